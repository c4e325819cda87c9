// CTA-per-cell operations: one thread block integrates one grid cell.
//
// For mechanisms whose LU is too large for the warp-per-cell tables (a few
// hundred species with a fill of tens of thousands of entries and hundreds
// of thousands of Schur updates), one warp per cell has too little
// parallelism and too little shared memory.  Here the cell's LU lives in the
// block's shared memory and every heavy operation (f, Jacobian, the
// factorization of I - gamma*J, the triangular solves) runs on all warps of
// the block.  The BDF control (the same Cell code as the warp-per-cell
// kernel) runs on warp 0: when it needs a heavy operation it writes a
// command, releases the other warps at a named barrier, and takes part in
// the operation itself; the other warps loop on commands until warp 0 sends
// OP_EXIT at the end of the cell.
//
// Barrier discipline (all barriers are `bar.sync 1, kThreads`, executed by
// whole warps): warp 0 passes one barrier per command it publishes and then
// the operation's own barriers; the other warps pass one barrier per command
// they read and the same operation's barriers.  Every operation ends on a
// barrier, so warp 0 writes the next command only after every warp has read
// the previous one.
//
// The factorization is right-looking, one barrier per pivot: the updates of
// pivot k (targets (i, j), i, j > k) never touch column k or row k, so they
// run in parallel.  Each target receives its updates in increasing pivot
// order, as in the row-wise (up-looking) form.  The trailing dense block of
// the LU (up to 112 x 112) lives in registers for the whole factorization:
// the block's threads form a 16 x 16 grid, thread (p, q) holding the dense
// entries (p + 16 s, q + 16 t); every pivot is a rank-1 update of those
// registers from two vectors exchanged through shared memory (the pivot's
// column of multipliers and its row of U), so the dense block's Schur
// updates cost no shared-memory traffic.  The sparse head pivots update the
// head rows and the dense rows' head columns in shared memory from
// tabulated update records and the dense block through the same exchange
// (their columns and rows scattered into zeroed vectors); each thread's
// records of the next pivot are loaded while the current one runs, and each
// column's L entries are scaled right after its pivot's barrier.  The exchange
// vectors rotate over three buffers, so a pivot's scatter never meets a
// slower warp's reads of the previous pivot's vectors and each buffer is
// zeroed two pivots after its use.
//
// The solves read their tables from shared memory (a section of the blob
// each block copies once): the sparse head by row levels, the dense rows'
// head columns and the head rows' dense columns one row per warp, and the
// dense block's triangles by panels of 16 columns (half a warp solves the
// panel's triangle with shuffles, every thread then updates one row beyond
// it).
#pragma once

namespace blk {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTile = 7;    // factorization: dense entries per thread and dimension
constexpr int kMaxDense = campb::kBlockMaxDense;  // = 16 * kTile
static_assert(kMaxDense == 16 * kTile, "dense block tiling");
constexpr int kXBuf = 3 * 2 * kMaxDense;  // exchange vectors (LT elements)

enum Op : int { OP_EXIT = 0, OP_F = 1, OP_JAC = 2, OP_FACTOR = 3, OP_SOLVE = 4 };

struct Cmd {
  int op, ret;
  const double* y;
  double* out;
  double h;  // guard step (f, J) or gamma (factorization)
};

struct Tab {
  const uint32_t *rx_word, *rx_vptr, *fg_ptr, *fg_ent, *jg_ptr, *jg_mid, *jg_w0;
  const uint32_t *lk_ptr, *lk_mid, *tg_ptr, *lk;
  const uint64_t* hrec;
  const uint16_t *jg_w1, *jg_row, *lu_src, *dep_state, *stage;
  const double *coef, *atol;
  int n, n_rxn, n_jac, n_lu, r0, n_hf, n_hb, sg_len;
  int sg_rowptr, sg_diag, sg_ub, sg_perm, sg_hf_ptr, sg_hf_rows, sg_hb_ptr, sg_hb_rows;
  int sg_ndoff, sg_ndcol, sg_dbase, sg_hlk, sg_hmid, sg_htg;
};

__device__ __forceinline__ Tab make_tab(const char* b) {
  const campb::BlockOff& o = *reinterpret_cast<const campb::BlockOff*>(b);
  Tab t;
  t.rx_word = (const uint32_t*)(b + o.rx_word);
  t.rx_vptr = (const uint32_t*)(b + o.rx_vptr);
  t.fg_ptr = (const uint32_t*)(b + o.fg_ptr);
  t.fg_ent = (const uint32_t*)(b + o.fg_ent);
  t.jg_ptr = (const uint32_t*)(b + o.jg_ptr);
  t.jg_mid = (const uint32_t*)(b + o.jg_mid);
  t.jg_w0 = (const uint32_t*)(b + o.jg_w0);
  t.lk_ptr = (const uint32_t*)(b + o.lk_ptr);
  t.lk_mid = (const uint32_t*)(b + o.lk_mid);
  t.tg_ptr = (const uint32_t*)(b + o.tg_ptr);
  t.jg_w1 = (const uint16_t*)(b + o.jg_w1);
  t.jg_row = (const uint16_t*)(b + o.jg_row);
  t.lu_src = (const uint16_t*)(b + o.lu_src);
  t.lk = (const uint32_t*)(b + o.lk);
  t.hrec = (const uint64_t*)(b + o.hrec);
  t.dep_state = (const uint16_t*)(b + o.dep_state);
  t.stage = (const uint16_t*)(b + o.stage);
  t.coef = (const double*)(b + o.coef);
  t.atol = (const double*)(b + o.atol);
  t.n = o.n;
  t.n_rxn = o.n_rxn;
  t.n_jac = o.n_jac;
  t.n_lu = o.n_lu;
  t.r0 = o.r0;
  t.n_hf = o.n_hf;
  t.n_hb = o.n_hb;
  t.sg_len = o.sg_len;
  t.sg_rowptr = o.sg_rowptr;
  t.sg_diag = o.sg_diag;
  t.sg_ub = o.sg_ub;
  t.sg_perm = o.sg_perm;
  t.sg_hf_ptr = o.sg_hf_ptr;
  t.sg_hf_rows = o.sg_hf_rows;
  t.sg_hb_ptr = o.sg_hb_ptr;
  t.sg_hb_rows = o.sg_hb_rows;
  t.sg_ndoff = o.sg_ndoff;
  t.sg_ndcol = o.sg_ndcol;
  t.sg_dbase = o.sg_dbase;
  t.sg_hlk = o.sg_hlk;
  t.sg_hmid = o.sg_hmid;
  t.sg_htg = o.sg_htg;
  return t;
}

__device__ __forceinline__ void bsync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory");
}

template <typename T>
__device__ __forceinline__ T lane_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// the per-cell arrays an operation works on (shared memory unless noted)
template <typename LT>
struct Ctx {
  Tab t;
  const double* keff;  // rate constants (global, per block)
  double* part;        // term rates (f)
  double* jpart;       // rate partials (J; global, per block)
  LT* xbuf;            // the factorization's exchange vectors (over part)
  LT* J;         // solver Jacobian slots (global)
  LT* LU;
  LT* dinv;
  LT* z;
  double* rhs;   // right-hand side and solution of the solves
  // the staged solve tables
  const uint16_t *rowptr, *diag, *ub, *perm, *hf_ptr, *hf_rows, *hb_ptr, *hb_rows;
  const uint16_t *ndoff, *ndcol, *dbase;
  const uint16_t *hlk, *hmid, *htg;  // head pivots' L-list and target pointers
};

// f(y) into out (src/time_derivative.c:90-97 with the negative-yield guard
// of src/rxns/rxn_arrhenius.c:153-160); the caller has checked y >= -SMALL
template <typename LT>
__device__ __noinline__ void op_f(const Ctx<LT>& c, const double* y, double* out, double h) {
  const Tab& t = c.t;
  double* rates = c.part;
  #pragma unroll 1
  for (int r = threadIdx.x; r < t.n_rxn; r += kThreads) {
    const uint32_t w = __ldg(t.rx_word + r);
    const int nv = w >> 30;
    double rate = c.keff[r];
    if (nv > 0) rate *= state_of(y[w & 1023u]);
    if (nv > 1) rate *= state_of(y[(w >> 10) & 1023u]);
    if (nv > 2) rate *= state_of(y[(w >> 20) & 1023u]);
    rates[r] = rate;
  }
  bsync();
  #pragma unroll 1
  for (int i = threadIdx.x; i < t.n; i += kThreads) {
    const double yi = state_of(y[i]);
    double P0 = 0.0, L0 = 0.0, P1 = 0.0, L1 = 0.0;
    const uint32_t e1 = __ldg(t.fg_ptr + i + 1);
    uint32_t e = __ldg(t.fg_ptr + i);
    #pragma unroll 1
    for (; e + 1 < e1; e += 2) {
      const uint32_t w0 = __ldg(t.fg_ent + e), w1 = __ldg(t.fg_ent + e + 1);
      const double r0 = rates[w0 & 0xFFFFu], r1 = rates[w1 & 0xFFFFu];
      const double c0 = __ldg(t.coef + ((w0 >> 16) & 0x7FFFu));
      const double c1 = __ldg(t.coef + ((w1 >> 16) & 0x7FFFu));
      const double v0 = ((w0 >> 31) && !(-r0 * c0 * h <= yi)) ? 0.0 : r0 * c0;
      const double v1 = ((w1 >> 31) && !(-r1 * c1 * h <= yi)) ? 0.0 : r1 * c1;
      P0 += v0 > 0.0 ? v0 : 0.0;
      L0 += v0 < 0.0 ? -v0 : 0.0;
      P1 += v1 > 0.0 ? v1 : 0.0;
      L1 += v1 < 0.0 ? -v1 : 0.0;
    }
    if (e < e1) {
      const uint32_t w0 = __ldg(t.fg_ent + e);
      const double r0 = rates[w0 & 0xFFFFu];
      const double c0 = __ldg(t.coef + ((w0 >> 16) & 0x7FFFu));
      const double v0 = ((w0 >> 31) && !(-r0 * c0 * h <= yi)) ? 0.0 : r0 * c0;
      P0 += v0 > 0.0 ? v0 : 0.0;
      L0 += v0 < 0.0 ? -v0 : 0.0;
    }
    const double P = P0 + P1, L = L0 + L1;
    out[i] = (P + L != 0.0) ? P - L : 0.0;
  }
  bsync();
}

// solver Jacobian slots at y (src/rxns/rxn_arrhenius.c:178-212): losses,
// then guarded products; the caller has checked y >= -SMALL
template <typename LT>
__device__ __noinline__ void op_jac(const Ctx<LT>& c, const double* y, double h) {
  const Tab& t = c.t;
  double* part = c.jpart;
  #pragma unroll 1
  for (int r = threadIdx.x; r < t.n_rxn; r += kThreads) {
    const uint32_t w = __ldg(t.rx_word + r);
    const int nv = w >> 30;
    const int base = (int)__ldg(t.rx_vptr + r);
    const double k = c.keff[r];
    if (nv == 1) {
      part[base] = k;
    } else if (nv == 2) {
      const double y0 = state_of(y[w & 1023u]), y1 = state_of(y[(w >> 10) & 1023u]);
      part[base] = k * y1;
      part[base + 1] = k * y0;
    } else if (nv == 3) {
      const double y0 = state_of(y[w & 1023u]), y1 = state_of(y[(w >> 10) & 1023u]);
      const double y2 = state_of(y[(w >> 20) & 1023u]);
      part[base] = k * y1 * y2;
      part[base + 1] = k * y0 * y2;
      part[base + 2] = k * y0 * y1;
    }
  }
  bsync();
  #pragma unroll 1
  for (int e = threadIdx.x; e < t.n_jac; e += kThreads) {
    const double yrow = state_of(y[__ldg(t.jg_row + e)]);
    double P = 0.0, L = 0.0;
    const uint32_t gm = __ldg(t.jg_mid + e), g1 = __ldg(t.jg_ptr + e + 1);
    uint32_t g = __ldg(t.jg_ptr + e);
    #pragma unroll 1
    for (; g < gm; ++g) L += part[__ldg(t.jg_w0 + g) & 0xFFFFu];
    #pragma unroll 1
    for (; g < g1; ++g) {
      const uint32_t w0 = __ldg(t.jg_w0 + g);
      const double p = part[w0 & 0xFFFFu];
      const double cf = __ldg(t.coef + (w0 >> 16));
      const double yi = state_of(y[__ldg(t.jg_w1 + g) - 1]);
      P += -p * yi * cf * h <= yrow ? cf * p : 0.0;
    }
    c.J[e] = (LT)(P - L);
  }
  bsync();
}

// LU = I - gamma*J factored in place; false when a pivot is zero or not
// finite (its reciprocal is then 0).  Every thread computes the same
// pivots, so the result is the same in all of them.
template <typename LT>
__device__ __noinline__ bool op_factor(const Ctx<LT>& c, double gamma) {
  const Tab& t = c.t;
  LT* LU = c.LU;
  const int tid = threadIdx.x;
  const int n = t.n, r0 = t.r0, m = n - r0;
  #pragma unroll 1
  for (int p = tid; p < t.n_lu; p += kThreads) {
    const int s = __ldg(t.lu_src + p);
    double v = (s & 0x7FFF) ? -gamma * (double)c.J[(s & 0x7FFF) - 1] : 0.0;
    if (s & 0x8000) v += 1.0;
    LU[p] = (LT)v;
  }
  #pragma unroll 1
  for (int e = tid; e < kXBuf; e += kThreads) c.xbuf[e] = (LT)0;
  bsync();
  // this thread's entries of the dense block: (p + 16 s, q + 16 u)
  const int p = tid >> 4, q = tid & 15;
  LT a[kTile][kTile];
  #pragma unroll
  for (int s = 0; s < kTile; ++s)
  #pragma unroll
    for (int u = 0; u < kTile; ++u) {
      const int di = p + 16 * s, dj = q + 16 * u;
      a[s][u] = (di < m && dj < m) ? LU[c.dbase[di] + r0 + dj] : (LT)0;
    }
  bool bad = false;
  // sparse head pivots.  A pivot's work is a list of update records
  // (target, L entry, U entry) and its column's L entries; thread tid takes
  // records tid + 256 j and L entry tid.  The first kPre records and the L
  // entry of pivot k + 1 are loaded while pivot k runs, so the L2 latency
  // of the tables overlaps the previous pivot's work and barrier.
  constexpr int kPre = 4;
  constexpr uint64_t kNone = ~0ull;
  uint64_t rq[kPre];
  uint32_t lq = 0xFFFFFFFFu;
  auto fetch = [&](int k) {
    const int q0 = c.htg[k], nq = c.htg[k + 1] - q0;
    #pragma unroll
    for (int j = 0; j < kPre; ++j)
      rq[j] = tid + kThreads * j < nq ? __ldg(t.hrec + q0 + tid + kThreads * j) : kNone;
    const int e0 = c.hlk[k], ne = c.hlk[k + 1] - e0;
    lq = tid < ne ? __ldg(t.lk + e0 + tid) : 0xFFFFFFFFu;
  };
  if (r0 > 0) fetch(0);
  #pragma unroll 1
  for (int k = 0; k < r0; ++k) {
    LT* lb = c.xbuf + (k % 3) * (2 * kMaxDense);
    LT* ubf = lb + kMaxDense;
    const LT piv = LU[c.diag[k]];
    const bool pb = (piv == (LT)0) || !isfinite((double)piv);
    bad |= pb;
    const LT dk = pb ? (LT)0 : (LT)(1.0 / (double)piv);
    if (tid == 0) c.dinv[k] = dk;
    // the buffer two pivots on (last read before the previous barrier)
    LT* nb = c.xbuf + ((k + 1) % 3) * (2 * kMaxDense);
    #pragma unroll 1
    for (int e = tid; e < 2 * kMaxDense; e += kThreads) nb[e] = (LT)0;
    uint64_t cr[kPre];
    #pragma unroll
    for (int j = 0; j < kPre; ++j) cr[j] = rq[j];
    const uint32_t cl = lq;
    if (k + 1 < r0) fetch(k + 1);
    // the tabulated updates (targets of one pivot are distinct)
    #pragma unroll
    for (int j = 0; j < kPre; ++j) {
      const uint64_t r = cr[j];
      if (r != kNone) {
        const int tg = (int)(r & 0xFFFFu), lp = (int)((r >> 16) & 0xFFFFu);
        const int up = (int)((r >> 32) & 0xFFFFu);
        LU[tg] -= (LU[lp] * dk) * LU[up];
      }
    }
    const int q0 = c.htg[k], nq = c.htg[k + 1] - q0;
    #pragma unroll 1
    for (int e = tid + kThreads * kPre; e < nq; e += kThreads) {
      const uint64_t r = __ldg(t.hrec + q0 + e);
      const int tg = (int)(r & 0xFFFFu), lp = (int)((r >> 16) & 0xFFFFu);
      const int up = (int)((r >> 32) & 0xFFFFu);
      LU[tg] -= (LU[lp] * dk) * LU[up];
    }
    // the dense rows' multipliers into the exchange column
    const int e0 = c.hlk[k], ne = c.hlk[k + 1] - e0;
    if (cl != 0xFFFFFFFFu && (int)(cl >> 16) >= r0) lb[(cl >> 16) - r0] = LU[cl & 0xFFFFu] * dk;
    #pragma unroll 1
    for (int e = tid + kThreads; e < ne; e += kThreads) {
      const uint32_t w = __ldg(t.lk + e0 + e);
      if ((int)(w >> 16) >= r0) lb[(w >> 16) - r0] = LU[w & 0xFFFFu] * dk;
    }
    // row k's U entries in dense columns into the exchange row
    const int uh = c.ub[k], u1 = c.rowptr[k + 1];
    const uint16_t* cols = c.ndcol + c.ndoff[k] - c.rowptr[k];
    #pragma unroll 1
    for (int b = uh + tid; b < u1; b += kThreads) ubf[cols[b] - r0] = LU[b];
    bsync();
    // column k's L entries scaled (nothing reads or writes them until the
    // solves: the next pivots' updates lie right of column k)
    if (cl != 0xFFFFFFFFu) LU[cl & 0xFFFFu] *= dk;
    #pragma unroll 1
    for (int e = tid + kThreads; e < ne; e += kThreads) LU[__ldg(t.lk + e0 + e) & 0xFFFFu] *= dk;
    LT lv[kTile], uv[kTile];
    #pragma unroll
    for (int s = 0; s < kTile; ++s) lv[s] = (p + 16 * s < m) ? lb[p + 16 * s] : (LT)0;
    #pragma unroll
    for (int u = 0; u < kTile; ++u) uv[u] = (q + 16 * u < m) ? ubf[q + 16 * u] : (LT)0;
    #pragma unroll
    for (int s = 0; s < kTile; ++s)
    #pragma unroll
      for (int u = 0; u < kTile; ++u) a[s][u] -= lv[s] * uv[u];
  }
  // dense pivots: kk = 16 s0 + kq, held by the threads with q == kq
  // (column), p == kq (row) and both (pivot)
  #pragma unroll
  for (int s0 = 0; s0 < kTile; ++s0) {
    #pragma unroll 1
    for (int kq = 0; kq < 16; ++kq) {
      const int kk = 16 * s0 + kq;
      if (kk >= m) break;
      const int k = r0 + kk;
      LT* lb = c.xbuf + (k % 3) * (2 * kMaxDense);
      LT* ubf = lb + kMaxDense;
      if (q == kq) {
        #pragma unroll
        for (int s = 0; s < kTile; ++s) {
          const int di = p + 16 * s;
          if (di > kk && di < m) lb[di] = a[s][s0];
        }
        if (p == kq) {
          // the pivot's owner publishes its reciprocal (0 for a zero or
          // non-finite pivot), so no other thread divides
          const LT pv = a[s0][s0];
          const bool pbad = (pv == (LT)0) || !isfinite((double)pv);
          lb[kk] = pbad ? (LT)0 : (LT)(1.0 / (double)pv);
        }
      }
      if (p == kq) {
        #pragma unroll
        for (int u = 0; u < kTile; ++u) {
          const int dj = q + 16 * u;
          if (dj > kk && dj < m) ubf[dj] = a[s0][u];
        }
      }
      bsync();
      const LT dk = lb[kk];
      bad |= dk == (LT)0;
      if (tid == 0) c.dinv[k] = dk;
      LT lv[kTile], uv[kTile];
      #pragma unroll
      for (int s = 0; s < kTile; ++s) {
        const int di = p + 16 * s;
        lv[s] = (di > kk && di < m) ? lb[di] * dk : (LT)0;
      }
      #pragma unroll
      for (int u = 0; u < kTile; ++u) {
        const int dj = q + 16 * u;
        uv[u] = (dj > kk && dj < m) ? ubf[dj] : (LT)0;
      }
      // branch-free: lv / uv are zero outside the trailing rows / columns,
      // so the update leaves row kk, column kk and the rest unchanged there
      #pragma unroll
      for (int s = 0; s < kTile; ++s) {
        const bool sc = q == kq && p + 16 * s > kk;
        a[s][s0] = sc ? a[s][s0] * dk : a[s][s0];
      }
      // tile rows / columns wholly at or before the pivot are finished:
      // the branch is the same for the whole block
      #pragma unroll
      for (int s = 0; s < kTile; ++s) {
        if (16 * s + 15 > kk) {
          #pragma unroll
          for (int u = 0; u < kTile; ++u)
            if (16 * u + 15 > kk) a[s][u] -= lv[s] * uv[u];
        }
      }
    }
  }
  #pragma unroll
  for (int s = 0; s < kTile; ++s)
  #pragma unroll
    for (int u = 0; u < kTile; ++u) {
      const int di = p + 16 * s, dj = q + 16 * u;
      if (di < m && dj < m) LU[c.dbase[di] + r0 + dj] = a[s][u];
    }
  bsync();
  return !bad;
}

// sum of row[cc] * x[cc] over one panel's columns c0..c1-1 (at most 16):
// four partial sums, so the loads and products overlap
template <typename LT>
__device__ __forceinline__ LT panel_dot(const LT* row, const LT* x, int c0, int c1) {
  LT a0 = (LT)0, a1 = (LT)0, a2 = (LT)0, a3 = (LT)0;
  if (c1 - c0 == 16) {
    #pragma unroll
    for (int cc = 0; cc < 16; cc += 4) {
      a0 += row[c0 + cc] * x[c0 + cc];
      a1 += row[c0 + cc + 1] * x[c0 + cc + 1];
      a2 += row[c0 + cc + 2] * x[c0 + cc + 2];
      a3 += row[c0 + cc + 3] * x[c0 + cc + 3];
    }
  } else {
    #pragma unroll 1
    for (int cc = c0; cc < c1; ++cc) a0 += row[cc] * x[cc];
  }
  return (a0 + a1) + (a2 + a3);
}

// rhs <- (LU)^{-1} rhs, through z in the LU's type
template <typename LT>
__device__ __noinline__ void op_solve(const Ctx<LT>& c) {
  const Tab& t = c.t;
  const LT* LU = c.LU;
  LT* z = c.z;
  const int n = t.n, r0 = t.r0, m = n - r0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  #pragma unroll 1
  for (int k = tid; k < n; k += kThreads) z[k] = (LT)c.rhs[c.perm[k]];
  bsync();
  // forward: head rows by levels
  #pragma unroll 1
  for (int l = 0; l < t.n_hf; ++l) {
    const int p1 = c.hf_ptr[l + 1];
    #pragma unroll 1
    for (int pp = c.hf_ptr[l] + tid; pp < p1; pp += kThreads) {
      const int i = c.hf_rows[pp];
      const int q0 = c.rowptr[i], ne = c.diag[i] - q0;
      const uint16_t* cols = c.ndcol + c.ndoff[i];
      LT acc = z[i];
      #pragma unroll 4
      for (int e = 0; e < ne; ++e) acc -= LU[q0 + e] * z[cols[e]];
      z[i] = acc;
    }
    bsync();
  }
  if (r0 > 0) {
    // forward: the head columns of the dense rows, one row per warp
    #pragma unroll 2
    for (int i = r0 + warp; i < n; i += kWarps) {
      const int q0 = c.rowptr[i], e0 = c.ndoff[i], ne = c.ndoff[i + 1] - e0;
      LT v = (LT)0;
      #pragma unroll 2
      for (int e = lane; e < ne; e += 32) v += LU[q0 + e] * z[c.ndcol[e0 + e]];
      v = lane_sum(v);
      if (lane == 0) z[i] -= v;
    }
    bsync();
  }
  // the dense block by panels of 16 columns: half of warp 0 solves the
  // panel's triangle (a lane per row, the column value broadcast by a
  // shuffle), then every thread updates one row beyond the panel
  const int np = (m + 15) / 16;
  #pragma unroll 1
  for (int pp = 0; pp < np; ++pp) {
    const int c0 = 16 * pp, c1 = min(c0 + 16, m), w = c1 - c0;
    if (warp == 0) {
      const int d = c0 + (lane & 15);
      const bool own = lane < w;
      LT zi = own ? z[r0 + d] : (LT)0;
      const LT* ri = LU + (own ? c.dbase[d] + r0 : 0);
      // unrolled: the row's entries load ahead of the shuffle chain
      #pragma unroll
      for (int kk = 0; kk < 15; ++kk) {
        if (kk < w - 1) {
          const LT lk = ri[c0 + kk];
          const LT zk = __shfl_sync(0xffffffffu, zi, kk);
          const LT v = zi - lk * zk;
          zi = lane > kk ? v : zi;
        }
      }
      if (own) z[r0 + d] = zi;
    }
    bsync();
    if (c1 < m) {
      #pragma unroll 1
      for (int d = c1 + tid; d < m; d += kThreads) {
        const LT* ri = LU + c.dbase[d] + r0;
        z[r0 + d] -= panel_dot(ri, z + r0, c0, c1);
      }
      bsync();
    }
  }
  // backward, last panel first: the panel's triangle finished by each
  // row's pivot reciprocal, then the rows above the panel
  #pragma unroll 1
  for (int pp = np - 1; pp >= 0; --pp) {
    const int c0 = 16 * pp, c1 = min(c0 + 16, m), w = c1 - c0;
    if (warp == 0) {
      const int d = c0 + (lane & 15);
      const bool own = lane < w;
      LT zi = own ? z[r0 + d] : (LT)0;
      const LT di = own ? c.dinv[r0 + d] : (LT)0;
      const LT* ri = LU + (own ? c.dbase[d] + r0 : 0);
      #pragma unroll
      for (int kk = 15; kk >= 0; --kk) {
        if (kk < w) {
          const LT uk = ri[c0 + kk];
          zi = lane == kk ? zi * di : zi;
          const LT zk = __shfl_sync(0xffffffffu, zi, kk);
          const LT v = zi - uk * zk;
          zi = lane < kk ? v : zi;
        }
      }
      if (own) z[r0 + d] = zi;
    }
    bsync();
    if (c0 > 0) {
      #pragma unroll 1
      for (int d = tid; d < c0; d += kThreads) {
        const LT* ri = LU + c.dbase[d] + r0;
        z[r0 + d] -= panel_dot(ri, z + r0, c0, c1);
      }
      bsync();
    }
  }
  if (r0 > 0) {
    // backward: the dense columns of the head rows, one row per warp
    #pragma unroll 2
    for (int i = warp; i < r0; i += kWarps) {
      const int q0 = c.rowptr[i], e0 = c.ndoff[i] - q0;
      const int q1 = c.rowptr[i + 1];
      LT v = (LT)0;
      #pragma unroll 2
      for (int qq = c.ub[i] + lane; qq < q1; qq += 32) v += LU[qq] * z[c.ndcol[e0 + qq]];
      v = lane_sum(v);
      if (lane == 0) z[i] -= v;
    }
    bsync();
    // backward: head rows by levels
    #pragma unroll 1
    for (int l = 0; l < t.n_hb; ++l) {
      const int p1 = c.hb_ptr[l + 1];
      #pragma unroll 1
      for (int pp = c.hb_ptr[l] + tid; pp < p1; pp += kThreads) {
        const int i = c.hb_rows[pp];
        const uint16_t* cols = c.ndcol + c.ndoff[i] - c.rowptr[i];
        LT acc = z[i];
        const int q1 = c.ub[i];
        #pragma unroll 4
        for (int qq = c.diag[i] + 1; qq < q1; ++qq) acc -= LU[qq] * z[cols[qq]];
        z[i] = acc * c.dinv[i];
      }
      bsync();
    }
  }
  #pragma unroll 1
  for (int k = tid; k < n; k += kThreads) c.rhs[c.perm[k]] = (double)z[k];
  bsync();
}

// runs one command on this thread (every thread of the block calls it with
// the same command); returns the factorization's failure flag
template <typename LT>
__device__ __noinline__ int exec(const Ctx<LT>& c, int op, const double* y, double* out,
                                 double h) {
  switch (op) {
    case OP_F:
      op_f<LT>(c, y, out, h);
      return 0;
    case OP_JAC:
      op_jac<LT>(c, y, h);
      return 0;
    case OP_FACTOR:
      return op_factor<LT>(c, h) ? 0 : 1;
    default:
      op_solve<LT>(c);
      return 0;
  }
}

// warp 0: publish a command, release the other warps, run it with them
template <typename LT>
__device__ __forceinline__ int call(Cmd* cmd, const Ctx<LT>& c, int op, const double* y,
                                    double* out, double h) {
  if ((threadIdx.x & 31) == 0) {
    cmd->op = op;
    cmd->y = y;
    cmd->out = out;
    cmd->h = h;
  }
  __syncwarp();
  bsync();
  return exec<LT>(c, op, y, out, h);
}

// warps 1..: run commands until OP_EXIT
template <typename LT>
__device__ void serve(const Cmd* cmd, const Ctx<LT>& c) {
  #pragma unroll 1
  for (;;) {
    bsync();
    const int op = cmd->op;
    if (op == OP_EXIT) return;
    exec<LT>(c, op, cmd->y, cmd->out, cmd->h);
  }
}

__device__ __forceinline__ void finish(Cmd* cmd) {
  if ((threadIdx.x & 31) == 0) cmd->op = OP_EXIT;
  __syncwarp();
  bsync();
}

}  // namespace blk
