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
// run in parallel, and the L entries of column k are scaled by the pivot's
// reciprocal during pivot k + 1 (nothing reads or writes them there).  Each
// target receives its updates in increasing pivot order, as in the row-wise
// (up-looking) form.  The trailing dense block of the LU is addressed without
// tables; the sparse head uses tabulated targets.  The solves handle the
// sparse head by row levels and the dense block by panels of 32 columns: one
// warp solves the panel's triangle with shuffles, all warps update the rows
// beyond it (one row per warp, one column per lane).
#pragma once

namespace blk {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

enum Op : int { OP_EXIT = 0, OP_F = 1, OP_JAC = 2, OP_FACTOR = 3, OP_SOLVE = 4 };

struct Cmd {
  int op, ret;
  const double* y;
  double* out;
  double h;  // guard step (f, J) or gamma (factorization)
};

struct Tab {
  const uint32_t *rx_word, *rx_vptr, *fg_ptr, *fg_ent, *jg_ptr, *jg_mid, *jg_w0;
  const uint32_t *lk_ptr, *tg_ptr;
  const uint16_t *jg_w1, *jg_row, *lu_src, *lu_perm, *lu_rowptr, *lu_col, *lu_diag;
  const uint16_t *dpos, *ub, *lk_pos, *tg, *hf_ptr, *hf_rows, *hb_ptr, *hb_rows, *dep_state;
  const double *coef, *atol;
  int n, n_rxn, n_jac, n_lu, r0, n_hf, n_hb;
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
  t.tg_ptr = (const uint32_t*)(b + o.tg_ptr);
  t.jg_w1 = (const uint16_t*)(b + o.jg_w1);
  t.jg_row = (const uint16_t*)(b + o.jg_row);
  t.lu_src = (const uint16_t*)(b + o.lu_src);
  t.lu_perm = (const uint16_t*)(b + o.lu_perm);
  t.lu_rowptr = (const uint16_t*)(b + o.lu_rowptr);
  t.lu_col = (const uint16_t*)(b + o.lu_col);
  t.lu_diag = (const uint16_t*)(b + o.lu_diag);
  t.dpos = (const uint16_t*)(b + o.dpos);
  t.ub = (const uint16_t*)(b + o.ub);
  t.lk_pos = (const uint16_t*)(b + o.lk_pos);
  t.tg = (const uint16_t*)(b + o.tg);
  t.hf_ptr = (const uint16_t*)(b + o.hf_ptr);
  t.hf_rows = (const uint16_t*)(b + o.hf_rows);
  t.hb_ptr = (const uint16_t*)(b + o.hb_ptr);
  t.hb_rows = (const uint16_t*)(b + o.hb_rows);
  t.dep_state = (const uint16_t*)(b + o.dep_state);
  t.coef = (const double*)(b + o.coef);
  t.atol = (const double*)(b + o.atol);
  t.n = o.n;
  t.n_rxn = o.n_rxn;
  t.n_jac = o.n_jac;
  t.n_lu = o.n_lu;
  t.r0 = o.r0;
  t.n_hf = o.n_hf;
  t.n_hb = o.n_hb;
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
  const double* keff;
  double* part;  // term rates (f) or rate partials (J)
  LT* J;         // solver Jacobian slots (global)
  LT* LU;
  LT* dinv;
  LT* z;
  double* rhs;   // right-hand side and solution of the solves
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
  double* part = c.part;
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
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  #pragma unroll 1
  for (int p = threadIdx.x; p < t.n_lu; p += kThreads) {
    const int s = __ldg(t.lu_src + p);
    double v = (s & 0x7FFF) ? -gamma * (double)c.J[(s & 0x7FFF) - 1] : 0.0;
    if (s & 0x8000) v += 1.0;
    LU[p] = (LT)v;
  }
  bsync();
  const int n = t.n, r0 = t.r0;
  bool bad = false;
  LT dprev = (LT)0;
  #pragma unroll 1
  for (int k = 0; k < n; ++k) {
    const LT piv = LU[__ldg(t.lu_diag + k)];
    const bool pb = (piv == (LT)0) || !isfinite((double)piv);
    bad |= pb;
    const LT dk = pb ? (LT)0 : (LT)(1.0 / (double)piv);
    if (threadIdx.x == 0) c.dinv[k] = dk;
    // scale the L entries of column k - 1 (its updates ran at pivot k - 1)
    if (k > 0) {
      const int kp = k - 1;
      if (kp < r0) {
        const uint32_t a1 = __ldg(t.lk_ptr + kp + 1);
        #pragma unroll 1
        for (uint32_t a = __ldg(t.lk_ptr + kp) + threadIdx.x; a < a1; a += kThreads)
          LU[__ldg(t.lk_pos + a)] *= dprev;
      } else {
        #pragma unroll 1
        for (int i = k + threadIdx.x; i < n; i += kThreads)
          LU[__ldg(t.dpos + i - r0) + (kp - r0)] *= dprev;
      }
    }
    if (k < r0) {
      const uint32_t a0 = __ldg(t.lk_ptr + k), na = __ldg(t.lk_ptr + k + 1) - a0;
      const int u0 = __ldg(t.lu_diag + k) + 1;
      const int nu = (int)__ldg(t.lu_rowptr + k + 1) - u0;
      const uint16_t* tg = t.tg + __ldg(t.tg_ptr + k);
      #pragma unroll 1
      for (uint32_t a = warp; a < na; a += kWarps) {
        const LT l = LU[__ldg(t.lk_pos + a0 + a)] * dk;
        const uint16_t* ta = tg + (size_t)a * nu;
        #pragma unroll 2
        for (int b = lane; b < nu; b += 32) {
          const int d = __ldg(ta + b);
          LU[d] -= l * LU[u0 + b];
        }
      }
    } else {
      // dense block: rows and columns k+1..n-1
      const LT* uk = LU + (__ldg(t.dpos + k - r0) - r0);
      #pragma unroll 1
      for (int i = k + 1 + warp; i < n; i += kWarps) {
        LT* ri = LU + (__ldg(t.dpos + i - r0) - r0);
        const LT l = ri[k] * dk;
        #pragma unroll 2
        for (int j = k + 1 + lane; j < n; j += 32) ri[j] -= l * uk[j];
      }
    }
    bsync();
    dprev = dk;
  }
  return !bad;
}

// rhs <- (LU)^{-1} rhs, through z in the LU's type
template <typename LT>
__device__ __noinline__ void op_solve(const Ctx<LT>& c) {
  const Tab& t = c.t;
  const LT* LU = c.LU;
  LT* z = c.z;
  const int n = t.n, r0 = t.r0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  #pragma unroll 1
  for (int k = threadIdx.x; k < n; k += kThreads) z[k] = (LT)c.rhs[__ldg(t.lu_perm + k)];
  bsync();
  // forward: head rows by levels
  #pragma unroll 1
  for (int l = 0; l < t.n_hf; ++l) {
    const int p1 = __ldg(t.hf_ptr + l + 1);
    #pragma unroll 1
    for (int p = __ldg(t.hf_ptr + l) + threadIdx.x; p < p1; p += kThreads) {
      const int i = __ldg(t.hf_rows + p);
      LT acc = z[i];
      const int d = __ldg(t.lu_diag + i);
      #pragma unroll 1
      for (int q = __ldg(t.lu_rowptr + i); q < d; ++q) acc -= LU[q] * z[__ldg(t.lu_col + q)];
      z[i] = acc;
    }
    bsync();
  }
  // forward: the head columns of the dense rows, one row per warp
  if (r0 > 0) {
    #pragma unroll 1
    for (int i = r0 + warp; i < n; i += kWarps) {
      const int q1 = __ldg(t.dpos + i - r0);
      LT v = (LT)0;
      #pragma unroll 1
      for (int q = __ldg(t.lu_rowptr + i) + lane; q < q1; q += 32)
        v += LU[q] * z[__ldg(t.lu_col + q)];
      v = lane_sum(v);
      if (lane == 0) z[i] -= v;
    }
    bsync();
  }
  // forward: dense block by panels
  #pragma unroll 1
  for (int c0 = r0; c0 < n; c0 += 32) {
    const int c1 = min(c0 + 32, n), w = c1 - c0;
    if (warp == 0) {
      const int i = c0 + lane;
      const bool own = lane < w;
      LT zi = own ? z[i] : (LT)0;
      const LT* ri = own ? LU + (__ldg(t.dpos + i - r0) - r0) : LU;
      #pragma unroll 1
      for (int kk = 0; kk < w - 1; ++kk) {
        const LT zk = __shfl_sync(0xffffffffu, zi, kk);
        if (own && lane > kk) zi -= ri[c0 + kk] * zk;
      }
      if (own) z[i] = zi;
    }
    bsync();
    if (c1 < n) {
      const LT zc = lane < w ? z[c0 + lane] : (LT)0;
      #pragma unroll 1
      for (int i = c1 + warp; i < n; i += kWarps) {
        const LT* ri = LU + (__ldg(t.dpos + i - r0) - r0);
        LT v = lane < w ? ri[c0 + lane] * zc : (LT)0;
        v = lane_sum(v);
        if (lane == 0) z[i] -= v;
      }
      bsync();
    }
  }
  // backward: dense block by panels, last first
  const int np = (n - r0 + 31) / 32;
  #pragma unroll 1
  for (int pp = np - 1; pp >= 0; --pp) {
    const int c0 = r0 + 32 * pp, c1 = min(c0 + 32, n), w = c1 - c0;
    if (warp == 0) {
      const int i = c0 + lane;
      const bool own = lane < w;
      LT zi = own ? z[i] : (LT)0;
      const LT di = own ? c.dinv[i] : (LT)0;
      const LT* ri = own ? LU + (__ldg(t.dpos + i - r0) - r0) : LU;
      #pragma unroll 1
      for (int kk = w - 1; kk >= 0; --kk) {
        if (lane == kk) zi *= di;
        const LT zk = __shfl_sync(0xffffffffu, zi, kk);
        if (own && lane < kk) zi -= ri[c0 + kk] * zk;
      }
      if (own) z[i] = zi;
    }
    bsync();
    if (c0 > r0) {
      const LT zc = lane < w ? z[c0 + lane] : (LT)0;
      #pragma unroll 1
      for (int i = r0 + warp; i < c0; i += kWarps) {
        const LT* ri = LU + (__ldg(t.dpos + i - r0) - r0);
        LT v = lane < w ? ri[c0 + lane] * zc : (LT)0;
        v = lane_sum(v);
        if (lane == 0) z[i] -= v;
      }
      bsync();
    }
  }
  if (r0 > 0) {
    // backward: the dense columns of the head rows, one row per warp
    #pragma unroll 1
    for (int i = warp; i < r0; i += kWarps) {
      const int q1 = __ldg(t.lu_rowptr + i + 1);
      LT v = (LT)0;
      #pragma unroll 1
      for (int q = __ldg(t.ub + i) + lane; q < q1; q += 32) v += LU[q] * z[__ldg(t.lu_col + q)];
      v = lane_sum(v);
      if (lane == 0) z[i] -= v;
    }
    bsync();
    // backward: head rows by levels
    #pragma unroll 1
    for (int l = 0; l < t.n_hb; ++l) {
      const int p1 = __ldg(t.hb_ptr + l + 1);
      #pragma unroll 1
      for (int p = __ldg(t.hb_ptr + l) + threadIdx.x; p < p1; p += kThreads) {
        const int i = __ldg(t.hb_rows + p);
        LT acc = z[i];
        const int q1 = __ldg(t.ub + i);
        #pragma unroll 1
        for (int q = __ldg(t.lu_diag + i) + 1; q < q1; ++q) acc -= LU[q] * z[__ldg(t.lu_col + q)];
        z[i] = acc * c.dinv[i];
      }
      bsync();
    }
  }
  #pragma unroll 1
  for (int k = threadIdx.x; k < n; k += kThreads) c.rhs[__ldg(t.lu_perm + k)] = (double)z[k];
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
