// Per-cell stiff chemistry solve on sm_100a.
//
// One warp integrates one grid cell over a whole host time step with its own
// variable-order BDF (the CVODE algorithm: Nordsieck history, Newton
// iteration on I - gamma*J, WRMS local error test, step and order control).
// The kernel is persistent: each warp pulls the next cell index from a
// global counter when its cell finishes, so cells with very different
// stiffness keep every SM busy until the tail.
//
// Lane l of a warp owns the dependent variables l, l+32, l+64, ... for the
// element-wise vector work; the rate, Jacobian and LU phases are spread over
// the lanes by reaction, Jacobian entry and LU row, with row-level
// schedules computed on the host so that no two lanes write the same word.
// Everything a warp touches during the integration lives in its slice of
// shared memory except the saved Jacobian, which sits in a per-warp global
// slot (L2-resident: a few MB for all resident warps).
//
// Precision: the plain form is FP64 throughout.  The mixed form keeps the
// saved Jacobian, the LU factors and the triangular solves in FP32 and
// everything else (rates, residual, state, error test, step control) in
// FP64; the Newton iteration then acts as iterative refinement.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "bdf_consts.hpp"
#include "blob.hpp"
#include "engine.hpp"
#include "rates.cuh"

namespace campb {

#define FULLMASK 0xffffffffu

// CVODE's BDF constants and outcome codes, shared with the lane kernel
using namespace bdf;

constexpr int DO_ERROR_TEST = 100, PREDICT_AGAIN = 101, TRY_AGAIN = 102;

// ---------------------------------------------------------------------------
// Device tables
// ---------------------------------------------------------------------------
// Cells (warps) per block of the solve kernel: its launch bound leaves 168
// registers per thread, enough to keep the BDF state without spilling.
constexpr int kMaxCellsPerBlock = 12;
constexpr int kMaxCellsAero = 8;  // cells per block of the aerosol form

struct Layout {  // per-warp shared-memory slice (byte offsets; -1 = not in it)
  int zn, ewt, acor, y, ftemp, tempv, rates, keff, fscr, lu, z, dinv, ctl, bytes;
};

struct SolveArgs {
  DevMech m;
  BlobOff off;
  const void* blob;  // table blob in global memory (copied to shared)
  int tab_bytes;     // shared-memory bytes reserved for the tables
  int stage_bytes;   // blob bytes staged into them
  int* err;
  Layout lay;
  double* state;
  const double* env;
  const double* photo;
  const int* order;
  int n_cells;
  int* counter;
  CellStats* stats;
  void* jscratch;  // per-warp saved Jacobian slots
  double* hist;    // per-warp Nordsieck history zn[LMAX][n] + rate constants
  int hist_stride; // doubles per warp in hist
  const double* tspan = nullptr;  // per-cell (t0, t1); null: t0, t1 for all
  double t0, t1, rtol;
  int max_steps, maxncf, maxnef;
  int lu_mode;
};

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(FULLMASK, v, o));
  return v;
}
__device__ __forceinline__ bool warp_any(bool p) { return __any_sync(FULLMASK, p) != 0; }
__device__ __forceinline__ bool warp_all(bool p) { return __all_sync(FULLMASK, p) != 0; }
__device__ __forceinline__ int warp_isum(int v) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULLMASK, v, o));
  return v;
}

// value the reference's f sees for a solver variable: y above -SMALL is used
// as is, anything else (only exactly -SMALL reaches here) becomes TINY
// (src/camp_solver.c:805-833)
__device__ __forceinline__ double state_of(double y) { return y > -kSmall ? y : kTiny; }

// Device loops carry `#pragma unroll 1` unless unrolling is wanted: the
// solve kernel is bound by instruction fetch (a warp per cell, each at its own
// point of the BDF control flow), so compact code beats unrolled code here.

// one out-of-line copy each of pow, division and square root for the BDF
// control code (IEEE results, identical to the inline forms)
__device__ __noinline__ double dpow(double x, double y) { return pow(x, y); }
__device__ __noinline__ double ddiv(double a, double b) { return a / b; }
__device__ __noinline__ double dsqrt(double a) { return sqrt(a); }


// ---------------------------------------------------------------------------
// Shared-memory tables (blob.hpp) as typed pointers
// ---------------------------------------------------------------------------
struct Tab {
  const uint32_t* rx_word;
  const uint16_t* rx_vptr;
  const double* coef;
  const uint32_t* fg_ent;
  const uint16_t *fg_unit, *fg_lane, *fg_split;
  const uint32_t* jg_w0;
  const uint16_t *jg_w1, *jg_ptr, *jg_mid, *jg_lupos, *jg_row, *jg_lane, *jg_slots;
  const uint16_t *lu_perm, *lu_diag, *lu_src, *fa_ptr;
  const uint32_t* fa;
  const uint16_t* fb_lane;
  const uint32_t *fb_unit, *fb_pair;
  const uint16_t* fw_lane;
  const uint32_t *fw_unit, *fw_pair;
  const uint16_t *bw_lane;
  const uint32_t *bw_unit, *bw_pair;
  const uint16_t* dep_state;
  const double* atol;
  const uint16_t *lu_rowptr, *lu_col;
  const uint32_t *upd_ptr, *upd;
  const uint16_t *si_rec, *si_elem, *jg_umid, *aq_rec, *aq_sp, *aq_cp;
  const double *si_ef, *aq_sm, *aq_cpm, *aq_sim;
  int n, n_rxn, n_jac, n_lu, n_fsplit, n_plev, n_flev, n_blev, n_simpol, has_ug, n_aq;
};

__device__ __forceinline__ Tab make_tab(const char* b) {
  const BlobOff& o = *reinterpret_cast<const BlobOff*>(b);
  Tab t;
  t.rx_word = (const uint32_t*)(b + o.rx_word);
  t.rx_vptr = (const uint16_t*)(b + o.rx_vptr);
  t.coef = (const double*)(b + o.coef);
  t.fg_ent = (const uint32_t*)(b + o.fg_ent);
  t.fg_unit = (const uint16_t*)(b + o.fg_unit);
  t.fg_lane = (const uint16_t*)(b + o.fg_lane);
  t.fg_split = (const uint16_t*)(b + o.fg_split);
  t.jg_w0 = (const uint32_t*)(b + o.jg_w0);
  t.jg_w1 = (const uint16_t*)(b + o.jg_w1);
  t.jg_ptr = (const uint16_t*)(b + o.jg_ptr);
  t.jg_mid = (const uint16_t*)(b + o.jg_mid);
  t.jg_lupos = (const uint16_t*)(b + o.jg_lupos);
  t.jg_row = (const uint16_t*)(b + o.jg_row);
  t.jg_lane = (const uint16_t*)(b + o.jg_lane);
  t.jg_slots = (const uint16_t*)(b + o.jg_slots);
  t.lu_perm = (const uint16_t*)(b + o.lu_perm);
  t.lu_diag = (const uint16_t*)(b + o.lu_diag);
  t.lu_src = (const uint16_t*)(b + o.lu_src);
  t.fa_ptr = (const uint16_t*)(b + o.fa_ptr);
  t.fa = (const uint32_t*)(b + o.fa);
  t.si_rec = (const uint16_t*)(b + o.si_rec);
  t.si_elem = (const uint16_t*)(b + o.si_elem);
  t.si_ef = (const double*)(b + o.si_ef);
  t.jg_umid = (const uint16_t*)(b + o.jg_umid);
  t.n_simpol = o.n_simpol;
  t.has_ug = o.has_ug;
  t.aq_rec = (const uint16_t*)(b + o.aq_rec);
  t.aq_sp = (const uint16_t*)(b + o.aq_sp);
  t.aq_sm = (const double*)(b + o.aq_sm);
  t.aq_sim = (const double*)(b + o.aq_sim);
  t.aq_cp = (const uint16_t*)(b + o.aq_cp);
  t.aq_cpm = (const double*)(b + o.aq_cpm);
  t.n_aq = o.n_aq;
  t.fb_lane = (const uint16_t*)(b + o.fb_lane);
  t.fb_unit = (const uint32_t*)(b + o.fb_unit);
  t.fb_pair = (const uint32_t*)(b + o.fb_pair);
  t.fw_lane = (const uint16_t*)(b + o.fw_lane);
  t.fw_unit = (const uint32_t*)(b + o.fw_unit);
  t.fw_pair = (const uint32_t*)(b + o.fw_pair);
  t.bw_lane = (const uint16_t*)(b + o.bw_lane);
  t.bw_unit = (const uint32_t*)(b + o.bw_unit);
  t.bw_pair = (const uint32_t*)(b + o.bw_pair);
  t.dep_state = (const uint16_t*)(b + o.dep_state);
  t.atol = (const double*)(b + o.atol);
  t.lu_rowptr = (const uint16_t*)(b + o.lu_rowptr);
  t.lu_col = (const uint16_t*)(b + o.lu_col);
  t.upd_ptr = (const uint32_t*)(b + o.upd_ptr);
  t.upd = (const uint32_t*)(b + o.upd);
  t.n = o.n;
  t.n_rxn = o.n_rxn;
  t.n_jac = o.n_jac;
  t.n_lu = o.n_lu;
  t.n_fsplit = o.n_fsplit;
  t.n_plev = o.n_plev;
  t.n_flev = o.n_flev;
  t.n_blev = o.n_blev;
  return t;
}

// Copies the table blob into the front of the block's shared memory with one
// bulk (TMA) copy completed on an mbarrier.  The wait is bounded: a copy of
// at most 64 KB from this GPU's memory completes in microseconds, and the
// first limit (2^24 polls, each suspending in try_wait) is seconds.  On
// timeout the block records the error flag that the host reads after the
// launch, then waits again for its own copy, with a four times longer limit,
// so that the block does not leave while the copy may still write its shared
// memory; only if that wait also runs out (the memory system no longer
// answers, and the host already sees the error) does it return false with
// the copy outstanding.
__device__ bool stage_tables(char* dst, const void* src, int bytes, unsigned long long* bar,
                             int* err_flag) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            (unsigned)__cvta_generic_to_shared(dst)),
        "l"(src), "r"(bytes), "r"(b)
        : "memory");
  }
  auto wait = [&](long limit) {
    unsigned done = 0;
    #pragma unroll 1
    for (long it = 0; it < limit && !done; ++it)
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(b)
          : "memory");
    return done != 0;
  };
  bool ok = wait(1L << 24);
  if (!ok) {
    atomicExch(err_flag, 1);
    wait(1L << 26);
  }
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

// ---------------------------------------------------------------------------
// Right-hand side f(y) and Jacobian
// ---------------------------------------------------------------------------
// Reaction rates k * prod(y) into rates[]; returns (warp-uniform) whether
// any rate is negative, which only a reactant in (-SMALL, 0) can cause.
__device__ __forceinline__ bool rates_of(const Tab& t, const double* y, const double* keff,
                                         double* rates, int lane) {
  bool neg = false;
  #pragma unroll 1
  for (int r = lane; r < t.n_rxn; r += 32) {
    const uint32_t w = t.rx_word[r];
    const int nv = w >> 30;
    double rate = keff[r];
    if (nv > 0) rate *= state_of(y[w & 1023u]);
    if (nv > 1) rate *= state_of(y[(w >> 10) & 1023u]);
    if (nv > 2) rate *= state_of(y[(w >> 20) & 1023u]);
    rates[r] = rate;
    neg |= rate < 0.0;
  }
  return warp_any(neg);
}

// ---------------------------------------------------------------------------
// Sub-models: the species they compute, before every f and J
// ---------------------------------------------------------------------------
// ZSR aerosol water of one phase instance
// (src/sub_models/sub_model_ZSR_aerosol_water.c:225-305, Jacobian :318-437)
// from its program (SubProgram in model.hpp); P, when given, receives the
// partials of the water against the gas-phase water and the ions.  Ion
// concentrations use the program's reciprocal factors (the reference divides
// by count, MW and 1000 in turn: equal to rounding).
__device__ double zsr_water(const int* I, const double* F, const double* y, double ppm,
                            double* P) {
  const double a_w = ppm * state_of(y[I[1]]);
  const int npair = I[2];
  double W = 1.0e-30;  // MINIMUM_WATER_MASS_
  int ii = 3, fi = 0;
  #pragma unroll 1
  for (int x = 0; x < npair; ++x) {
    const int type = I[ii++];
    if (type == 1) {  // Jacobson et al. (1996)
      const int ci = I[ii], ai = I[ii + 1], ny = I[ii + 2];
      const int pg = I[ii + 3], pc = I[ii + 4], pa = I[ii + 5];
      ii += 6;
      const double low = F[fi], fc = F[fi + 1], fa = F[fi + 2];
      const double* Y = F + fi + 3;
      fi += 3 + ny;
      const bool above = a_w > low;
      const double j_aw = above ? a_w : low;
      // Y_0 + Y_1 a + ... and its derivative in a, by Horner's rule
      double mol = 0.0, dm = 0.0;
      #pragma unroll 1
      for (int k = ny - 1; k >= 0; --k) {
        dm = dm * j_aw + mol;
        mol = mol * j_aw + Y[k];
      }
      const double cat = state_of(y[ci]) * fc, an = state_of(y[ai]) * fa;
      // smooth minimum of the ion concentrations (smoothing factor -100)
      const double ec = exp(-100.0 * cat), ea = exp(-100.0 * an);
      const double inv_e = ddiv(1.0, ec + ea);
      const double conc = (cat * ec + an * ea) * inv_e;
      const double inv_m2 = ddiv(1.0, mol * mol);
      W += conc * inv_m2 * 1000.0;
      if (P) {
        const double dcc = (ec * ec + ec * ea * (1.0 + 100.0 * an - 100.0 * cat)) * inv_e * inv_e;
        const double dca = (ea * ea + ec * ea * (1.0 + 100.0 * cat - 100.0 * an)) * inv_e * inv_e;
        P[pg] += -2.0 * conc * inv_m2 * ddiv(1000.0, mol) * (above ? dm * ppm : 0.0);
        P[pa] += inv_m2 * 1000.0 * dca * fa;
        P[pc] += inv_m2 * 1000.0 * dcc * fc;
      }
    } else if (type == 2) {  // EQSAM (Metzger et al., 2002)
      const int nion = I[ii], pg = I[ii + 1];
      ii += 2;
      const double pre = F[fi], zw = F[fi + 1];
      fi += 2;
      double e_aw = a_w > 0.99 ? 0.99 : a_w;
      e_aw = e_aw < 0.001 ? 0.001 : e_aw;
      const double base = pre * (ddiv(1.0, e_aw) - 1.0);
      const double mol = dpow(base, zw);
      const double inv_mol = ddiv(1.0, mol);
      double dmol = 0.0;
      if (P) {
        const double de = (a_w > 0.99 || a_w < 0.001) ? 0.0 : ppm;
        dmol = zw * dpow(base, zw - 1.0) * ddiv(-pre, e_aw * e_aw) * de;
      }
      #pragma unroll 1
      for (int k = 0; k < nion; ++k) {
        const int ion = I[ii], pid = I[ii + 1];
        ii += 2;
        const double inv_mw = F[fi++];
        double c = state_of(y[ion]);
        c = c > 0.0 ? c : 0.0;
        W += c * inv_mw * inv_mol;
        if (P) {
          P[pg] += -c * inv_mw * inv_mol * inv_mol * dmol;
          P[pid] += (c > 0.0 ? 1.0 : 0.0) * inv_mw * inv_mol;
        }
      }
    }
  }
  return W;
}

// PD-FiTE activity coefficient of one ion pair in one phase instance
// (src/sub_models/sub_model_PDFiTE.c:167-259, Jacobian :273-432; Topping et
// al. 2009, eq. 15) from its program; P, when given, receives its partials
// against the gas-phase water and every ion.  Moles per concentration and
// the partials' factors are the program's reciprocals; 1 / omega is taken
// once.
__device__ double pdfite_gamma(const int* I, const double* F, const double* y, double ppm,
                               double* P) {
  double a_w = ppm * state_of(y[I[1]]);
  a_w = a_w < 0.0 ? 0.0 : (a_w > 1.0 ? 1.0 : a_w);
  const int npair = I[2], x = I[3], ninter = I[4], pw = I[5];
  const int* pr = I + 6;              // per pair: cation, anion, stoichiometry, 2 param ids
  const int* it = pr + 5 * npair;     // per interaction: pair, B count
  const double* fb = F + 2 * npair;   // per interaction: min RH, max RH, B...
  auto cn = [&](int j) { return state_of(y[pr[5 * j]]) * F[2 * j]; };
  auto an = [&](int j) { return state_of(y[pr[5 * j + 1]]) * F[2 * j + 1]; };
  double omega = 0.0;
  #pragma unroll 1
  for (int j = 0; j < npair; ++j)
    if (j != x) omega += 2.0 * pr[5 * j + 2] * cn(j) * an(j);
  const double inv_omega = omega > 0.0 ? ddiv(1.0, omega) : 0.0;
  auto in_range = [&](double lo, double hi) {
    return !((a_w <= lo || a_w > hi) && !(a_w <= 0.0 && lo <= 0.0));
  };
  double lng = 0.0;
  int fi = 0;
  #pragma unroll 1
  for (int k = 0; k < ninter; ++k) {
    const int j = it[2 * k], nb = it[2 * k + 1];
    const double lo = fb[fi], hi = fb[fi + 1];
    const double* B = fb + fi + 2;
    fi += 2 + nb;
    if (!in_range(lo, hi)) continue;
    double li = 0.0;
    #pragma unroll 1
    for (int z = nb - 1; z >= 0; --z) li = li * a_w + B[z];
    if (j == x)
      lng += li;
    else if (omega > 0.0)
      lng += li * cn(j) * an(j) * inv_omega;
  }
  const double g = exp(lng);
  if (P) {
    fi = 0;
    #pragma unroll 1
    for (int k = 0; k < ninter; ++k) {
      const int j = it[2 * k], nb = it[2 * k + 1];
      const double lo = fb[fi], hi = fb[fi + 1];
      const double* B = fb + fi + 2;
      fi += 2 + nb;
      if (!in_range(lo, hi)) continue;
      double li = 0.0, dli = 0.0;
      #pragma unroll 1
      for (int z = nb - 1; z >= 0; --z) {
        dli = dli * a_w + li;
        li = li * a_w + B[z];
      }
      dli *= ppm;
      if (j == x) {
        P[pw] += g * dli;
      } else if (omega > 0.0) {
        const double cj = cn(j), aj = an(j);
        P[pr[5 * j + 3]] += g * li * aj * F[2 * j] * inv_omega;
        P[pr[5 * j + 4]] += g * li * cj * F[2 * j + 1] * inv_omega;
        P[pw] += g * cj * aj * inv_omega * dli;
        const double s = -g * li * cj * aj * inv_omega * inv_omega * 2.0;
        #pragma unroll 1
        for (int q = 0; q < npair; ++q) {
          if (q == x) continue;
          const double sq = s * pr[5 * q + 2];
          P[pr[5 * q + 3]] += sq * an(q) * F[2 * q];
          P[pr[5 * q + 4]] += sq * cn(q) * F[2 * q + 1];
        }
      }
    }
  }
  return g;
}

// Every computed species, one lane each, into cv; with P, also the
// parameter Jacobian (P zeroed first; element ids index it)
__device__ __noinline__ void sub_model_eval(const char* tb, const double* y, const double* keff,
                                            double* cv, double* P, int lane) {
  const BlobOff& o = *reinterpret_cast<const BlobOff*>(tb);
  if (P) {
    #pragma unroll 1
    for (int i = lane; i < o.n_pj; i += 32) P[i] = 0.0;
    __syncwarp();
  }
  const uint32_t* rec = (const uint32_t*)(tb + o.sm_rec);
  const int* I0 = (const int*)(tb + o.sm_int);
  const double* F0 = (const double*)(tb + o.sm_flt);
  const double ppm = keff[o.sm_keff];
  #pragma unroll 1
  for (int c = lane; c < o.n_cv; c += 32) {
    const int* I = I0 + rec[2 * c];
    const double* F = F0 + rec[2 * c + 1];
    cv[c] = I[0] == 1 ? zsr_water(I, F, y, ppm, P) : pdfite_gamma(I, F, y, ppm, P);
  }
  __syncwarp();
}

// SIMPOL phase transfer, one lane per instance
// (src/rxns/rxn_SIMPOL_phase_transfer.c:337-450 and 463-744, the total-mass
// branch of the modal/binned representation): the mode's or bin's number
// concentration from its volume, the phase's mass and mean molecular weight,
// and the condensation and evaporation rates.  Per-cell constants c (keff
// slots n_rxn + 8 k): condensation rate constant, K_eq, 1/(kg m-3 -> ppm),
// number factor, activity coefficient, and the volume, mass and moles of the
// floors and constant species.  The representation's radius partials are
// zero (its radii do not depend on the state) and are left out.
struct SimpolState {
  double N, cond, evap, evap_rate, m, mol, inv_k;
};
__device__ __forceinline__ SimpolState simpol_state(const Tab& t, int k, const double* y,
                                                    const double* keff, const double* cv) {
  const uint16_t* rec = t.si_rec + 8 * k;
  const double* c = keff + t.n_rxn + 8 * k;
  double V = c[5], m = c[6], mol = c[7];
  const int e0 = rec[3], e1 = e0 + rec[2];
  #pragma unroll 1
  for (int e = e0; e < e1; ++e) {
    const double ye = state_of(y[t.si_elem[e]]);
    const double* f = t.si_ef + 3 * e;
    V += ye * f[0];
    mol += ye * f[1];
    m += ye * f[2];
  }
  SimpolState s;
  s.N = V * c[3];
  s.m = m;
  s.mol = mol;
  s.inv_k = c[2];
  // k_c K_eq MW / m = k_c K_eq / moles
  s.evap_rate = ddiv(c[0] * c[1], mol) * c[4];
  // HL with a water that a sub-model computes: evaporation per water
  if (rec[5]) s.evap_rate = ddiv(s.evap_rate, cv[rec[5] - 1]);
  s.cond = c[0] * state_of(y[rec[0]]);
  s.evap = s.evap_rate * state_of(y[rec[1]]);
  return s;
}

// the four pseudo-rates per instance; returns (warp-uniform) whether any is
// negative
__device__ __noinline__ bool simpol_rates(const char* tb, const double* y, const double* keff,
                                          const double* cv, double* rates, int lane) {
  const Tab t = make_tab(tb);
  bool neg = false;
  #pragma unroll 1
  for (int k = lane; k < t.n_simpol; k += 32) {
    const SimpolState s = simpol_state(t, k, y, keff, cv);
    double* r = rates + t.n_rxn + 4 * k;
    r[0] = s.N * s.evap;            // gas gain
    r[1] = s.N * s.cond;            // gas loss
    r[2] = s.N * s.evap * s.inv_k;  // aerosol loss
    r[3] = s.N * s.cond * s.inv_k;  // aerosol gain
    neg |= r[0] < 0.0 || r[1] < 0.0 || r[2] < 0.0 || r[3] < 0.0;
  }
  return warp_any(neg);
}

// Jacobian partials per instance: gas-gas loss, aerosol-gas and gas-aerosol
// productions, aerosol-aerosol loss, then per dependent element the gas
// row's production and loss and the aerosol row's loss and production; an
// HL instance whose water a sub-model computes adds the gas and aerosol
// rows against that water (src/rxns/rxn_HL_phase_transfer.c:383-404)
__device__ __noinline__ void simpol_partials(const char* tb, const double* y, const double* keff,
                                             const double* cv, double* part, int lane) {
  const Tab t = make_tab(tb);
  #pragma unroll 1
  for (int k = lane; k < t.n_simpol; k += 32) {
    const uint16_t* rec = t.si_rec + 8 * k;
    const double* c = keff + t.n_rxn + 8 * k;
    const SimpolState s = simpol_state(t, k, y, keff, cv);
    double* p = part + rec[4];
    p[0] = s.N * c[0];
    p[1] = s.N * c[0] * s.inv_k;
    p[2] = s.N * s.evap_rate;
    p[3] = s.N * s.evap_rate * s.inv_k;
    if (rec[5]) {
      const double w = cv[rec[5] - 1];
      p[4] = -ddiv(s.N * s.evap, w);
      p[5] = ddiv(s.N * s.evap * s.inv_k, w);
      continue;
    }
    // d evap / d mass = -evap / m, d evap / d MW = evap / MW = evap mol / m
    const double dedm = -ddiv(s.evap, s.m);
    const double dedw = dedm * -s.mol;
    const double inv_mol2 = ddiv(1.0, s.mol * s.mol);
    const int e0 = rec[3], nd = rec[2];
    #pragma unroll 1
    for (int j = 0; j < nd; ++j) {
      const double* f = t.si_ef + 3 * (e0 + j);
      const double num = c[3] * f[0];
      const double dm = f[2];
      const double dw = f[2] != 0.0 ? (s.mol - f[1] * s.m) * inv_mol2 : 0.0;
      const double gp = s.evap * num + s.N * dedm * dm + s.N * dedw * dw;
      const double gl = s.cond * num;
      p[4 + 4 * j] = gp;
      p[5 + 4 * j] = gl;
      p[6 + 4 * j] = s.evap * s.inv_k * num + (s.N * dedm * dm + s.N * dedw * dw) * s.inv_k;
      p[7 + 4 * j] = gl * s.inv_k;
    }
  }
}

// Aqueous equilibrium, one lane per instance
// (src/rxns/rxn_aqueous_equilibrium.c:266-393, 403-540): the forward and
// reverse rates from the per-cell constants (keff slots: forward, reverse,
// with the constant species, water powers and activity coefficient folded
// in) times (c m) of each dependent reactant or product slot.
// A water or activity coefficient that a sub-model computes (rec[6], rec[7])
// enters here: 1 / W per reactant and per product after the first, the
// activity coefficient on the reverse rate, and no reaction below the
// minimum water (keff slot + 2); so do computed reactants and products
// (c m of each, rec[8], rec[9]).
__device__ __forceinline__ void aq_fr(const Tab& t, const uint16_t* rec, const double* y,
                                      const double* keff, const double* cv, double* rf,
                                      double* rr) {
  const int S = rec[0], R = rec[1], s0 = rec[2];
  double f = keff[rec[5]], r = keff[rec[5] + 1];
  #pragma unroll 1
  for (int k = 0; k < S; ++k) {
    const double v = state_of(y[t.aq_sp[s0 + k]]) * t.aq_sm[s0 + k];
    if (k < R)
      f *= v;
    else
      r *= v;
  }
  #pragma unroll 1
  for (int j = rec[8]; j < rec[8] + rec[9]; ++j) {
    const double v = cv[t.aq_cp[j] & 0x7FFF] * t.aq_cpm[j];
    if (t.aq_cp[j] & 0x8000)
      f *= v;
    else
      r *= v;
  }
  const int wcv = rec[6] & 0xFF;
  if (wcv) {
    const double w = cv[wcv - 1];
    if (w < keff[rec[5] + 2]) {
      f = r = 0.0;
    } else {
      const int nr = (rec[6] >> 8) & 0xF, np = rec[6] >> 12;
      #pragma unroll 1
      for (int i = 1; i < nr; ++i) f = ddiv(f, w);
      #pragma unroll 1
      for (int i = 1; i < np; ++i) r = ddiv(r, w);
    }
  }
  if (rec[7]) r *= cv[rec[7] - 1];
  *rf = f;
  *rr = r;
}

// per dependent slot a loss and a gain pseudo-rate: a reactant loses
// rf / m and gains rr / m, a product the reverse; returns (warp-uniform)
// whether any is negative
__device__ __noinline__ bool aq_rates(const char* tb, const double* y, const double* keff,
                                      const double* cv, double* rates, int lane) {
  const Tab t = make_tab(tb);
  bool neg = false;
  #pragma unroll 1
  for (int q = lane; q < t.n_aq; q += 32) {
    const uint16_t* rec = t.aq_rec + 12 * q;
    double rf, rr;
    aq_fr(t, rec, y, keff, cv, &rf, &rr);
    const int S = rec[0], R = rec[1], s0 = rec[2];
    double* r = rates + rec[3];
    #pragma unroll 1
    for (int k = 0; k < S; ++k) {
      const double im = t.aq_sim[s0 + k];
      r[2 * k] = (k < R ? rf : rr) * im;
      r[2 * k + 1] = (k < R ? rr : rf) * im;
      neg |= r[2 * k] < 0.0 || r[2 * k + 1] < 0.0;
    }
  }
  return warp_any(neg);
}

// partials: independent slot a (rate rf for a reactant, rr for a product,
// divided by its concentration), row slot k (divided by its m); zero when
// the rate is zero, as the reference skips those.  Then, for a water a
// sub-model computes, each row slot against it, and for a computed
// activity coefficient each row slot against that
// (src/rxns/rxn_aqueous_equilibrium.c:486-537).
__device__ __noinline__ void aq_partials(const char* tb, const double* y, const double* keff,
                                         const double* cv, double* part, int lane) {
  const Tab t = make_tab(tb);
  #pragma unroll 1
  for (int q = lane; q < t.n_aq; q += 32) {
    const uint16_t* rec = t.aq_rec + 12 * q;
    double rf, rr;
    aq_fr(t, rec, y, keff, cv, &rf, &rr);
    const int S = rec[0], R = rec[1], s0 = rec[2];
    double* p = part + rec[4];
    #pragma unroll 1
    for (int a = 0; a < S; ++a) {
      const double rate = a < R ? rf : rr;
      const double rc = rate != 0.0 ? ddiv(rate, state_of(y[t.aq_sp[s0 + a]])) : 0.0;
      #pragma unroll 1
      for (int k = 0; k < S; ++k) p[a * S + k] = rc * t.aq_sim[s0 + k];
    }
    p += S * S;
    const int wcv = rec[6] & 0xFF;
    if (wcv) {
      // d rate_f / d W = -(n_r - 1) rate_f / W, likewise the reverse
      const double w = cv[wcv - 1];
      const int nr = (rec[6] >> 8) & 0xF, np = rec[6] >> 12;
      const double dfw = ddiv(rf * (nr - 1), w), drw = ddiv(rr * (np - 1), w);
      #pragma unroll 1
      for (int k = 0; k < S; ++k) p[k] = (k < R ? dfw - drw : drw - dfw) * t.aq_sim[s0 + k];
      p += S;
    }
    if (rec[7]) {
      const double dg = ddiv(rr, cv[rec[7] - 1]);
      #pragma unroll 1
      for (int k = 0; k < S; ++k) {
        const double v = dg * t.aq_sim[s0 + k];
        p[k] = k < R ? v : -v;
      }
      p += S;
    }
    // computed reactants / products as independent species: a loss where
    // the participant and the row are both reactants or both products
    #pragma unroll 1
    for (int j = rec[8]; j < rec[8] + rec[9]; ++j, p += S) {
      const bool jr = (t.aq_cp[j] & 0x8000) != 0;
      const double rate = jr ? rf : rr;
      const double rc = rate != 0.0 ? ddiv(rate, cv[t.aq_cp[j] & 0x7FFF]) : 0.0;
      #pragma unroll 1
      for (int k = 0; k < S; ++k) {
        const double v = rc * t.aq_sim[s0 + k];
        p[k] = jr == (k < R) ? -v : v;
      }
    }
  }
}

// Both aerosol passes behind one call, so that the wrappers below keep a
// single call site each (the solve kernel's register allocation follows
// them).
__device__ __noinline__ bool aero_rates(const char* tb, const double* y, const double* keff,
                                        const double* cv, double* rates, int lane) {
  const bool neg = simpol_rates(tb, y, keff, cv, rates, lane);
  return aq_rates(tb, y, keff, cv, rates, lane) || neg;
}
__device__ __noinline__ void aero_partials(const char* tb, const double* y, const double* keff,
                                           const double* cv, double* part, int lane) {
  simpol_partials(tb, y, keff, cv, part, lane);
  aq_partials(tb, y, keff, cv, part, lane);
}

// Returns 1 (recoverable) when some y < -SMALL, else writes f into out.
// When rp/rl are given, the production and loss sums are written too.
// Species lists are processed in lane-balanced units; lists split over
// several units are added up in a combine pass (fscr holds their partials).
__device__ __noinline__ int dev_f(const char* tb, const double* y, double h,
                                  const double* keff, double* rates, double* fscr,
                                  double* out, int lane, double* rp = nullptr,
                                  double* rl = nullptr, bool neg_extra = false) {
  const Tab t = make_tab(tb);
  bool bad = false;
  #pragma unroll 1
  for (int i = lane; i < t.n; i += 32) bad |= y[i] < -kSmall;
  if (warp_any(bad)) return 1;
  const bool negrate = rates_of(t, y, keff, rates, lane) || neg_extra;
  __syncwarp();
  const uint4* fg_unit = (const uint4*)t.fg_unit;
  const int u1 = t.fg_lane[lane + 1];
  #pragma unroll 1
  for (int u = t.fg_lane[lane]; u < u1; ++u) {
    // unit record: species | first entry, end of losses | end of
    // non-negative-yield products, end | slot
    const uint4 rec = fg_unit[u];
    const int sp = rec.x & 0xFFFFu, b = rec.x >> 16;
    const int m1 = rec.y & 0xFFFFu, m2 = rec.y >> 16;
    const int e = rec.z & 0xFFFFu, slot = rec.z >> 16;
    const double yi = state_of(y[sp]);
    double P0 = 0.0, L0 = 0.0, P1 = 0.0, L1 = 0.0;
    if (!negrate && yi >= 0.0 && h >= 0.0) {
      // common path: every rate >= 0 and the product concentration >= 0, so
      // each group's sign is known and the negative-yield guard
      // (src/rxns/rxn_arrhenius.c:153-160) can only fail for negative yields
      int k = b;
      #pragma unroll 1
      for (; k + 1 < m1; k += 2) {
        L0 += rates[t.fg_ent[k] & 0xFFFFu];
        L1 += rates[t.fg_ent[k + 1] & 0xFFFFu];
      }
      if (k < m1) L0 += rates[t.fg_ent[k] & 0xFFFFu];
      #pragma unroll 1
      for (k = m1; k + 1 < m2; k += 2) {
        const uint32_t w0 = t.fg_ent[k], w1 = t.fg_ent[k + 1];
        P0 += __dmul_rn(rates[w0 & 0xFFFFu], t.coef[(w0 >> 16) & 0x7FFFu]);
        P1 += __dmul_rn(rates[w1 & 0xFFFFu], t.coef[(w1 >> 16) & 0x7FFFu]);
      }
      if (k < m2) {
        const uint32_t w0 = t.fg_ent[k];
        P0 += __dmul_rn(rates[w0 & 0xFFFFu], t.coef[(w0 >> 16) & 0x7FFFu]);
      }
      #pragma unroll 1
      for (k = m2; k < e; ++k) {
        const uint32_t w0 = t.fg_ent[k];
        const double v = __dmul_rn(rates[w0 & 0xFFFFu], -t.coef[(w0 >> 16) & 0x7FFFu]);
        L1 += v * h <= yi ? v : 0.0;
      }
    } else {
      // any sign: classify every term, guard every product term
      int k = b;
      #pragma unroll 1
      for (; k + 1 < e; k += 2) {
        const uint32_t w0 = t.fg_ent[k], w1 = t.fg_ent[k + 1];
        const double r0 = rates[w0 & 0xFFFFu], r1 = rates[w1 & 0xFFFFu];
        const double c0 = t.coef[(w0 >> 16) & 0x7FFFu], c1 = t.coef[(w1 >> 16) & 0x7FFFu];
        const double v0 = ((w0 >> 31) && !(-r0 * c0 * h <= yi)) ? 0.0 : r0 * c0;
        const double v1 = ((w1 >> 31) && !(-r1 * c1 * h <= yi)) ? 0.0 : r1 * c1;
        P0 += v0 > 0.0 ? v0 : 0.0;
        L0 += v0 < 0.0 ? -v0 : 0.0;
        P1 += v1 > 0.0 ? v1 : 0.0;
        L1 += v1 < 0.0 ? -v1 : 0.0;
      }
      if (k < e) {
        const uint32_t w0 = t.fg_ent[k];
        const double r0 = rates[w0 & 0xFFFFu];
        const double c0 = t.coef[(w0 >> 16) & 0x7FFFu];
        const double v0 = ((w0 >> 31) && !(-r0 * c0 * h <= yi)) ? 0.0 : r0 * c0;
        P0 += v0 > 0.0 ? v0 : 0.0;
        L0 += v0 < 0.0 ? -v0 : 0.0;
      }
    }
    const double P = P0 + P1, L = L0 + L1;
    if (slot == 0xFFFF) {
      out[sp] = (P + L != 0.0) ? P - L : 0.0;
      if (rp) rp[sp] = P;
      if (rl) rl[sp] = L;
    } else {
      fscr[2 * slot] = P;
      fscr[2 * slot + 1] = L;
    }
  }
  __syncwarp();
  #pragma unroll 1
  for (int s = lane; s < t.n_fsplit; s += 32) {
    const int sp = t.fg_split[3 * s], first = t.fg_split[3 * s + 1], cnt = t.fg_split[3 * s + 2];
    double P = 0.0, L = 0.0;
    #pragma unroll 1
    for (int j = 0; j < cnt; ++j) {
      P += fscr[2 * (first + j)];
      L += fscr[2 * (first + j) + 1];
    }
    out[sp] = (P + L != 0.0) ? P - L : 0.0;
    if (rp) rp[sp] = P;
    if (rl) rl[sp] = L;
  }
  __syncwarp();
  return 0;
}

// Solver Jacobian values into Jout (indexed by CSC entry; each lane writes the
// entries of its balanced slot list); production and loss parts into jp/jl
// when given (src/rxns/rxn_arrhenius.c:178-212).
// One product entry of a solver-Jacobian slot: the partial times its yield
// adds to the production part when the negative-yield guard lets the product
// term apply (src/rxns/rxn_arrhenius.c:201-207).
__device__ __forceinline__ double jac_prod(const Tab& t, const double* part, const double* y,
                                           double yrow, double h, int g) {
  const uint32_t w0 = t.jg_w0[g];
  const double p = part[w0 & 0xFFFFu];
  const double c = t.coef[w0 >> 16];
  const double yi = state_of(y[t.jg_w1[g] - 1]);
  return -p * yi * c * h <= yrow ? __dmul_rn(c, p) : 0.0;
}

template <typename JT>
__device__ __noinline__ int dev_jac(const char* tb, const double* y, double h,
                                    const double* keff, double* part, JT* Jout, int lane,
                                    double* jp = nullptr, double* jl = nullptr) {
  const Tab t = make_tab(tb);
  bool bad = false;
  #pragma unroll 1
  for (int i = lane; i < t.n; i += 32) bad |= y[i] < -kSmall;
  if (warp_any(bad)) return 1;
  // d rate / d y_k for every variable reactant occurrence k
  #pragma unroll 1
  for (int r = lane; r < t.n_rxn; r += 32) {
    const uint32_t w = t.rx_word[r];
    const int nv = w >> 30, base = t.rx_vptr[r];
    const double k = keff[r];
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
  __syncwarp();
  const int s1 = t.jg_lane[lane + 1];
  #pragma unroll 1
  for (int s = t.jg_lane[lane]; s < s1; ++s) {
    const int e = t.jg_slots[s];
    const double yrow = state_of(y[t.jg_row[e]]);
    // loss partials [g0, gm) add to L as they are; product partials
    // [gm, g1) are guarded; two entries per iteration into alternating sums
    double P0 = 0.0, L0 = 0.0, P1 = 0.0, L1 = 0.0;
    const int gm = t.jg_mid[e], g1 = t.jg_ptr[e + 1];
    int g = t.jg_ptr[e];
    if (t.has_ug) {
      // unguarded productions (SIMPOL) lead the slot
      const int gu = t.jg_umid[e];
      #pragma unroll 1
      for (; g < gu; ++g) P0 += part[t.jg_w0[g] & 0xFFFFu];
    }
    #pragma unroll 1
    for (; g + 1 < gm; g += 2) {
      L0 += part[t.jg_w0[g] & 0xFFFFu];
      L1 += part[t.jg_w0[g + 1] & 0xFFFFu];
    }
    if (g < gm) L0 += part[t.jg_w0[g] & 0xFFFFu];
    #pragma unroll 1
    for (g = gm; g + 1 < g1; g += 2) {
      P0 += jac_prod(t, part, y, yrow, h, g);
      P1 += jac_prod(t, part, y, yrow, h, g + 1);
    }
    if (g < g1) P0 += jac_prod(t, part, y, yrow, h, g);
    const double P = P0 + P1, L = L0 + L1;
    Jout[e] = (JT)(P - L);
    if (jp) jp[e] = P;
    if (jl) jl[e] = L;
  }
  __syncwarp();
  return 0;
}

// f and J of a mechanism with SIMPOL, HL or aqueous equilibrium instances:
// their pseudo-rates or
// partials first (slots after the terms', which the mass-action passes do
// not write, made visible to the gathers by their warp barrier), then the
// usual evaluation.  Separate functions, so that the plain f and J keep
// their register use.
//
// With sub-models, their computed species come first (after the pseudo-rates
// in the f scratch, after the partials in the J scratch), then for J the
// parameter Jacobian P and the virtual slots V (rate partials against the
// computed species), which the chain folds into the solver slots:
// J[row][j] += V[row][c] * P[c][j] (src/camp_solver.c:1063-1106).  Where
// the production / loss split jp / jl is asked for, each chained term adds to
// the production part when positive and to the loss part when negative.
__device__ __noinline__ int dev_f_aero(const char* tb, const double* y, double h,
                                       const double* keff, double* rates, double* fscr,
                                       double* out, int lane, double* rp = nullptr,
                                       double* rl = nullptr) {
  const BlobOff& o = *reinterpret_cast<const BlobOff*>(tb);
  double* cv = rates + o.n_rates;
  if (o.n_cv > 0) sub_model_eval(tb, y, keff, cv, nullptr, lane);
  const bool neg = aero_rates(tb, y, keff, cv, rates, lane);
  return dev_f(tb, y, h, keff, rates, fscr, out, lane, rp, rl, neg);
}
template <typename JT>
__device__ __noinline__ int dev_jac_aero(const char* tb, const double* y, double h,
                                         const double* keff, double* part, JT* Jout, int lane,
                                         double* jp = nullptr, double* jl = nullptr) {
  const BlobOff& o = *reinterpret_cast<const BlobOff*>(tb);
  double* cv = part + o.n_part_all;
  double* P = cv + o.n_cv;
  double* V = P + o.n_pj;
  if (o.n_cv > 0) sub_model_eval(tb, y, keff, cv, P, lane);
  aero_partials(tb, y, keff, cv, part, lane);
  const int r = dev_jac<JT>(tb, y, h, keff, part, Jout, lane, jp, jl);
  if (r != 0 || o.n_chain == 0) return r;
  const uint16_t* vptr = (const uint16_t*)(tb + o.jv_ptr);
  const uint16_t* vpart = (const uint16_t*)(tb + o.jv_part);
  #pragma unroll 1
  for (int v = lane; v < o.n_virt; v += 32) {
    double s = 0.0;
    #pragma unroll 1
    for (int g = vptr[v]; g < vptr[v + 1]; ++g) s += part[vpart[g]];
    V[v] = s;
  }
  __syncwarp();
  const uint16_t* tgt = (const uint16_t*)(tb + o.ch_tgt);
  const uint16_t* cptr = (const uint16_t*)(tb + o.ch_ptr);
  const uint32_t* ent = (const uint32_t*)(tb + o.ch_ent);
  #pragma unroll 1
  for (int g = lane; g < o.n_chain; g += 32) {
    double s = (double)Jout[tgt[g]], sp = 0.0, sl = 0.0;
    #pragma unroll 1
    for (int e = cptr[g]; e < cptr[g + 1]; ++e) {
      const double v = V[ent[e] & 0xFFFFu] * P[ent[e] >> 16];
      s += v;
      sp += v > 0.0 ? v : 0.0;
      sl += v < 0.0 ? -v : 0.0;
    }
    Jout[tgt[g]] = (JT)s;
    if (jp) {
      jp[tgt[g]] += sp;
      jl[tgt[g]] += sl;
    }
  }
  __syncwarp();
  return 0;
}
__device__ __forceinline__ bool has_simpol(const char* tb) {
  const BlobOff* o = reinterpret_cast<const BlobOff*>(tb);
  return o->n_simpol > 0 || o->n_aq > 0 || o->n_cv > 0;
}

// ---------------------------------------------------------------------------
// LU of M = I - gamma*J on the fixed order, and the triangular solves
// ---------------------------------------------------------------------------
// One level of a grouped phase: every unit of this lane subtracts its pair
// products from its target, acc[target] -= sum a[pa] * x[pb].  A unit that
// carries a pivot (factorization only) then stores the reciprocal of its
// final value, the pivot, in dinv; the return value flags a zero or
// non-finite pivot.
template <int MODE, typename LT, typename XT>
__device__ __forceinline__ bool grouped_level(const uint16_t* rnd, const uint32_t* rec,
                                              const uint32_t* pair, int level, LT* acc,
                                              const LT* a, const XT* x, LT* dinv, int lane) {
  // MODE 0: plain; 1: a unit carrying pivot k stores dinv[k] = 1 / (its
  // final value) (factorization); 2: a unit carrying pivot k scales its final
  // value by dinv[k] (backward substitution).  Round r hands this lane the
  // record rec[32 r + lane]; a no-op record targets the spare accumulator
  // slot with no pairs and no pivot, so every lane runs the same code.
  bool bad = false;
  const uint2* rec2 = (const uint2*)rec;
  const int r1 = rnd[level + 1];
  #pragma unroll 1
  for (int r = rnd[level]; r < r1; ++r) {
    const uint2 w = rec2[32 * r + lane];
    const int tgt = w.x & 0xFFFFu, cnt = w.x >> 16;
    const int p0 = w.y & 0xFFFFu, piv = w.y >> 16;
    LT s0 = acc[tgt], s1 = (LT)0;
    int p = p0;
    #pragma unroll 1
    for (; p + 1 < p0 + cnt; p += 2) {
      const uint32_t q0 = pair[p], q1 = pair[p + 1];
      s0 -= a[q0 & 0xFFFFu] * (LT)x[q0 >> 16];
      s1 -= a[q1 & 0xFFFFu] * (LT)x[q1 >> 16];
    }
    if (p < p0 + cnt) {
      const uint32_t q0 = pair[p];
      s0 -= a[q0 & 0xFFFFu] * (LT)x[q0 >> 16];
    }
    LT s = s0 + s1;
    if (MODE == 1 && piv) {
      const bool pbad = (s == (LT)0) || !isfinite((double)s);
      bad |= pbad;
      dinv[piv - 1] = pbad ? (LT)0 : (LT)1 / s;
    }
    if (MODE == 2 && piv) s *= dinv[piv - 1];
    acc[tgt] = s;
  }
  return bad;
}

// M = I - gamma*J scattered into the LU pattern, then a right-looking
// factorization level by level: reciprocal pivots of the level, scaled L
// columns, Schur updates grouped by target.  Returns false on a zero or
// non-finite pivot.
template <typename LT>
__device__ __noinline__ bool dev_form_factor(const char* tb, const LT* J, double gamma,
                                             LT* LU, LT* dinv, int lane) {
  const Tab t = make_tab(tb);
  // M = I - gamma*J in one pass over the LU positions (fill-in starts at 0)
  #pragma unroll 1
  for (int q = lane; q < t.n_lu; q += 32) {
    const uint32_t src = t.lu_src[q];
    const int e = (int)(src & 0x7FFFu) - 1;
    LT v = e >= 0 ? (LT)(-gamma * (double)J[e]) : (LT)0;
    if (src & 0x8000u) v += (LT)1;
    LU[q] = v;
  }
  __syncwarp();
  bool bad = grouped_level<1, LT, LT>(t.fb_lane, t.fb_unit, t.fb_pair, 0, LU, LU, LU, dinv, lane);
  __syncwarp();
  #pragma unroll 1
  for (int lv = 0; lv < t.n_plev; ++lv) {
    const int a1 = t.fa_ptr[lv + 1];
    #pragma unroll 1
    for (int i = t.fa_ptr[lv] + lane; i < a1; i += 32) {
      const uint32_t w = t.fa[i];
      LU[w & 0xFFFFu] *= dinv[w >> 16];
    }
    __syncwarp();
    bad |= grouped_level<1, LT, LT>(t.fb_lane, t.fb_unit, t.fb_pair, lv + 1, LU, LU, LU, dinv, lane);
    __syncwarp();
  }
  return !warp_any(bad);
}

// b (original variable order, FP64) <- M^{-1} b
template <typename LT>
__device__ __noinline__ void dev_lsolve(const char* tb, const LT* LU, const LT* dinv,
                                        double* b, LT* z, int lane) {
  const Tab t = make_tab(tb);
  #pragma unroll 1
  for (int k = lane; k < t.n; k += 32) z[k] = (LT)b[t.lu_perm[k]];
  __syncwarp();
  #pragma unroll 1
  for (int lv = 0; lv < t.n_flev; ++lv) {
    grouped_level<0, LT, LT>(t.fw_lane, t.fw_unit, t.fw_pair, lv, z, LU, z, (LT*)nullptr, lane);
    __syncwarp();
  }
  #pragma unroll 1
  for (int g = 0; g < t.n_blev; ++g) {
    grouped_level<2, LT, LT>(t.bw_lane, t.bw_unit, t.bw_pair, g, z, LU, z, (LT*)dinv, lane);
    __syncwarp();
  }
  #pragma unroll 1
  for (int k = lane; k < t.n; k += 32) b[t.lu_perm[k]] = (double)z[k];
  __syncwarp();
}

// Sequential mode: lane 0 factors row by row (IKJ order, the same update
// lists the oracle's dense-row elimination follows) and runs both triangular
// solves; the other lanes wait at the closing __syncwarp.  Fewer phases and
// higher instruction-level parallelism than the level schedule, at the price
// of issue slots.
template <typename LT>
__device__ __noinline__ bool dev_form_factor_seq(const char* tb, const LT* J, double gamma,
                                                 LT* LU, LT* dinv, int lane) {
  const Tab t = make_tab(tb);
  #pragma unroll 1
  for (int q = lane; q < t.n_lu; q += 32) LU[q] = (LT)0;
  __syncwarp();
  const int s1 = t.jg_lane[lane + 1];
  #pragma unroll 1
  for (int s = t.jg_lane[lane]; s < s1; ++s) {
    const int e = t.jg_slots[s];
    LU[t.jg_lupos[e]] = (LT)(-gamma * (double)J[e]);
  }
  __syncwarp();
  #pragma unroll 1
  for (int i = lane; i < t.n; i += 32) LU[t.lu_diag[i]] += (LT)1;
  __syncwarp();
  bool bad = false;
  if (lane == 0) {
    #pragma unroll 1
    for (int i = 0; i < t.n; ++i) {
      const int d = t.lu_diag[i];
      #pragma unroll 1
      for (int q = t.lu_rowptr[i]; q < d; ++q) {
        const LT l = LU[q] * dinv[t.lu_col[q]];
        LU[q] = l;
        const uint32_t p1 = t.upd_ptr[q + 1];
        uint32_t p = t.upd_ptr[q];
        #pragma unroll 1
        for (; p + 1 < p1; p += 2) {
          const uint32_t u0 = t.upd[p], u1 = t.upd[p + 1];
          const LT a0 = LU[u0 & 0xFFFFu], a1 = LU[u1 & 0xFFFFu];
          LU[u0 >> 16] -= l * a0;
          LU[u1 >> 16] -= l * a1;
        }
        if (p < p1) {
          const uint32_t u0 = t.upd[p];
          LU[u0 >> 16] -= l * LU[u0 & 0xFFFFu];
        }
      }
      const LT piv = LU[d];
      const bool pbad = (piv == (LT)0) || !isfinite((double)piv);
      bad |= pbad;
      dinv[i] = pbad ? (LT)0 : (LT)1 / piv;
    }
  }
  __syncwarp();
  return !warp_any(bad);
}

template <typename LT>
__device__ __noinline__ void dev_lsolve_seq(const char* tb, const LT* LU, const LT* dinv,
                                            double* b, LT* z, int lane) {
  const Tab t = make_tab(tb);
  #pragma unroll 1
  for (int k = lane; k < t.n; k += 32) z[k] = (LT)b[t.lu_perm[k]];
  __syncwarp();
  if (lane == 0) {
    #pragma unroll 1
    for (int i = 0; i < t.n; ++i) {
      LT s0 = z[i], s1 = (LT)0;
      const int d = t.lu_diag[i];
      int q = t.lu_rowptr[i];
      #pragma unroll 1
      for (; q + 1 < d; q += 2) {
        s0 -= LU[q] * z[t.lu_col[q]];
        s1 -= LU[q + 1] * z[t.lu_col[q + 1]];
      }
      if (q < d) s0 -= LU[q] * z[t.lu_col[q]];
      z[i] = s0 + s1;
    }
    #pragma unroll 1
    for (int i = t.n - 1; i >= 0; --i) {
      LT s0 = z[i], s1 = (LT)0;
      const int d = t.lu_diag[i], q1 = t.lu_rowptr[i + 1];
      int q = d + 1;
      #pragma unroll 1
      for (; q + 1 < q1; q += 2) {
        s0 -= LU[q] * z[t.lu_col[q]];
        s1 -= LU[q + 1] * z[t.lu_col[q + 1]];
      }
      if (q < q1) s0 -= LU[q] * z[t.lu_col[q]];
      z[i] = (s0 + s1) * dinv[i];
    }
  }
  __syncwarp();
  #pragma unroll 1
  for (int k = lane; k < t.n; k += 32) b[t.lu_perm[k]] = (double)z[k];
  __syncwarp();
}

// ---------------------------------------------------------------------------
// BDF integrator state of one cell (warp-uniform scalars)
// ---------------------------------------------------------------------------
#include "block.cuh"

// One cell's CVODE BDF integration, run by one warp (lane-strided vector
// loops, warp reductions).  BLK: the CTA-per-cell form, whose heavy
// operations (f, J, factorization, solves) run on the whole block through
// blk::call (block.cuh) while this warp keeps the control.
template <typename LT, bool AERO, bool BLK = false>
struct Cell {
  const char* tb;     // shared-memory tables
  blk::Cmd* cmd;      // CTA form: the command slot and the operations' arrays
  const blk::Ctx<LT>* bx;
  const double* atol;
  int lu_mode;        // 0 = level schedule over the lanes, 1 = one lane
  int lane, n;
  double* zb;  // Nordsieck history: column j at zb + j*n
  double *ewt, *acor, *y, *ftemp, *tempv, *rates, *keff, *fscr;
  LT *LU, *z, *J, *dinv;
  double rtol;
  int max_steps, maxncf, maxnef;
  double h0;
  // method state
  int q, qprime, qwait, L, jcur;
  double h, hprime, hscale, eta, etamax, hu, next_h, tn;
  double *tau, *tq, *l;  // per-warp shared scalars (all lanes hold equal values)
  double rl1, gamma, gammap, gamrat, crate, acnrm, saved_tq5;
  double etaqm1, etaq, etaqp1;
  int nst, nfe, nsetups, netf, nni, ncfn, nje, nstlp, nstlj;

  __device__ double wrms(const double* v) const {
    double s = 0.0;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      double t = v[i] * ewt[i];
      s += t * t;
    }
    return dsqrt(ddiv(warp_sum(s), (double)n));
  }
  __device__ int f(const double* yy, double* out) {
    if constexpr (BLK) {
      bool bad = false;
      #pragma unroll 1
      for (int i = lane; i < n; i += 32) bad |= yy[i] < -kSmall;
      if (warp_any(bad)) return 1;
      blk::call<LT>(cmd, *bx, blk::OP_F, yy, out, h > 0.0 ? h : h0);
      return 0;
    } else if constexpr (AERO)
      return dev_f_aero(tb, yy, h > 0.0 ? h : h0, keff, rates, fscr, out, lane);
    else
      return dev_f(tb, yy, h > 0.0 ? h : h0, keff, rates, fscr, out, lane);
  }
  __device__ bool set_ewt(const double* yy) {
    bool bad = false;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      double w = rtol * fabs(yy[i]) + atol[i];
      bad |= !(w > 0.0);
      ewt[i] = ddiv(1.0, w);
    }
    __syncwarp();
    return !warp_any(bad);
  }
  __device__ void rescale() {
    double factor = eta;
    #pragma unroll 1
    for (int j = 1; j <= q; ++j) {
      #pragma unroll 1
      for (int i = lane; i < n; i += 32) (zb + (j) * n)[i] *= factor;
      factor *= eta;
    }
    __syncwarp();
    h = hscale * eta;
    next_h = h;
    hscale = h;
  }
  // zn <- zn * Pascal(q) (sign +1) or its inverse (sign -1), one element's
  // q+1 history values at a time in registers: for k = 1..q, j = q..k,
  // zn[j-1] += sign * zn[j]
  __device__ void pascal(double sign) {
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      double v[LMAX];
#pragma unroll
      for (int j = 0; j < LMAX; ++j) v[j] = (j <= q) ? zb[j * n + i] : 0.0;
#pragma unroll
      for (int k = 1; k <= QMAX; ++k)
#pragma unroll
        for (int j = QMAX; j >= 1; --j)
          if (k <= q && j >= k && j <= q) v[j - 1] += sign * v[j];
#pragma unroll
      for (int j = 0; j < QMAX; ++j)
        if (j < q) zb[j * n + i] = v[j];
    }
    __syncwarp();
  }
  __device__ void predict() {
    tn += h;
    pascal(1.0);
  }
  __device__ void restore(double saved_t) {
    tn = saved_t;
    pascal(-1.0);
  }
  // l and tq of the fixed-leading-coefficient BDF formula
  __device__ void set() {
    double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
    l[0] = l[1] = xi_inv = xistar_inv = 1.0;
    #pragma unroll 1
    for (int i = 2; i <= q; ++i) l[i] = 0.0;
    alpha0 = alpha0_hat = -1.0;
    hsum = h;
    if (q > 1) {
      #pragma unroll 1
      for (int j = 2; j < q; ++j) {
        hsum += tau[j - 1];
        xi_inv = ddiv(h, hsum);
        alpha0 -= ddiv(1.0, (double)j);
        #pragma unroll 1
        for (int i = j; i >= 1; --i) l[i] += l[i - 1] * xi_inv;
      }
      alpha0 -= ddiv(1.0, (double)q);
      xistar_inv = -l[1] - alpha0;
      hsum += tau[q - 1];
      xi_inv = ddiv(h, hsum);
      alpha0_hat = -l[1] - xi_inv;
      #pragma unroll 1
      for (int i = q; i >= 1; --i) l[i] += l[i - 1] * xistar_inv;
    }
    double A1 = 1.0 - alpha0_hat + alpha0;
    double A2 = 1.0 + q * A1;
    tq[2] = fabs(ddiv(A1, alpha0 * A2));
    tq[5] = fabs(ddiv(A2 * xistar_inv, l[q] * xi_inv));
    if (qwait == 1) {
      if (q > 1) {
        double C = ddiv(xistar_inv, l[q]);
        double A3 = alpha0 + ddiv(1.0, (double)q);
        double A4 = alpha0_hat + xi_inv;
        double Cpinv = ddiv(1.0 - A4 + A3, A3);
        tq[1] = fabs(C * Cpinv);
      } else {
        tq[1] = 1.0;
      }
      hsum += tau[q];
      xi_inv = ddiv(h, hsum);
      double A5 = alpha0 - ddiv(1.0, (double)(q + 1));
      double A6 = alpha0_hat - xi_inv;
      double Cppinv = ddiv(1.0 - A6 + A5, A2);
      tq[3] = fabs(ddiv(Cppinv, xi_inv * (q + 2) * A5));
    }
    tq[4] = ddiv(NLSCOEF, tq[2]);
    rl1 = ddiv(1.0, l[1]);
    gamma = h * rl1;
    if (nst == 0) gammap = gamma;
    gamrat = (nst > 0) ? ddiv(gamma, gammap) : 1.0;
  }
  __device__ void increase_order() {
    #pragma unroll 1
    for (int i = 0; i <= QMAX; ++i) l[i] = 0.0;
    l[2] = 1.0;
    double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = hscale;
    if (q > 1) {
      #pragma unroll 1
      for (int j = 1; j < q; ++j) {
        hsum += tau[j + 1];
        double xi = ddiv(hsum, hscale);
        prod *= xi;
        alpha0 -= ddiv(1.0, (double)(j + 1));
        alpha1 += ddiv(1.0, xi);
        #pragma unroll 1
        for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xiold + l[i - 1];
        xiold = xi;
      }
    }
    double A1 = ddiv(-alpha0 - alpha1, prod);
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      double top = A1 * (zb + (QMAX) * n)[i];
      (zb + (q + 1) * n)[i] = top;
      #pragma unroll 1
      for (int j = 2; j <= q; ++j) (zb + (j) * n)[i] += l[j] * top;
    }
    __syncwarp();
  }
  __device__ void decrease_order() {
    #pragma unroll 1
    for (int i = 0; i <= QMAX; ++i) l[i] = 0.0;
    l[2] = 1.0;
    double hsum = 0.0;
    #pragma unroll 1
    for (int j = 1; j <= q - 2; ++j) {
      hsum += tau[j];
      double xi = ddiv(hsum, hscale);
      #pragma unroll 1
      for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xi + l[i - 1];
    }
    #pragma unroll 1
    for (int i = lane; i < n; i += 32)
      #pragma unroll 1
      for (int j = 2; j < q; ++j) (zb + (j) * n)[i] -= l[j] * (zb + (q) * n)[i];
    __syncwarp();
  }
  __device__ void adjust_order(int dq) {
    if (dq == 1)
      increase_order();
    else if (dq == -1)
      decrease_order();
  }
  __device__ void adjust_params() {
    if (qprime != q) {
      adjust_order(qprime - q);
      q = qprime;
      L = q + 1;
      qwait = L;
    }
    rescale();
  }
  // J reuse rule of the CVODE direct linear solver interface; returns 0, or
  // >0 for a recoverable failure
  __device__ int lsetup(int convfail, const double* ypred) {
    double dgamma = fabs(ddiv(gamma, gammap) - 1.0);
    bool jbad = (nst == 0) || (nst > nstlj + MSBJ) ||
                ((convfail == FAIL_BAD_J) && (dgamma < DGMAX_J)) || (convfail == FAIL_OTHER);
    if (!jbad) {
      jcur = 0;
    } else {
      nje++;
      nstlj = nst;
      jcur = 1;
      int jr;
      if constexpr (BLK) {
        bool bad = false;
        #pragma unroll 1
        for (int i = lane; i < n; i += 32) bad |= ypred[i] < -kSmall;
        if (warp_any(bad)) return 1;
        blk::call<LT>(cmd, *bx, blk::OP_JAC, ypred, nullptr, h > 0.0 ? h : h0);
        jr = 0;
      } else if constexpr (AERO) {
        jr = dev_jac_aero<LT>(tb, ypred, h > 0.0 ? h : h0, keff, rates, J, lane);
      } else {
        jr = dev_jac<LT>(tb, ypred, h > 0.0 ? h : h0, keff, rates, J, lane);
      }
      if (jr) return 1;
    }
    if constexpr (BLK) return blk::call<LT>(cmd, *bx, blk::OP_FACTOR, nullptr, nullptr, gamma);
    const bool ok = lu_mode ? dev_form_factor_seq<LT>(tb, J, gamma, LU, dinv, lane)
                            : dev_form_factor<LT>(tb, J, gamma, LU, dinv, lane);
    return ok ? 0 : 1;
  }
  __device__ int newton(bool projected) {
    int mm = 0;
    double del, delp = 0.0;
    #pragma unroll 1
    for (;;) {
      #pragma unroll 1
      for (int i = lane; i < n; i += 32)
        tempv[i] = gamma * ftemp[i] - (rl1 * (zb + (1) * n)[i] + acor[i]);
      __syncwarp();
      if constexpr (BLK)
        blk::call<LT>(cmd, *bx, blk::OP_SOLVE, nullptr, nullptr, 0.0);
      else if (lu_mode)
        dev_lsolve_seq<LT>(tb, LU, dinv, tempv, z, lane);
      else
        dev_lsolve<LT>(tb, LU, dinv, tempv, z, lane);
      if (gamrat != 1.0) {
        double s = ddiv(2.0, 1.0 + gamrat);
        #pragma unroll 1
        for (int i = lane; i < n; i += 32) tempv[i] *= s;
      }
      nni++;
      del = wrms(tempv);
      #pragma unroll 1
      for (int i = lane; i < n; i += 32) {
        acor[i] += tempv[i];
        y[i] = (zb + (0) * n)[i] + acor[i];
      }
      __syncwarp();
      if (mm > 0) crate = fmax(CRDOWN * crate, ddiv(del, delp));
      double dcon = ddiv(del * fmin(1.0, crate), tq[4]);
      if (dcon <= 1.0) {
        acnrm = (mm == 0 && !projected) ? del : wrms(acor);
        jcur = 0;
        return NL_OK;
      }
      ++mm;
      if ((mm == MAXCOR) || ((mm >= 2) && (del > RDIV * delp)))
        return jcur ? NL_CONV_FAIL : NL_TRY_AGAIN;
      delp = del;
      int r = f(y, ftemp);
      nfe++;
      if (r > 0) return jcur ? NL_RHS_RECVR : NL_TRY_AGAIN;
    }
  }
  // non-negativity of the converged iterate (CVODE's cvCheckConstraints
  // with constraint >= 0 on every component)
  __device__ int check_constraints() {
    bool viol = false;
    double s = 0.0;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32)
      if (y[i] < 0.0) {
        viol = true;
        double t = y[i] * ewt[i];
        s += t * t;
      }
    if (!warp_any(viol)) return NL_OK;
    double vnorm = dsqrt(ddiv(warp_sum(s), (double)n));
    if (vnorm <= tq[4]) {
      #pragma unroll 1
      for (int i = lane; i < n; i += 32)
        if (y[i] < 0.0) {
          acor[i] -= y[i];
          y[i] = 0.0;
        }
      __syncwarp();
      acnrm = wrms(acor);
      return NL_OK;
    }
    double e = 1.0e300;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32)
      if (y[i] < 0.0) {
        double qv = ddiv(zb[i], zb[i] - y[i]);
        e = fmin(e, qv);
      }
    e = warp_min(e) * 0.9;
    eta = e > 0.1 ? e : 0.1;
    return NL_CONSTR_RECVR;
  }
  __device__ bool start_guess() {
    bool proj = false;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      double a = (zb + (0) * n)[i] < 0.0 ? -(zb + (0) * n)[i] : 0.0;
      proj |= a != 0.0;
      acor[i] = a;
      y[i] = (zb + (0) * n)[i] + a;
    }
    __syncwarp();
    return warp_any(proj);
  }
  __device__ int nls(int nflag) {
    int convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL)) ? NO_FAILURES : FAIL_OTHER;
    bool call_setup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (nst == 0) ||
                      (nst >= nstlp + MSBP) || (fabs(gamrat - 1.0) > DGMAX);
    bool projected = start_guess();
    #pragma unroll 1
    for (;;) {
      int r = f(y, ftemp);
      nfe++;
      if (r > 0) return NL_RHS_RECVR;
      if (call_setup) {
        int ier = lsetup(convfail, y);
        nsetups++;
        call_setup = false;
        gamrat = crate = 1.0;
        gammap = gamma;
        nstlp = nst;
        if (ier > 0) return NL_CONV_FAIL;
      }
      int ier = newton(projected);
      if (ier == NL_OK) return check_constraints();
      if (ier != NL_TRY_AGAIN) return ier;
      call_setup = true;
      convfail = FAIL_BAD_J;
      projected = start_guess();
    }
  }
  __device__ int handle_nflag(int* nflag, double saved_t, int* ncf) {
    int nf = *nflag;
    if (nf == NL_OK) return DO_ERROR_TEST;
    ncfn++;
    restore(saved_t);
    (*ncf)++;
    etamax = 1.0;
    if (*ncf == maxncf) return nf == NL_RHS_RECVR ? REPTD_RHSFUNC_ERR : CONV_FAILURE;
    if (nf != NL_CONSTR_RECVR) eta = ETACF;
    *nflag = PREV_CONV_FAIL;
    rescale();
    return PREDICT_AGAIN;
  }
  __device__ int error_test(int* nflag, double saved_t, int* nef, double* dsm) {
    *dsm = acnrm * tq[2];
    if (*dsm <= 1.0) return OK;
    (*nef)++;
    netf++;
    *nflag = PREV_ERR_FAIL;
    restore(saved_t);
    if (*nef == maxnef) return ERR_FAILURE;
    etamax = 1.0;
    if (*nef <= MXNEF1) {
      eta = ddiv(1.0, dpow(BIAS2 * *dsm, ddiv(1.0, (double)L)) + ADDON);
      eta = fmax(ETAMIN, eta);
      if (*nef >= SMALL_NEF) eta = fmin(eta, ETAMXF);
      rescale();
      return TRY_AGAIN;
    }
    if (q > 1) {
      eta = ETAMIN;
      adjust_order(-1);
      L = q;
      q--;
      qwait = L;
      rescale();
      return TRY_AGAIN;
    }
    eta = ETAMIN;
    h *= eta;
    next_h = h;
    hscale = h;
    qwait = LONG_WAIT;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) y[i] = zb[i];
    __syncwarp();
    int r = f(y, tempv);
    nfe++;
    if (r > 0) return UNREC_RHSFUNC_ERR;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) (zb + (1) * n)[i] = h * tempv[i];
    __syncwarp();
    return TRY_AGAIN;
  }
  __device__ void complete_step() {
    nst++;
    hu = h;
    #pragma unroll 1
    for (int i = q; i >= 2; --i) tau[i] = tau[i - 1];
    if ((q == 1) && (nst > 1)) tau[2] = tau[1];
    tau[1] = h;
    const bool save = (qwait - 1 == 1) && (q != QMAX);
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      const double a = acor[i];
      #pragma unroll 1
      for (int j = 0; j <= q; ++j) (zb + (j) * n)[i] += l[j] * a;
      if (save) (zb + (QMAX) * n)[i] = a;
    }
    __syncwarp();
    qwait--;
    if (save) {
      saved_tq5 = tq[5];
    }
  }
  __device__ void set_eta() {
    if (eta < THRESH) {
      eta = 1.0;
      hprime = h;
    } else {
      eta = fmin(eta, etamax);
      hprime = h * eta;
    }
  }
  __device__ void prepare_next_step(double dsm) {
    if (etamax == 1.0) {
      qwait = qwait > 2 ? qwait : 2;
      qprime = q;
      hprime = h;
      eta = 1.0;
      return;
    }
    etaq = ddiv(1.0, dpow(BIAS2 * dsm, ddiv(1.0, (double)L)) + ADDON);
    if (qwait != 0) {
      eta = etaq;
      qprime = q;
      set_eta();
      return;
    }
    qwait = 2;
    etaqm1 = 0.0;
    if (q > 1) {
      double ddn = wrms((zb + (q) * n)) * tq[1];
      etaqm1 = ddiv(1.0, dpow(BIAS1 * ddn, ddiv(1.0, (double)q)) + ADDON);
    }
    etaqp1 = 0.0;
    if (q != QMAX && saved_tq5 != 0.0) {
      double cquot = ddiv(tq[5], saved_tq5) * dpow(ddiv(h, tau[2]), (double)L);
      #pragma unroll 1
      for (int i = lane; i < n; i += 32) tempv[i] = acor[i] - cquot * (zb + (QMAX) * n)[i];
      double dup = wrms(tempv) * tq[3];
      etaqp1 = ddiv(1.0, dpow(BIAS3 * dup, ddiv(1.0, (double)(L + 1))) + ADDON);
    }
    double etam = fmax(etaqm1, fmax(etaq, etaqp1));
    if (etam < THRESH) {
      eta = 1.0;
      qprime = q;
    } else if (etam == etaq) {
      eta = etaq;
      qprime = q;
    } else if (etam == etaqm1) {
      eta = etaqm1;
      qprime = q - 1;
    } else {
      eta = etaqp1;
      qprime = q + 1;
      #pragma unroll 1
      for (int i = lane; i < n; i += 32) (zb + (QMAX) * n)[i] = acor[i];
      __syncwarp();
    }
    set_eta();
  }
  __device__ int step() {
    double saved_t = tn, dsm = 0.0;
    int ncf = 0, nef = 0, nflag = FIRST_CALL;
    if ((nst > 0) && (hprime != h)) adjust_params();
    #pragma unroll 1
    for (;;) {
      predict();
      set();
      nflag = nls(nflag);
      int kflag = handle_nflag(&nflag, saved_t, &ncf);
      if (kflag == PREDICT_AGAIN) continue;
      if (kflag != DO_ERROR_TEST) return kflag;
      int eflag = error_test(&nflag, saved_t, &nef, &dsm);
      if (eflag == TRY_AGAIN) continue;
      if (eflag != OK) return eflag;
      break;
    }
    complete_step();
    prepare_next_step(dsm);
    etamax = (nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) acor[i] *= tq[2];
    __syncwarp();
    return OK;
  }
  // CVodeReInit + CVodeSetInitStep(h0) + CVode(tout, CV_NORMAL); y (shared)
  // holds the initial values and receives the interpolated solution
  __device__ int integrate(double t0, double tout) {
    #pragma unroll 1
    for (int i = 0; i <= LMAX; ++i) tau[i] = 0.0;
    #pragma unroll 1
    for (int i = 0; i < 6; ++i) tq[i] = 0.0;
    q = 1;
    L = 2;
    qwait = L;
    etamax = ETAMX1;
    qprime = 1;
    nst = nfe = nsetups = netf = nni = ncfn = nje = 0;
    nstlp = nstlj = 0;
    saved_tq5 = 0.0;
    crate = 1.0;
    jcur = 0;
    hu = 0.0;
    tn = t0;
    gammap = gamma = 0.0;
    h = 0.0;
    h0 = tout - t0;
    eta = 1.0;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) {
      (zb + (0) * n)[i] = y[i];
      #pragma unroll 1
      for (int j = 1; j < LMAX; ++j) (zb + (j) * n)[i] = 0.0;
    }
    __syncwarp();
    if (!set_ewt((zb + (0) * n))) return ILL_INPUT;
    next_h = 0.0;
    if (f(y, (zb + (1) * n))) return REPTD_RHSFUNC_ERR;
    nfe++;
    h = h0;
    // a zero initial step makes CVODE estimate one (cvHin), which refuses an
    // output time at the initial time
    if (h0 == 0.0) return TOO_CLOSE;
    if ((tout - t0) * h < 0.0) return ILL_INPUT;
    hscale = h;
    hprime = h;
    #pragma unroll 1
    for (int i = lane; i < n; i += 32) (zb + (1) * n)[i] *= h;
    __syncwarp();
    int nstloc = 0;
    #pragma unroll 1
    for (;;) {
      next_h = h;
      if (nst > 0 && !set_ewt((zb + (0) * n))) return ILL_INPUT;
      if (max_steps > 0 && nstloc >= max_steps) return TOO_MUCH_WORK;
      double tolsf = UROUND * wrms((zb + (0) * n));
      if (tolsf > 1.0) return TOO_MUCH_ACC;
      int kflag = step();
      if (kflag != OK) return kflag;
      nstloc++;
      if ((tn - tout) * h >= 0.0) {
        double s = (tout - tn) / h;
        #pragma unroll 1
        for (int i = lane; i < n; i += 32) {
          double v = (zb + (q) * n)[i];
          #pragma unroll 1
          for (int j = q - 1; j >= 0; --j) v = (zb + (j) * n)[i] + s * v;
          y[i] = v;
        }
        __syncwarp();
        next_h = hprime;
        return OK;
      }
    }
  }
};

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
template <typename LT, bool AERO>
__device__ void bind_cell(Cell<LT, AERO>& c, const SolveArgs& a, const char* tab, char* base,
                          int gwarp, int lane) {
  c.tb = tab;
  c.atol = make_tab(tab).atol;
  c.lane = lane;
  c.n = a.off.n;
  // per-warp global slab: [Nordsieck history when it is not in shared
  // memory] [rate constants when they are not in shared memory]
  double* slab = a.hist ? a.hist + (size_t)gwarp * a.hist_stride : nullptr;
  c.zb = a.lay.zn >= 0 ? (double*)(base + a.lay.zn) : slab;
  double* ctl = (double*)(base + a.lay.ctl);
  c.tau = ctl;
  c.tq = ctl + (LMAX + 2);
  c.l = ctl + (LMAX + 2) + 8;
  c.ewt = (double*)(base + a.lay.ewt);
  c.acor = (double*)(base + a.lay.acor);
  c.y = (double*)(base + a.lay.y);
  c.ftemp = (double*)(base + a.lay.ftemp);
  c.tempv = (double*)(base + a.lay.tempv);
  c.rates = (double*)(base + a.lay.rates);
  c.keff = a.lay.keff >= 0 ? (double*)(base + a.lay.keff)
                           : slab + (a.lay.zn >= 0 ? 0 : (size_t)LMAX * a.off.n);
  c.fscr = (double*)(base + a.lay.fscr);
  c.LU = (LT*)(base + a.lay.lu);
  c.z = (LT*)(base + a.lay.z);
  c.dinv = (LT*)(base + a.lay.dinv);
  c.J = (LT*)a.jscratch + (size_t)gwarp * a.off.n_jac;
  c.rtol = a.rtol;
  c.max_steps = a.max_steps;
  c.maxncf = a.maxncf;
  c.maxnef = a.maxnef;
  c.lu_mode = a.lu_mode;
}

// AERO: the mechanism has SIMPOL, HL, aqueous equilibrium or sub-models,
// whose out-of-line evaluations take registers that the gas-phase form keeps
// for itself; that form runs fewer cells per block.
template <typename LT, bool AERO>
__global__ void __launch_bounds__(32 * (AERO ? kMaxCellsAero : kMaxCellsPerBlock), 1)
    solve_kernel(SolveArgs a) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long tma_bar;
  if (!stage_tables(smem, a.blob, a.stage_bytes, &tma_bar, a.err)) return;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * (blockDim.x >> 5) + wib;
  char* base = smem + a.tab_bytes + (size_t)wib * a.lay.bytes;
  Cell<LT, AERO> c;
  bind_cell<LT, AERO>(c, a, smem, base, gwarp, lane);
  const DevMech& m = a.m;
  const uint16_t* dep_state = make_tab(smem).dep_state;
  #pragma unroll 1
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(a.counter, 1);
    idx = __shfl_sync(FULLMASK, idx, 0);
    if (idx >= a.n_cells) break;
    const int cell = a.order ? a.order[idx] : idx;
    double* st = a.state + (size_t)cell * m.n_state;
    // solver_run: dependent values clamped to >= TINY, constants clamped in
    // place (src/camp_solver.c:554-567)
    #pragma unroll 1
    for (int i = lane; i < c.n; i += 32) {
      double v = st[dep_state[i]];
      c.y[i] = v > kTiny ? v : kTiny;
    }
    #pragma unroll 1
    for (int j = lane; j < m.n_const; j += 32) {
      int s = ldg(m.const_state + j);
      double v = st[s];
      st[s] = v > kTiny ? v : kTiny;
    }
    __syncwarp();
    const double T = a.env[2 * (size_t)cell], P = a.env[2 * (size_t)cell + 1];
    compute_keff(m, st, T, P, a.photo ? a.photo + (size_t)cell * m.n_photo : nullptr,
                 c.keff, lane);
    const double t0 = a.tspan ? a.tspan[2 * (size_t)cell] : a.t0;
    const double t1 = a.tspan ? a.tspan[2 * (size_t)cell + 1] : a.t1;
    int flag = c.integrate(t0, t1);
    if (flag == OK) {
      #pragma unroll 1
      for (int i = lane; i < c.n; i += 32) st[dep_state[i]] = c.y[i] > 0.0 ? c.y[i] : 0.0;
      if constexpr (AERO) {
        // the species the sub-models compute, at the final concentrations
        const BlobOff& o = *reinterpret_cast<const BlobOff*>(smem);
        if (o.n_cv > 0) {
          __syncwarp();
          double* cv = c.rates + o.n_rates;
          sub_model_eval(smem, c.y, c.keff, cv, nullptr, lane);
          const uint16_t* cs = (const uint16_t*)(smem + o.sm_state);
          #pragma unroll 1
          for (int k = lane; k < o.n_cv; k += 32) st[cs[k]] = cv[k];
        }
      }
    }
    if (lane == 0) {
      CellStats s;
      s.status = flag;
      s.nst = c.nst;
      s.nfe = c.nfe;
      s.nsetups = c.nsetups;
      s.netf = c.netf;
      s.nni = c.nni;
      s.ncfn = c.ncfn;
      s.nje = c.nje;
      s.hu = c.hu;
      s.hcur = c.next_h;
      a.stats[cell] = s;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// CTA-per-cell kernel (block.cuh): one block per cell; warp 0 runs the BDF
// control, every warp runs its f, J, factorization and solves
// ---------------------------------------------------------------------------
struct BlkLayout {  // byte offsets in the block's shared memory (zn -1: global)
  int ctx, ctl, y, ewt, acor, ftemp, tempv, part, dinv, z, zn, sg, lu, bytes;
};

struct BlkArgs {
  DevMech m;
  const char* blob;  // BlockOff tables in global memory
  BlkLayout lay;
  double* state;
  const double* env;
  const double* photo;
  const int* order;
  const double* tspan;
  int n_cells;
  int* counter;
  CellStats* stats;
  void* jscratch;    // per-block solver Jacobian slots
  double* hist;      // per-block Nordsieck history when not in shared memory
  int hist_stride;   // doubles per block in hist
  double* gscr;      // per-block rate constants and rate partials
  int gscr_stride;   // doubles per block in gscr
  double t0, t1, rtol;
  int max_steps, maxncf, maxnef;
};

// FP32 LU: half the shared memory, two cells per SM, so the register budget
// is that of two blocks
template <typename LT>
__global__ void __launch_bounds__(blk::kThreads, sizeof(LT) == 4 ? 2 : 1)
    block_kernel(BlkArgs a) {
  extern __shared__ __align__(16) char smem[];
  __shared__ blk::Cmd cmd;
  __shared__ int s_idx;
  const BlkLayout& L = a.lay;
  blk::Ctx<LT>* cx = reinterpret_cast<blk::Ctx<LT>*>(smem + L.ctx);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    blk::Ctx<LT> c;
    c.t = blk::make_tab(a.blob);
    c.keff = a.gscr + (size_t)blockIdx.x * a.gscr_stride;
    c.jpart = a.gscr + (size_t)blockIdx.x * a.gscr_stride + c.t.n_rxn;
    c.part = (double*)(smem + L.part);
    c.xbuf = (LT*)(smem + L.part);
    c.J = (LT*)a.jscratch + (size_t)blockIdx.x * c.t.n_jac;
    c.LU = (LT*)(smem + L.lu);
    c.dinv = (LT*)(smem + L.dinv);
    c.z = (LT*)(smem + L.z);
    c.rhs = (double*)(smem + L.tempv);
    const uint16_t* sg = (const uint16_t*)(smem + L.sg);
    c.rowptr = sg + c.t.sg_rowptr;
    c.diag = sg + c.t.sg_diag;
    c.ub = sg + c.t.sg_ub;
    c.perm = sg + c.t.sg_perm;
    c.hf_ptr = sg + c.t.sg_hf_ptr;
    c.hf_rows = sg + c.t.sg_hf_rows;
    c.hb_ptr = sg + c.t.sg_hb_ptr;
    c.hb_rows = sg + c.t.sg_hb_rows;
    c.ndoff = sg + c.t.sg_ndoff;
    c.ndcol = sg + c.t.sg_ndcol;
    c.dbase = sg + c.t.sg_dbase;
    c.hlk = sg + c.t.sg_hlk;
    c.hmid = sg + c.t.sg_hmid;
    c.htg = sg + c.t.sg_htg;
    *cx = c;
  }
  {
    // the solve's tables into shared memory (16-byte units)
    const campb::BlockOff& o = *reinterpret_cast<const campb::BlockOff*>(a.blob);
    const uint4* src = reinterpret_cast<const uint4*>(a.blob + o.stage);
    uint4* dst = reinterpret_cast<uint4*>(smem + L.sg);
    #pragma unroll 1
    for (int e = threadIdx.x; e < o.sg_len / 8; e += blk::kThreads) dst[e] = src[e];
  }
  blk::bsync();
  const DevMech& m = a.m;
  #pragma unroll 1
  for (;;) {
    if (threadIdx.x == 0) s_idx = atomicAdd(a.counter, 1);
    blk::bsync();
    const int idx = s_idx;
    if (idx >= a.n_cells) break;
    if (warp != 0) {
      blk::serve<LT>(&cmd, *cx);
      continue;
    }
    Cell<LT, false, true> c;
    c.tb = nullptr;
    c.cmd = &cmd;
    c.bx = cx;
    c.atol = cx->t.atol;
    c.lane = lane;
    c.n = cx->t.n;
    c.zb = L.zn >= 0 ? (double*)(smem + L.zn) : a.hist + (size_t)blockIdx.x * a.hist_stride;
    double* ctl = (double*)(smem + L.ctl);
    c.tau = ctl;
    c.tq = ctl + (LMAX + 2);
    c.l = ctl + (LMAX + 2) + 8;
    c.ewt = (double*)(smem + L.ewt);
    c.acor = (double*)(smem + L.acor);
    c.y = (double*)(smem + L.y);
    c.ftemp = (double*)(smem + L.ftemp);
    c.tempv = (double*)(smem + L.tempv);
    c.rates = (double*)(smem + L.part);
    c.keff = const_cast<double*>(cx->keff);
    c.fscr = nullptr;
    c.LU = cx->LU;
    c.z = cx->z;
    c.dinv = cx->dinv;
    c.J = cx->J;
    c.rtol = a.rtol;
    c.max_steps = a.max_steps;
    c.maxncf = a.maxncf;
    c.maxnef = a.maxnef;
    c.lu_mode = 0;
    const uint16_t* dep_state = cx->t.dep_state;
    const int cell = a.order ? a.order[idx] : idx;
    double* st = a.state + (size_t)cell * m.n_state;
    // solver_run: dependent values clamped to >= TINY, constants clamped in
    // place (src/camp_solver.c:554-567)
    #pragma unroll 1
    for (int i = lane; i < c.n; i += 32) {
      const double v = st[__ldg(dep_state + i)];
      c.y[i] = v > kTiny ? v : kTiny;
    }
    #pragma unroll 1
    for (int j = lane; j < m.n_const; j += 32) {
      const int s = ldg(m.const_state + j);
      const double v = st[s];
      st[s] = v > kTiny ? v : kTiny;
    }
    __syncwarp();
    const double T = a.env[2 * (size_t)cell], P = a.env[2 * (size_t)cell + 1];
    compute_keff(m, st, T, P, a.photo ? a.photo + (size_t)cell * m.n_photo : nullptr, c.keff,
                 lane);
    __syncwarp();
    const double t0 = a.tspan ? a.tspan[2 * (size_t)cell] : a.t0;
    const double t1 = a.tspan ? a.tspan[2 * (size_t)cell + 1] : a.t1;
    const int flag = c.integrate(t0, t1);
    if (flag == OK) {
      #pragma unroll 1
      for (int i = lane; i < c.n; i += 32)
        st[__ldg(dep_state + i)] = c.y[i] > 0.0 ? c.y[i] : 0.0;
    }
    if (lane == 0) {
      CellStats s;
      s.status = flag;
      s.nst = c.nst;
      s.nfe = c.nfe;
      s.nsetups = c.nsetups;
      s.netf = c.netf;
      s.nni = c.nni;
      s.ncfn = c.ncfn;
      s.nje = c.nje;
      s.hu = c.hu;
      s.hcur = c.next_h;
      a.stats[cell] = s;
    }
    blk::finish(&cmd);
  }
}

struct EvalArgs {
  DevMech m;
  BlobOff off;
  const void* blob;
  int tab_bytes;
  int stage_bytes;
  int* err;
  Layout lay;
  const double* state;
  const double* env;
  const double* photo;
  int n_cells;
  double h;
  double *rp, *rl, *f, *jp, *jl, *jv;
  int do_jac;
};

__global__ void eval_kernel(EvalArgs a) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long tma_bar;
  if (!stage_tables(smem, a.blob, a.stage_bytes, &tma_bar, a.err)) return;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int cell = blockIdx.x * (blockDim.x >> 5) + wib;
  if (cell >= a.n_cells) return;
  char* base = smem + a.tab_bytes + (size_t)wib * a.lay.bytes;
  const Tab t = make_tab(smem);
  const DevMech& m = a.m;
  double* y = (double*)(base + a.lay.y);
  double* rates = (double*)(base + a.lay.rates);
  double* keff = (double*)(base + a.lay.keff);
  double* fscr = (double*)(base + a.lay.fscr);
  const double* st = a.state + (size_t)cell * m.n_state;
  #pragma unroll 1
  for (int i = lane; i < t.n; i += 32) y[i] = st[t.dep_state[i]];
  __syncwarp();
  compute_keff(m, st, a.env[2 * cell], a.env[2 * cell + 1],
               a.photo ? a.photo + (size_t)cell * m.n_photo : nullptr, keff, lane);
  if (!a.do_jac) {
    double* out = (double*)(base + a.lay.ftemp);
    if (has_simpol(smem))
      dev_f_aero(smem, y, a.h, keff, rates, fscr, out, lane, a.rp + (size_t)cell * t.n,
                 a.rl + (size_t)cell * t.n);
    else
      dev_f(smem, y, a.h, keff, rates, fscr, out, lane, a.rp + (size_t)cell * t.n,
            a.rl + (size_t)cell * t.n);
    #pragma unroll 1
    for (int i = lane; i < t.n; i += 32) a.f[(size_t)cell * t.n + i] = out[i];
  } else {
    if (has_simpol(smem))
      dev_jac_aero<double>(smem, y, a.h, keff, rates, a.jv + (size_t)cell * t.n_jac, lane,
                           a.jp + (size_t)cell * t.n_jac, a.jl + (size_t)cell * t.n_jac);
    else
      dev_jac<double>(smem, y, a.h, keff, rates, a.jv + (size_t)cell * t.n_jac, lane,
                      a.jp + (size_t)cell * t.n_jac, a.jl + (size_t)cell * t.n_jac);
  }
}

// ---------------------------------------------------------------------------
// Finite-difference audit of the analytic Jacobian (debug tool)
// ---------------------------------------------------------------------------
// The counterpart of the reference's check_Jac (src/camp_solver.c:1146-1257)
// for one warp per cell: every element of column j of the solver Jacobian is
// compared with a forward-difference estimate over steps dx = x_j * 10^-12
// ... 10^0, as the reference's GSL forward derivative does: the differences
// at dx and dx/2 give the Richardson estimate 2 D(dx/2) - D(dx) and an error
// estimate (their difference plus the rounding of f, 4 eps (P + L) / (dx/2)
// from the production and loss sums).  An element passes at the first step
// where |J - estimate| < max(abs_tol, 1.2 error estimate) or the relative
// difference is below rel_tol.  Columns whose concentration is below SMALL
// are skipped, as in the reference.  Per cell: the number of elements that
// never passed and the largest best-step relative difference among them.
struct CheckArgs {
  EvalArgs e;        // tables, layout, state, env, photo, h; e.jv: J scratch
  double rel_tol, abs_tol;
  double* best;      // [n_cells * n_jac] best relative difference per element
  double* worst;     // [n_cells]
  int* nfail;        // [n_cells]
};

__global__ void jac_check_kernel(CheckArgs c) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long tma_bar;
  const EvalArgs& a = c.e;
  if (!stage_tables(smem, a.blob, a.stage_bytes, &tma_bar, a.err)) return;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int cell = blockIdx.x * (blockDim.x >> 5) + wib;
  if (cell >= a.n_cells) return;
  char* base = smem + a.tab_bytes + (size_t)wib * a.lay.bytes;
  const Tab t = make_tab(smem);
  const DevMech& m = a.m;
  double* y = (double*)(base + a.lay.y);
  double* f0 = (double*)(base + a.lay.ftemp);
  double* f1 = (double*)(base + a.lay.tempv);
  double* f2 = (double*)(base + a.lay.zn);
  double* rp0 = (double*)(base + a.lay.acor);
  double* rl0 = (double*)(base + a.lay.ewt);
  double* rates = (double*)(base + a.lay.rates);
  double* keff = (double*)(base + a.lay.keff);
  double* fscr = (double*)(base + a.lay.fscr);
  double* J = a.jv + (size_t)cell * t.n_jac;
  double* best = c.best + (size_t)cell * t.n_jac;
  const double* st = a.state + (size_t)cell * m.n_state;
  #pragma unroll 1
  for (int i = lane; i < t.n; i += 32) y[i] = st[t.dep_state[i]];
  __syncwarp();
  compute_keff(m, st, a.env[2 * cell], a.env[2 * cell + 1],
               a.photo ? a.photo + (size_t)cell * m.n_photo : nullptr, keff, lane);
  const bool aero = has_simpol(smem);
  if (dev_f_aero(smem, y, a.h, keff, rates, fscr, f0, lane, rp0, rl0) ||
      (aero ? dev_jac_aero<double>(smem, y, a.h, keff, rates, J, lane)
            : dev_jac<double>(smem, y, a.h, keff, rates, J, lane))) {
    if (lane == 0) {
      c.nfail[cell] = -1;
      c.worst[cell] = -1.0;
    }
    return;
  }
  #pragma unroll 1
  for (int e = lane; e < t.n_jac; e += 32) best[e] = -1.0;  // -1: not checked
  __syncwarp();
  #pragma unroll 1
  for (int j = 0; j < t.n; ++j) {
    const double x = y[j];
    if (x < kSmall) continue;
    const int e0 = ldg(m.jac_colptr + j), e1 = ldg(m.jac_colptr + j + 1);
    #pragma unroll 1
    for (int e = e0 + lane; e < e1; e += 32) best[e] = 1.0e300;
    __syncwarp();
    #pragma unroll 1
    for (double scale = 1.0e-12; scale <= 1.0; scale *= 10.0) {
      const double dx = x * scale;
      if (lane == 0) y[j] = x + dx;
      __syncwarp();
      int r = dev_f_aero(smem, y, a.h, keff, rates, fscr, f1, lane);
      if (lane == 0) y[j] = x + 0.5 * dx;
      __syncwarp();
      r |= dev_f_aero(smem, y, a.h, keff, rates, fscr, f2, lane);
      if (lane == 0) y[j] = x;
      __syncwarp();
      if (r) continue;
      bool all = true;
      #pragma unroll 1
      for (int e = e0 + lane; e < e1; e += 32) {
        const int i = ldg(m.jg_row + e);
        const double d1 = (f1[i] - f0[i]) / dx, d2 = (f2[i] - f0[i]) / (0.5 * dx);
        const double est = 2.0 * d2 - d1;
        const double err = fabs(d1 - d2) + 4.0 * UROUND * (rp0[i] + rl0[i]) / (0.5 * dx);
        const double diff = fabs(J[e] - est);
        const double rel = est != 0.0 ? diff / fabs(est) : (diff == 0.0 ? 0.0 : 1.0);
        const bool pass = diff < fmax(c.abs_tol, 1.2 * err) || rel < c.rel_tol;
        best[e] = pass ? 0.0 : fmin(best[e], rel);
        all &= best[e] == 0.0;
      }
      __syncwarp();
      if (warp_all(all)) break;
    }
  }
  int fails = 0;
  double worst = 0.0;
  #pragma unroll 1
  for (int e = lane; e < t.n_jac; e += 32) {
    if (best[e] > 0.0) {
      ++fails;
      worst = fmax(worst, best[e]);
    }
  }
  fails = warp_isum(fails);
  worst = warp_max(worst);
  if (lane == 0) {
    c.nfail[cell] = fails;
    c.worst[cell] = worst;
  }
}

// ---------------------------------------------------------------------------
// Host side of the engine
// ---------------------------------------------------------------------------
#define CK(call)                                                        \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) {                                            \
      *err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      return false;                                                     \
    }                                                                   \
  } while (0)

bool lanes_launch(const DevMech& m, const void* d_blob, const LaneOff& off, double* d_state,
                  const double* d_env, const double* d_photo, const int* d_order, int n_cells,
                  int* d_counter, CellStats* d_stats, void** scr64, size_t* cap64,
                  void** scrlt, size_t* caplt, double t0, double t1, const SolveSettings& s,
                  int sm_count, int max_smem, void* stream, std::string* err);

// Precision audit: per cell, the Jacobian at its state, M = I - h J
// factored on the fixed order in precision LT and solved for a right-hand
// side of tolerance size (b_i = +-(rtol |y_i| + atol_i), signs from a fixed
// hash of i); the solution goes to x.  Run once in FP64 and once in FP32, the
// host compares them in the error-weighted norm: the accuracy the mixed
// form's Newton iteration has to refine.
struct PrecArgs {
  EvalArgs e;   // tables, layout (LU in LT), state, env, photo, h
  void* jbuf;   // [n_cells * n_jac] of LT
  double rtol;
  double* x;    // [n_cells * n]
  int* bad;     // [n_cells]: 1 when f / J or the factorization failed
};

template <typename LT>
__global__ void precision_kernel(PrecArgs p) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long tma_bar;
  const EvalArgs& a = p.e;
  if (!stage_tables(smem, a.blob, a.stage_bytes, &tma_bar, a.err)) return;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int cell = blockIdx.x * (blockDim.x >> 5) + wib;
  if (cell >= a.n_cells) return;
  char* base = smem + a.tab_bytes + (size_t)wib * a.lay.bytes;
  const Tab t = make_tab(smem);
  const DevMech& m = a.m;
  double* y = (double*)(base + a.lay.y);
  double* rates = (double*)(base + a.lay.rates);
  double* keff = (double*)(base + a.lay.keff);
  double* b = (double*)(base + a.lay.tempv);
  LT* LU = (LT*)(base + a.lay.lu);
  LT* z = (LT*)(base + a.lay.z);
  LT* dinv = (LT*)(base + a.lay.dinv);
  LT* J = (LT*)p.jbuf + (size_t)cell * t.n_jac;
  const double* st = a.state + (size_t)cell * m.n_state;
  #pragma unroll 1
  for (int i = lane; i < t.n; i += 32) y[i] = st[t.dep_state[i]];
  __syncwarp();
  compute_keff(m, st, a.env[2 * cell], a.env[2 * cell + 1],
               a.photo ? a.photo + (size_t)cell * m.n_photo : nullptr, keff, lane);
  int r = has_simpol(smem) ? dev_jac_aero<LT>(smem, y, a.h, keff, rates, J, lane)
                           : dev_jac<LT>(smem, y, a.h, keff, rates, J, lane);
  bool ok = r == 0 && dev_form_factor<LT>(smem, J, a.h, LU, dinv, lane);
  if (ok) {
    #pragma unroll 1
    for (int i = lane; i < t.n; i += 32) {
      const double s = p.rtol * fabs(y[i]) + t.atol[i];
      b[i] = ((i * 2654435761u) >> 13) & 1u ? s : -s;
    }
    __syncwarp();
    dev_lsolve<LT>(smem, LU, dinv, b, z, lane);
    #pragma unroll 1
    for (int i = lane; i < t.n; i += 32) p.x[(size_t)cell * t.n + i] = b[i];
  }
  if (lane == 0) p.bad[cell] = ok ? 0 : 1;
}

struct Engine::Impl {
  DevMech m{};
  BlobOff off{};
  void* d_blob = nullptr;
  // the warp-per-cell tables use 16-bit encodings; a mechanism beyond them
  // (e.g. an LU with hundreds of thousands of Schur updates) runs on the
  // lane-per-cell kernel only, and warp_why says why
  bool warp_ok = true, lanes_ok = true, blk_ok = false;
  std::string warp_why, lanes_why, blk_why;
  BlockOff boff{};
  void* d_bblob = nullptr;
  LaneOff loff{};
  void* d_lblob = nullptr;
  void *d_scr64 = nullptr, *d_scrlt = nullptr;
  size_t c_scr64 = 0, c_scrlt = 0;
  void* d_tables = nullptr;
  int capacity = 0;
  int n_state = 0, n_photo = 0;
  int sm_count = 0, max_smem = 0;
  // buffers
  void *d_state = nullptr, *d_env = nullptr, *d_photo = nullptr, *d_order = nullptr;
  size_t c_state = 0, c_env = 0, c_photo = 0, c_order = 0;
  void* d_stats = nullptr;
  size_t c_stats = 0;
  int* d_counter = nullptr;
  void* d_jscratch = nullptr;
  size_t c_jscratch = 0;
  void* d_hist = nullptr;
  size_t c_hist = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool ev_pending = false;
  // the device step (counter reset + solve kernel) as an instantiated graph;
  // its kernel node's launch shape and arguments are updated per launch
  cudaGraph_t graph = nullptr;  // kept: its node handles address the exec's nodes
  cudaGraphExec_t gexec = nullptr;
  cudaGraphNode_t gkernel = nullptr;
  int gprecision = -1, ggrid = 0, gblock = 0;
  size_t gsmem = 0;
};

Engine::Engine() : impl_(new Impl) {}

Engine::~Engine() {
  Impl* I = impl_;
  cudaFree(I->d_tables);
  cudaFree(I->d_blob);
  cudaFree(I->d_lblob);
  cudaFree(I->d_bblob);
  cudaFree(I->d_scr64);
  cudaFree(I->d_scrlt);
  cudaFree(I->d_state);
  cudaFree(I->d_env);
  cudaFree(I->d_photo);
  cudaFree(I->d_order);
  cudaFree(I->d_stats);
  cudaFree(I->d_counter);
  cudaFree(I->d_jscratch);
  cudaFree(I->d_hist);
  if (I->ev0) cudaEventDestroy(I->ev0);
  if (I->ev1) cudaEventDestroy(I->ev1);
  if (I->gexec) cudaGraphExecDestroy(I->gexec);
  if (I->graph) cudaGraphDestroy(I->graph);
  delete I;
}

bool Engine::ensure(void** p, size_t* cap, size_t bytes, std::string* err) {
  if (*cap >= bytes && *p) return true;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  CK(cudaMalloc(p, bytes > 0 ? bytes : 16));
  *cap = bytes;
  return true;
}

namespace {
// packs host vectors into one device blob; returns device pointers
struct Packer {
  std::vector<char> blob;
  std::vector<std::pair<size_t, const void**>> fix;
  template <typename T>
  void add(const std::vector<T>& v, const T** dst) {
    size_t off = (blob.size() + 15) & ~size_t(15);
    blob.resize(off + std::max<size_t>(v.size(), 1) * sizeof(T), 0);
    if (!v.empty()) memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
    fix.push_back({off, (const void**)dst});
  }
};
}  // namespace

bool Engine::init(const Model& model, const std::vector<double>& atol_dep, int capacity,
                  std::string* err) {
  Impl* I = impl_;
  const Tables& t = model.tables();
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&I->sm_count, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaDeviceGetAttribute(&I->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  DevMech& m = I->m;
  m.n = t.n;
  m.n_state = t.n_state;
  m.n_rxn = t.n_rxn;
  m.n_part = t.n_part;
  m.n_jac = t.n_jac;
  m.n_lu = t.n_lu;
  m.n_photo = t.n_photo;
  m.n_flev = t.n_flev;
  m.n_blev = t.n_blev;
  std::vector<int> cst;
  for (int i = 0; i < t.n_state; ++i)
    if (model.var_type()[i] == VAR_CONSTANT) cst.push_back(i);
  m.n_const = (int)cst.size();
  // SIMPOL instances (device-side constants; see rates.cuh)
  std::vector<double> si_prm, si_dp, si_cinv_rho, si_cinv_mw, si_cin;
  std::vector<int> si_type, si_kind, si_gmd, si_gsd, si_act, si_water, si_wcv, si_nph,
      si_cptr(1, 0), si_cidx;
  for (const SimpolInst& si : t.simpol) {
    si_prm.insert(si_prm.end(), si.prm, si.prm + 10);
    si_type.push_back(si.type);
    si_kind.push_back(si.kind);
    si_gmd.push_back(si.gmd_col);
    si_gsd.push_back(si.gsd_col);
    si_dp.push_back(si.bin_dp);
    si_act.push_back(si.act);
    si_water.push_back(si.water);
    si_wcv.push_back(si.water_cv);
    si_nph.push_back(si.n_phases);
    const size_t ne = si.type == RXN_SIMPOL_PHASE_TRANSFER ? si.elem.size() : 0;
    for (size_t j = 0; j < ne; ++j) {
      if (model.var_type()[si.elem[j]] == VAR_VARIABLE) continue;
      si_cidx.push_back(si.elem[j]);
      si_cinv_rho.push_back(si.inv_rho[j]);
      si_cinv_mw.push_back(si.inv_mw[j]);
      si_cin.push_back(si.in_phase[j] ? 1.0 : 0.0);
    }
    si_cptr.push_back((int)si_cidx.size());
  }
  m.n_simpol = t.n_simpol;
  // aqueous equilibrium instances (device-side constants; see rates.cuh)
  std::vector<double> aq_prm, aq_cm;
  std::vector<int> aq_int, aq_cptr(1, 0), aq_cidx, aq_cr;
  for (const AqInst& q : t.aq) {
    aq_prm.insert(aq_prm.end(), {q.A, q.C, q.kr, q.thr});
    aq_int.insert(aq_int.end(), {q.water, q.act, (int)q.react.size(), (int)q.prod.size(),
                                 q.water_cv, q.act_cv});
    for (int pass = 0; pass < 2; ++pass) {
      const std::vector<int>& list = pass == 0 ? q.react : q.prod;
      for (size_t i = 0; i < list.size(); ++i) {
        if (model.var_type()[list[i]] == VAR_VARIABLE) continue;
        if (std::find(q.cp_state.begin(), q.cp_state.end(), list[i]) != q.cp_state.end())
          continue;  // computed by a sub-model: applied per evaluation
        aq_cidx.push_back(list[i]);
        aq_cm.push_back(q.m2m[(pass == 0 ? 0 : q.react.size()) + i]);
        aq_cr.push_back(pass == 0 ? 1 : 0);
      }
    }
    aq_cptr.push_back((int)aq_cidx.size());
  }
  m.n_aq = t.n_aq;
  m.sm_keff = t.sm_keff;
  Packer pk;
  pk.add(aq_prm, &m.aq_prm);
  pk.add(aq_cm, &m.aq_cm);
  pk.add(aq_int, &m.aq_int);
  pk.add(aq_cptr, &m.aq_cptr);
  pk.add(aq_cidx, &m.aq_cidx);
  pk.add(aq_cr, &m.aq_cr);
  pk.add(si_prm, &m.si_prm);
  pk.add(si_type, &m.si_type);
  pk.add(si_kind, &m.si_kind);
  pk.add(si_gmd, &m.si_gmd_col);
  pk.add(si_gsd, &m.si_gsd_col);
  pk.add(si_act, &m.si_act);
  pk.add(si_water, &m.si_water);
  pk.add(si_wcv, &m.si_wcv);
  pk.add(si_nph, &m.si_nph);
  pk.add(si_cptr, &m.si_cptr);
  pk.add(si_cidx, &m.si_cidx);
  pk.add(si_dp, &m.si_dp);
  pk.add(si_cinv_rho, &m.si_cinv_rho);
  pk.add(si_cinv_mw, &m.si_cinv_mw);
  pk.add(si_cin, &m.si_cin);
  pk.add(t.rx_type, &m.rx_type);
  pk.add(t.rx_nreact, &m.rx_nreact);
  pk.add(t.rx_fpar, &m.rx_fpar);
  pk.add(t.rx_photo, &m.rx_photo);
  pk.add(t.fpar, &m.fpar);
  pk.add(t.rx_cptr, &m.rx_cptr);
  pk.add(t.rx_cidx, &m.rx_cidx);
  pk.add(t.rx_vptr, &m.rx_vptr);
  pk.add(t.rx_vdep, &m.rx_vdep);
  pk.add(t.fg_ptr, &m.fg_ptr);
  pk.add(t.fg_rxn, &m.fg_rxn);
  pk.add(t.fg_prod, &m.fg_prod);
  pk.add(t.fg_coef, &m.fg_coef);
  pk.add(t.jg_ptr, &m.jg_ptr);
  pk.add(t.jg_part, &m.jg_part);
  pk.add(t.jg_ind, &m.jg_ind);
  pk.add(t.jg_lupos, &m.jg_lupos);
  pk.add(t.jg_row, &m.jg_row);
  pk.add(model.device_colptr(), &m.jac_colptr);
  pk.add(t.jg_coef, &m.jg_coef);
  pk.add(t.lu_perm, &m.lu_perm);
  pk.add(t.lu_rowptr, &m.lu_rowptr);
  pk.add(t.lu_col, &m.lu_col);
  pk.add(t.lu_diag, &m.lu_diag);
  pk.add(t.upd_ptr, &m.upd_ptr);
  pk.add(t.upd_src, &m.upd_src);
  pk.add(t.upd_dst, &m.upd_dst);
  pk.add(t.fl_ptr, &m.fl_ptr);
  pk.add(t.fl_rows, &m.fl_rows);
  pk.add(t.bl_ptr, &m.bl_ptr);
  pk.add(t.bl_rows, &m.bl_rows);
  pk.add(t.dep_state, &m.dep_state);
  pk.add(cst, &m.const_state);
  pk.add(atol_dep, &m.atol);
  if (I->d_tables) cudaFree(I->d_tables);
  I->d_tables = nullptr;
  CK(cudaMalloc(&I->d_tables, pk.blob.size()));
  CK(cudaMemcpy(I->d_tables, pk.blob.data(), pk.blob.size(), cudaMemcpyHostToDevice));
  for (auto& f : pk.fix) *f.second = (const void*)((char*)I->d_tables + f.first);
  std::vector<uint8_t> blob;
  if (I->d_blob) cudaFree(I->d_blob);
  I->d_blob = nullptr;
  I->warp_why.clear();
  I->warp_ok = build_blob(t, atol_dep, &blob, &I->off, &I->warp_why);
  if (I->warp_ok) {
    CK(cudaMalloc(&I->d_blob, blob.size()));
    CK(cudaMemcpy(I->d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  }
  std::vector<uint8_t> lblob;
  if (I->d_lblob) cudaFree(I->d_lblob);
  I->d_lblob = nullptr;
  I->lanes_why.clear();
  I->lanes_ok = build_lane_blob(t, atol_dep, &lblob, &I->loff, &I->lanes_why);
  std::vector<uint8_t> bblob;
  if (I->d_bblob) cudaFree(I->d_bblob);
  I->d_bblob = nullptr;
  I->blk_why.clear();
  I->blk_ok = build_block_blob(t, atol_dep, &bblob, &I->boff, &I->blk_why);
  if (I->blk_ok) {
    CK(cudaMalloc(&I->d_bblob, bblob.size()));
    CK(cudaMemcpy(I->d_bblob, bblob.data(), bblob.size(), cudaMemcpyHostToDevice));
  }
  if (!I->warp_ok && !I->lanes_ok && !I->blk_ok) {
    *err = "mechanism fits no kernel: " + I->warp_why + "; " + I->lanes_why + "; " +
           I->blk_why;
    return false;
  }
  if (I->lanes_ok) {
    CK(cudaMalloc(&I->d_lblob, lblob.size()));
    CK(cudaMemcpy(I->d_lblob, lblob.data(), lblob.size(), cudaMemcpyHostToDevice));
  }
  I->capacity = capacity;
  I->n_state = t.n_state;
  I->n_photo = t.n_photo;
  if (!I->d_counter) CK(cudaMalloc((void**)&I->d_counter, sizeof(int) * 4));
  if (!I->ev0) {
    CK(cudaEventCreate(&I->ev0));
    CK(cudaEventCreate(&I->ev1));
  }
  return true;
}

// per-warp shared-memory slice; the solve kernel keeps the Nordsieck history
// and the rate constants in global memory (with_hist = false), which leaves
// room for more resident cells
static Layout make_layout(const BlobOff& o, int lt_size, bool with_hist,
                          bool keff_in_smem) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t r = off;
    off = (off + bytes + 15) & ~size_t(15);
    return (int)r;
  };
  const size_t vec = sizeof(double) * o.n;
  L.zn = with_hist ? take(vec * LMAX) : -1;
  L.ewt = take(vec);
  L.acor = take(vec);
  L.y = take(vec);
  L.ftemp = take(vec);
  L.tempv = take(vec);
  // the f scratch (pseudo-rates, then the computed species) and the J
  // scratch (partials, computed species, parameter partials, virtual slots)
  L.rates = take(sizeof(double) * std::max(o.n_rates + o.n_cv,
                                           o.n_part_all + o.n_cv + o.n_pj + o.n_virt));
  L.keff = keff_in_smem ? take(sizeof(double) * o.n_keff) : -1;
  L.fscr = take(sizeof(double) * 2 * std::max(1, o.n_fscratch));
  // one spare slot each: the target of the grouped phases' no-op records
  L.lu = take((size_t)lt_size * (o.n_lu + 1));
  L.z = take((size_t)lt_size * (o.n + 1));
  L.dinv = take((size_t)lt_size * o.n);
  // control block: tau[LMAX + 2], tq[8], l[LMAX + 1]
  L.ctl = take(sizeof(double) * (LMAX + 2 + 8 + LMAX + 1));
  L.bytes = (int)off;
  return L;
}

// shared-memory bytes of the staged tables: the one-lane LU mode also needs
// the row-wise LU tables at the end of the blob
static int stage_bytes_of(const BlobOff& o, int lu_mode) {
  return lu_mode ? o.bytes : o.stage_bytes;
}
static int tab_bytes_of(const BlobOff& o, int lu_mode) {
  return (stage_bytes_of(o, lu_mode) + 127) & ~127;
}

// Geometry and launch of the warp-per-cell kernel shared by the solver's own
// launches and the serving slots.  Scratch pointers come from the caller.
// the solve kernel's form for a mechanism: aerosol reactions or sub-models
// take the AERO instance (fewer cells per block, see solve_kernel)
static bool aero_form(const BlobOff& o) { return o.n_simpol > 0 || o.n_aq > 0 || o.n_cv > 0; }
static int max_cells_of(const BlobOff& o) {
  return aero_form(o) ? kMaxCellsAero : kMaxCellsPerBlock;
}
static void* solve_kernel_fn(const BlobOff& o, int precision) {
  if (aero_form(o))
    return precision == 1 ? (void*)solve_kernel<float, true> : (void*)solve_kernel<double, true>;
  return precision == 1 ? (void*)solve_kernel<float, false> : (void*)solve_kernel<double, false>;
}

struct WarpLaunch {
  int grid = 0, warps = 0, tab = 0, lt = 8;
  Layout lay{};
  size_t smem = 0;
};

static bool plan_warp_launch(const BlobOff& off, int sm_count, int max_smem,
                             const SolveSettings& s, int n_cells, int max_blocks,
                             WarpLaunch* w, std::string* err) {
  w->lt = s.precision == 1 ? 4 : 8;
  w->lay = make_layout(off, w->lt, s.hist_global == 0, true);
  w->tab = tab_bytes_of(off, s.lu_mode);
  int max_warps = (max_smem - w->tab) / w->lay.bytes;
  if (max_warps < 1) {
    *err = "mechanism too large for the shared-memory layout (" +
           std::to_string(w->lay.bytes) + " bytes per cell)";
    return false;
  }
  int warps = s.warps_per_block > 0 ? std::min(s.warps_per_block, max_warps) : max_warps;
  warps = std::min(warps, max_cells_of(off));
  int bps = std::max(1, s.blocks_per_sm);
  while (bps > 1 && (size_t)bps * (w->tab + warps * w->lay.bytes) > (size_t)max_smem) --bps;
  int grid = std::min(sm_count * bps, std::max(1, max_blocks));
  // no more warps than cells
  if ((long)grid * warps > n_cells) grid = std::max(1, (int)((n_cells + warps - 1) / warps));
  w->grid = grid;
  w->warps = warps;
  w->smem = (size_t)w->tab + (size_t)warps * w->lay.bytes;
  return true;
}

static int hist_stride_of(const BlobOff& off, const SolveSettings& s) {
  // global slab per warp for the Nordsieck history when it is not in shared
  // memory, rounded to 256-byte rows (the rate constants stay in shared
  // memory: they sit on the dependent path of every f and J evaluation)
  return s.hist_global ? (LMAX * off.n + 31) & ~31 : 0;
}

static bool launch_warp_kernel(SolveArgs& a, const WarpLaunch& w, int precision,
                               cudaStream_t st, std::string* err) {
  void* func = solve_kernel_fn(a.off, precision);
  CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w.smem));
  void* args[] = {&a};
  CK(cudaLaunchKernel(func, dim3(w.grid), dim3(w.warps * 32), args, w.smem, st));
  return true;
}

void Engine::fill_args(SolveArgs* a, const WarpLaunch& w, const SolveSettings& s, double* d_state,
                       const double* d_env, const double* d_photo, const int* d_order,
                       int n_cells, double t0, double t1) const {
  const Impl* I = impl_;
  a->m = I->m;
  a->off = I->off;
  a->blob = I->d_blob;
  a->tab_bytes = w.tab;
  a->stage_bytes = stage_bytes_of(I->off, s.lu_mode);
  a->lay = w.lay;
  a->state = d_state;
  a->env = d_env;
  a->photo = I->m.n_photo > 0 ? d_photo : nullptr;
  a->order = d_order;
  a->n_cells = n_cells;
  a->t0 = t0;
  a->t1 = t1;
  a->rtol = s.rtol;
  a->max_steps = s.max_steps;
  a->maxncf = s.max_conv_fails;
  a->maxnef = s.max_conv_fails;
  a->lu_mode = s.lu_mode;
}

// shared-memory layout of one block of the CTA-per-cell kernel
static BlkLayout make_blk_layout(const BlockOff& o, int lt, bool zn_in_smem) {
  BlkLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const int r = (int)off;
    off = (off + bytes + 15) & ~size_t(15);
    return r;
  };
  const size_t n = (size_t)o.n;
  L.ctx = take(sizeof(blk::Ctx<double>));
  L.ctl = take(sizeof(double) * (LMAX + 2 + 8 + LMAX + 1));
  L.y = take(8 * n);
  L.ewt = take(8 * n);
  L.acor = take(8 * n);
  L.ftemp = take(8 * n);
  L.tempv = take(8 * n);
  // term rates, and during a factorization its exchange vectors (the rate
  // constants and partials live in global scratch)
  L.part = take(std::max(8 * (size_t)o.n_rxn, (size_t)lt * blk::kXBuf));
  L.dinv = take((size_t)lt * n);
  L.z = take((size_t)lt * n);
  L.zn = zn_in_smem ? take(8 * LMAX * n) : -1;
  L.sg = take(2 * (size_t)o.sg_len);
  L.lu = take((size_t)lt * o.n_lu);
  L.bytes = (int)off;
  return L;
}

static void* block_kernel_fn(int precision) {
  return precision == 1 ? (void*)block_kernel<float> : (void*)block_kernel<double>;
}

struct BlkLaunch {
  int grid = 0, lt = 8, per_sm = 0;
  BlkLayout lay{};
};

// the layout that fits the most blocks per SM (the Nordsieck history in
// shared memory on a tie), one block per cell at most
static bool plan_blk_launch(const BlockOff& o, int sm_count, int max_smem, int precision,
                            int n_cells, BlkLaunch* b, std::string* err) {
  b->lt = precision == 1 ? 4 : 8;
  void* fn = block_kernel_fn(precision);
  // the kernel's static shared memory (the command slot) counts against the
  // same per-block limit
  cudaFuncAttributes fa{};
  CK(cudaFuncGetAttributes(&fa, fn));
  const int max_dyn = max_smem - (int)fa.sharedSizeBytes;
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn));
  b->per_sm = 0;
  for (int zs = 1; zs >= 0; --zs) {
    const BlkLayout L = make_blk_layout(o, b->lt, zs == 1);
    if (L.bytes > max_dyn) continue;
    int nb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, blk::kThreads, (size_t)L.bytes));
    if (nb > b->per_sm) {
      b->per_sm = nb;
      b->lay = L;
    }
  }
  if (b->per_sm < 1) {
    *err = "mechanism too large for the CTA-per-cell shared-memory layout";
    return false;
  }
  b->grid = std::max(1, std::min(sm_count * b->per_sm, n_cells));
  return true;
}

bool Engine::block_tables() const { return impl_->blk_ok; }

int Engine::effective_kernel(const SolveSettings& s) const {
  if (s.kernel != 0) return s.kernel;
  if (impl_->warp_ok) return 0;
  return impl_->blk_ok ? 2 : 1;
}

bool Engine::launch_block(double* d_state, const double* d_env, const double* d_photo,
                          const int* d_order, int n_cells, double t0, double t1,
                          const SolveSettings& s, void* stream, std::string* err) {
  Impl* I = impl_;
  if (!I->blk_ok) {
    *err = "the CTA-per-cell kernel cannot run this mechanism: " + I->blk_why;
    return false;
  }
  cudaStream_t st = (cudaStream_t)stream;
  BlkLaunch b;
  if (!plan_blk_launch(I->boff, I->sm_count, I->max_smem, s.precision, n_cells, &b, err))
    return false;
  if (!ensure(&I->d_stats, &I->c_stats, sizeof(CellStats) * (size_t)n_cells, err)) return false;
  if (!ensure(&I->d_jscratch, &I->c_jscratch, (size_t)b.lt * I->boff.n_jac * b.grid, err))
    return false;
  const int hist_stride = b.lay.zn >= 0 ? 0 : (LMAX * I->boff.n + 31) & ~31;
  const int gscr_stride = (I->boff.n_rxn + I->boff.n_part + 31) & ~31;
  if (!ensure(&I->d_hist, &I->c_hist,
              sizeof(double) * (size_t)(hist_stride + gscr_stride) * b.grid, err))
    return false;
  BlkArgs a{};
  a.m = I->m;
  a.blob = (const char*)I->d_bblob;
  a.lay = b.lay;
  a.state = d_state;
  a.env = d_env;
  a.photo = I->m.n_photo > 0 ? d_photo : nullptr;
  a.order = d_order;
  a.tspan = nullptr;
  a.n_cells = n_cells;
  a.counter = I->d_counter;
  a.stats = (CellStats*)I->d_stats;
  a.jscratch = I->d_jscratch;
  a.hist = (double*)I->d_hist;
  a.hist_stride = hist_stride;
  a.gscr = (double*)I->d_hist + (size_t)hist_stride * b.grid;
  a.gscr_stride = gscr_stride;
  a.t0 = t0;
  a.t1 = t1;
  a.rtol = s.rtol;
  a.max_steps = s.max_steps;
  a.maxncf = s.max_conv_fails;
  a.maxnef = s.max_conv_fails;
  void* fn = block_kernel_fn(s.precision);
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, b.lay.bytes));
  void* args[] = {&a};
  CK(cudaEventRecord(I->ev0, st));
  CK(cudaMemsetAsync(I->d_counter, 0, sizeof(int), st));
  CK(cudaLaunchKernel(fn, dim3(b.grid), dim3(blk::kThreads), args, (size_t)b.lay.bytes, st));
  CK(cudaEventRecord(I->ev1, st));
  I->ev_pending = true;
  ++launches_;
  return true;
}

bool Engine::launch_solve(double* d_state, const double* d_env, const double* d_photo,
                          const int* d_order, int n_cells, double t0, double t1,
                          const SolveSettings& s, void* stream, std::string* err) {
  Impl* I = impl_;
  if (n_cells <= 0) return true;
  cudaStream_t st = (cudaStream_t)stream;
  const int kern = effective_kernel(s);
  if (kern == 2)
    return launch_block(d_state, d_env, d_photo, d_order, n_cells, t0, t1, s, stream, err);
  if (kern == 1) {
    if (!I->lanes_ok) {
      *err = "the lane-per-cell kernel cannot run this mechanism: " + I->lanes_why;
      return false;
    }
    if (!ensure(&I->d_stats, &I->c_stats, sizeof(CellStats) * (size_t)n_cells, err)) return false;
    CK(cudaEventRecord(I->ev0, st));
    if (!lanes_launch(I->m, I->d_lblob, I->loff, d_state, d_env, d_photo, d_order, n_cells,
                      I->d_counter, (CellStats*)I->d_stats, &I->d_scr64, &I->c_scr64,
                      &I->d_scrlt, &I->c_scrlt, t0, t1, s, I->sm_count, I->max_smem, stream,
                      err))
      return false;
    CK(cudaEventRecord(I->ev1, st));
    I->ev_pending = true;
    ++launches_;
    return true;
  }
  WarpLaunch w;
  if (!plan_warp_launch(I->off, I->sm_count, I->max_smem, s, n_cells, I->sm_count * 64, &w, err))
    return false;
  const long total_warps = (long)w.grid * w.warps;
  if (!ensure(&I->d_stats, &I->c_stats, sizeof(CellStats) * (size_t)n_cells, err)) return false;
  if (!ensure(&I->d_jscratch, &I->c_jscratch, (size_t)w.lt * I->m.n_jac * total_warps, err))
    return false;
  const int hist_stride = hist_stride_of(I->off, s);
  if (hist_stride &&
      !ensure(&I->d_hist, &I->c_hist, sizeof(double) * (size_t)hist_stride * total_warps, err))
    return false;
  SolveArgs a;
  fill_args(&a, w, s, d_state, d_env, d_photo, d_order, n_cells, t0, t1);
  a.err = I->d_counter + 1;
  a.counter = I->d_counter;
  a.stats = (CellStats*)I->d_stats;
  a.jscratch = I->d_jscratch;
  a.hist = (double*)I->d_hist;
  a.hist_stride = hist_stride;
  CK(cudaEventRecord(I->ev0, st));
  if (s.use_graph) {
    if (!launch_graph(a, w, s.precision, st, err)) return false;
  } else {
    CK(cudaMemsetAsync(I->d_counter, 0, sizeof(int), st));
    if (!launch_warp_kernel(a, w, s.precision, st, err)) return false;
  }
  CK(cudaEventRecord(I->ev1, st));
  I->ev_pending = true;
  ++launches_;
  return true;
}

bool Engine::launch_graph(SolveArgs& a, const WarpLaunch& w, int precision, void* stream,
                          std::string* err) {
  Impl* I = impl_;
  cudaStream_t st = (cudaStream_t)stream;
  void* func = solve_kernel_fn(a.off, precision);
  CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w.smem));
  void* args[] = {&a};
  cudaKernelNodeParams kp{};
  kp.func = func;
  kp.gridDim = dim3(w.grid);
  kp.blockDim = dim3(w.warps * 32);
  kp.sharedMemBytes = (unsigned)w.smem;
  kp.kernelParams = args;
  // an instantiated kernel node takes new arguments but keeps its launch
  // shape: a new shape (fewer cells than resident warps, other settings)
  // instantiates the graph again
  if (!I->gexec || I->gprecision != precision || I->ggrid != w.grid ||
      I->gblock != w.warps * 32 || I->gsmem != w.smem) {
    if (I->gexec) cudaGraphExecDestroy(I->gexec);
    if (I->graph) cudaGraphDestroy(I->graph);
    I->gexec = nullptr;
    I->graph = nullptr;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    I->graph = g;
    cudaMemsetParams mp{};
    mp.dst = I->d_counter;
    mp.value = 0;
    mp.elementSize = sizeof(int);
    mp.width = 1;
    mp.height = 1;
    cudaGraphNode_t mset = nullptr;
    cudaError_t e = cudaGraphAddMemsetNode(&mset, g, nullptr, 0, &mp);
    if (e == cudaSuccess) e = cudaGraphAddKernelNode(&I->gkernel, g, &mset, 1, &kp);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&I->gexec, g, 0);
    if (e != cudaSuccess) {
      *err = std::string("solve graph: ") + cudaGetErrorString(e);
      I->gexec = nullptr;
      return false;
    }
    I->gprecision = precision;
    I->ggrid = w.grid;
    I->gblock = w.warps * 32;
    I->gsmem = w.smem;
  } else {
    CK(cudaGraphExecKernelNodeSetParams(I->gexec, I->gkernel, &kp));
  }
  CK(cudaGraphLaunch(I->gexec, st));
  return true;
}

bool Engine::warp_tables(std::string* err) const {
  if (impl_->warp_ok) return true;
  *err = "this entry point runs the warp-per-cell kernel, whose tables this mechanism "
         "exceeds (" + impl_->warp_why + "); solver_run and the device runs use the "
         "block-per-cell or lane-per-cell kernel for it";
  return false;
}

bool Engine::lane_tables() const { return impl_->lanes_ok; }

size_t Engine::slot_scratch_bytes(const SolveSettings& s, int max_blocks) const {
  const Impl* I = impl_;
  if (!I->warp_ok) return 0;
  WarpLaunch w;
  std::string err;
  if (!plan_warp_launch(I->off, I->sm_count, I->max_smem, s, 1 << 30, max_blocks, &w, &err))
    return 0;
  const size_t warps = (size_t)w.grid * w.warps;
  const size_t j = ((size_t)w.lt * I->m.n_jac * warps + 255) & ~size_t(255);
  const size_t h = sizeof(double) * (size_t)hist_stride_of(I->off, s) * warps;
  return 256 + j + h;
}

bool Engine::launch_solve_slot(double* d_state, const double* d_env, const double* d_photo,
                               CellStats* d_stats, const double* d_tspan, int n_cells,
                               const SolveSettings& s, char* scratch, size_t scratch_bytes,
                               int max_blocks, void* stream, std::string* err) {
  Impl* I = impl_;
  if (n_cells <= 0) return true;
  if (s.kernel != 0) {
    *err = "serving slots run the warp-per-cell kernel only";
    return false;
  }
  if (!warp_tables(err)) return false;
  cudaStream_t st = (cudaStream_t)stream;
  WarpLaunch w;
  if (!plan_warp_launch(I->off, I->sm_count, I->max_smem, s, n_cells, max_blocks, &w, err))
    return false;
  const size_t warps = (size_t)w.grid * w.warps;
  const size_t jb = ((size_t)w.lt * I->m.n_jac * warps + 255) & ~size_t(255);
  const int hist_stride = hist_stride_of(I->off, s);
  if (256 + jb + sizeof(double) * (size_t)hist_stride * warps > scratch_bytes) {
    *err = "slot scratch too small for this launch";
    return false;
  }
  int* counter = (int*)scratch;
  CK(cudaMemsetAsync(counter, 0, 2 * sizeof(int), st));
  SolveArgs a;
  fill_args(&a, w, s, d_state, d_env, d_photo, nullptr, n_cells, 0.0, 0.0);
  a.tspan = d_tspan;
  a.err = counter + 1;
  a.counter = counter;
  a.stats = d_stats;
  a.jscratch = scratch + 256;
  a.hist = hist_stride ? (double*)(scratch + 256 + jb) : nullptr;
  a.hist_stride = hist_stride;
  if (!launch_warp_kernel(a, w, s.precision, st, err)) return false;
  ++launches_;
  return true;
}

int Engine::sm_count() const { return impl_->sm_count; }

int Engine::max_cells_per_block(const SolveSettings& s) const {
  const Impl* I = impl_;
  if (s.kernel != 0 || !I->warp_ok) return 0;
  const int lt = s.precision == 1 ? 4 : 8;
  const Layout lay = make_layout(I->off, lt, s.hist_global == 0, true);
  return std::min(max_cells_of(I->off),
                  std::max(0, (I->max_smem - tab_bytes_of(I->off, s.lu_mode)) / lay.bytes));
}

bool Engine::read_last_ms(void* stream) {
  (void)stream;
  Impl* I = impl_;
  if (!I->ev_pending) return true;
  if (cudaEventSynchronize(I->ev1) != cudaSuccess) return false;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, I->ev0, I->ev1);
  last_ms_ = ms;
  I->ev_pending = false;
  return true;
}

bool Engine::fetch_stats(std::vector<CellStats>* out, int n_cells, void* stream,
                         std::string* err) {
  Impl* I = impl_;
  out->resize(n_cells);
  if (n_cells <= 0) return true;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(out->data(), I->d_stats, sizeof(CellStats) * n_cells,
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  read_last_ms(stream);
  return true;
}

bool Engine::sync(void* stream, std::string* err) {
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  read_last_ms(stream);
  return true;
}

double* Engine::d_state_buf(int n_cells, std::string* err) {
  if (!ensure(&impl_->d_state, &impl_->c_state, sizeof(double) * (size_t)n_cells * impl_->n_state,
              err))
    return nullptr;
  return (double*)impl_->d_state;
}
double* Engine::d_env_buf(int n_cells, std::string* err) {
  if (!ensure(&impl_->d_env, &impl_->c_env, sizeof(double) * 2 * (size_t)n_cells, err))
    return nullptr;
  return (double*)impl_->d_env;
}
double* Engine::d_photo_buf(int n_cells, std::string* err) {
  if (!ensure(&impl_->d_photo, &impl_->c_photo,
              sizeof(double) * (size_t)n_cells * std::max(1, impl_->n_photo), err))
    return nullptr;
  return (double*)impl_->d_photo;
}
int* Engine::d_order_buf(int n_cells, std::string* err) {
  if (!ensure(&impl_->d_order, &impl_->c_order, sizeof(int) * (size_t)n_cells, err))
    return nullptr;
  return (int*)impl_->d_order;
}

// temporary device buffer of the evaluation hooks, freed on every return
struct DevBuf {
  double* p = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc((void**)&p, sizeof(double) * std::max<size_t>(1, n)); }
};

bool Engine::eval_deriv(const double* h_state, const double* h_env, const double* h_photo,
                        int n_cells, double h, double* r_p, double* r_l, double* f,
                        std::string* err) {
  Impl* I = impl_;
  if (!warp_tables(err)) return false;
  const DevMech& m = I->m;
  size_t ns = (size_t)n_cells * m.n_state, nn = (size_t)n_cells * m.n;
  DevBuf bs, be, bp, bo;
  CK(bs.alloc(ns));
  CK(be.alloc(2 * (size_t)n_cells));
  CK(bp.alloc((size_t)n_cells * m.n_photo));
  CK(bo.alloc(3 * nn));
  double *ds = bs.p, *de = be.p, *dp = bp.p, *dout = bo.p;
  CK(cudaMemcpy(ds, h_state, sizeof(double) * ns, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(de, h_env, sizeof(double) * 2 * n_cells, cudaMemcpyHostToDevice));
  if (m.n_photo > 0 && h_photo)
    CK(cudaMemcpy(dp, h_photo, sizeof(double) * n_cells * m.n_photo, cudaMemcpyHostToDevice));
  EvalArgs a{};
  a.m = m;
  a.off = I->off;
  a.blob = I->d_blob;
  a.tab_bytes = tab_bytes_of(I->off, 1);
  a.stage_bytes = I->off.bytes;
  a.err = I->d_counter + 1;
  a.lay = make_layout(I->off, 8, true, true);
  a.state = ds;
  a.env = de;
  a.photo = (m.n_photo > 0 && h_photo) ? dp : nullptr;
  a.n_cells = n_cells;
  a.h = h;
  a.rp = dout;
  a.rl = dout + nn;
  a.f = dout + 2 * nn;
  a.do_jac = 0;
  int warps = std::max(1, std::min(8, (I->max_smem - a.tab_bytes) / a.lay.bytes));
  size_t smem = (size_t)a.tab_bytes + (size_t)warps * a.lay.bytes;
  CK(cudaFuncSetAttribute(eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  eval_kernel<<<(n_cells + warps - 1) / warps, warps * 32, smem>>>(a);
  CK(cudaGetLastError());
  ++launches_;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(r_p, a.rp, sizeof(double) * nn, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(r_l, a.rl, sizeof(double) * nn, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(f, a.f, sizeof(double) * nn, cudaMemcpyDeviceToHost));
  return true;
}

bool Engine::eval_jac(const double* h_state, const double* h_env, const double* h_photo,
                      int n_cells, double h, double* jp, double* jl, std::string* err) {
  Impl* I = impl_;
  if (!warp_tables(err)) return false;
  const DevMech& m = I->m;
  size_t ns = (size_t)n_cells * m.n_state, nj = (size_t)n_cells * m.n_jac;
  DevBuf bs, be, bp, bo;
  CK(bs.alloc(ns));
  CK(be.alloc(2 * (size_t)n_cells));
  CK(bp.alloc((size_t)n_cells * m.n_photo));
  CK(bo.alloc(3 * nj));
  double *ds = bs.p, *de = be.p, *dp = bp.p, *dout = bo.p;
  CK(cudaMemcpy(ds, h_state, sizeof(double) * ns, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(de, h_env, sizeof(double) * 2 * n_cells, cudaMemcpyHostToDevice));
  if (m.n_photo > 0 && h_photo)
    CK(cudaMemcpy(dp, h_photo, sizeof(double) * n_cells * m.n_photo, cudaMemcpyHostToDevice));
  EvalArgs a{};
  a.m = m;
  a.off = I->off;
  a.blob = I->d_blob;
  a.tab_bytes = tab_bytes_of(I->off, 1);
  a.stage_bytes = I->off.bytes;
  a.err = I->d_counter + 1;
  a.lay = make_layout(I->off, 8, true, true);
  a.state = ds;
  a.env = de;
  a.photo = (m.n_photo > 0 && h_photo) ? dp : nullptr;
  a.n_cells = n_cells;
  a.h = h;
  a.jp = dout;
  a.jl = dout + nj;
  a.jv = dout + 2 * nj;
  a.do_jac = 1;
  int warps = std::max(1, std::min(8, (I->max_smem - a.tab_bytes) / a.lay.bytes));
  size_t smem = (size_t)a.tab_bytes + (size_t)warps * a.lay.bytes;
  CK(cudaFuncSetAttribute(eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  eval_kernel<<<(n_cells + warps - 1) / warps, warps * 32, smem>>>(a);
  CK(cudaGetLastError());
  ++launches_;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(jp, a.jp, sizeof(double) * nj, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(jl, a.jl, sizeof(double) * nj, cudaMemcpyDeviceToHost));
  return true;
}

bool Engine::check_precision(const double* h_state, const double* h_env,
                             const double* h_photo, int n_cells, double h, double rtol,
                             double* rel_err, std::string* err) {
  Impl* I = impl_;
  if (!warp_tables(err)) return false;
  const DevMech& m = I->m;
  const int n = m.n;
  const size_t ns = (size_t)n_cells * m.n_state, nx = (size_t)n_cells * n;
  DevBuf bs, be, bp, bj, bx;
  CK(bs.alloc(ns));
  CK(be.alloc(2 * (size_t)n_cells));
  CK(bp.alloc((size_t)n_cells * m.n_photo));
  CK(bj.alloc((size_t)n_cells * m.n_jac));
  CK(bx.alloc(2 * nx + (size_t)n_cells));
  CK(cudaMemcpy(bs.p, h_state, sizeof(double) * ns, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(be.p, h_env, sizeof(double) * 2 * n_cells, cudaMemcpyHostToDevice));
  if (m.n_photo > 0 && h_photo)
    CK(cudaMemcpy(bp.p, h_photo, sizeof(double) * n_cells * m.n_photo, cudaMemcpyHostToDevice));
  std::vector<double> x(2 * nx);
  std::vector<int> bad(2 * (size_t)n_cells);
  for (int pass = 0; pass < 2; ++pass) {
    PrecArgs p{};
    EvalArgs& a = p.e;
    a.m = m;
    a.off = I->off;
    a.blob = I->d_blob;
    a.tab_bytes = tab_bytes_of(I->off, 1);
    a.stage_bytes = I->off.bytes;
    a.err = I->d_counter + 1;
    a.lay = make_layout(I->off, pass == 0 ? 8 : 4, true, true);
    a.state = bs.p;
    a.env = be.p;
    a.photo = (m.n_photo > 0 && h_photo) ? bp.p : nullptr;
    a.n_cells = n_cells;
    a.h = h;
    p.jbuf = bj.p;
    p.rtol = rtol;
    p.x = bx.p + (size_t)pass * nx;
    p.bad = (int*)(bx.p + 2 * nx);
    const int warps = std::max(1, std::min(8, (I->max_smem - a.tab_bytes) / a.lay.bytes));
    const size_t smem = (size_t)a.tab_bytes + (size_t)warps * a.lay.bytes;
    void* func = pass == 0 ? (void*)precision_kernel<double> : (void*)precision_kernel<float>;
    CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void* args[] = {&p};
    CK(cudaLaunchKernel(func, dim3((n_cells + warps - 1) / warps), dim3(warps * 32), args, smem,
                        0));
    CK(cudaGetLastError());
    ++launches_;
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(x.data() + (size_t)pass * nx, p.x, sizeof(double) * nx,
                  cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(bad.data() + (size_t)pass * n_cells, p.bad, sizeof(int) * n_cells,
                  cudaMemcpyDeviceToHost));
  }
  // weights as the kernel's right-hand side: rtol |y| + atol per dependent
  // variable (the atol of the blob, in dependent order)
  std::vector<double> atol(n);
  CK(cudaMemcpy(atol.data(), (const char*)I->d_blob + I->off.atol, sizeof(double) * n,
                cudaMemcpyDeviceToHost));
  std::vector<int> dep_state(n);
  {
    std::vector<uint16_t> ds(n);
    CK(cudaMemcpy(ds.data(), (const char*)I->d_blob + I->off.dep_state, sizeof(uint16_t) * n,
                  cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) dep_state[i] = ds[i];
  }
  for (int c = 0; c < n_cells; ++c) {
    if (bad[c] || bad[(size_t)n_cells + c]) {
      rel_err[c] = -1.0;
      continue;
    }
    double num = 0.0, den = 0.0;
    for (int i = 0; i < n; ++i) {
      const double s = rtol * std::fabs(h_state[(size_t)c * m.n_state + dep_state[i]]) + atol[i];
      const double x64 = x[(size_t)c * n + i], x32 = x[nx + (size_t)c * n + i];
      num += ((x32 - x64) / s) * ((x32 - x64) / s);
      den += (x64 / s) * (x64 / s);
    }
    rel_err[c] = den > 0.0 ? std::sqrt(num / den) : 0.0;
  }
  return true;
}

bool Engine::check_jac(const double* h_state, const double* h_env, const double* h_photo,
                       int n_cells, double h, double rel_tol, double abs_tol, double* worst,
                       int* nfail, std::string* err) {
  Impl* I = impl_;
  if (!warp_tables(err)) return false;
  const DevMech& m = I->m;
  const size_t ns = (size_t)n_cells * m.n_state, nj = (size_t)n_cells * m.n_jac;
  double *ds = nullptr, *de = nullptr, *dp = nullptr, *dj = nullptr, *db = nullptr,
         *dw = nullptr;
  int* dn = nullptr;
  bool ok = false;
  do {
    if (cudaMalloc(&ds, sizeof(double) * ns) != cudaSuccess ||
        cudaMalloc(&de, sizeof(double) * 2 * n_cells) != cudaSuccess ||
        cudaMalloc(&dp, sizeof(double) * std::max<size_t>(1, (size_t)n_cells * m.n_photo)) !=
            cudaSuccess ||
        cudaMalloc(&dj, sizeof(double) * nj) != cudaSuccess ||
        cudaMalloc(&db, sizeof(double) * nj) != cudaSuccess ||
        cudaMalloc(&dw, sizeof(double) * n_cells) != cudaSuccess ||
        cudaMalloc(&dn, sizeof(int) * n_cells) != cudaSuccess) {
      *err = "check_jac: device allocation failed";
      break;
    }
    cudaMemcpy(ds, h_state, sizeof(double) * ns, cudaMemcpyHostToDevice);
    cudaMemcpy(de, h_env, sizeof(double) * 2 * n_cells, cudaMemcpyHostToDevice);
    if (m.n_photo > 0 && h_photo)
      cudaMemcpy(dp, h_photo, sizeof(double) * n_cells * m.n_photo, cudaMemcpyHostToDevice);
    CheckArgs c{};
    EvalArgs& a = c.e;
    a.m = m;
    a.off = I->off;
    a.blob = I->d_blob;
    a.tab_bytes = tab_bytes_of(I->off, 1);
    a.stage_bytes = I->off.bytes;
    a.err = I->d_counter + 1;
    a.lay = make_layout(I->off, 8, true, true);
    a.state = ds;
    a.env = de;
    a.photo = (m.n_photo > 0 && h_photo) ? dp : nullptr;
    a.n_cells = n_cells;
    a.h = h;
    a.jv = dj;
    c.rel_tol = rel_tol;
    c.abs_tol = abs_tol;
    c.best = db;
    c.worst = dw;
    c.nfail = dn;
    const int warps = std::max(1, std::min(8, (I->max_smem - a.tab_bytes) / a.lay.bytes));
    const size_t smem = (size_t)a.tab_bytes + (size_t)warps * a.lay.bytes;
    if (cudaFuncSetAttribute(jac_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess) {
      *err = "check_jac: shared memory attribute";
      break;
    }
    jac_check_kernel<<<(n_cells + warps - 1) / warps, warps * 32, smem>>>(c);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      *err = std::string("check_jac: ") + cudaGetErrorString(e);
      break;
    }
    ++launches_;
    cudaMemcpy(worst, dw, sizeof(double) * n_cells, cudaMemcpyDeviceToHost);
    cudaMemcpy(nfail, dn, sizeof(int) * n_cells, cudaMemcpyDeviceToHost);
    ok = true;
  } while (false);
  cudaFree(ds);
  cudaFree(de);
  cudaFree(dp);
  cudaFree(dj);
  cudaFree(db);
  cudaFree(dw);
  cudaFree(dn);
  return ok;
}

// ---------------------------------------------------------------------------
// Solve without device allocation
//
// Some callers cannot allocate device memory while they run: a host model
// that hands the whole device heap to its own pool allocator up front, or a
// code that runs this solve inside a region where cudaMalloc is not allowed.
// For them the solve's scratch (the cell counter, the error flag and each
// resident cell's saved Jacobian) lives in one fixed static device array of
// kStaticScratchBytes that every GPU loading this library holds until the
// process exits.  Calls share the array and it keeps the last call's
// contents; the counter and flag are cleared by every call, the Jacobian
// slots are always written before they are read.  Two such calls that
// overlap on the GPU (different streams, or different solvers on one device)
// race on the array.  This path records no timing events and no per-cell
// statistics in the solver (the caller's d_stats receives them), so
// last_kernel_ms and get_cell_stats keep describing the solver's last
// regular run.  The Nordsieck history stays in shared memory whatever the
// solver's layout setting.
// ---------------------------------------------------------------------------
constexpr size_t kStaticScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr size_t kStaticHeadBytes = 256;                 // counter, error flag
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of the static scratch on the current device.  The host-side
// name g_static_scratch is only a stand-in, so the address is looked up once
// per device (with that device current) and kept for the life of the
// process; a caller that resets a device's primary context (cudaDeviceReset)
// must not use this path on that device afterwards.

static bool static_scratch_address(char** out, std::string* err) {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    *err = "device index out of range for the static scratch table";
    return false;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_static_scratch));
    addr[dev] = p;
  }
  *out = (char*)addr[dev];
  return true;
}

bool Engine::run_solve_static(double* d_state, const double* d_env, const double* d_photo,
                              CellStats* d_stats, int n_cells, double t0, double t1,
                              const SolveSettings& s, void* stream, std::string* err) {
  Impl* I = impl_;
  if (!warp_tables(err)) return false;
  if (n_cells <= 0) return true;
  if (!d_state || !d_env || !d_stats || (I->m.n_photo > 0 && !d_photo)) {
    *err = "state, env, stats (and photolysis rates, when the mechanism has photolysis) "
           "must be device buffers";
    return false;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int lt = s.precision == 1 ? 4 : 8;
  Layout lay = make_layout(I->off, lt, true, true);
  const int tab = tab_bytes_of(I->off, s.lu_mode);
  int warps = (I->max_smem - tab) / lay.bytes;
  if (warps < 1) {
    *err = "mechanism too large for the shared-memory layout (" + std::to_string(lay.bytes) +
           " bytes per cell)";
    return false;
  }
  if (s.warps_per_block > 0) warps = std::min(warps, s.warps_per_block);
  warps = std::min(warps, max_cells_of(I->off));
  // one resident cell keeps n_jac Jacobian values (the kernel indexes them
  // by warp); the static array bounds the number of resident cells
  const size_t per_warp = (size_t)lt * I->m.n_jac;
  const size_t fit = (kStaticScratchBytes - kStaticHeadBytes) / per_warp;
  if (fit < (size_t)I->sm_count) {
    *err = "the mechanism needs " + std::to_string(per_warp) +
           " bytes of scratch per resident cell; the static scratch of " +
           std::to_string(kStaticScratchBytes) + " bytes holds " + std::to_string(fit) +
           ", fewer than one per SM (" + std::to_string(I->sm_count) + ")";
    return false;
  }
  warps = std::min(warps, (int)(fit / (size_t)I->sm_count));
  int grid = I->sm_count;
  if ((long)grid * warps > n_cells) grid = std::max(1, (n_cells + warps - 1) / warps);
  char* base = nullptr;
  if (!static_scratch_address(&base, err)) return false;
  int* counter = (int*)base;
  CK(cudaMemsetAsync(counter, 0, kStaticHeadBytes, st));
  SolveArgs a;
  a.m = I->m;
  a.off = I->off;
  a.blob = I->d_blob;
  a.tab_bytes = tab;
  a.stage_bytes = stage_bytes_of(I->off, s.lu_mode);
  a.err = counter + 1;
  a.lay = lay;
  a.state = d_state;
  a.env = d_env;
  a.photo = I->m.n_photo > 0 ? d_photo : nullptr;
  a.order = nullptr;
  a.n_cells = n_cells;
  a.counter = counter;
  a.stats = d_stats;
  a.jscratch = base + kStaticHeadBytes;
  a.hist = nullptr;
  a.hist_stride = 0;
  a.t0 = t0;
  a.t1 = t1;
  a.rtol = s.rtol;
  a.max_steps = s.max_steps;
  a.maxncf = s.max_conv_fails;
  a.maxnef = s.max_conv_fails;
  a.lu_mode = s.lu_mode;
  const size_t smem = (size_t)tab + (size_t)warps * lay.bytes;
  // set on every call: the regular entry points set the same kernel's limit
  // to their own launch's size
  CK(cudaFuncSetAttribute(solve_kernel_fn(I->off, s.precision),
                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  void* args[] = {&a};
  CK(cudaLaunchKernel(solve_kernel_fn(I->off, s.precision), dim3(grid), dim3(warps * 32), args,
                      smem, st));
  ++launches_;
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, counter + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (flag) {
    *err = "solve kernel: the table stage into shared memory did not complete";
    return false;
  }
  return true;
}

}  // namespace campb
