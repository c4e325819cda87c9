// Lane-per-cell solve: every lane of a warp integrates its own grid cell.
//
// All cells share one mechanism, so the sparse structure of f, J and the LU
// is the same for every lane: each warp instruction of the rate, Jacobian,
// factorization and triangular-solve loops does the work of 32 cells, with
// warp-uniform table reads (broadcast from shared memory) and per-cell data
// in a lane-interleaved layout (element e of a lane's array at [e*32 + lane])
// that makes every data access a conflict-free shared-memory access or a
// coalesced global access.
//
// Each lane runs the CVODE BDF method as a resumable state machine: its
// control code runs until it needs a heavy operation (f, Jacobian + LU
// factorization, factorization, triangular solve), records the request and
// returns.  The warp loop then executes each heavy operation once for all the
// lanes that requested it, in a fixed order, and resumes those lanes' control
// code right after, so lanes of a warp that are at different points of their
// integrations still share the expensive instructions.  A lane that finishes
// its cell takes the next one from a global counter, so cells with very
// different stiffness keep every lane busy until the tail of the run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "bdf_consts.hpp"
#include "blob.hpp"
#include "engine.hpp"
#include "rates.cuh"

namespace campb {
namespace lanes {

using namespace bdf;

#define FULL 0xffffffffu
// element e of a lane-interleaved array
#define AT(p, e) (p)[(size_t)(e) << 5]

enum Op : int { OP_NONE = 0, OP_F = 1, OP_JAC = 2, OP_FACTOR = 3, OP_SOLVE = 4, OP_EXIT = 5 };
enum FArg : int { F_ZN0_ZN1 = 0, F_Y_FTEMP = 1, F_ZN0_TEMPV = 2 };
enum Resume : int {
  R_NEW = 0, R_INIT_F, R_NLS_F, R_SETUP, R_NEWTON_SOLVE, R_NEWTON_F, R_RESTART_F, R_EXIT
};

struct Tab {
  const uint32_t *rx_word, *rx_part, *upd_ptr, *upd;
  const uint16_t *rx_pptr, *rx_jptr, *jpos, *lu_perm, *lu_rowptr, *lu_col, *lu_diag, *dep_state;
  const double *coef, *atol;
  int n, n_rxn, n_lu;
};

__device__ __forceinline__ Tab make_tab(const char* b) {
  const LaneOff& o = *reinterpret_cast<const LaneOff*>(b);
  Tab t;
  t.rx_word = (const uint32_t*)(b + o.rx_word);
  t.rx_part = (const uint32_t*)(b + o.rx_part);
  t.upd_ptr = (const uint32_t*)(b + o.upd_ptr);
  t.upd = (const uint32_t*)(b + o.upd);
  t.rx_pptr = (const uint16_t*)(b + o.rx_pptr);
  t.rx_jptr = (const uint16_t*)(b + o.rx_jptr);
  t.jpos = (const uint16_t*)(b + o.jpos);
  t.lu_perm = (const uint16_t*)(b + o.lu_perm);
  t.lu_rowptr = (const uint16_t*)(b + o.lu_rowptr);
  t.lu_col = (const uint16_t*)(b + o.lu_col);
  t.lu_diag = (const uint16_t*)(b + o.lu_diag);
  t.dep_state = (const uint16_t*)(b + o.dep_state);
  t.coef = (const double*)(b + o.coef);
  t.atol = (const double*)(b + o.atol);
  t.n = o.n;
  t.n_rxn = o.n_rxn;
  t.n_lu = o.n_lu;
  return t;
}

// where each per-cell array lives (element offsets within the warp's global
// or shared region, in units of the array's element type x 32 lanes)
struct LaneLayout {
  // FP64 arrays in global scratch
  int zn, ewt, acor, ftemp, tempv, P, L, keff, J, dinv, w64;  // w64: doubles per lane
  // arrays that may sit in shared memory (flag) or global scratch
  int y_smem, lu_smem, z_smem;
  int y_off, lu_off, z_off;  // element offsets in their region
  int w64_extra;             // extra FP64 words per lane in global (y when not in smem)
  int wlt;                   // LT words per lane in global (LU, z when not in smem)
  int smem_bytes_per_warp;   // bytes of per-warp shared memory
};

struct LaneArgs {
  DevMech m;
  const void* blob;
  int tab_bytes;   // shared-memory bytes of the staged tables (0 when global)
  int tab_global;  // 1: tables too large for shared memory, read from global
  LaneLayout lay;
  double* state;
  const double* env;
  const double* photo;
  const int* order;
  int n_cells;
  int* counter;
  int* err;
  CellStats* stats;
  double* scratch64;  // per-warp FP64 regions
  void* scratchlt;    // per-warp LT regions
  double t0, t1, rtol;
  int max_steps, maxncf, maxnef;
};

// Per-lane integration state.  Vector members point at this lane's slot of a
// lane-interleaved array (use AT to index).
template <typename LT>
struct LS {
  double* zn;  // column j at zn + j*n*32
  double *ewt, *acor, *ftemp, *tempv, *y, *P, *L, *keff, *J, *dinv;
  LT *LU, *z;
  int n;
  // request
  int op, farg, resume;
  int fret, jret, fok;
  // cell
  int cell, flag;
  double h0, t0, tout;
  // method state
  int q, qprime, qwait, Lq, jcur;
  double h, hprime, hscale, eta, etamax, hu, next_h, tn;
  double tau[LMAX + 2], tq[6], l[LMAX];
  double rl1, gamma, gammap, gamrat, crate, acnrm, saved_tq5;
  double saved_t, del, delp, dsm;
  int nst, nfe, nsetups, netf, nni, ncfn, nje, nstlp, nstlj, nstloc;
  int ncf, nef, nflag, convfail, call_setup, projected, mnewt, nls;
};

__device__ __forceinline__ double state_of(double y) { return y > -kSmall ? y : kTiny; }

// ---------------------------------------------------------------------------
// Heavy operations (executed by all lanes that requested them together)
// ---------------------------------------------------------------------------

// f(y) into out; 1 when some y < -SMALL (recoverable failure).  Reactions
// are visited in mechanism order and their contributions split by sign into
// production and loss sums (src/time_derivative.c:90-97), with the
// negative-yield guard of the reference (src/rxns/rxn_arrhenius.c:153-160).
template <typename LT>
__device__ __noinline__ int op_f(const char* tb, LS<LT>* s, const double* y, double* out,
                                 double h) {
  const Tab t = make_tab(tb);
  const int n = t.n;
  bool bad = false;
  for (int i = 0; i < n; ++i) bad |= AT(y, i) < -kSmall;
  if (bad) return 1;
  double* P = s->P;
  double* L = s->L;
  for (int i = 0; i < n; ++i) {
    AT(P, i) = 0.0;
    AT(L, i) = 0.0;
  }
  const double* keff = s->keff;
  for (int r = 0; r < t.n_rxn; ++r) {
    const uint32_t w = t.rx_word[r];
    const int nv = w >> 30;
    double rate = AT(keff, r);
    if (nv > 0) rate *= state_of(AT(y, w & 1023u));
    if (nv > 1) rate *= state_of(AT(y, (w >> 10) & 1023u));
    if (nv > 2) rate *= state_of(AT(y, (w >> 20) & 1023u));
    if (rate == 0.0) continue;
    const int p1 = t.rx_pptr[r + 1];
    for (int p = t.rx_pptr[r]; p < p1; ++p) {
      const uint32_t pe = t.rx_part[p];
      const int sp = pe & 1023u;
      const double c = t.coef[(pe >> 10) & 0x7FFFu];
      if ((pe >> 31) && !(-rate * c * h <= state_of(AT(y, sp)))) continue;
      const double v = rate * c;
      if (v > 0.0)
        AT(P, sp) += v;
      else
        AT(L, sp) -= v;
    }
  }
  for (int i = 0; i < n; ++i) {
    const double p = AT(P, i), l = AT(L, i);
    AT(out, i) = (p + l != 0.0) ? p - l : 0.0;
  }
  return 0;
}

// Jacobian of f at y accumulated in LU layout (src/rxns/rxn_arrhenius.c:178-212)
template <typename LT>
__device__ __noinline__ int op_jac(const char* tb, LS<LT>* s, const double* y, double h) {
  const Tab t = make_tab(tb);
  bool bad = false;
  for (int i = 0; i < t.n; ++i) bad |= AT(y, i) < -kSmall;
  if (bad) return 1;
  double* J = s->J;
  for (int q = 0; q < t.n_lu; ++q) AT(J, q) = 0.0;
  const double* keff = s->keff;
  for (int r = 0; r < t.n_rxn; ++r) {
    const uint32_t w = t.rx_word[r];
    const int nv = w >> 30;
    if (nv == 0) continue;
    const double k = AT(keff, r);
    int d[3] = {(int)(w & 1023u), (int)((w >> 10) & 1023u), (int)((w >> 20) & 1023u)};
    double yv[3];
    for (int v = 0; v < nv; ++v) yv[v] = state_of(AT(y, d[v]));
    const int p0 = t.rx_pptr[r], np = t.rx_pptr[r + 1] - p0;
    int jp = t.rx_jptr[r];
    for (int kv = 0; kv < nv; ++kv) {
      double part = k;
      for (int v = 0; v < nv; ++v)
        if (v != kv) part *= yv[v];
      const double yind = yv[kv];
      for (int p = 0; p < np; ++p, ++jp) {
        const uint32_t pe = t.rx_part[p0 + p];
        const int pos = t.jpos[jp];
        if (!(pe >> 31)) {  // a loss (sources have no reactants, so never reach here)
          AT(J, pos) -= part;
        } else {
          const double c = t.coef[(pe >> 10) & 0x7FFFu];
          if (-part * yind * c * h <= state_of(AT(y, pe & 1023u))) AT(J, pos) += c * part;
        }
      }
    }
  }
  return 0;
}

// M = I - gamma*J in LU layout, factored row by row on the fixed order
template <typename LT>
__device__ __noinline__ int op_factor(const char* tb, LS<LT>* s) {
  const Tab t = make_tab(tb);
  LT* LU = s->LU;
  const double* J = s->J;
  double* dinv = s->dinv;
  const double g = s->gamma;
  for (int q = 0; q < t.n_lu; ++q) AT(LU, q) = (LT)(-g * AT(J, q));
  for (int i = 0; i < t.n; ++i) AT(LU, t.lu_diag[i]) += (LT)1;
  bool bad = false;
  for (int i = 0; i < t.n; ++i) {
    const int d = t.lu_diag[i];
    for (int q = t.lu_rowptr[i]; q < d; ++q) {
      const LT l = AT(LU, q) * (LT)AT(dinv, t.lu_col[q]);
      AT(LU, q) = l;
      // the update list of L entry (i, k) targets distinct entries of row i
      // and reads row k, so a group's loads can all be issued before its
      // stores: eight updates wait for one memory latency instead of eight
      const uint32_t p1 = t.upd_ptr[q + 1];
      uint32_t p = t.upd_ptr[q];
      for (; p + 8 <= p1; p += 8) {
        uint32_t u[8];
        LT a[8], b[8];
        #pragma unroll
        for (int j = 0; j < 8; ++j) u[j] = t.upd[p + j];
        #pragma unroll
        for (int j = 0; j < 8; ++j) {
          a[j] = AT(LU, u[j] >> 16);
          b[j] = AT(LU, u[j] & 0xFFFFu);
        }
        #pragma unroll
        for (int j = 0; j < 8; ++j) AT(LU, u[j] >> 16) = a[j] - l * b[j];
      }
      for (; p < p1; ++p) {
        const uint32_t u = t.upd[p];
        AT(LU, u >> 16) -= l * AT(LU, u & 0xFFFFu);
      }
    }
    const LT piv = AT(LU, d);
    const bool pb = (piv == (LT)0) || !isfinite((double)piv);
    bad |= pb;
    AT(dinv, i) = pb ? 0.0 : 1.0 / (double)piv;
  }
  return bad ? 0 : 1;
}

// tempv <- M^{-1} tempv
template <typename LT>
__device__ __noinline__ void op_solve(const char* tb, LS<LT>* s) {
  const Tab t = make_tab(tb);
  const LT* LU = s->LU;
  LT* z = s->z;
  double* b = s->tempv;
  const double* dinv = s->dinv;
  for (int k = 0; k < t.n; ++k) AT(z, k) = (LT)AT(b, t.lu_perm[k]);
  for (int i = 0; i < t.n; ++i) {
    LT acc = AT(z, i);
    const int d = t.lu_diag[i];
    for (int q = t.lu_rowptr[i]; q < d; ++q) acc -= AT(LU, q) * AT(z, t.lu_col[q]);
    AT(z, i) = acc;
  }
  for (int i = t.n - 1; i >= 0; --i) {
    LT acc = AT(z, i);
    const int d = t.lu_diag[i], q1 = t.lu_rowptr[i + 1];
    for (int q = d + 1; q < q1; ++q) acc -= AT(LU, q) * AT(z, t.lu_col[q]);
    AT(z, i) = acc * (LT)AT(dinv, i);
  }
  for (int k = 0; k < t.n; ++k) AT(b, t.lu_perm[k]) = (double)AT(z, k);
}

// ---------------------------------------------------------------------------
// Control (CVODE BDF, restated per lane)
// ---------------------------------------------------------------------------
template <typename LT>
struct Ctl {
  LS<LT>* s;
  const char* tb;
  int n;
  __device__ double* Z(int j) const { return s->zn + ((size_t)j * n << 5); }
  __device__ double wrms(const double* v) const {
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
      const double t = AT(v, i) * AT(s->ewt, i);
      acc += t * t;
    }
    return sqrt(acc / n);
  }
  __device__ bool set_ewt(const double* yy, const double* atol, double rtol) const {
    bool ok = true;
    for (int i = 0; i < n; ++i) {
      const double w = rtol * fabs(AT(yy, i)) + atol[i];
      ok &= w > 0.0;
      AT(s->ewt, i) = 1.0 / w;
    }
    return ok;
  }
  __device__ void rescale() const {
    double factor = s->eta;
    for (int j = 1; j <= s->q; ++j) {
      double* zj = Z(j);
      for (int i = 0; i < n; ++i) AT(zj, i) *= factor;
      factor *= s->eta;
    }
    s->h = s->hscale * s->eta;
    s->next_h = s->h;
    s->hscale = s->h;
  }
  __device__ void predict() const {
    s->tn += s->h;
    const int q = s->q;
    for (int k = 1; k <= q; ++k)
      for (int j = q; j >= k; --j) {
        double *a = Z(j - 1), *b = Z(j);
        for (int i = 0; i < n; ++i) AT(a, i) += AT(b, i);
      }
  }
  __device__ void restore(double saved_t) const {
    s->tn = saved_t;
    const int q = s->q;
    for (int k = 1; k <= q; ++k)
      for (int j = q; j >= k; --j) {
        double *a = Z(j - 1), *b = Z(j);
        for (int i = 0; i < n; ++i) AT(a, i) -= AT(b, i);
      }
  }
  __device__ void set() const {
    const int q = s->q;
    double* l = s->l;
    double* tau = s->tau;
    double* tq = s->tq;
    double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
    l[0] = l[1] = xi_inv = xistar_inv = 1.0;
    for (int i = 2; i <= q; ++i) l[i] = 0.0;
    alpha0 = alpha0_hat = -1.0;
    hsum = s->h;
    if (q > 1) {
      for (int j = 2; j < q; ++j) {
        hsum += tau[j - 1];
        xi_inv = s->h / hsum;
        alpha0 -= 1.0 / j;
        for (int i = j; i >= 1; --i) l[i] += l[i - 1] * xi_inv;
      }
      alpha0 -= 1.0 / q;
      xistar_inv = -l[1] - alpha0;
      hsum += tau[q - 1];
      xi_inv = s->h / hsum;
      alpha0_hat = -l[1] - xi_inv;
      for (int i = q; i >= 1; --i) l[i] += l[i - 1] * xistar_inv;
    }
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    tq[2] = fabs(A1 / (alpha0 * A2));
    tq[5] = fabs(A2 * xistar_inv / (l[q] * xi_inv));
    if (s->qwait == 1) {
      if (q > 1) {
        const double C = xistar_inv / l[q];
        const double A3 = alpha0 + 1.0 / q;
        const double A4 = alpha0_hat + xi_inv;
        const double Cpinv = (1.0 - A4 + A3) / A3;
        tq[1] = fabs(C * Cpinv);
      } else {
        tq[1] = 1.0;
      }
      hsum += tau[q];
      xi_inv = s->h / hsum;
      const double A5 = alpha0 - 1.0 / (q + 1);
      const double A6 = alpha0_hat - xi_inv;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
    }
    tq[4] = NLSCOEF / tq[2];
    s->rl1 = 1.0 / l[1];
    s->gamma = s->h * s->rl1;
    if (s->nst == 0) s->gammap = s->gamma;
    s->gamrat = (s->nst > 0) ? s->gamma / s->gammap : 1.0;
  }
  __device__ void increase_order() const {
    double* l = s->l;
    const int q = s->q;
    for (int i = 0; i <= QMAX; ++i) l[i] = 0.0;
    l[2] = 1.0;
    double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = s->hscale;
    if (q > 1) {
      for (int j = 1; j < q; ++j) {
        hsum += s->tau[j + 1];
        const double xi = hsum / s->hscale;
        prod *= xi;
        alpha0 -= 1.0 / (j + 1);
        alpha1 += 1.0 / xi;
        for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xiold + l[i - 1];
        xiold = xi;
      }
    }
    const double A1 = (-alpha0 - alpha1) / prod;
    double *top = Z(q + 1), *acc = Z(QMAX);
    for (int i = 0; i < n; ++i) AT(top, i) = A1 * AT(acc, i);
    for (int j = 2; j <= q; ++j) {
      double* zj = Z(j);
      for (int i = 0; i < n; ++i) AT(zj, i) += l[j] * AT(top, i);
    }
  }
  __device__ void decrease_order() const {
    double* l = s->l;
    const int q = s->q;
    for (int i = 0; i <= QMAX; ++i) l[i] = 0.0;
    l[2] = 1.0;
    double hsum = 0.0;
    for (int j = 1; j <= q - 2; ++j) {
      hsum += s->tau[j];
      const double xi = hsum / s->hscale;
      for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xi + l[i - 1];
    }
    double* zq = Z(q);
    for (int j = 2; j < q; ++j) {
      double* zj = Z(j);
      for (int i = 0; i < n; ++i) AT(zj, i) -= l[j] * AT(zq, i);
    }
  }
  __device__ void adjust_params() const {
    if (s->qprime != s->q) {
      if (s->qprime - s->q == 1)
        increase_order();
      else if (s->qprime - s->q == -1)
        decrease_order();
      s->q = s->qprime;
      s->Lq = s->q + 1;
      s->qwait = s->Lq;
    }
    rescale();
  }
  __device__ bool start_guess() const {
    bool proj = false;
    double* z0 = Z(0);
    for (int i = 0; i < n; ++i) {
      const double v = AT(z0, i);
      const double a = v < 0.0 ? -v : 0.0;
      proj |= a != 0.0;
      AT(s->acor, i) = a;
      AT(s->y, i) = v + a;
    }
    return proj;
  }
  __device__ int check_constraints() const {
    bool viol = false;
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
      const double v = AT(s->y, i);
      if (v < 0.0) {
        viol = true;
        const double t = v * AT(s->ewt, i);
        acc += t * t;
      }
    }
    if (!viol) return NL_OK;
    if (sqrt(acc / n) <= s->tq[4]) {
      for (int i = 0; i < n; ++i)
        if (AT(s->y, i) < 0.0) {
          AT(s->acor, i) -= AT(s->y, i);
          AT(s->y, i) = 0.0;
        }
      s->acnrm = wrms(s->acor);
      return NL_OK;
    }
    double e = 1.0e300;
    double* z0 = Z(0);
    for (int i = 0; i < n; ++i) {
      const double v = AT(s->y, i);
      if (v < 0.0) {
        const double z = AT(z0, i);
        e = fmin(e, z / (z - v));
      }
    }
    e *= 0.9;
    s->eta = e > 0.1 ? e : 0.1;
    return NL_CONSTR_RECVR;
  }
  __device__ void complete_step() const {
    s->nst++;
    s->hu = s->h;
    const int q = s->q;
    for (int i = q; i >= 2; --i) s->tau[i] = s->tau[i - 1];
    if ((q == 1) && (s->nst > 1)) s->tau[2] = s->tau[1];
    s->tau[1] = s->h;
    for (int j = 0; j <= q; ++j) {
      double* zj = Z(j);
      const double lj = s->l[j];
      for (int i = 0; i < n; ++i) AT(zj, i) += lj * AT(s->acor, i);
    }
    s->qwait--;
    if ((s->qwait == 1) && (q != QMAX)) {
      double* zq = Z(QMAX);
      for (int i = 0; i < n; ++i) AT(zq, i) = AT(s->acor, i);
      s->saved_tq5 = s->tq[5];
    }
  }
  __device__ void set_eta() const {
    if (s->eta < THRESH) {
      s->eta = 1.0;
      s->hprime = s->h;
    } else {
      s->eta = fmin(s->eta, s->etamax);
      s->hprime = s->h * s->eta;
    }
  }
  __device__ void prepare_next_step(double dsm) const {
    if (s->etamax == 1.0) {
      s->qwait = s->qwait > 2 ? s->qwait : 2;
      s->qprime = s->q;
      s->hprime = s->h;
      s->eta = 1.0;
      return;
    }
    const double etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / s->Lq) + ADDON);
    if (s->qwait != 0) {
      s->eta = etaq;
      s->qprime = s->q;
      set_eta();
      return;
    }
    s->qwait = 2;
    double etaqm1 = 0.0;
    if (s->q > 1) {
      const double ddn = wrms(Z(s->q)) * s->tq[1];
      etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / s->q) + ADDON);
    }
    double etaqp1 = 0.0;
    if (s->q != QMAX && s->saved_tq5 != 0.0) {
      const double cquot = (s->tq[5] / s->saved_tq5) * pow(s->h / s->tau[2], (double)s->Lq);
      double* zq = Z(QMAX);
      for (int i = 0; i < n; ++i) AT(s->tempv, i) = AT(s->acor, i) - cquot * AT(zq, i);
      const double dup = wrms(s->tempv) * s->tq[3];
      etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (s->Lq + 1)) + ADDON);
    }
    const double etam = fmax(etaqm1, fmax(etaq, etaqp1));
    if (etam < THRESH) {
      s->eta = 1.0;
      s->qprime = s->q;
    } else if (etam == etaq) {
      s->eta = etaq;
      s->qprime = s->q;
    } else if (etam == etaqm1) {
      s->eta = etaqm1;
      s->qprime = s->q - 1;
    } else {
      s->eta = etaqp1;
      s->qprime = s->q + 1;
      double* zq = Z(QMAX);
      for (int i = 0; i < n; ++i) AT(zq, i) = AT(s->acor, i);
    }
    set_eta();
  }
};

template <typename LT>
__device__ void lane_new_cell(const LaneArgs& a, const char* tb, LS<LT>* s, int lane);

// Runs this lane's control code from its resume point until the next heavy
// operation request (or the end of all work).
template <typename LT>
__device__ __noinline__ void advance(const LaneArgs& a, const char* tb, LS<LT>* s, int lane) {
  const Tab t = make_tab(tb);
  Ctl<LT> c{s, tb, t.n};
  const int n = t.n;
  int ier = 0;
  switch (s->resume) {
    case R_NEW: goto L_NEW;
    case R_INIT_F: goto L_INIT_F;
    case R_NLS_F: goto L_NLS_F;
    case R_SETUP: goto L_SETUP;
    case R_NEWTON_SOLVE: goto L_NEWTON_SOLVE;
    case R_NEWTON_F: goto L_NEWTON_F;
    case R_RESTART_F: goto L_RESTART_F;
    default: s->op = OP_EXIT; return;
  }

L_NEW:
  lane_new_cell<LT>(a, tb, s, lane);
  if (s->cell < 0) {
    s->resume = R_EXIT;
    s->op = OP_EXIT;
    return;
  }
  if (!c.set_ewt(c.Z(0), t.atol, a.rtol)) {
    s->flag = ILL_INPUT;
    goto L_DONE;
  }
  s->next_h = 0.0;
  s->op = OP_F;
  s->farg = F_ZN0_ZN1;
  s->resume = R_INIT_F;
  return;

L_INIT_F:
  if (s->fret) {
    s->flag = REPTD_RHSFUNC_ERR;
    goto L_DONE;
  }
  s->nfe++;
  s->h = s->h0;
  if (s->h0 == 0.0) {  // CVODE's cvHin refuses tout == t0
    s->flag = TOO_CLOSE;
    goto L_DONE;
  }
  if ((s->tout - s->t0) * s->h < 0.0) {
    s->flag = ILL_INPUT;
    goto L_DONE;
  }
  s->hscale = s->h;
  s->hprime = s->h;
  {
    double* z1 = c.Z(1);
    for (int i = 0; i < n; ++i) AT(z1, i) *= s->h;
  }
  s->nstloc = 0;

L_LOOP_TOP:
  s->next_h = s->h;
  if (s->nst > 0 && !c.set_ewt(c.Z(0), t.atol, a.rtol)) {
    s->flag = ILL_INPUT;
    goto L_DONE;
  }
  if (a.max_steps > 0 && s->nstloc >= a.max_steps) {
    s->flag = TOO_MUCH_WORK;
    goto L_DONE;
  }
  if (UROUND * c.wrms(c.Z(0)) > 1.0) {
    s->flag = TOO_MUCH_ACC;
    goto L_DONE;
  }
  s->saved_t = s->tn;
  s->ncf = s->nef = 0;
  s->nflag = FIRST_CALL;
  s->dsm = 0.0;
  if ((s->nst > 0) && (s->hprime != s->h)) c.adjust_params();

L_ATTEMPT:
  c.predict();
  c.set();
  s->convfail =
      ((s->nflag == FIRST_CALL) || (s->nflag == PREV_ERR_FAIL)) ? NO_FAILURES : FAIL_OTHER;
  s->call_setup = (s->nflag == PREV_CONV_FAIL) || (s->nflag == PREV_ERR_FAIL) ||
                  (s->nst == 0) || (s->nst >= s->nstlp + MSBP) ||
                  (fabs(s->gamrat - 1.0) > DGMAX);
  s->projected = c.start_guess();

L_NLS_LOOP:
  s->op = OP_F;
  s->farg = F_Y_FTEMP;
  s->resume = R_NLS_F;
  return;

L_NLS_F:
  s->nfe++;
  if (s->fret) {
    s->nls = NL_RHS_RECVR;
    goto L_AFTER_NLS;
  }
  if (s->call_setup) {
    const double dgamma = fabs(s->gamma / s->gammap - 1.0);
    const bool jbad = (s->nst == 0) || (s->nst > s->nstlj + MSBJ) ||
                      ((s->convfail == FAIL_BAD_J) && (dgamma < DGMAX_J)) ||
                      (s->convfail == FAIL_OTHER);
    if (jbad) {
      s->nje++;
      s->nstlj = s->nst;
      s->jcur = 1;
      s->op = OP_JAC;
    } else {
      s->jcur = 0;
      s->op = OP_FACTOR;
    }
    s->resume = R_SETUP;
    return;
  }
  goto L_NEWTON_START;

L_SETUP:
  // the Jacobian request runs the factorization right after it
  ier = (s->jret || !s->fok) ? 1 : 0;
  s->nsetups++;
  s->call_setup = 0;
  s->gamrat = s->crate = 1.0;
  s->gammap = s->gamma;
  s->nstlp = s->nst;
  if (ier > 0) {
    s->nls = NL_CONV_FAIL;
    goto L_AFTER_NLS;
  }

L_NEWTON_START:
  s->mnewt = 0;
  s->delp = 0.0;

L_NEWTON_ITER:
  {
    double* z1 = c.Z(1);
    for (int i = 0; i < n; ++i)
      AT(s->tempv, i) = s->gamma * AT(s->ftemp, i) - (s->rl1 * AT(z1, i) + AT(s->acor, i));
  }
  s->op = OP_SOLVE;
  s->resume = R_NEWTON_SOLVE;
  return;

L_NEWTON_SOLVE:
  {
    if (s->gamrat != 1.0) {
      const double sc = 2.0 / (1.0 + s->gamrat);
      for (int i = 0; i < n; ++i) AT(s->tempv, i) *= sc;
    }
    s->nni++;
    s->del = c.wrms(s->tempv);
    double* z0 = c.Z(0);
    for (int i = 0; i < n; ++i) {
      const double acv = AT(s->acor, i) + AT(s->tempv, i);
      AT(s->acor, i) = acv;
      AT(s->y, i) = AT(z0, i) + acv;
    }
    if (s->mnewt > 0) s->crate = fmax(CRDOWN * s->crate, s->del / s->delp);
    const double dcon = s->del * fmin(1.0, s->crate) / s->tq[4];
    if (dcon <= 1.0) {
      s->acnrm = (s->mnewt == 0 && !s->projected) ? s->del : c.wrms(s->acor);
      s->jcur = 0;
      s->nls = c.check_constraints();
      goto L_AFTER_NLS;
    }
    s->mnewt++;
    if ((s->mnewt == MAXCOR) || ((s->mnewt >= 2) && (s->del > RDIV * s->delp))) {
      ier = s->jcur ? NL_CONV_FAIL : NL_TRY_AGAIN;
      goto L_NLS_RETRY;
    }
    s->delp = s->del;
    s->op = OP_F;
    s->farg = F_Y_FTEMP;
    s->resume = R_NEWTON_F;
    return;
  }

L_NEWTON_F:
  s->nfe++;
  if (s->fret) {
    ier = s->jcur ? NL_RHS_RECVR : NL_TRY_AGAIN;
    goto L_NLS_RETRY;
  }
  goto L_NEWTON_ITER;

L_NLS_RETRY:
  if (ier == NL_TRY_AGAIN) {
    s->call_setup = 1;
    s->convfail = FAIL_BAD_J;
    s->projected = c.start_guess();
    goto L_NLS_LOOP;
  }
  s->nls = ier;

L_AFTER_NLS:
  if (s->nls != NL_OK) {
    s->ncfn++;
    c.restore(s->saved_t);
    s->ncf++;
    s->etamax = 1.0;
    if (s->ncf == a.maxncf) {
      s->flag = (s->nls == NL_RHS_RECVR) ? REPTD_RHSFUNC_ERR : CONV_FAILURE;
      goto L_DONE;
    }
    if (s->nls != NL_CONSTR_RECVR) s->eta = ETACF;
    s->nflag = PREV_CONV_FAIL;
    c.rescale();
    goto L_ATTEMPT;
  }
  s->dsm = s->acnrm * s->tq[2];
  if (s->dsm > 1.0) {
    s->nef++;
    s->netf++;
    s->nflag = PREV_ERR_FAIL;
    c.restore(s->saved_t);
    if (s->nef == a.maxnef) {
      s->flag = ERR_FAILURE;
      goto L_DONE;
    }
    s->etamax = 1.0;
    if (s->nef <= MXNEF1) {
      s->eta = 1.0 / (pow(BIAS2 * s->dsm, 1.0 / s->Lq) + ADDON);
      s->eta = fmax(ETAMIN, s->eta);
      if (s->nef >= SMALL_NEF) s->eta = fmin(s->eta, ETAMXF);
      c.rescale();
      goto L_ATTEMPT;
    }
    if (s->q > 1) {
      s->eta = ETAMIN;
      c.decrease_order();
      s->Lq = s->q;
      s->q--;
      s->qwait = s->Lq;
      c.rescale();
      goto L_ATTEMPT;
    }
    s->eta = ETAMIN;
    s->h *= s->eta;
    s->next_h = s->h;
    s->hscale = s->h;
    s->qwait = LONG_WAIT;
    s->op = OP_F;
    s->farg = F_ZN0_TEMPV;
    s->resume = R_RESTART_F;
    return;
  }
  c.complete_step();
  c.prepare_next_step(s->dsm);
  s->etamax = (s->nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
  for (int i = 0; i < n; ++i) AT(s->acor, i) *= s->tq[2];
  s->nstloc++;
  if ((s->tn - s->tout) * s->h >= 0.0) {
    const double sc = (s->tout - s->tn) / s->h;
    for (int i = 0; i < n; ++i) {
      double v = AT(c.Z(s->q), i);
      for (int j = s->q - 1; j >= 0; --j) v = AT(c.Z(j), i) + sc * v;
      AT(s->y, i) = v;
    }
    s->next_h = s->hprime;
    s->flag = OK;
    goto L_DONE;
  }
  goto L_LOOP_TOP;

L_RESTART_F:
  s->nfe++;
  if (s->fret) {
    s->flag = UNREC_RHSFUNC_ERR;
    goto L_DONE;
  }
  {
    double* z1 = c.Z(1);
    for (int i = 0; i < n; ++i) AT(z1, i) = s->h * AT(s->tempv, i);
  }
  goto L_ATTEMPT;

L_DONE:
  {
    double* st = a.state + (size_t)s->cell * a.m.n_state;
    if (s->flag == OK)
      for (int i = 0; i < n; ++i) {
        const double v = AT(s->y, i);
        st[t.dep_state[i]] = v > 0.0 ? v : 0.0;
      }
    CellStats cs;
    cs.status = s->flag;
    cs.nst = s->nst;
    cs.nfe = s->nfe;
    cs.nsetups = s->nsetups;
    cs.netf = s->netf;
    cs.nni = s->nni;
    cs.ncfn = s->ncfn;
    cs.nje = s->nje;
    cs.hu = s->hu;
    cs.hcur = s->next_h;
    a.stats[s->cell] = cs;
  }
  goto L_NEW;
}

// Takes the next cell (or marks the lane idle), loads its state and rate
// constants and resets the method (CVodeReInit with h0 = t1 - t0).
template <typename LT>
__device__ void lane_new_cell(const LaneArgs& a, const char* tb, LS<LT>* s, int lane) {
  const Tab t = make_tab(tb);
  const DevMech& m = a.m;
  const int idx = atomicAdd(a.counter, 1);
  if (idx >= a.n_cells) {
    s->cell = -1;
    return;
  }
  const int cell = a.order ? a.order[idx] : idx;
  s->cell = cell;
  double* st = a.state + (size_t)cell * m.n_state;
  // solver_run clamps (src/camp_solver.c:554-567)
  for (int j = 0; j < m.n_const; ++j) {
    const int k = ldg(m.const_state + j);
    const double v = st[k];
    st[k] = v > kTiny ? v : kTiny;
  }
  double* z0 = s->zn;
  for (int i = 0; i < t.n; ++i) {
    const double v = st[t.dep_state[i]];
    AT(z0, i) = v > kTiny ? v : kTiny;
    AT(s->y, i) = AT(z0, i);
  }
  for (int j = 1; j < LMAX; ++j) {
    double* zj = s->zn + ((size_t)j * t.n << 5);
    for (int i = 0; i < t.n; ++i) AT(zj, i) = 0.0;
  }
  const double T = a.env[2 * (size_t)cell], P = a.env[2 * (size_t)cell + 1];
  const double* photo = a.photo ? a.photo + (size_t)cell * m.n_photo : nullptr;
  for (int r = 0; r < m.n_rxn; ++r) {
    double k = rate_constant(m, r, T, P, photo);
    for (int cc = ldg(m.rx_cptr + r); cc < ldg(m.rx_cptr + r + 1); ++cc) {
      const double v = st[ldg(m.rx_cidx + cc)];
      k *= v > kTiny ? v : kTiny;
    }
    AT(s->keff, r) = k;
  }
  for (int i = 0; i < LMAX + 2; ++i) s->tau[i] = 0.0;
  for (int i = 0; i < 6; ++i) s->tq[i] = 0.0;
  for (int i = 0; i < LMAX; ++i) s->l[i] = 0.0;
  s->t0 = a.t0;
  s->tout = a.t1;
  s->h0 = a.t1 - a.t0;
  s->q = 1;
  s->Lq = 2;
  s->qwait = 2;
  s->etamax = ETAMX1;
  s->qprime = 1;
  s->nst = s->nfe = s->nsetups = s->netf = s->nni = s->ncfn = s->nje = 0;
  s->nstlp = s->nstlj = 0;
  s->saved_tq5 = 0.0;
  s->crate = 1.0;
  s->jcur = 0;
  s->hu = 0.0;
  s->tn = a.t0;
  s->gammap = s->gamma = 0.0;
  s->h = 0.0;
  s->eta = 1.0;
  s->flag = OK;
  (void)lane;
}

template <typename LT>
__global__ void __launch_bounds__(512, 1) lane_kernel(LaneArgs a) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long tma_bar;
  // stage the tables (bulk copy, bounded wait); tables larger than shared
  // memory stay in global memory, where every read is warp-uniform (one
  // broadcast line through L1, the lines shared by all warps in L2)
  if (!a.tab_global) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(&tma_bar);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int bytes = reinterpret_cast<const LaneOff*>(a.blob)->bytes;
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes)
                   : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              (unsigned)__cvta_generic_to_shared(smem)),
          "l"(a.blob), "r"(bytes), "r"(b)
          : "memory");
    }
    unsigned done = 0;
    for (long it = 0; it < (1L << 24) && !done; ++it)
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(b)
          : "memory");
    if (!done) {
      atomicExch(a.err, 1);
      for (long it = 0; it < (1L << 24) && !done; ++it)
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(b)
            : "memory");
    }
    if (!__syncthreads_and(done ? 1 : 0)) return;
  }
  const char* tb = a.tab_global ? (const char*)a.blob : smem;
  const Tab t = make_tab(tb);
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * (blockDim.x >> 5) + wib;
  const LaneLayout& L = a.lay;
  char* wsm = smem + a.tab_bytes + (size_t)wib * L.smem_bytes_per_warp;
  double* g64 = a.scratch64 + (size_t)gwarp * (L.w64 + L.w64_extra) * 32 + lane;
  LT* glt = (LT*)a.scratchlt + (size_t)gwarp * L.wlt * 32 + lane;
  LS<LT> s;
  s.n = t.n;
  s.zn = g64 + (size_t)L.zn * 32;
  s.ewt = g64 + (size_t)L.ewt * 32;
  s.acor = g64 + (size_t)L.acor * 32;
  s.ftemp = g64 + (size_t)L.ftemp * 32;
  s.tempv = g64 + (size_t)L.tempv * 32;
  s.P = g64 + (size_t)L.P * 32;
  s.L = g64 + (size_t)L.L * 32;
  s.keff = g64 + (size_t)L.keff * 32;
  s.J = g64 + (size_t)L.J * 32;
  s.dinv = g64 + (size_t)L.dinv * 32;
  s.y = L.y_smem ? (double*)(wsm) + (size_t)L.y_off * 32 + lane : g64 + (size_t)L.y_off * 32;
  s.LU = L.lu_smem ? (LT*)(wsm) + (size_t)L.lu_off * 32 + lane : glt + (size_t)L.lu_off * 32;
  s.z = L.z_smem ? (LT*)(wsm) + (size_t)L.z_off * 32 + lane : glt + (size_t)L.z_off * 32;
  s.resume = R_NEW;
  s.op = OP_NONE;
  s.fret = s.jret = 0;
  s.fok = 1;
  advance<LT>(a, tb, &s, lane);
  for (;;) {
    if (s.op == OP_F) {
      const double* in = (s.farg == F_Y_FTEMP) ? s.y : s.zn;
      double* out = (s.farg == F_ZN0_ZN1) ? s.zn + ((size_t)t.n << 5)
                                          : (s.farg == F_Y_FTEMP ? s.ftemp : s.tempv);
      s.fret = op_f<LT>(tb, &s, in, out, s.h > 0.0 ? s.h : s.h0);
      advance<LT>(a, tb, &s, lane);
    }
    if (s.op == OP_JAC) {
      s.jret = op_jac<LT>(tb, &s, s.y, s.h > 0.0 ? s.h : s.h0);
      s.fok = s.jret ? 0 : op_factor<LT>(tb, &s);
      advance<LT>(a, tb, &s, lane);
    }
    if (s.op == OP_FACTOR) {
      s.jret = 0;
      s.fok = op_factor<LT>(tb, &s);
      advance<LT>(a, tb, &s, lane);
    }
    if (s.op == OP_SOLVE) {
      op_solve<LT>(tb, &s);
      advance<LT>(a, tb, &s, lane);
    }
    if (__all_sync(FULL, s.op == OP_EXIT)) break;
  }
}

}  // namespace lanes

// ---------------------------------------------------------------------------
// Host side: layout and launch
// ---------------------------------------------------------------------------
static bool lane_layout(const LaneOff& o, int lt_size, int max_smem_block, int tab_bytes,
                        int warps_per_block, int place, lanes::LaneLayout* out, int* warps) {
  lanes::LaneLayout L{};
  const int n = o.n;
  int off = 0;
  L.zn = off; off += bdf::LMAX * n;
  L.ewt = off; off += n;
  L.acor = off; off += n;
  L.ftemp = off; off += n;
  L.tempv = off; off += n;
  L.P = off; off += n;
  L.L = off; off += n;
  L.keff = off; off += o.n_rxn;
  L.J = off; off += o.n_lu;
  L.dinv = off; off += n;
  L.w64 = off;
  // place: bit 0 = y in shared, bit 1 = LU in shared, bit 2 = z in shared
  L.y_smem = place & 1;
  L.lu_smem = (place >> 1) & 1;
  L.z_smem = (place >> 2) & 1;
  size_t sm = 0;  // bytes per lane in shared memory
  int e64 = 0, elt = 0;
  if (L.y_smem) {
    L.y_off = (int)(sm / 8);
    sm += 8 * (size_t)n;
  } else {
    L.y_off = L.w64 + e64;
    e64 += n;
  }
  // LT arrays in shared memory follow y, in units of LT
  size_t lt_base = (sm + lt_size - 1) / lt_size;
  size_t lt_sm = 0;
  if (L.lu_smem) {
    L.lu_off = (int)(lt_base + lt_sm);
    lt_sm += o.n_lu;
  } else {
    L.lu_off = elt;
    elt += o.n_lu;
  }
  if (L.z_smem) {
    L.z_off = (int)(lt_base + lt_sm);
    lt_sm += n;
  } else {
    L.z_off = elt;
    elt += n;
  }
  size_t per_lane = (lt_base + lt_sm) * lt_size;
  L.smem_bytes_per_warp = (int)(((per_lane * 32) + 127) & ~size_t(127));
  L.w64_extra = e64;
  L.wlt = std::max(elt, 1);
  int w = warps_per_block;
  const int avail = max_smem_block - tab_bytes;
  if (avail < 0) return false;
  const int fit = L.smem_bytes_per_warp > 0 ? avail / std::max(1, L.smem_bytes_per_warp) : 16;
  if (fit < 1) return false;
  if (w <= 0) w = std::min(fit, 16);
  w = std::min(w, std::min(fit, 16));
  *warps = w;
  *out = L;
  return true;
}


#define LCK(call)                                                 \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) {                                      \
      *err = std::string(#call) + ": " + cudaGetErrorString(e_);  \
      return false;                                               \
    }                                                             \
  } while (0)

static bool grow(void** p, size_t* cap, size_t bytes, std::string* err) {
  if (*p && *cap >= bytes) return true;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  LCK(cudaMalloc(p, bytes > 0 ? bytes : 16));
  *cap = bytes;
  return true;
}

// Launches the lane-per-cell solve (one block per SM, warps per block from
// the shared-memory layout).  Scratch buffers grow on demand.
bool lanes_launch(const DevMech& m, const void* d_blob, const LaneOff& off, double* d_state,
                  const double* d_env, const double* d_photo, const int* d_order, int n_cells,
                  int* d_counter, CellStats* d_stats, void** scr64, size_t* cap64,
                  void** scrlt, size_t* caplt, double t0, double t1, const SolveSettings& s,
                  int sm_count, int max_smem, void* stream, std::string* err) {
  cudaStream_t st = (cudaStream_t)stream;
  const int lt = s.precision == 1 ? 4 : 8;
  int tab = (off.bytes + 127) & ~127;
  int tab_global = 0;
  lanes::LaneLayout L;
  int warps = 0;
  // the requested placement with the tables staged, else everything per lane
  // in global memory, else the tables in global memory too (mechanisms whose
  // LU schedule alone exceeds shared memory)
  if (!lane_layout(off, lt, max_smem, tab, s.warps_per_block, s.lane_place, &L, &warps) &&
      !lane_layout(off, lt, max_smem, tab, s.warps_per_block, 0, &L, &warps)) {
    tab = 0;
    tab_global = 1;
    if (!lane_layout(off, lt, max_smem, 0, s.warps_per_block, s.lane_place, &L, &warps) &&
        !lane_layout(off, lt, max_smem, 0, s.warps_per_block, 0, &L, &warps)) {
      *err = "lane layout does not fit shared memory";
      return false;
    }
  }
  int grid = sm_count * std::max(1, s.blocks_per_sm);
  const long lanes_total = (long)grid * warps * 32;
  if (lanes_total > n_cells) grid = std::max(1, (int)((n_cells + warps * 32 - 1) / (warps * 32)));
  const size_t total_warps = (size_t)grid * warps;
  if (!grow(scr64, cap64, total_warps * (size_t)(L.w64 + L.w64_extra) * 32 * 8, err)) return false;
  if (!grow(scrlt, caplt, total_warps * (size_t)L.wlt * 32 * lt, err)) return false;
  LCK(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  lanes::LaneArgs a;
  a.m = m;
  a.blob = d_blob;
  a.tab_bytes = tab;
  a.tab_global = tab_global;
  a.lay = L;
  a.state = d_state;
  a.env = d_env;
  a.photo = m.n_photo > 0 ? d_photo : nullptr;
  a.order = d_order;
  a.n_cells = n_cells;
  a.counter = d_counter;
  a.err = d_counter + 1;
  a.stats = d_stats;
  a.scratch64 = (double*)*scr64;
  a.scratchlt = *scrlt;
  a.t0 = t0;
  a.t1 = t1;
  a.rtol = s.rtol;
  a.max_steps = s.max_steps;
  a.maxncf = s.max_conv_fails;
  a.maxnef = s.max_conv_fails;
  const size_t smem = (size_t)tab + (size_t)warps * L.smem_bytes_per_warp;
  if (s.precision == 1) {
    LCK(cudaFuncSetAttribute(lanes::lane_kernel<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lanes::lane_kernel<float><<<grid, warps * 32, smem, st>>>(a);
  } else {
    LCK(cudaFuncSetAttribute(lanes::lane_kernel<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lanes::lane_kernel<double><<<grid, warps * 32, smem, st>>>(a);
  }
  LCK(cudaGetLastError());
  return true;
}

}  // namespace campb
