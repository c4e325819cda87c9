// Rate constants of the gas-phase reaction types on the device, shared by the
// solve kernels.  DevMech points at the per-reaction rate-law parameters in
// global memory; these are read once per cell per host step.
#pragma once

#include <cuda_runtime.h>

#include "bdf_consts.hpp"
#include "model.hpp"

namespace campb {

struct DevMech {
  int n, n_state, n_rxn, n_part, n_jac, n_lu, n_photo, n_flev, n_blev;
  int n_const;
  const int *rx_type, *rx_nreact, *rx_fpar, *rx_photo;
  const double* fpar;
  const int *rx_cptr, *rx_cidx, *rx_vptr, *rx_vdep;
  const int *fg_ptr, *fg_rxn, *fg_prod;
  const double* fg_coef;
  const int *jg_ptr, *jg_part, *jg_ind, *jg_lupos, *jg_row;
  const int* jac_colptr;  // solver Jacobian CSC column pointers
  const double* jg_coef;
  const int *lu_perm, *lu_rowptr, *lu_col, *lu_diag;
  const int *upd_ptr, *upd_src, *upd_dst;
  const int *fl_ptr, *fl_rows, *bl_ptr, *bl_rows;
  const int *dep_state, *const_state;
  const double* atol;  // per dependent variable
};

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
  return __ldg(p);
}

// ---------------------------------------------------------------------------
// Rate constants (update_env_state of the gas types)
// ---------------------------------------------------------------------------
static __device__ double rate_constant(const DevMech& m, int r, double T, double P,
                                const double* photo_cell) {
  const double* f = m.fpar + ldg(m.rx_fpar + r);
  const int nr = ldg(m.rx_nreact + r);
  switch (ldg(m.rx_type + r)) {
    case RXN_ARRHENIUS:  // src/rxns/rxn_arrhenius.c:103-118
      return f[0] * exp(f[2] / T) * (f[1] == 0.0 ? 1.0 : pow(T / f[3], f[1])) *
             (f[4] == 0.0 ? 1.0 : (1.0 + f[4] * P)) * pow(f[5] * P / T, (double)(nr - 1));
    case RXN_TROE: {  // src/rxns/rxn_troe.c:118-140
      double conv = f[9] * P / T;
      double k0 = f[0] * (f[2] == 0.0 ? 1.0 : exp(f[2] / T)) *
                  (f[1] == 0.0 ? 1.0 : pow(T / 300.0, f[1])) * conv;
      double kinf = k0 / (f[3] * (f[5] == 0.0 ? 1.0 : exp(f[5] / T)) *
                          (f[4] == 0.0 ? 1.0 : pow(T / 300.0, f[4])));
      double e = log10(kinf) / f[7];
      return (k0 / (1.0 + kinf)) * pow(f[6], 1.0 / (1.0 + e * e)) *
             pow(conv, (double)(nr - 1)) * f[8];
    }
    case RXN_CMAQ_H2O2: {  // src/rxns/rxn_CMAQ_H2O2.c:106-125
      double conv = f[6] * P / T;
      return (f[0] * (f[2] == 0.0 ? 1.0 : exp(f[2] / T)) *
                  (f[1] == 0.0 ? 1.0 : pow(T / 300.0, f[1])) +
              f[3] * (f[5] == 0.0 ? 1.0 : exp(f[5] / T)) *
                  (f[4] == 0.0 ? 1.0 : pow(T / 300.0, f[4])) * conv) *
             pow(conv, (double)(nr - 1));
    }
    case RXN_CMAQ_OH_HNO3: {  // src/rxns/rxn_CMAQ_OH_HNO3.c:110-133
      double conv = f[10] * P / T;
      double k2 = f[3] * (f[5] == 0.0 ? 1.0 : exp(f[5] / T)) *
                  (f[4] == 0.0 ? 1.0 : pow(T / 300.0, f[4]));
      double k3 = f[6] * (f[8] == 0.0 ? 1.0 : exp(f[8] / T)) *
                  (f[7] == 0.0 ? 1.0 : pow(T / 300.0, f[7])) * conv;
      return (f[0] * (f[2] == 0.0 ? 1.0 : exp(f[2] / T)) *
                  (f[1] == 0.0 ? 1.0 : pow(T / 300.0, f[1])) +
              k3 / (1.0 + k3 / k2)) *
             pow(conv, (double)(nr - 1)) * f[9];
    }
    case RXN_PHOTOLYSIS:        // src/rxns/rxn_photolysis.c:137-148
    case RXN_FIRST_ORDER_LOSS:  // src/rxns/rxn_first_order_loss.c:118-130
    case RXN_EMISSION:          // src/rxns/rxn_emission.c:109-120
    case RXN_WET_DEPOSITION:    // src/rxns/rxn_wet_deposition.c:124-136
      // SCALING_ * BASE_RATE_, the base rate being the cell's host-set value
      return f[0] * (photo_cell ? photo_cell[ldg(m.rx_photo + r)] : 0.0);
  }
  return 0.0;
}

// k of every reaction times the (clamped) constant-species concentrations it
// multiplies; constant species are clamped to TINY as solver_run does.
static __device__ void compute_keff(const DevMech& m, const double* cell_state,
                             double T, double P, const double* photo_cell,
                             double* keff, int lane) {
  for (int r = lane; r < m.n_rxn; r += 32) {
    double k = rate_constant(m, r, T, P, photo_cell);
    for (int c = ldg(m.rx_cptr + r); c < ldg(m.rx_cptr + r + 1); ++c) {
      double s = cell_state[ldg(m.rx_cidx + c)];
      k *= s > bdf::kTiny ? s : bdf::kTiny;
    }
    keff[r] = k;
  }
  __syncwarp();
}


}  // namespace campb
