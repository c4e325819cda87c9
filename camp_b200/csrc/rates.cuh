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
  // SIMPOL and HL instances: reaction type, the reaction's float
  // parameters (10 slots), section kind, GMD / GSD columns (modes) or bin
  // diameter, activity coefficient state index (-1: none), HL water state
  // index, phases of the mode or bin, and (SIMPOL) its constant (not
  // dependent) mass species: state index, 1/density, 1/MW and in-phase flag
  int n_simpol;
  const double* si_prm;
  const int *si_type, *si_kind, *si_gmd_col, *si_gsd_col, *si_act, *si_water, *si_nph,
      *si_cptr, *si_cidx;
  const int* si_wcv;  // HL: computed water index, -1 for a constant water
  const double *si_dp, *si_cinv_rho, *si_cinv_mw, *si_cin;
  // aqueous equilibrium instances: A, C, k_reverse and the minimum water;
  // water and activity coefficient state indices (-1: none), reactant /
  // product counts and the computed-species indices of the water and the
  // activity coefficient (-1: constant); the constant (not dependent)
  // reactants and products: state index, 1e3 / MW, reactant flag
  int n_aq;
  const double *aq_prm, *aq_cm;
  const int *aq_int, *aq_cptr, *aq_cidx, *aq_cr;
  // keff slot of the sub-models' PPM_TO_RH_ (-1: no sub-models)
  int sm_keff;
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

// Per-cell constants of SIMPOL instance k into c[0..7]: the transition-
// regime condensation rate constant k_c = 4 pi r D f(Kn, alpha) (src/util.h:
// 50-135), K_eq, 1 / (kg m-3 -> ppm), the number factor of the mode or bin,
// the activity coefficient, and the volume floors (one minimum mass per
// phase of the mode or bin) plus the constant species' volume, mass and
// moles (src/rxns/rxn_SIMPOL_phase_transfer.c:220-262,
// src/aero_reps/aero_rep_modal_binned_mass.c:176-236,
// src/aero_phase_solver.c:14-19,88-147).  A mode's radius and number factor
// follow from the cell's GMD / GSD columns.
//
// An HL instance (src/rxns/rxn_HL_phase_transfer.c:209-247, 262-330) fills
// the same slots so that the SIMPOL rate formulas give its rates: number
// factor, activity, volume and mass 1, and "moles" K_H * water, so that the
// evaporation rate constant k_c K_eq / moles is k_c / (K_H water), K_H being
// the Henry's law constant in kg_x / kg_H2O / ppm and the water the cell's
// (constant) aerosol-phase water.
static __device__ void simpol_constants(const DevMech& m, int k,
                                                     const double* cell_state, double T,
                                                     double P, const double* photo_cell,
                                                     double* c) {
  constexpr double R = 8.314472, PI = 3.14159265358979323846;
  const double* f = m.si_prm + 10 * k;
  const bool hl = ldg(m.si_type + k) == RXN_HL_PHASE_TRANSFER;
  double alpha = 0.1;
  if (f[0] != 0.0 || f[1] != 0.0) {
    const double del_g = f[0] - T * f[1];
    alpha = exp(-del_g / (R * T));
    alpha = alpha / (1.0 + alpha);
  }
  const double mfp = 3.0 * f[2] / sqrt(8.0 * R * T / (PI * (hl ? f[7] : f[9])));
  double radius, nfac;
  if (ldg(m.si_kind + k) == SECTION_MODAL) {
    const double gmd = photo_cell ? photo_cell[ldg(m.si_gmd_col + k)] : 0.0;
    const double gsd = photo_cell ? photo_cell[ldg(m.si_gsd_col + k)] : 0.0;
    const double lg = log(gsd);
    radius = gmd / 2.0 * exp(5.0 * lg * lg / 2.0);
    nfac = 6.0 / (PI * pow(gmd, 3.0) * exp(9.0 / 2.0 * pow(lg, 2.0)));
  } else {
    const double dp = ldg(m.si_dp + k);
    radius = dp / 2.0;
    nfac = 3.0 / (4.0 * PI) / pow(dp / 2.0, 3.0);
  }
  const double kn = mfp / radius;
  const double fs = (0.75 * alpha * (1.0 + kn)) /
                    (kn * kn + (1.0 + 0.283 * alpha) * kn + 0.75 * alpha);
  c[0] = 4.0 * PI * radius * f[2] * fs;
  if (hl) {
    double kh = f[4] * P * 1.0e-6;
    if (f[5] != 0.0) kh *= exp(f[5] * (1.0 / T - 1.0 / 298.0));
    kh *= f[7];
    const double w = cell_state[ldg(m.si_water + k)];
    c[1] = 1.0;
    c[2] = 1.0 / (f[6] * T / P);
    c[3] = c[4] = c[5] = c[6] = 1.0;
    // a computed water is applied per evaluation (simpol_state)
    c[7] = ldg(m.si_wcv + k) >= 0 ? kh : kh * (w > bdf::kTiny ? w : bdf::kTiny);
    return;
  }
  double vp = f[4] / T + f[5] + f[6] * T + f[7] * log(T);
  vp = 101325.0 * pow(10.0, vp);
  c[1] = vp / P / f[9] * 1.0e6;
  c[2] = 1.0 / (f[8] * T / P);
  c[3] = nfac;
  const int act = ldg(m.si_act + k);
  c[4] = act >= 0 ? cell_state[act] : 1.0;
  double vol = ldg(m.si_nph + k) * (1.0e-25 / 1800.0), mass = 1.0e-25, mol = 1.0e-25 / 0.1;
  for (int j = ldg(m.si_cptr + k); j < ldg(m.si_cptr + k + 1); ++j) {
    double v = cell_state[ldg(m.si_cidx + j)];
    v = v > bdf::kTiny ? v : bdf::kTiny;
    vol += v * ldg(m.si_cinv_rho + j);
    mass += v * ldg(m.si_cin + j);
    mol += v * ldg(m.si_cinv_mw + j);
  }
  c[5] = vol;
  c[6] = mass;
  c[7] = mol;
}

// Forward and reverse rate constants of every aqueous equilibrium instance
// (src/rxns/rxn_aqueous_equilibrium.c:244-262, 278-305), one lane per
// instance, into keff[3 q], keff[3 q + 1], with the constant factors folded
// in: k_f = K_eq k_r times (c m) of each constant reactant and 1 / W per
// reactant after the first; k_r times the activity coefficient, (c m) of
// each constant product and 1 / W per product after the first.  Both are
// zero when the water is below its minimum (:331-336).  A water or activity
// coefficient that a sub-model computes is left out here and applied per
// evaluation (aq_fr), with the minimum water in keff[3 q + 2].  Out of line and
// over plain pointers, so that mechanisms without these reactions keep the
// solve kernel's register allocation.
static __device__ __noinline__ void aq_constants(const double* prm, const int* ii,
                                                 const int* cptr, const int* cidx,
                                                 const double* cm, const int* cr, int n_aq,
                                                 const double* cell_state, double T,
                                                 double* keff, int lane) {
  for (int q = lane; q < n_aq; q += 32) {
    const double* f = prm + 4 * q;
    const int* iq = ii + 6 * q;
    double* c = keff + 3 * q;
    const bool wdyn = ldg(iq + 4) >= 0, gdyn = ldg(iq + 5) >= 0;
    double w = cell_state[ldg(iq)];
    w = w > bdf::kTiny ? w : bdf::kTiny;
    c[2] = ldg(f + 3);
    if (!wdyn && w < ldg(f + 3)) {
      c[0] = c[1] = 0.0;
      continue;
    }
    const double eq = f[1] == 0.0 ? f[0] : f[0] * exp(f[1] * (1.0 / T - 1.0 / 298.0));
    double kf = eq * f[2], kr = f[2];
    const int act = ldg(iq + 1);
    if (act >= 0 && !gdyn) kr *= cell_state[act];
    for (int j = ldg(cptr + q); j < ldg(cptr + q + 1); ++j) {
      double v = cell_state[ldg(cidx + j)];
      v = (v > bdf::kTiny ? v : bdf::kTiny) * ldg(cm + j);
      if (ldg(cr + j))
        kf *= v;
      else
        kr *= v;
    }
    if (!wdyn) {
      for (int i = 1; i < ldg(iq + 2); ++i) kf /= w;
      for (int i = 1; i < ldg(iq + 3); ++i) kr /= w;
    }
    c[0] = kf;
    c[1] = kr;
  }
}

// k of every reaction times the (clamped) constant-species concentrations it
// multiplies; constant species are clamped to TINY as solver_run does.  The
// SIMPOL constants follow the terms' (keff[n_rxn + 8 k ..]), then the
// aqueous equilibrium ones (keff[n_rxn + 8 n_simpol + 3 q ..]), then the
// sub-models' PPM_TO_RH_.
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
  for (int k = lane; k < m.n_simpol; k += 32)
    simpol_constants(m, k, cell_state, T, P, photo_cell, keff + m.n_rxn + 8 * k);
  if (m.n_aq > 0)
    aq_constants(m.aq_prm, m.aq_int, m.aq_cptr, m.aq_cidx, m.aq_cm, m.aq_cr, m.n_aq, cell_state,
                 T, keff + m.n_rxn + 8 * m.n_simpol, lane);
  if (m.sm_keff >= 0 && lane == 0) {
    // PPM_TO_RH_: the MOSAIC water vapour pressure fit
    // (src/sub_models/sub_model_ZSR_aerosol_water.c:198-214)
    double a = 1.0 - 373.15 / T;
    a = (((-0.1299 * a - 0.6445) * a - 1.976) * a + 13.3185) * a;
    keff[m.sm_keff] = P / (101325.0 * exp(a)) / 1.0e6;
  }
  __syncwarp();
}


}  // namespace campb
