// Host-side mechanism model: packed reaction data, Jacobian sparsity, the
// fixed elimination order of the per-cell LU and the flat tables the device
// kernels read.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace campb {

// reaction type ids, src/rxn_solver.c:19-35
enum : int {
  RXN_ARRHENIUS = 1,
  RXN_TROE = 2,
  RXN_CMAQ_H2O2 = 3,
  RXN_CMAQ_OH_HNO3 = 4,
  RXN_PHOTOLYSIS = 5,
  RXN_HL_PHASE_TRANSFER = 6,
  RXN_AQUEOUS_EQUILIBRIUM = 7,
  RXN_FIRST_ORDER_LOSS = 12,
  RXN_EMISSION = 13,
  RXN_WET_DEPOSITION = 14,
  RXN_SIMPOL_PHASE_TRANSFER = 10,
};

// sub-model type ids, src/sub_model_solver.c:16-18
enum : int { SUB_MODEL_ZSR_AEROSOL_WATER = 2, SUB_MODEL_PDFITE = 3 };

// aerosol representation types, src/aero_rep_solver.c:19-20; section types
// of the modal/binned mass representation
enum : int { AERO_REP_MODAL_BINNED_MASS = 2 };
enum : int { SECTION_BINNED = 1, SECTION_MODAL = 2 };

// Types whose rate the host sets per cell through rxn_update_data
// (src/rxn_solver.c:735-760): k = SCALING_ * BASE_RATE_.
inline bool host_rate_type(int type) {
  return type == RXN_PHOTOLYSIS || type == RXN_FIRST_ORDER_LOSS || type == RXN_EMISSION ||
         type == RXN_WET_DEPOSITION;
}

// One phase instance of a SIMPOL or HL phase-transfer reaction (its
// partitioning into one phase of one mode or bin).  Elements are the mass
// species (variable, constant, PSSA) of every phase of the mode or bin in
// state order: the number concentration depends on all of them, the phase
// mass and mean molecular weight on those of the instance's phase
// (src/aero_reps/aero_rep_modal_binned_mass.c:86-125).  HL registers the
// same elements, but its partials over them are zero for this
// representation (radii do not depend on the state and its number
// concentration is 1, src/rxns/rxn_HL_phase_transfer.c:386-399): they
// take no part in the device tables.
struct SimpolInst {
  int type = RXN_SIMPOL_PHASE_TRANSFER;  // or RXN_HL_PHASE_TRANSFER
  int rxn = 0, x = 0;              // reaction, instance within it
  int gas = 0, aero = 0, act = -1;  // state indices (act: -1 when none)
  int water = -1;                   // HL: aerosol-phase water (state index)
  int rep = 0, section = 0, bin = 0, phase = 0;
  int kind = SECTION_MODAL;
  int gmd_col = -1, gsd_col = -1;   // host-set columns of a mode's GMD / GSD
  double bin_dp = 0.0;              // bin diameter [m] (bins)
  int n_phases = 0;                 // phases of the mode or bin (volume floors)
  // the reaction's float parameters: DELTA_H DELTA_S DIFF_COEFF PRE_C_AVG
  // B1..B4 CONV MW (SIMPOL, src/rxns/rxn_SIMPOL_phase_transfer.c:31-40) or
  // DELTA_H DELTA_S DIFF_COEFF PRE_C_AVG A C CONV MW (HL,
  // src/rxns/rxn_HL_phase_transfer.c:29-36)
  double prm[10] = {0.0};
  std::vector<int> elem;            // state indices
  std::vector<double> inv_rho, inv_mw;  // 1/density; 1/MW in the phase, else 0
  std::vector<char> in_phase;
  int water_cv = -1;                // HL: the water's computed-species index, -1 if constant
};

// One phase instance of an aqueous equilibrium reaction
// (src/rxns/rxn_aqueous_equilibrium.c:27-56): forward rate
// k_f prod(c_i m_i) / W^(n_r - 1), reverse rate k_r gamma prod(c_j m_j) /
// W^(n_p - 1), with m = 1e3 / MW (mass fraction -> M), W the aerosol-phase
// water and gamma the ion pair's activity coefficient; each reactant loses
// the forward rate / m_i and gains the reverse rate / m_i, each product the
// reverse.  W and gamma are constant species, so per cell the constant
// factors fold into two rate constants and the dependent species keep
// mass-action form.
struct AqInst {
  int rxn = 0, p = 0;                 // reaction, phase instance within it
  std::vector<int> react, prod;       // state indices
  std::vector<double> m2m;            // MASS_FRAC_TO_M_: reactants, then products
  int water = -1, act = -1;           // state indices (act: -1 when none)
  double A = 1.0, C = 0.0, kr = 0.0;  // equilibrium constant parameters, k_reverse
  double thr = 0.0;                   // water below which the reaction is off
  // computed-species indices of the water and the activity coefficient when
  // a sub-model computes them (-1: a constant species, folded per cell)
  int water_cv = -1, act_cv = -1;
  // reactants and products that a sub-model computes (the water of
  // H2O_aq <=> H+ + OH-): state index, computed index, 1e3 / MW, reactant
  // flag; they enter the rates per evaluation, not per cell
  std::vector<int> cp_state, cp_cv;
  std::vector<double> cp_m;
  std::vector<char> cp_r;
};

// One species that a sub-model computes from the state before every f and J
// (src/sub_model_solver.c:300-333): the aerosol-phase water of a ZSR phase
// instance or the activity coefficient of a PD-FiTE ion pair, with a compact
// program for its value and for its row of the parameter Jacobian.
//   ZSR water (kind 1), ints: kind, gas-water dependent index, pair count,
//     then per ion pair its type and
//       Jacobson: cation, anion (dependent indices), Y count, parameter ids
//                 of d/d(gas water), d/d(cation), d/d(anion);
//       EQSAM: ion count, parameter id of d/d(gas water), per ion its
//              dependent index and parameter id;
//     floats per pair: Jacobson: low RH, 1 / (cation count x cation MW x
//     1000), the same for the anion, Y...; EQSAM: NW 55.51 18.01 / MW / 1000,
//     ZW, 1 / ion MW of each ion.
//   PD-FiTE activity of pair x (kind 2), ints: kind, gas-water dependent
//     index, pair count, x, interaction count, parameter id of d/d(gas
//     water), per pair j: cation, anion (dependent indices), cation + anion
//     stoichiometry, parameter ids of d/d(cation j), d/d(anion j); per
//     interaction: its pair, B count;
//     floats: per pair 1 / (cation MW x 1e6), 1 / (anion MW x 1e6) (moles
//     per concentration, also the partials' factors); per interaction min
//     RH, max RH, B...
struct SubProgram {
  int state = -1;  // state index of the computed species
  std::vector<int> ints;
  std::vector<double> flts;
};

// kinds of f gather entries (Tables::fg_prod)
enum : int { FG_LOSS = 0, FG_PRODUCT = 1, FG_SOURCE = 2 };

// state variable types, src/camp_common.h:34-38
enum : int { VAR_VARIABLE = 1, VAR_CONSTANT = 2 };

// One mass-action term: rate = k * prod(reactants); the rate is lost by each
// reactant and gained, times its yield, by each product.  A product is
// guarded (dropped when a negative yield would take it below zero within one
// step, src/rxns/rxn_arrhenius.c:153-160) unless the term is a zero-order
// source (EMISSION, src/rxns/rxn_emission.c:133-147), which has no guard.
struct Term {
  std::vector<int> react, prod;  // state indices
  std::vector<double> yield;
  bool source = false;
  // positions in Model::rxn_int of the DERIV_ID of each reactant then each
  // product, and of the JAC_ID of each (reactant, reactant-or-product) pair
  std::vector<int> deriv_at, jac_at;
};

// One reaction's view into the packed arrays, with its mass-action terms:
// one for the gas types, FIRST_ORDER_LOSS and EMISSION, one per species for
// WET_DEPOSITION (each species is lost at the shared rate constant).
struct Rxn {
  int type = 0;
  int int_off = 0;    // first int after the type slot in Model::rxn_int
  int float_off = 0;  // first float parameter
  int env_off = 0;    // first env parameter within a cell's rxn_env_data
  int n_int_prop = 2, n_float_prop = 0;  // head blocks of the packed data
  int rid_at = -1;    // position of RXN_ID_ in Model::rxn_int, -1 if none
  std::vector<Term> terms;
};

// Flat tables that drive the device code.  All indices are int32.
struct Tables {
  int n = 0;        // dependent variables
  int n_state = 0;  // state variables per cell
  int n_rxn = 0;     // mass-action terms (Rxn::terms of every reaction)
  int n_part = 0;   // variable-reactant occurrences (rate partials)
  int n_jac = 0;    // live solver Jacobian entries (Model::device_colptr)
  int n_lu = 0;     // L+U entries
  int n_photo = 0;  // host-rate columns (reactions of a host_rate_type)
  int n_flev = 0, n_blev = 0;
  int max_fgather = 0;

  // per term: type, number of reactants (incl. constants), packed float
  // parameters (the type's head block), host-rate column (-1 if none)
  std::vector<int> rx_type, rx_nreact, rx_fpar, rx_photo;
  std::vector<double> fpar;
  // constant reactants (state index), variable reactants (dependent index)
  std::vector<int> rx_cptr, rx_cidx, rx_vptr, rx_vdep;
  // f gather by dependent species: term, coefficient, kind (FG_LOSS,
  // FG_PRODUCT: guarded, FG_SOURCE: unguarded gain of a zero-order term).
  // Terms n_rxn + 4 k + (0..3) are the SIMPOL pseudo-rates of instance k:
  // gas gain (evaporation), gas loss (condensation), aerosol loss, gain.
  std::vector<int> fg_ptr, fg_rxn, fg_prod;
  // SIMPOL: instances, their per-cell constants (keff slots n_rxn + 8 k ..),
  // and their Jacobian partials (part slots from si_part0[k])
  int n_simpol = 0;
  std::vector<SimpolInst> simpol;
  std::vector<int> si_part0;
  // aqueous equilibrium instances: per-cell constants at keff slots
  // aq_keff0 (forward, reverse), pseudo-rates from aq_rate0 (a loss and a
  // gain per dependent species slot), partials from aq_part0 (per dependent
  // independent slot, every dependent row slot)
  int n_aq = 0;
  std::vector<AqInst> aq;
  std::vector<int> aq_keff0, aq_rate0, aq_part0;
  // sub-models: the computed species (per-cell values written before every
  // f and J after the rates or partials), their programs, the parameter
  // Jacobian size (its element ids index the parameter partials), and the
  // per-cell constant PPM_TO_RH_ at keff slot sm_keff
  int n_cv = 0, n_pj = 0, sm_keff = -1;
  std::vector<SubProgram> cv;
  // rate partials against computed species gather into virtual Jacobian
  // slots (a variable row, a computed column; each partial adds with
  // coefficient 1), which the chain then folds into the solver slots:
  // J[ch_tgt[g]] += sum over [ch_ptr[g], ch_ptr[g+1]) of V[ch_v] * P[ch_p]
  // (src/camp_solver.c:1096-1106 with J_params)
  int n_virt = 0;
  std::vector<int> jv_ptr, jv_part, jv_row;
  std::vector<int> ch_tgt, ch_ptr, ch_v, ch_p;
  int n_part_all = 0;  // n_part + SIMPOL and aqueous partials
  int n_keff = 0;      // n_rxn + 8 n_simpol + 2 n_aq
  int n_rates = 0;     // n_rxn + 4 n_simpol + aqueous pseudo-rates
  std::vector<double> fg_coef;
  // J gather by live solver Jacobian entry (CSC order); jg_ind: -1 loss,
  // -2 unguarded product (phase transfer), else the guard's independent
  // species
  std::vector<int> jg_ptr, jg_part, jg_ind, jg_lupos, jg_row;
  std::vector<double> jg_coef;
  // LU structure in pivot order
  std::vector<int> lu_perm, lu_iperm, lu_rowptr, lu_col, lu_diag;
  std::vector<int> upd_ptr, upd_src, upd_dst;  // per L entry position
  std::vector<int> fl_ptr, fl_rows;            // forward / factor row levels
  std::vector<int> bl_ptr, bl_rows;            // backward row levels
  std::vector<int> dep_state;                  // dependent index -> state index
  // Right-looking factorization by pivot levels (pivots whose rows and
  // columns no other pivot of the level updates).  Per level: pivots whose
  // reciprocal is taken (fd), L entries scaled by their pivot reciprocal
  // (fa: position, pivot), and the Schur updates grouped by target (fb).
  // Forward / backward solves by column levels, grouped by target.
  // A grouped phase is: units (target, first pair, pair count) and pairs
  // (two positions); units are spread over 32 lanes per level.
  struct Grouped {
    int n_levels = 0;
    std::vector<int> lane_ptr;  // n_levels * 33 unit indices
    std::vector<int> unit_target, unit_begin, unit_count, unit_recip;
    std::vector<int> pair_a, pair_b;
  };
  int n_plev = 0;
  std::vector<int> fa_ptr, fa_pos, fa_piv;
  Grouped fb, fwd, bwd;
};

class Model {
 public:
  Model(int n_state_var, int n_cells, const int* var_type, int n_rxn,
        int n_rxn_int, int n_rxn_float, int n_rxn_env);

  // rxn_add_condensed_data (src/rxn_solver.c:658-700)
  bool add_rxn(int type, int n_int, int n_float, int n_env, const int* ints,
               const double* floats, std::string* err);
  // aero_phase_add_condensed_data (src/aero_phase_solver.c:175-202) and
  // aero_rep_add_condensed_data (src/aero_rep_solver.c:443-484); the
  // modal/binned mass representation only
  bool add_aero_phase(int n_int, int n_float, const int* ints, const double* floats,
                      std::string* err);
  bool add_aero_rep(int type, int n_int, int n_float, int n_env, const int* ints,
                    const double* floats, std::string* err);
  int n_aero_phase() const { return (int)aph_int_.size(); }
  int n_aero_rep() const { return (int)arep_int_.size(); }
  // condensed data of phase / representation k (representations: the
  // element counts are written at solver_initialize)
  const std::vector<int>& aero_phase_int(int k) const { return aph_int_[k]; }
  const std::vector<double>& aero_phase_float(int k) const { return aph_flt_[k]; }
  const std::vector<int>& aero_rep_int(int k) const { return arep_int_[k]; }
  const std::vector<double>& aero_rep_float(int k) const { return arep_flt_[k]; }
  // modes of every representation, (representation, section) in order: the
  // GMD / GSD host-set columns after the reaction columns
  const std::vector<std::pair<int, int>>& modes() const { return modes_; }
  // sub_model_add_condensed_data (src/sub_model_solver.c:425-470): ZSR
  // aerosol water and PD-FiTE activity; ints without the type slot
  bool add_sub_model(int type, int n_int, int n_float, int n_env, const int* ints,
                     const double* floats, std::string* err);
  int n_sub_model() const { return (int)sub_type_.size(); }
  int sub_model_type(int k) const { return sub_type_[k]; }
  const std::vector<int>& sub_model_int(int k) const { return sub_int_[k]; }
  const std::vector<double>& sub_model_float(int k) const { return sub_flt_[k]; }
  // the sub-model parameter Jacobian (CSC over state variables, with the
  // dummy element (0, 0)) and the solver Jacobian fold as (solver id,
  // reaction-Jacobian id, parameter id) triplets
  const std::vector<int>& param_colptr() const { return pj_colptr_; }
  const std::vector<int>& param_rowid() const { return pj_rowid_; }
  const std::vector<int>& jac_map() const { return jac_map_; }
  // aero_rep_update_data for the modal/binned representation: the id and
  // the section of a GMD (what 0) / GSD (what 1) update -> its column, or -1
  int aero_column(int rep_id, int section, int what) const;

  // get_jac_init (src/camp_solver.c:1417-1712) for a gas-phase model:
  // reaction Jacobian, DERIV_ID/JAC_ID, solver Jacobian; then the LU
  // elimination order and the device tables.  Returns false on error.
  bool build(std::string* err);
  // the absolute tolerances solver_initialize receives (per state
  // variable): they set the aqueous equilibrium's minimum water
  // (src/rxns/rxn_aqueous_equilibrium.c:222-227)
  void set_abs_tol(const double* abs_tol) { abs_tol_.assign(abs_tol, abs_tol + n_state_); }

  int n_state() const { return n_state_; }
  int n_cells() const { return n_cells_; }
  int n_dep() const { return n_dep_; }
  int n_rxn() const { return n_rxn_; }
  int n_added() const { return n_added_; }
  int n_rxn_env() const { return n_env_; }
  const std::vector<int>& var_type() const { return var_type_; }
  const std::vector<int>& rxn_int() const { return rxn_int_; }
  const std::vector<double>& rxn_float() const { return rxn_float_; }
  const std::vector<Rxn>& rxns() const { return rxns_; }
  // the solver Jacobian as the reference builds it (every registered
  // variable x variable element, src/camp_solver.c:1559-1633)
  const std::vector<int>& solver_colptr() const { return sj_colptr_; }
  const std::vector<int>& solver_rowid() const { return sj_rowid_; }
  // its live entries, the ones some reaction can make non-zero, which the
  // LU and the device tables use (every entry for mechanisms without HL
  // phase transfer), and the solver entry of each
  const std::vector<int>& device_colptr() const { return dj_colptr_; }
  const std::vector<int>& device_rowid() const { return dj_rowid_; }
  const std::vector<int>& device_to_solver() const { return dj_to_sj_; }
  const Tables& tables() const { return tab_; }
  bool built() const { return built_; }

  // host-rate columns: column of each reaction of a host_rate_type in
  // mechanism order (-1 for other types), and its RXN_ID_ value
  const std::vector<int>& photo_slot() const { return photo_slot_; }
  int photo_id(int rxn) const;
  int n_terms() const { return n_terms_; }
  // host-set columns: reaction rates, then the GMD and GSD of every mode
  int n_host_rate() const { return n_host_rate_ + 2 * (int)modes_.size(); }

 private:
  void build_rxn_jacobian();
  void update_ids();
  void build_solver_jacobian();
  void build_lu();
  void build_level_schedules(const std::vector<std::vector<int>>& pos,
                             const std::vector<int>& flev, int nfl,
                             const std::vector<int>& blev, int nbl);
  void build_tables();
  bool resolve_simpol(std::string* err);
  bool resolve_instance(SimpolInst* si, int phase, int ri, std::string* err);
  bool resolve_aq(std::string* err);
  bool resolve_sub_models(std::string* err);
  void build_param_jacobian();
  void build_sub_programs();
  int rxn_elem_id(int dep, int ind) const;
  int param_elem_id(int dep, int ind) const;

  int n_state_, n_cells_, n_dep_, n_rxn_;
  int n_added_ = 0, n_env_ = 0, n_terms_ = 0, n_host_rate_ = 0;
  std::vector<int> var_type_;
  std::vector<int> rxn_int_;
  std::vector<double> rxn_float_;
  std::vector<Rxn> rxns_;
  std::vector<int> photo_slot_;
  std::vector<std::vector<int>> aph_int_, arep_int_;
  std::vector<std::vector<double>> aph_flt_, arep_flt_;
  std::vector<int> arep_type_;
  std::vector<std::pair<int, int>> modes_;
  std::vector<SimpolInst> simpol_;
  std::vector<AqInst> aq_;
  // sub-models as added; computed species (state index -> computed index)
  std::vector<int> sub_type_;
  std::vector<std::vector<int>> sub_int_;
  std::vector<std::vector<double>> sub_flt_;
  std::vector<int> cv_state_, cv_of_;
  std::vector<int> pj_colptr_, pj_rowid_, jac_map_;
  std::vector<double> abs_tol_;
  std::vector<int> deriv_ids_;
  std::vector<int> rj_colptr_, rj_rowid_;
  std::vector<int> rl_colptr_, rl_rowid_;  // live subset of the reaction Jacobian
  std::vector<int> sj_colptr_, sj_rowid_;
  std::vector<int> dj_colptr_, dj_rowid_, dj_to_sj_;
  Tables tab_;
  bool built_ = false;
};

}  // namespace campb
