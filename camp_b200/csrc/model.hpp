// Host-side mechanism model: packed reaction data, Jacobian sparsity, the
// fixed elimination order of the per-cell LU and the flat tables the device
// kernels read.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace campb {

// reaction type ids, src/rxn_solver.c:19-35
enum : int {
  RXN_ARRHENIUS = 1,
  RXN_TROE = 2,
  RXN_CMAQ_H2O2 = 3,
  RXN_CMAQ_OH_HNO3 = 4,
  RXN_PHOTOLYSIS = 5,
  RXN_FIRST_ORDER_LOSS = 12,
  RXN_EMISSION = 13,
  RXN_WET_DEPOSITION = 14,
};

// Types whose rate the host sets per cell through rxn_update_data
// (src/rxn_solver.c:735-760): k = SCALING_ * BASE_RATE_.
inline bool host_rate_type(int type) {
  return type == RXN_PHOTOLYSIS || type == RXN_FIRST_ORDER_LOSS || type == RXN_EMISSION ||
         type == RXN_WET_DEPOSITION;
}

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
  int n_jac = 0;    // solver Jacobian entries
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
  // FG_PRODUCT: guarded, FG_SOURCE: unguarded gain of a zero-order term)
  std::vector<int> fg_ptr, fg_rxn, fg_prod;
  std::vector<double> fg_coef;
  // J gather by solver Jacobian entry (CSC order)
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

  // get_jac_init (src/camp_solver.c:1417-1712) for a gas-phase model:
  // reaction Jacobian, DERIV_ID/JAC_ID, solver Jacobian; then the LU
  // elimination order and the device tables.  Returns false on error.
  bool build(std::string* err);

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
  const std::vector<int>& solver_colptr() const { return sj_colptr_; }
  const std::vector<int>& solver_rowid() const { return sj_rowid_; }
  const Tables& tables() const { return tab_; }
  bool built() const { return built_; }

  // host-rate columns: column of each reaction of a host_rate_type in
  // mechanism order (-1 for other types), and its RXN_ID_ value
  const std::vector<int>& photo_slot() const { return photo_slot_; }
  int photo_id(int rxn) const;
  int n_terms() const { return n_terms_; }
  int n_host_rate() const { return n_host_rate_; }

 private:
  void build_rxn_jacobian();
  void update_ids();
  void build_solver_jacobian();
  void build_lu();
  void build_level_schedules(const std::vector<std::vector<int>>& pos,
                             const std::vector<int>& flev, int nfl,
                             const std::vector<int>& blev, int nbl);
  void build_tables();
  int rxn_elem_id(int dep, int ind) const;

  int n_state_, n_cells_, n_dep_, n_rxn_;
  int n_added_ = 0, n_env_ = 0, n_terms_ = 0, n_host_rate_ = 0;
  std::vector<int> var_type_;
  std::vector<int> rxn_int_;
  std::vector<double> rxn_float_;
  std::vector<Rxn> rxns_;
  std::vector<int> photo_slot_;
  std::vector<int> deriv_ids_;
  std::vector<int> rj_colptr_, rj_rowid_;
  std::vector<int> sj_colptr_, sj_rowid_;
  Tables tab_;
  bool built_ = false;
};

}  // namespace campb
