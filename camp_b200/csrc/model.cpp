// Host-side mechanism model.  See model.hpp.
#include "model.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace campb {

namespace {
// NUM_INT_PROP_ / NUM_FLOAT_PROP_ of the supported types (src/rxns/rxn_*.c
// headers)
bool type_layout(int type, int* n_int_prop, int* n_float_prop) {
  switch (type) {
    case RXN_ARRHENIUS: *n_int_prop = 2; *n_float_prop = 6; return true;
    case RXN_TROE: *n_int_prop = 2; *n_float_prop = 10; return true;
    case RXN_CMAQ_H2O2: *n_int_prop = 2; *n_float_prop = 7; return true;
    case RXN_CMAQ_OH_HNO3: *n_int_prop = 2; *n_float_prop = 11; return true;
    case RXN_PHOTOLYSIS: *n_int_prop = 3; *n_float_prop = 1; return true;
    case RXN_FIRST_ORDER_LOSS: *n_int_prop = 4; *n_float_prop = 1; return true;
    case RXN_EMISSION: *n_int_prop = 3; *n_float_prop = 1; return true;
    case RXN_WET_DEPOSITION: *n_int_prop = 2; *n_float_prop = 1; return true;
    case RXN_SIMPOL_PHASE_TRANSFER: *n_int_prop = 2; *n_float_prop = 10; return true;
    case RXN_HL_PHASE_TRANSFER: *n_int_prop = 2; *n_float_prop = 8; return true;
    case RXN_AQUEOUS_EQUILIBRIUM: *n_int_prop = 3; *n_float_prop = 5; return true;
    default: return false;
  }
}

// Column-wise registry of (dep, ind) pairs; a pair is stored once and the
// rows of each column are sorted when the matrix is built
// (src/Jacobian.c:105-188).
struct Registry {
  std::vector<std::vector<int>> cols;
  explicit Registry(int n) : cols(n) {}
  void add(int dep, int ind) {
    auto& c = cols[ind];
    if (std::find(c.begin(), c.end(), dep) == c.end()) c.push_back(dep);
  }
  void to_csc(std::vector<int>* colptr, std::vector<int>* rowid) {
    colptr->assign(cols.size() + 1, 0);
    rowid->clear();
    for (size_t c = 0; c < cols.size(); ++c) {
      std::sort(cols[c].begin(), cols[c].end());
      (*colptr)[c] = (int)rowid->size();
      rowid->insert(rowid->end(), cols[c].begin(), cols[c].end());
    }
    (*colptr)[cols.size()] = (int)rowid->size();
  }
};
}  // namespace

Model::Model(int n_state_var, int n_cells, const int* var_type, int n_rxn,
             int n_rxn_int, int n_rxn_float, int n_rxn_env)
    : n_state_(n_state_var), n_cells_(n_cells), n_dep_(0), n_rxn_(n_rxn) {
  var_type_.assign(var_type, var_type + n_state_var);
  for (int v : var_type_)
    if (v == VAR_VARIABLE) ++n_dep_;
  rxn_int_.reserve((size_t)std::max(0, n_rxn_int + n_rxn));
  rxn_float_.reserve((size_t)std::max(0, n_rxn_float));
  (void)n_rxn_env;
}

bool Model::add_rxn(int type, int n_int, int n_float, int n_env,
                    const int* ints, const double* floats, std::string* err) {
  if (n_added_ >= n_rxn_) {
    *err = "more reactions added than declared in solver_new";
    return false;
  }
  Rxn r;
  r.type = type;
  rxn_int_.push_back(type);
  r.int_off = (int)rxn_int_.size();
  rxn_int_.insert(rxn_int_.end(), ints, ints + n_int);
  r.float_off = (int)rxn_float_.size();
  rxn_float_.insert(rxn_float_.end(), floats, floats + n_float);
  r.env_off = n_env_;
  n_env_ += n_env;
  const int idx = n_added_++;
  // host-rate column, in mechanism order (known before solver_initialize so
  // that rxn_update_data can be called as soon as the reaction is added)
  photo_slot_.push_back(host_rate_type(type) ? n_host_rate_++ : -1);
  auto fail = [&](const std::string& msg) {
    *err = msg;
    rxns_.push_back(r);
    return false;
  };
  if (!type_layout(type, &r.n_int_prop, &r.n_float_prop))
    return fail("reaction type " + std::to_string(type) +
                " is not supported (ARRHENIUS, TROE, CMAQ_H2O2, CMAQ_OH_HNO3, PHOTOLYSIS, "
                "FIRST_ORDER_LOSS, EMISSION, WET_DEPOSITION, SIMPOL_PHASE_TRANSFER, "
                "HL_PHASE_TRANSFER and AQUEOUS_EQUILIBRIUM only)");
  const std::string malformed = "malformed packed data for reaction " + std::to_string(idx);
  if (n_int < r.n_int_prop || n_float < r.n_float_prop) return fail(malformed);
  const int o = r.int_off;  // rxn_int_ position of ints[0]
  switch (type) {
    case RXN_FIRST_ORDER_LOSS: {  // RXN_ID_ REACT_ DERIV_ID_ JAC_ID_ (rxn_first_order_loss.c:20-23)
      Term t;
      t.react = {ints[1] - 1};
      t.deriv_at = {o + 2};
      t.jac_at = {o + 3};
      r.terms.push_back(t);
      r.rid_at = o;
      break;
    }
    case RXN_EMISSION: {  // RXN_ID_ SPECIES_ DERIV_ID_ (rxn_emission.c:20-22)
      Term t;
      t.prod = {ints[1] - 1};
      t.yield = {1.0};
      t.source = true;
      t.deriv_at = {o + 2};
      r.terms.push_back(t);
      r.rid_at = o;
      break;
    }
    case RXN_WET_DEPOSITION: {  // RXN_ID_ NUM_SPEC_ REACT_(s) DERIV_ID_(s) JAC_ID_(s)
      const int ns = ints[1];  // (rxn_wet_deposition.c:20-30)
      if (ns < 0 || n_int < 2 + 3 * ns) return fail(malformed);
      for (int k = 0; k < ns; ++k) {
        Term t;
        t.react = {ints[2 + k] - 1};
        t.deriv_at = {o + 2 + ns + k};
        t.jac_at = {o + 2 + 2 * ns + k};
        r.terms.push_back(t);
      }
      r.rid_at = o;
      break;
    }
    case RXN_SIMPOL_PHASE_TRANSFER:  // src/rxns/rxn_SIMPOL_phase_transfer.c:37-78
    case RXN_HL_PHASE_TRANSFER: {    // src/rxns/rxn_HL_phase_transfer.c:37-63
      // no mass-action terms: the instances are resolved against the
      // aerosol representation at solver_initialize (both layouts hold
      // 4 + 13 n ints before the element lists)
      const int na = ints[0];
      if (na < 1 || n_int < 4 + 13 * na) return fail(malformed);
      if (ints[1] < 1 || ints[1] > n_state_)
        return fail("species index out of range in reaction " + std::to_string(idx));
      break;
    }
    case RXN_AQUEOUS_EQUILIBRIUM: {  // src/rxns/rxn_aqueous_equilibrium.c:27-56
      // resolved into instances at solver_initialize
      const int nr = ints[0], np = ints[1], P = ints[2], ns = nr + np;
      if (nr < 1 || np < 1 || P < 1 || n_int < 3 + P * (ns * (ns + 4) + 2) ||
          n_float < 5 + 2 * ns + 2 * P)
        return fail(malformed);
      for (int x = 0; x < P * (ns + 2); ++x) {  // reactants, products, water, activity
        const int sp = ints[3 + x];
        const bool act = x >= P * (ns + 1);
        if (act && sp == 0) continue;  // no ion pair
        if (sp < 1 || sp > n_state_)
          return fail("species index out of range in reaction " + std::to_string(idx));
      }
      break;
    }
    default: {  // NUM_REACT_ NUM_PROD_ [RXN_ID_] REACT_ PROD_ DERIV_ID_ JAC_ID_, yields
      const int nr = ints[0], np = ints[1];
      if (nr < 1 || np < 0 || n_int < r.n_int_prop + (nr + 2) * (nr + np) ||
          n_float < r.n_float_prop + np)
        return fail(malformed);
      Term t;
      const int p = r.n_int_prop;
      for (int k = 0; k < nr; ++k) t.react.push_back(ints[p + k] - 1);
      for (int k = 0; k < np; ++k) {
        t.prod.push_back(ints[p + nr + k] - 1);
        t.yield.push_back(floats[r.n_float_prop + k]);
      }
      for (int k = 0; k < nr + np; ++k) t.deriv_at.push_back(o + p + nr + np + k);
      for (int e = 0; e < nr * (nr + np); ++e) t.jac_at.push_back(o + p + 2 * (nr + np) + e);
      r.terms.push_back(t);
      if (type == RXN_PHOTOLYSIS) r.rid_at = o + 2;
    }
  }
  for (const Term& t : r.terms) {
    for (int sp : t.react)
      if (sp < 0 || sp >= n_state_) return fail("species index out of range in reaction " + std::to_string(idx));
    for (int sp : t.prod)
      if (sp < 0 || sp >= n_state_) return fail("species index out of range in reaction " + std::to_string(idx));
  }
  n_terms_ += (int)r.terms.size();
  rxns_.push_back(r);
  return true;
}

int Model::photo_id(int rxn) const {
  const Rxn& r = rxns_[rxn];
  return host_rate_type(r.type) && r.rid_at >= 0 ? rxn_int_[r.rid_at] : 0;
}

bool Model::add_aero_phase(int n_int, int n_float, const int* ints, const double* floats,
                           std::string* err) {
  // [NUM_STATE_VAR, SPEC_TYPE(x)], floats [MW(x), DENSITY(x)]
  // (src/aero_phase_solver.c:25-32)
  if (n_int < 1 || ints[0] < 0 || n_int < 1 + ints[0] || n_float < 2 * ints[0]) {
    *err = "malformed aerosol phase data";
    return false;
  }
  aph_int_.emplace_back(ints, ints + n_int);
  aph_flt_.emplace_back(floats, floats + n_float);
  return true;
}

bool Model::add_aero_rep(int type, int n_int, int n_float, int n_env, const int* ints,
                         const double* floats, std::string* err) {
  if (type != AERO_REP_MODAL_BINNED_MASS) {
    *err = "aerosol representation type " + std::to_string(type) +
           " is not supported (modal/binned mass only)";
    return false;
  }
  // NUM_SECTION_ INT_DATA_SIZE_ FLOAT_DATA_SIZE_ AERO_REP_ID_, section
  // locations, then per section its type, bins, phases and phase ids
  // (src/aero_reps/aero_rep_modal_binned_mass.c:28-84)
  if (n_int < 4 || ints[0] < 1 || n_int < 4 + 2 * ints[0] || n_env != 2 * ints[0]) {
    *err = "malformed aerosol representation data";
    return false;
  }
  const int ns = ints[0];
  for (int x = 0; x < ns; ++x) {
    const int li = ints[4 + x] - 1, lf = ints[4 + ns + x] - 1;
    if (li < 0 || li + 3 > n_int || lf < 0) {
      *err = "malformed aerosol representation data";
      return false;
    }
    const int nb = ints[li + 1], np = ints[li + 2];
    if (nb < 1 || np < 1 || li + 3 + 3 * nb * np > n_int || lf + 3 * nb > n_float) {
      *err = "malformed aerosol representation data";
      return false;
    }
    if (ints[li] == SECTION_MODAL) modes_.push_back({(int)arep_int_.size(), x});
  }
  arep_int_.emplace_back(ints, ints + n_int);
  arep_flt_.emplace_back(floats, floats + n_float);
  arep_type_.push_back(type);
  return true;
}

int Model::aero_column(int rep_id, int section, int what) const {
  if (what != 0 && what != 1) return -1;
  for (size_t k = 0; k < modes_.size(); ++k) {
    const auto& I = arep_int_[modes_[k].first];
    if (I[3] == rep_id && rep_id != 0 && modes_[k].second == section)
      return n_host_rate_ + 2 * (int)k + what;
  }
  return -1;
}

namespace {
// views of the packed SIMPOL data, 0-based within the reaction's ints
// (src/rxns/rxn_SIMPOL_phase_transfer.c:37-78)
struct SimpolView {
  int* I;
  int n;
  int gas() const { return I[1] - 1; }
  int aero(int x) const { return I[2 + x] - 1; }
  int act(int x) const { return I[2 + n + x] - 1; }
  int phase(int x) const { return I[2 + 2 * n + x] - 1; }
  int rep(int x) const { return I[2 + 3 * n + x] - 1; }
  int& deriv(int x) const { return I[2 + 4 * n + x]; }
  int& gas_act_jac(int x) const { return I[3 + 5 * n + x]; }
  int& aero_act_jac(int x) const { return I[3 + 6 * n + x]; }
  int& jac(int x) const { return I[3 + 7 * n + x]; }
  int iloc(int x) const { return I[4 + 10 * n + x] - 1; }
  int nelem(int x) const { return I[iloc(x)]; }
  int& phase_jac(int x, int set, int e) const { return I[iloc(x) + 1 + set * nelem(x) + e]; }
};
// views of the packed HL data, 0-based within the reaction's ints
// (src/rxns/rxn_HL_phase_transfer.c:37-63)
struct HlView {
  int* I;
  int n;
  int gas() const { return I[1] - 1; }
  int& deriv(int x) const { return I[2 + x]; }
  int& jac(int x) const { return I[3 + n + x]; }
  int iloc(int x) const { return I[4 + 6 * n + x] - 1; }
  int aero(int x) const { return I[iloc(x)] - 1; }
  int water(int x) const { return I[iloc(x) + 1] - 1; }
  int phase(int x) const { return I[iloc(x) + 2] - 1; }
  int rep(int x) const { return I[iloc(x) + 3] - 1; }
  int nelem(int x) const { return I[iloc(x) + 4]; }
  int& phase_jac(int x, int set, int e) const { return I[iloc(x) + 5 + set * nelem(x) + e]; }
};
// views of the packed aqueous equilibrium data, 0-based within the
// reaction's ints and floats (src/rxns/rxn_aqueous_equilibrium.c:27-56)
struct AqView {
  int* I;
  const double* F;
  int nr() const { return I[0]; }
  int np() const { return I[1]; }
  int P() const { return I[2]; }
  int react(int x) const { return I[3 + x] - 1; }
  int prod(int x) const { return I[3 + nr() * P() + x] - 1; }
  int water(int x) const { return I[3 + (nr() + np()) * P() + x] - 1; }
  int act(int x) const { return I[3 + (nr() + np() + 1) * P() + x] - 1; }
  int& deriv(int x) const { return I[3 + (nr() + np() + 2) * P() + x]; }
  int& jac(int x) const { return I[3 + (2 * (nr() + np()) + 2) * P() + x]; }
  double m2m(int x) const { return F[5 + x]; }
};
}  // namespace

// Aqueous equilibrium instances (one per phase instance of a reaction).
// The water and the ion pair's activity coefficient must be constant
// species: the reference's partials over them
// (src/rxns/rxn_aqueous_equilibrium.c:497-540) then fall outside the solver
// Jacobian, and per cell they are constants.
bool Model::resolve_aq(std::string* err) {
  aq_.clear();
  for (size_t ri = 0; ri < rxns_.size(); ++ri) {
    const Rxn& r = rxns_[ri];
    if (r.type != RXN_AQUEOUS_EQUILIBRIUM) continue;
    AqView v{&rxn_int_[r.int_off], &rxn_float_[r.float_off]};
    for (int p = 0; p < v.P(); ++p) {
      AqInst q;
      q.rxn = (int)ri;
      q.p = p;
      for (int i = 0; i < v.nr(); ++i) q.react.push_back(v.react(p * v.nr() + i));
      for (int i = 0; i < v.np(); ++i) q.prod.push_back(v.prod(p * v.np() + i));
      for (int i = 0; i < v.nr() + v.np(); ++i) q.m2m.push_back(v.m2m(i));
      q.water = v.water(p);
      q.act = v.act(p);
      q.A = v.F[0];
      q.C = v.F[1];
      q.kr = v.F[2];
      if (var_type_[q.water] == VAR_VARIABLE || (q.act >= 0 && var_type_[q.act] == VAR_VARIABLE)) {
        *err = "aqueous equilibrium reaction " + std::to_string(ri) +
               ": the aerosol-phase water and the ion pair must be constant (not variable) "
               "state variables";
        return false;
      }
      q.thr = abs_tol_.empty() ? 0.0 : 1.0e-4 * (abs_tol_[q.water] / 10.0);
      q.water_cv = cv_of_[q.water];
      q.act_cv = q.act >= 0 ? cv_of_[q.act] : -1;
      for (int pass = 0; pass < 2; ++pass) {
        const std::vector<int>& list = pass == 0 ? q.react : q.prod;
        for (size_t i = 0; i < list.size(); ++i) {
          if (cv_of_[list[i]] < 0) continue;
          q.cp_state.push_back(list[i]);
          q.cp_cv.push_back(cv_of_[list[i]]);
          q.cp_m.push_back(q.m2m[(pass == 0 ? 0 : q.react.size()) + i]);
          q.cp_r.push_back(pass == 0 ? 1 : 0);
        }
      }
      aq_.push_back(q);
    }
  }
  return true;
}

// Locates phase instance `phase` of representation si->rep the way the
// representation's C functions walk it (sections, then bins, then the phases
// of a bin, src/aero_reps/aero_rep_modal_binned_mass.c:300-330) and fills
// the section, bin, mode columns and element list of si; the element counts
// are written into the representation as its get_used_jac_elem does
// (:86-125).
bool Model::resolve_instance(SimpolInst* si, int phase, int ri, std::string* err) {
  const std::string what = (si->type == RXN_HL_PHASE_TRANSFER ? "HL reaction " : "SIMPOL reaction ") +
                           std::to_string(ri);
  if (si->rep < 0 || si->rep >= (int)arep_int_.size()) {
    *err = what + " names a missing aerosol representation";
    return false;
  }
  std::vector<int>& R = arep_int_[si->rep];
  const std::vector<double>& RF = arep_flt_[si->rep];
  const int ns = R[0];
  int idx = phase, found = 0;
  for (int s = 0; s < ns && !found; ++s) {
    const int li = R[4 + s] - 1;
    for (int b = 0; b < R[li + 1] && !found; ++b) {
      if (idx < R[li + 2]) {
        si->section = s;
        si->bin = b;
        si->phase = idx;
        found = 1;
      } else {
        idx -= R[li + 2];
      }
    }
  }
  if (!found) {
    *err = what + " names a missing phase instance";
    return false;
  }
  const int li = R[4 + si->section] - 1, lf = R[4 + ns + si->section] - 1;
  const int nb = R[li + 1], np = R[li + 2];
  si->kind = R[li];
  si->n_phases = np;
  si->bin_dp = RF[lf + 3 * si->bin];
  if (si->kind == SECTION_MODAL) {
    int k = 0;
    for (; k < (int)modes_.size(); ++k)
      if (modes_[k].first == si->rep && modes_[k].second == si->section) break;
    si->gmd_col = n_host_rate_ + 2 * k;
    si->gsd_col = si->gmd_col + 1;
  }
  for (int y = 0; y < np; ++y) {
    const int st0 = R[li + 3 + si->bin * np + y] - 1;
    const int ph = R[li + 3 + nb * np + si->bin * np + y] - 1;
    if (ph < 0 || ph >= (int)aph_int_.size()) {
      *err = "aerosol representation names a missing phase";
      return false;
    }
    const std::vector<int>& P = aph_int_[ph];
    const std::vector<double>& PF = aph_flt_[ph];
    int cnt = 0;
    for (int i = 0; i < P[0]; ++i) {
      const int t = P[1 + i];
      if (t != VAR_VARIABLE && t != VAR_CONSTANT && t != 3) continue;
      si->elem.push_back(st0 + i);
      si->inv_rho.push_back(1.0 / PF[P[0] + i]);
      si->inv_mw.push_back(y == si->phase ? 1.0 / PF[i] : 0.0);
      si->in_phase.push_back(y == si->phase ? 1 : 0);
      ++cnt;
    }
    R[li + 3 + 2 * nb * np + si->bin * np + y] = cnt;  // PHASE_NUM_JAC_ELEM_
  }
  for (int sp : {si->gas, si->aero})
    if (sp < 0 || sp >= n_state_ || var_type_[sp] != VAR_VARIABLE) {
      *err = what + ": the gas and aerosol species must be variable state variables";
      return false;
    }
  if (si->type == RXN_HL_PHASE_TRANSFER) {
    si->water_cv = si->water >= 0 && si->water < n_state_ ? cv_of_[si->water] : -1;
  } else {
    // a SIMPOL rate whose mode volume, phase mass or activity follows a
    // sub-model's output would need those partials chained as well
    bool computed = si->act >= 0 && si->act < n_state_ && cv_of_[si->act] >= 0;
    for (int e : si->elem) computed |= cv_of_[e] >= 0;
    if (computed) {
      *err = what + ": partitioning into a mode or bin that holds a species computed by a "
                    "sub-model is not supported";
      return false;
    }
  }
  return true;
}

// The instances of every SIMPOL and HL reaction against their
// representation, in mechanism order, with the state indices of their
// elements written into PHASE_JAC_ID_ as get_used_jac_elem does
// (src/rxns/rxn_SIMPOL_phase_transfer.c:86-151,
// src/rxns/rxn_HL_phase_transfer.c:72-138).
bool Model::resolve_simpol(std::string* err) {
  simpol_.clear();
  for (size_t ri = 0; ri < rxns_.size(); ++ri) {
    const Rxn& r = rxns_[ri];
    if (r.type == RXN_SIMPOL_PHASE_TRANSFER) {
      SimpolView v{&rxn_int_[r.int_off], rxn_int_[r.int_off]};
      for (int x = 0; x < v.n; ++x) {
        SimpolInst si;
        si.type = RXN_SIMPOL_PHASE_TRANSFER;
        si.rxn = (int)ri;
        si.x = x;
        for (int q = 0; q < 10; ++q) si.prm[q] = rxn_float_[r.float_off + q];
        si.gas = v.gas();
        si.aero = v.aero(x);
        si.act = v.act(x);
        si.rep = v.rep(x);
        if (!resolve_instance(&si, v.phase(x), (int)ri, err)) return false;
        if ((int)si.elem.size() > v.nelem(x)) {
          *err = "SIMPOL reaction " + std::to_string(ri) + ": more Jacobian elements than packed";
          return false;
        }
        for (int e = 0; e < v.nelem(x); ++e) {
          const int val = e < (int)si.elem.size() ? si.elem[e] : -1;
          v.phase_jac(x, 0, e) = val;
          v.phase_jac(x, 1, e) = val;
        }
        if (si.act >= 0 && (si.act >= n_state_ || var_type_[si.act] == VAR_VARIABLE)) {
          *err = "SIMPOL reaction " + std::to_string(ri) +
                 ": a variable activity coefficient is not supported";
          return false;
        }
        simpol_.push_back(si);
      }
    } else if (r.type == RXN_HL_PHASE_TRANSFER) {
      HlView v{&rxn_int_[r.int_off], rxn_int_[r.int_off]};
      for (int x = 0; x < v.n; ++x) {
        SimpolInst si;
        si.type = RXN_HL_PHASE_TRANSFER;
        si.rxn = (int)ri;
        si.x = x;
        for (int q = 0; q < 8; ++q) si.prm[q] = rxn_float_[r.float_off + q];
        si.gas = v.gas();
        si.aero = v.aero(x);
        si.water = v.water(x);
        si.rep = v.rep(x);
        if (!resolve_instance(&si, v.phase(x), (int)ri, err)) return false;
        if ((int)si.elem.size() > v.nelem(x)) {
          *err = "HL reaction " + std::to_string(ri) + ": more Jacobian elements than packed";
          return false;
        }
        for (int e = 0; e < v.nelem(x); ++e) {
          const int val = e < (int)si.elem.size() ? si.elem[e] : -1;
          v.phase_jac(x, 0, e) = val;
          v.phase_jac(x, 1, e) = val;
        }
        // the water divides the evaporation rate; a water that the solver
        // integrates would need its own partials (:365-373), which this
        // build does not evaluate
        if (si.water < 0 || si.water >= n_state_ || var_type_[si.water] == VAR_VARIABLE) {
          *err = "HL reaction " + std::to_string(ri) +
                 ": the aerosol-phase water must be a constant (not variable) state variable";
          return false;
        }
        simpol_.push_back(si);
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// Sub-models: ZSR aerosol water and PD-FiTE activity
// ---------------------------------------------------------------------------
namespace {
// Packed layouts (ints after the type slot) of
// src/sub_models/sub_model_ZSR_aerosol_water.c:27-71 and
// src/sub_models/sub_model_PDFiTE.c:21-64: NUM_PHASE, GAS_WATER_ID
// (1-based), NUM_ION_PAIR, the two data sizes, the phases' first state ids
// (1-based), then per ion pair its int and float block locations (1-based).
// Species ids of an ion pair are relative to the phase's first state id.
struct SubView {
  const int* I;
  const double* F;
  int np() const { return I[0]; }
  int gw() const { return I[1] - 1; }
  int npair() const { return I[2]; }
  int phase(int p) const { return I[5 + p] - 1; }
  int il(int x) const { return I[5 + np() + x] - 1; }
  int fl(int x) const { return I[5 + np() + npair() + x] - 1; }
  // ZSR: 1 = Jacobson et al. (1996), 2 = EQSAM
  int ztype(int x) const { return I[il(x)]; }
  int zj_ncat(int x) const { return I[il(x) + 1]; }
  int zj_nan(int x) const { return I[il(x) + 2]; }
  int zj_cat(int x) const { return I[il(x) + 3]; }
  int zj_an(int x) const { return I[il(x) + 4]; }
  int zj_ny(int x) const { return I[il(x) + 5]; }
  int ze_nion(int x) const { return I[il(x) + 1]; }
  int ze_ion(int x, int k) const { return I[il(x) + 2 + np() + k]; }
  // PD-FiTE
  int pd_act(int x) const { return I[il(x)]; }
  int pd_ncat(int x) const { return I[il(x) + 1]; }
  int pd_nan(int x) const { return I[il(x) + 2]; }
  int pd_cat(int x) const { return I[il(x) + 3]; }
  int pd_an(int x) const { return I[il(x) + 4]; }
  int pd_ninter(int x) const { return I[il(x) + 5]; }
  int pd_nb(int x, int y) const { return I[il(x) + 6 + (1 + 2 * npair()) * np() + y]; }
  int pd_pair(int x, int y) const {
    return I[il(x) + 6 + (1 + 2 * npair()) * np() + pd_ninter(x) + y] - 1;
  }
  int pd_loc(int x, int y) const {
    return I[il(x) + 6 + (1 + 2 * npair()) * np() + 2 * pd_ninter(x) + y] - 1;
  }
};
constexpr int kZsrJacobson = 1, kZsrEqsam = 2;
}  // namespace

bool Model::add_sub_model(int type, int n_int, int n_float, int n_env, const int* ints,
                          const double* floats, std::string* err) {
  if (type != SUB_MODEL_ZSR_AEROSOL_WATER && type != SUB_MODEL_PDFITE) {
    *err = "sub-model type " + std::to_string(type) +
           " is not supported (ZSR aerosol water and PD-FiTE activity are)";
    return false;
  }
  if (n_int < 5 || n_env != 1) {
    *err = "sub-model data does not have the ZSR / PD-FiTE layout";
    return false;
  }
  sub_type_.push_back(type);
  sub_int_.emplace_back(ints, ints + n_int);
  sub_flt_.emplace_back(floats, floats + n_float);
  return true;
}

// The parameter-Jacobian elements of sub-model k, (computed species, the
// species it is computed from), in the order get_used_jac_elem registers
// them (src/sub_models/sub_model_ZSR_aerosol_water.c:81-129,
// src/sub_models/sub_model_PDFiTE.c:73-97).
template <typename Fn>
static void for_sub_elements(int type, const SubView& v, Fn fn) {
  for (int p = 0; p < v.np(); ++p) {
    const int w = v.phase(p);
    if (type == SUB_MODEL_ZSR_AEROSOL_WATER) {
      fn(w, v.gw());
      for (int x = 0; x < v.npair(); ++x) {
        if (v.ztype(x) == kZsrJacobson) {
          fn(w, w + v.zj_cat(x));
          fn(w, w + v.zj_an(x));
        } else if (v.ztype(x) == kZsrEqsam) {
          for (int k = 0; k < v.ze_nion(x); ++k) fn(w, w + v.ze_ion(x, k));
        }
      }
    } else {
      for (int x = 0; x < v.npair(); ++x) {
        const int g = w + v.pd_act(x);
        fn(g, v.gw());
        for (int y = 0; y < v.npair(); ++y) {
          fn(g, w + v.pd_cat(y));
          fn(g, w + v.pd_an(y));
        }
      }
    }
  }
}

// The species the sub-models write (src/sub_models/sub_model_ZSR_aerosol_
// water.c:228-230: every phase instance's water; src/sub_models/
// sub_model_PDFiTE.c:196-256: each ion pair's activity coefficient up to the
// first pair without interactions), in sub-model, phase and pair order.
// Their inputs must be variable species and they themselves not variable; a
// reaction may use them only where the device evaluates them per f and J:
// as the aqueous equilibrium's water and activity coefficient and as HL's
// aerosol-phase water.
bool Model::resolve_sub_models(std::string* err) {
  cv_state_.clear();
  cv_of_.assign(n_state_, -1);
  auto state_ok = [&](int s) { return s >= 0 && s < n_state_; };
  for (size_t k = 0; k < sub_type_.size(); ++k) {
    const SubView v{sub_int_[k].data(), sub_flt_[k].data()};
    const std::string what = std::string(sub_type_[k] == SUB_MODEL_PDFITE ? "PD-FiTE" : "ZSR") +
                             " sub-model " + std::to_string(k);
    bool bad = false;
    for_sub_elements(sub_type_[k], v, [&](int dep, int ind) {
      if (!state_ok(dep) || !state_ok(ind)) {
        bad = true;
        return;
      }
      if (var_type_[ind] != VAR_VARIABLE || var_type_[dep] == VAR_VARIABLE) bad = true;
    });
    if (bad) {
      *err = what + ": its inputs (gas-phase water, ions) must be variable species and the "
                    "species it computes not variable";
      return false;
    }
    for (int p = 0; p < v.np(); ++p) {
      std::vector<int> out;
      if (sub_type_[k] == SUB_MODEL_ZSR_AEROSOL_WATER) {
        out.push_back(v.phase(p));
      } else {
        for (int x = 0; x < v.npair() && v.pd_ninter(x) > 0; ++x)
          out.push_back(v.phase(p) + v.pd_act(x));
      }
      for (int s : out) {
        if (cv_of_[s] >= 0) {
          *err = what + ": state variable " + std::to_string(s) +
                 " is computed by more than one sub-model";
          return false;
        }
        cv_of_[s] = (int)cv_state_.size();
        cv_state_.push_back(s);
      }
    }
  }
  // mass-action terms cannot take a computed species
  for (const Rxn& r : rxns_)
    for (const Term& t : r.terms)
      for (int s : t.react)
        if (cv_of_[s] >= 0) {
          *err = "a gas-phase reaction uses a species that a sub-model computes";
          return false;
        }
  return true;
}

int Model::param_elem_id(int dep, int ind) const {
  for (int e = pj_colptr_[ind]; e < pj_colptr_[ind + 1]; ++e)
    if (pj_rowid_[e] == dep) return e;
  return -1;
}

// Parameter Jacobian (src/camp_solver.c:1520-1550, src/sub_model_solver.c:
// 25-104): the dummy element (0, 0), which the fold uses as the unit
// parameter, then every sub-model element.  The interdependence elements
// (a sub-model computed from another's output) do not arise: every input is
// a variable species (resolve_sub_models).
void Model::build_param_jacobian() {
  Registry reg(n_state_);
  reg.add(0, 0);
  Registry local(n_state_);
  for (size_t k = 0; k < sub_type_.size(); ++k) {
    const SubView v{sub_int_[k].data(), sub_flt_[k].data()};
    for_sub_elements(sub_type_[k], v, [&](int dep, int ind) { local.add(dep, ind); });
  }
  std::vector<int> lcp, lri;
  local.to_csc(&lcp, &lri);
  for (int ind = 0; ind < n_state_; ++ind)
    for (int e = lcp[ind]; e < lcp[ind + 1]; ++e) reg.add(lri[e], ind);
  reg.to_csc(&pj_colptr_, &pj_rowid_);
}

// Per computed species its program (SubProgram) with the parameter ids of
// its partials.
void Model::build_sub_programs() {
  Tables& t = tab_;
  t.cv.assign(cv_state_.size(), SubProgram{});
  for (size_t c = 0; c < cv_state_.size(); ++c) t.cv[c].state = cv_state_[c];
  for (size_t k = 0; k < sub_type_.size(); ++k) {
    const SubView v{sub_int_[k].data(), sub_flt_[k].data()};
    const int gw = v.gw();
    for (int p = 0; p < v.np(); ++p) {
      const int w = v.phase(p);
      if (sub_type_[k] == SUB_MODEL_ZSR_AEROSOL_WATER) {
        SubProgram& g = t.cv[cv_of_[w]];
        g.ints = {1, deriv_ids_[gw], v.npair()};
        for (int x = 0; x < v.npair(); ++x) {
          const double* F = v.F + v.fl(x);
          if (v.ztype(x) == kZsrJacobson) {
            const int c = w + v.zj_cat(x), a = w + v.zj_an(x);
            g.ints.insert(g.ints.end(), {kZsrJacobson, deriv_ids_[c], deriv_ids_[a], v.zj_ny(x),
                                         param_elem_id(w, gw), param_elem_id(w, c),
                                         param_elem_id(w, a)});
            g.flts.insert(g.flts.end(), {F[0], 1.0 / (v.zj_ncat(x) * F[1] * 1000.0),
                                         1.0 / (v.zj_nan(x) * F[2] * 1000.0)});
            for (int y = 0; y < v.zj_ny(x); ++y) g.flts.push_back(F[3 + y]);
          } else if (v.ztype(x) == kZsrEqsam) {
            g.ints.insert(g.ints.end(), {kZsrEqsam, v.ze_nion(x), param_elem_id(w, gw)});
            for (int i = 0; i < v.ze_nion(x); ++i) {
              const int s = w + v.ze_ion(x, i);
              g.ints.insert(g.ints.end(), {deriv_ids_[s], param_elem_id(w, s)});
            }
            g.flts.insert(g.flts.end(), {F[0] * 55.51 * 18.01 / F[2] / 1000.0, F[1]});
            for (int i = 0; i < v.ze_nion(x); ++i) g.flts.push_back(1.0 / F[3 + i]);
          } else {
            g.ints.push_back(0);  // unknown pair type: contributes nothing
          }
        }
      } else {
        for (int x = 0; x < v.npair() && v.pd_ninter(x) > 0; ++x) {
          const int gs = w + v.pd_act(x);
          SubProgram& g = t.cv[cv_of_[gs]];
          g.ints = {2, deriv_ids_[gw], v.npair(), x, v.pd_ninter(x), param_elem_id(gs, gw)};
          for (int j = 0; j < v.npair(); ++j) {
            const int c = w + v.pd_cat(j), a = w + v.pd_an(j);
            g.ints.insert(g.ints.end(), {deriv_ids_[c], deriv_ids_[a], v.pd_ncat(j) + v.pd_nan(j),
                                         param_elem_id(gs, c), param_elem_id(gs, a)});
            const double* F = v.F + v.fl(j);
            g.flts.insert(g.flts.end(), {1.0 / (F[0] * 1.0e6), 1.0 / (F[1] * 1.0e6)});
          }
          for (int y = 0; y < v.pd_ninter(x); ++y) {
            g.ints.insert(g.ints.end(), {v.pd_pair(x, y), v.pd_nb(x, y)});
            const double* F = v.F + v.pd_loc(x, y);
            g.flts.insert(g.flts.end(), {F[0], F[1]});
            for (int z = 0; z < v.pd_nb(x, y); ++z) g.flts.push_back(F[2 + z]);
          }
        }
      }
    }
  }
}

int Model::rxn_elem_id(int dep, int ind) const {
  for (int e = rj_colptr_[ind]; e < rj_colptr_[ind + 1]; ++e)
    if (rj_rowid_[e] == dep) return e;
  return -1;
}

// Diagonal of every state variable plus, per mass-action term, each
// (reactant, reactant) and (product, reactant) pair (src/camp_solver.c:
// 1445-1460 and the get_used_jac_elem functions, e.g.
// src/rxns/rxn_arrhenius.c:44-60, rxn_first_order_loss.c:37-46,
// rxn_wet_deposition.c:38-49; EMISSION registers none).
//
// A second registry keeps the live elements only: all of the above except
// HL's elements, whose partials are zero for the modal/binned
// representation.  The reference's solver Jacobian keeps them as stored
// zeros; the LU built here leaves them out.
void Model::build_rxn_jacobian() {
  Registry reg(n_state_), live(n_state_);
  auto add = [&](int dep, int ind, bool is_live) {
    reg.add(dep, ind);
    if (is_live) live.add(dep, ind);
  };
  for (int i = 0; i < n_state_; ++i) add(i, i, true);
  for (const Rxn& r : rxns_)
    for (const Term& t : r.terms)
      for (int ind : t.react) {
        for (int d : t.react) add(d, ind, true);
        for (int d : t.prod) add(d, ind, true);
      }
  // SIMPOL (src/rxns/rxn_SIMPOL_phase_transfer.c:86-151): gas and aerosol
  // species against each other, the activity coefficient and the elements;
  // HL (src/rxns/rxn_HL_phase_transfer.c:72-138): the same with the
  // aerosol-phase water in place of the activity coefficient
  for (const SimpolInst& si : simpol_) {
    const bool hl = si.type == RXN_HL_PHASE_TRANSFER;
    add(si.gas, si.gas, true);
    add(si.aero, si.gas, true);
    add(si.gas, si.aero, true);
    add(si.aero, si.aero, true);
    if (hl) {
      add(si.gas, si.water, true);
      add(si.aero, si.water, true);
    } else if (si.act > 0) {
      add(si.gas, si.act, true);
      add(si.aero, si.act, true);
    }
    for (int e : si.elem) {
      add(si.gas, e, !hl);
      add(si.aero, e, !hl);
    }
  }
  // aqueous equilibrium (src/rxns/rxn_aqueous_equilibrium.c:70-127): the
  // forward and reverse mass-action pairs, water and activity coefficient
  for (const AqInst& q : aq_) {
    for (const std::vector<int>* ind : {&q.react, &q.prod})
      for (int i : *ind) {
        for (int d : q.react) add(d, i, true);
        for (int d : q.prod) add(d, i, true);
      }
    for (int d : q.react) add(d, q.water, true);
    for (int d : q.prod) add(d, q.water, true);
    if (q.act < 0) continue;
    for (int d : q.react) add(d, q.act, true);
    for (int d : q.prod) add(d, q.act, true);
  }
  reg.to_csc(&rj_colptr_, &rj_rowid_);
  live.to_csc(&rl_colptr_, &rl_rowid_);
}

// DERIV_ID and JAC_ID written back into the packed ints, as rxn_update_ids
// does (src/camp_solver.c:1491-1503, src/rxns/rxn_arrhenius.c:71-91,
// rxn_first_order_loss.c:56-69, rxn_emission.c:52-62).
void Model::update_ids() {
  deriv_ids_.assign(n_state_, -1);
  for (int i = 0, d = 0; i < n_state_; ++i)
    if (var_type_[i] == VAR_VARIABLE) deriv_ids_[i] = d++;
  for (const Rxn& r : rxns_)
    for (const Term& t : r.terms) {
      int k = 0;
      for (int s : t.react) rxn_int_[t.deriv_at[k++]] = deriv_ids_[s];
      for (int s : t.prod) rxn_int_[t.deriv_at[k++]] = deriv_ids_[s];
      int e = 0;
      for (int ind : t.react) {
        for (int d : t.react) rxn_int_[t.jac_at[e++]] = rxn_elem_id(d, ind);
        for (int d : t.prod) rxn_int_[t.jac_at[e++]] = rxn_elem_id(d, ind);
      }
    }
  // SIMPOL (src/rxns/rxn_SIMPOL_phase_transfer.c:160-205)
  for (const Rxn& r : rxns_) {
    if (r.type != RXN_SIMPOL_PHASE_TRANSFER) continue;
    SimpolView v{&rxn_int_[r.int_off], rxn_int_[r.int_off]};
    const int g = v.gas();
    v.deriv(0) = deriv_ids_[g];
    for (int x = 0; x < v.n; ++x) v.deriv(x + 1) = deriv_ids_[v.aero(x)];
    int ij = 0;
    v.jac(ij++) = rxn_elem_id(g, g);
    for (int x = 0; x < v.n; ++x) {
      const int a = v.aero(x);
      v.jac(ij++) = rxn_elem_id(a, g);
      v.jac(ij++) = rxn_elem_id(g, a);
      v.jac(ij++) = rxn_elem_id(a, a);
      if (v.act(x) > 0) {
        v.gas_act_jac(x) = rxn_elem_id(g, v.act(x));
        v.aero_act_jac(x) = rxn_elem_id(a, v.act(x));
      } else {
        v.gas_act_jac(x) = -1;
        v.aero_act_jac(x) = -1;
      }
      for (int e = 0; e < v.nelem(x); ++e) {
        if (v.phase_jac(x, 0, e) > 0) v.phase_jac(x, 0, e) = rxn_elem_id(g, v.phase_jac(x, 0, e));
        if (v.phase_jac(x, 1, e) > 0) v.phase_jac(x, 1, e) = rxn_elem_id(a, v.phase_jac(x, 1, e));
      }
    }
  }
  // aqueous equilibrium (src/rxns/rxn_aqueous_equilibrium.c:132-209; the
  // small concentrations it also sets are kept per instance, AqInst::thr)
  for (const Rxn& r : rxns_) {
    if (r.type != RXN_AQUEOUS_EQUILIBRIUM) continue;
    AqView v{&rxn_int_[r.int_off], &rxn_float_[r.float_off]};
    const int nr = v.nr(), np = v.np();
    int id = 0, ij = 0;
    for (int p = 0; p < v.P(); ++p) {
      for (int i = 0; i < nr; ++i) v.deriv(id++) = deriv_ids_[v.react(p * nr + i)];
      for (int i = 0; i < np; ++i) v.deriv(id++) = deriv_ids_[v.prod(p * np + i)];
    }
    for (int p = 0; p < v.P(); ++p) {
      std::vector<int> dep;
      for (int i = 0; i < nr; ++i) dep.push_back(v.react(p * nr + i));
      for (int i = 0; i < np; ++i) dep.push_back(v.prod(p * np + i));
      for (int ind : dep)
        for (int d : dep) v.jac(ij++) = rxn_elem_id(d, ind);
      for (int d : dep) v.jac(ij++) = rxn_elem_id(d, v.water(p));
      for (int d : dep) v.jac(ij++) = v.act(p) < 0 ? -1 : rxn_elem_id(d, v.act(p));
    }
  }
  // HL (src/rxns/rxn_HL_phase_transfer.c:149-186; the small water
  // concentration it also sets, :188-193, is never read)
  for (const Rxn& r : rxns_) {
    if (r.type != RXN_HL_PHASE_TRANSFER) continue;
    HlView v{&rxn_int_[r.int_off], rxn_int_[r.int_off]};
    const int g = v.gas();
    v.deriv(0) = deriv_ids_[g];
    for (int x = 0; x < v.n; ++x) v.deriv(x + 1) = deriv_ids_[v.aero(x)];
    int ij = 0;
    v.jac(ij++) = rxn_elem_id(g, g);
    for (int x = 0; x < v.n; ++x) {
      const int a = v.aero(x), w = v.water(x);
      v.jac(ij++) = rxn_elem_id(a, g);
      v.jac(ij++) = rxn_elem_id(g, a);
      v.jac(ij++) = rxn_elem_id(a, a);
      v.jac(ij++) = rxn_elem_id(g, w);
      v.jac(ij++) = rxn_elem_id(a, w);
      for (int e = 0; e < v.nelem(x); ++e) {
        if (v.phase_jac(x, 0, e) > 0) v.phase_jac(x, 0, e) = rxn_elem_id(g, v.phase_jac(x, 0, e));
        if (v.phase_jac(x, 1, e) > 0) v.phase_jac(x, 1, e) = rxn_elem_id(a, v.phase_jac(x, 1, e));
      }
    }
  }
}

// Solver Jacobian (src/camp_solver.c:1559-1633): a variable row keeps the
// variable columns of the reaction Jacobian, and a non-variable column c
// maps to every variable species j of a parameter element (c, j), so that
// J[row][j] += J_rxn[row][c] * J_params[c][j].  The fold's map lists the
// terms in reaction-Jacobian order (src/camp_solver.c:1649-1681).
//
// The same over the live reaction elements gives the device's Jacobian, with
// the solver entry of each of its entries; there only computed species map
// (a constant species, or a registered activity coefficient that PD-FiTE
// never writes, has zero parameter partials).
void Model::build_solver_jacobian() {
  auto build = [&](const std::vector<int>& rcp, const std::vector<int>& rri, bool live,
                   std::vector<int>* colptr, std::vector<int>* rowid) {
    Registry reg(n_state_);
    for (int ind = 0; ind < n_state_; ++ind)
      for (int e = rcp[ind]; e < rcp[ind + 1]; ++e) {
        const int dep = rri[e];
        if (var_type_[dep] != VAR_VARIABLE) continue;
        if (var_type_[ind] == VAR_VARIABLE) {
          reg.add(dep, ind);
          continue;
        }
        if (live && cv_of_[ind] < 0) continue;
        for (int j = 0; j < n_state_; ++j)
          if (var_type_[j] == VAR_VARIABLE && param_elem_id(ind, j) != -1) reg.add(dep, j);
      }
    std::vector<int> cp, ri;
    reg.to_csc(&cp, &ri);
    colptr->assign(n_dep_ + 1, 0);
    for (int c = 0; c < n_state_; ++c)
      if (deriv_ids_[c] >= 0) (*colptr)[deriv_ids_[c]] = cp[c];
    (*colptr)[n_dep_] = (int)ri.size();
    rowid->resize(ri.size());
    for (size_t e = 0; e < ri.size(); ++e) (*rowid)[e] = deriv_ids_[ri[e]];
  };
  build(rj_colptr_, rj_rowid_, false, &sj_colptr_, &sj_rowid_);
  build(rl_colptr_, rl_rowid_, true, &dj_colptr_, &dj_rowid_);
  auto sj_id = [&](int dep, int ind) {
    const int r = deriv_ids_[dep], c = deriv_ids_[ind];
    for (int e = sj_colptr_[c]; e < sj_colptr_[c + 1]; ++e)
      if (sj_rowid_[e] == r) return e;
    return -1;
  };
  jac_map_.clear();
  for (int ind = 0; ind < n_state_; ++ind)
    for (int e = rj_colptr_[ind]; e < rj_colptr_[ind + 1]; ++e) {
      const int dep = rj_rowid_[e];
      if (var_type_[dep] != VAR_VARIABLE) continue;
      if (var_type_[ind] == VAR_VARIABLE) {
        jac_map_.insert(jac_map_.end(), {sj_id(dep, ind), e, 0});
        continue;
      }
      for (int j = 0; j < n_state_; ++j) {
        const int pid = param_elem_id(ind, j);
        if (pid != -1 && var_type_[j] == VAR_VARIABLE)
          jac_map_.insert(jac_map_.end(), {sj_id(dep, j), e, pid});
      }
    }
  dj_to_sj_.assign(dj_rowid_.size(), -1);
  for (int c = 0; c < n_dep_; ++c) {
    int q = sj_colptr_[c];
    for (int e = dj_colptr_[c]; e < dj_colptr_[c + 1]; ++e) {
      while (sj_rowid_[q] != dj_rowid_[e]) ++q;  // both columns sorted, live a subset
      dj_to_sj_[e] = q;
    }
  }
}

// Fixed elimination order for the per-cell LU of I - gamma*J: diagonal
// pivots chosen greedily by minimum Markowitz count (r-1)(c-1) over the
// remaining submatrix, lowest index on ties.  The reference factors with
// KLU (partial pivoting, BTF + AMD ordering), whose source is not in the
// reference tree; M = I - gamma*J of a chemical Jacobian has a unit diagonal
// plus -gamma*J, whose diagonal entries are loss terms (<= 0), so diagonal
// pivots are the natural static choice.  A zero or non-finite pivot is
// reported as a recoverable setup failure by the device code.
void Model::build_lu() {
  const int n = n_dep_;
  Tables& t = tab_;
  std::vector<std::vector<char>> P(n, std::vector<char>(n, 0));
  for (int c = 0; c < n; ++c)
    for (int e = dj_colptr_[c]; e < dj_colptr_[c + 1]; ++e) P[dj_rowid_[e]][c] = 1;
  for (int i = 0; i < n; ++i) P[i][i] = 1;
  std::vector<char> done(n, 0);
  std::vector<int> rc(n), cc(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (P[i][j]) {
        rc[i]++;
        cc[j]++;
      }
  t.lu_perm.assign(n, 0);
  t.lu_iperm.assign(n, 0);
  for (int k = 0; k < n; ++k) {
    long best = -1;
    int bi = -1;
    for (int i = 0; i < n; ++i) {
      if (done[i]) continue;
      long s = (long)(rc[i] - 1) * (long)(cc[i] - 1);
      if (best < 0 || s < best) {
        best = s;
        bi = i;
      }
    }
    done[bi] = 1;
    t.lu_perm[k] = bi;
    t.lu_iperm[bi] = k;
    // remove pivot row/column from the active counts, then add fill
    for (int j = 0; j < n; ++j)
      if (!done[j] && P[bi][j]) cc[j]--;
    for (int i = 0; i < n; ++i)
      if (!done[i] && P[i][bi]) rc[i]--;
    for (int i = 0; i < n; ++i) {
      if (done[i] || !P[i][bi]) continue;
      for (int j = 0; j < n; ++j)
        if (!done[j] && P[bi][j] && !P[i][j]) {
          P[i][j] = 1;
          rc[i]++;
          cc[j]++;
        }
    }
  }
  // row-wise storage in pivot order, columns ascending
  t.lu_rowptr.assign(n + 1, 0);
  t.lu_col.clear();
  t.lu_diag.assign(n, 0);
  std::vector<std::vector<int>> pos(n, std::vector<int>(n, -1));
  for (int pi = 0; pi < n; ++pi) {
    t.lu_rowptr[pi] = (int)t.lu_col.size();
    int oi = t.lu_perm[pi];
    for (int pj = 0; pj < n; ++pj) {
      if (!P[oi][t.lu_perm[pj]]) continue;
      if (pj == pi) t.lu_diag[pi] = (int)t.lu_col.size();
      pos[pi][pj] = (int)t.lu_col.size();
      t.lu_col.push_back(pj);
    }
  }
  t.lu_rowptr[n] = (int)t.lu_col.size();
  t.n_lu = (int)t.lu_col.size();
  // update lists: for L entry (i,k) at position q, pairs (u_kj, a_ij), j > k
  t.upd_ptr.assign(t.n_lu + 1, 0);
  t.upd_src.clear();
  t.upd_dst.clear();
  std::vector<long> row_work(n, 0);
  for (int i = 0; i < n; ++i)
    for (int q = t.lu_rowptr[i]; q < t.lu_rowptr[i + 1]; ++q) {
      t.upd_ptr[q] = (int)t.upd_src.size();
      int k = t.lu_col[q];
      if (k >= i) continue;
      for (int p = t.lu_diag[k] + 1; p < t.lu_rowptr[k + 1]; ++p) {
        int j = t.lu_col[p];
        t.upd_src.push_back(p);
        t.upd_dst.push_back(pos[i][j]);
      }
      row_work[i] += 1 + (t.lu_rowptr[k + 1] - t.lu_diag[k] - 1);
    }
  t.upd_ptr[t.n_lu] = (int)t.upd_src.size();
  // factor / forward-solve levels: row i after every row k with L(i,k) != 0
  std::vector<int> flev(n, 0), blev(n, 0);
  int nfl = 0, nbl = 0;
  for (int i = 0; i < n; ++i) {
    int lv = 0;
    for (int q = t.lu_rowptr[i]; q < t.lu_diag[i]; ++q) lv = std::max(lv, flev[t.lu_col[q]] + 1);
    flev[i] = lv;
    nfl = std::max(nfl, lv + 1);
  }
  for (int i = n - 1; i >= 0; --i) {
    int lv = 0;
    for (int q = t.lu_diag[i] + 1; q < t.lu_rowptr[i + 1]; ++q) lv = std::max(lv, blev[t.lu_col[q]] + 1);
    blev[i] = lv;
    nbl = std::max(nbl, lv + 1);
  }
  auto levels = [&](const std::vector<int>& lev, int nl, std::vector<int>* ptr,
                    std::vector<int>* rows) {
    ptr->assign(nl + 1, 0);
    rows->clear();
    for (int l = 0; l < nl; ++l) {
      (*ptr)[l] = (int)rows->size();
      std::vector<int> r;
      for (int i = 0; i < n; ++i)
        if (lev[i] == l) r.push_back(i);
      // heaviest rows first so a strided assignment spreads the work
      std::stable_sort(r.begin(), r.end(),
                       [&](int a, int b) { return row_work[a] > row_work[b]; });
      rows->insert(rows->end(), r.begin(), r.end());
    }
    (*ptr)[nl] = (int)rows->size();
  };
  levels(flev, nfl, &t.fl_ptr, &t.fl_rows);
  levels(blev, nbl, &t.bl_ptr, &t.bl_rows);
  t.n_flev = nfl;
  t.n_blev = nbl;
  build_level_schedules(pos, flev, nfl, blev, nbl);
}

namespace {
// Longest-processing-time split of weighted units over 32 lanes; returns the
// units in lane order and fills lane_ptr (33 entries, offsets from base).
std::vector<int> lane_order(const std::vector<long>& w, int base, std::vector<int>* lane_ptr) {
  const int lanes = 32;
  std::vector<int> idx(w.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return w[a] > w[b]; });
  std::vector<long> load(lanes, 0);
  std::vector<std::vector<int>> per(lanes);
  for (int i : idx) {
    int best = 0;
    for (int l = 1; l < lanes; ++l)
      if (load[l] < load[best]) best = l;
    per[best].push_back(i);
    load[best] += w[i];
  }
  std::vector<int> out;
  for (int l = 0; l < lanes; ++l) {
    lane_ptr->push_back(base + (int)out.size());
    out.insert(out.end(), per[l].begin(), per[l].end());
  }
  lane_ptr->push_back(base + (int)out.size());
  return out;
}

// Appends one level of a grouped phase: targets with their pair lists.
void add_grouped_level(Tables::Grouped* g, const std::vector<int>& targets,
                       const std::vector<std::vector<std::pair<int, int>>>& pairs,
                       const std::vector<int>* recip = nullptr) {
  std::vector<long> w(targets.size());
  for (size_t u = 0; u < targets.size(); ++u) w[u] = 2 + (long)pairs[u].size();
  int base = (int)g->unit_target.size();
  std::vector<int> order = lane_order(w, base, &g->lane_ptr);
  for (int u : order) {
    g->unit_target.push_back(targets[u]);
    g->unit_begin.push_back((int)g->pair_a.size());
    g->unit_count.push_back((int)pairs[u].size());
    g->unit_recip.push_back(recip ? (*recip)[u] : 0);
    for (auto& pr : pairs[u]) {
      g->pair_a.push_back(pr.first);
      g->pair_b.push_back(pr.second);
    }
  }
  g->n_levels++;
}
}  // namespace

// Level schedules of the factorization and the triangular solves.
void Model::build_level_schedules(const std::vector<std::vector<int>>& pos,
                                  const std::vector<int>& flev, int nfl,
                                  const std::vector<int>& blev, int nbl) {
  Tables& t = tab_;
  const int n = n_dep_;
  auto has = [&](int i, int j) { return pos[i][j] >= 0; };
  // pivot k depends on k' < k when k' updates row k or column k
  std::vector<int> plev(n, 0);
  int npl = 0;
  for (int k = 0; k < n; ++k) {
    int lv = 0;
    for (int kk = 0; kk < k; ++kk)
      if (has(k, kk) || has(kk, k)) lv = std::max(lv, plev[kk] + 1);
    plev[k] = lv;
    npl = std::max(npl, lv + 1);
  }
  t.n_plev = npl;
  t.fa_ptr.assign(1, 0);
  t.fa_pos.clear();
  t.fa_piv.clear();
  t.fb = Tables::Grouped();
  // Grouped factor phase g (0..npl): g = 0 holds the reciprocals of the
  // level-0 pivots; g = l+1 holds the Schur updates of level l and the
  // reciprocals of the level-(l+1) pivots.  A pivot's reciprocal is taken by
  // the unit that last updates its diagonal in that phase, or by a unit of
  // its own when the diagonal was already final.  Unit targets are LU
  // positions; recip holds the pivot + 1 whose reciprocal the unit takes.
  auto emit_phase = [&](int g) {
    // Schur updates of level g-1
    std::vector<int> targets, recip;
    std::vector<std::vector<std::pair<int, int>>> pairs;
    std::vector<std::vector<int>> slot(n, std::vector<int>(n, -1));
    if (g > 0) {
      const int l = g - 1;
      for (int k = 0; k < n; ++k) {
        if (plev[k] != l) continue;
        for (int i = k + 1; i < n; ++i) {
          if (!has(i, k)) continue;
          for (int j = k + 1; j < n; ++j) {
            if (!has(k, j)) continue;
            int& sl = slot[i][j];
            if (sl < 0) {
              sl = (int)targets.size();
              targets.push_back(pos[i][j]);
              recip.push_back(0);
              pairs.emplace_back();
            }
            pairs[sl].push_back({pos[i][k], pos[k][j]});
          }
        }
      }
    }
    // reciprocals of the pivots of level g
    for (int k = 0; k < n; ++k) {
      if (plev[k] != g) continue;
      int sl = slot[k][k];
      if (sl >= 0) {
        recip[sl] = k + 1;
      } else {
        targets.push_back(pos[k][k]);
        recip.push_back(k + 1);
        pairs.emplace_back();
      }
    }
    add_grouped_level(&t.fb, targets, pairs, &recip);
  };
  for (int g = 0; g <= npl; ++g) {
    emit_phase(g);
    if (g == npl) break;
    for (int k = 0; k < n; ++k)
      if (plev[k] == g)
        for (int i = k + 1; i < n; ++i)
          if (has(i, k)) {
            t.fa_pos.push_back(pos[i][k]);
            t.fa_piv.push_back(k);
          }
    t.fa_ptr.push_back((int)t.fa_pos.size());
  }
  // forward substitution by forward levels: z_i -= l_ik z_k, k in the level
  t.fwd = Tables::Grouped();
  for (int l = 0; l < nfl; ++l) {
    std::vector<int> targets;
    std::vector<std::vector<std::pair<int, int>>> pairs;
    std::vector<int> slot(n, -1);
    for (int k = 0; k < n; ++k) {
      if (flev[k] != l) continue;
      for (int i = k + 1; i < n; ++i) {
        if (!has(i, k)) continue;
        if (slot[i] < 0) {
          slot[i] = (int)targets.size();
          targets.push_back(i);
          pairs.emplace_back();
        }
        pairs[slot[i]].push_back({pos[i][k], k});
      }
    }
    add_grouped_level(&t.fwd, targets, pairs);
  }
  // backward substitution in nbl phases: phase g applies z_i -= u_ik z_k for
  // the pivots k of level g-1 and finalises (z_k *= 1/u_kk) the pivots of
  // level g, each by the unit that last updates it or by a unit of its own
  t.bwd = Tables::Grouped();
  for (int g = 0; g < nbl; ++g) {
    std::vector<int> targets, fin;
    std::vector<std::vector<std::pair<int, int>>> pairs;
    std::vector<int> slot(n, -1);
    if (g > 0)
      for (int k = 0; k < n; ++k) {
        if (blev[k] != g - 1) continue;
        for (int i = 0; i < k; ++i) {
          if (!has(i, k)) continue;
          if (slot[i] < 0) {
            slot[i] = (int)targets.size();
            targets.push_back(i);
            fin.push_back(0);
            pairs.emplace_back();
          }
          pairs[slot[i]].push_back({pos[i][k], k});
        }
      }
    for (int k = 0; k < n; ++k) {
      if (blev[k] != g) continue;
      if (slot[k] >= 0) {
        fin[slot[k]] = k + 1;
      } else {
        targets.push_back(k);
        fin.push_back(k + 1);
        pairs.emplace_back();
      }
    }
    add_grouped_level(&t.bwd, targets, pairs, &fin);
  }
}

void Model::build_tables() {
  Tables& t = tab_;
  t.n = n_dep_;
  t.n_state = n_state_;
  t.n_rxn = n_terms_;
  t.n_jac = (int)dj_rowid_.size();
  t.dep_state.clear();
  for (int i = 0; i < n_state_; ++i)
    if (var_type_[i] == VAR_VARIABLE) t.dep_state.push_back(i);
  // rate laws and reactants, one entry per mass-action term; a reaction's
  // terms share its float head block and host-rate column
  t.rx_type.clear(); t.rx_nreact.clear(); t.rx_fpar.clear(); t.rx_photo.clear();
  t.fpar.clear();
  t.rx_cptr.assign(1, 0); t.rx_cidx.clear();
  t.rx_vptr.assign(1, 0); t.rx_vdep.clear();
  for (int ri = 0; ri < n_rxn_; ++ri) {
    const Rxn& r = rxns_[ri];
    const int fpar0 = (int)t.fpar.size();
    for (int k = 0; k < r.n_float_prop; ++k) t.fpar.push_back(rxn_float_[r.float_off + k]);
    for (const Term& tm : r.terms) {
      t.rx_type.push_back(r.type);
      t.rx_nreact.push_back((int)tm.react.size());
      t.rx_fpar.push_back(fpar0);
      t.rx_photo.push_back(photo_slot_[ri]);
      for (int s : tm.react) {
        if (var_type_[s] == VAR_VARIABLE)
          t.rx_vdep.push_back(deriv_ids_[s]);
        else
          t.rx_cidx.push_back(s);
      }
      t.rx_cptr.push_back((int)t.rx_cidx.size());
      t.rx_vptr.push_back((int)t.rx_vdep.size());
    }
  }
  t.n_photo = n_host_rate();
  t.n_part = (int)t.rx_vdep.size();
  // SIMPOL and HL instances: 4 pseudo-rates each after the terms' rates, 8
  // per-cell constants after the terms' rate constants, and their Jacobian
  // partials (4, plus 4 per dependent element for SIMPOL) after the terms'
  // partials
  t.simpol = simpol_;
  t.n_simpol = (int)simpol_.size();
  t.n_rates = t.n_rxn + 4 * t.n_simpol;
  t.n_keff = t.n_rxn + 8 * t.n_simpol;
  t.si_part0.clear();
  int n_part_all = t.n_part;
  for (const SimpolInst& si : simpol_) {
    t.si_part0.push_back(n_part_all);
    int nd = 0;
    if (si.type == RXN_SIMPOL_PHASE_TRANSFER)
      for (int e : si.elem) nd += var_type_[e] == VAR_VARIABLE;
    // HL with a computed water: the gas and aerosol rows against it
    n_part_all += 4 + 4 * nd + (si.water_cv >= 0 ? 2 : 0);
  }
  // aqueous equilibrium instances: 3 per-cell constants (forward, reverse,
  // minimum water) after the SIMPOL constants, a loss and a gain pseudo-rate
  // per dependent species slot after the SIMPOL pseudo-rates, per dependent
  // independent slot a partial for every dependent row slot, then per row
  // slot its partial against a computed water and against a computed
  // activity coefficient
  t.aq = aq_;
  t.n_aq = (int)aq_.size();
  t.aq_keff0.clear();
  t.aq_rate0.clear();
  t.aq_part0.clear();
  for (const AqInst& q : aq_) {
    int S = 0;
    for (int sp : q.react) S += var_type_[sp] == VAR_VARIABLE;
    for (int sp : q.prod) S += var_type_[sp] == VAR_VARIABLE;
    t.aq_keff0.push_back(t.n_keff);
    t.n_keff += 3;
    t.aq_rate0.push_back(t.n_rates);
    t.n_rates += 2 * S;
    t.aq_part0.push_back(n_part_all);
    n_part_all += S * S + S * (q.water_cv >= 0) + S * (q.act_cv >= 0) + S * (int)q.cp_cv.size();
  }
  t.n_part_all = n_part_all;
  // sub-models: computed species and their programs, PPM_TO_RH_ per cell
  build_sub_programs();
  t.n_cv = (int)cv_state_.size();
  t.n_pj = (int)pj_rowid_.size();
  t.sm_keff = -1;
  if (t.n_cv > 0) t.sm_keff = t.n_keff++;
  // f gather: per dependent species, in term order, reactant occurrences
  // (loss, coefficient -1) before products (coefficient yield)
  std::vector<std::vector<int>> frx(n_dep_), fpr(n_dep_);
  std::vector<std::vector<double>> fco(n_dep_);
  {
    int ti = 0, ks = 0, ka = 0;
    for (size_t ri = 0; ri < rxns_.size(); ++ri) {
      const Rxn& r = rxns_[ri];
      for (const Term& tm : r.terms) {
        int k = 0;
        for (size_t j = 0; j < tm.react.size(); ++j) {
          const int d = rxn_int_[tm.deriv_at[k++]];
          if (d < 0) continue;
          frx[d].push_back(ti); fco[d].push_back(-1.0); fpr[d].push_back(FG_LOSS);
        }
        for (size_t j = 0; j < tm.prod.size(); ++j) {
          const int d = rxn_int_[tm.deriv_at[k++]];
          if (d < 0) continue;
          frx[d].push_back(ti); fco[d].push_back(tm.yield[j]);
          fpr[d].push_back(tm.source ? FG_SOURCE : FG_PRODUCT);
        }
        ++ti;
      }
      // SIMPOL and HL at their place in the mechanism: the gas gains
      // evaporation and loses condensation, the aerosol species the reverse
      // (src/rxns/rxn_SIMPOL_phase_transfer.c:414-446,
      // src/rxns/rxn_HL_phase_transfer.c:323-339)
      for (; ks < t.n_simpol && simpol_[ks].rxn == (int)ri; ++ks) {
        const int base = t.n_rxn + 4 * ks;
        const int dg = deriv_ids_[simpol_[ks].gas], da = deriv_ids_[simpol_[ks].aero];
        frx[dg].push_back(base); fco[dg].push_back(1.0); fpr[dg].push_back(FG_SOURCE);
        frx[dg].push_back(base + 1); fco[dg].push_back(-1.0); fpr[dg].push_back(FG_LOSS);
        frx[da].push_back(base + 2); fco[da].push_back(-1.0); fpr[da].push_back(FG_LOSS);
        frx[da].push_back(base + 3); fco[da].push_back(1.0); fpr[da].push_back(FG_SOURCE);
      }
      // aqueous equilibrium: per dependent species slot its loss and gain
      // pseudo-rates (src/rxns/rxn_aqueous_equilibrium.c:361-390)
      for (; ka < t.n_aq && aq_[ka].rxn == (int)ri; ++ka) {
        int k = 0;
        for (const std::vector<int>* list : {&aq_[ka].react, &aq_[ka].prod})
          for (int sp : *list) {
            if (var_type_[sp] != VAR_VARIABLE) continue;
            const int d = deriv_ids_[sp], base = t.aq_rate0[ka] + 2 * k++;
            frx[d].push_back(base); fco[d].push_back(-1.0); fpr[d].push_back(FG_LOSS);
            frx[d].push_back(base + 1); fco[d].push_back(1.0); fpr[d].push_back(FG_SOURCE);
          }
      }
    }
  }
  t.fg_ptr.assign(n_dep_ + 1, 0);
  t.fg_rxn.clear(); t.fg_coef.clear(); t.fg_prod.clear();
  t.max_fgather = 0;
  for (int d = 0; d < n_dep_; ++d) {
    t.fg_ptr[d] = (int)t.fg_rxn.size();
    t.fg_rxn.insert(t.fg_rxn.end(), frx[d].begin(), frx[d].end());
    t.fg_coef.insert(t.fg_coef.end(), fco[d].begin(), fco[d].end());
    t.fg_prod.insert(t.fg_prod.end(), fpr[d].begin(), fpr[d].end());
    t.max_fgather = std::max(t.max_fgather, (int)frx[d].size());
  }
  t.fg_ptr[n_dep_] = (int)t.fg_rxn.size();
  // J gather: per solver Jacobian entry (column = independent species,
  // row = dependent species), in term order, for each variable independent
  // reactant occurrence: reactant rows (loss) then product rows
  std::vector<std::vector<int>> jpart(t.n_jac), jind(t.n_jac);
  std::vector<std::vector<double>> jco(t.n_jac);
  auto slot_of = [&](int row, int col) {
    for (int e = dj_colptr_[col]; e < dj_colptr_[col + 1]; ++e)
      if (dj_rowid_[e] == row) return e;
    return -1;
  };
  {
    int ti = 0;
    for (const Rxn& r : rxns_)
      for (const Term& tm : r.terms) {
        int kv = 0;
        for (int sind : tm.react) {
          if (var_type_[sind] != VAR_VARIABLE) continue;
          const int part = t.rx_vptr[ti] + kv++;
          const int cind = deriv_ids_[sind];
          for (int sd : tm.react) {
            if (var_type_[sd] != VAR_VARIABLE) continue;
            int e = slot_of(deriv_ids_[sd], cind);
            jpart[e].push_back(part); jco[e].push_back(-1.0); jind[e].push_back(-1);
          }
          for (size_t d = 0; d < tm.prod.size(); ++d) {
            const int sd = tm.prod[d];
            if (var_type_[sd] != VAR_VARIABLE) continue;
            int e = slot_of(deriv_ids_[sd], cind);
            jpart[e].push_back(part); jco[e].push_back(tm.yield[d]); jind[e].push_back(cind);
          }
        }
        ++ti;
      }
  }
  // SIMPOL and HL partials: losses (jg_ind -1) and unguarded productions
  // (-2) of the gas and aerosol rows against each other and, for SIMPOL,
  // every dependent element (src/rxns/rxn_SIMPOL_phase_transfer.c:615-744,
  // total-mass branch; src/rxns/rxn_HL_phase_transfer.c:412-439)
  for (int k = 0; k < t.n_simpol; ++k) {
    const SimpolInst& si = simpol_[k];
    const int p0 = t.si_part0[k];
    const int dg = deriv_ids_[si.gas], da = deriv_ids_[si.aero];
    auto add = [&](int row, int col, int part, bool loss) {
      int e = slot_of(row, col);
      jpart[e].push_back(part);
      jco[e].push_back(loss ? -1.0 : 1.0);
      jind[e].push_back(loss ? -1 : -2);
    };
    add(dg, dg, p0 + 0, true);
    add(da, dg, p0 + 1, false);
    add(dg, da, p0 + 2, false);
    add(da, da, p0 + 3, true);
    if (si.type != RXN_SIMPOL_PHASE_TRANSFER) continue;
    int j = 0;
    for (int es : si.elem) {
      if (var_type_[es] != VAR_VARIABLE) continue;
      const int de = deriv_ids_[es];
      add(dg, de, p0 + 4 + 4 * j, false);
      add(dg, de, p0 + 5 + 4 * j, true);
      add(da, de, p0 + 6 + 4 * j, true);
      add(da, de, p0 + 7 + 4 * j, false);
      ++j;
    }
  }
  // aqueous equilibrium partials: row slot b against independent slot a,
  // a loss where both are reactants or both products, else an unguarded
  // production (src/rxns/rxn_aqueous_equilibrium.c:436-479)
  for (int k = 0; k < t.n_aq; ++k) {
    const AqInst& q = aq_[k];
    std::vector<int> sd;
    std::vector<char> isr;
    for (int sp : q.react)
      if (var_type_[sp] == VAR_VARIABLE) sd.push_back(deriv_ids_[sp]), isr.push_back(1);
    for (int sp : q.prod)
      if (var_type_[sp] == VAR_VARIABLE) sd.push_back(deriv_ids_[sp]), isr.push_back(0);
    const int S = (int)sd.size(), p0 = t.aq_part0[k];
    for (int a = 0; a < S; ++a)
      for (int b = 0; b < S; ++b) {
        const bool loss = isr[a] == isr[b];
        const int e = slot_of(sd[b], sd[a]);
        jpart[e].push_back(p0 + a * S + b);
        jco[e].push_back(loss ? -1.0 : 1.0);
        jind[e].push_back(loss ? -1 : -2);
      }
  }
  // virtual slots: the live reaction-Jacobian elements of a variable row
  // against a computed species, ordered by column then row
  std::vector<int> vrow, vcol;
  std::vector<std::vector<int>> vpart;
  {
    auto vslot = [&](int dep_state, int cv_state) {
      for (size_t v = 0; v < vrow.size(); ++v)
        if (vrow[v] == dep_state && vcol[v] == cv_state) return (int)v;
      return -1;
    };
    for (int ind = 0; ind < n_state_; ++ind) {
      if (cv_of_[ind] < 0) continue;
      for (int e = rl_colptr_[ind]; e < rl_colptr_[ind + 1]; ++e)
        if (var_type_[rl_rowid_[e]] == VAR_VARIABLE) {
          vrow.push_back(rl_rowid_[e]);
          vcol.push_back(ind);
        }
    }
    vpart.assign(vrow.size(), {});
    // HL: the gas and aerosol rows against the computed water
    // (src/rxns/rxn_HL_phase_transfer.c:383-389, 398-404)
    for (int k = 0; k < t.n_simpol; ++k) {
      const SimpolInst& si = simpol_[k];
      if (si.water_cv < 0) continue;
      const int p0 = t.si_part0[k];
      vpart[vslot(si.gas, si.water)].push_back(p0 + 4);
      vpart[vslot(si.aero, si.water)].push_back(p0 + 5);
    }
    // aqueous equilibrium: every dependent row against the computed water
    // and activity coefficient (src/rxns/rxn_aqueous_equilibrium.c:486-537)
    for (int k = 0; k < t.n_aq; ++k) {
      const AqInst& q = aq_[k];
      std::vector<int> rows;
      for (const std::vector<int>* list : {&q.react, &q.prod})
        for (int sp : *list)
          if (var_type_[sp] == VAR_VARIABLE) rows.push_back(sp);
      const int S = (int)rows.size();
      int p = t.aq_part0[k] + S * S;
      if (q.water_cv >= 0)
        for (int b = 0; b < S; ++b) vpart[vslot(rows[b], q.water)].push_back(p++);
      if (q.act_cv >= 0)
        for (int b = 0; b < S; ++b) vpart[vslot(rows[b], q.act)].push_back(p++);
      // a computed reactant or product as an independent species
      // (src/rxns/rxn_aqueous_equilibrium.c:436-479)
      for (size_t j = 0; j < q.cp_state.size(); ++j)
        for (int b = 0; b < S; ++b) vpart[vslot(rows[b], q.cp_state[j])].push_back(p++);
    }
  }
  t.n_virt = (int)vrow.size();
  t.jv_ptr.assign(1, 0);
  t.jv_part.clear();
  t.jv_row.clear();
  for (int v = 0; v < t.n_virt; ++v) {
    t.jv_part.insert(t.jv_part.end(), vpart[v].begin(), vpart[v].end());
    t.jv_ptr.push_back((int)t.jv_part.size());
    t.jv_row.push_back(deriv_ids_[vrow[v]]);
  }
  // the chain, grouped by target device slot: V(row, c) * P(c, j) into
  // J(row, j) for every variable j of the computed species' parameter row
  {
    std::vector<std::vector<std::pair<int, int>>> by_slot(t.n_jac);
    for (int v = 0; v < t.n_virt; ++v)
      for (int j = 0; j < n_state_; ++j) {
        if (var_type_[j] != VAR_VARIABLE) continue;
        const int pid = param_elem_id(vcol[v], j);
        if (pid < 0) continue;
        by_slot[slot_of(deriv_ids_[vrow[v]], deriv_ids_[j])].push_back({v, pid});
      }
    t.ch_tgt.clear();
    t.ch_ptr.assign(1, 0);
    t.ch_v.clear();
    t.ch_p.clear();
    for (int e = 0; e < t.n_jac; ++e) {
      if (by_slot[e].empty()) continue;
      t.ch_tgt.push_back(e);
      for (const auto& vp : by_slot[e]) {
        t.ch_v.push_back(vp.first);
        t.ch_p.push_back(vp.second);
      }
      t.ch_ptr.push_back((int)t.ch_v.size());
    }
  }
  t.jg_ptr.assign(t.n_jac + 1, 0);
  t.jg_part.clear(); t.jg_coef.clear(); t.jg_ind.clear();
  t.jg_lupos.assign(t.n_jac, 0);
  t.jg_row.assign(t.n_jac, 0);
  for (int c = 0; c < n_dep_; ++c)
    for (int e = dj_colptr_[c]; e < dj_colptr_[c + 1]; ++e) {
      int pr = t.lu_iperm[dj_rowid_[e]], pc = t.lu_iperm[c];
      for (int q = t.lu_rowptr[pr]; q < t.lu_rowptr[pr + 1]; ++q)
        if (t.lu_col[q] == pc) t.jg_lupos[e] = q;
      t.jg_row[e] = dj_rowid_[e];
    }
  for (int e = 0; e < t.n_jac; ++e) {
    t.jg_ptr[e] = (int)t.jg_part.size();
    t.jg_part.insert(t.jg_part.end(), jpart[e].begin(), jpart[e].end());
    t.jg_coef.insert(t.jg_coef.end(), jco[e].begin(), jco[e].end());
    t.jg_ind.insert(t.jg_ind.end(), jind[e].begin(), jind[e].end());
  }
  t.jg_ptr[t.n_jac] = (int)t.jg_part.size();
}

bool Model::build(std::string* err) {
  if (n_added_ != n_rxn_) {
    *err = "solver_initialize called after " + std::to_string(n_added_) + " of " +
           std::to_string(n_rxn_) + " reactions were added";
    return false;
  }
  if (n_dep_ == 0) {
    *err = "no dependent (VARIABLE) state variables";
    return false;
  }
  if (!resolve_sub_models(err)) return false;
  if (!resolve_simpol(err)) return false;
  if (!resolve_aq(err)) return false;
  build_rxn_jacobian();
  update_ids();
  build_param_jacobian();
  build_solver_jacobian();
  build_lu();
  build_tables();
  built_ = true;
  return true;
}

}  // namespace campb
