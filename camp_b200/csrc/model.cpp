// Host-side mechanism model.  See model.hpp.
#include "model.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace campb {

namespace {
// NUM_INT_PROP_ / NUM_FLOAT_PROP_ of the gas types (src/rxns/rxn_*.c headers)
bool type_layout(int type, int* n_int_prop, int* n_float_prop) {
  switch (type) {
    case RXN_ARRHENIUS: *n_int_prop = 2; *n_float_prop = 6; return true;
    case RXN_TROE: *n_int_prop = 2; *n_float_prop = 10; return true;
    case RXN_CMAQ_H2O2: *n_int_prop = 2; *n_float_prop = 7; return true;
    case RXN_CMAQ_OH_HNO3: *n_int_prop = 2; *n_float_prop = 11; return true;
    case RXN_PHOTOLYSIS: *n_int_prop = 3; *n_float_prop = 1; return true;
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
  if (!type_layout(type, &r.n_int_prop, &r.n_float_prop)) {
    *err = "reaction type " + std::to_string(type) +
           " is not supported (gas-phase ARRHENIUS, TROE, CMAQ_H2O2, "
           "CMAQ_OH_HNO3 and PHOTOLYSIS only)";
    rxns_.push_back(r);
    ++n_added_;
    return false;
  }
  r.nr = n_int > 0 ? ints[0] : 0;
  r.np = n_int > 1 ? ints[1] : 0;
  int need_int = r.n_int_prop + (r.nr + 2) * (r.nr + r.np);
  int need_float = r.n_float_prop + r.np;
  rxns_.push_back(r);
  ++n_added_;
  if (r.nr < 1 || r.np < 0 || n_int < need_int || n_float < need_float) {
    *err = "malformed packed data for reaction " + std::to_string(n_added_ - 1);
    return false;
  }
  for (int k = 0; k < r.nr + r.np; ++k) {
    int s = ints[r.n_int_prop + k] - 1;
    if (s < 0 || s >= n_state_) {
      *err = "species index out of range in reaction " + std::to_string(n_added_ - 1);
      return false;
    }
  }
  return true;
}

int Model::photo_id(int rxn) const {
  const Rxn& r = rxns_[rxn];
  return r.type == RXN_PHOTOLYSIS ? rxn_int_[r.int_off + 2] : 0;
}

int Model::rxn_elem_id(int dep, int ind) const {
  for (int e = rj_colptr_[ind]; e < rj_colptr_[ind + 1]; ++e)
    if (rj_rowid_[e] == dep) return e;
  return -1;
}

#define REACT(r, x) (rxn_int_[(r).int_off + (r).n_int_prop + (x)] - 1)
#define PROD(r, x) (rxn_int_[(r).int_off + (r).n_int_prop + (r).nr + (x)] - 1)
#define DERIV_ID(r, x) rxn_int_[(r).int_off + (r).n_int_prop + (r).nr + (r).np + (x)]
#define JAC_ID(r, x) rxn_int_[(r).int_off + (r).n_int_prop + 2 * ((r).nr + (r).np) + (x)]
#define YIELD(r, x) rxn_float_[(r).float_off + (r).n_float_prop + (x)]

// Diagonal of every state variable plus, per reaction, each (reactant,
// reactant) and (product, reactant) pair (src/camp_solver.c:1445-1460 and
// the get_used_jac_elem functions, e.g. src/rxns/rxn_arrhenius.c:44-60).
void Model::build_rxn_jacobian() {
  Registry reg(n_state_);
  for (int i = 0; i < n_state_; ++i) reg.add(i, i);
  for (const Rxn& r : rxns_)
    for (int ind = 0; ind < r.nr; ++ind) {
      for (int d = 0; d < r.nr; ++d) reg.add(REACT(r, d), REACT(r, ind));
      for (int d = 0; d < r.np; ++d) reg.add(PROD(r, d), REACT(r, ind));
    }
  reg.to_csc(&rj_colptr_, &rj_rowid_);
}

// DERIV_ID and JAC_ID written back into the packed ints, as rxn_update_ids
// does (src/camp_solver.c:1491-1503, src/rxns/rxn_arrhenius.c:71-91).
void Model::update_ids() {
  deriv_ids_.assign(n_state_, -1);
  for (int i = 0, d = 0; i < n_state_; ++i)
    if (var_type_[i] == VAR_VARIABLE) deriv_ids_[i] = d++;
  for (const Rxn& r : rxns_) {
    for (int k = 0; k < r.nr; ++k) DERIV_ID(r, k) = deriv_ids_[REACT(r, k)];
    for (int k = 0; k < r.np; ++k) DERIV_ID(r, r.nr + k) = deriv_ids_[PROD(r, k)];
    int e = 0;
    for (int ind = 0; ind < r.nr; ++ind) {
      for (int d = 0; d < r.nr; ++d) JAC_ID(r, e++) = rxn_elem_id(REACT(r, d), REACT(r, ind));
      for (int d = 0; d < r.np; ++d) JAC_ID(r, e++) = rxn_elem_id(PROD(r, d), REACT(r, ind));
    }
  }
}

// Solver Jacobian: the variable x variable entries of the reaction Jacobian
// (src/camp_solver.c:1559-1633; a gas-phase model has no sub-model
// parameters, so every map entry has param_id 0).
void Model::build_solver_jacobian() {
  Registry reg(n_state_);
  for (int ind = 0; ind < n_state_; ++ind)
    for (int dep = 0; dep < n_state_; ++dep) {
      if (var_type_[dep] != VAR_VARIABLE || var_type_[ind] != VAR_VARIABLE) continue;
      if (rxn_elem_id(dep, ind) == -1) continue;
      reg.add(dep, ind);
    }
  std::vector<int> cp, ri;
  reg.to_csc(&cp, &ri);
  sj_colptr_.assign(n_dep_ + 1, 0);
  for (int c = 0; c < n_state_; ++c)
    if (deriv_ids_[c] >= 0) sj_colptr_[deriv_ids_[c]] = cp[c];
  sj_colptr_[n_dep_] = (int)ri.size();
  sj_rowid_.resize(ri.size());
  for (size_t e = 0; e < ri.size(); ++e) sj_rowid_[e] = deriv_ids_[ri[e]];
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
    for (int e = sj_colptr_[c]; e < sj_colptr_[c + 1]; ++e) P[sj_rowid_[e]][c] = 1;
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
  t.n_rxn = n_rxn_;
  t.n_jac = (int)sj_rowid_.size();
  t.dep_state.clear();
  for (int i = 0; i < n_state_; ++i)
    if (var_type_[i] == VAR_VARIABLE) t.dep_state.push_back(i);
  // rate laws and reactants
  t.rx_type.clear(); t.rx_nreact.clear(); t.rx_fpar.clear(); t.rx_photo.clear();
  t.fpar.clear();
  t.rx_cptr.assign(1, 0); t.rx_cidx.clear();
  t.rx_vptr.assign(1, 0); t.rx_vdep.clear();
  photo_slot_.assign(n_rxn_, -1);
  int n_photo = 0;
  for (int ri = 0; ri < n_rxn_; ++ri) {
    const Rxn& r = rxns_[ri];
    t.rx_type.push_back(r.type);
    t.rx_nreact.push_back(r.nr);
    t.rx_fpar.push_back((int)t.fpar.size());
    for (int k = 0; k < r.n_float_prop; ++k) t.fpar.push_back(rxn_float_[r.float_off + k]);
    if (r.type == RXN_PHOTOLYSIS) photo_slot_[ri] = n_photo++;
    t.rx_photo.push_back(photo_slot_[ri]);
    for (int k = 0; k < r.nr; ++k) {
      int s = REACT(r, k);
      if (var_type_[s] == VAR_VARIABLE)
        t.rx_vdep.push_back(deriv_ids_[s]);
      else
        t.rx_cidx.push_back(s);
    }
    t.rx_cptr.push_back((int)t.rx_cidx.size());
    t.rx_vptr.push_back((int)t.rx_vdep.size());
  }
  t.n_photo = n_photo;
  t.n_part = (int)t.rx_vdep.size();
  // f gather: per dependent species, in reaction order, reactant
  // occurrences (loss, coefficient -1) before products (coefficient yield)
  std::vector<std::vector<int>> frx(n_dep_), fpr(n_dep_);
  std::vector<std::vector<double>> fco(n_dep_);
  for (int ri = 0; ri < n_rxn_; ++ri) {
    const Rxn& r = rxns_[ri];
    for (int k = 0; k < r.nr; ++k) {
      int d = DERIV_ID(r, k);
      if (d < 0) continue;
      frx[d].push_back(ri); fco[d].push_back(-1.0); fpr[d].push_back(0);
    }
    for (int k = 0; k < r.np; ++k) {
      int d = DERIV_ID(r, r.nr + k);
      if (d < 0) continue;
      frx[d].push_back(ri); fco[d].push_back(YIELD(r, k)); fpr[d].push_back(1);
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
  // row = dependent species), in reaction order, for each variable
  // independent reactant occurrence: reactant rows (loss) then product rows
  std::vector<std::vector<int>> jpart(t.n_jac), jind(t.n_jac);
  std::vector<std::vector<double>> jco(t.n_jac);
  auto slot_of = [&](int row, int col) {
    for (int e = sj_colptr_[col]; e < sj_colptr_[col + 1]; ++e)
      if (sj_rowid_[e] == row) return e;
    return -1;
  };
  for (int ri = 0; ri < n_rxn_; ++ri) {
    const Rxn& r = rxns_[ri];
    int kv = 0;
    for (int ind = 0; ind < r.nr; ++ind) {
      int sind = REACT(r, ind);
      if (var_type_[sind] != VAR_VARIABLE) continue;
      int part = t.rx_vptr[ri] + kv++;
      int cind = deriv_ids_[sind];
      for (int d = 0; d < r.nr; ++d) {
        int sd = REACT(r, d);
        if (var_type_[sd] != VAR_VARIABLE) continue;
        int e = slot_of(deriv_ids_[sd], cind);
        jpart[e].push_back(part); jco[e].push_back(-1.0); jind[e].push_back(-1);
      }
      for (int d = 0; d < r.np; ++d) {
        int sd = PROD(r, d);
        if (var_type_[sd] != VAR_VARIABLE) continue;
        int e = slot_of(deriv_ids_[sd], cind);
        jpart[e].push_back(part); jco[e].push_back(YIELD(r, d)); jind[e].push_back(cind);
      }
    }
  }
  t.jg_ptr.assign(t.n_jac + 1, 0);
  t.jg_part.clear(); t.jg_coef.clear(); t.jg_ind.clear();
  t.jg_lupos.assign(t.n_jac, 0);
  t.jg_row.assign(t.n_jac, 0);
  for (int c = 0; c < n_dep_; ++c)
    for (int e = sj_colptr_[c]; e < sj_colptr_[c + 1]; ++e) {
      int pr = t.lu_iperm[sj_rowid_[e]], pc = t.lu_iperm[c];
      for (int q = t.lu_rowptr[pr]; q < t.lu_rowptr[pr + 1]; ++q)
        if (t.lu_col[q] == pc) t.jg_lupos[e] = q;
      t.jg_row[e] = sj_rowid_[e];
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
  build_rxn_jacobian();
  update_ids();
  build_solver_jacobian();
  build_lu();
  build_tables();
  built_ = true;
  return true;
}

}  // namespace campb
