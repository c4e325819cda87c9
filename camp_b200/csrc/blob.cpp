// Builds the compact shared-memory tables of the solve kernel (blob.hpp).
#include "blob.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>

#include "model.hpp"

namespace campb {

namespace {

constexpr int kLanes = 32;
constexpr uint16_t kNoSlot = 0xFFFF;

struct Writer {
  std::vector<uint8_t> buf;
  template <typename T>
  int put(const std::vector<T>& v) {
    size_t off = (buf.size() + 15) & ~size_t(15);
    buf.resize(off + std::max<size_t>(v.size(), 1) * sizeof(T), 0);
    if (!v.empty()) memcpy(buf.data() + off, v.data(), v.size() * sizeof(T));
    return (int)off;
  }
};

// Longest-processing-time assignment of weighted items to the 32 lanes.
std::vector<std::vector<int>> lpt(const std::vector<long>& weight) {
  std::vector<int> idx(weight.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return weight[a] > weight[b]; });
  std::vector<long> load(kLanes, 0);
  std::vector<std::vector<int>> lanes(kLanes);
  for (int i : idx) {
    int best = 0;
    for (int l = 1; l < kLanes; ++l)
      if (load[l] < load[best]) best = l;
    lanes[best].push_back(i);
    load[best] += weight[i];
  }
  return lanes;
}

}  // namespace

bool build_blob(const Tables& t, const std::vector<double>& atol_dep, std::vector<uint8_t>* blob,
                BlobOff* off, std::string* err) {
  const int n = t.n;
  if (n > 1023) {
    *err = "more than 1023 dependent variables";
    return false;
  }
  if (t.n_rates > 65535 || t.n_keff > 65535 || t.n_part_all > 65535 || t.n_lu > 65535 ||
      t.n_jac > 65535 ||
      (int)t.fg_rxn.size() > 65535 || (int)t.jg_part.size() > 65535 ||
      (int)t.fa_pos.size() > 65535) {
    *err = "mechanism exceeds the 16-bit table encodings";
    return false;
  }
  // coefficient table
  std::map<uint64_t, int> cid;
  std::vector<double> coef;
  auto coef_id = [&](double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    auto it = cid.find(b);
    if (it != cid.end()) return it->second;
    int id = (int)coef.size();
    coef.push_back(v);
    cid[b] = id;
    return id;
  };
  // reactions
  std::vector<uint32_t> rx_word(t.n_rxn);
  std::vector<uint16_t> rx_vptr(t.n_rxn + 1);
  for (int r = 0; r < t.n_rxn; ++r) {
    int v0 = t.rx_vptr[r], v1 = t.rx_vptr[r + 1];
    if (v1 - v0 > 3) {
      *err = "reaction " + std::to_string(r) + " has more than 3 variable reactants";
      return false;
    }
    uint32_t w = (uint32_t)(v1 - v0) << 30;
    for (int k = 0; k < v1 - v0; ++k) w |= (uint32_t)t.rx_vdep[v0 + k] << (10 * k);
    rx_word[r] = w;
    rx_vptr[r] = (uint16_t)v0;
  }
  rx_vptr[t.n_rxn] = (uint16_t)t.n_part;
  // f gather entries.  Each species list is regrouped, keeping reaction
  // order within a group: reactant occurrences (loss, coefficient -1), then
  // products with a non-negative yield, then products with a negative yield,
  // so that the device's common path adds each group without classifying
  // every term.  grp_end[2 * i + g] is the end of group g of species i.
  std::vector<uint32_t> fg_ent;
  fg_ent.reserve(t.fg_rxn.size());
  std::vector<int> grp_end(2 * n);
  for (int i = 0; i < n; ++i) {
    for (int g = 0; g < 3; ++g) {
      for (int e = t.fg_ptr[i]; e < t.fg_ptr[i + 1]; ++e) {
        const int eg = t.fg_prod[e] == FG_LOSS ? 0 : (t.fg_coef[e] >= 0.0 ? 1 : 2);
        if (eg != g) continue;
        int c = coef_id(t.fg_coef[e]);
        // bit 31: the term is guarded (a product; not a loss or a source)
        fg_ent.push_back((uint32_t)t.fg_rxn[e] | ((uint32_t)c << 16) |
                         ((uint32_t)(t.fg_prod[e] == FG_PRODUCT ? 1 : 0) << 31));
      }
      if (g < 2) grp_end[2 * i + g] = (int)fg_ent.size();
    }
  }
  // balanced f units: species lists longer than the per-lane share are split
  // into slots that a combine pass adds up
  const int total = t.fg_ptr[n];
  const int share = std::max(1, (total + kLanes - 1) / kLanes);
  struct Unit {
    int sp, b, e, slot;
  };
  auto clampi = [](int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); };
  std::vector<Unit> units;
  std::vector<uint16_t> split;
  int n_slots = 0;
  for (int i = 0; i < n; ++i) {
    int b = t.fg_ptr[i], e = t.fg_ptr[i + 1], c = e - b;
    if (c <= share) {
      units.push_back({i, b, e, kNoSlot});
      continue;
    }
    int k = (c + share - 1) / share;
    split.push_back((uint16_t)i);
    split.push_back((uint16_t)n_slots);
    split.push_back((uint16_t)k);
    for (int j = 0; j < k; ++j) {
      int ub = b + (int)((long)c * j / k), ue = b + (int)((long)c * (j + 1) / k);
      units.push_back({i, ub, ue, n_slots++});
    }
  }
  std::vector<long> uw(units.size());
  for (size_t u = 0; u < units.size(); ++u) uw[u] = 2 + (units[u].e - units[u].b);
  auto ulanes = lpt(uw);
  // unit record (8 x uint16, one 16-byte load): species, first entry, end
  // of its loss entries, end of its non-negative-yield products, end, slot
  std::vector<uint16_t> fg_unit, fg_lane(kLanes + 1, 0);
  for (int l = 0; l < kLanes; ++l) {
    fg_lane[l] = (uint16_t)(fg_unit.size() / 8);
    for (int u : ulanes[l]) {
      const Unit& x = units[u];
      fg_unit.push_back((uint16_t)x.sp);
      fg_unit.push_back((uint16_t)x.b);
      fg_unit.push_back((uint16_t)clampi(grp_end[2 * x.sp], x.b, x.e));
      fg_unit.push_back((uint16_t)clampi(grp_end[2 * x.sp + 1], x.b, x.e));
      fg_unit.push_back((uint16_t)x.e);
      fg_unit.push_back((uint16_t)x.slot);
      fg_unit.push_back(0);
      fg_unit.push_back(0);
    }
  }
  fg_lane[kLanes] = (uint16_t)(fg_unit.size() / 8);
  // J gather: each slot's partials regrouped: unguarded products (SIMPOL,
  // into the production part), losses (into the loss part) and guarded
  // products (into the production part); jg_umid[e] / jg_mid[e] are the
  // first loss / guarded product entry of slot e
  std::vector<uint32_t> jg_w0;
  std::vector<uint16_t> jg_w1, jg_mid(t.n_jac), jg_umid(t.n_jac);
  jg_w0.reserve(t.jg_part.size());
  jg_w1.reserve(t.jg_part.size());
  bool has_ug = false;
  for (int e = 0; e < t.n_jac; ++e) {
    for (int pass = 0; pass < 3; ++pass) {
      if (pass == 1) jg_umid[e] = (uint16_t)jg_w0.size();
      if (pass == 2) jg_mid[e] = (uint16_t)jg_w0.size();
      for (int g = t.jg_ptr[e]; g < t.jg_ptr[e + 1]; ++g) {
        const int kind = t.jg_ind[g] == -2 ? 0 : (t.jg_ind[g] == -1 ? 1 : 2);
        if (kind != pass) continue;
        has_ug |= kind == 0;
        int c = coef_id(t.jg_coef[g]);
        jg_w0.push_back((uint32_t)t.jg_part[g] | ((uint32_t)c << 16));
        jg_w1.push_back((uint16_t)(t.jg_ind[g] >= 0 ? t.jg_ind[g] + 1 : 0));
      }
    }
  }
  if (coef.size() > 32767) {
    *err = "too many distinct yields for the table encoding";
    return false;
  }
  std::vector<uint16_t> jg_ptr(t.n_jac + 1), jg_lupos(t.n_jac), jg_row(t.n_jac);
  for (int e = 0; e <= t.n_jac; ++e) jg_ptr[e] = (uint16_t)t.jg_ptr[e];
  // SIMPOL instance tables (dependent elements only: the constant ones are
  // folded into the per-cell constants)
  std::vector<uint16_t> si_rec, si_elem;
  std::vector<double> si_ef;
  for (int k = 0; k < t.n_simpol; ++k) {
    const SimpolInst& si = t.simpol[k];
    const int first = (int)si_elem.size();
    int nd = 0;
    // HL instances have no element partials (see SimpolInst)
    const size_t ne = si.type == RXN_SIMPOL_PHASE_TRANSFER ? si.elem.size() : 0;
    for (size_t j = 0; j < ne; ++j) {
      const int d = std::lower_bound(t.dep_state.begin(), t.dep_state.end(), si.elem[j]) -
                    t.dep_state.begin();
      if (d >= n || t.dep_state[d] != si.elem[j]) continue;  // not a dependent variable
      si_elem.push_back((uint16_t)d);
      si_ef.push_back(si.inv_rho[j]);
      si_ef.push_back(si.inv_mw[j]);
      si_ef.push_back(si.in_phase[j] ? 1.0 : 0.0);
      ++nd;
    }
    const auto dep_of = [&](int st) {
      return (int)(std::lower_bound(t.dep_state.begin(), t.dep_state.end(), st) -
                   t.dep_state.begin());
    };
    // rec[5]: HL's computed water + 1 (0: a constant water, folded per cell)
    const uint16_t rec[8] = {(uint16_t)dep_of(si.gas), (uint16_t)dep_of(si.aero),
                             (uint16_t)nd,                (uint16_t)first,
                             (uint16_t)t.si_part0[k],     (uint16_t)(si.water_cv + 1), 0, 0};
    si_rec.insert(si_rec.end(), rec, rec + 8);
  }
  for (int e = 0; e < t.n_jac; ++e) {
    jg_lupos[e] = (uint16_t)t.jg_lupos[e];
    jg_row[e] = (uint16_t)t.jg_row[e];
  }
  // per LU position: the solver-J slot that fills it (+1, 0 = none) and, in
  // bit 15, whether it is a diagonal (M = I - gamma*J in one pass)
  if (t.n_jac >= 32767) {
    *err = "too many Jacobian elements for the table encoding";
    return false;
  }
  std::vector<uint16_t> lu_src(t.n_lu, 0);
  for (int e = 0; e < t.n_jac; ++e) lu_src[t.jg_lupos[e]] = (uint16_t)(e + 1);
  for (int i = 0; i < n; ++i) lu_src[t.lu_diag[i]] |= 0x8000u;
  std::vector<long> jw(t.n_jac);
  for (int e = 0; e < t.n_jac; ++e) jw[e] = 2 + (t.jg_ptr[e + 1] - t.jg_ptr[e]);
  auto jlanes = lpt(jw);
  std::vector<uint16_t> jg_lane(kLanes + 1, 0), jg_slots;
  for (int l = 0; l < kLanes; ++l) {
    jg_lane[l] = (uint16_t)jg_slots.size();
    // longest slots first on every lane: the lanes of a warp step through
    // their k-th slots together, so slots of similar length line up and the
    // warp runs sum_k max_lane(len) ~ the per-lane total instead of far more
    std::vector<int> s = jlanes[l];
    std::stable_sort(s.begin(), s.end(), [&](int a, int b) {
      return t.jg_ptr[a + 1] - t.jg_ptr[a] > t.jg_ptr[b + 1] - t.jg_ptr[b];
    });
    for (int e : s) jg_slots.push_back((uint16_t)e);
  }
  jg_lane[kLanes] = (uint16_t)jg_slots.size();
  // LU
  auto u16 = [](const std::vector<int>& v) {
    std::vector<uint16_t> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = (uint16_t)v[i];
    return o;
  };
  std::vector<uint32_t> fa(t.fa_pos.size());
  for (size_t i = 0; i < fa.size(); ++i) fa[i] = (uint32_t)t.fa_pos[i] | ((uint32_t)t.fa_piv[i] << 16);
  // A grouped phase is stored as rounds: level l runs rounds
  // [rnd[l], rnd[l + 1]); round r gives lane k the record rec[32 r + k] of
  // its r-th unit (units of a lane in decreasing size) or, when the lane has
  // fewer units, a no-op record whose target is the spare slot `dummy` past
  // the end of the accumulator.  Records: target | count<<16, first pair |
  // (pivot+1)<<16.
  struct G {
    std::vector<uint16_t> rnd;
    std::vector<uint32_t> rec, pair;
  };
  auto pack = [&](const Tables::Grouped& g, G* o, int dummy) {
    o->rnd.assign(1, 0);
    o->rec.clear();
    for (int l = 0; l < g.n_levels; ++l) {
      int rounds = 0;
      for (int k = 0; k < kLanes; ++k)
        rounds = std::max(rounds, g.lane_ptr[33 * l + k + 1] - g.lane_ptr[33 * l + k]);
      for (int r = 0; r < rounds; ++r)
        for (int k = 0; k < kLanes; ++k) {
          const int u = g.lane_ptr[33 * l + k] + r;
          if (u < g.lane_ptr[33 * l + k + 1]) {
            o->rec.push_back((uint32_t)g.unit_target[u] | ((uint32_t)g.unit_count[u] << 16));
            o->rec.push_back((uint32_t)g.unit_begin[u] | ((uint32_t)g.unit_recip[u] << 16));
          } else {
            o->rec.push_back((uint32_t)dummy);
            o->rec.push_back(0u);
          }
        }
      o->rnd.push_back((uint16_t)(o->rnd.back() + rounds));
    }
    o->pair.resize(g.pair_a.size());
    for (size_t p = 0; p < g.pair_a.size(); ++p)
      o->pair[p] = (uint32_t)g.pair_a[p] | ((uint32_t)g.pair_b[p] << 16);
    return g.unit_target.size() <= 65535 && g.pair_a.size() <= 65535 && dummy <= 65535 &&
           o->rec.size() / 2 / kLanes <= 65535;
  };
  G gfb, gfw, gbw;
  if (!pack(t.fb, &gfb, t.n_lu) || !pack(t.fwd, &gfw, n) || !pack(t.bwd, &gbw, n)) {
    *err = "LU schedule exceeds the 16-bit table encodings";
    return false;
  }

  Writer w;
  // the offsets themselves lead the blob, so device code can rebuild its
  // table pointers from shared memory alone
  w.buf.resize(kBlobHeader, 0);
  static_assert(sizeof(BlobOff) <= kBlobHeader, "BlobOff must fit the blob header");
  BlobOff o{};
  o.n = n;
  o.n_rxn = t.n_rxn;
  o.n_part = t.n_part;
  o.n_jac = t.n_jac;
  o.n_lu = t.n_lu;
  o.n_coef = (int)coef.size();
  o.n_funits = (int)units.size();
  o.n_fsplit = (int)split.size() / 3;
  o.n_fscratch = n_slots;
  o.n_flev = t.n_flev;
  o.n_blev = t.n_blev;
  o.rx_word = w.put(rx_word);
  o.rx_vptr = w.put(rx_vptr);
  o.coef = w.put(coef);
  o.fg_ent = w.put(fg_ent);
  o.fg_unit = w.put(fg_unit);
  o.fg_lane = w.put(fg_lane);
  o.fg_split = w.put(split);
  o.jg_w0 = w.put(jg_w0);
  o.jg_w1 = w.put(jg_w1);
  o.jg_ptr = w.put(jg_ptr);
  o.jg_mid = w.put(jg_mid);
  o.jg_row = w.put(jg_row);
  o.jg_lane = w.put(jg_lane);
  o.jg_slots = w.put(jg_slots);
  o.has_ug = has_ug ? 1 : 0;
  o.jg_umid = w.put(jg_umid);
  o.n_simpol = t.n_simpol;
  o.n_keff = t.n_keff;
  o.n_rates = t.n_rates;
  o.n_part_all = t.n_part_all;
  o.si_rec = w.put(si_rec);
  o.si_elem = w.put(si_elem);
  o.si_ef = w.put(si_ef);
  // aqueous equilibrium instance records
  std::vector<uint16_t> aq_rec, aq_sp, aq_cp;
  std::vector<double> aq_sm, aq_cpm;
  for (int k = 0; k < t.n_aq; ++k) {
    const AqInst& q = t.aq[k];
    const int first = (int)aq_sp.size();
    int S = 0, R = 0;
    const auto dep_of = [&](int st) {
      const int d = (int)(std::lower_bound(t.dep_state.begin(), t.dep_state.end(), st) -
                          t.dep_state.begin());
      return d < n && t.dep_state[d] == st ? d : -1;
    };
    for (int pass = 0; pass < 2; ++pass) {
      const std::vector<int>& list = pass == 0 ? q.react : q.prod;
      for (size_t i = 0; i < list.size(); ++i) {
        const int d = dep_of(list[i]);
        if (d < 0) continue;
        aq_sp.push_back((uint16_t)d);
        aq_sm.push_back(q.m2m[(pass == 0 ? 0 : q.react.size()) + i]);
        ++S;
        R += pass == 0;
      }
    }
    // rec[6]: computed water + 1 (0: constant, folded per cell) | reactant
    // count << 8 | product count << 12 (constant species included: the
    // powers of the water); rec[7]: computed activity coefficient + 1
    const uint16_t wrec = (uint16_t)((q.water_cv + 1) | (q.react.size() << 8) |
                                     (q.prod.size() << 12));
    const int cp0 = (int)aq_cp.size();
    for (size_t j = 0; j < q.cp_cv.size(); ++j) {
      aq_cp.push_back((uint16_t)(q.cp_cv[j] | (q.cp_r[j] ? 0x8000 : 0)));
      aq_cpm.push_back(q.cp_m[j]);
    }
    const uint16_t rec[12] = {(uint16_t)S, (uint16_t)R, (uint16_t)first,
                              (uint16_t)t.aq_rate0[k], (uint16_t)t.aq_part0[k],
                              (uint16_t)t.aq_keff0[k], wrec, (uint16_t)(q.act_cv + 1),
                              (uint16_t)cp0, (uint16_t)q.cp_cv.size(), 0, 0};
    aq_rec.insert(aq_rec.end(), rec, rec + 12);
  }
  o.n_aq = t.n_aq;
  o.aq_rec = w.put(aq_rec);
  o.aq_sp = w.put(aq_sp);
  o.aq_sm = w.put(aq_sm);
  {
    std::vector<double> sim(aq_sm.size());
    for (size_t k = 0; k < sim.size(); ++k) sim[k] = 1.0 / aq_sm[k];
    o.aq_sim = w.put(sim);
  }
  o.aq_cp = w.put(aq_cp);
  o.aq_cpm = w.put(aq_cpm);
  // sub-model programs, virtual slots and the chain
  {
    std::vector<uint32_t> rec;
    std::vector<int32_t> ints;
    std::vector<double> flts;
    for (const SubProgram& g : t.cv) {
      rec.push_back((uint32_t)ints.size());
      rec.push_back((uint32_t)flts.size());
      ints.insert(ints.end(), g.ints.begin(), g.ints.end());
      flts.insert(flts.end(), g.flts.begin(), g.flts.end());
    }
    o.n_cv = t.n_cv;
    o.n_pj = t.n_pj;
    o.sm_keff = t.sm_keff;
    o.sm_rec = w.put(rec);
    std::vector<int> cv_state;
    for (const SubProgram& g : t.cv) cv_state.push_back(g.state);
    o.sm_state = w.put(u16(cv_state));
    o.sm_int = w.put(ints);
    o.sm_flt = w.put(flts);
    o.n_virt = t.n_virt;
    o.jv_ptr = w.put(u16(t.jv_ptr));
    o.jv_part = w.put(u16(t.jv_part));
    o.n_chain = (int)t.ch_tgt.size();
    o.ch_tgt = w.put(u16(t.ch_tgt));
    o.ch_ptr = w.put(u16(t.ch_ptr));
    std::vector<uint32_t> ent(t.ch_v.size());
    for (size_t i = 0; i < ent.size(); ++i)
      ent[i] = (uint32_t)t.ch_v[i] | ((uint32_t)t.ch_p[i] << 16);
    o.ch_ent = w.put(ent);
    if (t.n_cv > 254 || t.n_pj > 65535 || t.n_virt > 65535 || t.jv_part.size() > 65535 ||
        t.ch_v.size() > 65535) {
      *err = "sub-model tables exceed the 16-bit encodings";
      return false;
    }
  }
  o.n_plev = t.n_plev;
  o.lu_perm = w.put(u16(t.lu_perm));
  o.lu_src = w.put(lu_src);
  o.fa_ptr = w.put(u16(t.fa_ptr));
  o.fa = w.put(fa);
  o.fb_lane = w.put(gfb.rnd);
  o.fb_unit = w.put(gfb.rec);
  o.fb_pair = w.put(gfb.pair);
  o.fw_lane = w.put(gfw.rnd);
  o.fw_unit = w.put(gfw.rec);
  o.fw_pair = w.put(gfw.pair);
  o.bw_lane = w.put(gbw.rnd);
  o.bw_unit = w.put(gbw.rec);
  o.bw_pair = w.put(gbw.pair);
  o.dep_state = w.put(u16(t.dep_state));
  o.atol = w.put(atol_dep);
  // the one-lane LU tables come last: the level-scheduled mode stages only
  // the bytes before them into shared memory
  w.buf.resize((w.buf.size() + 15) & ~size_t(15), 0);
  o.stage_bytes = (int)w.buf.size();
  {
    std::vector<uint32_t> up(t.upd_ptr.begin(), t.upd_ptr.end()), ud(t.upd_src.size());
    for (size_t p = 0; p < ud.size(); ++p)
      ud[p] = (uint32_t)t.upd_src[p] | ((uint32_t)t.upd_dst[p] << 16);
    o.jg_lupos = w.put(jg_lupos);
    o.lu_diag = w.put(u16(t.lu_diag));
    o.lu_rowptr = w.put(u16(t.lu_rowptr));
    o.lu_col = w.put(u16(t.lu_col));
    o.upd_ptr = w.put(up);
    o.upd = w.put(ud);
  }
  w.buf.resize((w.buf.size() + 15) & ~size_t(15), 0);
  o.bytes = (int)w.buf.size();
  memcpy(w.buf.data(), &o, sizeof(o));
  blob->swap(w.buf);
  *off = o;
  return true;
}

}  // namespace campb

namespace campb {

bool build_lane_blob(const Tables& t, const std::vector<double>& atol_dep,
                     std::vector<uint8_t>* blob, LaneOff* off, std::string* err) {
  if (t.n_simpol > 0 || t.n_aq > 0 || t.n_cv > 0) {
    *err = "the lane-per-cell kernel does not evaluate SIMPOL, HL or aqueous equilibrium "
           "reactions or sub-models";
    return false;
  }
  const int n = t.n;
  if (n > 1023 || t.n_rxn > 65535 || t.n_lu > 65535) {
    *err = "mechanism exceeds the lane-kernel table encodings";
    return false;
  }
  std::map<uint64_t, int> cid;
  std::vector<double> coef;
  auto coef_id = [&](double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    auto it = cid.find(b);
    if (it != cid.end()) return it->second;
    int id = (int)coef.size();
    coef.push_back(v);
    cid[b] = id;
    return id;
  };
  // LU positions by (pivot row, pivot column)
  std::vector<std::vector<int>> pos(n, std::vector<int>(n, -1));
  for (int i = 0; i < n; ++i)
    for (int q = t.lu_rowptr[i]; q < t.lu_rowptr[i + 1]; ++q) pos[i][t.lu_col[q]] = q;
  // participants in term order: the variable reactant occurrences
  // (rx_vdep), then the variable products and sources (recovered from the f
  // gather lists, which hold every product of a term with its yield)
  struct Gain {
    int d;
    double c;
    bool guarded;
  };
  std::vector<std::vector<Gain>> prods(t.n_rxn);
  for (int d = 0; d < n; ++d)
    for (int e = t.fg_ptr[d]; e < t.fg_ptr[d + 1]; ++e)
      if (t.fg_prod[e] != FG_LOSS)
        prods[t.fg_rxn[e]].push_back({d, t.fg_coef[e], t.fg_prod[e] == FG_PRODUCT});
  std::vector<uint32_t> rx_word(t.n_rxn), rx_part;
  std::vector<uint16_t> rx_pptr(t.n_rxn + 1), rx_jptr(t.n_rxn + 1), jpos;
  for (int r = 0; r < t.n_rxn; ++r) {
    int v0 = t.rx_vptr[r], v1 = t.rx_vptr[r + 1];
    if (v1 - v0 > 3) {
      *err = "reaction " + std::to_string(r) + " has more than 3 variable reactants";
      return false;
    }
    uint32_t w = (uint32_t)(v1 - v0) << 30;
    for (int k = 0; k < v1 - v0; ++k) w |= (uint32_t)t.rx_vdep[v0 + k] << (10 * k);
    rx_word[r] = w;
    rx_pptr[r] = (uint16_t)rx_part.size();
    std::vector<int> sp;
    for (int k = v0; k < v1; ++k) {
      rx_part.push_back((uint32_t)t.rx_vdep[k] | ((uint32_t)coef_id(-1.0) << 10));
      sp.push_back(t.rx_vdep[k]);
    }
    for (const Gain& pr : prods[r]) {
      rx_part.push_back((uint32_t)pr.d | ((uint32_t)coef_id(pr.c) << 10) |
                        ((pr.guarded ? 1u : 0u) << 31));
      sp.push_back(pr.d);
    }
    rx_jptr[r] = (uint16_t)jpos.size();
    for (int k = v0; k < v1; ++k) {
      int col = t.lu_iperm[t.rx_vdep[k]];
      for (int s : sp) {
        int q = pos[t.lu_iperm[s]][col];
        if (q < 0) {
          *err = "internal: Jacobian entry outside the LU pattern";
          return false;
        }
        jpos.push_back((uint16_t)q);
      }
    }
  }
  rx_pptr[t.n_rxn] = (uint16_t)rx_part.size();
  rx_jptr[t.n_rxn] = (uint16_t)jpos.size();
  if (rx_part.size() > 65535 || jpos.size() > 65535 || coef.size() > 32767) {
    *err = "mechanism exceeds the lane-kernel table encodings";
    return false;
  }
  auto u16 = [](const std::vector<int>& v) {
    std::vector<uint16_t> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = (uint16_t)v[i];
    return o;
  };
  std::vector<uint32_t> up(t.upd_ptr.begin(), t.upd_ptr.end()), ud(t.upd_src.size());
  for (size_t p = 0; p < ud.size(); ++p)
    ud[p] = (uint32_t)t.upd_src[p] | ((uint32_t)t.upd_dst[p] << 16);
  Writer w;
  w.buf.resize(256, 0);
  static_assert(sizeof(LaneOff) <= 256, "LaneOff must fit the blob header");
  LaneOff o{};
  o.n = n;
  o.n_rxn = t.n_rxn;
  o.n_lu = t.n_lu;
  o.n_coef = (int)coef.size();
  o.n_part = (int)rx_part.size();
  o.n_jpos = (int)jpos.size();
  o.n_upd = (int)ud.size();
  o.rx_word = w.put(rx_word);
  o.rx_pptr = w.put(rx_pptr);
  o.rx_part = w.put(rx_part);
  o.rx_jptr = w.put(rx_jptr);
  o.jpos = w.put(jpos);
  o.coef = w.put(coef);
  o.lu_perm = w.put(u16(t.lu_perm));
  o.lu_rowptr = w.put(u16(t.lu_rowptr));
  o.lu_col = w.put(u16(t.lu_col));
  o.lu_diag = w.put(u16(t.lu_diag));
  o.upd_ptr = w.put(up);
  o.upd = w.put(ud);
  o.dep_state = w.put(u16(t.dep_state));
  o.atol = w.put(atol_dep);
  w.buf.resize((w.buf.size() + 15) & ~size_t(15), 0);
  o.bytes = (int)w.buf.size();
  memcpy(w.buf.data(), &o, sizeof(o));
  blob->swap(w.buf);
  *off = o;
  return true;
}

}  // namespace campb

namespace campb {

bool build_block_blob(const Tables& t, const std::vector<double>& atol_dep,
                      std::vector<uint8_t>* blob, BlockOff* off, std::string* err) {
  if (t.n_simpol > 0 || t.n_aq > 0 || t.n_cv > 0) {
    *err = "the CTA-per-cell kernel does not evaluate SIMPOL, HL or aqueous equilibrium "
           "reactions or sub-models";
    return false;
  }
  const int n = t.n;
  if (n < 1 || n > 1023 || t.n_rxn > 65535 || t.n_lu > 65535 || t.n_part > 65535 ||
      t.n_jac > 32767) {
    *err = "mechanism exceeds the CTA-kernel table encodings";
    return false;
  }
  std::map<uint64_t, int> cid;
  std::vector<double> coef;
  auto coef_id = [&](double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    auto it = cid.find(b);
    if (it != cid.end()) return it->second;
    int id = (int)coef.size();
    coef.push_back(v);
    cid[b] = id;
    return id;
  };
  // reactions
  std::vector<uint32_t> rx_word(t.n_rxn), rx_vptr(t.n_rxn + 1);
  for (int r = 0; r < t.n_rxn; ++r) {
    const int v0 = t.rx_vptr[r], v1 = t.rx_vptr[r + 1];
    if (v1 - v0 > 3) {
      *err = "reaction " + std::to_string(r) + " has more than 3 variable reactants";
      return false;
    }
    uint32_t w = (uint32_t)(v1 - v0) << 30;
    for (int k = 0; k < v1 - v0; ++k) w |= (uint32_t)t.rx_vdep[v0 + k] << (10 * k);
    rx_word[r] = w;
    rx_vptr[r] = (uint32_t)v0;
  }
  rx_vptr[t.n_rxn] = (uint32_t)t.rx_vptr[t.n_rxn];
  // f gather in the species lists' own order
  std::vector<uint32_t> fg_ptr(n + 1), fg_ent(t.fg_rxn.size());
  for (int i = 0; i <= n; ++i) fg_ptr[i] = (uint32_t)t.fg_ptr[i];
  for (size_t e = 0; e < fg_ent.size(); ++e)
    fg_ent[e] = (uint32_t)t.fg_rxn[e] | ((uint32_t)coef_id(t.fg_coef[e]) << 16) |
                ((uint32_t)(t.fg_prod[e] == FG_PRODUCT ? 1 : 0) << 31);
  // J gather: losses, then guarded products, per slot
  std::vector<uint32_t> jg_ptr(t.n_jac + 1), jg_mid(t.n_jac), jg_w0;
  std::vector<uint16_t> jg_w1, jg_row(t.n_jac);
  for (int e = 0; e < t.n_jac; ++e) {
    jg_ptr[e] = (uint32_t)jg_w0.size();
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) jg_mid[e] = (uint32_t)jg_w0.size();
      for (int g = t.jg_ptr[e]; g < t.jg_ptr[e + 1]; ++g) {
        if (t.jg_ind[g] == -2) {
          *err = "the CTA-per-cell kernel has no unguarded Jacobian products";
          return false;
        }
        if ((t.jg_ind[g] == -1) != (pass == 0)) continue;
        jg_w0.push_back((uint32_t)t.jg_part[g] | ((uint32_t)coef_id(t.jg_coef[g]) << 16));
        jg_w1.push_back((uint16_t)(t.jg_ind[g] >= 0 ? t.jg_ind[g] + 1 : 0));
      }
    }
    jg_row[e] = (uint16_t)t.jg_row[e];
  }
  jg_ptr[t.n_jac] = (uint32_t)jg_w0.size();
  if (coef.size() > 32767) {
    *err = "too many distinct yields for the table encoding";
    return false;
  }
  // LU: sorted rows, the diagonal in every row
  for (int i = 0; i < n; ++i) {
    for (int q = t.lu_rowptr[i] + 1; q < t.lu_rowptr[i + 1]; ++q)
      if (t.lu_col[q] <= t.lu_col[q - 1]) {
        *err = "internal: LU row columns not sorted";
        return false;
      }
    if (t.lu_col[t.lu_diag[i]] != i) {
      *err = "internal: LU diagonal position";
      return false;
    }
  }
  std::vector<uint16_t> lu_src(t.n_lu, 0);
  for (int e = 0; e < t.n_jac; ++e) lu_src[t.jg_lupos[e]] = (uint16_t)(e + 1);
  for (int i = 0; i < n; ++i) lu_src[t.lu_diag[i]] |= 0x8000u;
  // position lookup and the trailing dense block: the smallest r0 with every
  // (i, j), i, j >= r0, present
  std::vector<int> pos((size_t)n * n, -1);
  for (int i = 0; i < n; ++i)
    for (int q = t.lu_rowptr[i]; q < t.lu_rowptr[i + 1]; ++q)
      pos[(size_t)i * n + t.lu_col[q]] = q;
  int r0 = n - 1;
  for (int c = n - 2; c >= 0; --c) {
    bool full = true;
    for (int i = c; i < n && full; ++i)
      full = pos[(size_t)i * n + c] >= 0 && pos[(size_t)c * n + i] >= 0;
    if (!full) break;
    r0 = c;
  }
  if (n - r0 > kBlockMaxDense) {
    *err = "the LU's trailing dense block (" + std::to_string(n - r0) +
           " rows) exceeds the CTA kernel's " + std::to_string(kBlockMaxDense);
    return false;
  }
  std::vector<uint16_t> dpos(n - r0), ub(r0);
  for (int i = r0; i < n; ++i) dpos[i - r0] = (uint16_t)pos[(size_t)i * n + r0];
  for (int i = 0; i < r0; ++i) {
    int q = t.lu_rowptr[i + 1];
    while (q > t.lu_diag[i] + 1 && t.lu_col[q - 1] >= r0) --q;
    ub[i] = (uint16_t)q;
  }
  // head pivots: L entries of each column (row order), and the tabulated
  // update targets: head rows against every U entry of row k, dense rows
  // against the U entries in head columns
  std::vector<uint32_t> lk_ptr(r0 + 1, 0), lk_mid(std::max(r0, 1), 0), tg_ptr(r0 + 1, 0);
  std::vector<uint16_t> lk_pos, lk_row;
  std::vector<uint64_t> hrec;
  for (int k = 0; k < r0; ++k) {
    lk_ptr[k] = (uint32_t)lk_pos.size();
    tg_ptr[k] = (uint32_t)hrec.size();
    std::vector<int> rows;
    for (int i = k + 1; i < n; ++i) {
      const int q = pos[(size_t)i * n + k];
      if (q < 0) continue;
      rows.push_back(i);
      lk_pos.push_back((uint16_t)q);
      lk_row.push_back((uint16_t)i);
    }
    lk_mid[k] = (uint32_t)lk_ptr[k];
    for (int i : rows)
      if (i < r0) ++lk_mid[k];
    for (int pass = 0; pass < 2; ++pass)
      for (int i : rows) {
        if ((i >= r0) != (pass == 1)) continue;
        const int p1 = pass == 0 ? t.lu_rowptr[k + 1] : ub[k];
        const int lpos = pos[(size_t)i * n + k];
        for (int p = t.lu_diag[k] + 1; p < p1; ++p) {
          const int d = pos[(size_t)i * n + t.lu_col[p]];
          if (d < 0) {
            *err = "internal: LU fill pattern not closed";
            return false;
          }
          hrec.push_back((uint64_t)d | ((uint64_t)lpos << 16) | ((uint64_t)p << 32));
        }
      }
  }
  lk_ptr[r0] = (uint32_t)lk_pos.size();
  tg_ptr[r0] = (uint32_t)hrec.size();
  std::vector<uint32_t> lk(lk_pos.size());
  for (size_t e = 0; e < lk.size(); ++e) lk[e] = (uint32_t)lk_pos[e] | ((uint32_t)lk_row[e] << 16);
  // head row levels: forward over the L entries, backward over the U entries
  // with columns < r0 (the dense block's values reach head rows in one pass)
  std::vector<int> flev(r0, 0), blev(r0, 0);
  int n_hf = 0, n_hb = 0;
  for (int i = 0; i < r0; ++i) {
    int l = 0;
    for (int q = t.lu_rowptr[i]; q < t.lu_diag[i]; ++q) l = std::max(l, flev[t.lu_col[q]] + 1);
    flev[i] = l;
    n_hf = std::max(n_hf, l + 1);
  }
  for (int i = r0 - 1; i >= 0; --i) {
    int l = 0;
    for (int q = t.lu_diag[i] + 1; q < ub[i]; ++q) l = std::max(l, blev[t.lu_col[q]] + 1);
    blev[i] = l;
    n_hb = std::max(n_hb, l + 1);
  }
  auto levels = [&](const std::vector<int>& lev, int nl, std::vector<uint16_t>* ptr,
                    std::vector<uint16_t>* rows) {
    ptr->assign(nl + 1, 0);
    rows->clear();
    for (int l = 0; l < nl; ++l) {
      (*ptr)[l] = (uint16_t)rows->size();
      for (int i = 0; i < (int)lev.size(); ++i)
        if (lev[i] == l) rows->push_back((uint16_t)i);
    }
    (*ptr)[nl] = (uint16_t)rows->size();
  };
  std::vector<uint16_t> hf_ptr, hf_rows, hb_ptr, hb_rows;
  levels(flev, n_hf, &hf_ptr, &hf_rows);
  levels(blev, n_hb, &hb_ptr, &hb_rows);
  // the solve's staged section
  std::vector<uint16_t> stage;
  auto sec = [&](const std::vector<uint16_t>& v) {
    const int off = (int)stage.size();
    stage.insert(stage.end(), v.begin(), v.end());
    return off;
  };
  std::vector<uint16_t> ndoff(n + 1, 0), ndcol, dbase(n - r0);
  for (int i = 0; i < n; ++i) {
    ndoff[i] = (uint16_t)ndcol.size();
    const int q1 = i < r0 ? t.lu_rowptr[i + 1] : dpos[i - r0];
    for (int q = t.lu_rowptr[i]; q < q1; ++q) ndcol.push_back((uint16_t)t.lu_col[q]);
  }
  ndoff[n] = (uint16_t)ndcol.size();
  for (int i = r0; i < n; ++i) dbase[i - r0] = (uint16_t)(dpos[i - r0] - r0);
  if (ndcol.size() > 65535) {
    *err = "mechanism exceeds the CTA-kernel table encodings";
    return false;
  }
  auto u16 = [](const std::vector<int>& v) {
    std::vector<uint16_t> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = (uint16_t)v[i];
    return o;
  };
  Writer w;
  w.buf.resize(256, 0);
  static_assert(sizeof(BlockOff) <= 256, "BlockOff must fit the blob header");
  BlockOff o{};
  o.n = n;
  o.n_rxn = t.n_rxn;
  o.n_part = t.n_part;
  o.n_jac = t.n_jac;
  o.n_lu = t.n_lu;
  o.n_coef = (int)coef.size();
  o.r0 = r0;
  o.n_hf = n_hf;
  o.n_hb = n_hb;
  o.rx_word = w.put(rx_word);
  o.rx_vptr = w.put(rx_vptr);
  o.coef = w.put(coef);
  o.fg_ptr = w.put(fg_ptr);
  o.fg_ent = w.put(fg_ent);
  o.jg_ptr = w.put(jg_ptr);
  o.jg_mid = w.put(jg_mid);
  o.jg_w0 = w.put(jg_w0);
  o.jg_w1 = w.put(jg_w1);
  o.jg_row = w.put(jg_row);
  o.lu_src = w.put(lu_src);
  o.lu_perm = w.put(u16(t.lu_perm));
  o.lu_rowptr = w.put(u16(t.lu_rowptr));
  o.lu_col = w.put(u16(t.lu_col));
  o.lu_diag = w.put(u16(t.lu_diag));
  o.dpos = w.put(dpos);
  o.ub = w.put(ub);
  o.lk_ptr = w.put(lk_ptr);
  o.lk = w.put(lk);
  o.lk_mid = w.put(lk_mid);
  o.tg_ptr = w.put(tg_ptr);
  o.hrec = w.put(hrec);
  o.hf_ptr = w.put(hf_ptr);
  o.hf_rows = w.put(hf_rows);
  o.hb_ptr = w.put(hb_ptr);
  o.hb_rows = w.put(hb_rows);
  o.dep_state = w.put(u16(t.dep_state));
  o.atol = w.put(atol_dep);
  o.sg_rowptr = sec(u16(t.lu_rowptr));
  o.sg_diag = sec(u16(t.lu_diag));
  o.sg_ub = sec(ub);
  o.sg_perm = sec(u16(t.lu_perm));
  o.sg_hf_ptr = sec(hf_ptr);
  o.sg_hf_rows = sec(hf_rows);
  o.sg_hb_ptr = sec(hb_ptr);
  o.sg_hb_rows = sec(hb_rows);
  o.sg_ndoff = sec(ndoff);
  o.sg_ndcol = sec(ndcol);
  o.sg_dbase = sec(dbase);
  if (lk_ptr[r0] > 65535 || tg_ptr[r0] > 65535) {
    *err = "mechanism exceeds the CTA-kernel table encodings";
    return false;
  }
  std::vector<uint16_t> hlk(lk_ptr.begin(), lk_ptr.end()), hmid(r0), htg(tg_ptr.begin(), tg_ptr.end());
  for (int k = 0; k < r0; ++k) hmid[k] = (uint16_t)lk_mid[k];
  o.sg_hlk = sec(hlk);
  o.sg_hmid = sec(hmid);
  o.sg_htg = sec(htg);
  stage.resize((stage.size() + 7) & ~size_t(7), 0);  // whole 16-byte units
  o.sg_len = (int)stage.size();
  o.stage = w.put(stage);
  w.buf.resize((w.buf.size() + 15) & ~size_t(15), 0);
  o.bytes = (int)w.buf.size();
  memcpy(w.buf.data(), &o, sizeof(o));
  blob->swap(w.buf);
  *off = o;
  return true;
}

}  // namespace campb
