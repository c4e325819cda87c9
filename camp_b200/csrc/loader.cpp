// CAMP JSON input -> state layout and packed gas-phase reactions (loader.hpp).
#include "loader.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>

#include "json.hpp"

namespace campb {

namespace {

// state variable types, src/camp_common.h:34-38
constexpr int kUnknown = 0, kVariable = 1, kConstant = 2, kPssa = 3, kActivity = 4;
// reaction type ids, src/rxn_solver.c:19-35
constexpr int kArrhenius = 1, kTroe = 2, kCmaqH2O2 = 3, kCmaqOHHNO3 = 4, kPhotolysis = 5;
constexpr int kFirstOrderLoss = 12, kEmission = 13, kWetDeposition = 14;
constexpr int kHl = 6, kAqueous = 7, kSimpol = 10;
// aerosol representation and section types,
// src/aero_rep_solver.c:20, src/aero_reps/aero_rep_modal_binned_mass.c:25-26
constexpr int kModalBinned = 2, kBinned = 1, kModal = 2;
constexpr double kPi = 3.14159265358979323846;
// the Fortran packer's -9999.9 is a default-kind (single precision) literal
constexpr double kUnset = (double)-9999.9f;
// physical constants, src/constants.F90:37-41
constexpr double kBoltzmann = 1.3806505e-23;
constexpr double kAvogadro = 6.02214179e23;
constexpr double kGasConst = 8.314472;
constexpr double kDefaultAbsTol = 1.0e-14;  // src/chem_spec_data.F90:63

// Species in order of first appearance; later entries of the same name
// merge their properties (src/chem_spec_data.F90:320-338, 714-761).
struct SpeciesDb {
  struct Spec {
    int type = kUnknown;
    std::string phase;  // "" = not given (gas)
    std::vector<std::pair<std::string, const Json*>> props;
  };
  std::vector<std::string> names;
  std::map<std::string, Spec> spec;

  bool add(const Json& o, std::string* err) {
    const Json* jn = o.get("name");
    if (!jn || jn->kind != Json::String) {
      *err = "CHEM_SPEC without a name";
      return false;
    }
    const std::string& name = jn->str;
    int stype = kUnknown;
    std::string phase;
    if (!spec.count(name)) names.push_back(name);
    Spec& s = spec[name];
    for (const auto& kv : o.obj) {
      if (kv.first == "name" || kv.first == "type") continue;
      if (kv.first == "tracer type") {
        const std::string& v = kv.second.str;
        if (v == "VARIABLE") stype = kVariable;
        else if (v == "CONSTANT") stype = kConstant;
        else if (v == "PSSA") stype = kPssa;
        else if (v == "ION_PAIR" || v == "ACTIVITY_COEFF") stype = kActivity;
        else {
          *err = "unknown tracer type " + v + " for species " + name;
          return false;
        }
        if (v == "ION_PAIR") phase = "AEROSOL";
      } else if (kv.first == "phase") {
        phase = kv.second.str;
      } else {
        for (const auto& p : s.props)
          if (p.first == kv.first && kv.second.kind != Json::Object) {
            *err = "Duplicate property " + kv.first + " for species " + name;
            return false;
          }
        s.props.push_back({kv.first, &kv.second});
      }
    }
    if (stype != kUnknown) {
      if (s.type != kUnknown && s.type != stype) {
        *err = "Type mismatch for species " + name;
        return false;
      }
      s.type = stype;
    }
    if (!phase.empty()) {
      if (!s.phase.empty() && s.phase != phase) {
        *err = "Phase mismatch for species " + name;
        return false;
      }
      s.phase = phase;
    }
    return true;
  }
  bool is_gas(const std::string& n) const {
    const Spec& s = spec.at(n);
    return s.phase.empty() || s.phase == "GAS";
  }
  const Json* prop(const std::string& n, const std::string& key) const {
    for (const auto& p : spec.at(n).props)
      if (p.first == key) return p.second;
    return nullptr;
  }
  // a numeric property that must be present
  bool number(const std::string& n, const std::string& key, double* v, std::string* err) const {
    const Json* j = prop(n, key);
    bool ok = j != nullptr;
    if (ok) *v = as_number(*j, &ok);
    if (!ok) *err = "Missing or non-numeric '" + key + "' for species " + n;
    return ok;
  }
  int var_type(const std::string& n) const {
    int t = spec.at(n).type;
    return t == kUnknown ? kVariable : t;
  }
  double abs_tol(const std::string& n, bool* ok) const {
    double v = kDefaultAbsTol;
    for (const auto& p : spec.at(n).props)
      if (p.first == "absolute integration tolerance") v = as_number(*p.second, ok);
    return v;
  }
  static double as_number(const Json& j, bool* ok) {
    if (j.kind == Json::Number) return j.num;
    if (j.kind == Json::String) {
      char* end = nullptr;
      double v = std::strtod(j.str.c_str(), &end);
      if (end && *end == '\0' && end != j.str.c_str()) return v;
    }
    *ok = false;
    return 0.0;
  }
};

// one block of packed ints: [NUM_REACT, NUM_PROD, head.., REACT.., PROD..,
// DERIV_ID.. (0), JAC_ID.. (0)]
std::vector<int> int_block(int n_int_prop, const std::vector<int>& head,
                           const std::vector<int>& react, const std::vector<int>& prod) {
  const int nr = (int)react.size(), np = (int)prod.size();
  std::vector<int> ints((size_t)n_int_prop + (size_t)(nr + 2) * (nr + np), 0);
  ints[0] = nr;
  ints[1] = np;
  for (size_t k = 0; k < head.size(); ++k) ints[2 + k] = head[k];
  for (int k = 0; k < nr; ++k) ints[n_int_prop + k] = react[k];
  for (int k = 0; k < np; ++k) ints[n_int_prop + nr + k] = prod[k];
  return ints;
}

bool pack_reaction(const Json& r, const std::map<std::string, int>& gas_index, LoadedRxn* out,
                   std::string* err) {
  const Json* jt = r.get("type");
  const std::string type = jt ? jt->str : "";
  auto gas_id = [&](const std::string& n, int* id) {
    auto it = gas_index.find(n);
    if (it == gas_index.end()) {
      *err = "Missing species: " + n;
      return false;
    }
    *id = it->second;
    return true;
  };
  bool ok = true;
  auto num = [&](const char* key, double dflt) {
    const Json* j = r.get(key);
    return j ? SpeciesDb::as_number(*j, &ok) : dflt;
  };
  std::vector<int> react, prod;
  std::vector<double> ylds;
  if (const Json* jr = r.get("reactants"))
    for (const auto& kv : jr->obj) {
      int id;
      if (!gas_id(kv.first, &id)) return false;
      int qty = 1;
      if (const Json* q = kv.second.get("qty")) qty = (int)SpeciesDb::as_number(*q, &ok);
      for (int k = 0; k < qty; ++k) react.push_back(id);
    }
  if (const Json* jp = r.get("products"))
    for (const auto& kv : jp->obj) {
      int id;
      if (!gas_id(kv.first, &id)) return false;
      prod.push_back(id);
      const Json* y = kv.second.get("yield");
      ylds.push_back(y ? SpeciesDb::as_number(*y, &ok) : 1.0);
    }
  if (const Json* jl = r.get("rxn id")) out->label = jl->kind == Json::String ? jl->str : "";
  const Json* tu = r.get("time unit");
  const bool tunit_min = tu && tu->kind == Json::String && tu->str == "MIN";
  const double conv = kAvogadro / kGasConst * std::pow(10.0, -12.0);
  std::vector<double> f;
  if (type == "ARRHENIUS") {  // src/rxns/rxn_arrhenius.F90:150-287
    double A = num("A", 1.0);
    if (tunit_min) A = A / 60.0;
    double C;
    if (r.has("Ea")) {
      if (r.has("C")) {
        *err = "Received both Ea and C parameter for Arrhenius equation";
        return false;
      }
      C = -num("Ea", 0.0) / kBoltzmann;
    } else {
      C = num("C", 0.0);
    }
    const double D = num("D", 300.0), B = num("B", 0.0), E = num("E", 0.0);
    if (B != 0.0 && D == 0.0) {
      *err = "D cannot be zero if B is non-zero in Arrhenius reaction.";
      return false;
    }
    f = {A, B, C, D, E, conv};
    out->type = kArrhenius;
    out->ints = int_block(2, {}, react, prod);
    out->n_env = 1;
  } else if (type == "TROE") {  // src/rxns/rxn_troe.F90 initialize
    f = {num("k0_A", 1.0) * 1.0e6, num("k0_B", 0.0), num("k0_C", 0.0),
         num("kinf_A", 1.0),        num("kinf_B", 0.0), num("kinf_C", 0.0),
         num("Fc", 0.6),            num("N", 1.0),      tunit_min ? 1.0 / 60.0 : 1.0,
         conv};
    out->type = kTroe;
    out->ints = int_block(2, {}, react, prod);
    out->n_env = 1;
  } else if (type == "CMAQ_H2O2") {  // src/rxns/rxn_CMAQ_H2O2.F90 initialize
    double k1_A = num("k1_A", 1.0), k2_A = num("k2_A", 1.0);
    if (tunit_min) {
      k1_A = k1_A / 60.0;
      k2_A = k2_A / 60.0;
    }
    f = {k1_A, num("k1_B", 0.0), num("k1_C", 0.0), k2_A * 1.0e6, num("k2_B", 0.0),
         num("k2_C", 0.0), conv};
    out->type = kCmaqH2O2;
    out->ints = int_block(2, {}, react, prod);
    out->n_env = 1;
  } else if (type == "CMAQ_OH_HNO3") {  // src/rxns/rxn_CMAQ_OH_HNO3.F90 initialize
    f = {num("k0_A", 1.0),          num("k0_B", 0.0), num("k0_C", 0.0), num("k2_A", 1.0),
         num("k2_B", 0.0),          num("k2_C", 0.0), num("k3_A", 1.0) * 1.0e6,
         num("k3_B", 0.0),          num("k3_C", 0.0), tunit_min ? 1.0 / 60.0 : 1.0,
         conv};
    out->type = kCmaqOHHNO3;
    out->ints = int_block(2, {}, react, prod);
    out->n_env = 1;
  } else if (type == "PHOTOLYSIS") {  // src/rxns/rxn_photolysis.F90 initialize
    f = {num("scaling factor", 1.0)};
    out->type = kPhotolysis;
    out->ints = int_block(3, {-1}, react, prod);
    out->n_env = 2;
  } else if (type == "FIRST_ORDER_LOSS" || type == "EMISSION") {
    // src/rxns/rxn_first_order_loss.F90:169-220, rxn_emission.F90:166-217:
    // one gas species, RXN_ID_ = -1 until the host creates update data
    const bool loss = type == "FIRST_ORDER_LOSS";
    const Json* js = r.get("species");
    if (!js || js->kind != Json::String) {
      *err = std::string(loss ? "First-Order Loss" : "Emission") +
             " reaction is missing species name";
      return false;
    }
    int id;
    if (!gas_id(js->str, &id)) return false;
    f = {num("scaling factor", 1.0)};
    out->type = loss ? kFirstOrderLoss : kEmission;
    out->ints = loss ? std::vector<int>{-1, id, 0, 0} : std::vector<int>{-1, id, 0};
    out->n_env = 2;
  } else if (type == "WET_DEPOSITION") {
    *err = "WET_DEPOSITION removes the species of an aerosol phase, and the input defines no "
           "aerosol representation";
    return false;
  } else {
    *err = "reaction type " + type + " is not supported";
    return false;
  }
  if (!ok) {
    *err = "non-numeric reaction parameter in reaction " + out->label;
    return false;
  }
  f.insert(f.end(), ylds.begin(), ylds.end());
  out->floats = std::move(f);
  return true;
}

// --- aerosol phases and the modal/binned mass representation -----------

bool mass_species(int t) { return t == kVariable || t == kConstant || t == kPssa; }

// aero_phase_data_t%initialize (src/aero_phase_data.F90:306-385):
// [NUM_STATE_VAR, SPEC_TYPE(x)], floats [MW(x), DENSITY(x)]
bool pack_phase(const std::string& name, const std::vector<std::string>& species,
                const SpeciesDb& db, LoadedPhase* out, std::string* err) {
  out->name = name;
  out->species = species;
  const int n = (int)species.size();
  out->ints.assign(1 + n, 0);
  out->floats.assign(2 * n, 0.0);
  out->ints[0] = n;
  for (int i = 0; i < n; ++i) {
    const std::string& sp = species[i];
    if (!db.spec.count(sp)) {
      *err = "Missing property set for species '" + sp + "' in aerosol phase '" + name + "'";
      return false;
    }
    if (db.spec.at(sp).phase != "AEROSOL") {
      *err = "Trying to add non-aerosol phase species to aerosol phase " + name +
             "; species: " + sp;
      return false;
    }
    const int t = db.var_type(sp);
    out->ints[1 + i] = t;
    if (mass_species(t) && (!db.number(sp, "molecular weight [kg mol-1]", &out->floats[i], err) ||
                            !db.number(sp, "density [kg m-3]", &out->floats[n + i], err)))
      return false;
  }
  return true;
}

struct Section {
  std::string name;
  int kind = kModal, n_bins = 1;
  std::vector<int> phases;  // indices into the phase list
};

// A representation as the reaction packers query it (src/aero_rep_data.F90
// unique_names / spec_state_id / phase_ids / num_jac_elem).
struct Rep {
  LoadedRep data;
  int first_state = 0;  // 0-based state index of its first species
  std::vector<Section> sections;
  std::vector<std::string> unique;
  std::vector<int> instances;  // phase index of each instance, Fortran order

  // "section.[bin.]phase.species", optionally filtered by phase and species
  std::vector<std::string> names(const std::vector<LoadedPhase>& ph, const std::string* phase,
                                 const std::string* spec) const {
    std::vector<std::string> out;
    for (const Section& sec : sections)
      for (int pi : sec.phases) {
        if (phase && ph[pi].name != *phase) continue;
        for (int b = 0; b < sec.n_bins; ++b) {
          const std::string bin = sec.n_bins > 1 ? std::to_string(b + 1) + "." : "";
          for (const std::string& sp : ph[pi].species)
            if (!spec || sp == *spec) out.push_back(sec.name + "." + bin + ph[pi].name + "." + sp);
        }
      }
    return out;
  }
  int state_id(const std::string& un) const {  // 1-based
    for (size_t k = 0; k < unique.size(); ++k)
      if (unique[k] == un) return first_state + 1 + (int)k;
    return -1;
  }
  std::vector<int> phase_ids(const std::vector<LoadedPhase>& ph, const std::string& name) const {
    std::vector<int> out;
    for (size_t i = 0; i < instances.size(); ++i)
      if (ph[instances[i]].name == name) out.push_back((int)i + 1);
    return out;
  }
  // mass species of every phase of the instance's mode or bin
  // (src/aero_reps/aero_rep_modal_binned_mass.F90:964-996)
  int num_jac_elem(const std::vector<LoadedPhase>& ph, int phase_id) const {
    int start = 0, left = phase_id;
    for (const Section& sec : sections) {
      const int size = (int)sec.phases.size() * sec.n_bins;
      if (left <= size) {
        const int b = (left - 1) % sec.n_bins;
        int n = 0;
        for (size_t k = 0; k < sec.phases.size(); ++k) {
          const LoadedPhase& p = ph[instances[start + b + k * sec.n_bins]];
          for (int i = 0; i < p.ints[0]; ++i) n += mass_species(p.ints[1 + i]);
        }
        return n;
      }
      left -= size;
      start += size;
    }
    return 0;
  }
};

// aero_rep_modal_binned_mass_t%initialize
// (src/aero_reps/aero_rep_modal_binned_mass.F90:334-661) for a
// representation whose species start at 1-based state id first_state_1
bool pack_modal_binned(const Json& o, const std::vector<LoadedPhase>& phases, int first_state_1,
                       Rep* rep, std::string* err) {
  const std::string name = o.get("name") ? o.get("name")->str : "";
  const Json* secs = o.get("modes/bins");
  if (!secs || secs->kind != Json::Object || secs->obj.empty()) {
    *err = "No sections or bins specified for modal/binned mass aerosol representation '" + name +
           "'";
    return false;
  }
  bool ok = true;
  std::vector<const Json*> sj;
  for (const auto& kv : secs->obj) {
    Section sec;
    sec.name = kv.first;
    const Json* t = kv.second.get("type");
    const std::string type = t ? t->str : "";
    if (type == "MODAL") {
      sec.kind = kModal;
    } else if (type == "BINNED") {
      sec.kind = kBinned;
      const Json* nb = kv.second.get("bins");
      sec.n_bins = nb ? (int)SpeciesDb::as_number(*nb, &ok) : 0;
      if (!ok || sec.n_bins < 2) {
        *err = "Invalid number of bins for section '" + sec.name + "'";
        return false;
      }
    } else {
      *err = "Invalid type for section '" + sec.name + "'";
      return false;
    }
    const Json* pl = kv.second.get("phases");
    if (pl)
      for (const Json& pn : pl->arr) {
        int idx = -1;
        for (size_t k = 0; k < phases.size(); ++k)
          if (phases[k].name == pn.str) idx = (int)k;
        if (idx < 0) {
          *err = "Non-existant aerosol phase '" + pn.str + "' specified for mode '" + sec.name + "'";
          return false;
        }
        sec.phases.push_back(idx);
      }
    rep->sections.push_back(sec);
    sj.push_back(&kv.second);
  }
  const int ns = (int)rep->sections.size();
  int n_int = 4 + 2 * ns, n_float = 0;
  for (const Section& sec : rep->sections) {
    const int np = (int)sec.phases.size();
    n_int += 3 + 3 * sec.n_bins * np;
    n_float += 3 * sec.n_bins + 2 * sec.n_bins * np;
  }
  std::vector<int>& I = rep->data.ints;
  std::vector<double>& F = rep->data.floats;
  I.assign(n_int, 0);
  F.assign(n_float, 0.0);
  I[0] = ns;
  I[1] = n_int;
  I[2] = n_float;
  I[3] = -1;
  int loc_i = 4 + 2 * ns + 1, loc_f = 1, state = first_state_1;  // 1-based locations
  for (int x = 0; x < ns; ++x) {
    const Section& sec = rep->sections[x];
    I[4 + x] = loc_i;
    I[4 + ns + x] = loc_f;
    const int li = loc_i - 1, lf = loc_f - 1, nb = sec.n_bins, np = (int)sec.phases.size();
    I[li] = sec.kind;
    I[li + 1] = nb;
    I[li + 2] = np;
    if (sec.kind == kModal) {
      F[lf + 2] = kUnset;  // effective radius
      F[lf + 1] = kUnset;  // number concentration
    } else {
      const Json* jlo = sj[x]->get("minimum diameter [m]");
      const Json* jhi = sj[x]->get("maximum diameter [m]");
      const Json* jsc = sj[x]->get("scale");
      if (!jlo || !jhi || !jsc) {
        *err = "Missing diameter range or scale for bin '" + sec.name + "'";
        return false;
      }
      const double lo = SpeciesDb::as_number(*jlo, &ok), hi = SpeciesDb::as_number(*jhi, &ok);
      for (int b = 0; b < nb; ++b) {
        double dp;
        if (jsc->str == "LINEAR") {
          dp = lo + b * (hi - lo) / (nb - 1);
        } else if (jsc->str == "LOG") {
          const double d_log = (std::log10(hi) - std::log10(lo)) / (nb - 1);
          dp = std::pow(10.0, std::log10(lo) + b * d_log);
        } else {
          *err = "Invalid scale specified for bin '" + sec.name + "'";
          return false;
        }
        F[lf + 3 * b] = dp;
        F[lf + 3 * b + 2] = dp / 2.0;
        F[lf + 3 * b + 1] = kUnset;
      }
    }
    for (int y = 0; y < np; ++y)
      for (int b = 0; b < nb; ++b) {
        I[li + 3 + b * np + y] = state;                           // PHASE_STATE_ID_
        I[li + 3 + nb * np + b * np + y] = sec.phases[y] + 1;     // PHASE_MODEL_DATA_ID_
        state += (int)phases[sec.phases[y]].species.size();
        rep->instances.push_back(sec.phases[y]);
      }
    loc_i += 3 + 3 * nb * np;
    loc_f += 3 * nb + 2 * nb * np;
  }
  if (!ok) {
    *err = "non-numeric parameter in aerosol representation '" + name + "'";
    return false;
  }
  rep->data.type = kModalBinned;
  rep->data.name = name;
  rep->data.n_env = 2 * ns;
  rep->first_state = first_state_1 - 1;
  rep->unique = rep->names(phases, nullptr, nullptr);
  return true;
}

// N* -> enthalpy and entropy of the mass accommodation coefficient
// (src/rxns/rxn_SIMPOL_phase_transfer.F90, rxn_HL_phase_transfer.F90)
void n_star_terms(const SpeciesDb& db, const std::string& gas, double* dh, double* ds,
                  bool* ok) {
  *dh = *ds = 0.0;
  if (const Json* j = db.prop(gas, "N star")) {
    const double ns = SpeciesDb::as_number(*j, ok);
    *dh = (-10.0 * (ns - 1.0) + 7.53 * (std::pow(ns, 2.0 / 3.0) - 1.0) - 1.0) * 4184.0;
    *ds = (-32.0 * (ns - 1.0) + 9.21 * (std::pow(ns, 2.0 / 3.0) - 1.0) - 1.3) * 4.184;
  }
}

const std::string* json_str(const Json& r, const char* key) {
  const Json* j = r.get(key);
  return j && j->kind == Json::String ? &j->str : nullptr;
}

// One phase instance of a partitioning reaction: representation, species
// and second species (activity coefficient or water) unique names, phase id
struct Inst {
  int rep;
  std::string name, second;
  int phase_id;
};

// the instances of (phase, species) over every representation, with the
// second species' names beside them (an empty list when absent)
bool instances_of(const std::vector<Rep>& reps, const std::vector<LoadedPhase>& phases,
                  const std::string& phase, const std::string& spec, const std::string* second,
                  std::vector<Inst>* out, std::string* err) {
  for (size_t ri = 0; ri < reps.size(); ++ri) {
    const std::vector<std::string> names = reps[ri].names(phases, &phase, &spec);
    if (names.empty()) continue;
    std::vector<std::string> sec;
    if (second) {
      sec = reps[ri].names(phases, &phase, second);
      if (sec.size() != names.size()) {
        *err = "Missing species " + spec + " or " + *second + " in phase " + phase;
        return false;
      }
    }
    const std::vector<int> pids = reps[ri].phase_ids(phases, phase);
    for (size_t k = 0; k < names.size(); ++k)
      out->push_back({(int)ri, names[k], second ? sec[k] : "", pids[k]});
  }
  if (out->empty()) {
    *err = "No aerosol phase instances for partitioning of " + spec + " into " + phase;
    return false;
  }
  return true;
}

// rxn_SIMPOL_phase_transfer_t%initialize
// (src/rxns/rxn_SIMPOL_phase_transfer.F90:220-470)
bool pack_simpol(const Json& r, const SpeciesDb& db, const std::map<std::string, int>& gas_index,
                 const std::vector<Rep>& reps, const std::vector<LoadedPhase>& phases,
                 LoadedRxn* out, std::string* err) {
  const std::string* gas = json_str(r, "gas-phase species");
  const std::string* phase = json_str(r, "aerosol phase");
  const std::string* aero = json_str(r, "aerosol-phase species");
  const std::string* act = json_str(r, "aerosol-phase activity coefficient");
  if (!gas || !phase || !aero) {
    *err = "SIMPOL phase transfer reaction is missing a species or phase name";
    return false;
  }
  std::vector<Inst> inst;
  if (!instances_of(reps, phases, *phase, *aero, act, &inst, err)) return false;
  const int n = (int)inst.size();
  std::vector<int> ne(n);
  int E = 0;
  for (int x = 0; x < n; ++x) E += ne[x] = reps[inst[x].rep].num_jac_elem(phases, inst[x].phase_id);
  std::vector<int>& I = out->ints;
  std::vector<double>& F = out->floats;
  I.assign(4 + 13 * n + 2 * E, 0);
  F.assign(10 + 4 * E, 0.0);
  I[0] = n;
  auto g = gas_index.find(*gas);
  if (g == gas_index.end()) {
    *err = "Missing gas-phase species " + *gas;
    return false;
  }
  I[1] = g->second;
  int loc_i = 12 * n + 5, loc_f = 11;  // PHASE_INT_LOC_(1), PHASE_REAL_LOC_(1), 1-based
  for (int x = 0; x < n; ++x) {
    const Rep& rp = reps[inst[x].rep];
    I[4 + 10 * n + x] = loc_i;
    I[4 + 11 * n + x] = loc_f;
    I[loc_i - 1] = ne[x];                                            // NUM_AERO_PHASE_JAC_ELEM_
    I[2 + x] = rp.state_id(inst[x].name);                            // AERO_SPEC_
    I[2 + n + x] = act ? rp.state_id(inst[x].second) : -1;           // AERO_ACT_ID_
    I[2 + 2 * n + x] = inst[x].phase_id;                             // AERO_PHASE_ID_
    I[2 + 3 * n + x] = inst[x].rep + 1;                              // AERO_REP_ID_
    loc_i += 1 + 2 * ne[x];
    loc_f += 4 * ne[x];
  }
  bool ok = true;
  double mw, gas_mw, dh, ds;
  if (!db.spec.count(*aero) || !db.number(*aero, "molecular weight [kg mol-1]", &mw, err) ||
      !db.number(*gas, "diffusion coeff [m2 s-1]", &F[2], err) ||
      !db.number(*gas, "molecular weight [kg mol-1]", &gas_mw, err))
    return false;
  n_star_terms(db, *gas, &dh, &ds, &ok);
  const Json* b = r.get("B");
  if (!b || b->kind != Json::Array || b->arr.size() != 4) {
    *err = "Incorrect number of 'B' parameters";
    return false;
  }
  F[0] = dh;
  F[1] = ds;
  F[3] = std::sqrt(8.0 * kGasConst / (kPi * gas_mw));
  for (int k = 0; k < 4; ++k) F[4 + k] = SpeciesDb::as_number(b->arr[k], &ok);
  F[8] = kGasConst / mw * 1.0e6;
  F[9] = mw;
  if (!ok) {
    *err = "non-numeric SIMPOL parameter";
    return false;
  }
  out->type = kSimpol;
  out->n_env = 4;
  return true;
}

// rxn_HL_phase_transfer_t%initialize (src/rxns/rxn_HL_phase_transfer.F90:170-398)
bool pack_hl(const Json& r, const SpeciesDb& db, const std::map<std::string, int>& gas_index,
             const std::vector<Rep>& reps, const std::vector<LoadedPhase>& phases,
             LoadedRxn* out, std::string* err) {
  const std::string* gas = json_str(r, "gas-phase species");
  const std::string* phase = json_str(r, "aerosol phase");
  const std::string* aero = json_str(r, "aerosol-phase species");
  const std::string* water = json_str(r, "aerosol-phase water");
  if (!gas || !phase || !aero || !water) {
    *err = "HL phase transfer reaction is missing a species, phase or water name";
    return false;
  }
  std::vector<Inst> inst;
  if (!instances_of(reps, phases, *phase, *aero, water, &inst, err)) return false;
  const int n = (int)inst.size();
  std::vector<int> ne(n);
  int E = 0;
  for (int x = 0; x < n; ++x) E += ne[x] = reps[inst[x].rep].num_jac_elem(phases, inst[x].phase_id);
  std::vector<int>& I = out->ints;
  std::vector<double>& F = out->floats;
  I.assign(4 + 13 * n + 2 * E, 0);
  F.assign(8 + n + 2 * E, 0.0);
  I[0] = n;
  auto g = gas_index.find(*gas);
  if (g == gas_index.end()) {
    *err = "Missing gas-phase species " + *gas;
    return false;
  }
  I[1] = g->second;
  int loc_i = 8 * n + 5, loc_f = 9;  // PHASE_INT_LOC_(1), PHASE_REAL_LOC_(1), 1-based
  for (int x = 0; x < n; ++x) {
    const Rep& rp = reps[inst[x].rep];
    I[4 + 6 * n + x] = loc_i;
    I[4 + 7 * n + x] = loc_f;
    const int li = loc_i - 1;
    I[li] = rp.state_id(inst[x].name);       // AERO_SPEC_
    I[li + 1] = rp.state_id(inst[x].second);  // AERO_WATER_
    I[li + 2] = inst[x].phase_id;             // AERO_PHASE_ID_
    I[li + 3] = inst[x].rep + 1;              // AERO_REP_ID_
    I[li + 4] = ne[x];                        // NUM_AERO_PHASE_JAC_ELEM_
    loc_i += 5 + 2 * ne[x];
    loc_f += 1 + 2 * ne[x];
  }
  bool ok = true;
  double mw, gas_mw, dh, ds;
  if (!db.spec.count(*aero) || !db.number(*aero, "molecular weight [kg mol-1]", &mw, err) ||
      !db.number(*gas, "HLC(298K) [M Pa-1]", &F[4], err) ||
      !db.number(*gas, "HLC exp factor [K]", &F[5], err) ||
      !db.number(*gas, "diffusion coeff [m2 s-1]", &F[2], err) ||
      !db.number(*gas, "molecular weight [kg mol-1]", &gas_mw, err))
    return false;
  n_star_terms(db, *gas, &dh, &ds, &ok);
  if (!ok) {
    *err = "non-numeric N star for species " + *gas;
    return false;
  }
  F[0] = dh;
  F[1] = ds;
  F[3] = std::sqrt(8.0 * kGasConst / (kPi * gas_mw));
  F[6] = kGasConst / mw * 1.0e6;
  F[7] = mw;
  out->type = kHl;
  out->n_env = 4;
  return true;
}

// rxn_aqueous_equilibrium_t%initialize
// (src/rxns/rxn_aqueous_equilibrium.F90:170-493): reactant and product
// names (qty expanded), 1e3 / MW of each, and per phase instance the state
// ids of reactants, products, water and ion pair
bool pack_aqueous(const Json& r, const SpeciesDb& db, const std::vector<Rep>& reps,
                  const std::vector<LoadedPhase>& phases, LoadedRxn* out, std::string* err) {
  const std::string* phase = json_str(r, "aerosol phase");
  const std::string* water = json_str(r, "aerosol-phase water");
  if (!phase || !water) {
    *err = "Missing aerosol phase or aerosol-phase water for aqueous equilibrium reaction";
    return false;
  }
  bool ok = true;
  auto expand = [&](const char* key) {
    std::vector<std::string> names;
    if (const Json* b = r.get(key))
      for (const auto& kv : b->obj) {
        int qty = 1;
        if (const Json* q = kv.second.get("qty")) qty = (int)SpeciesDb::as_number(*q, &ok);
        for (int k = 0; k < qty; ++k) names.push_back(kv.first);
      }
    return names;
  };
  const std::vector<std::string> react = expand("reactants"), prod = expand("products");
  const int nr = (int)react.size(), np = (int)prod.size(), ns = nr + np;
  std::vector<int> present;
  int P = 0;
  for (size_t ri = 0; ri < reps.size(); ++ri)
    if (!reps[ri].phase_ids(phases, *phase).empty()) {
      present.push_back((int)ri);
      P += (int)reps[ri].names(phases, phase, water).size();
    }
  if (P == 0) {
    *err = "No aerosol phase '" + *phase + "' present.";
    return false;
  }
  std::vector<int>& I = out->ints;
  std::vector<double>& F = out->floats;
  I.assign(3 + P * (ns * (ns + 4) + 2), 0);
  F.assign(5 + 2 * ns + 2 * P, 0.0);
  I[0] = nr;
  I[1] = np;
  I[2] = P;
  const Json* ja = r.get("A");
  const Json* jc = r.get("C");
  const Json* jk = r.get("k_reverse");
  if (!jk) {
    *err = "Missing 'k_reverse' for aqueous equilibrium reaction";
    return false;
  }
  F[0] = ja ? SpeciesDb::as_number(*ja, &ok) : 1.0;
  F[1] = jc ? SpeciesDb::as_number(*jc, &ok) : 0.0;
  F[2] = SpeciesDb::as_number(*jk, &ok);
  const std::string* tu = json_str(r, "time_unit");
  if (tu && *tu == "MIN") F[2] = F[2] / 60.0;
  for (int k = 0; k < ns; ++k) {
    const std::string& name = k < nr ? react[k] : prod[k - nr];
    double mw;
    if (!db.spec.count(name) || !db.number(name, "molecular weight [kg mol-1]", &mw, err)) {
      *err = "Missing 'molecular weight' for species '" + name +
             "' in aqueous equilibrium reaction.";
      return false;
    }
    F[5 + k] = 1.0e3 / mw;
  }
  const std::string* ion = json_str(r, "ion pair");
  const int o_prod = 3 + nr * P, o_water = 3 + ns * P, o_act = o_water + P;
  int base = 0;
  for (int ri : present) {
    const Rep& rp = reps[ri];
    const std::vector<std::string> wn = rp.names(phases, phase, water);
    const int k = (int)wn.size();
    for (int j = 0; j < k; ++j) I[o_water + base + j] = rp.state_id(wn[j]);
    if (ion && !ion->empty()) {
      const std::vector<std::string> an = rp.names(phases, phase, ion);
      if ((int)an.size() != k || !db.spec.count(*ion) || db.var_type(*ion) != kActivity) {
        *err = "Ion pair '" + *ion + "' must have type 'ION_PAIR' and one instance per phase "
               "instance in an aqueous equilibrium reaction";
        return false;
      }
      for (int j = 0; j < k; ++j) I[o_act + base + j] = rp.state_id(an[j]);
    }
    for (int pass = 0; pass < 2; ++pass) {
      const std::vector<std::string>& names = pass == 0 ? react : prod;
      const int n = pass == 0 ? nr : np, o = pass == 0 ? 3 : o_prod;
      for (int i = 0; i < n; ++i) {
        const std::vector<std::string> un = rp.names(phases, phase, &names[i]);
        if ((int)un.size() != k) {
          *err = "Incorrect instances of '" + names[i] + "' in phase '" + *phase +
                 "' in an aqueous equilibrium reaction";
          return false;
        }
        for (int j = 0; j < k; ++j) I[o + (base + j) * n + i] = rp.state_id(un[j]);
      }
    }
    base += k;
  }
  if (!ok) {
    *err = "non-numeric aqueous equilibrium parameter";
    return false;
  }
  out->type = kAqueous;
  out->n_env = 1;
  return true;
}

// WET_DEPOSITION over every instance of a phase
// (src/rxns/rxn_wet_deposition.F90:172-254): RXN_ID_ NUM_SPEC_ REACT_(s)
// DERIV_ID_(s) JAC_ID_(s); SCALING_
bool pack_wet_deposition(const Json& r, const std::vector<Rep>& reps,
                         const std::vector<LoadedPhase>& phases, LoadedRxn* out,
                         std::string* err) {
  const std::string* phase = json_str(r, "aerosol phase");
  if (!phase) {
    *err = "Wet deposition reaction is missing an aerosol phase";
    return false;
  }
  std::vector<int> ids;
  for (const Rep& rp : reps)
    for (const std::string& un : rp.names(phases, phase, nullptr)) ids.push_back(rp.state_id(un));
  if (ids.empty()) {
    *err = "No aerosol phase instances for wet deposition of " + *phase;
    return false;
  }
  const int ns = (int)ids.size();
  out->ints.assign(2 + 3 * ns, 0);
  out->ints[0] = -1;
  out->ints[1] = ns;
  for (int k = 0; k < ns; ++k) out->ints[2 + k] = ids[k];
  bool ok = true;
  const Json* sc = r.get("scaling factor");
  out->floats = {sc ? SpeciesDb::as_number(*sc, &ok) : 1.0};
  if (!ok) {
    *err = "non-numeric wet deposition scaling factor";
    return false;
  }
  out->type = kWetDeposition;
  out->n_env = 2;
  return true;
}

// --- sub-models: ZSR aerosol water and PD-FiTE activity ------------------

// 1-based state ids of (phase, species) over every representation's
// instances, in representation and instance order
std::vector<int> instance_ids(const std::vector<Rep>& reps, const std::vector<LoadedPhase>& ph,
                              const std::string& phase, const std::string& spec) {
  std::vector<int> out;
  for (const Rep& r : reps)
    for (const std::string& un : r.names(ph, &phase, &spec)) out.push_back(r.state_id(un));
  return out;
}

// state id of spec relative to the aerosol water of the same instance; the
// same for every instance (the Fortran packers' relative ids)
bool relative_id(const std::vector<Rep>& reps, const std::vector<LoadedPhase>& ph,
                 const std::string& phase, const std::string& spec,
                 const std::vector<int>& water_ids, int* rel, std::string* err) {
  const std::vector<int> ids = instance_ids(reps, ph, phase, spec);
  if (ids.size() != water_ids.size() || ids.empty()) {
    *err = "Incorrect number of instances of '" + spec + "' in phase '" + phase + "'";
    return false;
  }
  *rel = ids[0] - water_ids[0];
  for (size_t k = 1; k < ids.size(); ++k)
    if (ids[k] - water_ids[k] != *rel) {
      *err = "'" + spec + "' is not at the same place in every instance of '" + phase + "'";
      return false;
    }
  return true;
}

// the two ions of a neutral ion pair: name, quantity, molecular weight, charge
struct Ion {
  std::string name;
  int qty;
  double mw;
  int charge;
};
bool ion_pair_ions(const Json& ions, const SpeciesDb& db, const std::string& what,
                   std::vector<Ion>* out, std::string* err) {
  if (ions.obj.size() != 2) {
    *err = "Invalid number of unique ions for ion pair in " + what;
    return false;
  }
  int total = 0;
  for (const auto& kv : ions.obj) {
    bool ok = true;
    int qty = 1;
    if (const Json* q = kv.second.get("qty")) qty = (int)SpeciesDb::as_number(*q, &ok);
    if (!db.spec.count(kv.first)) {
      *err = "Missing species properties for ion '" + kv.first + "' in " + what;
      return false;
    }
    double mw = 0.0, charge = 0.0;
    if (!db.number(kv.first, "molecular weight [kg mol-1]", &mw, err) ||
        !db.number(kv.first, "charge", &charge, err))
      return false;
    if ((int)charge == 0) {
      *err = "Neutral species '" + kv.first + "' not allowed in an ion pair in " + what;
      return false;
    }
    total += qty * (int)charge;
    out->push_back({kv.first, qty, mw, (int)charge});
  }
  if (total != 0) {
    *err = "Charge imbalance for an ion pair in " + what;
    return false;
  }
  return true;
}

// sub_model_ZSR_aerosol_water_t%initialize
// (src/sub_models/sub_model_ZSR_aerosol_water.F90:215-500): the layout the
// C sub-model reads (src/sub_models/sub_model_ZSR_aerosol_water.c:27-71),
// ion ids relative to the instance's water, Jacobian ids left at 0
bool pack_zsr(const Json& o, const SpeciesDb& db, const std::map<std::string, int>& gas_index,
              const std::vector<Rep>& reps, const std::vector<LoadedPhase>& ph,
              LoadedSubModel* out, std::string* err) {
  const std::string what = "ZSR aerosol water";
  const std::string* phase = json_str(o, "aerosol phase");
  const std::string* water = json_str(o, "aerosol-phase water");
  const std::string* gw = json_str(o, "gas-phase water");
  if (!phase || !water || !gw) {
    *err = what + ": missing aerosol phase, aerosol-phase water or gas-phase water";
    return false;
  }
  if (!db.spec.count(*water) || db.var_type(*water) != kConstant) {
    *err = "ZSR calculated species " + *water + " must be of tracer type CONSTANT";
    return false;
  }
  const std::vector<int> water_ids = instance_ids(reps, ph, *phase, *water);
  const int np = (int)water_ids.size();
  if (np == 0) {
    *err = "Aerosol phase '" + *phase + "' not present in any aerosol representation for " + what;
    return false;
  }
  const Json* pairs = o.get("ion pairs");
  if (!pairs || pairs->obj.empty()) {
    *err = "Empty ion pair set in " + what;
    return false;
  }
  if (!gas_index.count(*gw)) {
    *err = "Cannot find gas-phase water species '" + *gw + "' for " + what;
    return false;
  }
  const int n = (int)pairs->obj.size();
  int n_int = 5 + np + 2 * n, n_flt = 0;
  for (const auto& kv : pairs->obj) {
    const std::string* t = json_str(kv.second, "type");
    if (t && *t == "JACOBSON") {
      const Json* y = kv.second.get("Y_j");
      n_int += 6 + 3 * np;
      n_flt += 3 + (y ? (int)y->arr.size() : 0);
    } else if (t && *t == "EQSAM") {
      const Json* ions = kv.second.get("ions");
      const int ni = ions ? (int)ions->obj.size() : 0;
      n_int += 2 + np + (1 + np) * ni;
      n_flt += 3 + ni;
    } else {
      *err = "Invalid activity type specified for " + what;
      return false;
    }
  }
  std::vector<int> I(n_int, 0);
  std::vector<double> F(n_flt, 0.0);
  I[0] = np;
  I[1] = gas_index.at(*gw);
  I[2] = n;
  I[3] = n_int;
  I[4] = n_flt;
  for (int p = 0; p < np; ++p) I[5 + p] = water_ids[p];
  int ii = 5 + np + 2 * n, ff = 0, x = 0;
  bool ok = true;
  for (const auto& kv : pairs->obj) {
    const Json& pr = kv.second;
    I[5 + np + x] = ii + 1;
    I[5 + np + n + x] = ff + 1;
    ++x;
    if (*json_str(pr, "type") == "JACOBSON") {
      I[ii] = 1;
      const Json* y = pr.get("Y_j");
      const int ny = y ? (int)y->arr.size() : 0;
      I[ii + 5] = ny;
      for (int k = 0; k < ny; ++k) F[ff + 3 + k] = SpeciesDb::as_number(y->arr[k], &ok);
      const Json* low = pr.get("low RH");
      if (!low) {
        *err = "Missing 'low RH' value for ion pair '" + kv.first + "' in " + what;
        return false;
      }
      F[ff] = SpeciesDb::as_number(*low, &ok);
      const Json* ions = pr.get("ions");
      std::vector<Ion> ion;
      if (!ions || !ion_pair_ions(*ions, db, what, &ion, err)) {
        if (!ions) *err = "Missing ions for ion pair '" + kv.first + "' in " + what;
        return false;
      }
      for (const Ion& io : ion) {
        int rel = 0;
        if (!relative_id(reps, ph, *phase, io.name, water_ids, &rel, err)) return false;
        if (io.charge > 0) {
          I[ii + 1] = io.qty;
          F[ff + 1] = io.mw;
          I[ii + 3] = rel;
        } else {
          I[ii + 2] = io.qty;
          F[ff + 2] = io.mw;
          I[ii + 4] = rel;
        }
      }
      ii += 6 + 3 * np;
      ff += 3 + ny;
    } else {
      const Json* ions = pr.get("ions");
      const int ni = ions ? (int)ions->obj.size() : 0;
      const Json *nw = pr.get("NW"), *zw = pr.get("ZW"), *mw = pr.get("MW");
      if (!nw || !zw || !mw) {
        *err = "Missing NW, ZW or MW for ion pair '" + kv.first + "' in " + what;
        return false;
      }
      F[ff] = SpeciesDb::as_number(*nw, &ok);
      F[ff + 1] = SpeciesDb::as_number(*zw, &ok);
      F[ff + 2] = SpeciesDb::as_number(*mw, &ok);
      I[ii] = 2;
      I[ii + 1] = ni;
      for (int k = 0; k < ni; ++k) {
        const std::string& iname = ions->obj[k].first;
        double imw = 0.0;
        if (!db.spec.count(iname) || !db.number(iname, "molecular weight [kg mol-1]", &imw, err)) {
          *err = "Missing molecular weight for ion '" + iname + "' in " + what;
          return false;
        }
        F[ff + 3 + k] = imw;
        if (!relative_id(reps, ph, *phase, iname, water_ids, &I[ii + 2 + np + k], err))
          return false;
      }
      ii += 2 + np + (1 + np) * ni;
      ff += 3 + ni;
    }
  }
  if (!ok) {
    *err = "non-numeric parameter in " + what;
    return false;
  }
  out->type = 2;
  out->ints = std::move(I);
  out->floats = std::move(F);
  out->n_env = 1;
  return true;
}

// sub_model_PDFiTE_t%initialize (src/sub_models/sub_model_PDFiTE.F90:
// 250-700): the ion pairs of "calculate for" in order, then every further
// interaction partner in order of first appearance (no interactions of its
// own); ints and floats start at 9999 as the Fortran packer leaves unused
// slots
bool pack_pdfite(const Json& o, const SpeciesDb& db, const std::map<std::string, int>& gas_index,
                 const std::vector<Rep>& reps, const std::vector<LoadedPhase>& ph,
                 LoadedSubModel* out, std::string* err) {
  const std::string what = "PD-FiTE activity sub-model";
  const std::string* phase = json_str(o, "aerosol phase");
  const std::string* water = json_str(o, "aerosol-phase water");
  const std::string* gw = json_str(o, "gas-phase water");
  if (!phase || !water || !gw) {
    *err = what + ": missing aerosol phase, aerosol-phase water or gas-phase water";
    return false;
  }
  const std::vector<int> water_ids = instance_ids(reps, ph, *phase, *water);
  const int np = (int)water_ids.size();
  if (np == 0) {
    *err = "Aerosol phase '" + *phase + "' not present in any aerosol representation for " + what;
    return false;
  }
  if (!gas_index.count(*gw)) {
    *err = "Cannot find gas-phase water species '" + *gw + "' for " + what;
    return false;
  }
  const Json* calc = o.get("calculate for");
  std::vector<std::string> names;
  int n_inter = 0, n_flt_inter = 0;
  if (calc)
    for (const auto& kv : calc->obj) names.push_back(kv.first);
  if (calc)
    for (const auto& kv : calc->obj) {
      const Json* inter = kv.second.get("interactions");
      if (!inter) continue;
      for (const Json& it : inter->arr) {
        ++n_inter;
        const Json* b = it.get("B");
        n_flt_inter += 2 + (b ? (int)b->arr.size() : 0);
        const std::string* ip = json_str(it, "ion pair");
        if (!ip) {
          *err = "Missing ion pair of an interaction in " + what;
          return false;
        }
        if (std::find(names.begin(), names.end(), *ip) == names.end()) names.push_back(*ip);
      }
    }
  const int n = (int)names.size(), n_calc = calc ? (int)calc->obj.size() : 0;
  const int n_int = 5 + np + 3 * n_inter + (8 + (1 + 2 * n) * np) * n;
  const int n_flt = n_flt_inter + 4 * n;
  std::vector<int> I(n_int, 9999);
  std::vector<double> F(n_flt, 9999.0);
  I[0] = np;
  I[1] = gas_index.at(*gw);
  I[2] = n;
  I[3] = n_int;
  I[4] = n_flt;
  for (int p = 0; p < np; ++p) I[5 + p] = water_ids[p];
  int ii = 5 + np + 2 * n, ff = 0;
  bool ok = true;
  for (int x = 0; x < n; ++x) {
    const std::string& pname = names[x];
    I[5 + np + x] = ii + 1;
    I[5 + np + n + x] = ff + 1;
    if (!db.spec.count(pname) || db.var_type(pname) != kActivity) {
      *err = "Ion pair '" + pname + "' must have type ION_PAIR in " + what;
      return false;
    }
    if (!relative_id(reps, ph, *phase, pname, water_ids, &I[ii], err)) return false;
    const Json* ions = db.prop(pname, "ions");
    std::vector<Ion> ion;
    if (!ions || !ion_pair_ions(*ions, db, what, &ion, err)) {
      if (!ions) *err = "Missing ions for ion pair '" + pname + "' in " + what;
      return false;
    }
    for (const Ion& io : ion) {
      int rel = 0;
      if (!relative_id(reps, ph, *phase, io.name, water_ids, &rel, err)) return false;
      if (io.charge > 0) {
        I[ii + 1] = io.qty;
        F[ff] = io.mw;
        I[ii + 3] = rel;
      } else {
        I[ii + 2] = io.qty;
        F[ff + 1] = io.mw;
        I[ii + 4] = rel;
      }
    }
    ff += 4;
    const int base = ii;
    ii += 6 + (1 + 2 * n) * np;
    if (x < n_calc) {
      const Json* inter = calc->obj[x].second.get("interactions");
      const int ni = inter ? (int)inter->arr.size() : 0;
      I[base + 5] = ni;
      const int ob = base + 6 + (1 + 2 * n) * np;
      for (int y = 0; y < ni; ++y) {
        const Json& it = inter->arr[y];
        I[ob + 2 * ni + y] = ff + 1;
        I[ob + ni + y] =
            (int)(std::find(names.begin(), names.end(), *json_str(it, "ion pair")) -
                  names.begin()) + 1;
        const Json *lo = it.get("min RH"), *hi = it.get("max RH"), *b = it.get("B");
        if (!lo || !hi || !b) {
          *err = "Missing min RH, max RH or B for ion pair '" + pname + "' in " + what;
          return false;
        }
        const double vlo = SpeciesDb::as_number(*lo, &ok), vhi = SpeciesDb::as_number(*hi, &ok);
        if (!(vlo >= 0.0 && vlo < 1.0) || !(vhi > 0.0 && vhi <= 1.0)) {
          *err = "Invalid RH range for ion pair '" + pname + "' in " + what;
          return false;
        }
        const int nb = (int)b->arr.size();
        I[ob + y] = nb;
        F[ff] = vlo;
        F[ff + 1] = vhi;
        for (int z = 0; z < nb; ++z) F[ff + 2 + z] = SpeciesDb::as_number(b->arr[z], &ok);
        ff += 2 + nb;
        ii += 3;
      }
    } else {
      I[base + 5] = 0;
    }
  }
  if (!ok) {
    *err = "non-numeric parameter in " + what;
    return false;
  }
  out->type = 3;
  out->ints = std::move(I);
  out->floats = std::move(F);
  out->n_env = 1;
  return true;
}

}  // namespace

int LoadedMechanism::n_int() const {
  int k = 0;
  for (const auto& r : rxns) k += (int)r.ints.size();
  return k;
}
int LoadedMechanism::n_float() const {
  int k = 0;
  for (const auto& r : rxns) k += (int)r.floats.size();
  return k;
}
int LoadedMechanism::n_env() const {
  int k = 0;
  for (const auto& r : rxns) k += r.n_env;
  return k;
}

bool load_mechanism_json(const std::vector<std::string>& files, LoadedMechanism* out,
                         std::string* err) {
  std::vector<Json> docs(files.size());
  SpeciesDb db;
  std::vector<std::pair<std::string, std::vector<const Json*>>> mechs;
  std::vector<std::pair<std::string, std::vector<std::string>>> phase_json;
  std::vector<const Json*> rep_json, sub_json;
  bool have_rel = false;
  // camp_core keeps the sub-models in priority order: a new one goes before
  // the first of larger priority (src/camp_core.F90:575-605; ZSR 1, PD-FiTE 2,
  // src/sub_models/sub_model_ZSR_aerosol_water.F90:705-714,
  // src/sub_models/sub_model_PDFiTE.F90:865-874)
  auto priority = [](const Json* o) {
    const Json* t = o->get("type");
    return t && t->str == "SUB_MODEL_ZSR_AEROSOL_WATER" ? 1.0 : 2.0;
  };
  for (size_t f = 0; f < files.size(); ++f) {
    if (!read_json_file(files[f], &docs[f], err)) return false;
    const Json* data = docs[f].get("camp-data");
    if (!data) continue;
    for (const Json& o : data->arr) {
      const Json* t = o.get("type");
      const std::string type = t ? t->str : "";
      if (type == "CHEM_SPEC") {
        if (!db.add(o, err)) return false;
      } else if (type == "MECHANISM") {
        const std::string name = o.get("name") ? o.get("name")->str : "";
        std::vector<const Json*>* list = nullptr;
        for (auto& m : mechs)
          if (m.first == name) list = &m.second;
        if (!list) {
          mechs.push_back({name, {}});
          list = &mechs.back().second;
        }
        if (const Json* rx = o.get("reactions"))
          for (const Json& r : rx->arr) list->push_back(&r);
      } else if (type == "AERO_PHASE") {
        // phases of the same name merge their species lists
        const std::string name = o.get("name") ? o.get("name")->str : "";
        std::vector<std::string>* list = nullptr;
        for (auto& ph : phase_json)
          if (ph.first == name) list = &ph.second;
        if (!list) {
          phase_json.push_back({name, {}});
          list = &phase_json.back().second;
        }
        if (const Json* sp = o.get("species"))
          for (const Json& j : sp->arr) list->push_back(j.str);
      } else if (type.rfind("AERO_REP_", 0) == 0) {
        if (type != "AERO_REP_MODAL_BINNED_MASS") {
          *err = "aerosol representation " + type + " is not supported";
          return false;
        }
        rep_json.push_back(&o);
      } else if (type.rfind("SUB_MODEL_", 0) == 0) {
        if (type != "SUB_MODEL_ZSR_AEROSOL_WATER" && type != "SUB_MODEL_PDFITE") {
          *err = "sub-model " + type + " is not supported";
          return false;
        }
        const std::string name = o.get("name") ? o.get("name")->str : "";
        for (const Json* q : sub_json)
          if (q->get("name") && q->get("name")->str == name) {
            *err = "sub-model '" + name + "' is defined twice";
            return false;
          }
        size_t at = 0;
        while (at < sub_json.size() && !(priority(&o) < priority(sub_json[at]))) ++at;
        sub_json.insert(sub_json.begin() + (long)at, &o);
      } else if (type == "RELATIVE_TOLERANCE") {
        bool ok = true;
        const double v = o.get("value") ? SpeciesDb::as_number(*o.get("value"), &ok) : 0.0;
        if (!ok || !(v > 0.0 && v < 1.0)) {
          *err = "Invalid relative tolerance";
          return false;
        }
        out->rel_tol = v;
        have_rel = true;
      }
    }
  }
  if (!have_rel) out->rel_tol = 1.0e-8;
  std::map<std::string, int> gas_index;
  out->species.clear();
  out->var_type.clear();
  out->abs_tol.clear();
  for (const auto& n : db.names) {
    if (!db.is_gas(n)) continue;
    out->species.push_back(n);
    gas_index[n] = (int)out->species.size();  // 1-based state index
    bool ok = true;
    out->var_type.push_back(db.var_type(n));
    out->abs_tol.push_back(db.abs_tol(n, &ok));
    if (!ok) {
      *err = "non-numeric absolute tolerance for species " + n;
      return false;
    }
  }
  // aerosol phases, then the representations' species after the gas phase
  // (src/camp_core.F90:660-760), each representation's id its position
  out->phases.clear();
  for (const auto& ph : phase_json) {
    LoadedPhase lp;
    if (!pack_phase(ph.first, ph.second, db, &lp, err)) return false;
    out->phases.push_back(std::move(lp));
  }
  std::vector<Rep> reps;
  int next_state = (int)out->species.size() + 1;
  for (const Json* o : rep_json) {
    Rep rp;
    if (!pack_modal_binned(*o, out->phases, next_state, &rp, err)) return false;
    next_state += (int)rp.unique.size();
    reps.push_back(std::move(rp));
  }
  out->reps.clear();
  for (size_t i = 0; i < reps.size(); ++i) {
    reps[i].data.ints[3] = (int)i + 1;  // AERO_REP_ID_ as set_id gives it
    out->reps.push_back(reps[i].data);
    for (const std::string& un : reps[i].unique) {
      const std::string sp = un.substr(un.rfind('.') + 1);
      bool ok = true;
      out->species.push_back(un);
      out->var_type.push_back(db.var_type(sp));
      out->abs_tol.push_back(db.abs_tol(sp, &ok));
      if (!ok) {
        *err = "non-numeric absolute tolerance for species " + sp;
        return false;
      }
    }
  }
  out->rxns.clear();
  for (const auto& m : mechs)
    for (const Json* r : m.second) {
      LoadedRxn lr;
      const Json* jt = r->get("type");
      const std::string type = jt ? jt->str : "";
      bool done;
      if (type == "SIMPOL_PHASE_TRANSFER")
        done = pack_simpol(*r, db, gas_index, reps, out->phases, &lr, err);
      else if (type == "HL_PHASE_TRANSFER")
        done = pack_hl(*r, db, gas_index, reps, out->phases, &lr, err);
      else if (type == "AQUEOUS_EQUILIBRIUM")
        done = pack_aqueous(*r, db, reps, out->phases, &lr, err);
      else if (type == "WET_DEPOSITION" && !reps.empty())
        done = pack_wet_deposition(*r, reps, out->phases, &lr, err);
      else
        done = pack_reaction(*r, gas_index, &lr, err);
      if (!done) return false;
      if (const Json* jl = r->get("rxn id")) lr.label = jl->kind == Json::String ? jl->str : "";
      out->rxns.push_back(std::move(lr));
    }
  // reaction ids of the host-rate types: one sequence in mechanism order, as
  // generate_int_id (src/rand.F90:644-656) hands them out when the host
  // creates one update object per such reaction in that order
  int next_id = 1;
  for (auto& r : out->rxns) {
    if (r.type == kPhotolysis) r.ints[2] = next_id++;
    if (r.type == kFirstOrderLoss || r.type == kEmission || r.type == kWetDeposition)
      r.ints[0] = next_id++;
  }
  out->subs.clear();
  for (const Json* o : sub_json) {
    LoadedSubModel sm;
    const bool zsr = o->get("type")->str == "SUB_MODEL_ZSR_AEROSOL_WATER";
    if (!(zsr ? pack_zsr(*o, db, gas_index, reps, out->phases, &sm, err)
              : pack_pdfite(*o, db, gas_index, reps, out->phases, &sm, err)))
      return false;
    sm.name = o->get("name") ? o->get("name")->str : "";
    out->subs.push_back(std::move(sm));
  }
  out->name = mechs.empty() ? "mechanism" : mechs[0].first;
  return true;
}

}  // namespace campb
