// CAMP JSON input -> state layout and packed gas-phase reactions (loader.hpp).
#include "loader.hpp"

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
    *err = "WET_DEPOSITION removes the species of an aerosol phase, and aerosol phases are "
           "not read from JSON here; add it as packed data (rxn_add_condensed_data)";
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
  bool have_rel = false;
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
  out->rxns.clear();
  for (const auto& m : mechs)
    for (const Json* r : m.second) {
      LoadedRxn lr;
      if (!pack_reaction(*r, gas_index, &lr, err)) return false;
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
  out->name = mechs.empty() ? "mechanism" : mechs[0].first;
  return true;
}

}  // namespace campb
