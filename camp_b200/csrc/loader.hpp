// CAMP JSON input -> state layout and packed gas-phase reactions, in C++,
// so that C/C++ hosts can drive the solver without the Fortran camp_core
// (whose reading and packing this restates: src/camp_core.F90:303-798,
// src/chem_spec_data.F90, src/rxns/rxn_*.F90 initialize).
#pragma once

#include <string>
#include <vector>

namespace campb {

struct LoadedRxn {
  int type = 0;
  std::vector<int> ints;      // as rxn_add_condensed_data receives them
  std::vector<double> floats;
  int n_env = 0;
  std::string label;          // "rxn id"
};

struct LoadedMechanism {
  std::string name;
  std::vector<std::string> species;  // gas-phase species, state order
  std::vector<int> var_type;         // CHEM_SPEC_* per state variable
  std::vector<double> abs_tol;       // per state variable
  double rel_tol = 1.0e-8;
  std::vector<LoadedRxn> rxns;
  int n_int() const;
  int n_float() const;
  int n_env() const;
};

// Reads CAMP JSON files ({"camp-data": [...]} with CHEM_SPEC, MECHANISM and
// RELATIVE_TOLERANCE objects) and packs the gas-phase reactions.
// Reactions whose rate the host sets (PHOTOLYSIS, FIRST_ORDER_LOSS,
// EMISSION) get ids 1, 2, ... in mechanism order.
bool load_mechanism_json(const std::vector<std::string>& files, LoadedMechanism* out,
                         std::string* err);

}  // namespace campb
