// CAMP JSON input -> state layout, packed reactions, aerosol phases and
// representations, in C++, so that C/C++ hosts can drive the solver without
// the Fortran camp_core (whose reading and packing this restates:
// src/camp_core.F90:303-798, src/chem_spec_data.F90, src/rxns/rxn_*.F90
// initialize, src/aero_phase_data.F90, src/aero_reps/
// aero_rep_modal_binned_mass.F90).
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

// aero_phase_add_condensed_data / aero_rep_add_condensed_data arguments
struct LoadedPhase {
  std::string name;
  std::vector<std::string> species;
  std::vector<int> ints;
  std::vector<double> floats;
};
struct LoadedRep {
  int type = 0;
  std::string name;
  std::vector<int> ints;
  std::vector<double> floats;
  int n_env = 0;
};

// sub_model_add_condensed_data arguments (ints without the type slot)
struct LoadedSubModel {
  int type = 0;
  std::string name;
  std::vector<int> ints;
  std::vector<double> floats;
  int n_env = 0;
};

struct LoadedMechanism {
  std::string name;
  // state variables in order: the gas-phase species, then each aerosol
  // representation's "section.[bin.]phase.species" names
  std::vector<std::string> species;
  std::vector<int> var_type;         // CHEM_SPEC_* per state variable
  std::vector<double> abs_tol;       // per state variable
  double rel_tol = 1.0e-8;
  std::vector<LoadedRxn> rxns;
  std::vector<LoadedPhase> phases;
  std::vector<LoadedRep> reps;
  // ZSR aerosol water and PD-FiTE activity, in camp_core's priority order
  std::vector<LoadedSubModel> subs;
  int n_int() const;
  int n_float() const;
  int n_env() const;
};

// Reads CAMP JSON files ({"camp-data": [...]} with CHEM_SPEC, MECHANISM,
// RELATIVE_TOLERANCE, AERO_PHASE and AERO_REP_MODAL_BINNED_MASS objects) and
// packs the reactions: the gas-phase types, and SIMPOL_PHASE_TRANSFER,
// HL_PHASE_TRANSFER, AQUEOUS_EQUILIBRIUM and WET_DEPOSITION over the phase
// instances of the representations.  Reactions whose rate the host sets (PHOTOLYSIS,
// FIRST_ORDER_LOSS, EMISSION, WET_DEPOSITION) get ids 1, 2, ... in mechanism
// order; representations get ids 1, 2, ... in order.  SUB_MODEL_ZSR_AEROSOL_
// WATER and SUB_MODEL_PDFITE are packed in camp_core's priority order; other
// representation types and sub-models are refused.
bool load_mechanism_json(const std::vector<std::string>& files, LoadedMechanism* out,
                         std::string* err);

}  // namespace campb
