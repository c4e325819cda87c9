"""CAMP JSON input with aerosol phases, the modal/binned mass aerosol
representation and SIMPOL gas-particle partitioning, packed as the Fortran
``camp_core`` packs it for the C solver.

What is restated, from the reference's Fortran:

* the state layout (``src/camp_core.F90:660-760``): the gas-phase species,
  then each aerosol representation's species from the next state index;
* ``aero_phase_data_t%initialize`` (``src/aero_phase_data.F90:306-385``):
  ``[NUM_STATE_VAR, SPEC_TYPE(x)]``, floats ``[MW(x), DENSITY(x)]``;
* ``aero_rep_modal_binned_mass_t%initialize``
  (``src/aero_reps/aero_rep_modal_binned_mass.F90:334-661``): per mode or bin
  set its type, bin count, phase count, the state id, phase id and Jacobian
  element count of every phase instance, and the bin diameters; the unique
  names ``section.[bin.]phase.species`` (``:733-862``) give the state order,
  ``phase_ids`` (``src/aero_rep_data.F90``) and ``num_jac_elem`` (``:964-996``)
  the instance ids and element counts;
* ``rxn_SIMPOL_phase_transfer_t%initialize``
  (``src/rxns/rxn_SIMPOL_phase_transfer.F90:220-470``),
  ``rxn_HL_phase_transfer_t%initialize``
  (``src/rxns/rxn_HL_phase_transfer.F90:170-398``),
  ``rxn_aqueous_equilibrium_t%initialize``
  (``src/rxns/rxn_aqueous_equilibrium.F90:170-493``) and the WET_DEPOSITION
  packer over every instance of a phase
  (``src/rxns/rxn_wet_deposition.F90:172-254``).

* the ZSR aerosol-water and PD-FiTE activity sub-models
  (``src/sub_models/sub_model_ZSR_aerosol_water.F90:215-500``,
  ``src/sub_models/sub_model_PDFiTE.F90:250-700``), in camp_core's priority
  order.

Aerosol-representation ids (``AERO_REP_ID_``) are given 1, 2, ... as a host
does through ``set_id`` before it creates GMD/GSD update data.  Other aerosol
types (single particle, condensed-phase reactions, UNIFAC) are not packed
here.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import Iterable

import numpy as np

from .mechanism import (CHEM_SPEC_ACTIVITY_COEFF, CHEM_SPEC_CONSTANT, CHEM_SPEC_PSSA,
                        CHEM_SPEC_VARIABLE, RXN_WET_DEPOSITION, SUB_MODEL_PDFITE,
                        SUB_MODEL_ZSR_AEROSOL_WATER, Mechanism, PackedRxn, SubModel, _read_json,
                        _SpeciesDB, assign_rate_ids, pack_reaction)

AERO_REP_MODAL_BINNED_MASS = 2  # src/aero_rep_solver.c:20
RXN_HL_PHASE_TRANSFER = 6       # src/rxn_solver.c:24
RXN_AQUEOUS_EQUILIBRIUM = 7     # src/rxn_solver.c:25
RXN_SIMPOL_PHASE_TRANSFER = 10  # src/rxn_solver.c:26
BINNED, MODAL = 1, 2            # src/aero_reps/aero_rep_modal_binned_mass.c:25-26
UNIV_GAS_CONST = 8.314472       # src/constants.F90
# sub-model calculation priorities (lower first):
# src/sub_models/sub_model_ZSR_aerosol_water.F90:705-714,
# src/sub_models/sub_model_PDFiTE.F90:865-874
SUB_MODEL_PRIORITY = {"SUB_MODEL_ZSR_AEROSOL_WATER": 1.0, "SUB_MODEL_PDFITE": 2.0}
PI = 3.14159265358979323846
# the Fortran packer's -9999.9 is a default-kind (single precision) literal
UNSET = float(np.float32(-9999.9))


def _mass_species(t: int) -> bool:
    """Species that count towards phase mass and volume (and Jacobians)."""
    return t in (CHEM_SPEC_VARIABLE, CHEM_SPEC_CONSTANT, CHEM_SPEC_PSSA)


@dataclass
class AeroPhase:
    name: str
    species: list[str]
    types: list[int]
    ints: np.ndarray
    floats: np.ndarray

    @property
    def n_jac_elem(self) -> int:
        return sum(1 for t in self.types if _mass_species(t))

    def to_dict(self) -> dict:
        return {"name": self.name, "species": self.species, "types": self.types,
                "ints": [int(v) for v in self.ints], "floats": [float(v) for v in self.floats]}

    @classmethod
    def from_dict(cls, d: dict) -> "AeroPhase":
        return cls(d["name"], list(d["species"]), [int(v) for v in d["types"]],
                   np.asarray(d["ints"], np.int32), np.asarray(d["floats"], np.float64))


@dataclass
class Section:
    name: str
    kind: int                 # MODAL or BINNED
    n_bins: int
    phases: list[int]         # indices into the phase set
    gsd: float = 0.0          # modes: the JSON's geometric standard deviation
    gmd: float = 0.0          # modes: the JSON's geometric mean diameter [m]


@dataclass
class AeroRep:
    rep_type: int
    name: str
    ints: np.ndarray
    floats: np.ndarray
    n_env: int
    first_state: int          # 0-based state index of the first species
    sections: list[Section] = field(default_factory=list)
    unique_names: list[str] = field(default_factory=list)
    # phase instances in the Fortran order (section, phase, bin): phase index
    instances: list[int] = field(default_factory=list)

    def to_dict(self) -> dict:
        return {"rep_type": self.rep_type, "name": self.name,
                "ints": [int(v) for v in self.ints], "floats": [float(v) for v in self.floats],
                "n_env": self.n_env, "first_state": self.first_state,
                "sections": [vars(s) for s in self.sections],
                "unique_names": self.unique_names, "instances": self.instances}

    @classmethod
    def from_dict(cls, d: dict) -> "AeroRep":
        return cls(int(d["rep_type"]), d["name"], np.asarray(d["ints"], np.int32),
                   np.asarray(d["floats"], np.float64), int(d["n_env"]), int(d["first_state"]),
                   [Section(**s) for s in d["sections"]], list(d["unique_names"]),
                   [int(v) for v in d["instances"]])

    # --- the representation's queries used by the reaction packers ---------
    def names(self, phases: list[AeroPhase], phase_name: str | None = None,
              spec_name: str | None = None) -> list[str]:
        """unique_names with the Fortran filters, in its order."""
        out = []
        for sec in self.sections:
            for pi in sec.phases:
                ph = phases[pi]
                if phase_name is not None and ph.name != phase_name:
                    continue
                for b in range(sec.n_bins):
                    bin_str = f"{b + 1}." if sec.n_bins > 1 else ""
                    for sp in ph.species:
                        if spec_name is not None and sp != spec_name:
                            continue
                        out.append(f"{sec.name}.{bin_str}{ph.name}.{sp}")
        return out

    def state_id(self, unique_name: str) -> int:
        """1-based state id of a unique name (spec_state_id)."""
        return self.first_state + 1 + self.unique_names.index(unique_name)

    def phase_ids(self, phases: list[AeroPhase], phase_name: str) -> list[int]:
        return [i + 1 for i, pi in enumerate(self.instances) if phases[pi].name == phase_name]

    def num_jac_elem(self, phases: list[AeroPhase], phase_id: int) -> int:
        """Elements of all phases of the instance's mode or bin."""
        start = 0
        left = phase_id
        for sec in self.sections:
            size = len(sec.phases) * sec.n_bins
            if left <= size:
                b = (left - 1) % sec.n_bins
                return sum(phases[self.instances[start + b + k * sec.n_bins]].n_jac_elem
                           for k in range(len(sec.phases)))
            left -= size
            start += size
        raise ValueError(f"no phase instance {phase_id}")


def pack_aero_phase(name: str, species: list[str], db: _SpeciesDB) -> AeroPhase:
    types, mw, dens = [], [], []
    for sp in species:
        if sp not in db.props:
            raise KeyError(f"Missing property set for species '{sp}' in aerosol phase '{name}'")
        if (db.phase[sp] or "GAS") != "AEROSOL":
            raise ValueError(f"Trying to add non-aerosol phase species to aerosol phase {name}; "
                             f"species: {sp}")
        t = db.var_type_of(sp)
        types.append(t)
        if _mass_species(t):
            mw.append(float(db.props[sp]["molecular weight [kg mol-1]"]))
            dens.append(float(db.props[sp]["density [kg m-3]"]))
        else:
            mw.append(0.0)
            dens.append(0.0)
    ints = np.asarray([len(species)] + types, np.int32)
    floats = np.asarray(mw + dens, np.float64)
    return AeroPhase(name, list(species), types, ints, floats)


def pack_modal_binned(name: str, obj: dict, phases: list[AeroPhase],
                      first_state_1: int) -> AeroRep:
    """The modal/binned mass representation starting at 1-based state id
    ``first_state_1``; condensed data in the Fortran layout (1-based
    locations stored, as the C code subtracts one)."""
    secs_json = obj.get("modes/bins")
    if not secs_json:
        raise ValueError(f"No sections or bins specified for modal/binned mass aerosol "
                         f"representation '{name}'")
    by_name = {p.name: i for i, p in enumerate(phases)}
    sections = []
    for sname, sj in secs_json.items():
        kind = {"MODAL": MODAL, "BINNED": BINNED}[sj["type"]]
        nb = int(sj["bins"]) if kind == BINNED else 1
        plist = []
        for pn in sj["phases"]:
            if pn not in by_name:
                raise ValueError(f"Non-existant aerosol phase '{pn}' specified for mode '{sname}'")
            plist.append(by_name[pn])
        sec = Section(sname, kind, nb, plist)
        if kind == MODAL:
            sec.gmd = float(sj.get("geometric mean diameter [m]", 0.0))
            sec.gsd = float(sj.get("geometric standard deviation", 0.0))
        sections.append((sec, sj))
    ns = len(sections)
    n_int = 4 + 2 * ns + sum(3 + 3 * s.n_bins * len(s.phases) for s, _ in sections)
    n_float = sum(3 * s.n_bins + 2 * s.n_bins * len(s.phases) for s, _ in sections)
    ints = np.zeros(n_int, np.int32)
    floats = np.zeros(n_float, np.float64)
    ints[0], ints[1], ints[2], ints[3] = ns, n_int, n_float, -1
    loc_i, loc_f = 4 + 2 * ns + 1, 1   # next free 1-based locations
    state = first_state_1
    instances = []
    for x, (sec, sj) in enumerate(sections):
        ints[4 + x] = loc_i
        ints[4 + ns + x] = loc_f
        li, lf = loc_i - 1, loc_f - 1      # 0-based
        nb, npf = sec.n_bins, len(sec.phases)
        ints[li], ints[li + 1], ints[li + 2] = sec.kind, nb, npf
        if sec.kind == MODAL:
            floats[lf + 2] = UNSET   # effective radius
            floats[lf + 1] = UNSET   # number concentration
        else:
            lo, hi = float(sj["minimum diameter [m]"]), float(sj["maximum diameter [m]"])
            scale = sj["scale"]
            for b in range(nb):
                if scale == "LINEAR":
                    dp = lo + b * (hi - lo) / (nb - 1)
                elif scale == "LOG":
                    d_log = (math.log10(hi) - math.log10(lo)) / (nb - 1)
                    dp = 10.0 ** (math.log10(lo) + b * d_log)
                else:
                    raise ValueError(f"Invalid scale specified for bin '{sec.name}'")
                floats[lf + 3 * b] = dp
                floats[lf + 3 * b + 2] = dp / 2.0
                floats[lf + 3 * b + 1] = UNSET
        for y, pi in enumerate(sec.phases):
            for b in range(nb):
                ints[li + 3 + b * npf + y] = state                 # PHASE_STATE_ID_
                ints[li + 3 + nb * npf + b * npf + y] = pi + 1     # PHASE_MODEL_DATA_ID_
                state += len(phases[pi].species)
                instances.append(pi)
        loc_i += 3 + 3 * nb * npf
        loc_f += 3 * nb + 2 * nb * npf
    rep = AeroRep(AERO_REP_MODAL_BINNED_MASS, name, ints, floats, 2 * ns, first_state_1 - 1,
                  [s for s, _ in sections], [], instances)
    rep.unique_names = rep.names(phases)
    assert len(rep.unique_names) == state - first_state_1
    return rep


def pack_simpol(rxn: dict, db: _SpeciesDB, gas_index: dict[str, int], reps: list[AeroRep],
                phases: list[AeroPhase]) -> PackedRxn:
    gas = rxn["gas-phase species"]
    phase = rxn["aerosol phase"]
    aero = rxn["aerosol-phase species"]
    act = rxn.get("aerosol-phase activity coefficient")
    inst = []   # (rep index, unique name, act unique name, phase id)
    for ri, rep in enumerate(reps):
        names = rep.names(phases, phase, aero)
        if not names:
            continue
        acts = rep.names(phases, phase, act) if act else [None] * len(names)
        if len(acts) != len(names):
            raise ValueError("activity coefficient instances do not match the species")
        pids = rep.phase_ids(phases, phase)
        for k, nm in enumerate(names):
            inst.append((ri, nm, acts[k], pids[k]))
    if not inst:
        raise ValueError(f"No aerosol phase instances for SIMPOL partitioning of {aero}")
    n = len(inst)
    n_elem = [reps[ri].num_jac_elem(phases, pid) for ri, _, _, pid in inst]
    E = sum(n_elem)
    ints = np.zeros(4 + 13 * n + 2 * E, np.int32)
    floats = np.zeros(10 + 4 * E, np.float64)
    ints[0] = n
    if gas not in gas_index:
        raise KeyError(f"Missing gas-phase species {gas}")
    ints[1] = gas_index[gas]
    loc_i, loc_f = 12 * n + 5, 11  # PHASE_INT_LOC_(1), PHASE_REAL_LOC_(1), 1-based
    for x, (ri, nm, an, pid) in enumerate(inst):
        rep = reps[ri]
        ints[4 + 10 * n + x] = loc_i          # PHASE_INT_LOC_(x+1), 0-based 4+10n+x
        ints[4 + 11 * n + x] = loc_f          # PHASE_REAL_LOC_(x+1)
        ints[loc_i - 1] = n_elem[x]           # NUM_AERO_PHASE_JAC_ELEM_
        ints[2 + x] = rep.state_id(nm)        # AERO_SPEC_
        ints[2 + n + x] = rep.state_id(an) if an else -1   # AERO_ACT_ID_
        ints[2 + 2 * n + x] = pid             # AERO_PHASE_ID_
        ints[2 + 3 * n + x] = ri + 1          # AERO_REP_ID_
        loc_i += 1 + 2 * n_elem[x]
        loc_f += 4 * n_elem[x]
    gp = db.props[gas]
    ap = db.props[aero]
    mw = float(ap["molecular weight [kg mol-1]"])
    if "N star" in gp:
        ns = float(gp["N star"])
        dh = (-10.0 * (ns - 1.0) + 7.53 * (ns ** (2.0 / 3.0) - 1.0) - 1.0) * 4184.0
        ds = (-32.0 * (ns - 1.0) + 9.21 * (ns ** (2.0 / 3.0) - 1.0) - 1.3) * 4.184
    else:
        dh = ds = 0.0
    b = [float(v) for v in rxn["B"]]
    if len(b) != 4:
        raise ValueError("Incorrect number of 'B' parameters")
    floats[0], floats[1] = dh, ds
    floats[2] = float(gp["diffusion coeff [m2 s-1]"])
    floats[3] = math.sqrt(8.0 * UNIV_GAS_CONST / (PI * float(gp["molecular weight [kg mol-1]"])))
    floats[4:8] = b
    floats[8] = UNIV_GAS_CONST / mw * 1.0e6
    floats[9] = mw
    return PackedRxn(RXN_SIMPOL_PHASE_TRANSFER, ints, floats, 4, str(rxn.get("rxn id", "")))


def pack_hl(rxn: dict, db: _SpeciesDB, gas_index: dict[str, int], reps: list[AeroRep],
            phases: list[AeroPhase]) -> PackedRxn:
    """HL_PHASE_TRANSFER (src/rxns/rxn_HL_phase_transfer.F90:170-398).

    ints: ``[NUM_AERO_PHASE_, GAS_SPEC_, DERIV_ID_(0..n), JAC_ID_(0..5n),
    PHASE_INT_LOC_(n), PHASE_REAL_LOC_(n)]`` then per instance ``[AERO_SPEC_,
    AERO_WATER_, AERO_PHASE_ID_, AERO_REP_ID_, NUM_AERO_PHASE_JAC_ELEM_,
    PHASE_JAC_ID_(2 x elements)]``; floats: ``[DELTA_H_, DELTA_S_,
    DIFF_COEFF_, PRE_C_AVG_, A_, C_, CONV_, MW_]`` then per instance
    ``[SMALL_WATER_CONC_, EFF_RAD_JAC_ELEM_(e), NUM_CONC_JAC_ELEM_(e)]``."""
    gas = rxn["gas-phase species"]
    phase = rxn["aerosol phase"]
    aero = rxn["aerosol-phase species"]
    water = rxn.get("aerosol-phase water")
    if water is None:
        raise ValueError(f"Missing aerosol-phase water for HL partitioning of {gas} to {aero}")
    inst = []   # (rep index, species unique name, water unique name, phase id)
    for ri, rep in enumerate(reps):
        names = rep.names(phases, phase, aero)
        if not names:
            continue
        wnames = rep.names(phases, phase, water)
        if len(wnames) != len(names):
            raise ValueError(f"Missing species {aero} or {water} in phase {phase}")
        pids = rep.phase_ids(phases, phase)
        for k, nm in enumerate(names):
            inst.append((ri, nm, wnames[k], pids[k]))
    if not inst:
        raise ValueError(f"No aerosol phase instances for HL partitioning of {aero}")
    n = len(inst)
    n_elem = [reps[ri].num_jac_elem(phases, pid) for ri, _, _, pid in inst]
    E = sum(n_elem)
    ints = np.zeros(4 + 13 * n + 2 * E, np.int32)
    floats = np.zeros(8 + n + 2 * E, np.float64)
    ints[0] = n
    if gas not in gas_index:
        raise KeyError(f"Missing gas-phase species {gas}")
    ints[1] = gas_index[gas]
    loc_i, loc_f = 8 * n + 5, 9  # PHASE_INT_LOC_(1), PHASE_REAL_LOC_(1), 1-based
    for x, (ri, nm, wn, pid) in enumerate(inst):
        rep = reps[ri]
        ints[4 + 6 * n + x] = loc_i
        ints[4 + 7 * n + x] = loc_f
        li = loc_i - 1
        ints[li] = rep.state_id(nm)        # AERO_SPEC_
        ints[li + 1] = rep.state_id(wn)    # AERO_WATER_
        ints[li + 2] = pid                 # AERO_PHASE_ID_
        ints[li + 3] = ri + 1              # AERO_REP_ID_
        ints[li + 4] = n_elem[x]           # NUM_AERO_PHASE_JAC_ELEM_
        loc_i += 5 + 2 * n_elem[x]
        loc_f += 1 + 2 * n_elem[x]
    assert loc_i - 1 == ints.size and loc_f - 1 == floats.size
    gp = db.props[gas]
    ap = db.props[aero]
    mw = float(ap["molecular weight [kg mol-1]"])
    for key in ("HLC(298K) [M Pa-1]", "HLC exp factor [K]", "diffusion coeff [m2 s-1]",
                "molecular weight [kg mol-1]"):
        if key not in gp:
            raise KeyError(f"Missing '{key}' for gas-phase species {gas} of HL partitioning")
    if "N star" in gp:
        ns = float(gp["N star"])
        dh = (-10.0 * (ns - 1.0) + 7.53 * (ns ** (2.0 / 3.0) - 1.0) - 1.0) * 4184.0
        ds = (-32.0 * (ns - 1.0) + 9.21 * (ns ** (2.0 / 3.0) - 1.0) - 1.3) * 4.184
    else:
        dh = ds = 0.0
    floats[0], floats[1] = dh, ds
    floats[2] = float(gp["diffusion coeff [m2 s-1]"])
    # sqrt(8.0*R/(pi*MW)): the Fortran 8.0 is default-kind, R and pi are dp
    floats[3] = math.sqrt(8.0 * UNIV_GAS_CONST / (PI * float(gp["molecular weight [kg mol-1]"])))
    floats[4] = float(gp["HLC(298K) [M Pa-1]"])
    floats[5] = float(gp["HLC exp factor [K]"])
    floats[6] = UNIV_GAS_CONST / mw * 1.0e6
    floats[7] = mw
    return PackedRxn(RXN_HL_PHASE_TRANSFER, ints, floats, 4, str(rxn.get("rxn id", "")))


def pack_aqueous_equilibrium(rxn: dict, db: _SpeciesDB, reps: list[AeroRep],
                             phases: list[AeroPhase]) -> PackedRxn:
    """AQUEOUS_EQUILIBRIUM (src/rxns/rxn_aqueous_equilibrium.F90:170-493).

    ints: ``[NUM_REACT_, NUM_PROD_, NUM_AERO_PHASE_, REACT_(phase, r),
    PROD_(phase, p), WATER_(phase), ACTIVITY_COEFF_(phase), DERIV_ID_ ...,
    JAC_ID_ ...]``; floats: ``[A_, C_, RATE_CONST_REVERSE_, WATER_CONC_,
    ACTIVITY_COEFF_VALUE_, MASS_FRAC_TO_M_(r, p), REACT_CONC_(r),
    PROD_CONC_(p), SMALL_WATER_CONC_(phase), SMALL_CONC_(phase)]``; one env
    parameter (the forward rate constant)."""
    phase = rxn["aerosol phase"]
    water = rxn.get("aerosol-phase water")
    if water is None:
        raise ValueError("Missing aerosol-phase water for aqueous equilibrium reaction")

    def expand(block: dict) -> list[str]:
        out = []
        for name, props in (block or {}).items():
            out.extend([name] * int((props or {}).get("qty", 1)))
        return out

    react, prod = expand(rxn.get("reactants")), expand(rxn.get("products"))
    nr, np_ = len(react), len(prod)
    ns = nr + np_
    present = [ri for ri, rep in enumerate(reps) if rep.phase_ids(phases, phase)]
    n_phase = sum(len(reps[ri].names(phases, phase, water)) for ri in present)
    if n_phase == 0:
        raise ValueError(f"No aerosol phase '{phase}' present.")
    ints = np.zeros(3 + n_phase * (ns * (ns + 4) + 2), np.int32)
    floats = np.zeros(5 + 2 * ns + 2 * n_phase, np.float64)
    ints[0], ints[1], ints[2] = nr, np_, n_phase
    floats[0] = float(rxn.get("A", 1.0))
    floats[1] = float(rxn.get("C", 0.0))
    if "k_reverse" not in rxn:
        raise ValueError("Missing 'k_reverse' for aqueous equilibrium reaction")
    kr = float(rxn["k_reverse"])
    if str(rxn.get("time_unit", "")).strip() == "MIN":
        kr = kr / 60.0
    floats[2] = kr
    for k, name in enumerate(react + prod):
        if name not in db.props or "molecular weight [kg mol-1]" not in db.props[name]:
            raise KeyError(f"Missing 'molecular weight' for species '{name}' in aqueous "
                           f"equilibrium reaction.")
        floats[5 + k] = 1.0e3 / float(db.props[name]["molecular weight [kg mol-1]"])
    ion_pair = rxn.get("ion pair", "")
    o_prod = 3 + nr * n_phase
    o_water = 3 + ns * n_phase
    o_act = o_water + n_phase
    base = 0
    for ri in present:
        rep = reps[ri]
        wn = rep.names(phases, phase, water)
        k = len(wn)
        for j in range(k):
            ints[o_water + base + j] = rep.state_id(wn[j])
        if ion_pair:
            an = rep.names(phases, phase, ion_pair)
            if len(an) != k:
                raise ValueError(f"Incorrect instances of ion pair '{ion_pair}' in phase "
                                 f"'{phase}' in an aqueous equilibrium reaction")
            if db.var_type_of(ion_pair) != CHEM_SPEC_ACTIVITY_COEFF:
                raise ValueError(f"Ion pair '{ion_pair}' must have type 'ION_PAIR' to be used "
                                 f"as an ion pair in an aqueous equilibrium reaction.")
            for j in range(k):
                ints[o_act + base + j] = rep.state_id(an[j])
        for i, name in enumerate(react):
            un = rep.names(phases, phase, name)
            if len(un) != k:
                raise ValueError(f"Incorrect instances of reactant '{name}' in phase '{phase}' "
                                 f"in an aqueous equilibrium reaction")
            for j in range(k):
                ints[3 + (base + j) * nr + i] = rep.state_id(un[j])
        for i, name in enumerate(prod):
            un = rep.names(phases, phase, name)
            if len(un) != k:
                raise ValueError(f"Incorrect instances of product '{name}' in phase '{phase}' "
                                 f"in an aqueous equilibrium reaction")
            for j in range(k):
                ints[o_prod + (base + j) * np_ + i] = rep.state_id(un[j])
        base += k
    return PackedRxn(RXN_AQUEOUS_EQUILIBRIUM, ints, floats, 1, str(rxn.get("rxn id", "")))


def pack_wet_deposition_phase(rxn: dict, reps: list[AeroRep],
                              phases: list[AeroPhase]) -> PackedRxn:
    from .mechanism import pack_wet_deposition

    ids = []
    for rep in reps:
        ids += [rep.state_id(nm) for nm in rep.names(phases, rxn["aerosol phase"])]
    if not ids:
        raise ValueError(f"No aerosol phase instances for wet deposition of {rxn['aerosol phase']}")
    return pack_wet_deposition(ids, float(rxn.get("scaling factor", 1.0)), str(rxn.get("rxn id", "")))


def _instances(reps: list[AeroRep], phases: list[AeroPhase], phase: str,
               spec: str) -> list[int]:
    """1-based state ids of a species in every instance of a phase, over the
    representations in order (unique_names + spec_state_id)."""
    out = []
    for rep in reps:
        out += [rep.state_id(nm) for nm in rep.names(phases, phase, spec)]
    return out


def _relative_id(reps, phases, phase, spec, water_ids, what) -> int:
    """State id of spec relative to the aerosol water of the same instance,
    the same for every instance (the Fortran packers' relative ids)."""
    ids = _instances(reps, phases, phase, spec)
    if len(ids) != len(water_ids):
        raise ValueError(f"Incorrect number of instances of {what} '{spec}' in phase '{phase}'")
    rel = {i - w for i, w in zip(ids, water_ids)}
    if len(rel) != 1:
        raise ValueError(f"{what} '{spec}' is not at the same place in every instance")
    return rel.pop()


def _ion_pair_ions(ions: dict, db: _SpeciesDB, what: str) -> list[tuple[str, int, float, int]]:
    """(name, qty, molecular weight, charge) of the two ions of a pair, in
    their JSON order; the pair must be neutral."""
    if len(ions) != 2:
        raise ValueError(f"Invalid number of unique ions for ion pair in {what}: "
                         f"expected 2, got {len(ions)}")
    out = []
    total = 0
    for ion, props in ions.items():
        qty = int((props or {}).get("qty", 1))
        if ion not in db.props:
            raise KeyError(f"Missing species properties for ion '{ion}' in {what}")
        sp = db.props[ion]
        if "molecular weight [kg mol-1]" not in sp or "charge" not in sp:
            raise KeyError(f"Missing molecular weight or charge for ion '{ion}' in {what}")
        charge = int(sp["charge"])
        if charge == 0:
            raise ValueError(f"Neutral species '{ion}' not allowed in an ion pair in {what}")
        total += qty * charge
        out.append((ion, qty, float(sp["molecular weight [kg mol-1]"]), charge))
    if total != 0:
        raise ValueError(f"Charge imbalance for an ion pair in {what}: total charge {total}")
    return out


def pack_zsr_aerosol_water(obj: dict, db: _SpeciesDB, gas_index: dict[str, int],
                           reps: list[AeroRep], phases: list[AeroPhase]) -> SubModel:
    """SUB_MODEL_ZSR_AEROSOL_WATER
    (src/sub_models/sub_model_ZSR_aerosol_water.F90:215-500).

    ints: ``[NUM_PHASE_, GAS_WATER_ID_, NUM_ION_PAIR_, TOTAL_INT_PARAM_,
    TOTAL_FLOAT_PARAM_, PHASE_ID_(p), PAIR_INT_PARAM_LOC_(x),
    PAIR_FLOAT_PARAM_LOC_(x)]`` and per ion pair, JACOBSON: ``[TYPE_ 1,
    NUM_CATION_, NUM_ANION_, CATION_ID_, ANION_ID_, NUM_Y_, GAS_WATER_JAC_ID_
    (p), CATION_JAC_ID_(p), ANION_JAC_ID_(p)]``, floats ``[low_RH_,
    CATION_MW_, ANION_MW_, Y_(j)]``; EQSAM: ints ``[TYPE_ 2, NUM_ION_,
    GAS_WATER_JAC_ID_(p), ION_ID_(y), ION_JAC_ID_(p, y)]``, floats ``[NW_,
    ZW_, ION_PAIR_MW_, ION_MW_(y)]``.  Ion and water ids are relative to the
    phase instance's aerosol water; Jacobian ids are written by the solver.
    One env parameter (ppm of gas water -> relative humidity)."""
    what = "ZSR aerosol water"
    phase = obj["aerosol phase"]
    water = obj["aerosol-phase water"]
    if db.var_type_of(water) != CHEM_SPEC_CONSTANT:
        raise ValueError(f"ZSR calculated species {water} must be of tracer type CONSTANT")
    water_ids = _instances(reps, phases, phase, water)
    n_phase = len(water_ids)
    if n_phase == 0:
        raise ValueError(f"Aerosol phase '{phase}' not present in any aerosol representation "
                         f"for {what}")
    pairs = list((obj.get("ion pairs") or {}).items())
    if not pairs:
        raise ValueError(f"Empty ion pair set in {what}")
    n_int = 5 + n_phase + 2 * len(pairs)
    n_flt = 0
    for _, pr in pairs:
        if pr["type"] == "JACOBSON":
            n_int += 6 + 3 * n_phase
            n_flt += 3 + len(pr["Y_j"])
        elif pr["type"] == "EQSAM":
            n_ion = len(pr["ions"])
            n_int += 2 + n_phase + (1 + n_phase) * n_ion
            n_flt += 3 + n_ion
        else:
            raise ValueError(f"Invalid activity type specified for {what}: '{pr['type']}'")
    ints = np.zeros(n_int, np.int32)
    flts = np.zeros(n_flt, np.float64)
    gw = obj["gas-phase water"]
    if gw not in gas_index:
        raise KeyError(f"Cannot find gas-phase water species '{gw}' for {what}")
    ints[0:5] = (n_phase, gas_index[gw], len(pairs), n_int, n_flt)
    ints[5:5 + n_phase] = water_ids
    ii, ff = 5 + n_phase + 2 * len(pairs), 0
    for x, (pname, pr) in enumerate(pairs):
        ints[5 + n_phase + x] = ii + 1
        ints[5 + n_phase + len(pairs) + x] = ff + 1
        if pr["type"] == "JACOBSON":
            ints[ii] = 1
            ys = [float(v) for v in pr["Y_j"]]
            ints[ii + 5] = len(ys)
            flts[ff + 3:ff + 3 + len(ys)] = ys
            if "low RH" not in pr:
                raise KeyError(f"Missing 'low RH' value for ion pair '{pname}' in {what}")
            flts[ff] = float(pr["low RH"])
            for ion, qty, mw, charge in _ion_pair_ions(pr["ions"], db, what):
                rel = _relative_id(reps, phases, phase, ion, water_ids, "ion")
                if charge > 0:
                    ints[ii + 1], flts[ff + 1], ints[ii + 3] = qty, mw, rel
                else:
                    ints[ii + 2], flts[ff + 2], ints[ii + 4] = qty, mw, rel
            ii += 6 + 3 * n_phase
            ff += 3 + len(ys)
        else:
            ions = list(pr["ions"].keys())
            flts[ff], flts[ff + 1], flts[ff + 2] = float(pr["NW"]), float(pr["ZW"]), float(pr["MW"])
            ints[ii] = 2
            ints[ii + 1] = len(ions)
            for y, ion in enumerate(ions):
                if ion not in db.props or "molecular weight [kg mol-1]" not in db.props[ion]:
                    raise KeyError(f"Missing molecular weight for ion '{ion}' in {what}")
                flts[ff + 3 + y] = float(db.props[ion]["molecular weight [kg mol-1]"])
                ints[ii + 2 + n_phase + y] = _relative_id(reps, phases, phase, ion, water_ids,
                                                          "ion")
            ii += 2 + n_phase + (1 + n_phase) * len(ions)
            ff += 3 + len(ions)
    return SubModel(SUB_MODEL_ZSR_AEROSOL_WATER, ints, flts, 1, str(obj.get("name", "")))


def pack_pdfite(obj: dict, db: _SpeciesDB, gas_index: dict[str, int], reps: list[AeroRep],
                phases: list[AeroPhase]) -> SubModel:
    """SUB_MODEL_PDFITE (src/sub_models/sub_model_PDFiTE.F90:250-700).

    The ion pairs are those of "calculate for" in their order, then every
    further ion pair that only appears as an interaction partner, in order
    of first appearance (these get no interactions).  ints (initialised to
    9999): ``[NUM_PHASE_, GAS_WATER_ID_, NUM_ION_PAIRS_, TOTAL_INT_PARAM_,
    TOTAL_FLOAT_PARAM_, PHASE_ID_(p), PAIR_INT_PARAM_LOC_(x),
    PAIR_FLOAT_PARAM_LOC_(x)]``, per ion pair ``[ION_PAIR_ACT_ID_,
    NUM_CATION_, NUM_ANION_, CATION_ID_, ANION_ID_, NUM_INTER_,
    JAC_WATER_ID_(p), JAC_CATION_ID_(p, y), JAC_ANION_ID_(p, y), NUM_B_(i),
    INTER_SPEC_ID_(i), INTER_SPEC_LOC_(i)]``; floats (initialised to 9999)
    per ion pair ``[CATION_MW_, ANION_MW_, CATION_N_, ANION_N_]`` then per
    interaction ``[MIN_RH_, MAX_RH_, B_(z)]``.  One env parameter."""
    what = "PD-FiTE activity sub-model"
    phase = obj["aerosol phase"]
    water = obj["aerosol-phase water"]
    water_ids = _instances(reps, phases, phase, water)
    n_phase = len(water_ids)
    if n_phase == 0:
        raise ValueError(f"Aerosol phase '{phase}' not present in any aerosol representation "
                         f"for {what}")
    calc = list((obj.get("calculate for") or {}).items())
    names = [nm for nm, _ in calc]
    n_inter_total = 0
    for _, pr in calc:
        for it in pr["interactions"]:
            n_inter_total += 1
            if it["ion pair"] not in names:
                names.append(it["ion pair"])
    n = len(names)
    n_int = 5 + n_phase + 3 * n_inter_total + (8 + (1 + 2 * n) * n_phase) * n
    n_flt = sum(2 + len(it["B"]) for _, pr in calc for it in pr["interactions"]) + 4 * n
    ints = np.full(n_int, 9999, np.int32)
    flts = np.full(n_flt, 9999.0, np.float64)
    gw = obj["gas-phase water"]
    if gw not in gas_index:
        raise KeyError(f"Cannot find gas-phase water species '{gw}' for {what}")
    ints[0:5] = (n_phase, gas_index[gw], n, n_int, n_flt)
    ints[5:5 + n_phase] = water_ids
    ii, ff = 5 + n_phase + 2 * n, 0
    P = n_phase
    for x, pname in enumerate(names):
        ints[5 + P + x] = ii + 1
        ints[5 + P + n + x] = ff + 1
        if db.var_type_of(pname) != CHEM_SPEC_ACTIVITY_COEFF:
            raise ValueError(f"Ion pair '{pname}' must have type ION_PAIR in {what}")
        ints[ii] = _relative_id(reps, phases, phase, pname, water_ids, "ion pair")
        ions = db.props[pname].get("ions")
        if not ions:
            raise KeyError(f"Missing ions for ion pair '{pname}' in {what}")
        for ion, qty, mw, charge in _ion_pair_ions(ions, db, what):
            rel = _relative_id(reps, phases, phase, ion, water_ids, "ion")
            if charge > 0:
                ints[ii + 1], flts[ff], ints[ii + 3] = qty, mw, rel
            else:
                ints[ii + 2], flts[ff + 1], ints[ii + 4] = qty, mw, rel
        ff += 4
        base = ii
        ii += 6 + (1 + 2 * n) * P
        if x < len(calc):
            inters = calc[x][1]["interactions"]
            ni = len(inters)
            ints[base + 5] = ni
            o_b = base + 6 + (1 + 2 * n) * P
            for y, it in enumerate(inters):
                ints[o_b + 2 * ni + y] = ff + 1          # INTER_SPEC_LOC_
                ints[o_b + ni + y] = names.index(it["ion pair"]) + 1  # INTER_SPEC_ID_
                lo, hi = float(it["min RH"]), float(it["max RH"])
                if not (0.0 <= lo < 1.0) or not (0.0 < hi <= 1.0):
                    raise ValueError(f"Invalid RH range for ion pair '{pname}' in {what}")
                bs = [float(v) for v in it["B"]]
                ints[o_b + y] = len(bs)                    # NUM_B_
                flts[ff], flts[ff + 1] = lo, hi
                flts[ff + 2:ff + 2 + len(bs)] = bs
                ff += 2 + len(bs)
                ii += 3
        else:
            ints[base + 5] = 0
    return SubModel(SUB_MODEL_PDFITE, ints, flts, 1, str(obj.get("name", "")))


def load_aerosol_mechanism(files: Iterable[str], name: str | None = None) -> Mechanism:
    """Loads CAMP JSON input with aerosol phases and modal/binned mass
    representations (plus any gas-phase content), packed for the C solver.
    Host-rate reactions get ids 1, 2, ... in mechanism order and the
    representations ids 1, 2, ... in order."""
    db = _SpeciesDB()
    mechs: list[tuple[str, list[dict]]] = []
    phase_json: list[dict] = []
    rep_json: list[dict] = []
    sub_json: list[dict] = []
    rel_tol = None
    for path in files:
        for obj in _read_json(path).get("camp-data", []):
            t = obj.get("type")
            if t == "CHEM_SPEC":
                db.add(obj)
            elif t == "MECHANISM":
                for mname, mrx in mechs:
                    if mname == obj["name"]:
                        mrx.extend(obj.get("reactions", []))
                        break
                else:
                    mechs.append((obj["name"], list(obj.get("reactions", []))))
            elif t == "AERO_PHASE":
                for p in phase_json:
                    if p["name"] == obj["name"]:
                        p["species"] = list(p["species"]) + list(obj.get("species", []))
                        break
                else:
                    phase_json.append({"name": obj["name"], "species": list(obj.get("species", []))})
            elif t is not None and t.startswith("AERO_REP_"):
                if t != "AERO_REP_MODAL_BINNED_MASS":
                    raise NotImplementedError(f"aerosol representation {t} is not supported")
                rep_json.append(obj)
            elif t is not None and t.startswith("SUB_MODEL_"):
                if t not in SUB_MODEL_PRIORITY:
                    raise NotImplementedError(f"sub-model {t} is not supported")
                if any(o.get("name") == obj.get("name") for o in sub_json):
                    raise NotImplementedError(f"sub-model '{obj.get('name')}' is defined twice")
                # camp_core places a new sub-model before the first one of
                # larger priority value (src/camp_core.F90:575-605)
                at = next((i for i, o in enumerate(sub_json)
                           if SUB_MODEL_PRIORITY[t] < SUB_MODEL_PRIORITY[o["type"]]), len(sub_json))
                sub_json.insert(at, obj)
            elif t == "RELATIVE_TOLERANCE":
                rel_tol = float(obj["value"])
    gas = db.gas_species()
    gas_index = {n: i + 1 for i, n in enumerate(gas)}
    phases = [pack_aero_phase(p["name"], p["species"], db) for p in phase_json]
    reps = []
    state = len(gas) + 1
    for obj in rep_json:
        rep = pack_modal_binned(obj["name"], obj, phases, state)
        state += len(rep.unique_names)
        reps.append(rep)
    for i, rep in enumerate(reps):
        rep.ints[3] = i + 1   # AERO_REP_ID_ as set_id gives it

    def gas_id(n: str) -> int:
        if n not in gas_index:
            raise KeyError(f"Missing species: {n}")
        return gas_index[n]

    rxns = []
    for _, rx in mechs:
        for r in rx:
            if r["type"] == "SIMPOL_PHASE_TRANSFER":
                rxns.append(pack_simpol(r, db, gas_index, reps, phases))
            elif r["type"] == "HL_PHASE_TRANSFER":
                rxns.append(pack_hl(r, db, gas_index, reps, phases))
            elif r["type"] == "AQUEOUS_EQUILIBRIUM":
                rxns.append(pack_aqueous_equilibrium(r, db, reps, phases))
            elif r["type"] == "WET_DEPOSITION":
                rxns.append(pack_wet_deposition_phase(r, reps, phases))
            else:
                rxns.append(pack_reaction(r, gas_id))
    rate_ids = assign_rate_ids(rxns)
    subs = []
    for obj in sub_json:
        pack = pack_zsr_aerosol_water if obj["type"] == "SUB_MODEL_ZSR_AEROSOL_WATER" else pack_pdfite
        subs.append(pack(obj, db, gas_index, reps, phases))
    species = list(gas)
    var_type = [db.var_type_of(n) for n in gas]
    abs_tol = [db.abs_tol_of(n) for n in gas]
    for rep in reps:
        for un in rep.unique_names:
            sp = un.rsplit(".", 1)[1]
            species.append(un)
            var_type.append(db.var_type_of(sp))
            abs_tol.append(db.abs_tol_of(sp))
    props = {n: dict(db.props[n]) for n in gas}
    return Mechanism(
        name=name or (mechs[0][0] if mechs else "mechanism"), species=species,
        var_type=np.asarray(var_type, np.int32), abs_tol=np.asarray(abs_tol, np.float64),
        rel_tol=rel_tol if rel_tol is not None else 1.0e-8, rxns=rxns, rate_ids=rate_ids,
        species_props=props, aero_phases=phases, aero_reps=reps, sub_models=subs)


def modal_sections(mech: Mechanism) -> list[tuple[int, int]]:
    """(representation index, section index) of every mode: the GMD/GSD
    host-update targets, in representation then section order."""
    return [(ri, si) for ri, rep in enumerate(mech.aero_reps)
            for si, sec in enumerate(rep.sections) if sec.kind == MODAL]


def ion_pair_check(mech: Mechanism) -> int:
    """Number of activity-coefficient (ion-pair) state variables."""
    return int(np.count_nonzero(mech.var_type == CHEM_SPEC_ACTIVITY_COEFF))
