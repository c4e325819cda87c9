"""CAMP mechanism loading and packing (host side of the drop-in boundary).

The reference's Fortran layer reads the CAMP JSON input files, orders the
state array and packs every reaction into the ``int``/``double`` blocks that
``rxn_add_condensed_data`` receives (``src/camp_core.F90:303-798``,
``src/rxns/rxn_*.F90`` ``initialize``).  This module restates that layer for
the gas-phase reaction types of the cb05cl_ae5 mechanism, so that the C entry
points of ``libcamp_b200`` can be driven from Python exactly as the Fortran
caller drives them.

Packed layouts (one block per reaction, the type id is passed separately):

* ARRHENIUS (type 1, ``src/rxns/rxn_arrhenius.c:20-36``)
  ints  ``[NUM_REACT, NUM_PROD, REACT.., PROD.., DERIV_ID.., JAC_ID..]``
  reals ``[A, B, C, D, E, CONV, YIELD..]``; 1 env parameter (rate constant)
* TROE (type 2, ``src/rxns/rxn_troe.c:19-41``)
  reals ``[K0_A*1e6, K0_B, K0_C, KINF_A, KINF_B, KINF_C, FC, N, SCALING, CONV, YIELD..]``
* CMAQ_H2O2 (type 3, ``src/rxns/rxn_CMAQ_H2O2.c:20-37``)
  reals ``[k1_A, k1_B, k1_C, k2_A*1e6, k2_B, k2_C, CONV, YIELD..]``
* CMAQ_OH_HNO3 (type 4, ``src/rxns/rxn_CMAQ_OH_HNO3.c:20-41``)
  reals ``[k0_A, k0_B, k0_C, k2_A, k2_B, k2_C, k3_A*1e6, k3_B, k3_C, SCALING, CONV, YIELD..]``
* PHOTOLYSIS (type 5, ``src/rxns/rxn_photolysis.c:20-33``)
  ints  ``[NUM_REACT, NUM_PROD, RXN_ID, REACT.., PROD.., DERIV_ID.., JAC_ID..]``
  reals ``[SCALING, YIELD..]``; 2 env parameters (rate constant, base rate)

REACT/PROD are 1-based state indices; DERIV_ID and JAC_ID are left zero and
filled in by the solver when it builds the Jacobian sparsity.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Callable, Iterable

import numpy as np

# State variable types, src/camp_common.h:34-38
CHEM_SPEC_UNKNOWN_TYPE = 0
CHEM_SPEC_VARIABLE = 1
CHEM_SPEC_CONSTANT = 2
CHEM_SPEC_PSSA = 3
CHEM_SPEC_ACTIVITY_COEFF = 4

# Reaction type ids, src/rxn_factory.F90:212-228 (= src/rxn_solver.c:19-35)
RXN_ARRHENIUS = 1
RXN_TROE = 2
RXN_CMAQ_H2O2 = 3
RXN_CMAQ_OH_HNO3 = 4
RXN_PHOTOLYSIS = 5
RXN_FIRST_ORDER_LOSS = 12
RXN_EMISSION = 13
RXN_WET_DEPOSITION = 14

RXN_TYPE_IDS = {
    "ARRHENIUS": RXN_ARRHENIUS,
    "TROE": RXN_TROE,
    "CMAQ_H2O2": RXN_CMAQ_H2O2,
    "CMAQ_OH_HNO3": RXN_CMAQ_OH_HNO3,
    "PHOTOLYSIS": RXN_PHOTOLYSIS,
    "FIRST_ORDER_LOSS": RXN_FIRST_ORDER_LOSS,
    "EMISSION": RXN_EMISSION,
    "WET_DEPOSITION": RXN_WET_DEPOSITION,
}

# Types whose rate the host sets per cell through rxn_update_data
# (src/rxn_solver.c:735-760); each such reaction is one column of the
# per-cell base rates, in mechanism order.
HOST_RATE_TYPES = (RXN_PHOTOLYSIS, RXN_FIRST_ORDER_LOSS, RXN_EMISSION, RXN_WET_DEPOSITION)

# Physical constants, src/constants.F90:37-41
BOLTZMANN = 1.3806505e-23
AVOGADRO = 6.02214179e23
UNIV_GAS_CONST = 8.314472
# default species absolute tolerance, src/chem_spec_data.F90:63
DEFAULT_ABS_TOL = 1.0e-14
# #/cc -> ppm conversion prefactor set by the gas packers
CONV = AVOGADRO / UNIV_GAS_CONST * 10.0 ** (-12.0)


@dataclass
class PackedRxn:
    """One reaction as the Fortran caller hands it to rxn_add_condensed_data."""

    rxn_type: int
    ints: np.ndarray  # int32
    floats: np.ndarray  # float64
    n_env: int
    label: str = ""


SUB_MODEL_UNIFAC = 1             # src/sub_model_solver.c:16-18
SUB_MODEL_ZSR_AEROSOL_WATER = 2
SUB_MODEL_PDFITE = 3


@dataclass
class SubModel:
    """One sub-model as sub_model_add_condensed_data receives it."""

    sub_type: int
    ints: np.ndarray
    floats: np.ndarray
    n_env: int
    name: str = ""

    def to_dict(self) -> dict:
        return {"type": int(self.sub_type), "ints": [int(v) for v in self.ints],
                "floats": [float(v) for v in self.floats], "n_env": int(self.n_env),
                "name": self.name}

    @classmethod
    def from_dict(cls, d: dict) -> "SubModel":
        return cls(int(d["type"]), np.asarray(d["ints"], np.int32),
                   np.asarray(d["floats"], np.float64), int(d["n_env"]), d.get("name", ""))


@dataclass
class Mechanism:
    """State layout plus packed reactions for one solver instance."""

    name: str
    species: list[str]
    var_type: np.ndarray  # int32 [n_state_var]
    abs_tol: np.ndarray  # float64 [n_state_var]
    rel_tol: float
    rxns: list[PackedRxn]
    # RXN_ID_ of each reaction of a host-rate type -> its index in ``rxns``
    rate_ids: dict[int, int] = field(default_factory=dict)
    species_props: dict[str, dict] = field(default_factory=dict)
    # aerosol phases and representations as aero_phase_add_condensed_data /
    # aero_rep_add_condensed_data receive them (camp_b200.aerosol)
    aero_phases: list = field(default_factory=list)
    aero_reps: list = field(default_factory=list)
    # sub-models in the order sub_model_add_condensed_data receives them
    # (camp_core sorts them by priority: ZSR water before PD-FiTE activity)
    sub_models: list = field(default_factory=list)

    @property
    def n_state_var(self) -> int:
        return len(self.species)

    @property
    def n_dep_var(self) -> int:
        return int(np.count_nonzero(self.var_type == CHEM_SPEC_VARIABLE))

    @property
    def n_rxn(self) -> int:
        return len(self.rxns)

    @property
    def n_rxn_int_param(self) -> int:
        return int(sum(r.ints.size for r in self.rxns))

    @property
    def n_rxn_float_param(self) -> int:
        return int(sum(r.floats.size for r in self.rxns))

    @property
    def n_rxn_env_param(self) -> int:
        return int(sum(r.n_env for r in self.rxns))

    def aero_sizes(self) -> list[int]:
        """solver_new's aerosol counts: phases (count, ints, floats) and
        representations (count, ints, floats, env parameters)."""
        ph, rp = self.aero_phases, self.aero_reps
        return [len(ph), int(sum(p.ints.size for p in ph)), int(sum(p.floats.size for p in ph)),
                len(rp), int(sum(r.ints.size for r in rp)), int(sum(r.floats.size for r in rp)),
                int(sum(r.n_env for r in rp))]

    def sub_sizes(self) -> list[int]:
        """solver_new's sub-model counts: number, ints, floats, env parameters."""
        sm = self.sub_models
        return [len(sm), int(sum(m.ints.size for m in sm)), int(sum(m.floats.size for m in sm)),
                int(sum(m.n_env for m in sm))]

    def index(self, name: str) -> int:
        return self.species.index(name)

    def dep_index(self) -> np.ndarray:
        """State indices of the dependent (solver) variables, in order."""
        return np.nonzero(self.var_type == CHEM_SPEC_VARIABLE)[0]

    # --- serialisation of the packed form (fixtures travel without JSON) ---
    def to_dict(self) -> dict:
        return {
            "name": self.name,
            "species": list(self.species),
            "var_type": [int(v) for v in self.var_type],
            "abs_tol": [float(v) for v in self.abs_tol],
            "rel_tol": float(self.rel_tol),
            "rxns": [
                {
                    "type": int(r.rxn_type),
                    "ints": [int(v) for v in r.ints],
                    "floats": [float(v) for v in r.floats],
                    "n_env": int(r.n_env),
                    "label": r.label,
                }
                for r in self.rxns
            ],
            "rate_ids": {str(k): int(v) for k, v in self.rate_ids.items()},
            "init_conc": {
                n: float(p["init conc"]) for n, p in self.species_props.items() if "init conc" in p
            },
            "aero_phases": [p.to_dict() for p in self.aero_phases],
            "aero_reps": [r.to_dict() for r in self.aero_reps],
            "sub_models": [m.to_dict() for m in self.sub_models],
        }

    @classmethod
    def from_dict(cls, d: dict) -> "Mechanism":
        from .aerosol import AeroPhase, AeroRep

        rxns = [
            PackedRxn(
                int(r["type"]),
                np.asarray(r["ints"], dtype=np.int32),
                np.asarray(r["floats"], dtype=np.float64),
                int(r["n_env"]),
                r.get("label", ""),
            )
            for r in d["rxns"]
        ]
        return cls(
            name=d["name"],
            species=list(d["species"]),
            var_type=np.asarray(d["var_type"], dtype=np.int32),
            abs_tol=np.asarray(d["abs_tol"], dtype=np.float64),
            rel_tol=float(d["rel_tol"]),
            rxns=rxns,
            rate_ids={int(k): int(v)
                      for k, v in d.get("rate_ids", d.get("photo_ids", {})).items()},
            species_props={n: {"init conc": v} for n, v in d.get("init_conc", {}).items()},
            aero_phases=[AeroPhase.from_dict(p) for p in d.get("aero_phases", [])],
            aero_reps=[AeroRep.from_dict(r) for r in d.get("aero_reps", [])],
            sub_models=[SubModel.from_dict(m) for m in d.get("sub_models", [])],
        )

    def save(self, path: str) -> None:
        with open(path, "w") as fh:
            json.dump(self.to_dict(), fh, separators=(",", ":"))

    @classmethod
    def load(cls, path: str) -> "Mechanism":
        with open(path) as fh:
            return cls.from_dict(json.load(fh))

    def photolysis_rxns(self) -> list[int]:
        return [i for i, r in enumerate(self.rxns) if r.rxn_type == RXN_PHOTOLYSIS]

    def rate_rxns(self) -> list[int]:
        """Reactions of a host-rate type in mechanism order: column j of the
        per-cell base rates belongs to reaction rate_rxns()[j]."""
        return [i for i, r in enumerate(self.rxns) if r.rxn_type in HOST_RATE_TYPES]

    def rate_columns(self) -> list[tuple]:
        """Columns of the per-cell host-set values, in order: ("rxn", i) for
        every host-rate reaction (``rate_rxns``), then ("gmd", rep, section)
        and ("gsd", rep, section) for every mode of every aerosol
        representation (the targets of its GMD / GSD update data)."""
        cols: list[tuple] = [("rxn", i) for i in self.rate_rxns()]
        for ri, rep in enumerate(self.aero_reps):
            for si, sec in enumerate(rep.sections):
                if sec.kind == 2:  # MODAL
                    cols += [("gmd", ri, si), ("gsd", ri, si)]
        return cols

    def rate_id(self, rxn: int) -> int:
        """RXN_ID_ of a host-rate reaction (the id its update data carries)."""
        r = self.rxns[rxn]
        return int(r.ints[2] if r.rxn_type == RXN_PHOTOLYSIS else r.ints[0])


# ---------------------------------------------------------------------------
# JSON input
# ---------------------------------------------------------------------------


def _read_json(path: str) -> dict:
    with open(path) as fh:
        return json.load(fh)


def expand_config(config_path: str, path_map: Callable[[str], str] | None = None) -> list[str]:
    """File list of a CAMP config file (``{"camp-files": [...]}``).

    Relative entries are resolved against the config file's directory and then
    passed through ``path_map``, which lets a caller redirect the build-tree
    paths some reference configs use (``../../mechanisms_run/...``).
    """
    cfg = _read_json(config_path)
    base = os.path.dirname(os.path.abspath(config_path))
    out = []
    for f in cfg["camp-files"]:
        p = f if os.path.isabs(f) else os.path.normpath(os.path.join(base, f))
        out.append(path_map(p) if path_map else p)
    return out


class _SpeciesDB:
    """Restates the ordering/merging rules of src/chem_spec_data.F90.

    Species keep the order of their first appearance; later entries with the
    same name merge their properties (``add``, :714-761).  Unknown type
    defaults to VARIABLE and unknown phase to GAS (``initialize``, :320-338).
    """

    def __init__(self) -> None:
        self.names: list[str] = []
        self.props: dict[str, dict] = {}
        self.type: dict[str, int] = {}
        self.phase: dict[str, str] = {}

    def add(self, obj: dict) -> None:
        name = obj["name"]
        stype = CHEM_SPEC_UNKNOWN_TYPE
        phase = None
        props = {}
        for k, v in obj.items():
            if k == "name" or k == "type":
                continue
            if k == "tracer type":
                stype = {
                    "VARIABLE": CHEM_SPEC_VARIABLE,
                    "CONSTANT": CHEM_SPEC_CONSTANT,
                    "PSSA": CHEM_SPEC_PSSA,
                    "ION_PAIR": CHEM_SPEC_ACTIVITY_COEFF,
                    "ACTIVITY_COEFF": CHEM_SPEC_ACTIVITY_COEFF,
                }[v]
                if v == "ION_PAIR":
                    phase = "AEROSOL"
            elif k == "phase":
                phase = v
            else:
                props[k] = v
        if name not in self.props:
            self.names.append(name)
            self.props[name] = {}
            self.type[name] = CHEM_SPEC_UNKNOWN_TYPE
            self.phase[name] = None
        if stype != CHEM_SPEC_UNKNOWN_TYPE:
            old = self.type[name]
            if old not in (CHEM_SPEC_UNKNOWN_TYPE, stype):
                raise ValueError(f"Type mismatch for species {name}")
            self.type[name] = stype
        if phase is not None:
            old = self.phase[name]
            if old not in (None, phase):
                raise ValueError(f"Phase mismatch for species {name}")
            self.phase[name] = phase
        for k, v in props.items():
            if k in self.props[name] and not isinstance(v, dict):
                raise ValueError(f"Duplicate property {k} for species {name}")
            self.props[name][k] = v

    def gas_species(self) -> list[str]:
        return [n for n in self.names if (self.phase[n] or "GAS") == "GAS"]

    def var_type_of(self, name: str) -> int:
        t = self.type[name]
        return CHEM_SPEC_VARIABLE if t == CHEM_SPEC_UNKNOWN_TYPE else t

    def abs_tol_of(self, name: str) -> float:
        return float(self.props[name].get("absolute integration tolerance", DEFAULT_ABS_TOL))


def _expand_reactants(reactants: dict, gas_id: Callable[[str], int]) -> list[int]:
    out = []
    for name, props in reactants.items():
        sid = gas_id(name)
        qty = int((props or {}).get("qty", 1))
        out.extend([sid] * qty)
    return out


def _products(products: dict, gas_id: Callable[[str], int]) -> tuple[list[int], list[float]]:
    ids, ylds = [], []
    for name, props in products.items():
        ids.append(gas_id(name))
        ylds.append(float((props or {}).get("yield", 1.0)))
    return ids, ylds


def _int_block(n_int_prop: int, head: list[int], react: list[int], prod: list[int]) -> np.ndarray:
    nr, npd = len(react), len(prod)
    ints = np.zeros(n_int_prop + (nr + 2) * (nr + npd), dtype=np.int32)
    ints[0] = nr
    ints[1] = npd
    for i, v in enumerate(head):
        ints[2 + i] = v
    ints[n_int_prop : n_int_prop + nr] = react
    ints[n_int_prop + nr : n_int_prop + nr + npd] = prod
    return ints


def pack_species_rate(rtype: int, species: int, scaling: float = 1.0, label: str = "") -> PackedRxn:
    """FIRST_ORDER_LOSS or EMISSION of one state variable (1-based index),
    packed as src/rxns/rxn_first_order_loss.F90:169-220 and
    rxn_emission.F90:166-217 do: RXN_ID_ (-1 until the host assigns one),
    the species, then the DERIV_ID_ (and JAC_ID_) slots; SCALING_."""
    n_int = 4 if rtype == RXN_FIRST_ORDER_LOSS else 3
    ints = np.zeros(n_int, np.int32)
    ints[0], ints[1] = -1, species
    return PackedRxn(rtype, ints, np.asarray([scaling]), 2, label)


def pack_wet_deposition(species: list[int], scaling: float = 1.0, label: str = "") -> PackedRxn:
    """WET_DEPOSITION of the given state variables (1-based indices; the
    Fortran packer lists every species of the named aerosol phase in every
    instance of it, src/rxns/rxn_wet_deposition.F90:172-254): RXN_ID_,
    NUM_SPEC_, REACT_(s), DERIV_ID_(s), JAC_ID_(s); SCALING_."""
    ns = len(species)
    ints = np.zeros(2 + 3 * ns, np.int32)
    ints[0], ints[1] = -1, ns
    ints[2 : 2 + ns] = species
    return PackedRxn(RXN_WET_DEPOSITION, ints, np.asarray([scaling]), 2, label)


def pack_reaction(rxn: dict, gas_id: Callable[[str], int]) -> PackedRxn:
    """Packs one gas-phase reaction as its Fortran ``initialize`` does."""
    rtype = rxn["type"]
    if rtype not in RXN_TYPE_IDS:
        raise NotImplementedError(f"reaction type {rtype} is not supported")
    if rtype in ("FIRST_ORDER_LOSS", "EMISSION"):
        if "species" not in rxn:
            kind = "First-Order Loss" if rtype == "FIRST_ORDER_LOSS" else "Emission"
            raise ValueError(f"{kind} reaction is missing species name")
        return pack_species_rate(RXN_TYPE_IDS[rtype], gas_id(rxn["species"]),
                                 float(rxn.get("scaling factor", 1.0)),
                                 str(rxn.get("rxn id", "")))
    if rtype == "WET_DEPOSITION":
        raise NotImplementedError(
            "WET_DEPOSITION removes the species of an aerosol phase, and aerosol phases are "
            "not read from JSON here; build it with pack_wet_deposition")
    react = _expand_reactants(rxn["reactants"], gas_id)
    prod, ylds = _products(rxn.get("products", {}), gas_id)
    label = str(rxn.get("rxn id", ""))
    tunit_min = rxn.get("time unit") == "MIN"

    def g(key, default):
        return float(rxn.get(key, default))

    if rtype == "ARRHENIUS":  # src/rxns/rxn_arrhenius.F90:150-287
        A = g("A", 1.0)
        if tunit_min:
            A = A / 60.0
        if "Ea" in rxn:
            if "C" in rxn:
                raise ValueError("Received both Ea and C parameter for Arrhenius equation")
            C = -float(rxn["Ea"]) / BOLTZMANN
        else:
            C = g("C", 0.0)
        D = g("D", 300.0)
        B = g("B", 0.0)
        E = g("E", 0.0)
        if B != 0.0 and D == 0.0:
            raise ValueError("D cannot be zero if B is non-zero in Arrhenius reaction.")
        floats = [A, B, C, D, E, CONV] + ylds
        return PackedRxn(RXN_ARRHENIUS, _int_block(2, [], react, prod), np.asarray(floats), 1, label)
    if rtype == "TROE":  # src/rxns/rxn_troe.F90 initialize
        k0_A = g("k0_A", 1.0)
        scaling = 1.0 / 60.0 if tunit_min else 1.0
        floats = [
            k0_A * 1.0e6,
            g("k0_B", 0.0),
            g("k0_C", 0.0),
            g("kinf_A", 1.0),
            g("kinf_B", 0.0),
            g("kinf_C", 0.0),
            g("Fc", 0.6),
            g("N", 1.0),
            scaling,
            CONV,
        ] + ylds
        return PackedRxn(RXN_TROE, _int_block(2, [], react, prod), np.asarray(floats), 1, label)
    if rtype == "CMAQ_H2O2":  # src/rxns/rxn_CMAQ_H2O2.F90 initialize
        k1_A, k2_A = g("k1_A", 1.0), g("k2_A", 1.0)
        if tunit_min:
            k1_A, k2_A = k1_A / 60.0, k2_A / 60.0
        floats = [k1_A, g("k1_B", 0.0), g("k1_C", 0.0), k2_A * 1.0e6, g("k2_B", 0.0), g("k2_C", 0.0), CONV] + ylds
        return PackedRxn(RXN_CMAQ_H2O2, _int_block(2, [], react, prod), np.asarray(floats), 1, label)
    if rtype == "CMAQ_OH_HNO3":  # src/rxns/rxn_CMAQ_OH_HNO3.F90 initialize
        scaling = 1.0 / 60.0 if tunit_min else 1.0
        floats = [
            g("k0_A", 1.0),
            g("k0_B", 0.0),
            g("k0_C", 0.0),
            g("k2_A", 1.0),
            g("k2_B", 0.0),
            g("k2_C", 0.0),
            g("k3_A", 1.0) * 1.0e6,
            g("k3_B", 0.0),
            g("k3_C", 0.0),
            scaling,
            CONV,
        ] + ylds
        return PackedRxn(RXN_CMAQ_OH_HNO3, _int_block(2, [], react, prod), np.asarray(floats), 1, label)
    # PHOTOLYSIS, src/rxns/rxn_photolysis.F90 initialize; RXN_ID_ starts at -1
    floats = [g("scaling factor", 1.0)] + ylds
    return PackedRxn(RXN_PHOTOLYSIS, _int_block(3, [-1], react, prod), np.asarray(floats), 2, label)


def load_mechanism(files: Iterable[str], name: str | None = None) -> Mechanism:
    """Loads CAMP JSON input files and packs the gas-phase mechanism.

    Reactions whose rate the host sets (PHOTOLYSIS, FIRST_ORDER_LOSS,
    EMISSION) receive sequential ids (1, 2, ...) in mechanism order, which is
    what the reference's ``generate_int_id`` (src/rand.F90:644-656) hands out
    when a host model creates one update object per such reaction in that
    order (``test/chemistry/cb05cl_ae5/test_cb05cl_ae5.F90:293-310``).
    """
    db = _SpeciesDB()
    mechs: list[tuple[str, list[dict]]] = []
    rel_tol = None
    for path in files:
        data = _read_json(path)
        for obj in data.get("camp-data", []):
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
            elif t == "RELATIVE_TOLERANCE":
                v = float(obj["value"])
                if not (0.0 < v < 1.0):
                    raise ValueError(f"Invalid relative tolerance: {v}")
                rel_tol = v
    gas = db.gas_species()
    gas_index = {n: i + 1 for i, n in enumerate(gas)}

    def gas_id(n: str) -> int:
        if n not in gas_index:
            raise KeyError(f"Missing species: {n}")
        return gas_index[n]

    rxns: list[PackedRxn] = []
    for _, rx in mechs:
        for r in rx:
            rxns.append(pack_reaction(r, gas_id))
    rate_ids = assign_rate_ids(rxns)
    var_type = np.asarray([db.var_type_of(n) for n in gas], dtype=np.int32)
    abs_tol = np.asarray([db.abs_tol_of(n) for n in gas], dtype=np.float64)
    mech = Mechanism(
        name=name or (mechs[0][0] if mechs else "mechanism"),
        species=gas,
        var_type=var_type,
        abs_tol=abs_tol,
        rel_tol=rel_tol if rel_tol is not None else 1.0e-8,
        rxns=rxns,
        rate_ids=rate_ids,
        species_props={n: dict(db.props[n]) for n in gas},
    )
    return mech


def assign_rate_ids(rxns: list[PackedRxn]) -> dict[int, int]:
    """Gives every reaction of a host-rate type the next id of one sequence,
    in order, as a host creating one update object per such reaction does;
    returns id -> reaction index."""
    ids = {}
    for i, r in enumerate(rxns):
        if r.rxn_type not in HOST_RATE_TYPES:
            continue
        rid = len(ids) + 1
        r.ints[2 if r.rxn_type == RXN_PHOTOLYSIS else 0] = rid
        ids[rid] = i
    return ids


def reaction_summary(mech: Mechanism) -> dict:
    """Counts by type and by number of reactants (used by tests and docs)."""
    by_type: dict[int, int] = {}
    by_nr: dict[int, int] = {}
    for r in mech.rxns:
        by_type[r.rxn_type] = by_type.get(r.rxn_type, 0) + 1
        if r.rxn_type in (RXN_FIRST_ORDER_LOSS, RXN_WET_DEPOSITION):
            nr = 1
        elif r.rxn_type == RXN_EMISSION:
            nr = 0
        else:
            nr = int(r.ints[0])
        by_nr[nr] = by_nr.get(nr, 0) + 1
    return {"by_type": by_type, "by_n_react": by_nr}
