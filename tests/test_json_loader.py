"""The C++ reader/packer of CAMP JSON input (camp_b200_solver_from_json)
against the Python packer: the same state layout, tolerances and packed
reaction data, bit for bit (CPU only; no kernel runs)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from camp_b200 import _lib
from conftest import REF_ROOT

REF_CB05 = os.path.join(REF_ROOT, "mechanisms", "cb05cl_ae5")


def _cpp_solver(files, n_cells=2):
    lib = _lib.load()
    arr = (C.c_char_p * len(files))(*[f.encode() for f in files])
    h = lib.camp_b200_solver_from_json(arr, len(files), n_cells)
    assert h, _lib.last_error()
    return lib, h


def _compare(files, aerosol=False):
    from camp_b200.aerosol import load_aerosol_mechanism
    from camp_b200.mechanism import load_mechanism
    from camp_b200.solver import Solver

    mech = load_aerosol_mechanism(files) if aerosol else load_mechanism(files)
    lib, h = _cpp_solver(files)
    try:
        ns = lib.camp_b200_n_state_var(h)
        assert ns == mech.n_state_var
        buf = C.create_string_buffer(256)
        names = []
        for i in range(ns):
            lib.camp_b200_state_name(h, i, buf, 256)
            names.append(buf.value.decode())
        assert names == mech.species
        vt = np.zeros(ns, np.int32)
        lib.camp_b200_get_var_type(h, vt)
        np.testing.assert_array_equal(vt, mech.var_type)
        at = np.zeros(ns)
        rt = C.c_double()
        assert lib.camp_b200_json_tolerances(h, at, C.byref(rt)) == 0
        np.testing.assert_array_equal(at, mech.abs_tol)
        assert rt.value == mech.rel_tol
        # packed reaction data as added (before solver_initialize)
        py = Solver(mech, 2)
        ni = lib.camp_b200_rxn_int_data_size(h)
        assert ni == py.lib.camp_b200_rxn_int_data_size(py._h)
        a, b = np.zeros(ni, np.int32), np.zeros(ni, np.int32)
        lib.camp_b200_get_rxn_int_data(h, a)
        py.lib.camp_b200_get_rxn_int_data(py._h, b)
        np.testing.assert_array_equal(a, b)
        nf = lib.camp_b200_rxn_float_data_size(h)
        fa, fb = np.zeros(nf), np.zeros(nf)
        lib.camp_b200_get_rxn_float_data(h, fa)
        py.lib.camp_b200_get_rxn_float_data(py._h, fb)
        np.testing.assert_array_equal(fa, fb)
        # aerosol phases, representations and sub-models as added
        for which, objs in ((0, mech.aero_phases), (1, mech.aero_reps), (2, mech.sub_models)):
            for k, o in enumerate(objs):
                ni_, nf_ = C.c_int(), C.c_int()
                assert lib.camp_b200_get_aero_data(h, which, k, C.byref(ni_), C.byref(nf_),
                                                   None, None) == 0
                ia, fa_ = np.zeros(ni_.value, np.int32), np.zeros(nf_.value)
                lib.camp_b200_get_aero_data(h, which, k, None, None, ia.ctypes.data,
                                            fa_.ctypes.data)
                np.testing.assert_array_equal(ia, o.ints)
                np.testing.assert_array_equal(fa_, o.floats)
            assert lib.camp_b200_get_aero_data(h, which, len(objs), None, None, None,
                                               None) == -1
        py.free()
    finally:
        lib.solver_free(h)


def test_synthetic_mechanism(tmp_path):
    from camp_b200.synth import write_synthetic

    files, _ = write_synthetic(str(tmp_path), 60, 150, 3)
    _compare(files)


def test_every_gas_type_and_option(tmp_path):
    """CMAQ types, Ea instead of C, minute time units, repeated reactants,
    constant species, per-species tolerances, a relative tolerance, species
    merged across files, mechanisms merged by name."""
    sp1 = {"camp-data": [
        {"name": "A", "type": "CHEM_SPEC", "absolute integration tolerance": 1e-6},
        {"name": "B", "type": "CHEM_SPEC"},
        {"name": "M", "type": "CHEM_SPEC", "tracer type": "CONSTANT"},
        {"name": "RELTOL", "type": "RELATIVE_TOLERANCE", "value": 1e-5},
    ]}
    sp2 = {"camp-data": [
        {"name": "C", "type": "CHEM_SPEC"},
        {"name": "B", "type": "CHEM_SPEC", "description": "merged"},
    ]}
    mech = {"camp-data": [
        {"name": "m", "type": "MECHANISM", "reactions": [
            {"type": "ARRHENIUS", "reactants": {"A": {}, "B": {}}, "products": {"C": {"yield": 0.7}},
             "Ea": 2.0e-20, "B": -1.5, "D": 250.0, "E": 1.0e-6, "rxn id": "r1"},
            {"type": "ARRHENIUS", "reactants": {"B": {"qty": 2}}, "products": {"A": {}},
             "A": 3.0, "time unit": "MIN"},
            {"type": "TROE", "reactants": {"A": {}, "M": {}}, "products": {"B": {}},
             "k0_A": 5e-30, "k0_B": -2.0, "kinf_A": 1e-11, "Fc": 0.5, "N": 1.2},
        ]},
        {"name": "m", "type": "MECHANISM", "reactions": [
            {"type": "CMAQ_H2O2", "reactants": {"B": {"qty": 2}}, "products": {"C": {}},
             "k1_A": 2.3e-13, "k1_C": 600.0, "k2_A": 1.7e-33, "k2_C": 1000.0},
            {"type": "CMAQ_OH_HNO3", "reactants": {"A": {}, "C": {}}, "products": {"B": {}},
             "k0_A": 2.4e-14, "k0_C": 460.0, "k2_A": 2.7e-17, "k2_C": 2199.0,
             "k3_A": 6.5e-34, "k3_C": 1335.0},
            {"type": "PHOTOLYSIS", "reactants": {"C": {}}, "products": {"A": {}, "B": {"yield": -0.5}},
             "scaling factor": 2.0},
            {"type": "FIRST_ORDER_LOSS", "species": "A", "scaling factor": 0.5,
             "rxn id": "dep A"},
            {"type": "EMISSION", "species": "C", "rxn id": "emis C"},
            {"type": "PHOTOLYSIS", "reactants": {"A": {}}, "products": {"C": {}}},
        ]},
    ]}
    paths = []
    for name, obj in (("sp1.json", sp1), ("sp2.json", sp2), ("mech.json", mech)):
        p = os.path.join(tmp_path, name)
        with open(p, "w") as fh:
            json.dump(obj, fh)
        paths.append(p)
    _compare(paths)


REF_MOD37 = os.path.join(REF_ROOT, "mechanisms", "monarch_mod37")
REF_UNIT = os.path.join(REF_ROOT, "test", "unit_rxn_data")


@pytest.mark.skipif(not os.path.isdir(REF_MOD37), reason="reference tree not present")
def test_mod37_gas_from_reference_files():
    """cb05 with dry deposition (FIRST_ORDER_LOSS) and emissions (EMISSION),
    the gas-phase files of the shipped MONARCH mod37 configuration."""
    files = ["cb05_species.json", "cb05_abs_tol.json", "cb05_mechanism.json",
             "custom_species.json", "dry_deposition.json", "HERMES_emissions_rxns.json",
             "MEGAN_emissions_rxns.json"]
    _compare([os.path.join(REF_MOD37, f) for f in files])


@pytest.mark.skipif(not os.path.isdir(REF_UNIT), reason="reference tree not present")
@pytest.mark.parametrize("name", ["test_emission.json", "test_first_order_loss.json"])
def test_reference_unit_test_inputs(name):
    _compare([os.path.join(REF_UNIT, name)])


def test_wet_deposition_needs_packed_data(tmp_path):
    p = os.path.join(tmp_path, "wet.json")
    with open(p, "w") as fh:
        json.dump({"camp-data": [
            {"name": "A", "type": "CHEM_SPEC"},
            {"name": "m", "type": "MECHANISM", "reactions": [
                {"type": "WET_DEPOSITION", "aerosol phase": "rain"}]}]}, fh)
    lib = _lib.load()
    arr = (C.c_char_p * 1)(p.encode())
    assert not lib.camp_b200_solver_from_json(arr, 1, 1)
    assert "WET_DEPOSITION" in _lib.last_error()


@pytest.mark.skipif(not os.path.isdir(REF_CB05), reason="reference tree not present")
def test_cb05_from_reference_files():
    _compare([os.path.join(REF_CB05, "cb05cl_ae5_species.json"),
              os.path.join(REF_CB05, "cb05cl_ae5_mechanism.json")])


def test_errors_are_reported(tmp_path):
    p = os.path.join(tmp_path, "bad.json")
    with open(p, "w") as fh:
        fh.write('{"camp-data": [{"name": "m", "type": "MECHANISM", "reactions": '
                 '[{"type": "ARRHENIUS", "reactants": {"X": {}}, "products": {}}]}]}')
    lib = _lib.load()
    arr = (C.c_char_p * 1)(p.encode())
    assert not lib.camp_b200_solver_from_json(arr, 1, 1)
    assert "Missing species: X" in _lib.last_error()


@pytest.mark.skipif(not os.path.isdir(REF_MOD37), reason="reference tree not present")
def test_mod37_aerosol_from_reference_files():
    """The shipped mod37 files with the SOA scheme, aerosol phases, the
    MONARCH modal/binned representation (7 modes and bin sets), the wet
    deposition of cloud and rain water and its 35 HL partitioning
    reactions."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import MOD37_AERO_FILES

    _compare([os.path.join(REF_MOD37, f) for f in MOD37_AERO_FILES], aerosol=True)


@pytest.mark.skipif(not os.path.isdir(REF_MOD37), reason="reference tree not present")
def test_mod37_shipped_from_reference_files():
    """test/monarch/config_monarch_mod37.json as shipped: its ZSR
    aerosol-water and PD-FiTE activity sub-models packed by the C++ reader
    exactly as the Python packer does."""
    from camp_b200.mechanism import expand_config

    cfg = os.path.join(REF_ROOT, "test", "monarch", "config_monarch_mod37.json")
    files = expand_config(cfg, lambda p: p.replace("mechanisms_run", "mechanisms"))
    _compare(files, aerosol=True)


def test_aerosol_options(tmp_path):
    """A mode and LINEAR / LOG bin sets over two phases, a phase split over
    two objects, SIMPOL with an activity coefficient and with N*, HL and
    WET_DEPOSITION over every instance of a phase, species merged across
    files."""
    doc = {"camp-data": [
        {"name": "G1", "type": "CHEM_SPEC", "molecular weight [kg mol-1]": 0.1,
         "diffusion coeff [m2 s-1]": 1.0e-5, "N star": 2.5},
        {"name": "G2", "type": "CHEM_SPEC", "molecular weight [kg mol-1]": 0.05,
         "diffusion coeff [m2 s-1]": 1.2e-5, "HLC(298K) [M Pa-1]": 3.0e-4,
         "HLC exp factor [K]": 0.0},
        {"name": "O1", "type": "CHEM_SPEC", "phase": "AEROSOL",
         "molecular weight [kg mol-1]": 0.15, "density [kg m-3]": 1400.0},
        {"name": "W", "type": "CHEM_SPEC", "phase": "AEROSOL", "tracer type": "CONSTANT",
         "molecular weight [kg mol-1]": 0.018, "density [kg m-3]": 1000.0,
         "absolute integration tolerance": 1e-5},
        {"name": "X", "type": "CHEM_SPEC", "phase": "AEROSOL",
         "molecular weight [kg mol-1]": 0.05, "density [kg m-3]": 1000.0},
        {"name": "GAM", "type": "CHEM_SPEC", "tracer type": "ACTIVITY_COEFF", "phase": "AEROSOL"},
        {"name": "org", "type": "AERO_PHASE", "species": ["O1"]},
        {"name": "aq", "type": "AERO_PHASE", "species": ["W", "X"]},
        {"name": "org", "type": "AERO_PHASE", "species": ["GAM"]},
        {"name": "rep", "type": "AERO_REP_MODAL_BINNED_MASS", "modes/bins": {
            "fine": {"type": "MODAL", "phases": ["org", "aq"], "shape": "LOG_NORMAL",
                     "geometric mean diameter [m]": 1.0e-7, "geometric standard deviation": 1.8},
            "lin": {"type": "BINNED", "phases": ["aq"], "bins": 3, "scale": "LINEAR",
                    "minimum diameter [m]": 1.0e-6, "maximum diameter [m]": 5.0e-6},
            "log": {"type": "BINNED", "phases": ["org", "aq"], "bins": 4, "scale": "LOG",
                    "minimum diameter [m]": 1.0e-8, "maximum diameter [m]": 1.0e-5}}},
        {"name": "m", "type": "MECHANISM", "reactions": [
            {"type": "ARRHENIUS", "reactants": {"G1": {}}, "products": {"G2": {}}, "A": 1e-3},
            {"type": "SIMPOL_PHASE_TRANSFER", "gas-phase species": "G1", "aerosol phase": "org",
             "aerosol-phase species": "O1", "aerosol-phase activity coefficient": "GAM",
             "B": [-1.97e3, 2.91, 1.96e-3, -0.496]},
            {"type": "HL_PHASE_TRANSFER", "gas-phase species": "G2", "aerosol phase": "aq",
             "aerosol-phase species": "X", "aerosol-phase water": "W", "rxn id": "hl"},
            {"type": "WET_DEPOSITION", "aerosol phase": "aq", "scaling factor": 0.5},
            {"type": "PHOTOLYSIS", "reactants": {"G2": {}}, "products": {"G1": {}}},
        ]},
    ]}
    p = os.path.join(tmp_path, "aero.json")
    with open(p, "w") as fh:
        json.dump(doc, fh)
    _compare([p], aerosol=True)


@pytest.mark.parametrize("obj,msg", [
    ({"name": "sp", "type": "AERO_REP_SINGLE_PARTICLE"}, "AERO_REP_SINGLE_PARTICLE"),
    ({"name": "u", "type": "SUB_MODEL_UNIFAC"}, "SUB_MODEL_UNIFAC"),
    ({"name": "zsr", "type": "SUB_MODEL_ZSR_AEROSOL_WATER"}, "missing aerosol phase"),
])
def test_unsupported_aerosol_objects(tmp_path, obj, msg):
    p = os.path.join(tmp_path, "x.json")
    with open(p, "w") as fh:
        json.dump({"camp-data": [{"name": "A", "type": "CHEM_SPEC"}, obj]}, fh)
    lib = _lib.load()
    arr = (C.c_char_p * 1)(p.encode())
    assert not lib.camp_b200_solver_from_json(arr, 1, 1)
    assert msg in _lib.last_error()
