"""The C-ABI library without a GPU: it loads, exports every declared entry
point, and its host-side sparsity build is bit-exact with the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, REF_ROOT, ROOT, gpu_available


def header_functions():
    txt = open(os.path.join(ROOT, "include", "camp_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = "\n".join(l for l in txt.splitlines() if not l.lstrip().startswith("#"))
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)
    skip = {"extern", "if", "while", "sizeof"}
    return sorted({n for n in names if n not in skip})


def test_exports_every_declared_symbol(lib):
    from camp_b200 import _lib

    names = header_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/camp_b200.h but not exported"
    assert sorted(_lib.EXPORTED) == names


def test_sparsity_via_c_abi(golden, lib):
    from camp_b200.solver import Solver

    mech, ref = golden
    s = Solver(mech, 4)
    s.build_sparsity_only()
    if not gpu_available():
        assert not s.ready
    cp, ri = s.solver_jac()
    assert np.array_equal(cp, ref["solver_colptr"])
    assert np.array_equal(ri, ref["solver_rowid"])
    # DERIV_ID_/JAC_ID_ of every reaction, bit for bit
    assert np.array_equal(s.rxn_int_data(), ref["rxn_int_data"])
    # the fold J_solver += J_rxn * J_params, triplet for triplet (sub-model
    # parameters on the shipped mod37 configuration)
    assert np.array_equal(s.jac_map(), ref["jac_map"])
    perm = s.lu_order()
    assert sorted(perm.tolist()) == list(range(mech.n_dep_var))
    if mech.name == "cb05cl_ae5":
        assert s.n_lu() <= 748


def test_host_rate_columns(mod37, lib):
    """One base-rate column per PHOTOLYSIS / FIRST_ORDER_LOSS / EMISSION /
    WET_DEPOSITION reaction in mechanism order, each with its type and id,
    known as soon as the reactions are added."""
    from camp_b200.solver import Solver

    s = Solver(mech := mod37, 2)
    cols = mech.rate_rxns()
    assert s.n_photo == len(cols) == 107
    for j, i in enumerate(cols):
        assert s.rate_column(j) == (i, mech.rxns[i].rxn_type, mech.rate_id(i))
    assert lib.camp_b200_rate_column(s._h, len(cols), None, None, None) == -1


@pytest.mark.parametrize("kind", ["photolysis", "emission", "first_order_loss",
                                  "wet_deposition"])
def test_rate_update_data_layout(lib, kind):
    """int reaction id followed, unaligned, by the double base rate
    (src/rxns/rxn_photolysis.c:262-283, rxn_emission.c:192-213,
    rxn_first_order_loss.c:208-229, rxn_wet_deposition.c:218-239)."""
    ud = getattr(lib, f"rxn_{kind}_create_rate_update_data")()
    getattr(lib, f"rxn_{kind}_set_rate_update_data")(ud, 7, 2.5e-3)
    raw = C.string_at(ud, 12)
    assert int.from_bytes(raw[:4], "little", signed=True) == 7
    assert np.frombuffer(raw[4:12], np.float64)[0] == 2.5e-3
    lib.solver_free_update_data(ud)


def test_rejects_unsupported(cb05, lib):
    """Aerosol sub-models are refused at initialize with a readable error."""
    from camp_b200 import _lib

    m = cb05
    h = lib.solver_new(m.n_state_var, 1, np.ascontiguousarray(m.var_type, np.int32), m.n_rxn,
                       m.n_rxn_int_param, m.n_rxn_float_param, m.n_rxn_env_param,
                       0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0)
    for r in m.rxns:
        lib.rxn_add_condensed_data(r.rxn_type, r.ints.size, r.floats.size, r.n_env,
                                   np.ascontiguousarray(r.ints, np.int32),
                                   np.ascontiguousarray(r.floats), h)
    lib.solver_initialize(h, np.ascontiguousarray(m.abs_tol), 1e-4, 100, 10)
    assert lib.camp_b200_is_ready(h) == 0
    assert "sub-models" in _lib.last_error()
    st = np.zeros(m.n_state_var)
    env = np.array([298.0, 1e5])
    assert lib.solver_run(h, st, env, 0.0, 1.0) == 1
    lib.solver_free(h)


def test_packer_matches_fixture(cb05):
    """Re-packing the reference JSON reproduces the committed packed data."""
    ref = REF_ROOT
    if not os.path.isdir(ref):
        pytest.skip("reference tree absent")
    import sys

    sys.path.insert(0, GOLDEN)
    from make_golden import cb05_files

    from camp_b200.mechanism import load_mechanism, reaction_summary

    m = load_mechanism(cb05_files(ref), name="cb05cl_ae5")
    assert m.n_rxn == 186 and m.n_dep_var == 74
    summ = reaction_summary(m)
    assert summ["by_type"] == {5: 25, 1: 142, 2: 15, 4: 1, 3: 3}
    for a, b in zip(m.rxns, cb05.rxns):
        assert a.rxn_type == b.rxn_type
        assert np.array_equal(a.ints, b.ints)
        assert np.array_equal(a.floats, b.floats)


def test_mod37_packer_matches_fixture(mod37):
    ref = REF_ROOT
    if not os.path.isdir(ref):
        pytest.skip("reference tree absent")
    import sys

    sys.path.insert(0, GOLDEN)
    from make_golden import mod37_gas

    m = mod37_gas(ref)
    assert m.species == mod37.species
    assert len(m.rxns) == len(mod37.rxns) == 268
    for a, b in zip(m.rxns, mod37.rxns):
        assert a.rxn_type == b.rxn_type
        assert np.array_equal(a.ints, b.ints)
        assert np.array_equal(a.floats, b.floats)


def test_hl_elements_stay_out_of_the_lu(mod37_soa, mod37_aero, lib):
    """The reference registers every mass species of the cloud-and-rain mode
    against each HL gas and aerosol species (3827 solver Jacobian entries
    with mod37's aqueous equilibria, 863 without HL or those).  Those partials are zero for the modal/binned
    representation, so the exported sparsity keeps them while the LU leaves
    them out: it grows by the HL couplings only, where the full pattern
    fills to 4563 entries."""
    from camp_b200.solver import Solver

    sizes = []
    for m in (mod37_soa, mod37_aero):
        s = Solver(m, 2)
        s.build_sparsity_only()
        sizes.append((len(s.solver_jac()[1]), s.n_lu()))
    assert sizes[0][0] == 863 and sizes[1][0] == 3827
    assert sizes[1][1] <= 1.1 * sizes[0][1]


@pytest.mark.parametrize("case", ["hl", "aq"])
def test_variable_water_is_refused(tmp_path, case, lib):
    """HL and aqueous equilibrium divide by the aerosol-phase water; a water
    that the solver integrates would need its partials, which this build
    does not evaluate, so solver_initialize refuses it with a reason
    (before any device work)."""
    import json

    from conftest import aq_case, hl_case

    from camp_b200 import _lib
    from camp_b200.aerosol import load_aerosol_mechanism
    from camp_b200.solver import Solver

    (hl_case if case == "hl" else aq_case)(tmp_path)
    path = os.path.join(str(tmp_path), f"{case}.json")
    doc = json.load(open(path))
    for o in doc["camp-data"]:
        if o.get("name") == "H2O_aq":
            o["tracer type"] = "VARIABLE"
    with open(path, "w") as fh:
        json.dump(doc, fh)
    mech = load_aerosol_mechanism([path])
    s = Solver(mech, 2)
    s.build_sparsity_only()
    assert not s.ready
    assert "constant" in _lib.last_error()


def test_kernel_setting(cb05, lib):
    """camp_b200_set_kernel takes the three kernel forms (0 warp, 1 lane,
    2 block per cell) and refuses anything else; before solver_initialize
    camp_b200_get_kernel reports the setting."""
    from camp_b200.solver import Solver, SolverError

    s = Solver(cb05, 4)
    s.build_sparsity_only()
    for k in (2, 1, 0):
        s.set_kernel(k)
        if not s.ready:
            assert s.kernel() == k
    for bad in (-1, 3):
        with pytest.raises(SolverError, match="kernel must be 0, 1 or 2"):
            s.set_kernel(bad)
