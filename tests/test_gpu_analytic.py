"""Each gas-phase reaction type on the GPU against a closed-form solution.

The reference's per-reaction tests integrate A -> B -> C with two reactions
of one type and compare with the analytic solution
(test/unit_rxn_data/test_rxn_troe.F90, test_rxn_CMAQ_H2O2.F90,
test_rxn_CMAQ_OH_HNO3.F90, test_rxn_photolysis.F90,
test/unit_tests/rxns/unit_test_rxn_arrhenius.F90).  Here the same chain runs
through the C ABI in both precision forms.  The rate constants come from the
oracle's rate-constant code, which is pinned to the reference's C by the
golden fixture, so the comparison checks the device integrator:

    A = exp(-k1 t),  B = k1 / (k2 - k1) (exp(-k1 t) - exp(-k2 t)),  C = 1 - A - B.
"""
import os

import numpy as np
import pytest

from conftest import (CHAIN_CASES, CHAIN_ENV, CHAIN_PHOTO, chain_closed_form, chain_mechanism,
                      chain_rates, gpu_available)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

TIMES = (5.0, 20.0, 60.0)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("rtype", list(CHAIN_CASES))
def test_two_step_chain_matches_closed_form(tmp_path, rtype, precision):
    from camp_b200.solver import Solver

    mech, _ = chain_mechanism(tmp_path, rtype)
    k1, k2 = chain_rates(mech, rtype)
    n = len(TIMES)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(3, 1e-14), rel_tol=1e-9, max_steps=100000)
    s.set_precision(precision)
    if rtype == "PHOTOLYSIS":
        s.set_photo_rates(np.tile(np.array(CHAIN_PHOTO), (n, 1)))
    env = np.tile(np.array(CHAIN_ENV), (n, 1))
    out = np.zeros((n, 3))
    for c, t in enumerate(TIMES):  # one run per end time; cell c is kept from run c
        x = np.tile(np.array([1.0, 0.0, 0.0]), (n, 1))
        assert s.solve(x, env, 0.0, t) == 0, s.cell_stats()["status"]
        out[c] = x[c]
    np.testing.assert_allclose(out, chain_closed_form(k1, k2, TIMES), rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("rtype", ["ARRHENIUS", "PHOTOLYSIS"])
def test_chain_through_json_entry_point(tmp_path, rtype):
    """The same chain built by the C++ JSON reader (camp_b200_solver_from_json)
    instead of the Python packer."""
    import ctypes as C

    from camp_b200 import _lib

    mech, files = chain_mechanism(tmp_path, rtype)
    k1, k2 = chain_rates(mech, rtype)
    lib = _lib.load()
    paths = (C.c_char_p * len(files))(*[f.encode() for f in files])
    n = 2
    h = lib.camp_b200_solver_from_json(paths, len(files), n)
    assert h, _lib.last_error()
    try:
        lib.solver_initialize(h, np.full(3, 1e-14), 1e-9, 100000, 1000)
        assert lib.camp_b200_is_ready(h), _lib.last_error()
        if rtype == "PHOTOLYSIS":
            rates = np.ascontiguousarray(np.tile(np.array(CHAIN_PHOTO), (n, 1)).reshape(-1))
            lib.camp_b200_set_photo_rates(h, rates, n)
        state = np.ascontiguousarray(np.tile(np.array([1.0, 0.0, 0.0]), (n, 1)))
        env = np.ascontiguousarray(np.tile(np.array(CHAIN_ENV), (n, 1)))
        assert lib.solver_run(h, state.reshape(-1), env.reshape(-1), 0.0, 30.0) == 0
    finally:
        lib.solver_free(h)
    np.testing.assert_allclose(state, np.tile(chain_closed_form(k1, k2, [30.0]), (n, 1)),
                               rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("kind", ["EMISSION", "FIRST_ORDER_LOSS", "WET_DEPOSITION"])
def test_host_rate_types_known_answer(kind, precision):
    """The reference's EMISSION, FIRST_ORDER_LOSS and WET_DEPOSITION unit
    tests: rates set per cell through the update-data functions and
    rxn_update_data (the second one set, then reset), ten 1-s host steps
    through solver_run, against the closed forms."""
    from conftest import species_rate_case

    from camp_b200.solver import Solver

    mech, y0, first, rates, truth = species_rate_case(kind)
    n = 4
    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(y0.size, 1e-14), rel_tol=1e-10, max_steps=100000)
    s.set_precision(precision)
    cols = mech.rate_rxns()
    for c in range(n):
        for vals in (first, rates):
            for j, i in enumerate(cols):
                s.set_rate(c, mech.rxns[i].rxn_type, mech.rate_id(i), float(vals[j]))
    y = np.tile(y0, (n, 1))
    env = np.tile(np.array([298.0, 1.0e5]), (n, 1))
    out = []
    for step in range(10):
        assert s.solve(y, env, float(step), float(step + 1)) == 0, s.cell_stats()["status"]
        out.append(y.copy())
    out = np.stack(out)  # [step, cell, species]
    expect = truth(np.arange(1, 11))
    for c in range(n):
        np.testing.assert_allclose(out[:, c], expect, rtol=1e-7, atol=1e-14)


@pytest.mark.parametrize("precision", [0, 1])
def test_hl_closed_form(tmp_path, precision):
    """HL partitioning into one aqueous mode with constant water: the
    relaxation to the Henry's law equilibrium (conftest.hl_case) through
    the C ABI, the mode's GMD / GSD set per cell."""
    from conftest import HL_ENV, hl_case

    from camp_b200.solver import Solver

    mech, y0, cols, truth = hl_case(tmp_path)
    n = len(TIMES)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.array([1e-14, 1e-20, 1e-14]), rel_tol=1e-10, max_steps=100000)
    s.set_precision(precision)
    s.set_photo_rates(np.tile(cols, (n, 1)))
    env = np.tile(np.array(HL_ENV), (n, 1))
    out = np.zeros((n, 2))
    for c, t in enumerate(TIMES):
        x = np.tile(y0, (n, 1))
        assert s.solve(x, env, 0.0, t) == 0, s.cell_stats()["status"]
        out[c] = x[c, :2]
    np.testing.assert_allclose(out, truth(TIMES), rtol=1e-6, atol=1e-18)


def test_hl_through_json_entry_point(tmp_path):
    """The HL case read by the C++ JSON reader (camp_b200_solver_from_json:
    phases, the modal representation and the HL reaction packed in C++),
    its mode columns set through the representation's update data."""
    import ctypes as C

    from conftest import HL_ENV, HL_MODE, hl_case

    from camp_b200 import _lib

    _, y0, _, truth = hl_case(tmp_path)
    lib = _lib.load()
    paths = (C.c_char_p * 1)(os.path.join(str(tmp_path), "hl.json").encode())
    n = 2
    h = lib.camp_b200_solver_from_json(paths, 1, n)
    assert h, _lib.last_error()
    try:
        lib.solver_initialize(h, np.array([1e-14, 1e-20, 1e-14]), 1e-10, 100000, 1000)
        assert lib.camp_b200_is_ready(h), _lib.last_error()
        for what, val in (("gmd", HL_MODE[0]), ("gsd", HL_MODE[1])):
            ud = getattr(lib, f"aero_rep_modal_binned_mass_create_{what}_update_data")()
            getattr(lib, f"aero_rep_modal_binned_mass_set_{what}_update_data")(ud, 1, 0, val)
            for c in range(n):
                rep_id = C.c_int(0)
                lib.aero_rep_update_data(c, C.byref(rep_id), 2, ud, h)
            lib.solver_free_update_data(ud)
        state = np.ascontiguousarray(np.tile(y0, (n, 1)))
        env = np.ascontiguousarray(np.tile(np.array(HL_ENV), (n, 1)))
        assert lib.solver_run(h, state.reshape(-1), env.reshape(-1), 0.0, 30.0) == 0
    finally:
        lib.solver_free(h)
    np.testing.assert_allclose(state[:, :2], np.tile(truth([30.0])[0], (n, 1)), rtol=1e-6,
                               atol=1e-18)


@pytest.mark.parametrize("precision", [0, 1])
def test_aqueous_equilibrium_closed_form(tmp_path, precision):
    """A <-> B in one aqueous mode (conftest.aq_case) through the C ABI."""
    from conftest import AQ_ENV, aq_case

    from camp_b200.solver import Solver

    mech, y0, cols, truth = aq_case(tmp_path)
    n = len(TIMES)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.array([1e-14, 1e-20, 1e-20, 1e-14]), rel_tol=1e-10,
                 max_steps=100000)
    s.set_precision(precision)
    s.set_photo_rates(np.tile(cols, (n, 1)))
    env = np.tile(np.array(AQ_ENV), (n, 1))
    out = np.zeros((n, 2))
    for c, t in enumerate(TIMES):
        x = np.tile(y0, (n, 1))
        assert s.solve(x, env, 0.0, t) == 0, s.cell_stats()["status"]
        out[c] = x[c, 1:3]
    np.testing.assert_allclose(out, truth(TIMES), rtol=1e-6, atol=1e-20)
