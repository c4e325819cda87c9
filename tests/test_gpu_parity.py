"""GPU parity: the CUDA path through the C ABI against the reference's C
derivative/Jacobian (golden fixtures: cb05cl_ae5, the gas phase of MONARCH
mod37 with its deposition and emission reactions, mod37 with SIMPOL SOA
partitioning, with HL partitioning into cloud and rain water as well, and
the shipped mod37 test configuration with its ZSR aerosol-water and PD-FiTE
activity sub-models) and against the CPU oracle's solve."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL_FJ = 1e-12  # derivative / Jacobian parity with the reference's FP64 C code


@pytest.fixture(scope="module")
def solver_ref(golden):
    from camp_b200.solver import Solver

    mech, ref = golden
    nc = ref["state"].shape[0]
    s = Solver(mech, max(nc, 256))
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4)
    return s, ref


def test_deriv_matches_reference(solver_ref):
    solver, cb05_ref = solver_ref
    nc = cb05_ref["state"].shape[0]
    photo = np.zeros((solver.n_cells, solver.n_photo))
    photo[:nc] = cb05_ref["photo"]
    solver.set_photo_rates(photo)
    for ih, h in enumerate(cb05_ref["h"]):
        f, rp, rl = solver.eval_deriv(cb05_ref["state"], cb05_ref["env"], h)
        np.testing.assert_allclose(rp, cb05_ref["r_p"][ih], rtol=RTOL_FJ, atol=0)
        np.testing.assert_allclose(rl, cb05_ref["r_l"][ih], rtol=RTOL_FJ, atol=0)
        scale = cb05_ref["r_p"][ih] + cb05_ref["r_l"][ih]
        assert np.all(np.abs(f - cb05_ref["f"][ih]) <= RTOL_FJ * scale)


def test_jacobian_matches_reference(solver_ref):
    solver, cb05_ref = solver_ref
    nc = cb05_ref["state"].shape[0]
    photo = np.zeros((solver.n_cells, solver.n_photo))
    photo[:nc] = cb05_ref["photo"]
    solver.set_photo_rates(photo)
    for ih, h in enumerate(cb05_ref["h"]):
        j, jp, jl = solver.eval_jac(cb05_ref["state"], cb05_ref["env"], h)
        ref = cb05_ref["jac"][ih]
        assert np.all(np.abs(j - ref) <= RTOL_FJ * (np.abs(jp) + np.abs(jl)) + 1e-300)


def _run_both(cb05, n_cells, seed, precision=0, t1=60.0):
    """Solves the same seeded cells on the GPU and with the oracle at the same
    tolerances (rtol 1e-4, atol 1e-8 ppm), and with the oracle at tight
    tolerances (rtol 1e-8, atol 1e-12) as the accuracy yardstick."""
    import os

    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver
    from oracle.oracle import OracleModel

    cells = make_cells(cb05, n_cells, seed)
    atol = np.full(cb05.n_state_var, 1e-8)
    s = Solver(cb05, n_cells)
    s.initialize(abs_tol=atol, rel_tol=1e-4)
    s.set_precision(precision)
    s.set_photo_rates(cells.photo_rates)
    gpu_state = cells.state.copy()
    s.solve(gpu_state, cells.env, 0.0, t1)
    gstatus = s.cell_stats()["status"]
    om = OracleModel(cb05)
    nt = os.cpu_count() or 1
    _, status, _, cpu_state = om.solve(cells.state.copy(), cells.env, cells.photo_rates,
                                       0.0, t1, 1e-4, atol, n_threads=nt)
    _, tstatus, _, tight = om.solve(cells.state.copy(), cells.env, cells.photo_rates, 0.0, t1,
                                    1e-8, np.full(cb05.n_state_var, 1e-12),
                                    max_steps=100000, n_threads=nt)
    return gpu_state, gstatus, cpu_state, status, tight, tstatus


def _tol_units(cb05, x, truth, rows):
    """Per-cell max error in units of the loose tolerance (1e-4 |y| + 1e-8)."""
    dep = cb05.dep_index()
    y = truth[rows][:, dep]
    return (np.abs(x[rows][:, dep] - y) / (1e-4 * np.abs(y) + 1e-8)).max(axis=1)


def _check_solve(cb05, precision, seed, bulk_rel):
    g, gst, c, cst, tight, tst = _run_both(cb05, 96, seed, precision=precision)
    # the same cells succeed (and fail) on both sides
    assert np.mean(gst == cst) >= 0.95
    ok = (gst == 0) & (cst == 0)
    assert ok.sum() >= 0.5 * len(ok)
    # the bulk of the values agree far inside the tolerance
    dep = cb05.dep_index()
    x, y = g[ok][:, dep], c[ok][:, dep]
    big = np.abs(y) > 1e-6
    assert np.median(np.abs(x - y)[big] / np.abs(y)[big]) < bulk_rel
    # the GPU's error against a tight solution is the oracle's own error at
    # the same tolerances: two BDF runs at rtol 1e-4 differ by their global
    # errors, so their per-cell distance is compared as distributions
    both = ok & (tst == 0)
    assert both.sum() >= 0.4 * len(ok)
    eg = _tol_units(cb05, g, tight, both)
    ec = _tol_units(cb05, c, tight, both)
    assert np.median(eg) <= 2.0 * np.median(ec) + 1.0
    assert np.percentile(eg, 90) <= 2.0 * np.percentile(ec, 90) + 5.0


def test_fp64_solve_matches_oracle(cb05):
    _check_solve(cb05, precision=0, seed=11, bulk_rel=1e-7)


def test_mixed_solve_matches_oracle(cb05):
    _check_solve(cb05, precision=1, seed=12, bulk_rel=1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_mod37_gas_solve_matches_oracle(mod37, precision):
    """cb05 with dry deposition, emissions and wet deposition: the same
    outcome per cell and the oracle's accuracy at equal tolerances."""
    _check_solve(mod37, precision=precision, seed=13 + precision,
                 bulk_rel=1e-7 if precision == 0 else 1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_mod37_soa_solve_matches_oracle(mod37_soa, precision):
    """mod37 with SIMPOL partitioning into the modal/binned aerosol
    representation (cells carry per-mode GMD / GSD columns)."""
    _check_solve(mod37_soa, precision=precision, seed=17 + precision,
                 bulk_rel=1e-7 if precision == 0 else 1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_mod37_aero_solve_matches_oracle(mod37_aero, precision):
    """mod37 with SIMPOL and the 35 HL reactions into cloud and rain water
    (the LU without HL's zero element partials; the oracle factors the
    reference's full pattern)."""
    _check_solve(mod37_aero, precision=precision, seed=19 + precision,
                 bulk_rel=1e-7 if precision == 0 else 1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_mod37_shipped_solve_matches_oracle(mod37_shipped, precision):
    """The shipped MONARCH mod37 test configuration: the ZSR sub-model
    computes the sulfate mode's aerosol water and PD-FiTE four ion-pair
    activity coefficients before every f and J, and the Jacobian chains
    their parameter partials (J_rxn x J_params) into the solver Jacobian.

    Its fast aqueous equilibria make the outcome of a few log-uniform cells
    (TOO_MUCH_WORK or not) depend on roundoff, so the per-cell outcomes are
    held to the oracle's own floor: the oracle against itself with its
    inputs perturbed at the form's resolution (1e-15 FP64, 1e-7 mixed), and
    the FP64 values agree with the oracle's to a median of 1e-6 relative
    (1e-7 on the other mechanisms).  The same equilibria make M = I - gamma J
    so ill-conditioned (2-norm condition 1e14-1e17) that an FP32
    factorization's solve is off by up to 0.7 in the error-weighted norm
    (median 6e-4; at most 1e-2 on cb05cl_ae5 and mod37 without the
    sub-models; camp_b200_check_precision measures it): the mixed form's
    Newton iteration converges more slowly there, it finishes about 6 % fewer
    cells than the FP64 form (61 % against 67 % of 1e4 seeded cells) and its
    results are not at the oracle's accuracy, so for the mixed form this test
    checks the per-cell outcomes only, against the floor less those extra
    failures; the FP64 form meets the floor and the oracle's accuracy."""
    import os

    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver
    from oracle.oracle import OracleModel

    mech, n = mod37_shipped, 192
    cells = make_cells(mech, n, 23)
    atol = np.full(mech.n_state_var, 1e-8)
    s = Solver(mech, n)
    s.initialize(abs_tol=atol, rel_tol=1e-4)
    s.set_precision(precision)
    s.set_photo_rates(cells.photo_rates)
    g = cells.state.copy()
    s.solve(g, cells.env, 0.0, 60.0)
    gst = s.cell_stats()["status"]
    om = OracleModel(mech)
    nt = os.cpu_count() or 1
    _, cst, _, c = om.solve(cells.state.copy(), cells.env, cells.photo_rates, 0.0, 60.0, 1e-4,
                            atol, n_threads=nt)
    pert = cells.state.copy()
    dep = mech.dep_index()
    rng = np.random.default_rng(5)
    pert[:, dep] *= 1.0 + (1e-15 if precision == 0 else 1e-7) * rng.standard_normal((n, len(dep)))
    _, pst, _, _ = om.solve(pert, cells.env, cells.photo_rates, 0.0, 60.0, 1e-4, atol,
                            n_threads=nt)
    _, tst, _, tight = om.solve(cells.state.copy(), cells.env, cells.photo_rates, 0.0, 60.0,
                                1e-8, np.full(mech.n_state_var, 1e-12), max_steps=100000,
                                n_threads=nt)
    floor = float(np.mean(pst == cst))
    agree = float(np.mean(gst == cst))
    print(f"\nshipped mod37, precision {precision}: outcome agreement {agree:.3f}, oracle floor "
          f"{floor:.3f}; finished GPU {int((gst == 0).sum())}, oracle {int((cst == 0).sum())}")
    assert agree >= floor - (0.03 if precision == 0 else 0.08)
    ok = (gst == 0) & (cst == 0)
    assert ok.sum() >= 0.5 * n
    both = ok & (tst == 0)
    assert both.sum() >= 0.4 * n
    eg = _tol_units(mech, g, tight, both)
    ec = _tol_units(mech, c, tight, both)
    print(f"  error vs tight in tolerance units: GPU median {np.median(eg):.1f} p90 "
          f"{np.percentile(eg, 90):.1f}; oracle median {np.median(ec):.1f} p90 "
          f"{np.percentile(ec, 90):.1f}")
    if precision == 0:
        x, y = g[ok][:, dep], c[ok][:, dep]
        big = np.abs(y) > 1e-6
        assert np.median(np.abs(x - y)[big] / np.abs(y)[big]) < 1e-6
        assert np.median(eg) <= 2.0 * np.median(ec) + 1.0
        assert np.percentile(eg, 90) <= 2.0 * np.percentile(ec, 90) + 5.0


def test_aerosol_update_data_sets_columns(mod37_soa):
    """GMD / GSD through the reference's update-data path land in the
    cell's mode columns, the same values set_photo_rates takes."""
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    m = mod37_soa
    cells = make_cells(m, 3, 23)
    cols = m.rate_columns()
    a = Solver(m, 3)
    a.initialize(abs_tol=np.full(m.n_state_var, 1e-8), rel_tol=1e-4, max_steps=2000)
    a.set_photo_rates(cells.photo_rates)
    b = Solver(m, 3)
    b.initialize(abs_tol=np.full(m.n_state_var, 1e-8), rel_tol=1e-4, max_steps=2000)
    rates = cells.photo_rates.copy()
    aero = [j for j, c in enumerate(cols) if c[0] != "rxn"]
    rates[:, aero] = 0.0
    b.set_photo_rates(rates)
    rep_id = int(m.aero_reps[0].ints[3])
    for c in range(3):
        for j in aero:
            kind, _, sec = cols[j]
            b.set_aero(c, rep_id, sec, kind, cells.photo_rates[c, j])
    for j in aero:
        idx, typ, sec = b.rate_column(j)
        assert idx == -1 and typ in (-1, -2) and sec == cols[j][2]
    xa, xb = cells.state.copy(), cells.state.copy()
    a.solve(xa, cells.env, 0.0, 60.0)
    b.solve(xb, cells.env, 0.0, 60.0)
    np.testing.assert_array_equal(a.cell_stats()["status"], b.cell_stats()["status"])
    np.testing.assert_array_equal(xa, xb)


def test_failed_cells_keep_input_state(cb05):
    """A cell that cannot finish (max_steps 5) leaves its input state and
    reports TOO_MUCH_WORK, and solver_run returns 1."""
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    cells = make_cells(cb05, 8, 3)
    s = Solver(cb05, 8)
    s.initialize(abs_tol=np.full(cb05.n_state_var, 1e-8), rel_tol=1e-4, max_steps=5)
    s.set_photo_rates(cells.photo_rates)
    st = cells.state.copy()
    rc = s.solve(st, cells.env, 0.0, 60.0)
    cs = s.cell_stats()
    assert rc == 1
    assert np.all(cs["status"] == -1)
    dep = cb05.dep_index()
    assert np.array_equal(st[:, dep], cells.state[:, dep])
