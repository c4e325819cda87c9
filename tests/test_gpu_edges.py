"""Edge cases of the device solve through the C ABI: a zero-length host step,
a single cell, cells that start at zero or in the dark, runs on fewer cells
than the capacity, out-of-range sizes, and launch shapes that must not change
any cell's result."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL = 1e-12


def _solver(mech, n, precision=0, max_steps=3000):
    from camp_b200.solver import Solver

    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4, max_steps=max_steps)
    s.set_precision(precision)
    return s


def test_zero_length_step_is_too_close(cb05):
    """t_final == t_initial: CVODE's initial-step estimate refuses it
    (CV_TOO_CLOSE); every cell keeps its input and solver_run reports 1,
    as the oracle does."""
    from camp_b200.cells import make_cells
    from oracle.oracle import OracleModel

    cells = make_cells(cb05, 6, 2)
    s = _solver(cb05, 6)
    s.set_photo_rates(cells.photo_rates)
    st = cells.state.copy()
    assert s.solve(st, cells.env, 30.0, 30.0) == 1
    assert np.all(s.cell_stats()["status"] == -27)
    dep = cb05.dep_index()
    np.testing.assert_array_equal(st[:, dep], cells.state[:, dep])
    _, ost, _, _ = OracleModel(cb05).solve(cells.state.copy(), cells.env, cells.photo_rates,
                                           30.0, 30.0, 1e-4, np.full(cb05.n_state_var, 1e-8))
    assert np.all(ost == -27)


def test_single_cell_equals_cell_in_batch(cb05):
    from camp_b200.cells import make_cells

    cells = make_cells(cb05, 40, 8)
    big = _solver(cb05, 40)
    big.set_photo_rates(cells.photo_rates)
    all_out = cells.state.copy()
    big.solve(all_out, cells.env, 0.0, 60.0)
    for c in (0, 17, 39):
        one = _solver(cb05, 1)
        one.set_photo_rates(cells.photo_rates[c:c + 1])
        x = cells.state[c:c + 1].copy()
        one.solve(x, cells.env[c:c + 1], 0.0, 60.0)
        assert one.cell_stats()["status"][0] == big.cell_stats()["status"][c]
        np.testing.assert_allclose(x[0], all_out[c], rtol=RTOL, atol=0)


def test_zero_and_dark_cells_match_oracle(cb05):
    """All variable species at 0 (clamped to TINY on input) and cells without
    photolysis reach the oracle's outcome and values."""
    from camp_b200.cells import make_cells
    from camp_b200.mechanism import CHEM_SPEC_VARIABLE
    from oracle.oracle import OracleModel

    cells = make_cells(cb05, 4, 12)
    var = cb05.var_type == CHEM_SPEC_VARIABLE
    cells.state[0, var] = 0.0
    cells.photo_rates[1:3] = 0.0
    s = _solver(cb05, 4)
    s.set_photo_rates(cells.photo_rates)
    g = cells.state.copy()
    s.solve(g, cells.env, 0.0, 60.0)
    atol = np.full(cb05.n_state_var, 1e-8)
    _, ost, _, c = OracleModel(cb05).solve(cells.state.copy(), cells.env, cells.photo_rates,
                                           0.0, 60.0, 1e-4, atol)
    gst = s.cell_stats()["status"]
    np.testing.assert_array_equal(gst, ost)
    dep = cb05.dep_index()
    ok = gst == 0
    x, y = g[ok][:, dep], c[ok][:, dep]
    big = np.abs(y) > 1e-6
    assert np.median(np.abs(x - y)[big] / np.abs(y)[big]) < 1e-6


def test_fewer_cells_than_capacity_and_bounds(cb05):
    import torch

    from camp_b200.cells import make_cells
    from camp_b200.solver import SolverError

    n = 64
    cells = make_cells(cb05, n, 14)
    s = _solver(cb05, n, max_steps=1000)
    s.set_photo_rates(cells.photo_rates)
    dev = torch.device("cuda", 0)
    st = torch.from_numpy(cells.state).to(dev)
    env = torch.from_numpy(cells.env).to(dev)
    s.run_device(st, env, 20, 0.0, 60.0)
    out = st.cpu().numpy()
    # cells beyond the run are untouched
    np.testing.assert_array_equal(out[20:], cells.state[20:])
    assert not np.array_equal(out[:20], cells.state[:20])
    with pytest.raises(SolverError):
        s.run_device(st, env, n + 1, 0.0, 60.0)
    with pytest.raises(SolverError):
        s.run_device(st, env, 0, 0.0, 60.0)


@pytest.mark.parametrize("precision", [0, 1])
def test_launch_shape_does_not_change_results(cb05, precision):
    """Cells per block 1, 5 and automatic, and the one-lane LU mode, give
    the same per-cell results: each cell's arithmetic is fixed by the
    schedules, not by where it runs.  (The one-lane LU mode orders its
    updates differently, so it is compared to round-off.)"""
    from camp_b200.cells import make_cells

    n = 48
    cells = make_cells(cb05, n, 16)
    res = []
    for warps, lu in ((0, 0), (1, 0), (5, 0), (0, 1)):
        s = _solver(cb05, n, precision=precision, max_steps=800)
        s.set_photo_rates(cells.photo_rates)
        s.set_launch(warps, 1)
        s.set_lu_mode(lu)
        x = cells.state.copy()
        s.solve(x, cells.env, 0.0, 60.0)
        res.append((x, s.cell_stats()["status"]))
    for x, stt in res[1:3]:
        np.testing.assert_array_equal(stt, res[0][1])
        np.testing.assert_array_equal(x, res[0][0])
    # the one-lane LU: same outcomes on nearly all cells, values to tolerance
    assert np.mean(res[3][1] == res[0][1]) >= 0.9
