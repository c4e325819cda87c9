"""GPU parity: the CUDA path through the C ABI against the reference's C
derivative/Jacobian (golden fixture) and against the CPU oracle's solve."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL_FJ = 1e-12  # derivative / Jacobian parity with the reference's FP64 C code


@pytest.fixture(scope="module")
def solver(cb05, cb05_ref):
    from camp_b200.solver import Solver

    nc = cb05_ref["state"].shape[0]
    s = Solver(cb05, max(nc, 256))
    s.initialize(abs_tol=np.full(cb05.n_state_var, 1e-8), rel_tol=1e-4)
    return s


def test_deriv_matches_reference(solver, cb05_ref):
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


def test_jacobian_matches_reference(solver, cb05_ref):
    nc = cb05_ref["state"].shape[0]
    photo = np.zeros((solver.n_cells, solver.n_photo))
    photo[:nc] = cb05_ref["photo"]
    solver.set_photo_rates(photo)
    for ih, h in enumerate(cb05_ref["h"]):
        j, jp, jl = solver.eval_jac(cb05_ref["state"], cb05_ref["env"], h)
        ref = cb05_ref["jac"][ih]
        assert np.all(np.abs(j - ref) <= RTOL_FJ * (np.abs(jp) + np.abs(jl)) + 1e-300)


def _run_both(cb05, n_cells, seed, precision=0, t1=60.0):
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
    rc = s.solve(gpu_state, cells.env, 0.0, t1)
    gstats = s.cell_stats()
    om = OracleModel(cb05)
    nf, status, stats, cpu_state = om.solve(cells.state.copy(), cells.env, cells.photo_rates,
                                            0.0, t1, 1e-4, atol, n_threads=8)
    return cells, rc, gpu_state, gstats, status, cpu_state, stats


def _agreement(cb05, a, b, ok):
    dep = cb05.dep_index()
    x, y = a[ok][:, dep], b[ok][:, dep]
    big = (np.abs(y) > 1e-8)
    rel = np.abs(x - y)[big] / np.abs(y)[big]
    return rel.max() if rel.size else 0.0


def test_fp64_solve_matches_oracle(cb05):
    cells, rc, g, gs, status, c, cs = _run_both(cb05, 96, 11, precision=0)
    ok = (gs["status"] == 0) & (status == 0)
    # the same cells succeed on both sides
    assert np.mean(gs["status"] == status) >= 0.95
    assert ok.sum() >= 0.5 * len(ok)
    assert _agreement(cb05, g, c, ok) < 1e-3
    # and the bulk agree far more tightly than the 1e-3 bar
    dep = cb05.dep_index()
    x, y = g[ok][:, dep], c[ok][:, dep]
    big = np.abs(y) > 1e-8
    assert np.median(np.abs(x - y)[big] / np.abs(y)[big]) < 1e-8


def test_mixed_solve_matches_oracle(cb05):
    cells, rc, g, gs, status, c, cs = _run_both(cb05, 96, 12, precision=1)
    ok = (gs["status"] == 0) & (status == 0)
    assert ok.sum() >= 0.5 * len(ok)
    assert _agreement(cb05, g, c, ok) < 1e-3


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
