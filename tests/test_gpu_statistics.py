"""solver_get_statistics after a device solve, against the per-cell counters.

The reference integrates all cells of a call as one CVODE system and reports
that system's counters (src/camp_solver.c:725-791).  Here every cell has its
own integration, so each counter is the largest over the cells of the last
run (the coupled system takes at least as many steps as its stiffest cell),
the flag is the first failing cell's (in cell order, 0 when every cell
finished), the last and next step sizes are the smallest over the cells.
Fields with no per-cell counterpart keep the values the reference reports
outside CAMP_DEBUG builds or for a solver without the quantity:
DLS_RHS_evals 0 (no difference-quotient Jacobian), Jac_eval_fails 0,
RHS_evals_total and Jac_evals_total -1, RHS/Jac times 0 and
max_loss_precision 0."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]


@pytest.mark.parametrize("max_steps", [10000, 400])
def test_statistics_aggregate_the_cell_counters(cb05, max_steps):
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    n = 64
    cells = make_cells(cb05, n, 31)
    s = Solver(cb05, n)
    s.initialize(abs_tol=np.full(cb05.n_state_var, 1e-8), rel_tol=1e-4, max_steps=max_steps)
    s.set_photo_rates(cells.photo_rates)
    st = cells.state.copy()
    rc = s.solve(st, cells.env, 0.0, 60.0)
    cs = s.cell_stats()
    out = s.statistics()
    failed = np.nonzero(cs["status"] != 0)[0]
    assert rc == (1 if failed.size else 0)
    assert out["solver_flag"] == (int(cs["status"][failed[0]]) if failed.size else 0)
    if max_steps == 400:
        assert failed.size > 0  # the step cap makes some cells fail
    for key, col in (("num_steps", "nst"), ("RHS_evals", "nfe"), ("LS_setups", "nsetups"),
                     ("error_test_fails", "netf"), ("NLS_iters", "nni"),
                     ("NLS_convergence_fails", "ncfn"), ("DLS_Jac_evals", "nje")):
        assert out[key] == int(cs[col].max()), key
    assert out["num_steps"] <= max_steps
    assert out["last_time_step__s"] == pytest.approx(float(cs["hu"].min()), rel=0, abs=0)
    assert out["next_time_step__s"] == pytest.approx(float(cs["hcur"].min()), rel=0, abs=0)
    assert out["DLS_RHS_evals"] == 0 and out["Jac_eval_fails"] == 0
    assert out["RHS_evals_total"] == -1 and out["Jac_evals_total"] == -1
    assert out["RHS_time__s"] == 0.0 and out["Jac_time__s"] == 0.0
    assert out["max_loss_precision"] == 0.0
    # the counters are CVODE's: every step evaluates f at least once, and a
    # Jacobian evaluation comes with a linear-solver setup
    assert np.all(cs["nfe"] >= cs["nst"])
    assert np.all(cs["nsetups"] >= cs["nje"])
