"""Accuracy of the FP64 and mixed-precision solves against a tight FP64
solution (the oracle's BDF at rtol 1e-10, atol 1e-14), next to the oracle's
own accuracy at the same loose tolerances (rtol 1e-4, atol 1e-8 ppm).

Both GPU forms must reach the accuracy of the reference algorithm at equal
tolerances: per value, relative error against the tight solution, over the
cells that finish on every side and the values above the absolute
tolerance.  The printed table (pytest -s) is the accuracy statement for the
two forms."""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]


def test_equal_error_against_tight_oracle(cb05):
    from camp_b200.cells import make_cells
    from camp_b200.solver import FP64, MIXED, Solver
    from oracle.oracle import OracleModel

    n = 48
    cells = make_cells(cb05, n, 11)
    atol = np.full(cb05.n_state_var, 1e-8)
    nt = os.cpu_count() or 1
    om = OracleModel(cb05)
    _, tst, _, tight = om.solve(cells.state.copy(), cells.env, cells.photo_rates, 0.0, 60.0,
                                1e-10, np.full(cb05.n_state_var, 1e-14), max_steps=500000,
                                n_threads=nt)
    _, ost, _, loose = om.solve(cells.state.copy(), cells.env, cells.photo_rates, 0.0, 60.0,
                                1e-4, atol, n_threads=nt)
    out = {}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        s = Solver(cb05, n)
        s.initialize(abs_tol=atol, rel_tol=1e-4)
        s.set_precision(prec)
        s.set_photo_rates(cells.photo_rates)
        g = cells.state.copy()
        s.solve(g, cells.env, 0.0, 60.0)
        out[name] = (g, s.cell_stats()["status"])
    ok = (tst == 0) & (ost == 0) & (out["fp64"][1] == 0) & (out["mixed"][1] == 0)
    assert ok.sum() >= n // 3
    dep = cb05.dep_index()
    y = tight[ok][:, dep]
    big = np.abs(y) > 1e-8

    def rel(x):
        r = np.abs(x[ok][:, dep] - y)[big] / np.abs(y)[big]
        return float(np.median(r)), float(np.percentile(r, 99))

    ref_med, ref_p99 = rel(loose)
    print(f"\ncells finishing everywhere: {ok.sum()}/{n}")
    print(f"oracle BDF rtol 1e-4: median rel err {ref_med:.2e}, p99 {ref_p99:.2e}")
    for name in ("fp64", "mixed"):
        med, p99 = rel(out[name][0])
        print(f"GPU {name:5s} rtol 1e-4: median rel err {med:.2e}, p99 {p99:.2e}")
        # equal error: within a small factor of the reference algorithm's own
        assert med <= 3.0 * ref_med + 1e-9
        assert p99 <= 3.0 * ref_p99 + 1e-9
