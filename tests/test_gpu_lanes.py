"""The lane-per-cell and block-per-cell kernels, and the large synthetic
mechanism that only they run.

The lane kernel (one lane per cell, 32 cells of a warp sharing every table
read) and the block kernel (one thread block per cell, the cell's LU in
shared memory) are two more CUDA implementations of the same per-cell BDF
solve; on cb05cl_ae5 and the mod37 gas phase each must reach the warp
kernel's outcomes and values.  The synthetic 200-species / 600-reaction
mechanism has an LU of 18 681 entries with 622 765 Schur updates, beyond the
warp kernel's 16-bit schedules: solver_run uses the block kernel for it by
default (the lane kernel on request), and the warp-only entry points say why
they refuse.

The synthetic mechanism gains molecules in every reaction (1-4 unit-yield
products from 1-2 reactants), so its concentrations grow quickly: at a 300 s
host step the oracle's cells all stop at the 10 000-step limit (and at
200 000), so the parity case uses a 0.5 s host step, which every cell
finishes in a few hundred internal steps.
"""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

T_LARGE = 0.5  # host step of the large-mechanism parity case (s)


def _solve(mech, cells, precision, kernel, t1, max_steps):
    from camp_b200.solver import Solver

    s = Solver(mech, cells.n_cells)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4, max_steps=max_steps)
    s.set_precision(precision)
    if kernel is not None:
        s.set_kernel(kernel)
    s.set_photo_rates(cells.photo_rates)
    x = cells.state.copy()
    s.solve(x, cells.env, 0.0, t1)
    return s, x, s.cell_stats()["status"].copy()


def _tol_units(mech, x, truth, rows):
    """Per-cell max difference in units of the tolerance (1e-4 |y| + 1e-8)."""
    dep = mech.dep_index()
    y = truth[rows][:, dep]
    return (np.abs(x[rows][:, dep] - y) / (1e-4 * np.abs(y) + 1e-8)).max(axis=1)


def _tight(mech, cells, t1):
    """The oracle's BDF at rtol 1e-8, atol 1e-12: the accuracy yardstick."""
    from oracle.oracle import OracleModel

    _, st, _, y = OracleModel(mech).solve(cells.state.copy(), cells.env, cells.photo_rates, 0.0,
                                          t1, 1e-8, np.full(mech.n_state_var, 1e-12),
                                          max_steps=200000, n_threads=os.cpu_count() or 1)
    return y, st


def _same_accuracy(mech, a, b, tight, rows):
    """Two BDF runs at rtol 1e-4 differ by their global errors, so each is
    measured against the tight solution and their per-cell errors are
    compared as distributions (median and 90th percentile): a's within 2x
    (plus slack) of b's."""
    ea = _tol_units(mech, a, tight, rows)
    eb = _tol_units(mech, b, tight, rows)
    assert np.median(ea) <= 2.0 * np.median(eb) + 1.0, (np.median(ea), np.median(eb))
    assert np.percentile(ea, 90) <= 2.0 * np.percentile(eb, 90) + 5.0, (
        np.percentile(ea, 90), np.percentile(eb, 90))


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("which", ["cb05", "mod37"])
def test_lane_kernel_matches_warp_kernel(request, which, precision, kernel):
    """Same outcomes as the warp kernel, and the reference algorithm's
    accuracy (the oracle at equal tolerances), both against the tight
    solution.  The error distributions need a few dozen finishing cells: on
    ~20 cells the median of either kernel moves by 2x with the sample."""
    from camp_b200.cells import make_cells
    from oracle.oracle import OracleModel

    mech = request.getfixturevalue(which)
    cells = make_cells(mech, 64, 23)
    _, xw, sw = _solve(mech, cells, precision, 0, 60.0, 1500)
    _, xl, sl = _solve(mech, cells, precision, kernel, 60.0, 1500)
    assert np.mean(sw == sl) >= 0.9
    _, ost, _, yo = OracleModel(mech).solve(cells.state.copy(), cells.env, cells.photo_rates,
                                            0.0, 60.0, 1e-4, np.full(mech.n_state_var, 1e-8),
                                            max_steps=1500, n_threads=os.cpu_count() or 1)
    tight, tst = _tight(mech, cells, 60.0)
    ok = (sw == 0) & (sl == 0) & (ost == 0) & (tst == 0)
    assert ok.sum() >= 32
    _same_accuracy(mech, xl, yo, tight, ok)


@pytest.fixture(scope="module")
def large():
    import tempfile

    from camp_b200.synth import load_synthetic

    with tempfile.TemporaryDirectory() as td:
        return load_synthetic(td, 200, 600)


@pytest.mark.parametrize("kernel", [None, 1])
@pytest.mark.parametrize("precision", [0, 1])
def test_large_mechanism_matches_oracle(large, precision, kernel):
    """The default (block) and the lane kernel against the oracle."""
    from camp_b200.cells import make_cells
    from oracle.oracle import OracleModel

    mech, base = large
    cells = make_cells(mech, 32, 29, conc_lo=1e-8, photo_base=base)
    s, x, st = _solve(mech, cells, precision, kernel, T_LARGE, 10000)
    assert s.kernel() == (2 if kernel is None else kernel)
    nf, ost, _, y = OracleModel(mech).solve(cells.state.copy(), cells.env, cells.photo_rates,
                                            0.0, T_LARGE, 1e-4, np.full(mech.n_state_var, 1e-8),
                                            n_threads=os.cpu_count() or 1)
    assert np.mean(st == ost) >= 0.9
    tight, tst = _tight(mech, cells, T_LARGE)
    ok = (st == 0) & (ost == 0) & (tst == 0)
    assert ok.sum() >= 24
    _same_accuracy(mech, x, y, tight, ok)


def test_large_mechanism_warp_entry_points_refuse(large):
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver, SolverError

    mech, base = large
    cells = make_cells(mech, 4, 31, conc_lo=1e-8, photo_base=base)
    s = Solver(mech, 4)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4)
    assert s.ready
    s.set_photo_rates(cells.photo_rates)
    with pytest.raises(SolverError, match="warp-per-cell"):
        s.eval_deriv(cells.state, cells.env, 1.0)


def test_large_mechanism_autotune_keeps_block_kernel(large):
    """On a mechanism beyond the warp tables the autotuner times the
    block-per-cell kernel (the lane kernel only where no other has tables)
    and the tuned solver still solves."""
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    mech, base = large
    cells = make_cells(mech, 64, 33, conc_lo=1e-8, photo_base=base)
    s = Solver(mech, 64)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4)
    s.set_photo_rates(cells.photo_rates)
    tuned = s.autotune(cells.state, cells.env, 0.0, T_LARGE)
    assert tuned["kernel"] == 2 and tuned["sample_ms"] > 0
    x = cells.state.copy()
    s.solve(x, cells.env, 0.0, T_LARGE)
    assert np.mean(s.cell_stats()["status"] == 0) >= 0.9
