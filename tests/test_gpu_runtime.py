"""Runtime around the solve kernel on the GPU: the autotuner and the serving
loop (continuous batching).  Both must leave every cell's result unchanged:
a cell's integration does not depend on the launch configuration or on what
else runs on the GPU."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL = 1e-12  # same kernel, same cell: equal to round-off


def _solver(mech, n, precision=1, max_steps=3000):
    from camp_b200.solver import Solver

    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4, max_steps=max_steps)
    s.set_precision(precision)
    return s


def test_autotune_keeps_results(cb05):
    from camp_b200.cells import make_cells

    n = 400
    cells = make_cells(cb05, n, 31)
    s = _solver(cb05, n, max_steps=1500)
    s.set_photo_rates(cells.photo_rates)
    ref = cells.state.copy()
    s.solve(ref, cells.env, 0.0, 60.0)
    ref_status = s.cell_stats()["status"]
    tuned = s.autotune(cells.state, cells.env, 0.0, 60.0)
    # the lane-per-cell kernel is a candidate too; on cb05cl_ae5 the warp
    # kernel is the faster one
    assert tuned["kernel"] == 0
    assert 1 <= tuned["warps_per_block"] <= 16
    assert tuned["hist_global"] in (0, 1) and tuned["lu_mode"] in (0, 1)
    assert tuned["sample_ms"] > 0
    out = cells.state.copy()
    s.solve(out, cells.env, 0.0, 60.0)
    np.testing.assert_array_equal(s.cell_stats()["status"], ref_status)
    np.testing.assert_allclose(out, ref, rtol=RTOL, atol=0)


def test_serving_mix_equals_alone(cb05, mod37_aero):
    """Columns of cb05cl_ae5 and of mod37 with its aerosol chemistry
    (deposition, emissions, SIMPOL and HL partitioning, per-cell mode GMD /
    GSD), 10-200 cells and host steps of 60/300/900 s submitted back to back;
    each result equals the same column solved alone through solver_run."""
    from camp_b200.cells import make_cells, photo_base_rates
    from camp_b200.serve import Server

    mechs = [(cb05, photo_base_rates(cb05)), (mod37_aero, photo_base_rates(mod37_aero))]
    solvers = [_solver(m, 200) for m, _ in mechs]
    server = Server(n_slots=6, device_mb=512, host_mb=128)
    ids = [server.add_solver(s) for s in solvers]
    rng = np.random.Generator(np.random.PCG64(5))
    reqs = []
    for k in range(14):
        mi = 0 if rng.uniform() < 0.7 else 1
        n = int(rng.integers(10, 201))
        dt = float(rng.choice([60.0, 300.0, 900.0]))
        mech, base = mechs[mi]
        c = make_cells(mech, n, 100 + k, photo_base=base)
        st = c.state.copy()
        rid = server.submit(ids[mi], st, c.env, c.photo_rates, 0.0, dt)
        reqs.append((rid, mi, c, dt, st))
    assert server.pending() == len(reqs)
    lat = []
    for rid, mi, c, dt, st in reqs:
        rc, ms, out, stats = server.wait(rid)
        lat.append(ms)
        s = _solver(mechs[mi][0], c.n_cells)
        s.set_photo_rates(c.photo_rates)
        alone = c.state.copy()
        rc_alone = s.solve(alone, c.env, 0.0, dt)
        assert rc == rc_alone
        np.testing.assert_array_equal(stats["status"], s.cell_stats()["status"])
        np.testing.assert_allclose(out, alone, rtol=RTOL, atol=0)
    assert server.pending() == 0
    assert all(x > 0 for x in lat)
    server.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_resident_column_equals_successive_solver_runs(cb05, mod37_aero, precision):
    """Device-resident columns: three host steps of each column, submitted
    back to back and interleaved with ordinary requests, give the
    concentrations of three solver_run calls on the same cells (a column's
    steps run in order; its concentrations never leave the device between
    them)."""
    from camp_b200.cells import make_cells, photo_base_rates
    from camp_b200.serve import Server

    mechs = [(cb05, photo_base_rates(cb05)), (mod37_aero, photo_base_rates(mod37_aero))]
    solvers = [_solver(m, 160, precision=precision) for m, _ in mechs]
    server = Server(n_slots=4, device_mb=512, host_mb=128)
    ids = [server.add_solver(s) for s in solvers]
    cols = []
    for k, (mech, base) in enumerate(mechs):
        c = make_cells(mech, 60 + 40 * k, 300 + k, photo_base=base)
        cols.append((k, c, server.open_column(ids[k], c.state)))
    steps = (0.0, 60.0, 360.0, 1260.0)
    extra = []
    col_reqs = {cid: [] for _, _, cid in cols}
    for j in range(3):
        for k, c, cid in cols:
            col_reqs[cid].append(server.submit_column(cid, c.env, c.photo_rates, steps[j],
                                                      steps[j + 1]))
        # an ordinary request of cb05 between the column steps
        o = make_cells(cb05, 30, 400 + j, photo_base=mechs[0][1])
        st = o.state.copy()
        extra.append((server.submit(ids[0], st, o.env, o.photo_rates, 0.0, 60.0), o, st))
    for k, c, cid in cols:
        for rid in col_reqs[cid]:
            rc, ms, out, stats = server.wait(rid)
            assert rc in (0, 1) and out is None and ms > 0
        dev = server.read_column(cid)
        s = _solver(mechs[k][0], c.n_cells, precision=precision)
        s.set_photo_rates(c.photo_rates)
        ref = c.state.copy()
        for j in range(3):
            s.solve(ref, c.env, steps[j], steps[j + 1])
        np.testing.assert_allclose(dev, ref, rtol=RTOL, atol=0)
        server.close_column(cid)
    for rid, o, st in extra:
        rc, ms, out, stats = server.wait(rid)
        s = _solver(cb05, o.n_cells, precision=precision)
        s.set_photo_rates(o.photo_rates)
        alone = o.state.copy()
        s.solve(alone, o.env, 0.0, 60.0)
        np.testing.assert_allclose(out, alone, rtol=RTOL, atol=0)
    assert server.pending() == 0
    server.close()


def test_graph_launch_keeps_results(cb05):
    """The device step launched as a CUDA graph (updated per run) gives the
    results of the plain launches, over runs with changing arguments."""
    import torch

    from camp_b200.cells import make_cells

    n = 256
    cells = make_cells(cb05, n, 41)
    dev = torch.device("cuda", 0)
    env = torch.from_numpy(cells.env).to(dev)
    outs = []
    for graph in (False, True):
        s = _solver(cb05, n, max_steps=1500)
        s.set_photo_rates(cells.photo_rates)
        s.set_graph(graph)
        st = torch.from_numpy(cells.state).to(dev)
        res = []
        # same launch shape with new arguments (node update), then other shapes
        for dt in (60.0, 120.0, 300.0, 60.0):
            s.run_device(st, env, n if dt != 300.0 else n // 2, 0.0, dt)
            res.append((st.cpu().numpy().copy(), s.cell_stats(n // 2)["status"].copy()))
        outs.append(res)
    for (a, sa), (b, sb) in zip(*outs):
        np.testing.assert_array_equal(sa, sb)
        np.testing.assert_allclose(b, a, rtol=RTOL, atol=0)


def test_device_photolysis_rates(cb05):
    """Rates handed over in device memory give the results of host rates."""
    import torch

    from camp_b200.cells import make_cells

    n = 128
    cells = make_cells(cb05, n, 51)
    dev = torch.device("cuda", 0)
    env = torch.from_numpy(cells.env).to(dev)
    s = _solver(cb05, n, max_steps=1500)
    s.set_photo_rates(cells.photo_rates)
    a = torch.from_numpy(cells.state).to(dev)
    s.run_device(a, env, n, 0.0, 60.0)
    sa = s.cell_stats()["status"].copy()
    s.set_photo_rates(np.zeros_like(cells.photo_rates))  # host copy no longer matches
    s.set_photo_rates_device(torch.from_numpy(np.ascontiguousarray(cells.photo_rates)).to(dev))
    b = torch.from_numpy(cells.state).to(dev)
    s.run_device(b, env, n, 0.0, 60.0)
    np.testing.assert_array_equal(s.cell_stats()["status"], sa)
    np.testing.assert_allclose(b.cpu().numpy(), a.cpu().numpy(), rtol=RTOL, atol=0)
