"""Replica plumbing of the multi-GPU benchmark on CPU: two gloo ranks, each
with its own seeded cells, agree on the barrier and on the max over ranks of
their timed region, and compute the same whole-job throughput."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from camp_b200 import replicas
    from camp_b200.cells import make_cells
    from camp_b200.mechanism import Mechanism

    w, r, _ = replicas.init("gloo", timeout_s=60)
    mech = Mechanism.load(os.path.join(os.path.dirname(__file__), "golden", "cb05cl_ae5.mech.json"))
    cells = make_cells(mech, 8, replicas.rank_seed(100, r))
    replicas.barrier(w)
    local_seconds = 1.0 + r  # rank 1 is the slow one
    t = replicas.max_over_ranks(local_seconds, w)
    ok = replicas.sum_over_ranks(5 + r, w)  # cells that finished on each rank
    out.put((r, w, t, replicas.aggregate_throughput(8, 10, w, t), float(cells.state.sum()), ok))
    replicas.finalize(w)


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(2))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (r0, w0, t0, v0, s0, k0), (r1, w1, t1, v1, s1, k1) = res
    assert (r0, r1) == (0, 1) and w0 == w1 == 2
    assert t0 == t1 == 2.0  # max over ranks
    assert v0 == v1 == 2 * 8 * 10 / 2.0
    assert s0 != s1  # disjoint seeded cells per rank
    assert k0 == k1 == 11.0  # sum over ranks


def test_single_rank_needs_no_group(monkeypatch):
    from camp_b200 import replicas

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.init("gloo") == (1, 0, 0)
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.aggregate_throughput(100, 10, 1, 2.0) == 500.0
    assert replicas.sum_over_ranks(7, 1) == 7.0
