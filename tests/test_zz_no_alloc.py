"""The no-allocation entry point against the regular device entry point.

camp_b200_run_device_noalloc serves callers that cannot allocate device
memory while they run (a host model whose pool allocator owns the device
heap, or code running where cudaMalloc is not allowed): all buffers are the
caller's and the solve's scratch lives in a static device array inside the
library.  This test runs it twice in a row on the same inputs and checks each
result against camp_b200_run_device.  The file is named so that pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL = 1e-12  # both entry points run the same kernel: results agree to round-off


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_run_device(cb05, precision):
    import torch

    from camp_b200 import _lib
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    n = 300
    cells = make_cells(cb05, n, 21)
    s = Solver(cb05, n)
    s.initialize(abs_tol=np.full(cb05.n_state_var, 1e-8), rel_tol=1e-4, max_steps=2000)
    s.set_precision(precision)
    s.set_photo_rates(cells.photo_rates)
    dev = torch.device("cuda", 0)
    state0 = torch.from_numpy(cells.state).to(dev)
    env = torch.from_numpy(cells.env).to(dev)
    photo = torch.from_numpy(np.ascontiguousarray(cells.photo_rates)).to(dev)

    ref = state0.clone()
    s.run_device(ref, env, n, 0.0, 60.0)
    torch.cuda.synchronize()
    ref_stats = s.cell_stats(n)
    ref = ref.cpu().numpy()

    lib = _lib.load()
    stats_bytes = C.sizeof(_lib.CellStats) * n
    for call in range(2):
        out = state0.clone()
        d_stats = torch.full((stats_bytes,), 0xAB, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()
        rc = lib.camp_b200_run_device_noalloc(s._h, out.data_ptr(), env.data_ptr(),
                                              photo.data_ptr(), d_stats.data_ptr(), n,
                                              0.0, 60.0, None)
        assert rc == 0, _lib.last_error()
        st = (_lib.CellStats * n).from_buffer_copy(d_stats.cpu().numpy().tobytes())
        status = np.array([x.status for x in st])
        nst = np.array([x.nst for x in st])
        np.testing.assert_array_equal(status, ref_stats["status"], err_msg=f"call {call}")
        np.testing.assert_array_equal(nst, ref_stats["nst"], err_msg=f"call {call}")
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=RTOL, atol=0,
                                   err_msg=f"call {call}")


def test_noalloc_rejects_missing_buffers(cb05):
    from camp_b200 import _lib
    from camp_b200.solver import Solver

    s = Solver(cb05, 4)
    s.initialize(abs_tol=np.full(cb05.n_state_var, 1e-8), rel_tol=1e-4)
    lib = _lib.load()
    rc = lib.camp_b200_run_device_noalloc(s._h, None, None, None, None, 4, 0.0, 60.0, None)
    assert rc == -1
    assert "device buffers" in _lib.last_error()
