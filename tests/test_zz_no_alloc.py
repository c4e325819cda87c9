"""The no-allocation entry point against the regular device entry point.

camp_b200_run_device_noalloc serves callers that cannot allocate device
memory while they run (a host model whose pool allocator owns the device
heap, or code running where cudaMalloc is not allowed): all buffers are the
caller's and the solve's scratch lives in a static device array inside the
library.  This test runs it twice in a row on the same inputs and checks each
result against camp_b200_run_device, on cb05cl_ae5 and on MONARCH mod37 with
its SOA, cloud and aqueous aerosol chemistry (whose per-cell rate matrix
carries every aerosol mode's GMD and GSD after the host-set reaction rates).
The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL = 1e-12  # both entry points run the same kernel: results agree to round-off


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("which", ["cb05", "mod37_aero"])
def test_noalloc_matches_run_device(request, which, precision):
    import torch

    from camp_b200 import _lib
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    mech = request.getfixturevalue(which)
    n = 300 if which == "cb05" else 120
    cells = make_cells(mech, n, 21)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4, max_steps=2000)
    # the rate matrix the caller passes: host-set reaction rates, then the
    # GMD / GSD columns of the aerosol modes
    assert cells.photo_rates.shape[1] == s.n_photo
    n_mode_cols = sum(1 for c in mech.rate_columns() if c[0] != "rxn")
    assert (n_mode_cols > 0) == (which == "mod37_aero")
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
