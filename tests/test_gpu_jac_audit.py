"""Finite-difference audit of the device Jacobian (the counterpart of the
reference's check_Jac debug check) on seeded cb05 cell states and on the
shipped MONARCH mod37 configuration, whose Jacobian chains the ZSR and
PD-FiTE parameter partials."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]


@pytest.mark.parametrize("h", [1.0, 60.0])
@pytest.mark.parametrize("which", ["cb05", "mod37_shipped"])
def test_jacobian_matches_finite_differences(request, which, h):
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    mech = request.getfixturevalue(which)
    n = 16
    cells = make_cells(mech, n, 7)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4)
    s.set_photo_rates(cells.photo_rates)
    nfail, worst = s.check_jac(cells.state, cells.env, h)
    assert np.all(nfail >= 0)
    n_jac = s.lib.camp_b200_n_jac_elem(s._h)
    # every element agrees with the difference estimate within its error
    # estimate at some step (a guard switching inside every tried step would
    # be reported here, as by the reference's check)
    assert nfail.sum() <= 0.001 * n * n_jac, (nfail, worst)


@pytest.mark.parametrize("which,limit", [("cb05", 0.05), ("mod37_aero", 0.05)])
def test_precision_audit_small_where_mixed_is_at_equal_error(request, which, limit):
    """The FP32 solve of I - h J at internal step sizes of 0.01-1 s, against
    the FP64 one, in the error-weighted norm: well below 1 on the mechanisms
    whose mixed solves are at the oracle's accuracy (the Newton iteration
    refines it).  At a whole 60 s host step single mod37 cells reach 0.4."""
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    mech = request.getfixturevalue(which)
    n = 32
    cells = make_cells(mech, n, 23)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4)
    s.set_photo_rates(cells.photo_rates)
    for h in (0.01, 1.0):
        err = s.check_precision(cells.state, cells.env, h)
        ok = err >= 0.0
        assert ok.sum() >= n // 2
        print(f"\n{which} h {h}: FP32 solve error median {np.median(err[ok]):.1e} "
              f"max {err[ok].max():.1e}")
        assert err[ok].max() < limit, (h, err[ok].max())


def test_precision_audit_flags_the_shipped_configuration(mod37_shipped):
    """On the shipped mod37 configuration (computed sulfate-mode water in
    fast aqueous equilibria) the FP32 solve is far less accurate: the audit
    flags it, and the FP64 form is the one to use there."""
    from camp_b200.cells import make_cells
    from camp_b200.solver import Solver

    mech = mod37_shipped
    n = 32
    cells = make_cells(mech, n, 23)
    s = Solver(mech, n)
    s.initialize(abs_tol=np.full(mech.n_state_var, 1e-8), rel_tol=1e-4)
    s.set_photo_rates(cells.photo_rates)
    err = s.check_precision(cells.state, cells.env, 1.0)
    ok = err >= 0.0
    assert ok.sum() >= n // 2
    print(f"\nshipped mod37 h 1: FP32 solve error median {np.median(err[ok]):.1e} "
          f"max {err[ok].max():.1e}")
    assert err[ok].max() > 0.1
