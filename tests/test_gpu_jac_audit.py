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
