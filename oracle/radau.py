"""Independent integrator cross-check (TEST INFRASTRUCTURE ONLY).

SciPy's Radau IIA (order 5, ``scipy.integrate.Radau``) run on the reference's
own derivative and Jacobian (the reference C sources compiled into
``oracle/_ref/libcamp_ref.so``), one cell at a time.  It shares no code with
the restated BDF of ``camp_oracle.c`` or with the device solver, so it checks
two things the BDF cannot check on itself:

* the tight oracle (the restated BDF at rtol 1e-10) is the solution of the
  reference's ODE, not of a shared integrator bug;
* whether a cell that the BDF cannot finish is integrable at all under the
  reference's semantics.

The reference's f takes the integrator's current step as ``time_step``
(``CVodeGetCurrentStep``, src/camp_solver.c:872-876) and its negative-yield
product guard multiplies it (src/rxns/rxn_arrhenius.c:153-160).  Radau is
given the same: each f and J call sees the step of the collocation system
being solved (``guard_step=None``), or a fixed step when an experiment asks
for one.  Only ``tests/`` use this module.
"""
from __future__ import annotations

import numpy as np

SMALL = 1.0e-30
TINY = 1.0e-60


class _StepTracker:
    """Makes the step of the Radau collocation system visible to f and J."""

    def __init__(self):
        import scipy.integrate._ivp.radau as radau

        self.radau = radau
        self.h = None
        self._orig = radau.solve_collocation_system

    def __enter__(self):
        orig = self._orig

        def tracked(fun, t, y, h, *a, **k):
            self.h = abs(h)
            return orig(fun, t, y, h, *a, **k)

        self.radau.solve_collocation_system = tracked
        return self

    def __exit__(self, *exc):
        self.radau.solve_collocation_system = self._orig


def radau_cell(mech, state, env, rates_row, t0, t1, rtol, atol, guard_step=None,
               max_steps=20000, ref=None):
    """Integrates one cell with Radau on the reference's f/J.

    state: the cell's full state row; env: (T, P); rates_row: its host-set
    columns (``Mechanism.rate_columns`` order).  Constants are clamped to
    TINY and dependent values to >= TINY as solver_run does
    (src/camp_solver.c:554-567); a trial state below -SMALL makes f return
    NaN, which Radau treats as a failed Newton iteration (the reference's
    recoverable f failure, src/camp_solver.c:805-833).

    Returns (status, steps, t_reached, y_dep): status is "finished",
    "failed" (Radau's step became too small) or "running" (max_steps spent
    before t1)."""
    from .oracle import RefModel

    rm = ref if ref is not None else RefModel(mech, 1)
    dep = mech.dep_index()
    n = len(dep)
    cp, ri = rm.solver_jac()
    cols = np.repeat(np.arange(n), np.diff(cp))
    st = np.asarray(state, np.float64).copy()
    for i, vt in enumerate(mech.var_type):
        if vt == 2:
            st[i] = max(st[i], TINY)
    rm.set_cell(0, st, env)
    rm.set_rates(0, rates_row)
    rm.update_env(0)
    dt = t1 - t0

    with _StepTracker() as trk:
        def time_step():
            if guard_step is not None:
                return guard_step
            return trk.h if trk.h else dt

        def load(y):
            if np.any(y < -SMALL):
                return False
            rm.state[0, dep] = np.where(y > -SMALL, y, TINY)
            return True

        def f(t, y):
            if not load(y):
                return np.full(n, np.nan)
            return rm.deriv(0, time_step())[0]

        def jac(t, y):
            J = np.zeros((n, n))
            load(np.maximum(y, 0.0))
            js, _ = rm.jac(0, time_step())
            J[ri, cols] = js
            return J

        y0 = np.maximum(st[dep], TINY)
        solver = trk.radau.Radau(f, t0, y0, t1, rtol=rtol, atol=atol, jac=jac)
        k = 0
        while solver.status == "running" and k < max_steps:
            solver.step()
            k += 1
    return solver.status, k, float(solver.t), np.asarray(solver.y).copy()
