"""ctypes front end of the oracle libraries (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.  The product,
``camp_b200``, never imports it.

Two libraries live in ``oracle/_ref`` (built by ``oracle/Makefile``):

* ``libcamp_oracle.so`` - the CPU restatement in ``camp_oracle.c``: gas-phase
  f/J restated from the reference's ``src/rxns/rxn_*.c``, the sparsity build
  of ``src/camp_solver.c:1417-1712``, a sparse LU, and the CVODE BDF
  algorithm restated per cell.  Needs only gcc, so it builds anywhere.
* ``libcamp_ref.so`` - the reference's own reaction/derivative/Jacobian C
  sources compiled from the reference tree plus ``ref_glue.c``.  Present only
  where the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(REF_DIR, "libcamp_oracle.so")
REF_SO = os.path.join(REF_DIR, "libcamp_ref.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class OracleStats(C.Structure):
    _fields_ = [
        ("nst", C.c_long),
        ("nfe", C.c_long),
        ("nsetups", C.c_long),
        ("netf", C.c_long),
        ("nni", C.c_long),
        ("ncfn", C.c_long),
        ("nje", C.c_long),
        ("hu", C.c_double),
        ("hcur", C.c_double),
        ("flag", C.c_int),
        ("qu", C.c_int),
    ]


def build(with_ref: bool = True) -> None:
    """Builds the oracle libraries (the reference part only if its tree exists)."""
    target = "all" if with_ref else "oracle"
    cmd = ["make", "-s", "-C", HERE, target]
    ref = os.environ.get("CAMP_REFERENCE_ROOT")
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


_oracle_lib = None
_ref_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        lib = C.CDLL(ORACLE_SO)
        vp = C.c_void_p
        lib.om_new.restype = vp
        lib.om_new.argtypes = [C.c_int, _i32p, C.c_int]
        lib.om_add_rxn.restype = C.c_int
        lib.om_add_rxn.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f64p]
        lib.om_build.restype = C.c_int
        lib.om_build.argtypes = [vp]
        lib.om_set_abs_tol.argtypes = [vp, _f64p]
        lib.om_set_experiment.restype = C.c_int
        lib.om_set_experiment.argtypes = [vp, C.c_double, C.c_int]
        lib.om_free.argtypes = [vp]
        for name in (
            "om_n_dep_var",
            "om_n_rxn_env_data",
            "om_n_rxn_jac_elem",
            "om_n_solver_jac_elem",
            "om_n_lu_elem",
            "om_rxn_int_data_size",
            "om_n_param_jac_elem",
            "om_n_mapped_values",
        ):
            getattr(lib, name).restype = C.c_int
            getattr(lib, name).argtypes = [vp]
        lib.om_get_rxn_jac.argtypes = [vp, _i32p, _i32p]
        lib.om_get_solver_jac.argtypes = [vp, _i32p, _i32p]
        lib.om_get_rxn_int_data.argtypes = [vp, _i32p]
        lib.om_get_lu_order.argtypes = [vp, _i32p]
        lib.om_get_jac_map.argtypes = [vp, _i32p]
        lib.om_add_sub_model.restype = C.c_int
        lib.om_add_sub_model.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f64p]
        lib.om_set_photo_rate.restype = C.c_int
        lib.om_set_photo_rate.argtypes = [vp, _f64p, C.c_int, C.c_double]
        lib.om_set_rate.restype = C.c_int
        lib.om_set_rate.argtypes = [vp, _f64p, C.c_int, C.c_int, C.c_double]
        lib.om_add_aero_phase.restype = C.c_int
        lib.om_add_aero_phase.argtypes = [vp, C.c_int, C.c_int, _i32p, _f64p]
        lib.om_add_aero_rep.restype = C.c_int
        lib.om_add_aero_rep.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f64p]
        lib.om_set_aero_env.restype = C.c_int
        lib.om_set_aero_env.argtypes = [vp, _f64p, C.c_int, C.c_int, C.c_int, C.c_double]
        lib.om_update_env.argtypes = [vp, _f64p, _f64p]
        lib.om_deriv.argtypes = [vp, _f64p, _f64p, C.c_double, _f64p, _f64p, _f64p]
        lib.om_jac.argtypes = [vp, _f64p, _f64p, C.c_double, _f64p]
        lib.om_solve.restype = C.c_int
        lib.om_solve.argtypes = [
            vp, C.c_int, _f64p, _f64p, _f64p, C.c_double, C.c_double, C.c_double,
            _f64p, C.c_int, C.c_int, C.c_int, _i32p, C.POINTER(OracleStats),
        ]
        lib.om_solve_cb.restype = C.c_int
        lib.om_solve_cb.argtypes = [
            vp, C.c_int, _f64p, C.c_double, C.c_double, C.c_double, _f64p,
            C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p),
            _i32p, C.POINTER(OracleStats),
        ]
        _oracle_lib = lib
    return _oracle_lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(
                "oracle/_ref/libcamp_ref.so is absent (it is built from the reference tree)"
            )
        lib = C.CDLL(REF_SO)
        vp = C.c_void_p
        lib.ref_new.restype = vp
        lib.ref_new.argtypes = [C.c_int, C.c_int, _i32p] + [C.c_int] * 15
        lib.rxn_add_condensed_data.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f64p, vp]
        lib.ref_build.restype = C.c_int
        lib.ref_build.argtypes = [vp]
        lib.ref_set_abs_tol.argtypes = [vp, _f64p]
        for name in (
            "ref_n_dep_var",
            "ref_n_rxn_jac_elem",
            "ref_n_solver_jac_elem",
            "ref_n_mapped_values",
            "ref_n_rxn_env_data",
            "ref_rxn_int_data_size",
        ):
            getattr(lib, name).restype = C.c_int
            getattr(lib, name).argtypes = [vp]
        lib.ref_get_rxn_jac.argtypes = [vp, _i32p, _i32p]
        lib.ref_get_solver_jac.argtypes = [vp, _i32p, _i32p]
        lib.ref_get_jac_map.argtypes = [vp, _i32p]
        lib.ref_get_rxn_int_data.argtypes = [vp, _i32p]
        lib.ref_get_rxn_env_data.argtypes = [vp, C.c_int, _f64p]
        lib.ref_set_rxn_env_data.argtypes = [vp, C.c_int, _f64p]
        lib.ref_set_state.argtypes = [vp, _f64p, _f64p]
        lib.ref_update_env.argtypes = [vp, C.c_int]
        lib.ref_calc_deriv.argtypes = [vp, C.c_int, C.c_double, _f64p, _f64p, _f64p]
        lib.ref_calc_jac.argtypes = [vp, C.c_int, C.c_double, _f64p, _f64p]
        lib.ref_free.argtypes = [vp]
        lib.rxn_update_data.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, vp, vp]
        for kind in ("photolysis", "emission", "first_order_loss", "wet_deposition"):
            getattr(lib, f"rxn_{kind}_create_rate_update_data").restype = vp
            getattr(lib, f"rxn_{kind}_set_rate_update_data").argtypes = [vp, C.c_int, C.c_double]
        lib.sub_model_add_condensed_data.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p,
                                                     _f64p, vp]
        lib.aero_phase_add_condensed_data.argtypes = [C.c_int, C.c_int, _i32p, _f64p, vp]
        lib.aero_rep_add_condensed_data.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p,
                                                    _f64p, vp]
        lib.aero_rep_update_data.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, vp, vp]
        for what in ("gmd", "gsd"):
            getattr(lib, f"aero_rep_modal_binned_mass_create_{what}_update_data").restype = vp
            getattr(lib, f"aero_rep_modal_binned_mass_set_{what}_update_data").argtypes = [
                vp, C.c_int, C.c_int, C.c_double]
        _ref_lib = lib
    return _ref_lib


class OracleModel:
    """The oracle's restated mechanism, built from packed reaction blocks."""

    def __init__(self, mech):
        self.lib = oracle_lib()
        self.mech = mech
        self.h = self.lib.om_new(mech.n_state_var, np.ascontiguousarray(mech.var_type, np.int32), mech.n_rxn)
        for r in mech.rxns:
            rc = self.lib.om_add_rxn(
                self.h, r.rxn_type, r.ints.size, r.floats.size, r.n_env,
                np.ascontiguousarray(r.ints, np.int32), np.ascontiguousarray(r.floats, np.float64),
            )
            if rc != 0:
                raise ValueError(f"oracle rejected reaction type {r.rxn_type} (code {rc})")
        for p in mech.aero_phases:
            self.lib.om_add_aero_phase(self.h, p.ints.size, p.floats.size,
                                       np.ascontiguousarray(p.ints, np.int32),
                                       np.ascontiguousarray(p.floats, np.float64))
        for a in mech.aero_reps:
            if self.lib.om_add_aero_rep(self.h, a.rep_type, a.ints.size, a.floats.size, a.n_env,
                                        np.ascontiguousarray(a.ints, np.int32),
                                        np.ascontiguousarray(a.floats, np.float64)) != 0:
                raise ValueError(f"oracle rejected aerosol representation type {a.rep_type}")
        for sm in mech.sub_models:
            if self.lib.om_add_sub_model(self.h, sm.sub_type, sm.ints.size, sm.floats.size,
                                         sm.n_env, np.ascontiguousarray(sm.ints, np.int32),
                                         np.ascontiguousarray(sm.floats, np.float64)) != 0:
                raise ValueError(f"oracle rejected sub-model type {sm.sub_type}")
        rc = self.lib.om_build(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle sparsity build failed (code {rc})")
        # the mechanism's tolerances, as solver_initialize would pass them
        self.lib.om_set_abs_tol(self.h, np.ascontiguousarray(mech.abs_tol, np.float64))
        self.n_dep = self.lib.om_n_dep_var(self.h)
        self.n_env = self.lib.om_n_rxn_env_data(self.h)
        self.n_rxn_jac = self.lib.om_n_rxn_jac_elem(self.h)
        self.n_jac = self.lib.om_n_solver_jac_elem(self.h)
        self.n_lu = self.lib.om_n_lu_elem(self.h)

    def __del__(self):
        try:
            self.lib.om_free(self.h)
        except Exception:
            pass

    # positivity rules of set_experiment (camp_oracle.h)
    POS_PROJECT, POS_GUESS_HELPER, POS_GUESS_HELPER_ONLY, POS_NONE = 0, 1, 2, 3

    def set_experiment(self, guard_step: float = 0.0, positivity: int = 0) -> None:
        """Integrator experiment switches (camp_oracle.h om_set_experiment):
        a fixed time_step for f and J instead of the current step (0 = the
        reference's semantics), and the positivity rule."""
        if self.lib.om_set_experiment(self.h, float(guard_step), int(positivity)) != 0:
            raise ValueError("invalid experiment setting")

    def solver_jac(self):
        cp = np.zeros(self.n_dep + 1, np.int32)
        ri = np.zeros(max(self.n_jac, 1), np.int32)
        self.lib.om_get_solver_jac(self.h, cp, ri)
        return cp, ri[: self.n_jac]

    def rxn_jac(self):
        cp = np.zeros(self.mech.n_state_var + 1, np.int32)
        ri = np.zeros(max(self.n_rxn_jac, 1), np.int32)
        self.lib.om_get_rxn_jac(self.h, cp, ri)
        return cp, ri[: self.n_rxn_jac]

    def jac_map(self):
        """(solver id, reaction-Jacobian id, parameter id) per mapped value."""
        n = self.lib.om_n_mapped_values(self.h)
        out = np.zeros(3 * max(n, 1), np.int32)
        self.lib.om_get_jac_map(self.h, out)
        return out[: 3 * n].reshape(n, 3)

    def rxn_int_data(self):
        out = np.zeros(self.lib.om_rxn_int_data_size(self.h), np.int32)
        self.lib.om_get_rxn_int_data(self.h, out)
        return out

    def lu_order(self):
        out = np.zeros(self.n_dep, np.int32)
        self.lib.om_get_lu_order(self.h, out)
        return out

    def _set_rates(self, re, rates: dict[int, float]) -> None:
        """Host-set base rates by RXN_ID_ (the reaction's type is looked up)."""
        for rid, rate in rates.items():
            rtype = self.mech.rxns[self.mech.rate_ids[int(rid)]].rxn_type
            self.lib.om_set_rate(self.h, re, int(rtype), int(rid), float(rate))

    def rxn_env(self, env, photo_rates: dict[int, float] | None = None):
        """One cell's rate constants for env=(T, P) and host-set base rates
        keyed by RXN_ID_ (photolysis, first-order loss, emission, wet
        deposition)."""
        re = np.zeros(max(self.n_env, 1), np.float64)
        self._set_rates(re, photo_rates or {})
        self.lib.om_update_env(self.h, np.asarray(env, np.float64), re)
        return re

    def _set_row(self, re, row) -> None:
        """One cell's host-set columns (``Mechanism.rate_columns`` order)."""
        for j, col in enumerate(self.mech.rate_columns()):
            v = float(row[j])
            if col[0] == "rxn":
                i = col[1]
                self.lib.om_set_rate(self.h, re, self.mech.rxns[i].rxn_type,
                                     self.mech.rate_id(i), v)
            else:
                self.lib.om_set_aero_env(self.h, re, col[1], col[2], 0 if col[0] == "gmd" else 1, v)

    def rxn_env_row(self, env, row):
        """rxn_env from a full row of host-set columns (rates, GMD, GSD)."""
        re = np.zeros(max(self.n_env, 1), np.float64)
        self._set_row(re, row)
        self.lib.om_update_env(self.h, np.asarray(env, np.float64), re)
        return re

    def deriv(self, state, rxn_env, time_step):
        f = np.zeros(self.n_dep)
        rp = np.zeros(self.n_dep)
        rl = np.zeros(self.n_dep)
        self.lib.om_deriv(self.h, np.ascontiguousarray(state, np.float64), rxn_env, float(time_step), f, rp, rl)
        return f, rp, rl

    def jac(self, state, rxn_env, time_step):
        j = np.zeros(max(self.n_jac, 1))
        self.lib.om_jac(self.h, np.ascontiguousarray(state, np.float64), rxn_env, float(time_step), j)
        return j[: self.n_jac]

    def solve(self, state, env, photo_rates, t0, t1, rtol, abs_tol, max_steps=10000,
              max_conv_fails=1000, n_threads=1):
        """Per-cell solve; state [n_cells, n_state_var] is updated in place.

        photo_rates is [n_cells, n_photo] of host-set base rates, one column
        per host-rate reaction in mechanism order (``Mechanism.rate_rxns``).
        Returns (n_failed, status, stats, state)."""
        state = np.ascontiguousarray(state, np.float64)
        n_cells = state.shape[0]
        env = np.ascontiguousarray(env, np.float64).reshape(n_cells, 2)
        re = np.zeros((n_cells, max(self.n_env, 1)), np.float64)
        photo_rates = np.asarray(photo_rates, np.float64).reshape(n_cells, -1)
        if photo_rates.shape[1] != len(self.mech.rate_columns()):
            raise ValueError("photo_rates must have one column per host-set value")
        for c in range(n_cells):
            self._set_row(re[c], photo_rates[c])
        status = np.zeros(n_cells, np.int32)
        stats = (OracleStats * n_cells)()
        nf = self.lib.om_solve(
            self.h, n_cells, state, env, re, float(t0), float(t1), float(rtol),
            np.ascontiguousarray(abs_tol, np.float64), int(max_steps), int(max_conv_fails),
            int(n_threads), status, stats,
        )
        return nf, status, stats, state


class RefModel:
    """The reference's own C code for one or more cells (via ref_glue.c)."""

    def __init__(self, mech, n_cells: int = 1):
        self.lib = ref_lib()
        self.mech = mech
        self.n_cells = n_cells
        self.h = self.lib.ref_new(
            mech.n_state_var, n_cells, np.ascontiguousarray(mech.var_type, np.int32),
            mech.n_rxn, mech.n_rxn_int_param, mech.n_rxn_float_param, mech.n_rxn_env_param,
            *mech.aero_sizes(), *mech.sub_sizes(),
        )
        for r in mech.rxns:
            self.lib.rxn_add_condensed_data(
                r.rxn_type, r.ints.size, r.floats.size, r.n_env,
                np.ascontiguousarray(r.ints, np.int32), np.ascontiguousarray(r.floats, np.float64), self.h,
            )
        for p in mech.aero_phases:
            self.lib.aero_phase_add_condensed_data(p.ints.size, p.floats.size,
                                                   np.ascontiguousarray(p.ints, np.int32),
                                                   np.ascontiguousarray(p.floats, np.float64),
                                                   self.h)
        for a in mech.aero_reps:
            self.lib.aero_rep_add_condensed_data(a.rep_type, a.ints.size, a.floats.size, a.n_env,
                                                 np.ascontiguousarray(a.ints, np.int32),
                                                 np.ascontiguousarray(a.floats, np.float64),
                                                 self.h)
        for sm in mech.sub_models:
            self.lib.sub_model_add_condensed_data(sm.sub_type, sm.ints.size, sm.floats.size,
                                                  sm.n_env,
                                                  np.ascontiguousarray(sm.ints, np.int32),
                                                  np.ascontiguousarray(sm.floats, np.float64),
                                                  self.h)
        self.lib.ref_set_abs_tol(self.h, np.ascontiguousarray(mech.abs_tol, np.float64))
        rc = self.lib.ref_build(self.h)
        if rc != 0:
            raise RuntimeError(f"reference sparsity build failed ({rc})")
        self.n_dep = self.lib.ref_n_dep_var(self.h)
        self.n_rxn_jac = self.lib.ref_n_rxn_jac_elem(self.h)
        self.n_jac = self.lib.ref_n_solver_jac_elem(self.h)
        self.n_env = self.lib.ref_n_rxn_env_data(self.h)
        self.state = np.zeros((n_cells, mech.n_state_var))
        self.env = np.zeros((n_cells, 2))
        self.lib.ref_set_state(self.h, self.state.reshape(-1), self.env.reshape(-1))

    def solver_jac(self):
        cp = np.zeros(self.n_dep + 1, np.int32)
        ri = np.zeros(max(self.n_jac, 1), np.int32)
        self.lib.ref_get_solver_jac(self.h, cp, ri)
        return cp, ri[: self.n_jac]

    def rxn_jac(self):
        cp = np.zeros(self.mech.n_state_var + 1, np.int32)
        ri = np.zeros(max(self.n_rxn_jac, 1), np.int32)
        self.lib.ref_get_rxn_jac(self.h, cp, ri)
        return cp, ri[: self.n_rxn_jac]

    def jac_map(self):
        n = self.lib.ref_n_mapped_values(self.h)
        out = np.zeros(3 * max(n, 1), np.int32)
        self.lib.ref_get_jac_map(self.h, out)
        return out[: 3 * n].reshape(n, 3)

    def rxn_int_data(self):
        """Packed reaction ints (with type slots) after rxn_update_ids."""
        out = np.zeros(self.lib.ref_rxn_int_data_size(self.h), np.int32)
        self.lib.ref_get_rxn_int_data(self.h, out)
        return out

    def set_photo_rate(self, cell: int, photo_id: int, rate: float) -> None:
        """Goes through the reference's rxn_update_data path."""
        self.set_rate(cell, 5, photo_id, rate)

    def set_rate(self, cell: int, rxn_type: int, rxn_id: int, rate: float) -> None:
        """A host-rate update through the reference's own update-data
        functions of that type and its rxn_update_data."""
        kind = {5: "photolysis", 12: "first_order_loss", 13: "emission",
                14: "wet_deposition"}[int(rxn_type)]
        ud = getattr(self.lib, f"rxn_{kind}_create_rate_update_data")()
        getattr(self.lib, f"rxn_{kind}_set_rate_update_data")(ud, int(rxn_id), float(rate))
        cursor = C.c_int(0)
        self.lib.rxn_update_data(int(cell), C.byref(cursor), int(rxn_type), ud, self.h)

    def set_aero(self, cell: int, rep: int, section: int, what: str, value: float) -> None:
        """GMD or GSD of a mode through the reference's update data and
        aero_rep_update_data (which also sets the mode's effective radius)."""
        lib = self.lib
        ud = getattr(lib, f"aero_rep_modal_binned_mass_create_{what}_update_data")()
        rep_id = int(self.mech.aero_reps[rep].ints[3])
        getattr(lib, f"aero_rep_modal_binned_mass_set_{what}_update_data")(ud, rep_id, section,
                                                                            float(value))
        cursor = C.c_int(0)
        lib.aero_rep_update_data(int(cell), C.byref(cursor), 2, ud, self.h)

    def set_rates(self, cell: int, row) -> None:
        """One cell's host-set columns (``Mechanism.rate_columns`` order)."""
        for j, col in enumerate(self.mech.rate_columns()):
            if col[0] == "rxn":
                i = col[1]
                self.set_rate(cell, self.mech.rxns[i].rxn_type, self.mech.rate_id(i),
                              float(row[j]))
            else:
                self.set_aero(cell, col[1], col[2], col[0], float(row[j]))

    def set_cell(self, cell, state, env):
        self.state[cell, :] = state
        self.env[cell, :] = env

    def update_env(self, cell):
        self.lib.ref_update_env(self.h, int(cell))

    def rxn_env(self, cell):
        out = np.zeros(max(self.n_env, 1))
        self.lib.ref_get_rxn_env_data(self.h, int(cell), out)
        return out

    def deriv(self, cell, time_step):
        f = np.zeros(self.n_dep)
        rp = np.zeros(self.n_dep)
        rl = np.zeros(self.n_dep)
        self.lib.ref_calc_deriv(self.h, int(cell), float(time_step), f, rp, rl)
        return f, rp, rl

    def jac(self, cell, time_step):
        jr = np.zeros(max(self.n_rxn_jac, 1))
        js = np.zeros(max(self.n_jac, 1))
        self.lib.ref_calc_jac(self.h, int(cell), float(time_step), jr, js)
        return js[: self.n_jac], jr[: self.n_rxn_jac]


def _ref_cb_setup(lib):
    vp = C.c_void_p
    lib.ref_cell_ctx_new.restype = vp
    lib.ref_cell_ctx_new.argtypes = [vp, C.c_int, C.c_double]
    lib.ref_cell_ctx_free.argtypes = [vp]


def ref_solve(mech, state, env, photo_rates, t0, t1, rtol, abs_tol, max_steps=10000,
              max_conv_fails=1000, n_threads=None, chunk=None):
    """Per-cell solve with the reference's own f/J (compiled reference C code)
    driven by the restated BDF and sparse LU.  Cells are split over threads,
    each with its own reference model object: contiguous ranges, or, with
    ``chunk``, chunks of that many cells that the threads take in turn (so
    that a few slow cells do not leave the other threads idle).  state is
    updated in place (dependent variables of successful cells, as
    solver_run does).

    Returns (status, stats) arrays."""
    import os
    import threading

    rlib = ref_lib()
    _ref_cb_setup(rlib)
    olib = oracle_lib()
    om = OracleModel(mech)
    n_cells = state.shape[0]
    n_threads = n_threads or os.cpu_count() or 1
    n_threads = max(1, min(n_threads, n_cells))
    dep = mech.dep_index()
    atol_dep = np.ascontiguousarray(np.asarray(abs_tol, np.float64)[dep])
    status = np.zeros(n_cells, np.int32)
    stats = (OracleStats * n_cells)()
    f_ptr = C.cast(rlib.ref_cb_rhs, C.c_void_p)
    j_ptr = C.cast(rlib.ref_cb_jac, C.c_void_p)
    TINY = 1.0e-60

    def work(c0, c1):
        nc = c1 - c0
        rm = RefModel(mech, nc)
        for c in range(nc):
            st = state[c0 + c].copy()
            for i, vt in enumerate(mech.var_type):
                if vt == 2:
                    st[i] = max(st[i], TINY)
            rm.set_cell(c, st, env[c0 + c])
            rm.set_rates(c, photo_rates[c0 + c])
            rm.update_env(c)
        y = np.ascontiguousarray(np.maximum(state[c0:c1][:, dep], TINY))
        ctxs = (C.c_void_p * nc)(*[rlib.ref_cell_ctx_new(rm.h, c, t1 - t0) for c in range(nc)])
        st_out = np.zeros(nc, np.int32)
        sub = (OracleStats * nc)()
        olib.om_solve_cb(om.h, nc, y, float(t0), float(t1), float(rtol), atol_dep,
                         int(max_steps), int(max_conv_fails), f_ptr, j_ptr, ctxs, st_out, sub)
        for c in range(nc):
            rlib.ref_cell_ctx_free(ctxs[c])
            status[c0 + c] = st_out[c]
            stats[c0 + c] = sub[c]
            if st_out[c] == 0:
                state[c0 + c, dep] = np.maximum(y[c], 0.0)

    if chunk:
        lock = threading.Lock()
        nxt = [0]

        def pull():
            while True:
                with lock:
                    a = nxt[0]
                    nxt[0] = min(n_cells, a + chunk)
                if a >= n_cells:
                    return
                work(a, min(n_cells, a + chunk))

        th = [threading.Thread(target=pull) for _ in range(n_threads)]
    else:
        bounds = [int(n_cells * t / n_threads) for t in range(n_threads + 1)]
        th = [threading.Thread(target=work, args=(bounds[t], bounds[t + 1]))
              for t in range(n_threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return status, stats
