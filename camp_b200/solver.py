"""Python host API over libcamp_b200 — the mirror of ``camp_solver_data_t``.

The reference's Fortran ``camp_solver_data_t`` (src/camp_solver_data.F90)
creates the C solver with ``solver_new``, feeds it every reaction's packed
data with ``rxn_add_condensed_data``, calls ``solver_initialize`` and then
``solver_run`` once per host time step, and pushes per-cell host-set rates
(photolysis, emission, first-order loss, wet deposition) through
``rxn_update_data``.  :class:`Solver` makes the same calls, in the
same order, through the C ABI of ``libcamp_b200.so``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mechanism import (RXN_EMISSION, RXN_FIRST_ORDER_LOSS, RXN_PHOTOLYSIS, RXN_WET_DEPOSITION,
                        Mechanism)

_UPDATE_KIND = {RXN_PHOTOLYSIS: "photolysis", RXN_EMISSION: "emission",
                RXN_FIRST_ORDER_LOSS: "first_order_loss", RXN_WET_DEPOSITION: "wet_deposition"}

# solver defaults, src/camp_solver_data.F90:33-37
DEFAULT_MAX_STEPS = 10000
DEFAULT_MAX_CONV_FAILS = 1000

FP64 = 0
MIXED = 1


class SolverError(RuntimeError):
    pass


class Solver:
    """One CAMP solver instance for ``n_cells`` cells of ``mech``."""

    def __init__(self, mech: Mechanism, n_cells: int):
        self.lib = _lib.load()
        self.mech = mech
        self.n_cells = int(n_cells)
        self._h = self.lib.solver_new(
            mech.n_state_var, self.n_cells, np.ascontiguousarray(mech.var_type, np.int32),
            mech.n_rxn, mech.n_rxn_int_param, mech.n_rxn_float_param, mech.n_rxn_env_param,
            *mech.aero_sizes(), *mech.sub_sizes(),
        )
        if not self._h:
            raise SolverError(_lib.last_error())
        # reactions, then aerosol phases and representations, the order of
        # camp_solver_data%initialize (src/camp_solver_data.F90:635-700)
        for r in mech.rxns:
            self.lib.rxn_add_condensed_data(
                r.rxn_type, r.ints.size, r.floats.size, r.n_env,
                np.ascontiguousarray(r.ints, np.int32), np.ascontiguousarray(r.floats, np.float64),
                self._h,
            )
        for p in mech.aero_phases:
            self.lib.aero_phase_add_condensed_data(
                p.ints.size, p.floats.size, np.ascontiguousarray(p.ints, np.int32),
                np.ascontiguousarray(p.floats, np.float64), self._h)
        for a in mech.aero_reps:
            self.lib.aero_rep_add_condensed_data(
                a.rep_type, a.ints.size, a.floats.size, a.n_env,
                np.ascontiguousarray(a.ints, np.int32), np.ascontiguousarray(a.floats, np.float64),
                self._h)
        # sub-models in priority order (src/camp_solver_data.F90:700-720)
        for sm in mech.sub_models:
            self.lib.sub_model_add_condensed_data(
                sm.sub_type, sm.ints.size, sm.floats.size, sm.n_env,
                np.ascontiguousarray(sm.ints, np.int32), np.ascontiguousarray(sm.floats, np.float64),
                self._h)
        self.ready = False

    # ------------------------------------------------------------------
    def initialize(self, abs_tol=None, rel_tol: float | None = None,
                   max_steps: int = DEFAULT_MAX_STEPS,
                   max_conv_fails: int = DEFAULT_MAX_CONV_FAILS) -> None:
        """solver_initialize; abs_tol per state variable (default: mechanism's)."""
        atol = np.ascontiguousarray(self.mech.abs_tol if abs_tol is None else abs_tol, np.float64)
        if atol.size == 1:
            atol = np.full(self.mech.n_state_var, float(atol))
        rtol = self.mech.rel_tol if rel_tol is None else float(rel_tol)
        self.rtol = rtol
        self.atol = atol
        self.lib.solver_initialize(self._h, atol, rtol, int(max_steps), int(max_conv_fails))
        self.ready = bool(self.lib.camp_b200_is_ready(self._h))
        if not self.ready:
            raise SolverError(_lib.last_error())

    def build_sparsity_only(self, abs_tol=None, rel_tol=None) -> None:
        """solver_initialize without requiring a GPU: the host-side sparsity
        and packed-data update are done before any device work, so they can be
        inspected on a machine without CUDA devices."""
        atol = np.ascontiguousarray(self.mech.abs_tol if abs_tol is None else abs_tol, np.float64)
        rtol = self.mech.rel_tol if rel_tol is None else float(rel_tol)
        self.lib.solver_initialize(self._h, atol, rtol, DEFAULT_MAX_STEPS, DEFAULT_MAX_CONV_FAILS)
        self.ready = bool(self.lib.camp_b200_is_ready(self._h))

    def set_precision(self, mode: int) -> None:
        if self.lib.camp_b200_set_precision(self._h, int(mode)) != 0:
            raise SolverError(_lib.last_error())

    def set_launch(self, warps_per_block: int = 0, blocks_per_sm: int = 1) -> None:
        self.lib.camp_b200_set_launch(self._h, int(warps_per_block), int(blocks_per_sm))

    def autotune(self, state, env, t_initial: float, t_final: float) -> dict:
        """Times the candidate launch configurations on a sample of cells
        (host arrays; state is not modified) and keeps the fastest."""
        st = np.ascontiguousarray(state, np.float64)
        ev = np.ascontiguousarray(env, np.float64).reshape(-1, 2)
        n = st.shape[0]
        if self.lib.camp_b200_autotune(self._h, st.reshape(-1), ev.reshape(-1), n,
                                       float(t_initial), float(t_final)) != 0:
            raise SolverError(_lib.last_error())
        return self.tuning()

    def tuning(self) -> dict:
        w, hg, lu, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self.lib.camp_b200_get_tuning(self._h, C.byref(w), C.byref(hg), C.byref(lu),
                                      C.byref(ms))
        return {"warps_per_block": w.value, "hist_global": hg.value, "lu_mode": lu.value,
                "sample_ms": ms.value, "kernel": int(self.lib.camp_b200_get_kernel(self._h))}

    def set_graph(self, enable: bool) -> None:
        """Launch each run's device step as one CUDA graph."""
        self.lib.camp_b200_set_graph(self._h, int(bool(enable)))

    def set_layout(self, hist_global: int) -> None:
        """0: Nordsieck history and rate constants in shared memory; 1: in
        global memory (more resident cells per SM)."""
        if self.lib.camp_b200_set_layout(self._h, int(hist_global)) != 0:
            raise SolverError(_lib.last_error())

    def set_lu_mode(self, mode: int) -> None:
        if self.lib.camp_b200_set_lu_mode(self._h, int(mode)) != 0:
            raise SolverError(_lib.last_error())

    def set_kernel(self, kernel: int, place: int = -1) -> None:
        """0 = warp per cell, 1 = lane per cell (place: shared-memory bits),
        2 = block per cell."""
        if self.lib.camp_b200_set_kernel(self._h, int(kernel), int(place)) != 0:
            raise SolverError(_lib.last_error())

    def set_cost_ordering(self, enable: bool = True) -> None:
        self.lib.camp_b200_set_cost_ordering(self._h, 1 if enable else 0)

    # ------------------------------------------------------------------
    def solve(self, state: np.ndarray, env: np.ndarray, t_initial: float, t_final: float) -> int:
        """solver_run on host arrays; state [n_cells, n_state_var] in place."""
        if state.dtype != np.float64 or not state.flags.c_contiguous:
            raise TypeError("state must be a C-contiguous float64 array")
        # solver_run advances every cell the solver was created for
        if state.shape != (self.n_cells, self.mech.n_state_var):
            raise ValueError(f"state must be [{self.n_cells}, {self.mech.n_state_var}]")
        env = np.ascontiguousarray(env, np.float64)
        if env.size != 2 * self.n_cells:
            raise ValueError(f"env must hold {self.n_cells} (T, P) pairs")
        return int(self.lib.solver_run(self._h, state.reshape(-1), env.reshape(-1),
                                       float(t_initial), float(t_final)))

    def run_device(self, d_state, d_env, n_cells: int, t_initial: float, t_final: float,
                   stream=None) -> int:
        """Device-resident run; d_state/d_env are torch CUDA tensors or raw
        device pointers (int)."""
        ps = d_state.data_ptr() if hasattr(d_state, "data_ptr") else int(d_state)
        pe = d_env.data_ptr() if hasattr(d_env, "data_ptr") else int(d_env)
        st = None
        if stream is not None:
            st = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        rc = self.lib.camp_b200_run_device(self._h, ps, pe, int(n_cells), float(t_initial),
                                           float(t_final), st)
        if rc < 0:
            raise SolverError(_lib.last_error())
        return rc

    def launch_device(self, d_state, d_env, n_cells: int, t_initial: float, t_final: float,
                      stream=None) -> None:
        ps = d_state.data_ptr() if hasattr(d_state, "data_ptr") else int(d_state)
        pe = d_env.data_ptr() if hasattr(d_env, "data_ptr") else int(d_env)
        st = None
        if stream is not None:
            st = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        if self.lib.camp_b200_launch_device(self._h, ps, pe, int(n_cells), float(t_initial),
                                            float(t_final), st) < 0:
            raise SolverError(_lib.last_error())

    def sync_status(self, stream=None) -> int:
        st = None
        if stream is not None:
            st = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        rc = self.lib.camp_b200_sync_status(self._h, st)
        if rc < 0:
            raise SolverError(_lib.last_error())
        return rc

    # ------------------------------------------------------------------
    def set_photo_rate(self, cell: int, photo_id: int, base_rate: float) -> None:
        """Photolysis update through the reference's rxn_update_data path."""
        self.set_rate(cell, RXN_PHOTOLYSIS, photo_id, base_rate)

    def set_rate(self, cell: int, rxn_type: int, rxn_id: int, base_rate: float) -> None:
        """Base rate of the reaction of a host-rate type with RXN_ID_ rxn_id,
        through the update-data functions of that type and rxn_update_data."""
        kind = _UPDATE_KIND[rxn_type]
        ud = getattr(self.lib, f"rxn_{kind}_create_rate_update_data")()
        getattr(self.lib, f"rxn_{kind}_set_rate_update_data")(ud, int(rxn_id), float(base_rate))
        cursor = C.c_int(0)
        self.lib.rxn_update_data(int(cell), C.byref(cursor), int(rxn_type), ud, self._h)
        self.lib.solver_free_update_data(ud)

    def set_aero(self, cell: int, rep_id: int, section: int, what: str, value: float) -> None:
        """GMD [m] (what "gmd") or GSD ("gsd") of a mode of the modal/binned
        representation with that id, through its update data and
        aero_rep_update_data."""
        ud = getattr(self.lib, f"aero_rep_modal_binned_mass_create_{what}_update_data")()
        getattr(self.lib, f"aero_rep_modal_binned_mass_set_{what}_update_data")(
            ud, int(rep_id), int(section), float(value))
        cursor = C.c_int(0)
        self.lib.aero_rep_update_data(int(cell), C.byref(cursor), 2, ud, self._h)
        self.lib.solver_free_update_data(ud)

    def rate_column(self, column: int) -> tuple[int, int, int]:
        """(reaction index, type, RXN_ID_) of a host-rate column."""
        vals = [C.c_int() for _ in range(3)]
        if self.lib.camp_b200_rate_column(self._h, int(column), *[C.byref(v) for v in vals]):
            raise SolverError(_lib.last_error())
        return tuple(int(v.value) for v in vals)

    def set_photo_rates_device(self, d_rates, n_cells: int | None = None) -> None:
        """Photolysis rates already in device memory (torch CUDA tensor or
        pointer; None returns to the host rates)."""
        if d_rates is None:
            self.lib.camp_b200_set_photo_rates_device(self._h, None, 0)
            self._d_photo_ref = None
            return
        ptr = d_rates.data_ptr() if hasattr(d_rates, "data_ptr") else int(d_rates)
        n = self.n_cells if n_cells is None else int(n_cells)
        self._d_photo_ref = d_rates  # keep the buffer alive while in use
        if self.lib.camp_b200_set_photo_rates_device(self._h, ptr, n) != 0:
            raise SolverError(_lib.last_error())

    @property
    def n_photo(self) -> int:
        return int(self.lib.camp_b200_n_photo(self._h))

    def set_photo_rates(self, rates: np.ndarray) -> None:
        """Host-set base rates [n_cells, n_photo]: one column per reaction of
        a host-rate type (photolysis, first-order loss, emission, wet
        deposition) in mechanism order; this sets the same values a loop of
        rxn_update_data calls would (see rate_column for a column's id)."""
        rates = np.ascontiguousarray(rates, np.float64)
        n = rates.shape[0]
        if rates.ndim != 2 or rates.shape[1] != self.n_photo:
            raise ValueError("rates must have one column per host-rate reaction")
        self.lib.camp_b200_set_photo_rates(self._h, rates.reshape(-1), n)

    # ------------------------------------------------------------------
    def statistics(self) -> dict:
        ints = [C.c_int() for _ in range(9)]
        dbl = [C.c_double() for _ in range(2)]
        ints2 = [C.c_int() for _ in range(3)]
        dbl2 = [C.c_double() for _ in range(3)]
        self.lib.solver_get_statistics(self._h, *[C.byref(x) for x in ints],
                                       *[C.byref(x) for x in dbl], *[C.byref(x) for x in ints2],
                                       *[C.byref(x) for x in dbl2])
        keys = ["solver_flag", "num_steps", "RHS_evals", "LS_setups", "error_test_fails",
                "NLS_iters", "NLS_convergence_fails", "DLS_Jac_evals", "DLS_RHS_evals"]
        out = {k: v.value for k, v in zip(keys, ints)}
        out["last_time_step__s"] = dbl[0].value
        out["next_time_step__s"] = dbl[1].value
        out.update({k: v.value for k, v in zip(["Jac_eval_fails", "RHS_evals_total",
                                                 "Jac_evals_total"], ints2)})
        out.update({k: v.value for k, v in zip(["RHS_time__s", "Jac_time__s",
                                                 "max_loss_precision"], dbl2)})
        return out

    def cell_stats(self, n_cells: int | None = None) -> np.ndarray:
        n = self.n_cells if n_cells is None else int(n_cells)
        arr = (_lib.CellStats * n)()
        self.lib.camp_b200_get_cell_stats(self._h, arr, n)
        dt = np.dtype([("status", np.int32), ("nst", np.int32), ("nfe", np.int32),
                       ("nsetups", np.int32), ("netf", np.int32), ("nni", np.int32),
                       ("ncfn", np.int32), ("nje", np.int32), ("hu", np.float64),
                       ("hcur", np.float64)])
        return np.frombuffer(bytes(arr), dtype=dt).copy()

    def kernel(self) -> int:
        """The kernel solver_run uses: 0 warp, 1 lane, 2 block per cell."""
        return int(self.lib.camp_b200_get_kernel(self._h))

    def kernel_launches(self) -> int:
        return int(self.lib.camp_b200_kernel_launches(self._h))

    def last_kernel_ms(self) -> float:
        return float(self.lib.camp_b200_last_kernel_ms(self._h))

    # ------------------------------------------------------------------
    def solver_jac(self):
        n = self.lib.camp_b200_n_dep_var(self._h)
        nnz = self.lib.camp_b200_n_jac_elem(self._h)
        cp = np.zeros(n + 1, np.int32)
        ri = np.zeros(max(nnz, 1), np.int32)
        if self.lib.camp_b200_get_solver_jac(self._h, cp, ri) != 0:
            raise SolverError("sparsity not built")
        return cp, ri[:nnz]

    def rxn_int_data(self) -> np.ndarray:
        out = np.zeros(self.lib.camp_b200_rxn_int_data_size(self._h), np.int32)
        self.lib.camp_b200_get_rxn_int_data(self._h, out)
        return out

    def jac_map(self) -> np.ndarray:
        """The solver-Jacobian fold as (solver id, reaction-Jacobian id,
        parameter id) rows."""
        n = self.lib.camp_b200_n_mapped_values(self._h)
        if n < 0:
            raise SolverError("sparsity not built")
        out = np.zeros(3 * max(n, 1), np.int32)
        self.lib.camp_b200_get_jac_map(self._h, out)
        return out[: 3 * n].reshape(n, 3)

    def lu_order(self) -> np.ndarray:
        out = np.zeros(self.lib.camp_b200_n_dep_var(self._h), np.int32)
        self.lib.camp_b200_get_lu_order(self._h, out)
        return out

    def n_lu(self) -> int:
        return int(self.lib.camp_b200_n_lu_elem(self._h))

    def block_tables(self) -> bytes:
        """The block-per-cell kernel's tables as built on the host (the
        BlockOff header, then its sections)."""
        n = int(self.lib.camp_b200_get_block_tables(self._h, None, 0))
        if n < 0:
            raise SolverError(_lib.last_error())
        buf = (C.c_uint8 * n)()
        self.lib.camp_b200_get_block_tables(self._h, buf, n)
        return bytes(buf)

    def check_jac(self, state, env, h: float, rel_tol: float = 1e-4, abs_tol: float = 1e-9):
        """Finite-difference audit of the device Jacobian at these states;
        returns (n_failed per cell, worst relative difference per cell)."""
        state = np.ascontiguousarray(state, np.float64)
        env = np.ascontiguousarray(env, np.float64)
        nc = state.shape[0]
        worst = np.zeros(nc, np.float64)
        nfail = np.zeros(nc, np.int32)
        if self.lib.camp_b200_check_jac(self._h, state.reshape(-1), env.reshape(-1), nc,
                                        float(h), float(rel_tol), float(abs_tol), worst,
                                        nfail) < 0:
            raise SolverError(_lib.last_error())
        return nfail, worst

    def check_precision(self, state, env, h: float) -> np.ndarray:
        """Per cell, the error-weighted RMS difference of the FP32 and FP64
        solves of I - h J at these states (see camp_b200_check_precision)."""
        state = np.ascontiguousarray(state, np.float64)
        env = np.ascontiguousarray(env, np.float64)
        nc = state.shape[0]
        out = np.zeros(nc, np.float64)
        if self.lib.camp_b200_check_precision(self._h, state.reshape(-1), env.reshape(-1), nc,
                                              float(h), out) < 0:
            raise SolverError(_lib.last_error())
        return out

    def eval_deriv(self, state, env, h):
        state = np.ascontiguousarray(state, np.float64)
        nc = state.shape[0]
        n = self.lib.camp_b200_n_dep_var(self._h)
        rp, rl, f = (np.zeros(nc * n) for _ in range(3))
        if self.lib.camp_b200_eval_deriv(self._h, state.reshape(-1),
                                         np.ascontiguousarray(env, np.float64).reshape(-1),
                                         nc, float(h), rp, rl, f) != 0:
            raise SolverError(_lib.last_error())
        return f.reshape(nc, n), rp.reshape(nc, n), rl.reshape(nc, n)

    def eval_jac(self, state, env, h):
        state = np.ascontiguousarray(state, np.float64)
        nc = state.shape[0]
        nnz = self.lib.camp_b200_n_jac_elem(self._h)
        jp, jl = np.zeros(nc * nnz), np.zeros(nc * nnz)
        if self.lib.camp_b200_eval_jac(self._h, state.reshape(-1),
                                       np.ascontiguousarray(env, np.float64).reshape(-1),
                                       nc, float(h), jp, jl) != 0:
            raise SolverError(_lib.last_error())
        jp, jl = jp.reshape(nc, nnz), jl.reshape(nc, nnz)
        return jp - jl, jp, jl

    def free(self) -> None:
        if self._h:
            self.lib.solver_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
