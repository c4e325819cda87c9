"""Python handle on the serving loop of libcamp_b200 (camp_b200_server_*).

Column solves of different sizes, mechanisms and host steps are submitted as
they arrive; the library's dispatcher thread admits them in arrival order as
slots and memory free up and runs them concurrently on the GPU (continuous
batching).  See include/camp_b200.h for the C interface.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .solver import Solver, SolverError


class Server:
    def __init__(self, n_slots: int = 8, device_mb: float = 2048.0, host_mb: float = 512.0):
        self.lib = _lib.load()
        self._h = self.lib.camp_b200_server_new(int(n_slots), float(device_mb), float(host_mb))
        if not self._h:
            raise SolverError(_lib.last_error())
        self._keep: dict[int, tuple] = {}
        self._cols: dict[int, tuple] = {}
        self._mech_nstate: list[int] = []

    def add_solver(self, solver: Solver) -> int:
        """Registers an initialised solver; returns its mechanism index."""
        m = self.lib.camp_b200_server_add_solver(self._h, solver._h)
        if m < 0:
            raise SolverError(_lib.last_error())
        self._mech_nstate.append(solver.mech.n_state_var)
        return m

    def submit(self, mech: int, state: np.ndarray, env: np.ndarray, photo: np.ndarray | None,
               t_initial: float, t_final: float) -> int:
        """Queues a column; ``state`` [n, n_state_var] is updated by wait()."""
        st = np.ascontiguousarray(state, np.float64)
        ev = np.ascontiguousarray(env, np.float64)
        ph = None if photo is None or photo.size == 0 else np.ascontiguousarray(photo, np.float64)
        n = st.shape[0]
        rid = self.lib.camp_b200_server_submit(
            self._h, int(mech), st.ctypes.data, ev.ctypes.data,
            ph.ctypes.data if ph is not None else None, n, float(t_initial), float(t_final))
        if rid < 0:
            raise SolverError(_lib.last_error())
        self._keep[rid] = (st, ev, ph, state, st.shape[0])
        return rid

    def wait(self, rid: int):
        """Returns (rc, latency_ms, state, stats) of a request."""
        st, ev, ph, orig, n = self._keep.pop(rid)
        lat = C.c_double()
        stats = (_lib.CellStats * n)()
        rc = self.lib.camp_b200_server_wait(self._h, int(rid), C.byref(lat), stats, n)
        if rc < 0:
            raise SolverError(_lib.last_error())
        if orig is not None and orig is not st:
            orig[...] = st
        status = np.array([x.status for x in stats], np.int32)
        nst = np.array([x.nst for x in stats], np.int32)
        return rc, lat.value, st, {"status": status, "nst": nst}

    def pending(self) -> int:
        return int(self.lib.camp_b200_server_pending(self._h))

    # device-resident columns ------------------------------------------
    def open_column(self, mech: int, state: np.ndarray) -> int:
        """Copies a column's concentrations [n, n_state_var] to the device
        once; returns the column id."""
        st = np.ascontiguousarray(state, np.float64)
        cid = self.lib.camp_b200_server_open_column(self._h, int(mech), st.ctypes.data,
                                                    st.shape[0])
        if cid < 0:
            raise SolverError(_lib.last_error())
        self._cols[cid] = (int(mech), st.shape)
        return cid

    def submit_column(self, column: int, env: np.ndarray, photo: np.ndarray | None,
                      t_initial: float, t_final: float) -> int:
        """Queues one host step of a resident column; wait() returns its
        (rc, latency_ms, None, stats)."""
        ev = np.ascontiguousarray(env, np.float64)
        ph = None if photo is None or photo.size == 0 else np.ascontiguousarray(photo, np.float64)
        rid = self.lib.camp_b200_server_submit_column(
            self._h, int(column), ev.ctypes.data, ph.ctypes.data if ph is not None else None,
            float(t_initial), float(t_final))
        if rid < 0:
            raise SolverError(_lib.last_error())
        self._keep[rid] = (None, ev, ph, None, self._cols[column][1][0])
        return rid

    def read_column(self, column: int) -> np.ndarray:
        out = np.zeros(self._cols[column][1], np.float64)
        if self.lib.camp_b200_server_read_column(self._h, int(column), out.ctypes.data) != 0:
            raise SolverError(_lib.last_error())
        return out

    def close_column(self, column: int) -> None:
        if self.lib.camp_b200_server_close_column(self._h, int(column)) != 0:
            raise SolverError(_lib.last_error())
        self._cols.pop(column, None)

    def close(self) -> None:
        if self._h:
            self.lib.camp_b200_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
