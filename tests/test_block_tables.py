"""Tables of the block-per-cell kernel, checked on the CPU.

The block-per-cell kernel (camp_b200/csrc/block.cuh) factors I - gamma*J
right-looking, one pivot at a time: the sparse head pivots from tabulated
update targets, the trailing dense block of the LU by computed addresses, the
L entries of column k scaled during pivot k + 1; it solves the head rows by
levels and the dense block by panels of 32 columns.  These tests replay that
schedule in numpy on the tables the library builds (every index the kernel
reads comes from them) for a random matrix with the mechanism's LU pattern,
and check the factors and the solution against dense linear algebra.  They
also check the tables' invariants: the dense block is dense, each head
pivot's targets are the pattern's (L entry, U entry) products, the levels
respect every dependency.
"""
import struct

import numpy as np
import pytest

FIELDS = ("bytes n n_rxn n_part n_jac n_lu n_coef r0 n_hf n_hb rx_word rx_vptr coef fg_ptr "
          "fg_ent jg_ptr jg_mid jg_w0 jg_w1 jg_row lu_src lu_perm lu_rowptr lu_col lu_diag "
          "dpos ub lk_ptr lk_pos tg_ptr tg hf_ptr hf_rows hb_ptr hb_rows dep_state atol").split()


def parse(blob: bytes) -> dict:
    """Arrays of the tables, by the BlockOff header (blob.hpp)."""
    o = dict(zip(FIELDS, struct.unpack_from(f"<{len(FIELDS)}i", blob, 0)))
    n, r0 = o["n"], o["r0"]

    def arr(name, dtype, count):
        return np.frombuffer(blob, dtype=dtype, count=count, offset=o[name]).astype(np.int64)

    t = dict(o)
    t["lu_perm"] = arr("lu_perm", np.uint16, n)
    t["lu_rowptr"] = arr("lu_rowptr", np.uint16, n + 1)
    t["lu_col"] = arr("lu_col", np.uint16, o["n_lu"])
    t["lu_diag"] = arr("lu_diag", np.uint16, n)
    t["lu_src"] = arr("lu_src", np.uint16, o["n_lu"])
    t["dpos"] = arr("dpos", np.uint16, n - r0)
    t["ub"] = arr("ub", np.uint16, r0)
    t["lk_ptr"] = arr("lk_ptr", np.uint32, r0 + 1)
    t["lk_pos"] = arr("lk_pos", np.uint16, int(t["lk_ptr"][-1]))
    t["tg_ptr"] = arr("tg_ptr", np.uint32, r0 + 1)
    t["tg"] = arr("tg", np.uint16, int(t["tg_ptr"][-1]))
    t["hf_ptr"] = arr("hf_ptr", np.uint16, o["n_hf"] + 1)
    t["hf_rows"] = arr("hf_rows", np.uint16, int(t["hf_ptr"][-1]))
    t["hb_ptr"] = arr("hb_ptr", np.uint16, o["n_hb"] + 1)
    t["hb_rows"] = arr("hb_rows", np.uint16, int(t["hb_ptr"][-1]))
    return t


def pattern(t) -> np.ndarray:
    n = t["n"]
    P = np.zeros((n, n), bool)
    for i in range(n):
        P[i, t["lu_col"][t["lu_rowptr"][i]:t["lu_rowptr"][i + 1]]] = True
    return P


def factor(t, LU):
    """op_factor's schedule on the values LU (in place); returns dinv."""
    n, r0 = t["n"], t["r0"]
    diag, rowptr, dpos = t["lu_diag"], t["lu_rowptr"], t["dpos"]
    dinv = np.zeros(n)
    dprev = 0.0
    for k in range(n):
        dk = 1.0 / LU[diag[k]]
        dinv[k] = dk
        if k > 0:
            kp = k - 1
            if kp < r0:
                LU[t["lk_pos"][t["lk_ptr"][kp]:t["lk_ptr"][kp + 1]]] *= dprev
            else:
                LU[dpos[k - r0:] + (kp - r0)] *= dprev
        if k < r0:
            lk = t["lk_pos"][t["lk_ptr"][k]:t["lk_ptr"][k + 1]]
            u0 = diag[k] + 1
            nu = rowptr[k + 1] - u0
            tg = t["tg"][t["tg_ptr"][k]:t["tg_ptr"][k] + len(lk) * nu].reshape(len(lk), nu)
            upd = np.outer(LU[lk] * dk, LU[u0:u0 + nu])
            # targets of one pivot are distinct: a plain scatter
            assert len(np.unique(tg)) == tg.size
            LU[tg.ravel()] -= upd.ravel()
        else:
            uk = dpos[k - r0] - r0
            for i in range(k + 1, n):
                ri = dpos[i - r0] - r0
                l = LU[ri + k] * dk
                LU[ri + k + 1:ri + n] -= l * LU[uk + k + 1:uk + n]
        dprev = dk
    return dinv


def solve(t, LU, dinv, rhs):
    """op_solve's schedule: rhs (dependent order) -> M^{-1} rhs."""
    n, r0 = t["n"], t["r0"]
    perm, rowptr, col, diag, dpos, ub = (t["lu_perm"], t["lu_rowptr"], t["lu_col"],
                                         t["lu_diag"], t["dpos"], t["ub"])
    z = rhs[perm].copy()
    for lv in range(t["n_hf"]):
        rows = t["hf_rows"][t["hf_ptr"][lv]:t["hf_ptr"][lv + 1]]
        new = {i: z[i] - LU[rowptr[i]:diag[i]] @ z[col[rowptr[i]:diag[i]]] for i in rows}
        for i, v in new.items():
            z[i] = v
    for i in range(r0, n):
        q0, q1 = rowptr[i], dpos[i - r0]
        z[i] -= LU[q0:q1] @ z[col[q0:q1]]
    for c0 in range(r0, n, 32):
        c1 = min(c0 + 32, n)
        for i in range(c0, c1):
            ri = dpos[i - r0] - r0
            z[i] -= LU[ri + c0:ri + i] @ z[c0:i]
        for i in range(c1, n):
            ri = dpos[i - r0] - r0
            z[i] -= LU[ri + c0:ri + c1] @ z[c0:c1]
    np_ = (n - r0 + 31) // 32
    for pp in range(np_ - 1, -1, -1):
        c0 = r0 + 32 * pp
        c1 = min(c0 + 32, n)
        for i in range(c1 - 1, c0 - 1, -1):
            ri = dpos[i - r0] - r0
            z[i] = (z[i] - LU[ri + i + 1:ri + c1] @ z[i + 1:c1]) * dinv[i]
        for i in range(r0, c0):
            ri = dpos[i - r0] - r0
            z[i] -= LU[ri + c0:ri + c1] @ z[c0:c1]
    for i in range(r0):
        q0, q1 = ub[i], rowptr[i + 1]
        z[i] -= LU[q0:q1] @ z[col[q0:q1]]
    for lv in range(t["n_hb"]):
        rows = t["hb_rows"][t["hb_ptr"][lv]:t["hb_ptr"][lv + 1]]
        new = {i: (z[i] - LU[diag[i] + 1:ub[i]] @ z[col[diag[i] + 1:ub[i]]]) * dinv[i]
               for i in rows}
        for i, v in new.items():
            z[i] = v
    out = np.zeros(n)
    out[perm] = z
    return out


def _tables(mech):
    from camp_b200.solver import Solver

    s = Solver(mech, 4)
    s.build_sparsity_only()
    return parse(s.block_tables())


@pytest.fixture(scope="module")
def large_mech():
    import tempfile

    from camp_b200.synth import load_synthetic

    with tempfile.TemporaryDirectory() as td:
        mech, _ = load_synthetic(td, 200, 600)
    return mech


def _check(t, seed):
    n = t["n"]
    P = pattern(t)
    rng = np.random.default_rng(seed)
    A = np.where(P, rng.uniform(-1.0, 1.0, (n, n)), 0.0)
    A[np.arange(n), np.arange(n)] = n + rng.uniform(0.0, 1.0, n)
    LU = np.array([A[i, c] for i in range(n)
                   for c in t["lu_col"][t["lu_rowptr"][i]:t["lu_rowptr"][i + 1]]])
    dinv = factor(t, LU)
    # the factors reproduce A (pivot order)
    L = np.eye(n)
    U = np.zeros((n, n))
    for i in range(n):
        for q in range(t["lu_rowptr"][i], t["lu_rowptr"][i + 1]):
            c = t["lu_col"][q]
            if c < i:
                L[i, c] = LU[q]
            else:
                U[i, c] = LU[q]
    assert np.allclose(L @ U, A, rtol=1e-12, atol=1e-12 * n)
    assert np.allclose(dinv, 1.0 / np.diag(U), rtol=1e-14)
    # the solve in dependent order: M x = b with M[perm][:, perm] = A
    b = rng.uniform(-1.0, 1.0, n)
    x = solve(t, LU, dinv, b)
    perm = t["lu_perm"]
    M = np.zeros((n, n))
    M[np.ix_(perm, perm)] = A
    assert np.allclose(M @ x, b, rtol=1e-10, atol=1e-12)


def _invariants(t):
    n, r0 = t["n"], t["r0"]
    P = pattern(t)
    assert P[r0:, r0:].all()
    assert r0 == 0 or not (P[r0 - 1:, r0 - 1].all() and P[r0 - 1, r0 - 1:].all())
    for i in range(r0, n):
        assert t["lu_col"][t["dpos"][i - r0]] == r0
    for k in range(r0):
        rows = np.nonzero(P[k + 1:, k])[0] + k + 1
        lk = t["lk_pos"][t["lk_ptr"][k]:t["lk_ptr"][k + 1]]
        assert len(lk) == len(rows)
    flev = np.full(n, -1)
    for lv in range(t["n_hf"]):
        for i in t["hf_rows"][t["hf_ptr"][lv]:t["hf_ptr"][lv + 1]]:
            deps = t["lu_col"][t["lu_rowptr"][i]:t["lu_diag"][i]]
            assert all(0 <= flev[d] < lv for d in deps)
            flev[i] = lv
    assert (flev[:r0] >= 0).all()
    blev = np.full(n, -1)
    for lv in range(t["n_hb"]):
        for i in t["hb_rows"][t["hb_ptr"][lv]:t["hb_ptr"][lv + 1]]:
            deps = t["lu_col"][t["lu_diag"][i] + 1:t["ub"][i]]
            assert all(0 <= blev[d] < lv for d in deps)
            blev[i] = lv
    assert (blev[:r0] >= 0).all()


def test_large_mechanism_tables(large_mech):
    t = _tables(large_mech)
    assert t["n"] == 200 and t["n_lu"] == 18681
    # the 200-species mechanism's LU ends in a dense 112 x 112 block
    assert t["r0"] == 88
    _invariants(t)
    _check(t, 3)


@pytest.mark.parametrize("which", ["cb05", "mod37"])
def test_gas_mechanism_tables(request, which):
    t = _tables(request.getfixturevalue(which))
    _invariants(t)
    _check(t, 5)


def test_aerosol_mechanism_has_no_block_tables(mod37_aero):
    from camp_b200.solver import Solver, SolverError

    s = Solver(mod37_aero, 4)
    s.build_sparsity_only()
    with pytest.raises(SolverError, match="CTA-per-cell"):
        s.block_tables()
