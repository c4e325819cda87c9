"""Tables of the block-per-cell kernel, checked on the CPU.

The block-per-cell kernel (camp_b200/csrc/block.cuh) factors I - gamma*J
right-looking, one pivot at a time: the sparse head pivots' updates of the
head rows and of the dense rows' head columns from tabulated targets, their
updates of the trailing dense block and the dense pivots' by that block's
addressing (the kernel keeps it in registers), the head L entries of column
k scaled during pivot k + 1; it solves the head rows by levels, the border
entries one row at a time and the dense block's triangles in order, all
from the staged table section.  These tests replay that schedule in numpy on
the tables the library builds (every index the kernel reads comes from
them) for a random matrix with the mechanism's LU pattern, and check the
factors and the solution against dense linear algebra.  They also check the
tables' invariants: the dense block is dense, the staged section matches the
LU structure, the levels respect every dependency.
"""
import struct

import numpy as np
import pytest

FIELDS = ("bytes n n_rxn n_part n_jac n_lu n_coef r0 n_hf n_hb rx_word rx_vptr coef fg_ptr "
          "fg_ent jg_ptr jg_mid jg_w0 jg_w1 jg_row lu_src lu_perm lu_rowptr lu_col lu_diag "
          "dpos ub lk_ptr lk lk_mid tg_ptr hrec hf_ptr hf_rows hb_ptr hb_rows "
          "dep_state atol stage sg_len sg_rowptr sg_diag sg_ub sg_perm sg_hf_ptr sg_hf_rows "
          "sg_hb_ptr sg_hb_rows sg_ndoff sg_ndcol sg_dbase sg_hlk sg_hmid sg_htg").split()
MAX_DENSE = 112


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
    lk = arr("lk", np.uint32, int(t["lk_ptr"][-1]))
    t["lk_pos"], t["lk_row"] = lk & 0xFFFF, lk >> 16
    t["lk_mid"] = arr("lk_mid", np.uint32, r0)
    t["tg_ptr"] = arr("tg_ptr", np.uint32, r0 + 1)
    rec = np.frombuffer(blob, dtype=np.uint64, count=int(t["tg_ptr"][-1]), offset=o["hrec"])
    t["rec_tg"] = (rec & 0xFFFF).astype(np.int64)
    t["rec_l"] = ((rec >> 16) & 0xFFFF).astype(np.int64)
    t["rec_u"] = ((rec >> 32) & 0xFFFF).astype(np.int64)
    t["hf_ptr"] = arr("hf_ptr", np.uint16, o["n_hf"] + 1)
    t["hf_rows"] = arr("hf_rows", np.uint16, int(t["hf_ptr"][-1]))
    t["hb_ptr"] = arr("hb_ptr", np.uint16, o["n_hb"] + 1)
    t["hb_rows"] = arr("hb_rows", np.uint16, int(t["hb_ptr"][-1]))
    sg = arr("stage", np.uint16, o["sg_len"])
    assert o["stage"] % 16 == 0 and o["sg_len"] % 8 == 0
    lens = {"rowptr": n + 1, "diag": n, "ub": r0, "perm": n, "hf_ptr": o["n_hf"] + 1,
            "hf_rows": len(t["hf_rows"]), "hb_ptr": o["n_hb"] + 1, "hb_rows": len(t["hb_rows"]),
            "ndoff": n + 1}
    t["sg"] = {k: sg[o["sg_" + k]:o["sg_" + k] + v] for k, v in lens.items()}
    t["sg"]["ndcol"] = sg[o["sg_ndcol"]:o["sg_ndcol"] + int(t["sg"]["ndoff"][-1])]
    t["sg"]["dbase"] = sg[o["sg_dbase"]:o["sg_dbase"] + n - r0]
    t["sg"]["hlk"] = sg[o["sg_hlk"]:o["sg_hlk"] + r0 + 1]
    t["sg"]["hmid"] = sg[o["sg_hmid"]:o["sg_hmid"] + r0]
    t["sg"]["htg"] = sg[o["sg_htg"]:o["sg_htg"] + r0 + 1]
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
    m = n - r0
    sg = t["sg"]
    diag, rowptr, ub, ndoff, ndcol, dbase = (sg["diag"], sg["rowptr"], sg["ub"], sg["ndoff"],
                                             sg["ndcol"], sg["dbase"])
    # the dense block, as the kernel's registers hold it
    A = np.array([[LU[dbase[i] + r0 + j] for j in range(m)] for i in range(m)])
    dinv = np.zeros(n)
    dense_pos = set()
    for i in range(m):
        dense_pos.update(range(dbase[i] + r0, dbase[i] + r0 + m))
    for k in range(r0):
        dk = 1.0 / LU[diag[k]]
        dinv[k] = dk
        a0, am, a1 = sg["hlk"][k], sg["hmid"][k], sg["hlk"][k + 1]
        u0, uh, u1 = diag[k] + 1, ub[k], rowptr[k + 1]
        nu, nuh = u1 - u0, uh - u0
        q0, q1 = sg["htg"][k], sg["htg"][k + 1]
        assert q1 - q0 == (am - a0) * nu + (a1 - am) * nuh
        assert all(t["lk_row"][a0:am] < r0) and all(t["lk_row"][am:a1] >= r0)
        tg, lp, up = t["rec_tg"][q0:q1], t["rec_l"][q0:q1], t["rec_u"][q0:q1]
        # the records' L entries are column k's, their U entries row k's
        assert set(lp) <= set(t["lk_pos"][a0:a1]) and all((up >= u0) & (up < u1))
        # every target of one pivot is distinct, and none is in the dense block
        assert len(np.unique(tg)) == tg.size and not dense_pos & set(tg.tolist())
        upd = (LU[lp] * dk) * LU[up]
        ld = LU[t["lk_pos"][am:a1]] * dk
        LU[tg] -= upd
        # column k's L entries scaled after its updates
        LU[t["lk_pos"][a0:a1]] *= dk
        # the exchange column and row into the dense block
        lcol = np.zeros(m)
        lcol[t["lk_row"][am:a1] - r0] = ld
        urow = np.zeros(m)
        cols = ndcol[ndoff[k] - rowptr[k] + np.arange(uh, u1)]
        assert all(cols >= r0)
        urow[cols - r0] = LU[uh:u1]
        A -= np.outer(lcol, urow)
    for kk in range(m):
        k = r0 + kk
        dk = 1.0 / A[kk, kk]
        dinv[k] = dk
        A[kk + 1:, kk] *= dk
        A[kk + 1:, kk + 1:] -= np.outer(A[kk + 1:, kk], A[kk, kk + 1:])
    for i in range(m):
        LU[dbase[i] + r0:dbase[i] + r0 + m] = A[i]
    return dinv


def solve(t, LU, dinv, rhs):
    """op_solve's schedule on the staged tables: rhs (dependent order) ->
    M^{-1} rhs."""
    n, r0 = t["n"], t["r0"]
    m = n - r0
    sg = t["sg"]
    perm, rowptr, diag, ub, ndoff, ndcol, dbase = (sg["perm"], sg["rowptr"], sg["diag"],
                                                   sg["ub"], sg["ndoff"], sg["ndcol"],
                                                   sg["dbase"])

    def cols(i, q0, q1):  # columns of positions q0..q1 of row i (non-dense entries)
        return ndcol[ndoff[i] + q0 - rowptr[i]:ndoff[i] + q1 - rowptr[i]]

    z = rhs[perm].copy()
    for lv in range(t["n_hf"]):
        rows = sg["hf_rows"][sg["hf_ptr"][lv]:sg["hf_ptr"][lv + 1]]
        new = {i: z[i] - LU[rowptr[i]:diag[i]] @ z[cols(i, rowptr[i], diag[i])] for i in rows}
        for i, v in new.items():
            z[i] = v
    for i in range(r0, n):
        ne = ndoff[i + 1] - ndoff[i]
        z[i] -= LU[rowptr[i]:rowptr[i] + ne] @ z[ndcol[ndoff[i]:ndoff[i] + ne]]
    npan = (m + 15) // 16  # dense block by panels of 16 columns
    for pp in range(npan):
        c0, c1 = 16 * pp, min(16 * pp + 16, m)
        for kk in range(c0, c1):  # the panel's triangle
            for d in range(kk + 1, c1):
                z[r0 + d] -= LU[dbase[d] + r0 + kk] * z[r0 + kk]
        for d in range(c1, m):  # the rows beyond it
            z[r0 + d] -= LU[dbase[d] + r0 + c0:dbase[d] + r0 + c1] @ z[r0 + c0:r0 + c1]
    for pp in range(npan - 1, -1, -1):
        c0, c1 = 16 * pp, min(16 * pp + 16, m)
        for kk in range(c1 - 1, c0 - 1, -1):
            z[r0 + kk] *= dinv[r0 + kk]
            for d in range(c0, kk):
                z[r0 + d] -= LU[dbase[d] + r0 + kk] * z[r0 + kk]
        for d in range(c0):
            z[r0 + d] -= LU[dbase[d] + r0 + c0:dbase[d] + r0 + c1] @ z[r0 + c0:r0 + c1]
    for i in range(r0):
        z[i] -= LU[ub[i]:rowptr[i + 1]] @ z[cols(i, ub[i], rowptr[i + 1])]
    for lv in range(t["n_hb"]):
        rows = sg["hb_rows"][sg["hb_ptr"][lv]:sg["hb_ptr"][lv + 1]]
        new = {i: (z[i] - LU[diag[i] + 1:ub[i]] @ z[cols(i, diag[i] + 1, ub[i])]) * dinv[i]
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
    assert n - r0 <= MAX_DENSE
    # the staged section is the LU structure
    sg = t["sg"]
    for k in ("rowptr", "diag", "perm"):
        assert np.array_equal(sg[k], t["lu_" + k])
    assert np.array_equal(sg["ub"], t["ub"])
    assert np.array_equal(sg["dbase"], t["dpos"] - r0)
    assert np.array_equal(sg["hlk"], t["lk_ptr"]) and np.array_equal(sg["hmid"], t["lk_mid"])
    assert np.array_equal(sg["htg"], t["tg_ptr"])
    for i in range(n):
        q1 = t["lu_rowptr"][i + 1] if i < r0 else t["dpos"][i - r0]
        assert np.array_equal(sg["ndcol"][sg["ndoff"][i]:sg["ndoff"][i + 1]],
                              t["lu_col"][t["lu_rowptr"][i]:q1])
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


def test_dense_block_beyond_registers_is_refused():
    """A larger random mechanism (250 species, 800 reactions) fills to a
    dense trailing block of more than 112 rows, beyond the 16 x 16 threads x
    7 x 7 entries the factorization holds in registers: the tables refuse it
    with the reason, and such a mechanism runs on the lane-per-cell kernel."""
    import tempfile

    from camp_b200.solver import Solver, SolverError
    from camp_b200.synth import load_synthetic

    with tempfile.TemporaryDirectory() as td:
        mech, _ = load_synthetic(td, 250, 800)
    s = Solver(mech, 4)
    s.build_sparsity_only()
    with pytest.raises(SolverError, match=r"trailing dense block \(\d+ rows\) exceeds"):
        s.block_tables()
