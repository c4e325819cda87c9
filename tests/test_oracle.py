"""The CPU oracle pinned against the reference's own C code.

The golden fixtures (tests/golden/*_ref.npz) hold the reference's sparsity,
rate constants, derivative and Jacobian on seeded cells of cb05cl_ae5 and of
the gas phase of MONARCH mod37 (cb05 plus FIRST_ORDER_LOSS dry deposition,
EMISSION and WET_DEPOSITION), computed by the reference's C sources
(tests/golden/make_golden.py).  The oracle's restatement must reproduce the
sparsity and packed ints bit-exactly and the numbers to 1e-12 relative.
"""
import numpy as np
import pytest

from oracle.oracle import OracleModel, ref_available


@pytest.fixture(scope="module")
def om(cb05):
    return OracleModel(cb05)


@pytest.fixture(scope="module")
def gom(golden):
    mech, ref = golden
    return OracleModel(mech), ref


def test_sparsity_bit_exact(gom):
    om, ref = gom
    cp, ri = om.solver_jac()
    assert np.array_equal(cp, ref["solver_colptr"])
    assert np.array_equal(ri, ref["solver_rowid"])
    rcp, rri = om.rxn_jac()
    assert np.array_equal(rcp, ref["rxn_colptr"])
    assert np.array_equal(rri, ref["rxn_rowid"])
    # DERIV_ID_/JAC_ID_ written back into the packed ints
    assert np.array_equal(om.rxn_int_data(), ref["rxn_int_data"])
    # the fold J_solver += J_rxn * J_params, entry for entry
    assert np.array_equal(om.jac_map(), ref["jac_map"])


def test_sizes(om):
    assert om.n_dep == 74
    assert om.n_jac == 671
    assert om.n_rxn_jac == 716


def _photo_dict(row):
    return {pid + 1: float(row[pid]) for pid in range(row.size)}


def test_rate_constants(gom):
    om, ref = gom
    for c in range(ref["state"].shape[0]):
        re = om.rxn_env_row(ref["env"][c], ref["photo"][c])
        n = ref["rxn_env"].shape[1]  # the aerosol GMD/GSD follow in the oracle's buffer
        np.testing.assert_allclose(re[:n], ref["rxn_env"][c], rtol=1e-15, atol=0)


def test_deriv_and_jacobian(gom):
    om, ref = gom
    for ih, h in enumerate(ref["h"]):
        for c in range(ref["state"].shape[0]):
            re = om.rxn_env_row(ref["env"][c], ref["photo"][c])
            re[:ref["rxn_env"].shape[1]] = ref["rxn_env"][c]
            st = ref["state"][c]
            f, rp, rl = om.deriv(st, re, h)
            np.testing.assert_allclose(rp, ref["r_p"][ih][c], rtol=1e-12, atol=0)
            np.testing.assert_allclose(rl, ref["r_l"][ih][c], rtol=1e-12, atol=0)
            scale = ref["r_p"][ih][c] + ref["r_l"][ih][c]
            assert np.all(np.abs(f - ref["f"][ih][c]) <= 1e-12 * scale)
            j = om.jac(st, re, h)
            jr = ref["jac"][ih][c]
            assert np.all(np.abs(j - jr) <= 1e-12 * np.abs(jr) + 1e-300)


def test_mod37_soa_composition(mod37_soa):
    """The SOA fixture: 4 SIMPOL reactions into one mode, the modal/binned
    representation's 99 aerosol state variables after the 86 gas species,
    and the GMD/GSD columns of its five modes after the reaction rates."""
    from camp_b200.mechanism import reaction_summary

    m = mod37_soa
    assert reaction_summary(m)["by_type"][10] == 4
    rep = m.aero_reps[0]
    assert rep.first_state == 86 and len(rep.unique_names) == 99 == m.n_state_var - 86
    cols = m.rate_columns()
    assert [c[0] for c in cols[-10:]] == ["gmd", "gsd"] * 5
    assert all(c[0] == "rxn" for c in cols[:-10])


def test_mod37_aero_composition(mod37_soa, mod37_aero):
    """The aerosol fixture: the SOA fixture's state plus 35 HL reactions into
    the "clouds and rain" mode, whose water (H2O_aq) is a constant species;
    the reference registers the mode's elements against the gas and aerosol
    species (3803 solver Jacobian entries)."""
    from camp_b200.aerosol import RXN_HL_PHASE_TRANSFER
    from camp_b200.cells import hl_water_indices
    from camp_b200.mechanism import reaction_summary

    m = mod37_aero
    assert reaction_summary(m)["by_type"][RXN_HL_PHASE_TRANSFER] == 35
    assert m.species == mod37_soa.species
    water = hl_water_indices(m)
    assert [m.species[i] for i in water] == ["clouds and rain.cloud and rain water.H2O_aq"]
    assert all(m.var_type[i] == 2 for i in water)
    for r in m.rxns:
        if r.rxn_type == RXN_HL_PHASE_TRANSFER:
            iloc = r.ints[4 + 6] - 1  # PHASE_INT_LOC_(1) of a single instance
            assert r.ints[0] == 1 and r.ints.size == 4 + 13 + 2 * r.ints[iloc + 4]


def test_mod37_gas_composition(mod37):
    """The mod37 gas-phase fixture holds every host-rate type: its rate
    columns are photolysis, dry deposition, emissions and the wet
    deposition, with ids 1..n in mechanism order."""
    from camp_b200.mechanism import reaction_summary

    by_type = reaction_summary(mod37)["by_type"]
    assert by_type[12] == 45 and by_type[13] == 36 and by_type[14] == 1 and by_type[5] == 25
    cols = mod37.rate_rxns()
    assert [mod37.rate_id(i) for i in cols] == list(range(1, len(cols) + 1))
    assert sorted(mod37.rate_ids) == list(range(1, len(cols) + 1))


@pytest.mark.skipif(not ref_available(), reason="reference build absent")
@pytest.mark.parametrize("which", ["cb05", "mod37", "mod37_soa", "mod37_aero"])
def test_live_against_reference_build(request, which):
    """Fresh random states through the reference build and the oracle."""
    from camp_b200.cells import make_cells
    from oracle.oracle import RefModel

    mech = request.getfixturevalue(which)
    om = OracleModel(mech)
    cells = make_cells(mech, 5, 777)
    ref = RefModel(mech, 5)
    for c in range(5):
        ref.set_cell(c, cells.state[c], cells.env[c])
        ref.set_rates(c, cells.photo_rates[c])
        ref.update_env(c)
        re = om.rxn_env_row(cells.env[c], cells.photo_rates[c])
        assert np.array_equal(re[:ref.n_env], ref.rxn_env(c)[:ref.n_env])
        for h in (1e-3, 30.0):
            ref.set_rates(c, cells.photo_rates[c])  # this cell's mode radii
            f1, p1, l1 = ref.deriv(c, h)
            f2, p2, l2 = om.deriv(cells.state[c], re, h)
            np.testing.assert_allclose(p2, p1, rtol=1e-12, atol=0)
            np.testing.assert_allclose(l2, l1, rtol=1e-12, atol=0)
            j1, _ = ref.jac(c, h)
            j2 = om.jac(cells.state[c], re, h)
            assert np.all(np.abs(j2 - j1) <= 1e-12 * np.abs(j1) + 1e-300)


def test_lu_fill_vs_kpp(om):
    """Fill of the Markowitz order against KPP's generated cb05 LU
    (LU_NONZERO = 748, test/chemistry/cb05cl_ae5/cb05cl_ae5_Parameters.f90)."""
    assert om.n_lu <= 748


def test_bdf_consecutive_first_order(cb05):
    """A -> B -> C with first-order rates against the closed form, the check
    the reference's per-reaction unit tests make
    (test/unit_rxn_data/test_rxn_photolysis.F90:288-311)."""
    from camp_b200.mechanism import Mechanism, PackedRxn

    k1, k2 = 0.05, 0.3
    # two photolysis reactions, base rates k1 and k2
    rx = []
    for (a, b) in ((1, 2), (2, 3)):
        ints = np.zeros(3 + (1 + 2) * 2, np.int32)
        ints[0], ints[1], ints[2], ints[3], ints[4] = 1, 1, len(rx) + 1, a, b
        rx.append(PackedRxn(5, ints, np.array([1.0, 1.0]), 2))
    mech = Mechanism("abc", ["A", "B", "C"], np.array([1, 1, 1], np.int32),
                     np.full(3, 1e-12), 1e-10, rx, {1: 0, 2: 1})
    om = OracleModel(mech)
    t = 40.0
    y0 = np.array([[1.0, 0.0, 0.0]])
    nf, status, stats, out = om.solve(y0.copy(), np.array([[298.0, 1e5]]),
                                      np.array([[k1, k2]]), 0.0, t, 1e-10, np.full(3, 1e-14))
    assert nf == 0 and status[0] == 0
    A = np.exp(-k1 * t)
    B = k1 / (k2 - k1) * (np.exp(-k1 * t) - np.exp(-k2 * t))
    C = 1.0 - A - B
    np.testing.assert_allclose(out[0], [A, B, C], rtol=1e-7, atol=1e-12)


@pytest.mark.parametrize("rtype", ["ARRHENIUS", "TROE", "CMAQ_H2O2", "CMAQ_OH_HNO3",
                                   "PHOTOLYSIS"])
def test_bdf_chain_per_reaction_type(tmp_path, rtype):
    """The A -> B -> C chain of every gas-phase type, read from CAMP JSON,
    against the closed form; the GPU counterpart runs the same chains."""
    from conftest import CHAIN_ENV, CHAIN_PHOTO, chain_closed_form, chain_mechanism, chain_rates

    mech, _ = chain_mechanism(tmp_path, rtype)
    k1, k2 = chain_rates(mech, rtype)
    assert 1e-2 < k1 < 1.0 and 1e-2 < k2 < 1.0 and abs(k1 - k2) > 1e-2
    photo = np.array([CHAIN_PHOTO]) if rtype == "PHOTOLYSIS" else np.zeros((1, 0))
    out = []
    for t in (5.0, 60.0):
        nf, status, _, x = OracleModel(mech).solve(np.array([[1.0, 0.0, 0.0]]),
                                                   np.array([CHAIN_ENV]), photo, 0.0, t, 1e-9,
                                                   np.full(3, 1e-14), max_steps=100000)
        assert nf == 0
        out.append(x[0])
    np.testing.assert_allclose(out, chain_closed_form(k1, k2, [5.0, 60.0]), rtol=1e-7,
                               atol=1e-12)


def test_zero_length_step_is_too_close(cb05):
    """CVODE refuses tout == t0 when it must estimate the initial step
    (cvHin: CV_TOO_CLOSE, -27); the cell keeps its input."""
    from camp_b200.cells import make_cells
    from oracle.oracle import OracleModel

    cells = make_cells(cb05, 2, 4)
    nf, status, _, out = OracleModel(cb05).solve(cells.state.copy(), cells.env,
                                                 cells.photo_rates, 5.0, 5.0, 1e-4,
                                                 np.full(cb05.n_state_var, 1e-8))
    assert nf == 2 and list(status) == [-27, -27]
    np.testing.assert_array_equal(out, cells.state)


@pytest.mark.parametrize("kind", ["EMISSION", "FIRST_ORDER_LOSS", "WET_DEPOSITION"])
def test_host_rate_types_known_answer(kind):
    """The reference's unit-test systems for the host-rate types, integrated
    over ten 1-s host steps, against their closed forms."""
    from conftest import species_rate_case

    mech, y0, _, rates, truth = species_rate_case(kind)
    om = OracleModel(mech)
    y = y0[None, :].copy()
    out = []
    for step in range(10):
        nf, status, _, y = om.solve(y, np.array([[298.0, 1.0e5]]), rates[None, :], float(step),
                                    float(step + 1), 1e-10, np.full(y0.size, 1e-14),
                                    max_steps=100000)
        assert nf == 0, status
        out.append(y[0].copy())
    np.testing.assert_allclose(out, truth(np.arange(1, 11)), rtol=1e-7, atol=1e-14)


@pytest.mark.skipif(not ref_available(), reason="reference build absent")
@pytest.mark.parametrize("kind", ["EMISSION", "FIRST_ORDER_LOSS", "WET_DEPOSITION"])
def test_host_rate_updates_match_reference(kind):
    """Rate updates through the reference's own update-data functions (a
    value, then a reset) give the oracle's rate constants, f and J."""
    from conftest import species_rate_case
    from oracle.oracle import RefModel

    mech, y0, first, rates, _ = species_rate_case(kind)
    om = OracleModel(mech)
    ref = RefModel(mech, 1)
    ref.set_cell(0, y0, np.array([298.0, 1.0e5]))
    ref.set_rates(0, first)
    ref.set_rates(0, rates)
    ref.update_env(0)
    re = om.rxn_env([298.0, 1.0e5], {i + 1: float(r) for i, r in enumerate(rates)})
    assert np.array_equal(re, ref.rxn_env(0))
    assert np.array_equal(om.rxn_int_data(), ref.rxn_int_data())
    f1, p1, l1 = ref.deriv(0, 1.0)
    f2, p2, l2 = om.deriv(y0, re, 1.0)
    np.testing.assert_allclose(p2, p1, rtol=1e-15, atol=0)
    np.testing.assert_allclose(l2, l1, rtol=1e-15, atol=0)
    j1, _ = ref.jac(0, 1.0)
    np.testing.assert_allclose(om.jac(y0, re, 1.0), j1, rtol=1e-15, atol=0)


def test_hl_closed_form(tmp_path):
    """HL partitioning into one aqueous mode (constant water) relaxes to the
    Henry's law equilibrium at the rate the reference's rate constants give,
    G + K G_aq conserved."""
    from conftest import HL_ENV, hl_case

    mech, y0, cols, truth = hl_case(tmp_path)
    om = OracleModel(mech)
    abs_tol = np.array([1e-14, 1e-20, 1e-14])
    out = []
    for t in (5.0, 20.0, 60.0):
        nf, status, _, y = om.solve(y0[None, :].copy(), np.array([HL_ENV]), cols[None, :], 0.0,
                                    t, 1e-10, abs_tol, max_steps=100000)
        assert nf == 0, status
        out.append(y[0, :2])
    np.testing.assert_allclose(out, truth([5.0, 20.0, 60.0]), rtol=1e-7, atol=1e-18)


def test_aqueous_equilibrium_closed_form(tmp_path):
    """A <-> B in one aqueous mode (constant water and ion pair) relaxes to
    the equilibrium ratio k_r gamma / k_f at the rate k_f + k_r gamma."""
    from conftest import AQ_ENV, aq_case

    mech, y0, cols, truth = aq_case(tmp_path)
    om = OracleModel(mech)
    abs_tol = np.array([1e-14, 1e-20, 1e-20, 1e-14])
    out = []
    for t in (5.0, 20.0, 60.0):
        nf, status, _, y = om.solve(y0[None, :].copy(), np.array([AQ_ENV]), cols[None, :], 0.0,
                                    t, 1e-10, abs_tol, max_steps=100000)
        assert nf == 0, status
        out.append(y[0, 1:3])
    np.testing.assert_allclose(out, truth([5.0, 20.0, 60.0]), rtol=1e-7, atol=1e-20)
