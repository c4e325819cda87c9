import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# the reference source tree (read only by the CPU tests that re-pack its
# JSON input or compile its C sources; they skip when it is absent)
REF_ROOT = os.environ.get("CAMP_REFERENCE_ROOT", "/root/reference")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cb05():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "cb05cl_ae5.mech.json"))


@pytest.fixture(scope="session")
def cb05_ref():
    return dict(np.load(os.path.join(GOLDEN, "cb05cl_ae5_ref.npz")))


# golden fixtures made by tests/golden/make_golden.py from the reference's C
# code: cb05cl_ae5, the gas phase of MONARCH mod37 (cb05 with dry
# deposition, emissions and the wet deposition of one aqueous phase), and
# mod37 with its SOA scheme (SIMPOL partitioning into the modal/binned
# aerosol representation), mod37 with SOA, cloud/rain HL and aqueous
# equilibria, and the shipped MONARCH mod37 test configuration
# (test/monarch/config_monarch_mod37.json), whose aerosol water and ion-pair
# activity coefficients the ZSR and PD-FiTE sub-models compute
GOLDEN_MECHS = ("cb05cl_ae5", "monarch_mod37_gas", "monarch_mod37_soa", "monarch_mod37_aero",
                "monarch_mod37_shipped")


@pytest.fixture(scope="session")
def mod37():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "monarch_mod37_gas.mech.json"))


@pytest.fixture(scope="session")
def mod37_soa():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "monarch_mod37_soa.mech.json"))


@pytest.fixture(scope="session")
def mod37_aero():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "monarch_mod37_aero.mech.json"))


@pytest.fixture(scope="session")
def mod37_shipped():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "monarch_mod37_shipped.mech.json"))


@pytest.fixture(scope="session", params=GOLDEN_MECHS)
def golden(request):
    """(mechanism, reference outputs) of each golden fixture."""
    from camp_b200.mechanism import Mechanism

    tag = request.param
    return (Mechanism.load(os.path.join(GOLDEN, f"{tag}.mech.json")),
            dict(np.load(os.path.join(GOLDEN, f"{tag}_ref.npz"))))


@pytest.fixture(scope="session")
def lib():
    from camp_b200 import build, _lib

    build.build()
    return _lib.load()


# A -> B -> C with two first-order reactions of one type, the analytic check
# of the reference's per-reaction tests (test/unit_rxn_data/test_rxn_troe.F90,
# test_rxn_CMAQ_H2O2.F90, test_rxn_CMAQ_OH_HNO3.F90, test_rxn_photolysis.F90,
# test/unit_tests/rxns/unit_test_rxn_arrhenius.F90).  Parameters are chosen
# so that both rate constants lie in 1e-2..1 s-1 at CHAIN_ENV.
CHAIN_ENV = (280.0, 9.0e4)  # T (K), P (Pa)
CHAIN_PHOTO = (0.03, 0.2)   # photolysis base rates of the two reactions
CHAIN_CASES = {
    "ARRHENIUS": ({"A": 0.05, "C": -100.0}, {"A": 0.4, "B": 1.5, "D": 290.0}),
    "TROE": ({"k0_A": 1e-21, "kinf_A": 1e-1},
             {"k0_A": 4e-21, "k0_B": -1.0, "kinf_A": 2.0, "Fc": 0.5}),
    "CMAQ_H2O2": ({"k1_A": 0.02, "k2_A": 1e-21},
                  {"k1_A": 0.1, "k1_C": -50.0, "k2_A": 2e-21, "k2_C": 100.0}),
    "CMAQ_OH_HNO3": ({"k0_A": 0.03, "k2_A": 1e-2, "k3_A": 1e-21},
                     {"k0_A": 0.08, "k0_C": 20.0, "k2_A": 0.5, "k3_A": 3e-21}),
    "PHOTOLYSIS": ({"scaling factor": 1.0}, {"scaling factor": 2.0}),
}


def chain_mechanism(tmp_dir, rtype):
    """The A -> B -> C mechanism of type rtype, written as CAMP JSON input
    files under tmp_dir and loaded; returns (mechanism, json files)."""
    import json

    from camp_b200.mechanism import load_mechanism

    p1, p2 = CHAIN_CASES[rtype]
    species = {"camp-data": [{"name": n, "type": "CHEM_SPEC"} for n in "ABC"]}
    rxns = [dict(type=rtype, reactants={"A": {}}, products={"B": {}}, **p1),
            dict(type=rtype, reactants={"B": {}}, products={"C": {}}, **p2)]
    mech = {"camp-data": [{"name": "abc", "type": "MECHANISM", "reactions": rxns}]}
    files = [os.path.join(str(tmp_dir), "species.json"),
             os.path.join(str(tmp_dir), "mechanism.json")]
    for f, obj in zip(files, (species, mech)):
        with open(f, "w") as fh:
            json.dump(obj, fh)
    return load_mechanism(files), files


def chain_rates(mech, rtype):
    """k1, k2 of the chain from the oracle's rate-constant code."""
    from oracle.oracle import OracleModel

    photo = {1: CHAIN_PHOTO[0], 2: CHAIN_PHOTO[1]} if rtype == "PHOTOLYSIS" else None
    re = OracleModel(mech).rxn_env(CHAIN_ENV, photo)
    stride = 2 if rtype == "PHOTOLYSIS" else 1  # env parameters per reaction
    return float(re[0]), float(re[stride])


def chain_closed_form(k1, k2, times):
    """[A, B, C] at each time from A0 = 1, B0 = C0 = 0."""
    times = np.asarray(times, np.float64)
    a = np.exp(-k1 * times)
    b = k1 / (k2 - k1) * (np.exp(-k1 * times) - np.exp(-k2 * times))
    return np.stack([a, b, 1.0 - a - b], axis=1)


def species_rate_case(kind):
    """The systems of the reference's EMISSION, FIRST_ORDER_LOSS and
    WET_DEPOSITION unit tests (test/unit_rxn_data/test_rxn_emission.F90:
    112-121,245-286, test_rxn_first_order_loss.F90:112-121,245-286,
    test_rxn_wet_deposition.F90:119-128,314-367), packed directly.

    Returns (mechanism, y0, first_rates, rates, truth): the second reaction's
    base rate is first set to first_rates and then reset to rates, as those
    tests do; truth(t) is the closed form at times t, [len(t), n_state]."""
    from camp_b200.mechanism import (RXN_EMISSION, RXN_FIRST_ORDER_LOSS, Mechanism,
                                     assign_rate_ids, pack_species_rate, pack_wet_deposition)

    if kind in ("EMISSION", "FIRST_ORDER_LOSS"):
        rtype = RXN_EMISSION if kind == "EMISSION" else RXN_FIRST_ORDER_LOSS
        rxns = [pack_species_rate(rtype, 1, 1.0, "rxn A"), pack_species_rate(rtype, 2, 12.3, "rxn B")]
        names, y0 = ["A", "B"], np.array([1.0, 1.0])
        first = np.array([0.954, 42.11 if kind == "EMISSION" else 432.3])
        rates = np.array([0.954, 1.0e-2])
        k = np.array([0.954, 1.0e-2 * 12.3])
        if kind == "EMISSION":
            def truth(t):
                return y0[None, :] + k[None, :] * np.asarray(t, float)[:, None]
        else:
            def truth(t):
                return y0[None, :] * np.exp(-k[None, :] * np.asarray(t, float)[:, None])
    else:
        # two instances (1, 2) of phases rain (A, B) and cloud (B, C)
        names = ["1.rain.A", "1.rain.B", "1.cloud.B", "1.cloud.C",
                 "2.rain.A", "2.rain.B", "2.cloud.B", "2.cloud.C"]
        y0 = np.array([1.0, 2.2, 1.7, 2.4, 2.5, 0.7, 1.6, 1.9])
        rxns = [pack_wet_deposition([1, 2, 5, 6], 1.0, "rxn rain"),
                pack_wet_deposition([3, 4, 7, 8], 12.3, "rxn cloud")]
        first = np.array([0.954, 43912.5])
        rates = np.array([0.954, 1.0e-2])
        krow = np.array([0.954, 0.954, 0.123, 0.123, 0.954, 0.954, 0.123, 0.123])

        def truth(t):
            return y0[None, :] * np.exp(-krow[None, :] * np.asarray(t, float)[:, None])
    ids = assign_rate_ids(rxns)
    n = len(names)
    mech = Mechanism(kind.lower(), names, np.ones(n, np.int32), np.full(n, 1.0e-12), 1.0e-10,
                     rxns, ids)
    return mech, y0, first, rates, truth


# One HL_PHASE_TRANSFER reaction of gas G into "G_aq" of a single aqueous
# mode whose water is a constant species: with the modal/binned
# representation's number concentration of 1 the system is linear,
#   dG/dt = k_c G_aq / (K_H W) - k_c G,   dG_aq/dt = -(dG/dt) / K,
# G + K G_aq is conserved and both relax at lambda = k_c (1 + 1 / (K_H W K)).
HL_ENV = (272.5, 101253.3)              # T (K), P (Pa)
HL_MODE = (2.0e-5, 1.5)                 # GMD (m), GSD
HL_WATER = 1.0e-6                       # kg m-3
HL_LAMBDA = 0.1                         # s-1, sets the Henry's law constant
HL_Y0 = (0.5, 1.0e-6)                   # G (ppm), G_aq (kg m-3)
HL_D, HL_MW, HL_C = 1.5e-5, 0.048, 2300.0


def hl_rates(T, P, gmd, gsd, hlc):
    """k_c, K_H and the kg m-3 -> ppm factor K of the reference's HL
    (src/rxns/rxn_HL_phase_transfer.c:209-247, src/util.h:50-135): mass
    accommodation 0.1 (no N*), the mode's effective radius."""
    R, PI = 8.314472, np.pi
    alpha = 0.1
    mfp = 3.0 * HL_D / np.sqrt(8.0 * R * T / (PI * HL_MW))
    r = gmd / 2.0 * np.exp(5.0 * np.log(gsd) ** 2 / 2.0)
    kn = mfp / r
    fs = 0.75 * alpha * (1.0 + kn) / (kn * kn + (1.0 + 0.283 * alpha) * kn + 0.75 * alpha)
    kc = 4.0 * PI * r * HL_D * fs
    kh = hlc * P * 1.0e-6 * np.exp(HL_C * (1.0 / T - 1.0 / 298.0)) * HL_MW
    K = R / HL_MW * 1.0e6 * T / P
    return kc, kh, K


def hl_case(tmp_dir):
    """(mechanism, y0, host columns (GMD, GSD), closed form G, G_aq at t)."""
    import json

    from camp_b200.aerosol import load_aerosol_mechanism

    T, P = HL_ENV
    kc, kh1, K = hl_rates(T, P, *HL_MODE, 1.0)
    # the Henry's law constant that gives the chosen relaxation rate
    hlc = kc / ((HL_LAMBDA - kc) * HL_WATER * K) / kh1
    doc = {"camp-data": [
        {"name": "G", "type": "CHEM_SPEC", "molecular weight [kg mol-1]": HL_MW,
         "diffusion coeff [m2 s-1]": HL_D, "HLC(298K) [M Pa-1]": hlc,
         "HLC exp factor [K]": HL_C, "absolute integration tolerance": 1e-14},
        {"name": "G_aq", "type": "CHEM_SPEC", "phase": "AEROSOL",
         "molecular weight [kg mol-1]": HL_MW, "density [kg m-3]": 1000.0,
         "absolute integration tolerance": 1e-20},
        {"name": "H2O_aq", "type": "CHEM_SPEC", "phase": "AEROSOL", "tracer type": "CONSTANT",
         "molecular weight [kg mol-1]": 0.01801528, "density [kg m-3]": 1000.0},
        {"name": "aqueous", "type": "AERO_PHASE", "species": ["G_aq", "H2O_aq"]},
        {"name": "rep", "type": "AERO_REP_MODAL_BINNED_MASS", "modes/bins": {
            "the mode": {"type": "MODAL", "phases": ["aqueous"], "shape": "LOG_NORMAL",
                         "geometric mean diameter [m]": HL_MODE[0],
                         "geometric standard deviation": HL_MODE[1]}}},
        {"name": "hl", "type": "MECHANISM", "reactions": [
            {"type": "HL_PHASE_TRANSFER", "gas-phase species": "G",
             "aerosol phase": "aqueous", "aerosol-phase species": "G_aq",
             "aerosol-phase water": "H2O_aq"}]},
    ]}
    path = os.path.join(str(tmp_dir), "hl.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    mech = load_aerosol_mechanism([path], name="hl")
    assert mech.species == ["G", "the mode.aqueous.G_aq", "the mode.aqueous.H2O_aq"]
    y0 = np.array([HL_Y0[0], HL_Y0[1], HL_WATER])
    cols = np.array(HL_MODE)
    kc, kh, K = hl_rates(T, P, *HL_MODE, hlc)
    lam = kc * (1.0 + 1.0 / (kh * HL_WATER * K))
    assert abs(lam - HL_LAMBDA) < 1e-12 * HL_LAMBDA
    total = HL_Y0[0] + K * HL_Y0[1]
    g_eq = total / (1.0 + K * kh * HL_WATER)

    def truth(times):
        g = g_eq + (HL_Y0[0] - g_eq) * np.exp(-lam * np.asarray(times, np.float64))
        return np.stack([g, (total - g) / K], axis=-1)

    return mech, y0, cols, truth


# One AQUEOUS_EQUILIBRIUM reaction A <-> B in one aqueous mode, water and the
# ion pair's activity coefficient constant species: in molar amounts
# a = A m_A, b = B m_B (m = 1e3 / MW) it is linear,
#   da/dt = -k_f a + k_r g b,  db/dt = -da/dt,
# relaxing at k_f + k_r g to a / b = k_r g / k_f.
AQ_ENV = (285.0, 9.5e4)
AQ_PRM = {"A": 2.0, "C": 300.0, "k_reverse": 0.04}
AQ_GAMMA = 1.5
AQ_MW = (0.06, 0.09)                    # A, B (kg mol-1)
AQ_Y0 = (2.0e-9, 5.0e-10)               # A, B (kg m-3)


def aq_case(tmp_dir):
    """(mechanism, y0, host columns (GMD, GSD), closed form A, B at t)."""
    import json

    from camp_b200.aerosol import load_aerosol_mechanism

    doc = {"camp-data": [
        {"name": "AQA", "type": "CHEM_SPEC", "phase": "AEROSOL",
         "molecular weight [kg mol-1]": AQ_MW[0], "density [kg m-3]": 1000.0,
         "absolute integration tolerance": 1e-20},
        {"name": "AQB", "type": "CHEM_SPEC", "phase": "AEROSOL",
         "molecular weight [kg mol-1]": AQ_MW[1], "density [kg m-3]": 1000.0,
         "absolute integration tolerance": 1e-20},
        {"name": "H2O_aq", "type": "CHEM_SPEC", "phase": "AEROSOL", "tracer type": "CONSTANT",
         "molecular weight [kg mol-1]": 0.01801528, "density [kg m-3]": 1000.0},
        {"name": "A-B", "type": "CHEM_SPEC", "tracer type": "ION_PAIR"},
        {"name": "aqueous", "type": "AERO_PHASE", "species": ["H2O_aq", "AQA", "AQB", "A-B"]},
        {"name": "rep", "type": "AERO_REP_MODAL_BINNED_MASS", "modes/bins": {
            "the mode": {"type": "MODAL", "phases": ["aqueous"], "shape": "LOG_NORMAL",
                         "geometric mean diameter [m]": 2.0e-7,
                         "geometric standard deviation": 1.6}}},
        {"name": "aq", "type": "MECHANISM", "reactions": [
            dict({"type": "AQUEOUS_EQUILIBRIUM", "aerosol phase": "aqueous",
                  "aerosol-phase water": "H2O_aq", "ion pair": "A-B",
                  "reactants": {"AQA": {}}, "products": {"AQB": {}}}, **AQ_PRM)]},
    ]}
    path = os.path.join(str(tmp_dir), "aq.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    mech = load_aerosol_mechanism([path], name="aq")
    names = ["the mode.aqueous." + n for n in ("H2O_aq", "AQA", "AQB", "A-B")]
    assert mech.species == names
    y0 = np.array([1.0e-6, AQ_Y0[0], AQ_Y0[1], AQ_GAMMA])
    T = AQ_ENV[0]
    kf = AQ_PRM["A"] * np.exp(AQ_PRM["C"] * (1.0 / T - 1.0 / 298.0)) * AQ_PRM["k_reverse"]
    kr = AQ_PRM["k_reverse"] * AQ_GAMMA
    ma, mb = 1.0e3 / AQ_MW[0], 1.0e3 / AQ_MW[1]
    a0, b0 = AQ_Y0[0] * ma, AQ_Y0[1] * mb
    lam = kf + kr
    a_eq = (a0 + b0) * kr / lam

    def truth(times):
        a = a_eq + (a0 - a_eq) * np.exp(-lam * np.asarray(times, np.float64))
        return np.stack([a / ma, (a0 + b0 - a) / mb], axis=-1)

    return mech, y0, np.array([2.0e-7, 1.6]), truth
