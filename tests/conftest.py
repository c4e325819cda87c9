import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_ROOT = "/root/reference"
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
# aerosol representation)
GOLDEN_MECHS = ("cb05cl_ae5", "monarch_mod37_gas", "monarch_mod37_soa")


@pytest.fixture(scope="session")
def mod37():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "monarch_mod37_gas.mech.json"))


@pytest.fixture(scope="session")
def mod37_soa():
    from camp_b200.mechanism import Mechanism

    return Mechanism.load(os.path.join(GOLDEN, "monarch_mod37_soa.mech.json"))


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
