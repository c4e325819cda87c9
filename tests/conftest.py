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
