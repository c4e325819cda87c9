"""The seeded synthetic mechanism generator (the large-mechanism workload):
reaction mix, parameter ranges, determinism, and that the packer and the
sparsity builder accept it."""
import json

import numpy as np


def test_mix_and_ranges():
    from camp_b200.synth import synthetic_json

    species, mech, photo_base = synthetic_json(200, 600, 1234)
    names = [s["name"] for s in species["camp-data"]]
    assert len(names) == 200 and len(set(names)) == 200
    rxns = mech["camp-data"][0]["reactions"]
    assert len(rxns) == 600
    kinds = {"bi": 0, "first": 0, "troe": 0, "photo": 0}
    for r in rxns:
        nreact = sum(p.get("qty", 1) for p in r["reactants"].values())
        assert 1 <= len(r["products"]) <= 4
        if r["type"] == "ARRHENIUS" and nreact == 2:
            kinds["bi"] += 1
            assert 1e-14 <= r["A"] <= 1e-10 and -3000.0 <= r["C"] <= 0.0
        elif r["type"] == "ARRHENIUS":
            kinds["first"] += 1
            assert nreact == 1 and 1e-6 <= r["A"] <= 1e2
        elif r["type"] == "TROE":
            kinds["troe"] += 1
            assert nreact == 2 and 1e-33 <= r["k0_A"] <= 1e-28 and 1e-12 <= r["kinf_A"] <= 1e-10
            assert r["Fc"] == 0.6 and r["N"] == 1.0
        else:
            assert r["type"] == "PHOTOLYSIS" and nreact == 1
            kinds["photo"] += 1
    assert kinds == {"bi": 300, "first": 180, "troe": 60, "photo": 60}
    assert photo_base.size == 60 and np.all((photo_base >= 1e-6) & (photo_base <= 1e-2))


def test_deterministic_and_packs(tmp_path):
    from camp_b200.solver import Solver
    from camp_b200.synth import load_synthetic, synthetic_json

    a = json.dumps(synthetic_json(200, 600, 99)[1])
    b = json.dumps(synthetic_json(200, 600, 99)[1])
    assert a == b
    mech, base = load_synthetic(str(tmp_path), 40, 100, 7)
    assert mech.n_state_var == 40 and mech.n_rxn == 100
    s = Solver(mech, 4)
    s.build_sparsity_only()
    assert s.lib.camp_b200_n_jac_elem(s._h) > 0
    assert s.n_lu() >= s.lib.camp_b200_n_jac_elem(s._h)
