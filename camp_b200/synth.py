"""Seeded synthetic gas-phase mechanism for the large-mechanism workload.

The workload is 200 species and 600 reactions: 50 % bimolecular Arrhenius
(A log-uniform 1e-14..1e-10 cm3 molec-1 s-1, C = -Ea/R with Ea/R uniform in
0..3000 K), 30 % first-order Arrhenius (A log-uniform 1e-6..1e2 s-1), 10 %
Troe fall-off (k0 log-uniform 1e-33..1e-28, kinf log-uniform 1e-12..1e-10,
Fc 0.6, N 1) and 10 % photolysis (base J log-uniform 1e-6..1e-2 s-1, scaled
per cell by a factor in [0, 1]).  Reactant counts follow the rate law (one for
first-order and photolysis, two for bimolecular and Troe, the third body of
Troe being implicit as in CAMP); each reaction has 1-4 distinct products with
unit yield.  Reactants and products are drawn uniformly from the species.

The mechanism is written as CAMP JSON input files, so the same packer
(:func:`camp_b200.mechanism.load_mechanism`), oracle and solver handle it like
a shipped mechanism.  The generator is numpy ``PCG64`` with an explicit seed.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .mechanism import Mechanism, load_mechanism

SYNTH_SEED = 20241204


def synthetic_json(n_species: int = 200, n_rxn: int = 600, seed: int = SYNTH_SEED):
    """Returns (species_json, mechanism_json, photo_base) for the workload.

    photo_base[j] is the base rate of the j-th photolysis reaction in
    mechanism order (photolysis id j + 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    names = [f"S{i:03d}" for i in range(n_species)]
    n_bi = int(round(0.5 * n_rxn))
    n_first = int(round(0.3 * n_rxn))
    n_troe = int(round(0.1 * n_rxn))
    n_photo = n_rxn - n_bi - n_first - n_troe
    kinds = ["bi"] * n_bi + ["first"] * n_first + ["troe"] * n_troe + ["photo"] * n_photo
    kinds = [kinds[i] for i in rng.permutation(len(kinds))]

    def loguniform(lo, hi):
        return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))

    def reactants(k):
        out: dict[str, dict] = {}
        for s in rng.integers(0, n_species, k):
            nm = names[int(s)]
            out[nm] = {"qty": out[nm]["qty"] + 1} if nm in out else {"qty": 1}
        return {nm: ({} if p["qty"] == 1 else p) for nm, p in out.items()}

    def products():
        k = int(rng.integers(1, 5))
        pick = rng.choice(n_species, size=k, replace=False)
        return {names[int(s)]: {} for s in pick}

    rxns, photo_base = [], []
    for i, kind in enumerate(kinds):
        r = {"rxn id": f"SYN{i:04d}"}
        if kind == "bi":
            r.update(type="ARRHENIUS", reactants=reactants(2), products=products(),
                     A=loguniform(1e-14, 1e-10), C=-float(rng.uniform(0.0, 3000.0)))
        elif kind == "first":
            r.update(type="ARRHENIUS", reactants=reactants(1), products=products(),
                     A=loguniform(1e-6, 1e2))
        elif kind == "troe":
            r.update(type="TROE", reactants=reactants(2), products=products(),
                     k0_A=loguniform(1e-33, 1e-28), kinf_A=loguniform(1e-12, 1e-10),
                     Fc=0.6, N=1.0)
        else:
            r.update(type="PHOTOLYSIS", reactants=reactants(1), products=products())
            photo_base.append(loguniform(1e-6, 1e-2))
        rxns.append(r)
    species = {"camp-data": [{"name": nm, "type": "CHEM_SPEC"} for nm in names]}
    mech = {"camp-data": [{"name": "synthetic", "type": "MECHANISM", "reactions": rxns}]}
    return species, mech, np.asarray(photo_base, dtype=np.float64)


def write_synthetic(directory: str, n_species: int = 200, n_rxn: int = 600,
                    seed: int = SYNTH_SEED) -> tuple[list[str], np.ndarray]:
    """Writes the JSON files into ``directory``; returns (paths, photo_base)."""
    species, mech, photo_base = synthetic_json(n_species, n_rxn, seed)
    os.makedirs(directory, exist_ok=True)
    sp = os.path.join(directory, "synthetic_species.json")
    mp = os.path.join(directory, "synthetic_mechanism.json")
    with open(sp, "w") as fh:
        json.dump(species, fh)
    with open(mp, "w") as fh:
        json.dump(mech, fh)
    return [sp, mp], photo_base


def load_synthetic(directory: str, n_species: int = 200, n_rxn: int = 600,
                   seed: int = SYNTH_SEED) -> tuple[Mechanism, np.ndarray]:
    """Generates, writes and packs the synthetic mechanism."""
    paths, photo_base = write_synthetic(directory, n_species, n_rxn, seed)
    return load_mechanism(paths, "synthetic"), photo_base
