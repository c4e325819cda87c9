"""Seeded synthetic cell states for the benchmark and parity workloads.

Per-cell inputs follow the documented workload distributions:

* temperature uniform 260-310 K, pressure uniform 5e4-1.013e5 Pa;
* photolysis base rates = a fixed base set x one per-cell factor uniform in
  [0, 1] (the day/night stiffness spread).  The cb05cl_ae5 base set is the
  reference cb05 test's 1e-4 s^-1 for every photolysis reaction except jo2,
  which is 0 (``test/chemistry/cb05cl_ae5/test_cb05cl_ae5.F90:349-362``);
* the other host-set rates (emission in ppm s^-1, first-order loss and wet
  deposition in s^-1) = a fixed base set x a second per-cell factor uniform
  in [0.5, 1.5], drawn after everything else so that mechanisms without such
  reactions keep their streams;
* aerosol (mechanisms with a modal/binned representation, drawn last): per
  mode a geometric mean diameter log-uniform in 20-500 nm (the GSD is the
  representation's, 2.0 where it sets none) and a number concentration log-uniform in 1e7-1e10 m^-3,
  per bin a number concentration log-uniform in 1e3-1e6 m^-3 (bins reach
  15 um); the mode's or bin's volume is split over its mass species with
  uniform random weights into kg m^-3; activity coefficients are 1;
* initial concentrations of variable species log-uniform in
  [conc_lo, conc_hi] ppm; constant species keep their "init conc" value.

The generator is numpy ``PCG64`` with an explicit seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mechanism import (CHEM_SPEC_VARIABLE, RXN_EMISSION, RXN_FIRST_ORDER_LOSS, RXN_PHOTOLYSIS,
                        RXN_WET_DEPOSITION, Mechanism)

# base rates of the non-photolysis host-rate types: a surface emission
# tendency (ppm s^-1) and dry / wet deposition rate constants (s^-1)
EMISSION_BASE = 1.0e-8
FIRST_ORDER_LOSS_BASE = 2.0e-5
WET_DEPOSITION_BASE = 1.0e-4
# GSD of a mode whose representation input sets none (the MONARCH test
# configuration leaves GMD / GSD to the host's update data; the shipped mod37
# modes use 2.0-2.24)
DEFAULT_GSD = 2.0


@dataclass
class CellBatch:
    state: np.ndarray  # [n_cells, n_state_var] float64
    env: np.ndarray  # [n_cells, 2] (T K, P Pa)
    photo_rates: np.ndarray  # [n_cells, n_photo] host-set base rates, one column per
    #                          host-rate reaction (Mechanism.rate_rxns order)
    seed: int

    @property
    def n_cells(self) -> int:
        return self.state.shape[0]

    def slice(self, a: int, b: int) -> "CellBatch":
        return CellBatch(self.state[a:b].copy(), self.env[a:b].copy(), self.photo_rates[a:b].copy(), self.seed)


def photo_base_rates(mech: Mechanism, base: float = 1.0e-4, zero_labels=("jo2",)) -> np.ndarray:
    """Base rate per host-rate column: ``base`` for photolysis (0 for the
    listed reactions), the module's emission / deposition bases otherwise."""
    other = {RXN_EMISSION: EMISSION_BASE, RXN_FIRST_ORDER_LOSS: FIRST_ORDER_LOSS_BASE,
             RXN_WET_DEPOSITION: WET_DEPOSITION_BASE}
    cols = mech.rate_columns()
    out = np.zeros(len(cols), dtype=np.float64)
    for j, col in enumerate(cols):
        if col[0] != "rxn":
            sec = mech.aero_reps[col[1]].sections[col[2]]
            out[j] = sec.gmd if col[0] == "gmd" else sec.gsd
            continue
        r = mech.rxns[col[1]]
        if r.rxn_type == RXN_PHOTOLYSIS:
            out[j] = 0.0 if r.label in zero_labels else base
        else:
            out[j] = other[r.rxn_type]
    return out


def photolysis_columns(mech: Mechanism) -> np.ndarray:
    """Mask of the host-set columns that are photolysis reactions."""
    return np.asarray([c[0] == "rxn" and mech.rxns[c[1]].rxn_type == RXN_PHOTOLYSIS
                       for c in mech.rate_columns()], dtype=bool)


def hl_water_indices(mech: Mechanism) -> set[int]:
    """State indices of the aerosol-phase water that HL partitioning divides
    by (AERO_WATER_ of every instance,
    src/rxns/rxn_HL_phase_transfer.c:49-57)."""
    from .aerosol import RXN_HL_PHASE_TRANSFER

    out = set()
    for r in mech.rxns:
        if r.rxn_type != RXN_HL_PHASE_TRANSFER:
            continue
        n = int(r.ints[0])
        for x in range(n):
            iloc = int(r.ints[4 + 6 * n + x]) - 1
            out.add(int(r.ints[iloc + 1]) - 1)
    return out


def zsr_water_indices(mech: Mechanism) -> set[int]:
    """State indices of the aerosol-phase water that a ZSR sub-model
    computes (PHASE_ID_ of every instance,
    src/sub_models/sub_model_ZSR_aerosol_water.c:37-40)."""
    from .mechanism import SUB_MODEL_ZSR_AEROSOL_WATER

    out = set()
    for sm in mech.sub_models:
        if sm.sub_type == SUB_MODEL_ZSR_AEROSOL_WATER:
            n_phase = int(sm.ints[0])
            out.update(int(sm.ints[5 + p]) - 1 for p in range(n_phase))
    return out


def _aerosol_cells(mech: Mechanism, rng, state: np.ndarray, photo: np.ndarray) -> None:
    """Per-cell aerosol state and mode GMD/GSD columns (module docstring)."""
    from .aerosol import MODAL

    n_cells = state.shape[0]
    cols = mech.rate_columns()
    col_of = {c: j for j, c in enumerate(cols)}
    # cloud-like input only where HL partitions into a water that no
    # sub-model computes
    water = hl_water_indices(mech) - zsr_water_indices(mech)
    for ri, rep in enumerate(mech.aero_reps):
        inst = 0
        for si, sec in enumerate(rep.sections):
            nb = sec.n_bins

            def first_of(j: int) -> int:  # first state index of instance j
                return rep.first_state + sum(len(mech.aero_phases[q].species)
                                             for q in rep.instances[:j])

            cloud = any(first_of(j) + k in water
                        for j in range(inst, inst + len(sec.phases) * nb)
                        for k in range(len(mech.aero_phases[rep.instances[j]].species)))
            if cloud:
                # liquid water around the representation's own mode size
                if sec.kind == MODAL:
                    gmd = sec.gmd * np.exp(rng.uniform(np.log(0.5), np.log(2.0), n_cells))
                    photo[:, col_of[("gmd", ri, si)]] = gmd
                    photo[:, col_of[("gsd", ri, si)]] = np.full(n_cells, sec.gsd)
                lwc = np.exp(rng.uniform(np.log(1e-5), np.log(1e-3), (n_cells, nb)))
                for pi in sec.phases:
                    ph = mech.aero_phases[pi]
                    w = rng.uniform(0.0, 1.0, (n_cells, nb, len(ph.species)))
                    for b in range(nb):
                        first = first_of(inst)
                        dis = [k for k, t in enumerate(ph.types)
                               if t in (1, 2, 3) and first + k not in water]
                        wsum = w[:, b, dis].sum(axis=1) if dis else np.ones(n_cells)
                        share = lwc[:, b] / len(sec.phases)
                        for k, t in enumerate(ph.types):
                            if first + k in water:
                                state[:, first + k] = share
                            elif t in (1, 2, 3):
                                state[:, first + k] = share * 1.0e-3 * w[:, b, k] / wsum
                            else:
                                state[:, first + k] = 1.0
                        inst += 1
                continue
            if sec.kind == MODAL:
                gmd = np.exp(rng.uniform(np.log(20e-9), np.log(500e-9), n_cells))
                gsd = np.full(n_cells, sec.gsd if sec.gsd > 0.0 else DEFAULT_GSD)
                photo[:, col_of[("gmd", ri, si)]] = gmd
                photo[:, col_of[("gsd", ri, si)]] = gsd
                number = np.exp(rng.uniform(np.log(1e7), np.log(1e10), (n_cells, 1)))
                vol = number * (np.pi / 6.0 * gmd[:, None] ** 3 *
                                np.exp(4.5 * np.log(gsd[:, None]) ** 2))
            else:
                dp = rep.floats[rep.ints[4 + len(rep.sections) + si] - 1 + 3 * np.arange(nb)]
                number = np.exp(rng.uniform(np.log(1e3), np.log(1e6), (n_cells, nb)))
                vol = number * (4.0 / 3.0 * np.pi * (dp[None, :] / 2.0) ** 3)
            # instances of this section, Fortran order (phase, bin)
            for pi in sec.phases:
                ph = mech.aero_phases[pi]
                mass_idx = [k for k, t in enumerate(ph.types) if t in (1, 2, 3)]
                w = rng.uniform(0.0, 1.0, (n_cells, nb, len(mech.aero_phases[pi].species)))
                for b in range(nb):
                    first = rep.first_state + sum(
                        len(mech.aero_phases[q].species) for q in rep.instances[:inst])
                    wsum = w[:, b, mass_idx].sum(axis=1) if mass_idx else np.ones(n_cells)
                    for k, t in enumerate(ph.types):
                        if t in (1, 2, 3):
                            dens = ph.floats[len(ph.species) + k]
                            state[:, first + k] = (vol[:, b] / len(sec.phases) * w[:, b, k] /
                                                   wsum * dens)
                        else:
                            state[:, first + k] = 1.0
                    inst += 1


def make_cells(
    mech: Mechanism,
    n_cells: int,
    seed: int,
    conc_lo: float = 1.0e-6,
    conc_hi: float = 1.0e2,
    photo_base: np.ndarray | None = None,
    constants: dict[str, float] | None = None,
) -> CellBatch:
    rng = np.random.Generator(np.random.PCG64(seed))
    T = rng.uniform(260.0, 310.0, n_cells)
    P = rng.uniform(5.0e4, 1.013e5, n_cells)
    factor = rng.uniform(0.0, 1.0, n_cells)
    if photo_base is None:
        photo_base = photo_base_rates(mech)
    photo = factor[:, None] * np.asarray(photo_base)[None, :]
    ns = mech.n_state_var
    state = np.zeros((n_cells, ns))
    var = mech.var_type == CHEM_SPEC_VARIABLE
    nvar = int(np.count_nonzero(var))
    logc = rng.uniform(np.log(conc_lo), np.log(conc_hi), (n_cells, nvar))
    state[:, var] = np.exp(logc)
    for i, name in enumerate(mech.species):
        if var[i]:
            continue
        v = None
        if constants and name in constants:
            v = constants[name]
        elif "init conc" in mech.species_props.get(name, {}):
            v = float(mech.species_props[name]["init conc"])
        state[:, i] = 0.0 if v is None else v
    env = np.stack([T, P], axis=1)
    is_photo = photolysis_columns(mech)
    if photo.shape[1] and not is_photo.all():
        other = rng.uniform(0.5, 1.5, n_cells)
        photo[:, ~is_photo] = other[:, None] * np.asarray(photo_base)[None, ~is_photo]
    if mech.aero_reps:
        _aerosol_cells(mech, rng, state, photo)
    return CellBatch(state=state, env=env, photo_rates=photo, seed=seed)


def make_cells_near_init(mech: Mechanism, n_cells: int, seed: int,
                         spread: float = 3.0) -> CellBatch:
    """Cells around the mechanism's own initial state: every variable
    species at its "init conc" (the cb05cl_ae5 test's initial state,
    ``test/chemistry/cb05cl_ae5/cb05cl_ae5_init.json``; 0 where none is
    given) times a per-cell, per-species factor log-uniform in
    [1/spread, spread]; T, P and the host-set rates as in ``make_cells``.
    Unlike the log-uniform workload, whose radicals start up to 1e2 ppm, such
    cells have a solution that the tolerances determine: two runs that
    differ by roundoff agree to far inside 1e-3 on every species."""
    cells = make_cells(mech, n_cells, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 0x5EED))
    var = mech.var_type == CHEM_SPEC_VARIABLE
    init = np.asarray([float(mech.species_props.get(s, {}).get("init conc", 0.0))
                       for s in mech.species])
    fac = np.exp(rng.uniform(-np.log(spread), np.log(spread), (n_cells, mech.n_state_var)))
    cells.state[:, var] = (init[None, :] * fac)[:, var]
    return cells


def constant_values(mech: Mechanism) -> dict[str, float]:
    """'init conc' of each non-variable species (packed fixtures keep these)."""
    out = {}
    for i, name in enumerate(mech.species):
        if mech.var_type[i] != CHEM_SPEC_VARIABLE:
            v = mech.species_props.get(name, {}).get("init conc")
            if v is not None:
                out[name] = float(v)
    return out


def n_photo(mech: Mechanism) -> int:
    """Host-set columns of a mechanism."""
    return len(mech.rate_columns())
