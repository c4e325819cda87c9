"""Generates the committed golden fixtures from the reference (run here only).

    python tests/golden/make_golden.py [REFERENCE_ROOT [TAG ...]]

Outputs (all small):
  cb05cl_ae5.mech.json   packed cb05cl_ae5 mechanism as the Fortran caller
                         would hand it to rxn_add_condensed_data (packer:
                         camp_b200/mechanism.py), with the photolysis ids the
                         reference's cb05 test assigns
  monarch_mod37_gas.mech.json
                         the gas-phase part of the shipped MONARCH mod37
                         configuration (mechanisms/monarch_mod37: cb05, 45
                         FIRST_ORDER_LOSS dry-deposition and 36 EMISSION
                         reactions) plus its WET_DEPOSITION of the "cloud and
                         rain water" phase, whose 49 species are appended as
                         state variables (no aerosol representation is read;
                         the packed wet-deposition data lists their indices as
                         the Fortran packer would)
  monarch_mod37_soa.mech.json
                         the same gas phase with the shipped 2-product SOA
                         scheme (4 Arrhenius + 4 SIMPOL_PHASE_TRANSFER into
                         the "organic matter" mode) and the shipped aerosol
                         phases and MONARCH modal/binned mass representation
                         (7 modes and bin sets, 99 aerosol state variables);
                         its wet deposition acts on the cloud-and-rain phase
                         instance.  The sub-models of mod37 (ZSR water,
                         PDFiTE activity) are not restated and are left out
  monarch_mod37_aero.mech.json
                         the SOA fixture plus the shipped partitioning of 35
                         gas-phase species into cloud and rain water
                         (cloud_and_rain_partitioning.json: HL_PHASE_TRANSFER
                         into the "clouds and rain" mode, aerosol-phase water
                         H2O_aq a constant species) and the 5 aqueous
                         equilibria of the sulfate mode
                         (inorganic_reactions.json; their ion pairs'
                         activity coefficients are constant species here, as
                         without the PDFiTE sub-model)
  monarch_mod37_shipped.mech.json
                         test/monarch/config_monarch_mod37.json as shipped:
                         cb05cl_ae5, the SOA scheme, HL partitioning of SULF,
                         HNO3 and NH3 into the aqueous sulfate phase, its
                         aqueous equilibria, and the ZSR aerosol-water and
                         PD-FiTE activity sub-models that make the phase's
                         water and ion-pair activity coefficients functions
                         of the state
  cb05cl_ae5_ref.npz, monarch_mod37_gas_ref.npz, monarch_mod37_soa_ref.npz,
  monarch_mod37_aero_ref.npz, monarch_mod37_shipped_ref.npz
                         outputs of the reference's own C code
                         (oracle/_ref/libcamp_ref.so, compiled from the
                         reference sources) on seeded cell states:
                         sparsity (solver CSC, reaction CSC, jac_map, packed
                         ints after rxn_update_ids), per-cell rate constants,
                         production/loss/net derivative and solver Jacobian
                         at several time steps

The cell states follow the workload distribution (camp_b200/cells.py, seed
20241203) plus a few edge-case cells: concentrations exactly at TINY, a dark
cell (all photolysis rates zero), a cell where PAR is nearly exhausted so
the negative-yield guard of the reference switches contributions off, and,
for mechanisms with aqueous equilibria, a cell whose aerosol water is below
their minimum, which switches them off.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from camp_b200.cells import make_cells  # noqa: E402
from camp_b200.mechanism import (CHEM_SPEC_VARIABLE, assign_rate_ids, load_mechanism,  # noqa: E402
                                 pack_wet_deposition)

SEED = 20241203
H_VALUES = (1.0e-6, 1.0, 60.0)


def cb05_files(ref_root: str) -> list[str]:
    return [
        os.path.join(ref_root, "mechanisms/cb05cl_ae5/cb05cl_ae5_mechanism.json"),
        os.path.join(ref_root, "mechanisms/cb05cl_ae5/cb05cl_ae5_species.json"),
        os.path.join(ref_root, "test/chemistry/cb05cl_ae5/cb05cl_ae5_init.json"),
    ]


MOD37_GAS_FILES = ("cb05_species.json", "cb05_abs_tol.json", "cb05_mechanism.json",
                   "custom_species.json", "dry_deposition.json", "HERMES_emissions_rxns.json",
                   "MEGAN_emissions_rxns.json")
RAIN_PHASE = "cloud and rain water"


def mod37_gas(ref_root: str):
    import json

    base = os.path.join(ref_root, "mechanisms/monarch_mod37")
    mech = load_mechanism([os.path.join(base, f) for f in MOD37_GAS_FILES],
                          name="monarch_mod37_gas")
    with open(os.path.join(base, "aerosol_phases.json")) as fh:
        phases = {o["name"]: o["species"] for o in json.load(fh)["camp-data"]
                  if o.get("type") == "AERO_PHASE"}
    first = mech.n_state_var
    names = [f"{RAIN_PHASE}.{sp}" for sp in phases[RAIN_PHASE]]
    mech.species = mech.species + names
    mech.var_type = np.concatenate([mech.var_type,
                                    np.full(len(names), CHEM_SPEC_VARIABLE, np.int32)])
    mech.abs_tol = np.concatenate([mech.abs_tol, np.full(len(names), 1.0e-8)])
    mech.rxns.append(pack_wet_deposition(list(range(first + 1, first + len(names) + 1)),
                                         1.0, "rain loss"))
    mech.rate_ids = assign_rate_ids(mech.rxns)
    return mech


MOD37_SOA_FILES = MOD37_GAS_FILES + ("inorganic_species.json", "cloud_and_rain_species.json",
                                     "tsigaridis_2_product_SOA_scheme/species.json",
                                     "tsigaridis_2_product_SOA_scheme/mechanism.json",
                                     "aerosol_phases.json", "aerosol_representation.json",
                                     "wet_deposition.json")


def mod37_soa(ref_root: str):
    from camp_b200.aerosol import load_aerosol_mechanism

    base = os.path.join(ref_root, "mechanisms/monarch_mod37")
    return load_aerosol_mechanism([os.path.join(base, f) for f in MOD37_SOA_FILES],
                                  name="monarch_mod37_soa")


MOD37_AERO_FILES = MOD37_SOA_FILES + ("cloud_and_rain_partitioning.json",
                                      "inorganic_reactions.json")


def mod37_aero(ref_root: str):
    from camp_b200.aerosol import load_aerosol_mechanism

    base = os.path.join(ref_root, "mechanisms/monarch_mod37")
    return load_aerosol_mechanism([os.path.join(base, f) for f in MOD37_AERO_FILES],
                                  name="monarch_mod37_aero")


def mod37_shipped(ref_root: str):
    """test/monarch/config_monarch_mod37.json as shipped: cb05cl_ae5, the
    mod37 species, aerosol phases and representation, HL partitioning of
    SULF / HNO3 / NH3 with the ZSR aerosol-water sub-model, the PD-FiTE
    activity sub-model, the aqueous equilibria and the 2-product SOA scheme
    (the config's build-tree paths ``mechanisms_run`` map to ``mechanisms``)."""
    from camp_b200.aerosol import load_aerosol_mechanism
    from camp_b200.mechanism import expand_config

    cfg = os.path.join(ref_root, "test/monarch/config_monarch_mod37.json")
    files = expand_config(cfg, lambda p: p.replace("mechanisms_run", "mechanisms"))
    return load_aerosol_mechanism(files, name="monarch_mod37_shipped")


def edge_cells(mech, cells):
    """Appends edge-case cells to a seeded batch."""
    st, env, ph = cells.state.copy(), cells.env.copy(), cells.photo_rates.copy()
    extra_s, extra_e, extra_p = [], [], []
    var = mech.var_type == 1
    # concentrations at TINY
    s = st[0].copy()
    s[var] = 1.0e-60
    extra_s.append(s); extra_e.append([298.0, 101325.0]); extra_p.append(ph[0])
    # dark cell (every host-set reaction rate 0; GMD / GSD kept)
    dark = ph[1].copy()
    dark[[j for j, c in enumerate(mech.rate_columns()) if c[0] == "rxn"]] = 0.0
    extra_s.append(st[1].copy()); extra_e.append(env[1]); extra_p.append(dark)
    # PAR nearly exhausted while its negative-yield producers are abundant
    s = st[2].copy()
    s[mech.index("PAR")] = 1.0e-12
    for name in ("ROR", "OLE", "IOLE", "ISOP", "TERP"):
        if name in mech.species:
            s[mech.index(name)] = 50.0
    extra_s.append(s); extra_e.append([300.0, 1.0e5]); extra_p.append(ph[2])
    # aqueous equilibria: their water below the reaction's minimum
    # (1e-4 x absolute tolerance / 10), which switches them off
    water = set()
    for r in mech.rxns:
        if r.rxn_type == 7:  # AQUEOUS_EQUILIBRIUM
            nr, np_, nph = int(r.ints[0]), int(r.ints[1]), int(r.ints[2])
            water.update(int(r.ints[3 + (nr + np_) * nph + k]) - 1 for k in range(nph))
    if water:
        s = st[3].copy()
        for i in water:
            s[i] = 1.0e-4 * mech.abs_tol[i] / 10.0 / 10.0
        extra_s.append(s); extra_e.append(env[3]); extra_p.append(ph[3])
    return (np.vstack([st, np.asarray(extra_s)]), np.vstack([env, np.asarray(extra_e)]),
            np.vstack([ph, np.asarray(extra_p)]))


def main(ref_root: str, only: list[str] | None = None) -> None:
    sys.path.insert(0, ROOT)
    from oracle.oracle import build  # noqa: E402

    build(with_ref=True)
    makers = {
        "cb05cl_ae5": lambda: load_mechanism(cb05_files(ref_root), name="cb05cl_ae5"),
        "monarch_mod37_gas": lambda: mod37_gas(ref_root),
        "monarch_mod37_soa": lambda: mod37_soa(ref_root),
        "monarch_mod37_aero": lambda: mod37_aero(ref_root),
        "monarch_mod37_shipped": lambda: mod37_shipped(ref_root),
    }
    for tag, make in makers.items():
        if not only or tag in only:
            write_fixture(make(), tag)


def write_fixture(mech, tag: str) -> None:
    from oracle.oracle import RefModel  # noqa: E402

    mech.rel_tol = 1.0e-4
    mech.abs_tol[:] = 1.0e-8
    mech.save(os.path.join(HERE, f"{tag}.mech.json"))

    cells = make_cells(mech, 8, SEED)
    state, env, photo = edge_cells(mech, cells)
    nc = state.shape[0]
    ref = RefModel(mech, nc)
    out = {}
    cp, ri = ref.solver_jac()
    out["solver_colptr"], out["solver_rowid"] = cp, ri
    rcp, rri = ref.rxn_jac()
    out["rxn_colptr"], out["rxn_rowid"] = rcp, rri
    out["jac_map"] = ref.jac_map()
    out["rxn_int_data"] = ref.rxn_int_data()
    out["state"], out["env"], out["photo"] = state, env, photo
    out["h"] = np.asarray(H_VALUES)
    rxn_env, F, RP, RL, J = [], [], [], [], []
    for c in range(nc):
        ref.set_cell(c, state[c], env[c])
        ref.set_rates(c, photo[c])
        ref.update_env(c)
        rxn_env.append(ref.rxn_env(c))
    for h in H_VALUES:
        fs, rps, rls, js = [], [], [], []
        for c in range(nc):
            # the reference keeps a mode's effective radius per solver, not
            # per cell: apply this cell's GMD / GSD again before its f and J
            ref.set_rates(c, photo[c])
            f, rp, rl = ref.deriv(c, h)
            j, _ = ref.jac(c, h)
            fs.append(f); rps.append(rp); rls.append(rl); js.append(j)
        F.append(fs); RP.append(rps); RL.append(rls); J.append(js)
    out["rxn_env"] = np.asarray(rxn_env)
    out["f"], out["r_p"], out["r_l"], out["jac"] = (np.asarray(x) for x in (F, RP, RL, J))
    np.savez_compressed(os.path.join(HERE, f"{tag}_ref.npz"), **out)
    print(tag, "wrote", nc, "cells;", "jac nnz", len(ri), "rxn jac nnz", len(rri))


if __name__ == "__main__":
    # make_golden.py [REFERENCE_ROOT [TAG ...]]: all fixtures, or the named ones
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CAMP_REFERENCE_ROOT", "/root/reference"),
         sys.argv[2:] or None)
