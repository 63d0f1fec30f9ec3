"""Generates the golden fixtures of this directory by running the reference itself.

The reference's dose path is CUDA-only, so this script runs on a GPU machine with
the reference library built from the reference's own sources by
oracle/ref/build_ref.sh (oracle/_ref/librtd.so). For every case it stores the
reference's float32 dose grid and the per-layer batched radius counts the
reference prints with verbose=1 (complete_superposition.cu:476-495), together with
the arguments that regenerate the seeded inputs with subsecondpbs_b200.phantoms.

Usage: python tests/golden/make_golden.py --out <dir>
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from subsecondpbs_b200 import phantoms  # noqa: E402

# name -> (builder, kwargs, beam transform)
CASES = {
    "water_small": ("water_phantom_case", {"dims": [32, 32, 96], "n_side": 5, "energy_mev": 120.0}, None),
    "water_config1": ("water_phantom_case", {}, None),
    "hetero_small": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                            "e_range": [80.0, 120.0]}, None),
    "hetero_rot30": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                            "e_range": [80.0, 120.0]}, {"rotate": 30.0}),
    "hetero_legacy": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 2, "target_radius_mm": 12.0,
                                             "e_range": [90.0, 110.0]}, {"legacy": True}),
    # Nuclear halo (reference built with NUCLEAR_CORR=GAUSS_FIT, oracle/_ref/librtd_nuc.so),
    # synthetic halo tables on the proton axes (subsecondpbs_b200.tables.synthetic_nuclear_tables).
    "halo_small": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                          "e_range": [80.0, 120.0]}, {"nuclear": "GAUSS_FIT"}),
    # Water-equivalence import (the CarbonPBS rayweq contract): exporter depths in
    # place of the CT trace, spot positions as rayweq texel coordinates.
    "weq_small": ("weq_case", {}, None),
    # Carbon ions with the nuclear halo (synthetic carbon tables and their halo tables).
    "carbon_halo_small": ("carbon_case", {"dims": [64, 64, 48], "res": [2.0, 2.0, 2.0], "gantries": [90.0],
                                          "n_layers": 3, "e_range": [120.0, 200.0], "spots_per_layer": 40},
                          {"nuclear": "GAUSS_FIT"}),
    # The reference's own tables (reference_tables.npz, made by make_tables.py from
    # the reference's tables/ with its energyReader): configs 1 and 2 in small form,
    # a gantry of 30 deg, and the nuclear halo with the reference's
    # nuclear_weights_and_sigmas_fit.txt.
    "water_config1_rt": ("water_phantom_case", {}, {"tables": "reference"}),
    "hetero_small_rt": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                               "e_range": [80.0, 120.0]}, {"tables": "reference"}),
    "hetero_rot30_rt": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                               "e_range": [80.0, 120.0]}, {"tables": "reference", "rotate": 30.0}),
    "hetero_mid_rt": ("heterogeneous_case", {"dims": [96, 96, 64], "n_layers": 6, "target_radius_mm": 20.0,
                                             "e_range": [70.0, 150.0]}, {"tables": "reference"}),
    # The bench's headline beam (config 2): 256x256x160 CT, 20 layers 70-180 MeV, 3020 spots.
    "headline_rt": ("heterogeneous_case", {}, {"tables": "reference"}),
    "halo_small_rt": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                             "e_range": [80.0, 120.0]}, {"tables": "reference", "nuclear": "GAUSS_FIT"}),
    # CarbonPBS lateral profile model (sigma override and overall weight), which the
    # reference compiles but keeps off: made by the reference built with both switches
    # on (oracle/ref/build_ref.sh OFF profile, oracle/_ref/librtd_profile.so), with a
    # seeded profile table per layer (phantoms.with_carbon_profile), and with the
    # profile rows on their own energy axis.
    "profile_small_rt": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                                "e_range": [80.0, 120.0]}, {"tables": "reference", "profile": "layers"}),
    "profile_energy_rows_rt": ("heterogeneous_case", {"dims": [64, 64, 48], "n_layers": 3, "target_radius_mm": 14.0,
                                                      "e_range": [80.0, 120.0]},
                               {"tables": "reference", "profile": "energies"}),
}

REFERENCE_TABLES = Path(__file__).resolve().parent / "reference_tables.npz"


def reference_tables(nuclear: bool) -> dict:
    """The reference's tables (reference_tables.npz); without `nuclear` the halo
    tables are left out."""
    from subsecondpbs_b200 import tables

    t = tables.load_table_npz(REFERENCE_TABLES)
    if not nuclear:
        for k in ("nuc_weight_matrix", "nuc_sq_sigma_matrix", "nuclear_tables_aligned_to_primary_axis"):
            t.pop(k, None)
    return t


def build_case(name: str):
    builder, kw, tf = CASES[name]
    kw = {k: (tuple(v) if isinstance(v, list) else v) for k, v in kw.items()}
    case = getattr(phantoms, builder)(**kw)
    if tf and tf.get("tables") == "reference":
        case = dict(case)
        case["energy"] = reference_tables("nuclear" in tf)
    elif tf and "nuclear" in tf:
        from subsecondpbs_b200 import tables

        case = dict(case)
        case["energy"] = tables.synthetic_nuclear_tables(case["energy"])
    beam = case["beam"]
    if tf and "rotate" in tf:
        beam = phantoms.rotate_beam(beam, tf["rotate"])
    if tf and "profile" in tf:
        beam = phantoms.with_carbon_profile(beam, rows=tf["profile"])
    if tf and tf.get("legacy"):
        beam = phantoms.legacy_beam(beam)
    return case, beam


def main(argv=None) -> int:
    from oracle.ref import ref

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    a = ap.parse_args(argv)
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    for name in a.cases:
        case, beam = build_case(name)
        builder, kw, tf = CASES[name]
        nuclear = bool(tf and "nuclear" in tf)
        lib = ref.REF_LIB.parent / "librtd_nuc.so" if nuclear else ref.REF_LIB
        if tf and "profile" in tf:
            lib = ref.REF_LIB.parent / "librtd_profile.so"
        dose, batched, text = ref.run(case, beams=[beam], nuclear=nuclear, verbose=1, path=lib)
        build = f"NUCLEAR_CORR={tf['nuclear']}" if nuclear else "NUCLEAR_CORR=OFF"
        if tf and "profile" in tf:
            build += ", CarbonPBS profile switches on"
        meta = {"case": name, "builder": builder, "kwargs": kw, "transform": tf,
                "reference": f"Nelgcis/subsecondPBS subsecondWrapper built by oracle/ref/build_ref.sh ({build})",
                "dose_max": float(dose.max()), "dose_sum": float(dose.sum())}
        extra = {}
        if nuclear:
            extra["nuc_batched"] = np.asarray(ref.parse_batched(text, nuclear=True), np.int32).reshape(-1, 33)
        np.savez_compressed(out / f"{name}.npz", dose=dose.astype(np.float32),
                            batched=np.asarray(batched, np.int32).reshape(-1, 33), meta=json.dumps(meta), **extra)
        (out / f"{name}.log").write_text(text[-20000:])
        print(name, dose.shape, float(dose.max()), len(batched), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
