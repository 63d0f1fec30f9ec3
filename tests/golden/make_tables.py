"""Generates tests/golden/reference_tables.npz: the reference's own lookup tables.

Reads the text tables of a reference checkout (tables/: proton_cumul_ddd_data.txt,
density_Schneider2000_adj.txt, HU_to_SP_H&N_adj.txt, radiation_length.txt and
nuclear_weights_and_sigmas_fit.txt) with the reference's own parser,
energyReader (src/utils/energy_reader.cpp:21-185), built from its sources into
oracle/_ref/librtd_nuc.so by oracle/ref/build_ref.sh GAUSS_FIT (the nuclear build
also reads the halo tables). The package's parser, subsecondpbs_b200.tables.
energy_reader, must give bit-identical arrays, or the script stops. The archive
lets the tests and the benchmark use the reference's tables where the checkout is
not present (the GPU machine).

Usage: python tests/golden/make_tables.py [--reference <checkout>] [--out <npz>]
(the checkout defaults to $REFERENCE_DIR, else <repo>/../reference).
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from subsecondpbs_b200 import tables  # noqa: E402

REF_NUC_LIB = ROOT / "oracle" / "_ref" / "librtd_nuc.so"
FILES = (tables.PROTON_FILE, tables.DENSITY_FILE, tables.SP_FILE, tables.RRL_FILE, tables.NUCLEAR_FILE)


def default_checkout() -> Path:
    return Path(os.environ.get("REFERENCE_DIR", str(ROOT.parent / "reference")))


def reference_energy_reader(tables_dir: Path, lib_path: Path = REF_NUC_LIB) -> dict:
    """The reference's energyReader on `tables_dir`, as an energy dict (float32)."""
    lib = C.CDLL(str(lib_path))
    f = lib.ref_energy_reader
    f.restype = C.c_int
    sizes = (C.c_int * 6)()
    scales = (C.c_float * 3)()
    if f(str(tables_dir).encode(), sizes, scales, None, None, None, None) != 0:
        raise RuntimeError(f"reference energyReader failed on {tables_dir}")
    ns, ne, nd, nsp, nr, has_nuc = list(sizes)
    e = np.zeros(3 * ne, np.float32)
    cidd = np.zeros(ne * ns, np.float32)
    luts = np.zeros(nd + nsp + nr, np.float32)
    nuc = np.zeros(2 * ne * ns, np.float32)
    fp = C.POINTER(C.c_float)
    if f(str(tables_dir).encode(), sizes, scales, e.ctypes.data_as(fp), cidd.ctypes.data_as(fp),
         luts.ctypes.data_as(fp), nuc.ctypes.data_as(fp)) != 0:
        raise RuntimeError(f"reference energyReader failed on {tables_dir}")
    out = {
        "n_energies": ne, "n_energy_samples": ns,
        "energies_per_u": e[:ne], "peak_depths": e[ne:2 * ne], "scale_facts": e[2 * ne:],
        "cidd_matrix": cidd.reshape(ne, ns),
        "n_density_samples": nd, "density_scale_fact": float(scales[0]), "density_vector": luts[:nd],
        "n_sp_samples": nsp, "sp_scale_fact": float(scales[1]), "sp_vector": luts[nd:nd + nsp],
        "n_rrl_samples": nr, "rrl_scale_fact": float(scales[2]), "rrl_vector": luts[nd + nsp:],
    }
    if has_nuc:
        out["nuc_weight_matrix"] = nuc[:ne * ns].reshape(ne, ns)
        out["nuc_sq_sigma_matrix"] = nuc[ne * ns:].reshape(ne, ns)
        out["nuclear_tables_aligned_to_primary_axis"] = True
    return out


def same_tables(a: dict, b: dict) -> list:
    """Keys whose values differ (arrays compared bit for bit as float32)."""
    bad = []
    for k in sorted(set(a) | set(b)):
        if k not in a or k not in b:
            bad.append(k)
            continue
        x, y = a[k], b[k]
        if isinstance(x, np.ndarray) or isinstance(y, np.ndarray):
            x = np.asarray(x, np.float32)
            y = np.asarray(y, np.float32)
            if x.shape != y.shape or not np.array_equal(x.view(np.uint32), y.view(np.uint32)):
                bad.append(k)
        elif float(x) != float(y):
            bad.append(k)
    return bad


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(default_checkout()))
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "reference_tables.npz"))
    a = ap.parse_args(argv)
    tdir = Path(a.reference) / "tables"
    ref = reference_energy_reader(tdir)
    mine = tables.energy_reader(tdir, nuclear=True)
    bad = same_tables(ref, mine)
    if bad:
        raise SystemExit(f"tables.energy_reader differs from the reference's energyReader in: {bad}")
    digests = {f: hashlib.sha256((tdir / f).read_bytes()).hexdigest() for f in FILES}
    tables.save_table_npz(a.out, ref, source="Nelgcis/subsecondPBS tables/ read by its energyReader "
                          "(src/utils/energy_reader.cpp:21-185, NUCLEAR_CORR build)",
                          sha256=" ".join(f"{f}={d}" for f, d in digests.items()))
    print(a.out, Path(a.out).stat().st_size, "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
