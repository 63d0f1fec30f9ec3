"""ctypes driver of the reference library built by build_ref.sh (test
infrastructure only; runs where a GPU and oracle/_ref/ exist)."""
from __future__ import annotations

import ctypes as C
import os
import re
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE.parent / "_ref" / "librtd.so"


def available(path: Path = REF_LIB) -> bool:
    return path.exists()


def _load(path: Path = REF_LIB):
    from subsecondpbs_b200 import _lib as P

    lib = C.CDLL(str(path))
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int)
    lib.ref_subsecond_wrapper.restype = C.c_int
    lib.ref_subsecond_wrapper.argtypes = [fp, ip, fp, fp, fp, ip, fp, fp, C.POINTER(P.PbsBeamDesc), C.c_size_t,
                                          C.POINTER(P.PbsEnergyDesc), C.c_int, C.c_int, C.c_int]
    return lib


class _CaptureStdout:
    """Redirects the process-level stdout/stderr (C printf and std::cout) to a file."""

    def __enter__(self):
        import sys

        sys.stdout.flush()
        sys.stderr.flush()
        self.tmp = tempfile.TemporaryFile(mode="w+b")
        self.saved = (os.dup(1), os.dup(2))
        os.dup2(self.tmp.fileno(), 1)
        os.dup2(self.tmp.fileno(), 2)
        return self

    def __exit__(self, *exc):
        libc = C.CDLL(None)
        libc.fflush(None)
        os.dup2(self.saved[0], 1)
        os.dup2(self.saved[1], 2)
        os.close(self.saved[0])
        os.close(self.saved[1])
        self.tmp.seek(0)
        self.text = self.tmp.read().decode(errors="replace")
        self.tmp.close()


_BATCH = re.compile(r"Primary superposition batched launches:((?: \[rad=\d+:\d+\])*)")
_NUC_BATCH = re.compile(r"Nuclear superposition batched launches:((?: \[rad=\d+:\d+\])*)")
_ITEM = re.compile(r"\[rad=(\d+):(\d+)\]")


def parse_batched(text: str, nuclear: bool = False) -> list:
    """Per-layer batched radius counts (33 ints) the reference printed with verbose=1
    (complete_superposition.cu:486-495 primary, 660-669 nuclear halo)."""
    rows = []
    for m in (_NUC_BATCH if nuclear else _BATCH).finditer(text):
        row = [0] * 33
        for r, n in _ITEM.findall(m.group(1)):
            row[int(r)] = int(n)
        rows.append(row)
    return rows


def run(case: dict, beams=None, nuclear: bool = False, verbose: int = 1, path: Path = REF_LIB):
    """Run the reference on `case`; returns (dose float32 [Z][Y][X], per-layer batched
    counts parsed from its verbose output (list of 33-int lists), captured text)."""
    from subsecondpbs_b200 import _lib as P
    from subsecondpbs_b200.cudaCalDoseRTD import _with_luts

    lib = _load(path)
    beams = beams if beams is not None else [case["beam"]]
    descs, keep = [], []
    for b in beams:
        d, k = P.beam_desc(b)
        descs.append(d)
        keep.append(k)
    arr = (P.PbsBeamDesc * len(descs))(*descs)
    ed, ke = P.energy_desc(_with_luts(case["energy"], None))
    ct = np.ascontiguousarray(case["ct"], dtype=np.float32)
    dd = case["dose_dims"]
    dose = np.zeros((dd[2], dd[1], dd[0]), dtype=np.float32)
    fp = C.POINTER(C.c_float)
    with _CaptureStdout() as cap:
        rc = lib.ref_subsecond_wrapper(ct.ctypes.data_as(fp), P.int3(case["ct_dims"]), P.float3(case["ct_resolution"]),
                                       P.float3(case["ct_corner"]), dose.ctypes.data_as(fp), P.int3(dd),
                                       P.float3(case["dose_resolution"]), P.float3(case["dose_corner"]), arr,
                                       len(descs), C.byref(ed), 0, int(nuclear), int(verbose))
    if rc != 0:
        raise RuntimeError(f"reference returned {rc}:\n{cap.text[-2000:]}")
    del keep, ke
    return dose, parse_batched(cap.text), cap.text


def _headline_case():
    """The 256x256x160 heterogeneous CT with one 20-layer beam of 3020 spots on the
    reference's own proton tables (tests/golden/reference_tables.npz)."""
    from subsecondpbs_b200 import phantoms, tables

    t = tables.load_table_npz(HERE.parents[1] / "tests" / "golden" / "reference_tables.npz")
    t = {k: v for k, v in t.items() if not k.startswith("nuc")}
    return phantoms.heterogeneous_case(energy=t)


def time_reference(calls: int = 10, budget_s: float = 90.0, dose_out: str | None = None) -> dict:
    """Wall time of the reference's subsecondWrapper (host buffers in and out, as its
    callers use it) on the headline beam: one untimed call (module load, first-use
    set-up), then up to `calls` timed calls within `budget_s`; the median is reported.
    With `dose_out` the first call's dose is saved there (.npy)."""
    import time

    from subsecondpbs_b200 import _lib as P
    from subsecondpbs_b200.cudaCalDoseRTD import _with_luts

    case = _headline_case()
    lib = _load()
    bd, kb = P.beam_desc(case["beam"])
    ed, ke = P.energy_desc(_with_luts(case["energy"], None))
    ct = np.ascontiguousarray(case["ct"], dtype=np.float32)
    dd = case["dose_dims"]
    dose = np.zeros((dd[2], dd[1], dd[0]), dtype=np.float32)
    fp = C.POINTER(C.c_float)

    def call():
        dose[...] = 0.0
        with _CaptureStdout():
            rc = lib.ref_subsecond_wrapper(ct.ctypes.data_as(fp), P.int3(case["ct_dims"]),
                                           P.float3(case["ct_resolution"]), P.float3(case["ct_corner"]),
                                           dose.ctypes.data_as(fp), P.int3(dd), P.float3(case["dose_resolution"]),
                                           P.float3(case["dose_corner"]), C.byref(bd), 1, C.byref(ed), 0, 0, 0)
        if rc != 0:
            raise RuntimeError(f"reference returned {rc}")

    call()
    first_dose = dose.copy()
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < calls and (len(times) < 3 or time.perf_counter() < t_end):
        t = time.perf_counter()
        call()
        times.append((time.perf_counter() - t) * 1e3)
    # The first call's dose is the reference's answer; the last call's is compared with
    # it (the reference keeps state such as texture and memory caches across calls).
    drift = float(np.abs(dose.astype(np.float64) - first_dose).max() / max(float(first_dose.max()), 1e-30))
    if dose_out:
        np.save(dose_out, first_dose)
    del kb, ke
    return {"median_ms": float(np.median(times)), "calls": len(times), "times_ms": [round(x, 2) for x in times],
            "last_vs_first_call_max_diff_frac_dmax": drift}


if __name__ == "__main__":
    import argparse
    import json
    import sys

    sys.path.insert(0, str(HERE.parents[1]))
    ap = argparse.ArgumentParser(description="time the reference's subsecondWrapper on the headline beam")
    ap.add_argument("--calls", type=int, default=10)
    ap.add_argument("--budget-s", type=float, default=90.0)
    ap.add_argument("--dose-out", default=None)
    a = ap.parse_args()
    print(json.dumps(time_reference(a.calls, a.budget_s, a.dose_out)), flush=True)
