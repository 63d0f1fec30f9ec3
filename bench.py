#!/usr/bin/env python
"""Benchmark of the pencil-beam dose path: ms per beam dose on the heterogeneous
256x256x160 CT (2 mm) with one 20-layer proton beam of ~3000 spots.

One step = the whole dose of one beam: host planning, BEV tracing, spot->ray
fluence, IDD/sigma, tile binning, superposition, transfer into the FP64 dose grid
and the float readout of the grid, with CT and lookup tables resident in HBM.
`e2e` repeats the step through the C ABI (pbs_subsecond_wrapper) from pinned host
buffers, host<->device copies included. Under torchrun every rank computes one
beam of an opposed-beam plan (gantry 90/270) and the FP64 beam doses are summed
to rank 0 with one NCCL reduce per step (weak scaling).

The lookup tables are the reference's own (its tables/ files as its energyReader
reads them, kept in tests/golden/reference_tables.npz). On one GPU the line also
carries `reference_gpu`: the reference's own subsecondWrapper, built from its
sources by oracle/ref/build_ref.sh, timed on the same beam in a child process,
and its dose against this library's in the reference's BEV depth convention.

`--impl reference` times the reference path's CPU restatement (the oracle port)
on the host cores; the reference ships no CPU implementation of this path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ms per beam dose (256²×160, 3k spots); served plans/s, p50/p99 latency"
WORKLOAD = ("heterogeneous CT 256x256x160 at 2 mm (body ellipsoid, lung slab, 2 bone cylinders), "
            "1 proton beam at gantry 90 deg, 20 layers 70-180 MeV, 3020 spots on a 5 mm hex grid, "
            "7x7 subspots, 1 mm rays")
DATA = ("synthetic seeded phantom; the reference's own proton lookup tables (tables/ as read by its "
        "energyReader)")
TABLES = ROOT / "tests" / "golden" / "reference_tables.npz"
# The same `config` on both arms (the workload and how the L2 is treated between
# timed steps); run details of either arm go under `run`.
L2_NOTE = "GPU arm: L2 flushed between timed steps (256 MiB write outside the step events); CPU arm: not applicable"
CONFIG = {"workload": WORKLOAD, "l2": L2_NOTE}
REF_LIB = ROOT / "oracle" / "_ref" / "librtd.so"


def _proton_tables() -> dict:
    """The reference's proton tables without its nuclear halo tables."""
    from subsecondpbs_b200 import tables

    return {k: v for k, v in tables.load_table_npz(TABLES).items() if not k.startswith("nuc")}


def _headline_case() -> dict:
    from subsecondpbs_b200 import phantoms

    return phantoms.heterogeneous_case(energy=_proton_tables())


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU path (oracle/_ref/librtd.so)")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the secondary timings (spot-weight adjoint, carbon plan)")
    ap.add_argument("--serving-requests", type=int, default=1000, help="served stream length (0: skip)")
    ap.add_argument("--serving-slots", type=int, default=8)
    ap.add_argument("--serving-budget-mib", type=int, default=0, help="server HBM budget (0: 90%% of free)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [r.split(",") for r in Path(self.path).read_text().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _cpu_oracle_ms(case, budget_s=12.0, max_runs=20):
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    times = []
    dose = None
    t_end = time.perf_counter() + budget_s
    while len(times) < max_runs and (not times or time.perf_counter() < t_end):
        t = time.perf_counter()
        dose = O.dose(case, threads=threads)["dose"]
        times.append((time.perf_counter() - t) * 1e3)
    return statistics.median(times), threads, len(times), dose


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import oracle as O

    case = _headline_case()
    threads = os.cpu_count() or 1
    for _ in range(max(args.warmup, 1)):
        O.dose(case, threads=threads)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        O.dose(case, threads=threads)
        times.append((time.perf_counter() - t) * 1e3)
    ms = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": dict(CONFIG),
        "run": {"arm": "CPU restatement of the reference's dose path (the oracle port), all host threads"},
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "port",
                         "sample": f"full workload: {args.steps} beams after {args.warmup} warm-up beams"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _adjoint_cost(local: int, reps: int = 5) -> dict:
    """Inverse-planning gradient: the forward dose of four ~8000-spot beams on the
    64x64x128 water phantom and the FP64 least-squares objective (2 Gy in a 5 cm
    sphere, 0 Gy in a 2 cm shell), against the spot-weight adjoint of the same
    plan (all four beams), both synchronised wall-clock medians on one GPU."""
    import torch

    from subsecondpbs_b200 import phantoms
    from subsecondpbs_b200.autograd import with_weights
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    case = phantoms.inverse_planning_case(energy=_proton_tables())
    dev = torch.device("cuda", local)
    eng = DoseEngine(local)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    dd = case["dose_dims"]
    dose = torch.empty((dd[2], dd[1], dd[0]), dtype=torch.float64, device=dev)
    tt = torch.from_numpy(case["target"]).to(dev)
    ts = torch.from_numpy(case["shell"]).to(dev)
    p = case["prescription"]
    beams = [eng.prepare_beam(b) for b in case["beams"]]

    def forward():
        eng.reset_dose()
        for b in beams:
            eng.add_beam(b)
        eng.read_dose64(dose)
        eng.synchronize()
        return dose

    d = forward()
    s = p / float(d[tt].mean())
    beams = [eng.prepare_beam(with_weights(b, b["spot_weights"] * s)) for b in case["beams"]]
    n_spots = [int(np.sum(b["layer_spot_counts"])) for b in case["beams"]]

    def objective():
        d = forward()
        g = torch.zeros_like(d)
        g[tt] = 2.0 * (d[tt] - p)
        g[ts] = 2.0 * d[ts]
        j = float(((d[tt] - p) ** 2).sum() + (d[ts] ** 2).sum())
        torch.cuda.synchronize(dev)
        return j, g

    def adjoint(g):
        return [eng.adjoint_beam(b, g, n) for b, n in zip(beams, n_spots)]

    for _ in range(2):
        _, g = objective()
        adjoint(g)
    tf, ta = [], []
    for _ in range(reps):
        t = time.perf_counter()
        j, g = objective()
        tf.append((time.perf_counter() - t) * 1e3)
        t = time.perf_counter()
        adjoint(g)
        ta.append((time.perf_counter() - t) * 1e3)
    fwd, adj = statistics.median(tf), statistics.median(ta)
    return {"workload": "water 64x64x128 at 2 mm, 4 beams (gantry 0/90/180/270) x 36 layers x 225 spots",
            "spots": int(sum(n_spots)), "objective": "FP64 least squares on the GPU", "objective_value": j,
            "forward_ms": round(fwd, 3), "adjoint_ms": round(adj, 3), "adjoint_over_forward": round(adj / fwd, 3),
            "timing": f"median of {reps} synchronised wall-clock runs; forward includes the FP64 readout and "
                      "objective, adjoint includes the per-spot gradient readout"}


def _serving(local: int, n_requests: int, slots: int, budget_mib: int) -> dict:
    """Served mixed stream (seeded Poisson arrivals; CTs 128^3 and 256x256x160 at
    2 mm and 512x512x200 at 1 mm; 1-4 beams; heavy-tailed 500-20000 spots per
    field; 80/20 proton/carbon, carbon with the nuclear halo) through the
    continuous-batching server, against the plain pipeline that runs one request
    at a time through pbs_subsecond_wrapper."""
    from subsecondpbs_b200 import _lib, phantoms, serving
    from subsecondpbs_b200.precision import max_rel_err

    w = phantoms.serving_workload(n_requests=n_requests, proton_energy=_proton_tables())
    prepared = [[_lib.beam_desc(b) for b in phantoms.request_beams(w, r)] for r in w["requests"]]
    check = set(range(0, n_requests, max(1, n_requests // 16)))
    # Both sides are measured warm, as a long-running service: one untimed pass of the
    # whole stream first, so that the plain pipeline's context and the server's slots
    # hold their largest buffers and the server its per-field traces.
    serving.plain_pipeline(w, prepared, local)
    plain = serving.plain_pipeline(w, prepared, local, keep=check)
    ps = plain["service_s"] * 1e3
    device = serving.device_pipeline(w, prepared, local)
    srv = serving.DoseServer(local, slots=slots, hbm_budget_mib=budget_mib)
    srv.add_energy(0, w["energy"]["proton"])
    srv.add_energy(1, w["energy"]["carbon"])
    for p in w["patients"]:
        srv.add_patient(p["id"], p["ct"], p["ct_dims"], p["ct_resolution"], p["ct_corner"])
    serving.serve_workload(srv, w, prepared, arrivals=False)
    sat = serving.serve_workload(srv, w, prepared, arrivals=False, keep=check)
    rate = 0.8 * sat["plans_per_s"]
    poi = serving.serve_workload(srv, serving.with_rate(w, rate), prepared, arrivals=True)
    stats = srv.stats()
    srv.close()
    diffs = [max_rel_err(sat["doses"][i], plain["doses"][i], thr=0.0) for i in sorted(check)]

    def pct(a, q):
        return round(float(np.quantile(a, q)), 3)

    sl, pl = sat["latency_s"] * 1e3, poi["latency_s"] * 1e3
    return {
        "workload": f"{n_requests} requests, {len(w['patients'])} patients (CT 128^3@2mm, 256x256x160@2mm, "
                    "512x512x200@1mm), 1-4 beams of 500-20000 spots (Pareto 1.1), 80/20 proton/carbon+halo",
        "slots": slots, "hbm_budget_mib": budget_mib or "90% of free",
        "warmup": "one untimed pass of the whole stream on each side",
        "plain": {"plans_per_s": round(plain["plans_per_s"], 2), "p50_ms": pct(ps, 0.5), "p99_ms": pct(ps, 0.99),
                  "api": "pbs_subsecond_wrapper per request, pinned host CT and dose"},
        "saturated": {"plans_per_s": round(sat["plans_per_s"], 2), "p50_ms": pct(sl, 0.5), "p99_ms": pct(sl, 0.99),
                      "arrivals": "all at t=0"},
        "poisson": {"rate_hz": round(rate, 2), "plans_per_s": round(poi["plans_per_s"], 2), "p50_ms": pct(pl, 0.5),
                    "p99_ms": pct(pl, 0.99)},
        "device_serial": {"plans_per_s": round(device["plans_per_s"], 2),
                          "what": "the same requests' kernels back to back on one resident context per ion, "
                                  "CUDA-event device time per request (no host planning, uploads or copies)"},
        "served_over_plain": round(sat["plans_per_s"] / plain["plans_per_s"], 3),
        "served_over_device_serial": round(sat["plans_per_s"] / device["plans_per_s"], 3),
        "result_max_diff_vs_plain_frac_dmax": float(max(diffs)),
        "server_stats": {k: v for k, v in stats.items() if k in ("completed", "failed", "patient_loads",
                                                                  "evictions", "peak_bytes", "budget_bytes")},
    }


def _carbon_plan(local: int, reps: int = 3, with_dose: bool = False):
    """Carbon-ion plan with the nuclear halo (512x512x200 CT at 1 mm, three beams of
    40 layers 120-400 MeV/u, ~15,000 spots): device time of the whole plan on the
    context stream, median of `reps` after one warm-up."""
    import torch

    from subsecondpbs_b200 import phantoms
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    case = phantoms.carbon_case()
    eng = DoseEngine(local, nuclear_model=2)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    beams = [eng.prepare_beam(b) for b in case["beams"]]
    stream = torch.cuda.ExternalStream(eng.stream_handle, device=torch.device("cuda", local))
    ms = []
    for rep in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.reset_dose()
        for b in beams:
            eng.add_beam(b, nuclear_correction=True)
        e1.record(stream)
        eng.synchronize()
        if rep:
            ms.append(e0.elapsed_time(e1))
    dose = eng.read_dose64() if with_dose else None
    eng.close()
    out = {"workload": "carbon + nuclear halo (GAUSS_FIT), CT 512x512x200 at 1 mm, 3 beams (0/120/240 deg) x 40 "
                       "layers 120-400 MeV/u, 14,520 spots, 9x9 subspots",
           "ms_per_plan": round(statistics.median(ms), 3), "timing": f"CUDA events, median of {reps}"}
    return (out, dose, case) if with_dose else out


def _carbon_precision(case: dict, dose) -> dict:
    """Error of the carbon plan's dose against the FP64 oracle on the same inputs
    (halo included), over the box of voxels above 1 % of the oracle's maximum with a
    two-voxel margin (the gamma's neighbour shifts stay inside it)."""
    from oracle import oracle as O
    from subsecondpbs_b200 import precision as prec

    t = time.perf_counter()
    ref = O.dose(case, beams=case["beams"], nuclear_model=2, threads=os.cpu_count() or 1)["dose"]
    oracle_s = time.perf_counter() - t
    nz = np.nonzero(ref > 0.01 * ref.max())
    box = tuple(slice(max(int(a.min()) - 2, 0), min(int(a.max()) + 3, n)) for a, n in zip(nz, ref.shape))
    rep = prec.report(dose[box], ref[box], case["dose_resolution"])
    return dict(rep, reference="FP64 oracle, same inputs, nuclear halo GAUSS_FIT",
                region=f"voxels above 10 % of Dmax (box {[s.stop - s.start for s in box]} of {list(ref.shape)})",
                oracle_s=round(oracle_s, 1))


def _operator_export(local: int, n_spots: int = 1024, n_face: int = 256) -> dict:
    """Influence-matrix export of the headline beam's spots: the C ABI call
    (pbs_context_influence_csc: every column computed, compacted on the device and
    copied to host arrays) on `n_spots` spots, and the Python face (which adds the
    scipy CSC matrix) on `n_face` spots, wall time after a warm-up call each."""
    import ctypes as C
    import time

    from subsecondpbs_b200 import _lib
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    case = _headline_case()
    eng = DoseEngine(local)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    beam = eng.prepare_beam(case["beam"])
    bd, _keep = beam
    begin = 1000
    cap = 40000 * n_spots
    col_ptr = np.zeros(n_spots + 1, dtype=np.int64)
    rows = np.zeros(cap, dtype=np.int32)
    vals = np.zeros(cap, dtype=np.float32)
    nnz = C.c_longlong(0)

    def c_call(first):
        return eng._lib.pbs_context_influence_csc(
            eng._h, C.byref(bd), 0, first, n_spots, 0.0, col_ptr.ctypes.data_as(C.POINTER(C.c_longlong)),
            rows.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p), cap, C.byref(nnz))

    import torch

    free_gib = torch.cuda.mem_get_info(local)[0] / 2**30
    _lib.check(c_call(0))
    t = time.perf_counter()
    _lib.check(c_call(begin))
    c_ms = (time.perf_counter() - t) * 1e3
    entries = int(nnz.value)
    fcap = 40000 * n_face
    eng.influence_csc(beam, spot_begin=begin - n_face, spot_count=n_face, capacity=fcap)
    t = time.perf_counter()
    a = eng.influence_csc(beam, spot_begin=begin, spot_count=n_face, capacity=fcap)
    f_ms = (time.perf_counter() - t) * 1e3
    eng.close()
    return {"workload": f"{n_spots} spots of the headline beam (from spot {begin}), threshold 0",
            "ms": round(c_ms, 2), "ms_per_spot": round(c_ms / n_spots, 4), "entries": entries,
            "timing": "wall time of one pbs_context_influence_csc call (C ABI, host arrays) after a warm-up call",
            "device_free_gib_before": round(free_gib, 1),
            "python_face": {"spots": n_face, "ms": round(f_ms, 2), "ms_per_spot": round(f_ms / n_face, 4),
                            "entries": int(a.nnz), "what": "DoseEngine.influence_csc, scipy CSC matrix included"}}


def _upstream_cpu_conv(eng, stats: dict, spacing_mm: float, our_conv_ms: float, budget_s: float = 10.0) -> dict:
    """Stage-level CPU baseline of the spot-to-ray convolution: the upstream
    RayTraceDicom CPU Gaussian convolution (xConvCpu then yConvCpu,
    RayTraceDicom-main/src/cpu_convolution_1d.cpp, built from its sources into
    oracle/_ref/librtd_cpuconv.so by oracle/ref/build_upstream_conv.sh), single
    threaded as shipped, over a dense weight map of the headline beam's ray grid for
    each of its layers with the layer's entry sigma in ray pixels (3-sigma radius)."""
    lib_path = ROOT / "oracle" / "_ref" / "librtd_cpuconv.so"
    if not lib_path.exists():
        return {"unavailable": "oracle/_ref/librtd_cpuconv.so not built (oracle/ref/build_upstream_conv.sh needs the "
                               "reference sources)"}
    import ctypes as C
    import time

    lib = C.CDLL(str(lib_path))
    fp = C.POINTER(C.c_float)
    lib.upstream_x_conv_cpu.argtypes = [fp, fp, C.c_float, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int]
    lib.upstream_y_conv_cpu.argtypes = [fp, fp, C.c_float, C.c_uint, C.c_uint, C.c_uint, C.c_int]
    rx, ry = stats["ray_dims"]
    layers = []
    for l in range(stats["num_layers"]):
        sig = max(float(eng.layer_stats(l)["entry_sigma"][0]) / spacing_mm, 1e-3)
        layers.append((1.0 / (np.sqrt(2.0) * sig), int(np.ceil(3.0 * sig))))
    rng = np.random.Generator(np.random.PCG64(7))
    src = rng.random((ry, rx), dtype=np.float32)
    mid = np.zeros((ry, rx), np.float32)
    outs = [np.zeros((ry + 2 * rad, rx), np.float32) for _, rad in layers]

    def one_beam():
        for (rs, rad), out in zip(layers, outs):
            out[...] = 0.0
            lib.upstream_x_conv_cpu(src.ctypes.data_as(fp), mid.ctypes.data_as(fp), rs, rad, rx, rx, ry, 0)
            lib.upstream_y_conv_cpu(mid.ctypes.data_as(fp), out.ctypes.data_as(fp), rs, rad, ry, rx, rad)

    one_beam()
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < 3 or (len(times) < 50 and time.perf_counter() < t_end):
        t = time.perf_counter()
        one_beam()
        times.append((time.perf_counter() - t) * 1e3)
    ms = float(np.median(times))
    return {"stage": "spot-to-ray convolution", "impl": "upstream RayTraceDicom xConvCpu + yConvCpu "
            "(cpu_convolution_1d.cpp) built from its sources, 1 thread", "ms_per_beam": round(ms, 3),
            "ours_conv_ms": round(our_conv_ms, 4), "ratio": round(ms / max(our_conv_ms, 1e-9), 1),
            "sample": f"{len(layers)} layers on the {rx}x{ry} ray grid, median of {len(times)} beams"}


def _reference_gpu(local: int, case: dict, our_e2e_ms: float) -> dict | None:
    """The reference's own GPU path on the same beam and tables: its subsecondWrapper
    (built from its sources into oracle/_ref/librtd.so) timed in a child process,
    host buffers in and out as its callers use it. Its dose is then compared with
    this library's dose computed in the reference's BEV depth convention
    (PBS_OPT_COMPAT_BEV_Z_SHIFT), the one deliberate difference of the default path."""
    if not REF_LIB.exists():
        return {"unavailable": "oracle/_ref/librtd.so not built (oracle/ref/build_ref.sh needs the reference sources)"}
    from subsecondpbs_b200 import precision as prec
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    with tempfile.TemporaryDirectory() as d:
        dose_path = Path(d) / "ref_dose.npy"
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
        r = subprocess.run([sys.executable, "-m", "oracle.ref.ref", "--calls", "10", "--budget-s", "90",
                            "--dose-out", str(dose_path)], cwd=str(ROOT), capture_output=True, text=True,
                           timeout=600, env=env)
        if r.returncode != 0:
            return {"unavailable": f"reference run failed (rc {r.returncode}): {r.stderr.strip()[-300:]}"}
        timing = json.loads(r.stdout.strip().splitlines()[-1])
        ref_dose = np.load(dose_path)
    eng = DoseEngine(local, compat_bev_z_shift=True)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    eng.add_beam(case["beam"])
    ours = eng.read_dose()
    eng.close()
    agreement = prec.report(ours, ref_dose.astype(np.float64), case["dose_resolution"])
    return {"api": "reference subsecondWrapper (raytracedicom_wrapper.cu:2446) built from its sources for sm_100a "
                   "by oracle/ref/build_ref.sh, host buffers, verbose=0",
            "e2e_ms_median": round(timing["median_ms"], 3), "calls": timing["calls"],
            "reference_last_vs_first_call_max_diff_frac_dmax": timing.get("last_vs_first_call_max_diff_frac_dmax"),
            "ours_e2e_ms": round(our_e2e_ms, 4),
            "speedup_e2e": round(timing["median_ms"] / our_e2e_ms, 1),
            "dose_agreement": dict(agreement, against="this library with the reference's BEV depth shift, "
                                                      "same inputs (voxels above 10 % of Dmax)")}


def run_ours(args):
    import ctypes as C

    import torch
    import torch.distributed as dist

    from subsecondpbs_b200 import _lib, phantoms, sharding
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine, fp32_peak_tflops

    world, rank, local = _dist()
    if world > 1:
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    case = _headline_case()
    # N > 1: a plan of one beam per rank (opposed gantry angles), divided by the
    # sharding module's assignment; each rank computes its beam and the FP64 grids
    # are reduced on rank 0.
    plan = [case["beam"] if world == 1 else phantoms.rotate_beam(case["beam"], 90.0 + 180.0 * (k % 2))
            for k in range(world)]
    mine = sharding.assign_beams([sharding.beam_cost(b) for b in plan], world)[rank]
    beam = plan[mine[0]]
    dims = case["dose_dims"]
    n_vox = int(np.prod(dims))

    peak_fp32 = fp32_peak_tflops(local)

    eng = DoseEngine(local, stage_timing=True)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    stream = torch.cuda.ExternalStream(eng.stream_handle, device=dev)
    out = torch.empty((dims[2], dims[1], dims[0]), dtype=torch.float32, device=dev)
    d64 = torch.empty((dims[2], dims[1], dims[0]), dtype=torch.float64, device=dev) if world > 1 else None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    stage_acc = {k: [] for k in _lib.STAGES}
    prepared = eng.prepare_beam(beam)

    def step():
        eng.reset_dose()
        eng.add_beam(prepared)
        eng.read_dose(out)
        if d64 is not None:
            eng.read_dose64(d64)
            with torch.cuda.stream(stream):
                sharding.reduce_dose(d64, dst=0)

    for _ in range(args.warmup):
        step()
        eng.synchronize()
    stats = eng.beam_stats()

    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.25)
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    per_step = []
    t_begin.record(stream)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        per_step.append((e0, e1))
        for k, v in eng.stage_times().items():
            stage_acc[k].append(v)
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in per_step]
    ms = float(np.mean(step_ms))
    total_ms = t_begin.elapsed_time(t_end)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # End to end through the C ABI from pinned host buffers.
    lib = _lib.load()
    ct_pin = torch.from_numpy(np.ascontiguousarray(case["ct"], dtype=np.float32)).pin_memory()
    dose_pin = torch.zeros((dims[2], dims[1], dims[0]), dtype=torch.float32).pin_memory()
    from subsecondpbs_b200.cudaCalDoseRTD import _with_luts

    energy = _with_luts(case["energy"], None)
    bd, kb = _lib.beam_desc(beam)
    ed, ke = _lib.energy_desc(energy)
    fp = C.POINTER(C.c_float)
    ct_ptr = C.cast(C.c_void_p(ct_pin.data_ptr()), fp)
    dose_ptr = C.cast(C.c_void_p(dose_pin.data_ptr()), fp)

    def e2e_call():
        rc = lib.pbs_subsecond_wrapper(ct_ptr, _lib.int3(case["ct_dims"]), _lib.float3(case["ct_resolution"]),
                                       _lib.float3(case["ct_corner"]), dose_ptr, _lib.int3(dims),
                                       _lib.float3(case["dose_resolution"]), _lib.float3(case["dose_corner"]),
                                       C.byref(bd), 1, C.byref(ed), local, 0, 0)
        _lib.check(rc)

    for _ in range(2):
        dose_pin.zero_()
        e2e_call()
    e2e_times = []
    for _ in range(args.e2e_steps):
        # The caller's initial dose (zeros) is prepared outside the timed call.
        dose_pin.zero_()
        t = time.perf_counter()
        e2e_call()
        e2e_times.append((time.perf_counter() - t) * 1e3)
    e2e_ms = float(np.mean(e2e_times))
    copied = (C.c_ulonglong * 2)()
    _lib.check(lib.pbs_wrapper_copy_bytes(copied))
    h2d, d2h = int(copied[0]), int(copied[1])
    if world > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    if rank != 0:
        dist.destroy_process_group()
        return 0

    # Roofline of the dominant kernel (superposition, FP32 pipe) and per-stage HBM figures.
    sup_ms = float(np.mean(stage_acc["superpose"]))
    fma = float(stats["superpose_fma"])
    achieved = 2.0 * fma / (sup_ms * 1e-3) / 1e12
    traffic = None
    tfile = ROOT / "profiles" / "superpose_traffic.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get("dram_bytes_per_beam")
        except (ValueError, OSError):
            traffic = None
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_source = ("MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)" if "hbm_gbs" in peaks
                  else "fallback: 6.65 TB/s, an earlier copy-bandwidth measurement on this pool")
    rays = stats["ray_dims"][0] * stats["ray_dims"][1]
    pad = stats["superp_dims"][0] * stats["superp_dims"][1]
    S = stats["tracer_steps"]
    first = stats["first_inside"]
    idd_steps = sum(max(eng.layer_stats(l)["after_last_step"] - first, 0) for l in range(stats["num_layers"]))
    tb = stats["transfer_start"], stats["transfer_max"]
    box = int(np.prod([max(tb[1][i] - tb[0][i] + 1, 0) for i in range(3)]))
    stage_ms = {k: float(np.mean(v)) for k, v in stage_acc.items()}
    stage_bytes = {
        "trace": 8.0 * rays * S,                      # density + WEPL written
        "idd": 16.0 * pad * idd_steps,                # density + WEPL read, IDD + sigma written
        "transfer": 16.0 * box,                       # FP64 dose read-modify-write over the box
    }
    roof_stages = []
    for k, b in stage_bytes.items():
        if stage_ms[k] > 0:
            gbs = b / (stage_ms[k] * 1e-3) / 1e9
            roof_stages.append({"stage": k, "bound": "hbm", "achieved": round(gbs, 1), "peak": hbm_peak,
                                "unit": "GB/s", "frac": round(gbs / hbm_peak, 4), "algorithmic_bytes": b,
                                "peak_source": hbm_source})

    launches_per_step = int(stats["kernel_launches"]) + 2  # + dose reset and float readout
    cpu = None
    precision = None
    bench_dose = out.cpu().numpy() if world == 1 and not args.no_cpu_baseline else None

    adjoint = _adjoint_cost(local) if world == 1 and not args.no_adjoint else None
    served = (_serving(local, args.serving_requests, args.serving_slots, args.serving_budget_mib)
              if world == 1 and args.serving_requests > 0 else None)
    carbon = carbon_dose = carbon_case = None
    if world == 1 and not args.no_adjoint:
        carbon, carbon_dose, carbon_case = _carbon_plan(local, with_dose=True)
    operator = _operator_export(local) if world == 1 and not args.no_adjoint else None
    reference_gpu = _reference_gpu(local, case, e2e_ms) if world == 1 and not args.no_reference_gpu else None
    upstream_conv = (_upstream_cpu_conv(eng, stats, float(case["beam"]["ray_spacing"][0]), stage_ms["conv"])
                     if world == 1 and not args.no_cpu_baseline else None)
    # The CPU legs run the oracle on every host core: after the timed GPU legs, whose
    # host work they would otherwise share the cores with.
    if bench_dose is not None:
        cms, threads, runs, ref_dose = _cpu_oracle_ms(case)
        cpu = {"value": cms, "unit": "ms", "cores": threads, "kind": "port",
               "sample": f"full workload (one 20-layer beam) x {runs} runs, OpenMP over rays and steps"}
        # Error of the benchmarked result against the FP64 oracle on the same inputs.
        from subsecondpbs_b200 import precision as prec

        precision = dict(prec.report(bench_dose, ref_dose, case["dose_resolution"]),
                         reference="FP64 oracle, same inputs", arithmetic="FP32 rays/superposition, "
                         "int32 fixed-point tile footprints, Kahan WEPL, FP64 dose accumulation")
    if carbon is not None and not args.no_cpu_baseline:
        carbon["precision"] = _carbon_precision(carbon_case, carbon_dose)
    del carbon_dose, carbon_case

    line = {
        "metric": METRIC,
        "value": ms / world,
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": DATA,
        "config": dict(CONFIG),
        "run": {"beams_per_step": world, "parallelism": f"beam-sharded x{world}", "accumulation": "FP64 dose grid",
                "total_ms_incl_flush": total_ms},
        "roofline": {"kernel": "superpose_kernel", "bound": "fp32", "achieved": round(achieved, 3),
                     "peak": round(peak_fp32, 3), "unit": "TFLOP/s", "frac": round(achieved / peak_fp32, 4),
                     "traffic": traffic, "peak_source": "in-run FFMA microbenchmark (FP32 pipe, no tensor cores)",
                     "algorithmic_flops": 2.0 * fma},
        "roofline_stages": roof_stages,
        "stages_ms": stage_ms,
        "cpu_baseline": cpu,
        "cpu_stage_baseline": upstream_conv,
        "precision": precision,
        "adjoint": adjoint,
        "serving": served,
        "carbon_plan": carbon,
        "operator_export": operator,
        "e2e": {"value": e2e_ms / world, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "pbs_subsecond_wrapper (C ABI), pinned host buffers",
                "bytes": "measured by the library (pbs_wrapper_copy_bytes): traced CT box, initial and final dose "
                         "box, beam inputs, strided CT type samples; tables resident after the first call"},
        "reference_gpu": reference_gpu,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "plan": {"ray_dims": stats["ray_dims"], "tracer_steps": S, "live_tiles": stats["live_tiles"],
                 "superpose_fma": stats["superpose_fma"]},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    del kb, ke
    return 0


def main():
    args = _args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
