"""Dose-request serving on one GPU: Python face of the library's server
(pbs_server_*), a replay driver for seeded request streams, and the plain
one-request-at-a-time pipeline the server is measured against.

The server keeps `slots` resident contexts, each with its own CUDA stream and host
thread, and admits queued requests to free slots while their device bytes fit the
HBM budget next to the resident patient CTs and the other slots. Requests of
different patients, sizes and ions therefore run concurrently on the device: one
slot's H2D/D2H copies and host planning overlap the others' kernels.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .cudaCalDoseRTD import _with_luts


class DoseServer:
    """Continuous-batching dose server on GPU `gpu_id` (see include/subsecondpbs.h)."""

    def __init__(self, gpu_id: int = 0, slots: int = 4, hbm_budget_mib: int = 0, bypass_limit_s: float | None = None,
                 nuclear_model: int | None = None, layer_budget_mib: int | None = None, trace_cache: bool = True):
        self._lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self._lib.pbs_server_create(gpu_id, slots, hbm_budget_mib, C.byref(h)))
        self._h = h
        self._patients: dict[int, tuple] = {}
        self._keep: dict[int, object] = {}
        if not trace_cache:
            _lib.check(self._lib.pbs_server_set_trace_cache(self._h, 0))
        if bypass_limit_s is not None:
            _lib.check(self._lib.pbs_server_set_bypass_limit(self._h, float(bypass_limit_s)))
        if nuclear_model is not None:
            _lib.check(self._lib.pbs_server_set_option(self._h, _lib.PBS_OPT_NUCLEAR_MODEL, int(nuclear_model)))
        if layer_budget_mib is not None:
            _lib.check(self._lib.pbs_server_set_option(self._h, _lib.PBS_OPT_LAYER_BUDGET_MIB, int(layer_budget_mib)))

    def close(self) -> None:
        if self._h:
            self._lib.pbs_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_energy(self, energy_id: int, energy: dict, tables_dir: str | None = None) -> None:
        ed, keep = _lib.energy_desc(_with_luts(energy, tables_dir))
        _lib.check(self._lib.pbs_server_add_energy(self._h, int(energy_id), C.byref(ed)))
        del keep

    def add_patient(self, patient_id: int, ct, ct_dims, ct_resolution, ct_corner, dose_dims=None,
                    dose_resolution=None, dose_corner=None) -> None:
        """Registers a patient's CT (copied; any float CT type the wrapper accepts)
        and dose grid (default: the CT grid)."""
        ct = np.ascontiguousarray(ct, dtype=np.float32)
        dd = dose_dims if dose_dims is not None else ct_dims
        dr = dose_resolution if dose_resolution is not None else ct_resolution
        dc = dose_corner if dose_corner is not None else ct_corner
        _lib.check(self._lib.pbs_server_add_patient(
            self._h, int(patient_id), ct.ctypes.data_as(C.POINTER(C.c_float)), _lib.int3(ct_dims),
            _lib.float3(ct_resolution), _lib.float3(ct_corner), _lib.int3(dd), _lib.float3(dr), _lib.float3(dc)))
        self._patients[int(patient_id)] = (int(dd[2]), int(dd[1]), int(dd[0]))

    def add_case_patient(self, patient_id: int, case: dict) -> None:
        self.add_patient(patient_id, case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"],
                         case["dose_dims"], case["dose_resolution"], case["dose_corner"])

    def remove_patient(self, patient_id: int) -> None:
        _lib.check(self._lib.pbs_server_remove_patient(self._h, int(patient_id)))
        self._patients.pop(int(patient_id), None)

    def submit(self, patient_id: int, beams, energy_id: int = 0, nuclear_correction: bool = False) -> int:
        """Queues the dose of `beams` (beam dicts or `prepare_beam` tuples) for the
        patient; returns the request's ticket."""
        descs, keep = [], []
        for b in beams:
            d, k = b if isinstance(b, tuple) else _lib.beam_desc(b)
            descs.append(d)
            keep.append(k)
        arr = (_lib.PbsBeamDesc * len(descs))(*descs)
        t = C.c_ulonglong()
        _lib.check(self._lib.pbs_server_submit(self._h, int(patient_id), int(energy_id), arr, len(descs),
                                               int(bool(nuclear_correction)), C.byref(t)))
        self._keep[t.value] = int(patient_id)
        return t.value

    def wait(self, ticket: int, timeout: float = 120.0, copy: bool = True):
        """(dose float32 [Z][Y][X], {'submit_s', 'start_s', 'done_s', 'slot'}). With
        copy=False the array views the server's buffer, valid until release()."""
        ptr = C.POINTER(C.c_float)()
        times = (C.c_double * 3)()
        slot = C.c_int(-1)
        _lib.check(self._lib.pbs_server_wait(self._h, C.c_ulonglong(ticket), float(timeout), C.byref(ptr), times,
                                             C.byref(slot)))
        shape = self._patients[self._keep[ticket]]
        view = np.ctypeslib.as_array(ptr, shape=shape)
        info = {"submit_s": times[0], "start_s": times[1], "done_s": times[2], "slot": slot.value}
        return (view.copy() if copy else view), info

    def release(self, ticket: int) -> None:
        _lib.check(self._lib.pbs_server_release(self._h, C.c_ulonglong(ticket)))
        self._keep.pop(ticket, None)

    def result(self, ticket: int, timeout: float = 120.0):
        """wait() with a copy of the dose, then release()."""
        dose, info = self.wait(ticket, timeout, copy=True)
        self.release(ticket)
        return dose, info

    def times(self, ticket: int, timeout: float = 120.0) -> dict:
        """The request's phase times (waiting for it first), slot and reserved bytes."""
        ptr = C.POINTER(C.c_float)()
        _lib.check(self._lib.pbs_server_wait(self._h, C.c_ulonglong(ticket), float(timeout), C.byref(ptr), None,
                                             None))
        times = (C.c_double * 4)()
        slot = C.c_int(-1)
        est = C.c_longlong(0)
        _lib.check(self._lib.pbs_server_request_info(self._h, C.c_ulonglong(ticket), times, C.byref(slot),
                                                     C.byref(est)))
        return {"submit_s": times[0], "start_s": times[1], "enqueued_s": times[2], "done_s": times[3],
                "slot": slot.value, "est_bytes": est.value}

    def drain(self, timeout: float = 600.0) -> None:
        _lib.check(self._lib.pbs_server_drain(self._h, float(timeout)))

    def stats(self) -> dict:
        st = _lib.PbsServerStats()
        _lib.check(self._lib.pbs_server_stats(self._h, C.byref(st)))
        return _lib.struct_to_dict(st)

    def now(self) -> float:
        return float(self._lib.pbs_server_now(self._h))


ENERGY_IDS = {"proton": 0, "carbon": 1}


def serve_workload(server: DoseServer, workload: dict, prepared: list, arrivals: bool = True,
                   timeout: float = 600.0, keep: set | None = None) -> dict:
    """Replays `workload["requests"]` against a server holding the workload's
    patients and tables: each request is submitted at its arrival time (or all at
    once with arrivals=False) while a collector thread waits for the results in
    order and releases them (copies are kept for the request indices in `keep`).
    Returns per-request latencies (submit -> done, s), the served plans/s over the
    run (requests / (last done - first submit)) and the kept doses."""
    import queue
    import threading

    reqs = workload["requests"]
    pending: queue.Queue = queue.Queue()
    info: dict[int, dict] = {}
    doses: dict[int, np.ndarray] = {}
    errors: list = []

    def collect():
        while True:
            item = pending.get()
            if item is None:
                return
            i, t = item
            try:
                if keep is not None and i in keep:
                    doses[i], info[i] = server.result(t, timeout)
                else:
                    info[i] = server.times(t, timeout)
                    server.release(t)
            except Exception as ex:  # surfaced after the run
                errors.append((i, ex))

    th = threading.Thread(target=collect, daemon=True)
    th.start()
    t0 = time.perf_counter()
    try:
        for i, (r, beams) in enumerate(zip(reqs, prepared)):
            if arrivals:
                delay = r["arrival_s"] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            t = server.submit(r["patient"], beams, ENERGY_IDS[r["ion"]], nuclear_correction=r["ion"] == "carbon")
            pending.put((i, t))
    finally:
        pending.put(None)
        th.join()
    if errors:
        raise errors[0][1]
    lat = np.array([info[i]["done_s"] - info[i]["submit_s"] for i in range(len(reqs))])
    first = min(v["submit_s"] for v in info.values())
    last = max(v["done_s"] for v in info.values())
    return {"latency_s": lat, "plans_per_s": len(reqs) / (last - first), "wall_s": last - first, "doses": doses,
            "slots": [info[i]["slot"] for i in range(len(reqs))], "info": [info[i] for i in range(len(reqs))]}


def plain_pipeline(workload: dict, prepared: list, gpu_id: int = 0, keep: set | None = None) -> dict:
    """The plain one-request-at-a-time GPU pipeline: every request is one
    pbs_subsecond_wrapper call (CT up, beams, dose down) from pinned host buffers,
    after the previous one returned. Returns per-request service times (s) and
    plans/s = requests / the sum of the call times (host buffer preparation
    between calls is not counted)."""
    import torch

    lib = _lib.load()
    fp = C.POINTER(C.c_float)
    energies = {k: _lib.energy_desc(_with_luts(v, None)) for k, v in workload["energy"].items()}
    cts = {}
    for p in workload["patients"]:
        cts[p["id"]] = torch.from_numpy(np.ascontiguousarray(p["ct"], np.float32)).pin_memory()
    doses = {}
    kept: dict[int, np.ndarray] = {}
    times = []
    for r, beams in zip(workload["requests"], prepared):
        p = workload["patients"][r["patient"]]
        dd = p["dose_dims"]
        key = tuple(dd)
        if key not in doses:
            doses[key] = torch.zeros((dd[2], dd[1], dd[0]), dtype=torch.float32).pin_memory()
        dose = doses[key]
        dose.zero_()
        descs = (_lib.PbsBeamDesc * len(beams))(*[b[0] for b in beams])
        ed = energies[r["ion"]][0]
        t = time.perf_counter()
        rc = lib.pbs_subsecond_wrapper(C.cast(C.c_void_p(cts[p["id"]].data_ptr()), fp), _lib.int3(p["ct_dims"]),
                                       _lib.float3(p["ct_resolution"]), _lib.float3(p["ct_corner"]),
                                       C.cast(C.c_void_p(dose.data_ptr()), fp), _lib.int3(dd),
                                       _lib.float3(p["dose_resolution"]), _lib.float3(p["dose_corner"]), descs,
                                       len(beams), C.byref(ed), gpu_id, int(r["ion"] == "carbon"), 0)
        times.append(time.perf_counter() - t)
        _lib.check(rc)
        if keep is not None and r["index"] in keep:
            kept[r["index"]] = dose.numpy().copy()
    times = np.array(times)
    return {"service_s": times, "plans_per_s": len(times) / float(times.sum()), "doses": kept}


def device_pipeline(workload: dict, prepared: list, gpu_id: int = 0, passes: int = 2) -> dict:
    """The stream's GPU work alone, one request after the other: every request's beams
    and its float dose readout on one resident context per ion (the patient's CT and
    dose grid set outside the timed region when the patient changes), timed with CUDA
    events on the context's stream. Host planning, CT uploads and copies are not in
    the per-request times; plans/s = requests / the sum of those times. The last of
    `passes` passes over the stream is reported (the first grows the buffers)."""
    import torch

    from .cudaCalDoseRTD import DoseEngine

    dev = torch.device("cuda", gpu_id)
    engines: dict[str, DoseEngine] = {}
    current: dict[str, int] = {}
    outs: dict[tuple, torch.Tensor] = {}
    times = []
    for _ in range(passes):
        times = []
        for r, beams in zip(workload["requests"], prepared):
            ion = r["ion"]
            carbon = ion == "carbon"
            eng = engines.get(ion)
            if eng is None:
                eng = engines[ion] = DoseEngine(gpu_id)
                eng.set_energy(workload["energy"][ion])
                current[ion] = -1
            p = workload["patients"][r["patient"]]
            if current[ion] != r["patient"]:
                eng.set_ct(p["ct"], p["ct_dims"], p["ct_resolution"], p["ct_corner"])
                eng.set_dose_grid(p["dose_dims"], p["dose_resolution"], p["dose_corner"])
                eng.synchronize()
                current[ion] = r["patient"]
            dd = tuple(p["dose_dims"])
            if dd not in outs:
                outs[dd] = torch.empty((dd[2], dd[1], dd[0]), dtype=torch.float32, device=dev)
            stream = torch.cuda.ExternalStream(eng.stream_handle, device=dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.reset_dose()
            for b in beams:
                eng.add_beam(b, nuclear_correction=carbon)
            eng.read_dose(outs[dd])
            e1.record(stream)
            eng.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
    for eng in engines.values():
        eng.close()
    times = np.array(times)
    return {"device_s": times, "plans_per_s": len(times) / float(times.sum())}


def with_rate(workload: dict, rate_hz: float) -> dict:
    """The same requests with their Poisson arrival times rescaled to `rate_hz`."""
    f = workload["rate_hz"] / rate_hz
    reqs = [dict(r, arrival_s=r["arrival_s"] * f) for r in workload["requests"]]
    return dict(workload, requests=reqs, rate_hz=rate_hz)


class ServerPool:
    """One DoseServer per GPU of a node. Requests of a patient go to the GPU that
    already holds its CT and traces (the least loaded one at its first request),
    unless that GPU has `spill` more requests in flight than the least loaded one,
    in which case the request goes there and the patient becomes resident on both.
    Tickets are (gpu index, ticket) pairs."""

    def __init__(self, gpu_ids=(0,), slots: int = 8, hbm_budget_mib: int = 0, spill: int = 16, **kw):
        self.servers = [DoseServer(g, slots=slots, hbm_budget_mib=hbm_budget_mib, **kw) for g in gpu_ids]
        self.gpu_ids = list(gpu_ids)
        self.spill = spill
        self._home: dict[int, int] = {}
        self._inflight = [0] * len(self.servers)

    def close(self) -> None:
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_energy(self, energy_id: int, energy: dict, tables_dir: str | None = None) -> None:
        for s in self.servers:
            s.add_energy(energy_id, energy, tables_dir)

    def add_patient(self, patient_id: int, *args, **kw) -> None:
        for s in self.servers:
            s.add_patient(patient_id, *args, **kw)

    def _route(self, patient_id: int) -> int:
        least = min(range(len(self.servers)), key=lambda i: self._inflight[i])
        home = self._home.setdefault(patient_id, least)
        if self._inflight[home] - self._inflight[least] > self.spill:
            return least
        return home

    def submit(self, patient_id: int, beams, energy_id: int = 0, nuclear_correction: bool = False) -> tuple:
        i = self._route(patient_id)
        t = self.servers[i].submit(patient_id, beams, energy_id, nuclear_correction)
        self._inflight[i] += 1
        return (i, t)

    def result(self, ticket: tuple, timeout: float = 120.0):
        i, t = ticket
        try:
            return self.servers[i].result(t, timeout)
        finally:
            self._inflight[i] -= 1

    def stats(self) -> list:
        return [s.stats() for s in self.servers]
