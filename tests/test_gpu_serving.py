"""The dose-request server: every result is the same alone and in a concurrent
mix, admission respects the HBM budget (evicting idle patients), and bad
requests are refused at submit."""
import numpy as np
import pytest

from subsecondpbs_b200 import _lib, phantoms, serving

pytestmark = pytest.mark.gpu

# Through the server the dose path is deterministic (fixed-point BEV accumulation,
# one thread per dose voxel in the transfer): a request's dose is the same to the bit
# alone and in a concurrent mix. Against a separate resident context, which traces
# its own packed copy of the CT instead of the server's shared one, the doses agree
# to float rounding.
SAME_TOL = 2e-5

SMALL_CLASSES = (((96, 96, 80), (2.0, 2.0, 2.0)), ((128, 128, 96), (2.0, 2.0, 2.0)))


@pytest.fixture(scope="module")
def workload():
    return phantoms.serving_workload(n_requests=24, rate_hz=400.0, patients_per_class=2, ct_classes=SMALL_CLASSES,
                                     max_spots=3000, carbon_fraction=0.3)


def _server(w, **kw):
    srv = serving.DoseServer(0, **kw)
    srv.add_energy(0, w["energy"]["proton"])
    srv.add_energy(1, w["energy"]["carbon"])
    for p in w["patients"]:
        srv.add_patient(p["id"], p["ct"], p["ct_dims"], p["ct_resolution"], p["ct_corner"])
    return srv


def _alone(w):
    """Every request on its own resident context (no server), one at a time."""
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    out = []
    engines = {}
    for r in w["requests"]:
        p = w["patients"][r["patient"]]
        key = (p["id"], r["ion"])
        if key not in engines:
            eng = DoseEngine(0)
            eng.set_energy(w["energy"][r["ion"]])
            eng.set_ct(p["ct"], p["ct_dims"], p["ct_resolution"], p["ct_corner"])
            eng.set_dose_grid(p["dose_dims"], p["dose_resolution"], p["dose_corner"])
            engines[key] = eng
        eng = engines[key]
        eng.reset_dose()
        for b in phantoms.request_beams(w, r):
            eng.add_beam(b, nuclear_correction=r["ion"] == "carbon")
        out.append(eng.read_dose())
    for e in engines.values():
        e.close()
    return out


def _assert_same(a, b, what):
    scale = max(float(np.abs(b).max()), 1e-30)
    err = float(np.abs(a - b).max()) / scale
    assert err <= SAME_TOL, (what, err)


def test_results_same_alone_and_in_the_mix(workload):
    w = workload
    ref = _alone(w)
    assert all(d.max() > 0 for d in ref)
    prepared = [[_lib.beam_desc(b) for b in phantoms.request_beams(w, r)] for r in w["requests"]]
    with _server(w, slots=4) as srv:
        # All at once: up to four requests on the device together, patients
        # loading while others run.
        mix = serving.serve_workload(srv, w, prepared, arrivals=False, keep=set(range(len(w["requests"]))))
        assert len(set(mix["slots"])) > 1
        for i, d in mix["doses"].items():
            _assert_same(d, ref[i], ("mix", i))
        # One at a time through the same server: bit for bit the mix's result.
        for i, (r, beams) in enumerate(zip(w["requests"], prepared)):
            t = srv.submit(r["patient"], beams, serving.ENERGY_IDS[r["ion"]], r["ion"] == "carbon")
            d, _ = srv.result(t)
            _assert_same(d, ref[i], ("alone", i))
            assert np.array_equal(d, mix["doses"][i]), ("alone vs mix", i)
        st = srv.stats()
        assert st["failed"] == 0 and st["completed"] == 2 * len(w["requests"])
        assert st["patient_loads"] == len(w["patients"])  # loaded once, then resident
        # Every field geometry (the ion changes the ray grid and the steps) is traced
        # once; later beams reuse the resident trace.
        n_fields = len({(r["patient"], f, r["ion"]) for r in w["requests"] for f in r["fields"]})
        n_beams = sum(len(r["fields"]) for r in w["requests"])
        assert st["trace_loads"] == n_fields
        assert st["trace_hits"] == 2 * n_beams - n_fields


def test_poisson_arrivals_overlap_on_the_device(workload):
    w = workload
    prepared = [[_lib.beam_desc(b) for b in phantoms.request_beams(w, r)] for r in w["requests"]]
    with _server(w, slots=3) as srv:
        res = serving.serve_workload(srv, w, prepared, arrivals=True)
    assert res["plans_per_s"] > 0 and np.all(res["latency_s"] > 0)


@pytest.mark.parametrize("trace_cache", [False, True])
def test_budget_evicts_idle_patients(workload, trace_cache):
    w = workload
    prepared = [[_lib.beam_desc(b) for b in phantoms.request_beams(w, r)] for r in w["requests"]]
    ref = _alone(w)
    ct_all = sum(int(np.prod(p["ct_dims"])) * 4 for p in w["patients"])
    ct_max = max(int(np.prod(p["ct_dims"])) * 4 for p in w["patients"])
    with _server(w, slots=1, trace_cache=trace_cache) as probe:
        serving.serve_workload(probe, w, prepared, arrivals=False)
        st0 = probe.stats()
    per_slot = st0["slot_bytes"]  # the slot grown to the largest request
    traces_all = st0["resident_bytes"] - ct_all
    # One slot and room for the largest request plus part of the CTs and traces.
    if trace_cache:
        budget = per_slot + ct_all + 0.5 * traces_all
    else:
        budget = per_slot + 1.6 * ct_max
    with _server(w, slots=1, hbm_budget_mib=int(np.ceil(budget / 2**20)), trace_cache=trace_cache) as srv:
        res = serving.serve_workload(srv, w, prepared, arrivals=False, keep=set(range(len(w["requests"]))))
        st = srv.stats()
    for i, d in res["doses"].items():
        _assert_same(d, ref[i], ("budget", i))
    if trace_cache:
        assert st["trace_evictions"] > 0 and st["trace_loads"] > st0["trace_loads"], st
    else:
        assert st["evictions"] > 0 and st["patient_loads"] > len(w["patients"]), st
    assert st["peak_bytes"] <= st["budget_bytes"], st


def test_submit_refuses_bad_requests(workload):
    w = workload
    beams = phantoms.request_beams(w, w["requests"][0])
    with _server(w, slots=1, hbm_budget_mib=8) as srv:
        with pytest.raises(_lib.PbsError) as ex:
            srv.submit(999, beams, 0)
        assert ex.value.code == _lib.PBS_ERR_INVALID_ARGUMENT
        with pytest.raises(_lib.PbsError) as ex:
            srv.submit(w["requests"][0]["patient"], beams, 7)
        assert ex.value.code == _lib.PBS_ERR_INVALID_ARGUMENT
        # 8 MiB holds neither the dose grid nor the CT of this request.
        big = max(w["patients"], key=lambda p: int(np.prod(p["ct_dims"])))
        with pytest.raises(_lib.PbsError) as ex:
            srv.submit(big["id"], [big["fields"][0]["proton"]], 0)
        assert ex.value.code == _lib.PBS_ERR_OUT_OF_MEMORY
        assert srv.stats()["submitted"] == 0


def test_a_failing_request_does_not_stop_the_server(workload):
    """A carbon request with the halo against tables that carry no halo tables
    passes submit, fails on its slot with PBS_ERR_UNSUPPORTED, and the requests
    around it complete."""
    w = workload
    r0 = w["requests"][0]
    beams = phantoms.request_beams(w, r0)
    with _server(w, slots=2) as srv:
        ok1 = srv.submit(r0["patient"], beams, 0)
        bad = srv.submit(r0["patient"], beams, 0, nuclear_correction=True)  # proton tables: no halo tables
        ok2 = srv.submit(r0["patient"], beams, 0)
        d1, _ = srv.result(ok1)
        with pytest.raises(_lib.PbsError) as ex:
            srv.result(bad)
        assert ex.value.code == _lib.PBS_ERR_UNSUPPORTED
        srv.release(bad)
        d2, _ = srv.result(ok2)
        _assert_same(d2, d1, "around a failure")
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == 2


def test_patients_are_removed_only_when_idle(workload):
    w = workload
    r0 = w["requests"][0]
    with _server(w, slots=1) as srv:
        t = srv.submit(r0["patient"], phantoms.request_beams(w, r0), 0)
        srv.drain()
        srv.remove_patient(r0["patient"])
        with pytest.raises(_lib.PbsError):
            srv.submit(r0["patient"], phantoms.request_beams(w, r0), 0)
        srv.release(t)
        assert srv.stats()["resident_bytes"] >= 0


def test_server_pool_keeps_patients_home_and_results_unchanged(workload):
    """Two servers (both on GPU 0 here; one per GPU on a node): a patient's requests
    stay on the server holding its CT, and the results are the requests' doses."""
    w = workload
    ref = _alone(w)
    with serving.ServerPool(gpu_ids=(0, 0), slots=2) as pool:
        pool.add_energy(0, w["energy"]["proton"])
        pool.add_energy(1, w["energy"]["carbon"])
        for p in w["patients"]:
            pool.add_patient(p["id"], p["ct"], p["ct_dims"], p["ct_resolution"], p["ct_corner"])
        tickets = [pool.submit(r["patient"], phantoms.request_beams(w, r), serving.ENERGY_IDS[r["ion"]],
                               r["ion"] == "carbon") for r in w["requests"]]
        for i, t in enumerate(tickets):
            d, _ = pool.result(t)
            _assert_same(d, ref[i], ("pool", i))
        homes = {}
        for r, (g, _) in zip(w["requests"], tickets):
            homes.setdefault(r["patient"], set()).add(g)
        assert all(len(v) == 1 for v in homes.values())
        st = pool.stats()
        assert sum(s["completed"] for s in st) == len(w["requests"])
        assert min(s["completed"] for s in st) > 0
