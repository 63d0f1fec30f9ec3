"""The seeded serving stream: request mix, size classes, spot counts and arrivals."""
import numpy as np

from subsecondpbs_b200 import phantoms, serving

SMALL = (((48, 48, 40), (2.0, 2.0, 2.0)), ((64, 64, 48), (2.0, 2.0, 2.0)), ((80, 80, 40), (2.0, 2.0, 2.0)))


def test_stream_is_seeded_and_mixed():
    a = phantoms.serving_workload(n_requests=400, rate_hz=50.0, patients_per_class=2, ct_classes=SMALL)
    b = phantoms.serving_workload(n_requests=400, rate_hz=50.0, patients_per_class=2, ct_classes=SMALL)
    assert a["requests"] == b["requests"]
    assert all(np.array_equal(pa["ct"], pb["ct"]) for pa, pb in zip(a["patients"], b["patients"]))
    reqs = a["requests"]
    assert {len(r["fields"]) for r in reqs} == {1, 2, 3, 4}
    carbon = np.mean([r["ion"] == "carbon" for r in reqs])
    assert 0.12 < carbon < 0.28
    classes = np.bincount([a["patients"][r["patient"]]["size_class"] for r in reqs], minlength=3)
    assert classes.min() > 0.2 * len(reqs)
    gaps = np.diff([r["arrival_s"] for r in reqs])
    assert abs(gaps.mean() * 50.0 - 1.0) < 0.15
    spots = [f["spots"] for p in a["patients"] for f in p["fields"]]
    assert min(spots) >= 500 and max(spots) <= 20000
    # Request weights are per request; fields are per patient.
    r0 = reqs[0]
    w1 = phantoms.request_beams(a, r0)[0]["spot_weights"]
    w2 = phantoms.request_beams(a, dict(r0, seed=r0["seed"] + 1))[0]["spot_weights"]
    assert w1.shape == w2.shape and not np.array_equal(w1, w2)


def test_rate_rescaling_keeps_the_order():
    w = phantoms.serving_workload(n_requests=50, rate_hz=10.0, patients_per_class=1, ct_classes=SMALL)
    f = serving.with_rate(w, 40.0)
    t0 = np.array([r["arrival_s"] for r in w["requests"]])
    t1 = np.array([r["arrival_s"] for r in f["requests"]])
    assert np.allclose(t1, t0 / 4.0)
    assert [r["patient"] for r in f["requests"]] == [r["patient"] for r in w["requests"]]


def test_heavy_tail():
    rng = np.random.Generator(np.random.PCG64(3))
    n = np.array([phantoms.heavy_tailed_spots(rng) for _ in range(4000)])
    assert n.min() >= 500 and n.max() == 20000
    assert np.median(n) < 1500 and (n > 5000).mean() > 0.03
