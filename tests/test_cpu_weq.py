"""Water-equivalence import in the oracle (fillBevFromWeqVolumeKernel,
raytracedicom_wrapper.cu:1923-1989, and its planning, 3316-3395 and 3566-3640)."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms
from subsecondpbs_b200.cudaCalDoseRTD import plan_beam


@pytest.fixture(scope="module")
def weq():
    return phantoms.weq_case()


def test_header_drives_the_plan(weq):
    b = weq["beam"]
    h = b["water_equivalence"][:9]
    st = plan_beam(b, weq["energy"], weq["ct_dims"], weq["ct_resolution"], weq["ct_corner"], weq["dose_dims"],
                   weq["dose_resolution"], weq["dose_corner"])
    assert st["tracer_steps"] == int(round(h[2]))
    assert abs(st["fan_delta"][2]) == pytest.approx(h[1])
    # The header's origin is the CT start plane: the aligned start is unchanged.
    assert 0.5 * (st["source_dist"][0] + st["source_dist"][1]) - st["fan_corner"][2] == pytest.approx(h[0], abs=1e-3)
    assert st["lattice_dims"] == [int(h[8]), int(h[5])]


def test_oracle_reads_the_imported_depths(weq):
    r = O.dose(weq, capture=True)
    cap = r["capture"]
    pl = cap["plan"]
    h = weq["beam"]["water_equivalence"][:9]
    body = weq["weq"]
    RX, RY = pl["ray_x"], pl["ray_y"]
    xs = pl["cpb_corner"][0] + np.arange(RX) * pl["cpb_res"][0]
    ys = pl["cpb_corner"][1] + np.arange(RY) * pl["cpb_res"][1]
    wx = np.rint((xs - h[6]) / h[7]).astype(int)
    wy = np.rint((ys - h[3]) / h[4]).astype(int)
    inside_x = (wx >= 0) & (wx < body.shape[0])
    inside_y = (wy >= 0) & (wy < body.shape[1])
    want = np.zeros((pl["steps"], RY, RX), np.float32)
    for j in np.nonzero(inside_y)[0]:
        for i in np.nonzero(inside_x)[0]:
            want[:, j, i] = body[wx[i], wy[j], :]
    assert np.array_equal(cap["wepl"].astype(np.float32), want)
    # Entry one step past the first step with material; no entry outside the lattice.
    d = np.diff(np.concatenate([np.zeros((1, RY, RX), np.float32), want], axis=0), axis=0) / h[1]
    mat = d > 1e-4
    first = np.where(mat.any(axis=0), mat.argmax(axis=0) + 1, pl["steps"])
    assert np.array_equal(cap["first_inside"], first)
    assert r["dose"].max() > 0


def test_payload_shorter_than_header_is_refused(weq):
    beam = dict(weq["beam"])
    beam["water_equivalence"] = beam["water_equivalence"][:-1]
    with pytest.raises(RuntimeError, match="smaller than header"):
        O.dose(weq, beams=[beam])
