"""Host side of the CarbonPBS-contract entry points (cuFinalDose / calcDose /
cuCalDose / cuCalDose3 / debug_build_carbonpbs_context): argument conversion as
raytracedicom_pybind.cpp does it (no GPU needed)."""
import numpy as np
import pytest

from subsecondpbs_b200 import carbonpbs as cp
from subsecondpbs_b200 import phantoms
from subsecondpbs_b200 import cudaCalDoseRTD


@pytest.fixture(scope="module")
def export():
    case = phantoms.weq_case()
    return case, phantoms.carbonpbs_export(case)


def test_faces_are_exported():
    for name in ("cuFinalDose", "calcDose", "cuCalDose", "cuCalDose3", "debug_build_carbonpbs_context"):
        assert callable(getattr(cudaCalDoseRTD, name))
    assert cudaCalDoseRTD.calcDose is cudaCalDoseRTD.cuFinalDose is cudaCalDoseRTD.cuCalDose


def test_roi_index_forms():
    dims = (4, 5, 6)
    xyz = np.array([[1, 2, 3], [3, 4, 5], [0, 0, 0], [2, 1, 4]], np.int32)
    lin = xyz[:, 0] * 5 * 6 + xyz[:, 1] * 6 + xyz[:, 2]
    assert np.array_equal(cp.roi_linear_indices(xyz, dims), lin)
    assert np.array_equal(cp.roi_linear_indices(xyz.T.copy(), dims), lin)
    assert np.array_equal(cp.roi_linear_indices(xyz.reshape(-1), dims), lin)
    # A flat array whose triplets leave the grid is taken as linear indices.
    flat = np.array([100, 7, 9], np.int32)
    assert np.array_equal(cp.roi_linear_indices(flat, dims), flat)
    assert np.array_equal(cp.roi_linear_indices(np.array([5, 17], np.int32), dims), [5, 17])
    with pytest.raises(RuntimeError, match=r"\(N,3\) or \(3,N\)"):
        cp.roi_linear_indices(np.zeros((2, 4), np.int32), dims)


def test_vector_columns():
    a = np.arange(12, dtype=np.float32).reshape(4, 3)
    assert np.array_equal(cp._columns(a, 3), a.reshape(-1))
    assert np.array_equal(cp._columns(a.T.copy(), 3), a.reshape(-1))
    with pytest.raises(RuntimeError, match="does not match expected count"):
        cp._columns(a, 3, expected=5)
    with pytest.raises(RuntimeError, match="multiple of 2"):
        cp._columns(np.zeros(5, np.float32), 2)


def test_energy_from_idd_table():
    rng = np.random.Generator(np.random.PCG64(5))
    idd = rng.uniform(0.0, 1.0, (3, 50)).astype(np.float32)
    idd[0, 17] = 5.0
    e = cp.energy_from_carbonpbs(np.array([100.0, 150.0, 200.0], np.float32), idd, [2.0, 1.5, 50], tables_dir=None)
    assert np.allclose(e["cidd_matrix"], np.cumsum(idd * np.float32(1.5), axis=1), rtol=1e-6)
    assert np.all(e["scale_facts"] == np.float32(1.0) / np.float32(1.5))
    assert e["peak_depths"][0] == pytest.approx(2.0 + 1.5 * 17)
    assert e["nuclear_tables_aligned_to_primary_axis"]
    assert e["nuc_weight_matrix"].shape == (3, 50)
    # Short steps over a short span are centimetres.
    e = cp.energy_from_carbonpbs([100.0, 150.0, 200.0], idd, [0.0, 0.1, 50], tables_dir=None)
    assert e["scale_facts"][0] == pytest.approx(1.0)
    # A compacted depth axis (logical samples > stored) stretches the step.
    e = cp.energy_from_carbonpbs([100.0, 150.0, 200.0], idd, [0.0, 1.0, 100], tables_dir=None)
    assert e["scale_facts"][0] == pytest.approx(0.5)
    # Fewer IDD rows than energies: the trailing energies (or leading, by env).
    e = cp.energy_from_carbonpbs([90.0, 100.0, 150.0, 200.0], idd, [0.0, 1.0, 50], tables_dir=None)
    assert list(e["energies_per_u"]) == [100.0, 150.0, 200.0]
    with pytest.raises(RuntimeError, match="range"):
        cp.energy_from_carbonpbs([100.0, 150.0], idd, [0.0, 1.0, 50], tables_dir=None)
    with pytest.raises(RuntimeError, match=r"\[start, step, nSamples\]"):
        cp.energy_from_carbonpbs([100.0, 150.0, 200.0], idd, [0.0, 1.0], tables_dir=None)


def test_head_slice_from_environment(monkeypatch):
    idd = np.ones((2, 10), np.float32)
    monkeypatch.setenv("RTD_IDD_SLICE_MODE", "head")
    e = cp.energy_from_carbonpbs([90.0, 100.0, 150.0], idd, [0.0, 1.0, 10], tables_dir=None)
    assert list(e["energies_per_u"]) == [90.0, 100.0]


def test_layer_cutoffs_are_per_layer():
    counts = np.array([2, 3], np.int32)
    assert list(cp._layer_cutoffs(np.array([5, 5, 7, 7, 7], np.float32), counts)) == [5.0, 7.0]
    with pytest.raises(RuntimeError, match="varies within layer 1"):
        cp._layer_cutoffs(np.array([5, 5, 7, 8, 7], np.float32), counts)


def test_subspot_lut_remapped_to_layer_energies():
    lut_e = np.array([100.0, 200.0], np.float32)
    sub = np.zeros((2, 3, 5), np.float32)
    sub[0, :, 3:5] = 4.0
    sub[1, :, 3:5] = 2.0
    sub[0, :, 2] = 1.0
    out, sig = cp._remap_subspots(lut_e, sub, sub[:, 0, 3:5], np.array([150.0, 90.0], np.float32))
    assert np.allclose(sig, [[3.0, 3.0], [4.0, 4.0]])
    assert np.allclose(out[0, :, 2], 0.5)


def test_context_of_an_export(export):
    case, ex = export
    info = cp.debug_build_carbonpbs_context(**ex, tables_dir=None)
    b = case["beam"]
    assert info["rayWeqHeader"] == [float(v) for v in b["water_equivalence"][:9]]
    assert info["totalSpots"] == info["spotPositions"] == info["spotWeights"] == info["spotDirections"] == 93
    assert info["spotPositionsAreIndices"] is True
    assert info["layer_energies"] == [float(v) for v in b["energies"]]
    assert info["energyData_nEnergySamples"] == 400
    ctx = cp.build_carbonpbs_context(**ex, tables_dir=None)
    assert ctx["beam"]["ray_spacing"] == (1.0, 1.0)
    assert ctx["beam"]["steps"] == 64
    assert np.allclose(ctx["beam"]["spot_sigmas"], b["spot_sigmas"])


def test_context_errors(export):
    _, ex = export
    with pytest.raises(RuntimeError, match="9-value CarbonPBS header"):
        cp.build_carbonpbs_context(**dict(ex, rayweq=np.zeros(5, np.float32)), tables_dir=None)
    with pytest.raises(RuntimeError, match="all_energies length must match nPar"):
        cp.build_carbonpbs_context(**dict(ex, all_energies=np.zeros(3, np.float32)), tables_dir=None)
    with pytest.raises(RuntimeError, match="subspotdata must have shape"):
        cp.build_carbonpbs_context(**dict(ex, subspotdata=np.zeros((3, 4), np.float32)), tables_dir=None)
    with pytest.raises(RuntimeError, match="layerEnergy/layerInfo size mismatch"):
        cp.build_carbonpbs_context(**dict(ex, layerEnergy=np.zeros(2, np.float32)), tables_dir=None)
