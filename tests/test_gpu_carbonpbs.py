"""The CarbonPBS-contract entry points on the GPU: cuFinalDose (= calcDose =
cuCalDose) and cuCalDose3 give the dose of the converted beam in every output
layout, add onto the caller's dose, and agree with the oracle run on the same
converted inputs."""
import numpy as np
import pytest

from subsecondpbs_b200 import carbonpbs as cp
from subsecondpbs_b200 import phantoms
from subsecondpbs_b200.cudaCalDoseRTD import calcDose, cuCalDose3, cuFinalDose

from _parity import oracle_run
from test_gpu_parity import _dose_checks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def export():
    case = phantoms.weq_case()
    ex = phantoms.carbonpbs_export(case)
    ctx = cp.build_carbonpbs_context(**ex, tables_dir=None)
    return case, ex, ctx


def test_final_dose_layouts_and_accumulation(export):
    case, ex, ctx = export
    nx, ny, nz = ctx["dims"]
    flat = cuFinalDose(np.zeros(nx * ny * nz, np.float32), **ex, tables_dir=None)
    zyx = calcDose(np.zeros((nz, ny, nx), np.float32), **ex, tables_dir=None)
    xyz = cuFinalDose(np.zeros((nx, ny, nz), np.float32), **ex, tables_dir=None)
    ref = zyx.copy()
    assert ref.max() > 0
    scale = float(ref.max())
    assert np.abs(flat.reshape(nz, ny, nx) - ref).max() <= 2e-5 * scale
    assert np.abs(xyz.transpose(2, 1, 0) - ref).max() <= 2e-5 * scale
    # The result is added to what the caller's array holds.
    init = np.full((nz, ny, nx), 0.25 * scale, np.float32)
    acc = cuFinalDose(init, **ex, tables_dir=None)
    assert np.abs(acc - (ref + 0.25 * scale)).max() <= 2e-5 * scale
    with pytest.raises(RuntimeError, match="size does not match dims"):
        cuFinalDose(np.zeros(10, np.float32), **ex, tables_dir=None)
    with pytest.raises(RuntimeError, match="float32"):
        cuFinalDose(np.zeros((nz, ny, nx)), **ex, tables_dir=None)


def test_final_dose_matches_the_oracle_on_the_converted_inputs(export):
    case, ex, ctx = export
    nx, ny, nz = ctx["dims"]
    dose = cuFinalDose(np.zeros((nz, ny, nx), np.float32), **ex, tables_dir=None)
    conv = dict(case, beam=ctx["beam"], energy=ctx["energy"], ct=np.full(nx * ny * nz, 1000.0, np.float32))
    r = oracle_run(conv)
    _dose_checks(dose, r["dose"], case["dose_resolution"])


def _dose3_args(ex, nnz):
    return dict(weq_data=ex["rayweq"], roi_index=ex["roiIdx"], source_energies=ex["all_energies"],
                source=ex["sourcePos"], beam_dir=ex["tmpBeamDir"], beam_xdir=ex["bmxdir"], beam_ydir=ex["bmydir"],
                corner=ex["corner"], resolution=ex["resolution"], dims=ex["dims"], longitudal_cutoff=None,
                enelist=ex["enelist"], idddata=ex["idddata"], iddsetting=ex["iddsetting"], profiledata=None,
                profilesetting=None, beamparadata=None, subspot_data=ex["subspotdata"], layer_info=ex["layerInfo"],
                layer_energy=ex["layerEnergy"], outNNZ=nnz, idbeamxy=ex["idbeamxy"],
                num_particles_per_beam=ex["nPar"], cutoff=None, sad=ex["sad"], beam_para_pos=None,
                python_nnz_size=None, tables_dir=None)


def test_cal_dose3_exports_the_influence_matrix(export):
    """cuCalDose3's sparse outputs hold the spot-preserving influence matrix in the
    CarbonPBS caller's layout (x-major rows, per-column counts after a leading 0):
    weighted by the spot weights it gives the dose grid; a short buffer is left
    unwritten with the needed size in outNNZ."""
    case, ex, ctx = export
    nx, ny, nz = ctx["dims"]
    n_spots = ex["nPar"].size
    nnz = np.zeros(1, np.uint64)
    small = cuCalDose3(np.ones(16, np.float32), np.ones(n_spots + 1, np.int32), np.ones(16, np.int32),
                       **_dose3_args(ex, nnz))
    need = int(nnz[0])
    assert need > 16 and not small["out_cscdata"].any() and not small["out_cscrowind"].any()
    data, rows = np.zeros(need, np.float32), np.zeros(need, np.int32)
    ptr = np.zeros(n_spots + 1, np.int32)
    out = cuCalDose3(data, ptr, rows, **_dose3_args(ex, nnz))
    assert int(nnz[0]) == need and int(ptr.sum()) == need and ptr[0] == 0
    offs = np.cumsum(ptr.astype(np.int64))
    for j in range(0, n_spots, max(1, n_spots // 7)):
        assert np.all(np.diff(rows[offs[j]:offs[j + 1]]) > 0)
    import scipy.sparse as sp

    a = sp.csc_matrix((data, rows, offs), shape=(nx * ny * nz, n_spots))
    dose_xyz = out["dose_grid"]
    ad = (a @ ex["nPar"].astype(np.float64)).reshape(nx, ny, nz)
    dmax = float(dose_xyz.max())
    assert dmax > 0
    assert np.abs(ad - dose_xyz).max() <= 5e-3 * dmax


def test_dose_norm_is_the_row_norm_of_the_influence_matrix(export):
    """cuCalDoseNorm (CarbonPBS) = sum over spots of the squared unit-weight dose at
    each ROI voxel, computed on the device: equal to the squared row norms of the
    matrix cuCalDose3 exports."""
    case, ex, ctx = export
    nx, ny, nz = ctx["dims"]
    n_spots = ex["nPar"].size
    nnz = np.zeros(1, np.uint64)
    cuCalDose3(np.zeros(1, np.float32), np.zeros(n_spots + 1, np.int32), np.zeros(1, np.int32),
               **_dose3_args(ex, nnz))
    need = int(nnz[0])
    data, rows, ptr = np.zeros(need, np.float32), np.zeros(need, np.int32), np.zeros(n_spots + 1, np.int32)
    cuCalDose3(data, ptr, rows, **_dose3_args(ex, nnz))
    import scipy.sparse as sp

    a = sp.csc_matrix((data.astype(np.float64), rows, np.cumsum(ptr.astype(np.int64))),
                      shape=(nx * ny * nz, n_spots))
    want = np.asarray(a.multiply(a).sum(axis=1)).reshape(-1)
    hot = np.flatnonzero(want > 0.05 * want.max())
    roi = np.stack([hot // (ny * nz), (hot // nz) % ny, hot % nz], axis=1).astype(np.int32)
    norm = np.zeros(hot.size, np.float32)
    assert cp.cuCalDoseNorm(norm, ex["rayweq"], roi, ex["all_energies"], ex["sourcePos"], ex["tmpBeamDir"],
                            ex["bmxdir"], ex["bmydir"], ex["corner"], ex["resolution"], ex["dims"], None,
                            ex["enelist"], ex["idddata"], ex["iddsetting"], None, None, None, ex["subspotdata"],
                            ex["layerInfo"], ex["layerEnergy"], ex["idbeamxy"], ex["sad"], None, None,
                            tables_dir=None) == 1
    np.testing.assert_allclose(norm, want[hot], rtol=2e-5)


def test_roi_ct_changes_only_the_geometry_stand_in(export):
    """With an ROI the stand-in CT is water on the ROI and air elsewhere; the WEQ
    volume still carries the transport, so the dose is the same."""
    case, ex, ctx = export
    nx, ny, nz = ctx["dims"]
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    roi = np.stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)], axis=1)[::7].astype(np.int32)
    a = cuFinalDose(np.zeros((nz, ny, nx), np.float32), **ex, tables_dir=None)
    b = cuFinalDose(np.zeros((nz, ny, nx), np.float32), **dict(ex, roiIdx=roi), tables_dir=None)
    assert np.abs(a - b).max() <= 2e-5 * float(a.max())
