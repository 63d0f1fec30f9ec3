"""Dose-influence export (pbs_context_influence_csc) against the forward dose and
the spot-weight adjoint on the same context.

Dose is linear in the spot weights at a fixed set of live rays, so A . w must
reproduce the forward dose of w, and A^T g the adjoint's gradient for any
dose-grid vector g. Tolerance: 0.5 % of Dmax for the dose (the dose tolerance of
the parity tests; the export's float32 values and the forward's few-ulp atomics
noise are far below it); for A^T g, 1e-4 of the largest |A|^T |g|, the summed
magnitude of the terms each gradient entry adds up (a signed g cancels inside the
sums, so the entries themselves are no scale for float32 rounding)."""
import numpy as np
import pytest

from subsecondpbs_b200 import _lib

pytestmark = pytest.mark.gpu

SEED = 20261203
DOSE_TOL = 5e-3


def _engine(case):
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    eng = DoseEngine(0)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    return eng


def _weighted(case):
    beam = dict(case["beam"])
    n = int(np.sum(beam["layer_spot_counts"]))
    rng = np.random.Generator(np.random.PCG64(SEED))
    beam["spot_weights"] = rng.lognormal(0.0, 0.5, n).astype(np.float32)
    return beam, n


def _forward(eng, beam):
    eng.reset_dose()
    eng.add_beam(beam)
    return eng.read_dose64().ravel()


@pytest.fixture(scope="module")
def exported(hetero_small_case):
    eng = _engine(hetero_small_case)
    beam, n = _weighted(hetero_small_case)
    a = eng.influence_csc(beam)
    return eng, beam, n, a


def test_columns_reproduce_the_forward_dose(exported):
    eng, beam, n, a = exported
    assert a.shape == (int(np.prod(eng.dose_dims)), n)
    d = _forward(eng, beam)
    ad = a.astype(np.float64) @ beam["spot_weights"].astype(np.float64)
    dmax = d.max()
    assert dmax > 0
    assert np.abs(ad - d).max() <= DOSE_TOL * dmax
    # Rows ascend strictly inside every column; every stored value passes the threshold (0).
    for j in range(n):
        rows = a.indices[a.indptr[j]:a.indptr[j + 1]]
        assert np.all(np.diff(rows) > 0)
    assert np.all(a.data != 0)


def test_column_is_the_one_hot_forward(exported):
    eng, beam, n, a = exported
    for j in (0, n // 2, n - 1):
        one = dict(beam)
        w = np.zeros(n, dtype=np.float32)
        w[j] = 1.0
        one["spot_weights"] = w
        d = _forward(eng, one)
        col = a[:, j].toarray().ravel()
        scale = max(np.abs(d).max(), 1e-30)
        assert np.abs(col - d).max() <= 1e-5 * scale


def test_transpose_is_the_adjoint(exported):
    eng, beam, n, a = exported
    rng = np.random.Generator(np.random.PCG64(SEED + 1))
    g = rng.standard_normal(tuple(reversed(eng.dose_dims)))
    grad = eng.adjoint_beam(beam, g, n).astype(np.float64)
    atg = a.T.astype(np.float64) @ g.ravel()
    scale = (abs(a).T.astype(np.float64) @ np.abs(g).ravel()).max()
    assert np.abs(atg - grad).max() <= 1e-4 * scale


def test_batches_threshold_and_capacity(exported):
    eng, beam, n, a = exported
    begin, count = n // 3, min(17, n - n // 3)
    part = eng.influence_csc(beam, spot_begin=begin, spot_count=count)
    ref = a[:, begin:begin + count].toarray()
    scale = np.abs(a.data).max()
    assert np.abs(part.toarray() - ref).max() <= 1e-5 * scale
    t = 1e-3 * scale
    cut = eng.influence_csc(beam, threshold=t)
    assert cut.nnz < a.nnz and np.all(np.abs(cut.data) > t)
    assert np.abs(cut.toarray() - np.where(np.abs(a.toarray()) > t, a.toarray(), 0.0)).max() <= t * 1.001
    with pytest.raises(_lib.PbsError, match="capacity"):
        eng.influence_csc(beam, spot_count=2, capacity=1)
    empty = eng.influence_csc(beam, spot_begin=n, spot_count=0)
    assert empty.shape[1] == 0 and empty.nnz == 0
    # The export leaves the accumulator at zero.
    assert not eng.read_dose64().any()


def test_beam_without_a_lattice_is_refused(exported):
    """A spot off the lattice phase leaves the beam without a raw spot lattice; its
    dose would come from the legacy CPB fluence, which ignores per-spot weights, so
    the export refuses it and leaves the dose grid at zero."""
    eng, beam, n, a = exported
    off = dict(beam)
    pos = np.asarray(beam["spot_positions"], np.float32).reshape(-1, 2).copy()
    pos[n // 3, 0] += 0.3
    off["spot_positions"] = pos.reshape(-1)
    with pytest.raises(_lib.PbsError) as e:
        eng.influence_csc(off, spot_count=2)
    assert e.value.code == _lib.PBS_ERR_UNSUPPORTED
    assert "raw spot lattice" in str(e.value)
    assert not np.any(eng.read_dose64())


def test_spot_range_past_the_beam_is_refused(exported):
    eng, beam, n, a = exported
    with pytest.raises(_lib.PbsError) as e:
        eng.influence_csc(beam, spot_begin=n - 1, spot_count=2)
    assert e.value.code == _lib.PBS_ERR_INVALID_ARGUMENT
    with pytest.raises(_lib.PbsError):
        eng.influence_csc(beam, spot_begin=2, spot_count=n)


def test_export_is_bit_identical_across_calls_and_batches(exported):
    # Columns are computed 64 to a pass, each in its own BEV volume and dose buffer,
    # which the pass leaves zero: a second export and a sub-range starting inside a
    # pass reproduce the first bit for bit (the fixed-point superposition is
    # deterministic, the per-column buffers carry nothing over).
    eng, beam, n, a = exported
    assert n > 64
    again = eng.influence_csc(beam)
    assert np.array_equal(again.indptr, a.indptr) and np.array_equal(again.indices, a.indices)
    assert np.array_equal(again.data, a.data)
    for j in (63, 64):
        one = dict(beam)
        w = np.zeros(n, dtype=np.float32)
        w[j] = 1.0
        one["spot_weights"] = w
        d = _forward(eng, one)
        col = a[:, j].toarray().ravel()
        assert np.abs(col - d).max() <= 1e-5 * max(np.abs(d).max(), 1e-30)


def test_export_in_the_reference_depth_convention(hetero_small_case):
    # With the reference's BEV depth indexing each layer is superposed and
    # transferred through the dose grid on its own box, whose depth ends at the last
    # step any live ray of the layer reaches (wrapper.cu:4975-4990, 5343-5394). A
    # spot alone has fewer live rays than its whole layer, so its box can end
    # earlier: the columns are the one-hot forwards of that mode, while their sum
    # need not be the whole beam's dose there.
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    case = hetero_small_case
    eng = DoseEngine(0, compat_bev_z_shift=True)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    beam, n = _weighted(case)
    a = eng.influence_csc(beam)
    assert a.shape[1] == n and a.nnz > 0
    for j in (0, 64, n - 1):
        one = dict(beam)
        w = np.zeros(n, dtype=np.float32)
        w[j] = 1.0
        one["spot_weights"] = w
        d = _forward(eng, one)
        col = a[:, j].toarray().ravel()
        assert d.max() > 0
        assert np.abs(col - d).max() <= 1e-5 * d.max()
    eng.close()
