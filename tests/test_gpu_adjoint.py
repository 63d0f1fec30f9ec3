"""The spot-weight adjoint (pbs_context_adjoint_beam and the torch.autograd wrapper
around it) against the forward pass, central finite differences of the FP64
objective, and the FP64 gradient of the oracle.

The dose is linear in the spot weights at a fixed set of live rays, so
<G, D(w)> = <K^T G, w> holds for every dose-grid gradient G, and the least-squares
objective is quadratic, which makes its central differences exact up to rounding
for any step. The forward's float atomics make each dose evaluation differ from
the last by a few ulps; the finite-difference bound carries that noise, measured
on two evaluations at the same weights."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms
from subsecondpbs_b200.autograd import plan_dose, spot_counts, with_weights

pytestmark = pytest.mark.gpu

SEED = 20261203


def _engine(case):
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    eng = DoseEngine(0)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    return eng


def _sphere_masks(case, radius_mm, shell_mm):
    dd, res, corner = case["dose_dims"], case["dose_resolution"], case["dose_corner"]
    z, y, x = np.meshgrid(*(corner[i] + res[i] * np.arange(dd[i]) for i in (2, 1, 0)), indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    return r <= radius_mm, (r > radius_mm) & (r <= radius_mm + shell_mm)


def _objective(dose, target, shell, prescription):
    """FP64 least squares: (D - p)^2 over the target, D^2 over the shell."""
    return ((dose[target] - prescription) ** 2).sum() + (dose[shell] ** 2).sum()


def _forward(eng, beams):
    eng.reset_dose()
    for b in beams:
        eng.add_beam(b)
    return eng.read_dose64()


@pytest.mark.parametrize("signed", [False, True])
def test_adjoint_dot_product(hetero_small_case, signed):
    case = hetero_small_case
    eng = _engine(case)
    beam = case["beam"]
    dose = _forward(eng, [beam])
    rng = np.random.Generator(np.random.PCG64(SEED))
    g = rng.standard_normal(dose.shape) if signed else rng.uniform(0.0, 1.0, dose.shape)
    lhs = float((g * dose).sum())
    gw = eng.adjoint_beam(beam, g).astype(np.float64)
    rhs = float(gw @ beam["spot_weights"].astype(np.float64))
    scale = float((np.abs(g) * dose).sum())
    assert scale > 0
    assert abs(lhs - rhs) <= 2e-5 * scale, (lhs, rhs, scale)
    # A device gradient gives the same result as a host one.
    import torch

    gd = torch.from_numpy(g).to("cuda:0")
    gw2 = eng.adjoint_beam(beam, gd).astype(np.float64)
    assert np.abs(gw2 - gw).max() <= 1e-5 * np.abs(gw).max()


def test_adjoint_rotated_beams_dot_product(hetero_small_case):
    """Gantry angles that put the fan at an angle to the dose grid's axes."""
    case = hetero_small_case
    eng = _engine(case)
    rng = np.random.Generator(np.random.PCG64(SEED + 1))
    for angle in (30.0, 135.0):
        beam = phantoms.rotate_beam(case["beam"], angle)
        dose = _forward(eng, [beam])
        g = rng.uniform(-1.0, 1.0, dose.shape)
        lhs = float((g * dose).sum())
        rhs = float(eng.adjoint_beam(beam, g).astype(np.float64) @ beam["spot_weights"].astype(np.float64))
        scale = float((np.abs(g) * dose).sum())
        assert abs(lhs - rhs) <= 2e-5 * scale, (angle, lhs, rhs, scale)


def _scaled_weights(eng, beams, target, prescription):
    dose = _forward(eng, beams)
    s = prescription / float(dose[target].mean())
    return [with_weights(b, b["spot_weights"] * s) for b in beams]


def test_adjoint_finite_differences_inverse_planning():
    """Four beams of about 8000 spots on the water phantom; the objective's gradient
    from torch.autograd against central differences (step 1e-3 of the weight) on
    64 spots."""
    import torch

    case = phantoms.inverse_planning_case()
    target, shell, p = case["target"], case["shell"], case["prescription"]
    eng = _engine(case)
    beams = _scaled_weights(eng, case["beams"], target, p)
    tt = torch.from_numpy(target).to("cuda:0")
    ts = torch.from_numpy(shell).to("cuda:0")

    def objective(w):
        d = plan_dose(w, eng, beams)
        return ((d[tt] - p) ** 2).sum() + (d[ts] ** 2).sum()

    w0 = np.concatenate([b["spot_weights"] for b in beams]).astype(np.float32)
    assert w0.size == sum(spot_counts(beams)) and w0.size >= 4 * 8000
    w = torch.tensor(w0, dtype=torch.float64, device="cuda:0", requires_grad=True)
    j = objective(w)
    j.backward()
    grad = w.grad.detach().cpu().numpy()
    assert np.isfinite(grad).all() and np.abs(grad).max() > 0
    def eval_objective(wnp):
        wd = torch.from_numpy(wnp.astype(np.float64)).to("cuda:0")
        return float(objective(wd))

    with torch.no_grad():
        j0 = float(j)
        # The evaluation is deterministic (fixed-point BEV accumulation): repeated
        # runs agree to the bit.
        assert eval_objective(w0) == eval_objective(w0)
        rng = np.random.Generator(np.random.PCG64(SEED + 2))
        # Its rounding error is not: J(w + v) + J(w - v) - 2 J(w) for a random
        # relative change v of 1e-6 of every weight holds the second-order term
        # (about 1e-12 J, far below FP32 rounding) and the rounding errors of three
        # evaluations (variance 6 sigma^2).
        second = []
        for _ in range(8):
            v = (w0 * rng.uniform(-1e-6, 1e-6, w0.size)).astype(np.float32)
            second.append(eval_objective(w0 + v) + eval_objective(w0 - v) - 2.0 * eval_objective(w0))
        sigma = float(np.sqrt(np.mean(np.square(second)) / 6.0))
        idx = rng.choice(w0.size, 64, replace=False)
        fd = np.empty(idx.size)
        hs = np.empty(idx.size)
        for n, i in enumerate(idx):
            up, dn = w0.copy(), w0.copy()
            up[i] = np.float32(w0[i] * (1.0 + 1e-3))
            dn[i] = np.float32(w0[i] * (1.0 - 1e-3))
            hs[n] = float(up[i]) - float(dn[i])
            fd[n] = (eval_objective(up) - eval_objective(dn)) / hs[n]
    g = grad[idx]
    err = np.abs(fd - g)
    rel = err / np.maximum(np.abs(g), 1e-300)
    # Standard deviation of each central difference from the evaluations' rounding.
    sigma_fd = max(sigma, 1e-13 * j0) * np.sqrt(2.0) / hs
    bound = 1e-3 * np.abs(g) + 6.0 * sigma_fd
    print(f"J={j0:.6g} sigma(J)={sigma:.3g} max|g|={np.abs(g).max():.4g} median rel err={np.median(rel):.3g} "
          f"median sigma_fd/|g|={np.median(sigma_fd / np.abs(g)):.3g} worst err/bound={(err / bound).max():.3g}")
    assert (err <= bound).all(), list(zip(idx[err > bound], fd[err > bound], g[err > bound]))
    assert np.median(rel) < 1e-2


def test_adjoint_matches_fp64_oracle_gradient(hetero_small_case):
    """The FP64 gradient: exact central differences of the oracle's FP64 dose (linear
    in the weights) on a sample of spots, against the library's adjoint."""
    case = hetero_small_case
    target, shell = _sphere_masks(case, 20.0, 20.0)
    eng = _engine(case)
    beam = _scaled_weights(eng, [case["beam"]], target, 2.0)[0]
    w0 = beam["spot_weights"].astype(np.float32)
    d_or = O.dose(case, beams=[beam])["dose"]
    g_dose = np.zeros_like(d_or)
    g_dose[target] = 2.0 * (d_or[target] - 2.0)
    g_dose[shell] = 2.0 * d_or[shell]
    gpu = eng.adjoint_beam(beam, g_dose).astype(np.float64)
    rng = np.random.Generator(np.random.PCG64(SEED + 3))
    idx = np.concatenate([np.argsort(-np.abs(gpu))[:6], rng.choice(w0.size, 10, replace=False)])
    ref = np.empty(idx.size)
    for n, i in enumerate(idx):
        up, dn = w0.copy(), w0.copy()
        up[i] = np.float32(w0[i] * 1.001)
        dn[i] = np.float32(w0[i] * 0.999)
        dp = O.dose(case, beams=[with_weights(beam, up)])["dose"]
        dm = O.dose(case, beams=[with_weights(beam, dn)])["dose"]
        ref[n] = float((g_dose * (dp - dm)).sum()) / (float(up[i]) - float(dn[i]))
    err = np.abs(gpu[idx] - ref)
    scale = np.abs(ref).max()
    print(f"max|g|={scale:.4g} max err/max|g|={err.max() / scale:.3g} "
          f"worst rel err={np.max(err / np.maximum(np.abs(ref), 1e-3 * scale)):.3g}")
    assert scale > 0
    assert (err <= 5e-3 * scale).all(), list(zip(idx, gpu[idx], ref))


def test_adjoint_rejects_legacy_cpb_beams(hetero_small_case):
    """Beams without a spot lattice (the legacy CPB fluence) have no spot-weight
    adjoint: refused with PBS_ERR_UNSUPPORTED before any launch."""
    from subsecondpbs_b200 import _lib as L

    case = hetero_small_case
    eng = _engine(case)
    beam = phantoms.legacy_beam(case["beam"])
    dd = case["dose_dims"]
    with pytest.raises(L.PbsError):
        eng.adjoint_beam(beam, np.zeros((dd[2], dd[1], dd[0])))
