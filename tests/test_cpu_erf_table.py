"""Error bound of the superposition's erf table (csrc/superpose.cu): Abramowitz &
Stegun 7.1.26 (|erf error| <= 1.5e-7) with e^{-x^2} carried by a product
recurrence, evaluated here in float32 arithmetic as the kernel does it and
compared with double-precision erf differences."""
import math

import numpy as np

F = np.float32
P = F(0.3275911)
A = [F(v) for v in (0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429)]


def _erf(x, e):
    t = F(1) / (P * x + F(1))
    poly = t * (A[0] + t * (A[1] + t * (A[2] + t * (A[3] + t * A[4]))))
    return F(1) - poly * e


def _table(r, R):
    r = F(r)
    r2 = r * r
    step2 = F(np.exp(F(-2) * r2))
    e_ = F(np.exp(F(-0.25) * r2))
    g = step2
    prev = _erf(r * F(0.5), e_)
    out = [prev]
    for k in range(1, R + 1):
        e_ = F(e_ * g)
        g = F(g * step2)
        f = _erf(r * (F(k) + F(0.5)), e_)
        out.append(F(0.5) * (f - prev))
        prev = f
    return np.array(out, dtype=np.float64)


def _exact(r, R):
    r = float(F(r))
    out = [math.erf(0.5 * r)]
    for k in range(1, R + 1):
        out.append(0.5 * (math.erf(r * (k + 0.5)) - math.erf(r * (k - 0.5))))
    return np.array(out)


def test_erf_table_error_bound():
    worst = 0.0
    for r in np.linspace(0.05, 3.0, 300):
        worst = max(worst, float(np.abs(_table(r, 32) - _exact(r, 32)).max()))
    assert worst < 6e-7, worst


def test_erf_table_normalisation():
    # The symmetric sum e(0) + 2 sum e(k) telescopes to erf((R + 1/2) r).
    for r in (0.07, 0.2, 0.6, 1.5):
        t = _table(r, 32)
        total = t[0] + 2.0 * t[1:].sum()
        assert abs(total - math.erf(r * 32.5)) < 2e-6
