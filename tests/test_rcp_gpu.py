"""GPU: accuracy of the reciprocals the kernels use, evaluated by the
library's own device code (bgw_debug_rcp_probe) and compared with the IEEE
reciprocal 1/d (numpy, correctly rounded).

  rcp_refined (FP64 kernels): rcp.approx.ftz.f64 plus one third-order
      Newton-Householder step.  Bar: at most 1 ulp from 1/d for every d whose
      reciprocal is a normal double (2^-1022 <= d <= 2^1022), on 10^6
      log-uniform values and the binade edges.  Outside that range the
      approximation's flush-to-zero shows: a zero or subnormal d gives a
      non-finite result, a d whose reciprocal is subnormal gives 0.  (The
      kernels' denominators |wdiff|^2 never reach those ranges on physical
      inputs; the pole guard's select discards a non-finite reciprocal.)
  rcp.approx.ftz.f32 (mixed remainder): relative error below 2^-22 on the
      remainder's denominator range [(1 - 1/8)^6, (1 + 1/8)^6].
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    return np.abs(a.view(np.int64) - b.view(np.int64))


def test_refined_reciprocal_within_one_ulp(bgw):
    rng = np.random.default_rng(3)
    d = np.exp2(rng.uniform(-1021.0, 1021.0, 1_000_000))
    edges = np.array([2.0 ** k for k in (-1022, -1021, -100, -1, 0, 1, 100, 1021, 1022)])
    edges = np.concatenate([edges, np.nextafter(edges, 0), np.nextafter(edges, np.inf), [3.0, 7.0, 1.0 / 3.0]])
    x = np.concatenate([d, edges[(edges >= 2.0 ** -1022) & (edges <= 2.0 ** 1022)]])
    refined, seed, _ = bgw.rcp_probe(x)
    want = 1.0 / x
    u = _ulps(refined, want)
    assert u.max() <= 1, (u.max(), x[np.argmax(u)])
    exact = float(np.mean(u == 0))
    assert exact > 0.9, exact                                  # mostly correctly rounded
    assert np.max(np.abs(seed / want - 1.0)) < 1e-4           # the starting value's accuracy class


def test_refined_reciprocal_outside_the_normal_range(bgw):
    x = np.array([0.0, 5e-324, 2.0 ** -1030, 2.0 ** 1023, np.nextafter(2.0 ** 1023, np.inf)])
    refined, _, _ = bgw.rcp_probe(x)
    assert not np.isfinite(refined[0]) and not np.isfinite(refined[1]) and not np.isfinite(refined[2])
    assert refined[3] == 0.0 and refined[4] == 0.0           # 1/d subnormal: flushed to zero


def test_f32_reciprocal_on_the_remainder_range(bgw):
    lo, hi = (1 - 0.125) ** 6, (1 + 0.125) ** 6
    x = np.linspace(lo, hi, 200_001)
    _, _, f = bgw.rcp_probe(x)
    xf = x.astype(np.float32).astype(np.float64)
    rel = np.abs(f.astype(np.float64) * xf - 1.0)
    assert rel.max() < 2.0 ** -22, rel.max()
