"""GPU: FF asxDtemp / achDtemp_cor with an iw-dependent frequency argument
(BGW_FLAG_FF_WX_PER_IW: wx = freqevalmin - ekq + iw * freqevalstep, one
distinct output per evaluation point) against the oracle's restatement, in
FP64 (1e-12) and mixed precision (1e-9); the iw = 1 entry equals the
reference's value."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, l2c, rel_err

from bgwsigma import inputs as I
from cases import FF_CASES

pytestmark = pytest.mark.gpu

PER_IW = 8
SLICE_ALL = 4
MIXED_FF_RTOL = 1e-9


STAGED = 16


@pytest.mark.parametrize("precision,extra,rtol", [("fp64", 0, FP64_RTOL), ("mixed", 0, MIXED_FF_RTOL),
                                                  ("mixed", SLICE_ALL, MIXED_FF_RTOL),
                                                  ("mixed", STAGED, MIXED_FF_RTOL),
                                                  ("mixed", STAGED | SLICE_ALL, MIXED_FF_RTOL)])
@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_per_iw_vs_oracle(bgw, golden, oracle, cuda, name, precision, extra, rtol):
    f = FF_CASES[name]()
    achs, asx, cor = bgw.ff_sigma(f, precision=precision, flags=PER_IW | extra)
    assert rel_err(achs, oracle.achs(f)) < rtol
    assert rel_err(asx, oracle.asx(f, per_iw=True)) < rtol
    assert rel_err(cor, oracle.cor(f, per_iw=True)) < rtol
    if f.nfreqeval >= 2:
        ref = golden["ff"][name]["reference"]
        assert rel_err(asx[1], l2c(ref["asx"])[1]) < rtol
        assert rel_err(cor[1], l2c(ref["cor"])[1]) < rtol


def test_per_iw_separate_entry_points(bgw, oracle, cuda):
    f = FF_CASES["ff_small_seeded"]()
    assert rel_err(bgw.asxDtemp_Kernel(f, flags=PER_IW), oracle.asx(f, per_iw=True)) < FP64_RTOL
    assert rel_err(bgw.achDtemp_cor_Kernel(f, flags=PER_IW), oracle.cor(f, per_iw=True)) < FP64_RTOL
    assert rel_err(bgw.achsDtemp_Kernel(f, flags=PER_IW), oracle.achs(f)) < FP64_RTOL


@pytest.mark.parametrize("precision,extra,rtol", [("fp64", 0, FP64_RTOL), ("mixed", 0, MIXED_FF_RTOL),
                                                  ("mixed", SLICE_ALL, MIXED_FF_RTOL),
                                                  ("mixed", STAGED | SLICE_ALL, MIXED_FF_RTOL)])
@pytest.mark.parametrize("dims", [(300, 3, 2000, 600, 9, 4), (129, 7, 333, 257, 5, 6), (40, 0, 300, 64, 3, 3)])
def test_per_iw_ragged_shapes(bgw, oracle, cuda, dims, precision, extra, rtol):
    f = I.ff_seeded(*dims, seed=sum(dims) + 1)
    achs, asx, cor = bgw.ff_sigma(f, precision=precision, flags=PER_IW | extra)
    assert rel_err(achs, oracle.achs(f)) < rtol
    assert rel_err(asx, oracle.asx(f, per_iw=True)) < rtol
    assert rel_err(cor, oracle.cor(f, per_iw=True)) < rtol


def test_per_iw_outputs_distinct_and_deterministic(bgw, cuda):
    f = FF_CASES["ff_small_seeded"]()
    a = bgw.ff_sigma(f, flags=PER_IW)
    assert len(np.unique(np.round(a[2], 6))) > 1
    for _ in range(2):
        b = bgw.ff_sigma(f, flags=PER_IW)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_per_iw_device_memory_matches_host(bgw, cuda):
    f = FF_CASES["ff_ragged"]()
    h = bgw.ff_sigma(f, precision="mixed", flags=PER_IW | SLICE_ALL)
    d = bgw.ff_sigma(bgw.to_device(f, cuda), precision="mixed", flags=PER_IW | SLICE_ALL)
    for x, y in zip(h, d):
        assert np.array_equal(x, y.cpu().numpy())


def test_per_iw_fused_out_of_range_units_recomputed(bgw, oracle, cuda):
    """Per-iw outputs through the fused kernel with units that must be
    recomputed in FP64 (first 32 k of some rows scaled down)."""
    f = I.ff_seeded(120, 3, 2500, 260, 7, 5, seed=33)
    f.I_epsR_array = f.I_epsR_array.copy()
    f.I_epsA_array = f.I_epsA_array.copy()
    f.I_epsR_array[:, 50:140, :32] *= 1e-3
    f.I_epsA_array[:, 50:140, :32] *= 1e-3
    achs, asx, cor = bgw.ff_sigma(f, precision="mixed", flags=PER_IW)
    assert rel_err(achs, oracle.achs(f)) < MIXED_FF_RTOL
    assert rel_err(asx, oracle.asx(f, per_iw=True)) < MIXED_FF_RTOL
    assert rel_err(cor, oracle.cor(f, per_iw=True)) < MIXED_FF_RTOL
