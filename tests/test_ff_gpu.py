"""GPU parity of the FF sums (achsDtemp / asxDtemp / achDtemp_cor,
FF/ff.cpp:103-451) through the C ABI, against the reference's golden
outputs, the long-double oracle and closed-form known answers.
Tolerance: 1e-12 relative (plain FP64)."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, l2c, rel_err

from bgwsigma import inputs as I
from cases import FF_CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_golden_ff_sigma(bgw, golden, cuda, name):
    f = FF_CASES[name]()
    achs, asx, cor = bgw.ff_sigma(f)
    ref = golden["ff"][name]["reference"]
    orc = golden["ff"][name]["oracle"]
    assert rel_err(achs, l2c(ref["achs"])) < FP64_RTOL
    assert rel_err(asx[:f.nfreqeval], l2c(ref["asx"])) < FP64_RTOL
    assert rel_err(cor[:f.nfreqeval], l2c(ref["cor"])) < FP64_RTOL
    assert rel_err(achs, l2c(orc["achs"])) < FP64_RTOL
    assert rel_err(asx[:f.nfreqeval], l2c(orc["asx"])) < FP64_RTOL
    assert rel_err(cor[:f.nfreqeval], l2c(orc["cor"])) < FP64_RTOL


@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_golden_separate_entry_points(bgw, golden, cuda, name):
    f = FF_CASES[name]()
    ref = golden["ff"][name]["reference"]
    assert rel_err(bgw.achsDtemp_Kernel(f), l2c(ref["achs"])) < FP64_RTOL
    assert rel_err(bgw.asxDtemp_Kernel(f)[:f.nfreqeval], l2c(ref["asx"])) < FP64_RTOL
    assert rel_err(bgw.achDtemp_cor_Kernel(f)[:f.nfreqeval], l2c(ref["cor"])) < FP64_RTOL


def test_uniform_closed_forms(bgw, cuda):
    nb, nv, G, P, F, E = 64, 2, 512, 64, 15, 10
    achs, asx, cor = bgw.ff_sigma(I.ff_uniform(nb, nv, G, P, F, E))
    assert rel_err(achs, -0.125 * (1 + 1j) * nb * P * G) < FP64_RTOL
    assert rel_err(asx, np.full(E, 0.25 * (1 + 1j) * nv * P * G)) < FP64_RTOL
    assert rel_err(cor, np.full(E, -0.25j * 9 * P * G)) < FP64_RTOL


def test_device_memory_matches_host_bitwise(bgw, cuda):
    f = FF_CASES["ff_small_seeded"]()
    h = bgw.ff_sigma(f)
    d = bgw.ff_sigma(bgw.to_device(f, cuda))
    for a, b in zip(h, d):
        assert np.array_equal(a, b.cpu().numpy())


def test_deterministic_reruns(bgw, cuda):
    f = FF_CASES["ff_ragged"]()
    a = bgw.ff_sigma(f)
    for _ in range(3):
        b = bgw.ff_sigma(f)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_bad_index_reported(bgw, cuda):
    f = I.ff_seeded(8, 2, 128, 16, 4, 2, seed=4)
    f.inv_igp_index = f.inv_igp_index.copy()
    f.inv_igp_index[5] = 128          # == len(indinv): out of range
    with pytest.raises(bgw.BgwError) as e:
        bgw.ff_sigma(f)
    assert e.value.status == -2
    g = I.ff_seeded(8, 2, 128, 16, 4, 2, seed=4)
    assert bgw.ff_sigma(g)[0] is not None


def test_zero_eval_points_and_no_valence(bgw, oracle, cuda):
    f = I.ff_seeded(10, 0, 200, 20, 4, 0, seed=6)
    achs, asx, cor = bgw.ff_sigma(f)
    assert rel_err(achs, oracle.achs(f)) < FP64_RTOL


def test_benchmark_size(bgw, oracle, golden, cuda):
    """512 bands, nvband 2, ncouls 8192, ngpown 512, nFreq 15, nfreqeval 10."""
    f = I.ff_seeded(512, 2, 8192, 512, 15, 10, seed=1234)
    d = bgw.to_device(f, cuda)
    achs, asx, cor = bgw.ff_sigma(d)
    assert rel_err(achs.cpu().numpy(), oracle.achs(f)) < FP64_RTOL
    assert rel_err(asx.cpu().numpy(), oracle.asx(f)) < FP64_RTOL
    assert rel_err(cor.cpu().numpy(), oracle.cor(f)) < FP64_RTOL
    # ... and against the reference build's own outputs on the same inputs.
    ref = golden["full"]["ff_benchmark"]["reference"]
    assert rel_err(achs.cpu().numpy(), l2c(ref["achs"])) < FP64_RTOL
    assert rel_err(asx.cpu().numpy()[:f.nfreqeval], l2c(ref["asx"])) < FP64_RTOL
    assert rel_err(cor.cpu().numpy()[:f.nfreqeval], l2c(ref["cor"])) < FP64_RTOL
