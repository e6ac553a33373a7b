"""GPU: mixed-precision FF sums (BGW_PRECISION_MIXED): integer-slice
products on the tcgen05 tensor cores with FP64 recombination, against the
reference's golden outputs (FF/ff.cpp:103-451), the oracle and the FP64
path.  Tolerance: 1e-9 relative."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import l2c, rel_err

from bgwsigma import inputs as I
from cases import FF_CASES

pytestmark = pytest.mark.gpu

MIXED_FF_RTOL = 1e-9
# 0: fused kernel (slices cut inside the tensor-core kernel) for band groups
# of >= 8 rows (the default); 4 (FLAG_FF_SLICE_ALL): for every group;
# 16 (FLAG_FF_STAGED): digit buffers cut first, groups of >= 128 rows;
# 20: staged, every group of more than 16 rows.
ROUTES = [0, 4, 16, 20]


@pytest.mark.parametrize("flags", ROUTES)
@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_golden_ff_sigma_mixed(bgw, golden, cuda, name, flags):
    f = FF_CASES[name]()
    achs, asx, cor = bgw.ff_sigma(f, precision="mixed", flags=flags)
    ref = golden["ff"][name]["reference"]
    assert rel_err(achs, l2c(ref["achs"])) < MIXED_FF_RTOL
    assert rel_err(asx[:f.nfreqeval], l2c(ref["asx"])) < MIXED_FF_RTOL
    assert rel_err(cor[:f.nfreqeval], l2c(ref["cor"])) < MIXED_FF_RTOL


@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_golden_separate_entry_points_mixed(bgw, golden, cuda, name):
    f = FF_CASES[name]()
    ref = golden["ff"][name]["reference"]
    assert rel_err(bgw.achsDtemp_Kernel(f, precision="mixed"), l2c(ref["achs"])) < MIXED_FF_RTOL
    assert rel_err(bgw.asxDtemp_Kernel(f, precision="mixed")[:f.nfreqeval], l2c(ref["asx"])) < MIXED_FF_RTOL
    assert rel_err(bgw.achDtemp_cor_Kernel(f, precision="mixed")[:f.nfreqeval], l2c(ref["cor"])) < MIXED_FF_RTOL


@pytest.mark.parametrize("flags", ROUTES)
def test_uniform_closed_forms_mixed(bgw, cuda, flags):
    nb, nv, G, P, F, E = 64, 2, 512, 64, 15, 10
    achs, asx, cor = bgw.ff_sigma(I.ff_uniform(nb, nv, G, P, F, E), precision="mixed", flags=flags)
    assert rel_err(achs, -0.125 * (1 + 1j) * nb * P * G) < 1e-13
    assert rel_err(asx, np.full(E, 0.25 * (1 + 1j) * nv * P * G)) < 1e-13
    assert rel_err(cor, np.full(E, -0.25j * 9 * P * G)) < 1e-13


# Several 128-row tiles, three 256-column tiles, k not a multiple of 64,
# column count not a multiple of 256, many frequency groups; fewer k than one
# 32-k stage, a column tile with 3 real rows, one stage plus one k.
@pytest.mark.parametrize("flags", ROUTES)
@pytest.mark.parametrize("dims", [(300, 3, 2000, 600, 9, 4), (129, 1, 333, 257, 5, 3), (17, 0, 300, 256, 3, 1),
                                  (200, 2, 5000, 96, 6, 2), (40, 2, 20, 3, 4, 2), (97, 2, 33, 30, 3, 2)])
def test_ragged_shapes_vs_oracle(bgw, oracle, cuda, dims, flags):
    f = I.ff_seeded(*dims, seed=sum(dims))
    achs, asx, cor = bgw.ff_sigma(f, precision="mixed", flags=flags)
    assert rel_err(achs, oracle.achs(f)) < MIXED_FF_RTOL
    if f.nfreqeval:
        assert rel_err(asx, oracle.asx(f)) < MIXED_FF_RTOL
        assert rel_err(cor, oracle.cor(f)) < MIXED_FF_RTOL


@pytest.mark.parametrize("flags", ROUTES)
def test_mixed_close_to_fp64_at_scale(bgw, cuda, flags):
    """512 bands, 512 x 4096 slices, 8 frequencies: mixed vs the FP64 path."""
    import torch
    f = I.ff_seeded(512, 2, 4096, 512, 8, 4, seed=77)
    d = bgw.to_device(f, cuda)
    m = bgw.ff_sigma(d, precision="mixed", flags=flags)
    p = bgw.ff_sigma(d)
    torch.cuda.synchronize()
    for a, b in zip(m, p):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < MIXED_FF_RTOL


def test_deterministic_reruns_mixed(bgw, cuda):
    f = FF_CASES["ff_ragged"]()
    a = bgw.ff_sigma(f, precision="mixed", flags=4)
    for _ in range(3):
        b = bgw.ff_sigma(f, precision="mixed", flags=4)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_device_memory_matches_host_bitwise_mixed(bgw, cuda):
    f = FF_CASES["ff_small_seeded"]()
    h = bgw.ff_sigma(f, precision="mixed", flags=4)
    d = bgw.ff_sigma(bgw.to_device(f, cuda), precision="mixed", flags=4)
    for a, b in zip(h, d):
        assert np.array_equal(a, b.cpu().numpy())


def test_bad_index_reported_mixed(bgw, cuda):
    f = I.ff_seeded(40, 2, 128, 16, 4, 2, seed=4)
    f.inv_igp_index = f.inv_igp_index.copy()
    f.inv_igp_index[5] = 128          # == len(indinv): out of range
    with pytest.raises(bgw.BgwError) as e:
        bgw.ff_sigma(f, precision="mixed", flags=4)
    assert e.value.status == -2
    g = I.ff_seeded(40, 2, 128, 16, 4, 2, seed=4)
    assert bgw.ff_sigma(g, precision="mixed", flags=4)[0] is not None


def _first_block_small(f, rows, factor):
    """Scales k < 32 of the given G' rows of every I_epsR / I_epsA slice by
    `factor`: the fused kernel takes a row's digit scale from the first 32 k
    of each 2048-k unit, so with factor < 1/2 the later values of those rows
    do not fit and their units are recomputed in FP64."""
    f.I_epsR_array = f.I_epsR_array.copy()
    f.I_epsA_array = f.I_epsA_array.copy()
    f.I_epsR_array[:, rows, :32] *= factor
    f.I_epsA_array[:, rows, :32] *= factor
    return f


@pytest.mark.parametrize("flags", [0, 4])
@pytest.mark.parametrize("rows", [slice(0, 1), slice(100, 300), slice(None)])
def test_fused_out_of_range_units_recomputed(bgw, oracle, cuda, flags, rows):
    """Units with a value outside their first-block digit range (one row,
    a band of rows across two column tiles, every row) give the FP64 result
    for exactly those units."""
    f = _first_block_small(I.ff_seeded(90, 2, 3000, 300, 6, 3, seed=21), rows, 1e-3)
    achs, asx, cor = bgw.ff_sigma(f, precision="mixed", flags=flags)
    assert rel_err(achs, oracle.achs(f)) < MIXED_FF_RTOL
    assert rel_err(asx, oracle.asx(f)) < MIXED_FF_RTOL
    assert rel_err(cor, oracle.cor(f)) < MIXED_FF_RTOL


def test_fused_zero_first_block_and_nan(bgw, oracle, cuda):
    """A row whose first block is zero is recomputed in FP64; a NaN in a
    slice reaches the output as in the FP64 path."""
    f = _first_block_small(I.ff_seeded(60, 2, 2500, 140, 5, 2, seed=8), slice(3, 5), 0.0)
    achs, asx, cor = bgw.ff_sigma(f, precision="mixed")
    assert rel_err(achs, oracle.achs(f)) < MIXED_FF_RTOL
    assert rel_err(cor, oracle.cor(f)) < MIXED_FF_RTOL
    g = I.ff_seeded(60, 2, 2500, 140, 5, 2, seed=8)
    g.I_epsR_array = g.I_epsR_array.copy()
    g.I_epsR_array[1, 7, 2100] = np.nan
    m = bgw.ff_sigma(g, precision="mixed")
    p = bgw.ff_sigma(g)
    assert np.isnan(m[0]) == np.isnan(p[0])
    assert np.array_equal(np.isnan(m[2]), np.isnan(p[2]))


def test_fused_matches_staged(bgw, cuda):
    """The fused and staged integer paths agree to the digit truncation."""
    f = I.ff_seeded(256, 2, 4096, 384, 8, 4, seed=5)
    a = bgw.ff_sigma(f, precision="mixed")
    b = bgw.ff_sigma(f, precision="mixed", flags=bgw.FLAG_FF_STAGED | bgw.FLAG_FF_SLICE_ALL)
    for x, y in zip(a, b):
        assert rel_err(x, y) < MIXED_FF_RTOL
