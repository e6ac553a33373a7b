"""GPU: host-memory calls stage their inputs (pageable buffers through
page-locked slots filled by host threads; the GPP sum's aqsmtemp / aqsntemp
gathered to the columns it reads) -- results must not depend on how the
inputs arrive: pageable, pinned and device-resident inputs give bitwise equal
outputs where the evaluation order is the same, and agree with the oracle."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, rel_err

from bgwsigma import inputs as I

pytestmark = pytest.mark.gpu


def test_ff_pageable_pinned_device_agree(bgw, oracle, cuda):
    # 3 x 512 x 2048 complex per frequency array = 50 MB: above the staging
    # threshold and more than one 32 MiB slot.
    f = I.ff_seeded(40, 2, 2048, 512, 3, 2, seed=31)
    page = bgw.ff_sigma(f)
    pinned = bgw.ff_sigma(bgw.to_pinned(f))
    dev = bgw.ff_sigma(bgw.to_device(f, cuda))
    for a, b, c in zip(page, pinned, dev):
        assert np.array_equal(a, b)
        assert np.array_equal(a, c.cpu().numpy())
    assert rel_err(page[0], oracle.achs(f)) < FP64_RTOL
    assert rel_err(page[2], oracle.cor(f)) < FP64_RTOL


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_gpp_pageable_and_pinned_agree(bgw, oracle, cuda, algorithm):
    # ngpown 409 -> 6 row chunks on the host path; a permuted indinv makes
    # the column gather non-trivial.
    g = I.gpp_seeded(48, 2, 8192, 20, seed=32)
    page = bgw.noflagOCC_solver(g, algorithm=algorithm)
    pinned = bgw.noflagOCC_solver(bgw.to_pinned(g), algorithm=algorithm)
    assert np.array_equal(page, pinned)
    dev = bgw.noflagOCC_solver(bgw.to_device(g, cuda), algorithm=algorithm).cpu().numpy()
    assert rel_err(page, dev) < 1e-13        # device calls use one chunk: another summation order
    assert rel_err(page, oracle.gpp(g)) < FP64_RTOL


def test_gpp_host_gather_reports_bad_index(bgw, cuda):
    g = I.gpp_seeded(8, 2, 4096, 20, seed=33)
    g.inv_igp_index = g.inv_igp_index.copy()
    g.inv_igp_index[3] = len(g.indinv) + 5
    with pytest.raises(bgw.BgwError) as e:
        bgw.noflagOCC_solver(g)
    assert e.value.status == -2
    ok = I.gpp_seeded(8, 2, 4096, 20, seed=33)
    assert np.all(np.isfinite(bgw.noflagOCC_solver(ok)))


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_gpp_repeated_and_unordered_columns(bgw, oracle, cuda, algorithm):
    """inv_igp_index with repeated entries (several G' columns reading the same
    igp) and in no particular order: the host path gathers each column per
    row chunk; host, device and the oracle agree."""
    g = I.gpp_seeded(40, 2, 8192, 20, seed=34)                 # ngpown 409: several row chunks
    rng = np.random.default_rng(35)
    inv = g.inv_igp_index.copy()
    inv[::7] = inv[3]                                          # collisions
    g.inv_igp_index = np.ascontiguousarray(rng.permutation(inv).astype(np.int32))
    ref = oracle.gpp(g)
    host = bgw.noflagOCC_solver(g, algorithm=algorithm)
    assert rel_err(host, ref) < FP64_RTOL
    assert np.array_equal(host, bgw.noflagOCC_solver(bgw.to_pinned(g), algorithm=algorithm))
    dev = bgw.noflagOCC_solver(bgw.to_device(g, cuda), algorithm=algorithm).cpu().numpy()
    assert rel_err(dev, ref) < FP64_RTOL
