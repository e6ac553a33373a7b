"""CPU: the host twin of bgw_fill_uniform (bgwsigma.inputs.philox_uniform,
numpy's Philox bit generator) against an independent pure-Python
Philox4x64-10 written from the published round function (Salmon, Moraes,
Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), and the
counter-based properties the GPU fill relies on: any offset / sub-block of a
stream is the same values as the whole stream."""
from __future__ import annotations

import numpy as np
import pytest

from bgwsigma import inputs as I

_MASK = (1 << 64) - 1
_M0, _M1 = 0xD2E7470EE14C6C93, 0xCA5A826395121157      # round multipliers
_W0, _W1 = 0x9E3779B97F4A7C15, 0xBB67AE8584CAA73B      # key increments (golden ratio, sqrt(3) - 1)


def _philox4x64_10(ctr, key):
    c, k = list(ctr), list(key)
    for r in range(10):
        if r:
            k = [(k[0] + _W0) & _MASK, (k[1] + _W1) & _MASK]
        p0, p1 = _M0 * c[0], _M1 * c[2]
        c = [(p1 >> 64) ^ c[1] ^ k[0], p1 & _MASK, (p0 >> 64) ^ c[3] ^ k[1], p0 & _MASK]
    return c


def _words(n, seed, stream, offset=0):
    out = []
    for w in range(offset, offset + n):
        out.append(_philox4x64_10([w // 4 + 1, 0, 0, 0], [seed, stream])[w % 4])
    return out


@pytest.mark.parametrize("seed,stream,offset", [(0, 0, 0), (1234, 7, 0), (2**63 + 5, 3, 9), (42, 2**40, 1001)])
def test_host_twin_matches_published_round_function(seed, stream, offset):
    want = np.array(_words(13, seed, stream, offset), dtype=np.uint64)
    bg = np.random.Philox(key=seed + (stream << 64), counter=[offset // 4, 0, 0, 0])
    got = bg.random_raw(13 + offset % 4)[offset % 4:]
    assert np.array_equal(got, want)
    u = I.philox_uniform(13, seed, stream, offset, 0.0, 1.0, 0.0, 1.0)
    assert np.array_equal(u, (want >> np.uint64(11)).astype(np.float64) * 2.0 ** -53)


def test_offsets_and_ranges():
    whole = I.philox_uniform(1 << 12, 9, 1, 0, -1.0, 1.0, 0.5, 2.0)
    for off, n in ((0, 1), (1, 5), (3, 100), (4, 4096 - 4), (1027, 333)):
        assert np.array_equal(I.philox_uniform(n, 9, 1, off, -1.0, 1.0, 0.5, 2.0), whole[off:off + n])
    assert whole[0::2].min() >= -1.0 and whole[0::2].max() < 1.0
    assert whole[1::2].min() >= 0.5 and whole[1::2].max() < 2.0
    # Pieces of the host twin (2^22 words) join without a seam.
    big = I.philox_uniform((1 << 22) + 10, 3, 2, 5, 0.0, 1.0, 0.0, 1.0)
    assert np.array_equal(big[(1 << 22) - 3:], I.philox_uniform(13, 3, 2, 5 + (1 << 22) - 3, 0.0, 1.0, 0.0, 1.0))


def test_gpp_philox_row_blocks_are_slices_of_the_whole():
    g = I.gpp_philox(48, 2, 1500, 15, seed=3)             # ngpown 100
    for p0, p1 in ((0, 100), (0, 1), (37, 64), (99, 100)):
        s = I.gpp_philox(48, 2, 1500, 15, seed=3, rows=(p0, p1))
        assert s.ngpown == p1 - p0
        assert np.array_equal(s.wtilde_array, g.wtilde_array[p0:p1])
        assert np.array_equal(s.I_eps_array, g.I_eps_array[p0:p1])
        assert np.array_equal(s.inv_igp_index, g.inv_igp_index[p0:p1])
        for k in ("aqsmtemp", "aqsntemp", "vcoul", "indinv", "wx_array"):
            assert np.array_equal(getattr(s, k), getattr(g, k))
    w = g.wtilde_array
    assert 0.5 <= w.real.min() and w.real.max() < 2.0 and -0.01 <= w.imag.min() and w.imag.max() < 0.01


def test_gpp_philox_sums_to_oracle_of_shards(oracle):
    # The whole problem's sum equals the sum over row blocks generated alone.
    g = I.gpp_philox(16, 2, 900, 9, seed=8)               # ngpown 100
    parts = [oracle.gpp(I.gpp_philox(16, 2, 900, 9, seed=8, rows=r)) for r in ((0, 33), (33, 34), (34, 100))]
    whole = oracle.gpp(g)
    assert np.max(np.abs(np.sum(parts, axis=0) - whole)) / np.max(np.abs(whole)) < 1e-13
