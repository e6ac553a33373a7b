"""GPU: bgw_fill_uniform (Philox4x64-10 on the device) gives the same bits as
its host twin (numpy's Philox, bgwsigma.inputs.philox_uniform) for any
offset, length and alignment, into device and host memory; the GPP inputs
generated on the GPU (gpp_philox(device=...)) have the fingerprint of those
generated on the host, for the whole problem and for a G' row block."""
from __future__ import annotations

import numpy as np
import pytest

from bgwsigma import inputs as I
from conftest import FP64_RTOL, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,offset", [(1, 0), (3, 1), (4, 4), (7, 2), (1000, 0), (1001, 3), (65537, 5),
                                      (1 << 20, 123456789)])
def test_device_fill_matches_host_twin(bgw, cuda, n, offset):
    import torch
    want = I.philox_uniform(n, 77, 5, offset, -0.5, 0.5, 0.5, 2.0)
    buf = torch.full((n + 2,), -7.0, dtype=torch.float64, device=cuda)
    bgw.fill_uniform(buf[1:n + 1], 77, 5, offset, -0.5, 0.5, 0.5, 2.0)   # 8-byte aligned start
    got = buf.cpu().numpy()
    assert np.array_equal(got[1:n + 1], want)
    assert got[0] == -7.0 and got[n + 1] == -7.0                        # nothing written outside
    h = np.zeros(n)
    bgw.fill_uniform(h, 77, 5, offset, -0.5, 0.5, 0.5, 2.0)             # host memory: generated on the GPU
    assert np.array_equal(h, want)


def test_large_host_fill_pieces(bgw):
    n = (4 << 20) * 2 + 13                                              # three 32 MiB pieces
    h = np.empty(n)
    bgw.fill_uniform(h, 1, 2, 11, 0.0, 1.0, 0.0, 1.0)
    idx = np.array([0, 1, (4 << 20) - 1, 4 << 20, (8 << 20) + 1, n - 1])
    want = np.array([I.philox_uniform(1, 1, 2, 11 + int(i), 0.0, 1.0, 0.0, 1.0)[0] for i in idx])
    assert np.array_equal(h[idx], want)


def test_gpp_inputs_generated_on_gpu_match_host(bgw, cuda, oracle):
    host = I.gpp_philox(64, 2, 2048, 20, seed=21)
    dev = I.gpp_philox(64, 2, 2048, 20, seed=21, device=cuda)
    assert I.fingerprint(dev.map_arrays(lambda t: t.cpu().numpy())) == I.fingerprint(host)
    blk = I.gpp_philox(64, 2, 2048, 20, seed=21, rows=(17, 60), device=cuda)
    assert np.array_equal(blk.wtilde_array.cpu().numpy(), host.wtilde_array[17:60])
    assert np.array_equal(blk.I_eps_array.cpu().numpy(), host.I_eps_array[17:60])
    got = bgw.noflagOCC_solver(dev, algorithm="bandloop").cpu().numpy()
    assert rel_err(got, oracle.gpp(host, factored=True)) < FP64_RTOL
