"""GPU: bgw_noflagOCC_solver_noalloc, the GPP entry point for callers that
cannot allocate GPU memory (all of their device memory belongs to another
runtime or a preallocated pool, or they must never enter the CUDA allocator
because cudaMalloc/cudaFree can synchronise the device).  Its scratch is a
static device array inside the library, so it is checked here against the
regular, workspace-allocating bgw_noflagOCC_solver on two calls in a row
with different shapes: the second call must not see the first call's
leftovers.  This file is collected last and must also pass on its own in a
fresh process."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, rel_err

from bgwsigma import inputs as I

pytestmark = pytest.mark.gpu

NOALLOC_MAX_NGPOWN = 65536  # BGW_NOALLOC_MAX_NGPOWN in include/bgw_sigma.h


def _noalloc(bgw, d, out, stream=None):
    p = bgw._ptr
    return bgw.load().bgw_noflagOCC_solver_noalloc(
        d.number_bands, d.ngpown, d.ncouls, p(d.inv_igp_index), p(d.indinv), len(d.indinv), p(d.wx_array),
        p(d.wtilde_array), p(d.aqsmtemp), p(d.aqsntemp), p(d.I_eps_array), p(d.vcoul), p(out), -1, stream)


def test_noalloc_matches_regular_entry_point_twice_in_a_row(bgw, cuda):
    import torch
    cases = [I.gpp_seeded(64, 2, 2048, 20, seed=1234), I.gpp_seeded(37, 2, 3001, 7, seed=77)]
    dev_inputs = [bgw.to_device(g, cuda) for g in cases]
    expected = [bgw.noflagOCC_solver(d).cpu().numpy() for d in dev_inputs]
    outs = [torch.zeros(3, dtype=torch.complex128, device=cuda) for _ in cases]
    # Two calls in a row on the shared static scratch.
    for d, out in zip(dev_inputs, outs):
        assert _noalloc(bgw, d, out) == 0
    for out, want in zip(outs, expected):
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, want) < FP64_RTOL


def test_noalloc_warm_calls_allocate_nothing(bgw, cuda):
    """After one warm-up call (which may load the module and fetch the
    scratch address), further calls leave the device's free memory and
    torch's allocator untouched: nothing is allocated or freed."""
    import torch
    d = bgw.to_device(I.gpp_seeded(48, 2, 4096, 16, seed=12), cuda)
    out = torch.zeros(3, dtype=torch.complex128, device=cuda)
    assert _noalloc(bgw, d, out) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(5):
        assert _noalloc(bgw, d, out) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_on_a_stream_and_bad_index(bgw, cuda):
    import torch
    g = I.gpp_seeded(16, 2, 1024, 16, seed=8)
    d = bgw.to_device(g, cuda)
    want = bgw.noflagOCC_solver(d).cpu().numpy()
    stream = torch.cuda.Stream()
    out = torch.zeros(3, dtype=torch.complex128, device=cuda)
    torch.cuda.synchronize()
    assert _noalloc(bgw, d, out, stream.cuda_stream) == 0
    assert rel_err(out.cpu().numpy(), want) < FP64_RTOL
    bad = bgw.to_device(g, cuda)
    bad.inv_igp_index = bad.inv_igp_index.clone()
    bad.inv_igp_index[2] = len(g.indinv) + 3
    assert _noalloc(bgw, bad, out) == -2            # BGW_ERR_INDEX, status cleared per call
    assert _noalloc(bgw, d, out) == 0
    assert rel_err(out.cpu().numpy(), want) < FP64_RTOL


def test_noalloc_rejects_ngpown_beyond_scratch(bgw, cuda):
    import torch
    small = bgw.to_device(I.gpp_seeded(2, 1, 40, 20, seed=1), cuda)
    out = torch.zeros(3, dtype=torch.complex128, device=cuda)
    p = bgw._ptr
    st = bgw.load().bgw_noflagOCC_solver_noalloc(
        2, NOALLOC_MAX_NGPOWN + 1, NOALLOC_MAX_NGPOWN + 1, p(small.inv_igp_index), p(small.indinv),
        len(small.indinv), p(small.wx_array), p(small.wtilde_array), p(small.aqsmtemp), p(small.aqsntemp),
        p(small.I_eps_array), p(small.vcoul), p(out), -1, None)
    assert st == -1                                  # rejected on the host, nothing launched
