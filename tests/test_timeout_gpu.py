"""GPU: the timeout path of the kernels that stage their inputs through
bulk copies (GPP band loop FP64 and mixed, both GPP adjoint kernels, the
batched band loop, and the fused FF tensor-core kernel with its 2-CTA
pairs).

bgw_debug_inject_stall(step) makes the bounded wait of CTA-local step `step`
wait on a barrier that nothing ever completes, with a ~0.1 ms budget.  The
wait runs out, the kernel raises BGW_ERR_TIMEOUT, lets the copies still in
flight land (steps `step` and `step + 1`, on the phase each one really
occupies) and exits.  Steps 0 and 3 put the outstanding copies on the even
and the odd phase of the two barriers.  Afterwards the context must still
work: the next call, with the stall off, is bitwise equal to a run made
before the stall, which itself matches the oracle.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from bgwsigma import inputs as I
from conftest import FP64_RTOL, rel_err

pytestmark = pytest.mark.gpu

# 512 bands, ncouls 8192, 585 rows: the FP64 form has 2 band chunks x 4 G
# chunks per row, the mixed form (4096-element chunks, all 512 bands per
# step) 2 G chunks per row; every CTA of either persistent grid gets at
# least 4 steps, so every CTA reaches step 3.
DIMS = dict(number_bands=512, nvband=2, ncouls=8192, nodes_per_group=14)


@pytest.fixture(scope="module")
def gdev(cuda):
    import bgwsigma as bgw
    g = I.gpp_seeded(**DIMS, seed=71)
    assert g.ngpown >= 585
    return g, bgw.to_device(g, cuda)


def _expect_timeout(bgw, fn, step):
    bgw.inject_stall(step)
    try:
        with pytest.raises(bgw.BgwError) as ei:
            fn()
        assert ei.value.status == -6, ei.value  # BGW_ERR_TIMEOUT
    finally:
        bgw.inject_stall(-1)


@pytest.mark.parametrize("step", [0, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bandloop_timeout_then_recovers(bgw, oracle, gdev, step, precision):
    g, d = gdev
    call = lambda: bgw.noflagOCC_solver(d, algorithm="bandloop", precision=precision).cpu().numpy()  # noqa: E731
    before = call()
    if precision == "fp64":
        assert rel_err(before, oracle.gpp(g, factored=True)) < FP64_RTOL
    _expect_timeout(bgw, call, step)
    assert np.array_equal(call(), before)


@pytest.mark.parametrize("step", [0, 3])
def test_adjoint_timeout_then_recovers(bgw, gdev, step):
    g, d = gdev
    gc = [0.3 - 1.1j, 0.7 + 0.2j, -0.4 + 0.9j]

    def call():
        return [x.cpu().numpy() for x in bgw.noflagOCC_solver_backward(d, gc)]
    before = call()
    _expect_timeout(bgw, call, step)
    after = call()
    for a, b in zip(after, before):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("step", [0, 3])
def test_adjoint_bandloop_timeout_then_recovers(bgw, cuda, gdev, step):
    import torch
    g, d = gdev
    shift = np.linspace(-0.2, 0.2, g.number_bands)
    wxb = (np.asarray(g.wx_array)[None, :] + shift[:, None]).astype(np.float64)
    db = dataclasses.replace(d, wx_array=torch.as_tensor(np.ascontiguousarray(wxb), device=cuda), wx_band_stride=3)
    gc = [0.3 - 1.1j, 0.7 + 0.2j, -0.4 + 0.9j]

    def call():
        return [x.cpu().numpy() for x in bgw.noflagOCC_solver_backward(db, gc)]
    before = call()
    _expect_timeout(bgw, call, step)
    after = call()
    for a, b in zip(after, before):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("step", [0, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_timeout_then_recovers(bgw, cuda, step, precision):
    insts = [bgw.to_device(I.gpp_seeded(512, 2, 4096, 20, seed=80 + k), cuda) for k in range(3)]
    b = bgw.GppBatch(insts, algorithm="bandloop", precision=precision)
    before = b.execute().cpu().numpy().copy()
    b.close()
    bgw.inject_stall(step)
    try:
        bs = bgw.GppBatch(insts, algorithm="bandloop", precision=precision)  # the stall is captured here
    finally:
        bgw.inject_stall(-1)
    with pytest.raises(bgw.BgwError) as ei:
        bs.execute()
    assert ei.value.status == -6
    bs.close()
    b2 = bgw.GppBatch(insts, algorithm="bandloop", precision=precision)
    assert np.array_equal(b2.execute().cpu().numpy(), before)
    b2.close()


@pytest.mark.parametrize("step", [0, 3])
@pytest.mark.parametrize("flags", [0, 8])
def test_ff_fused_timeout_then_recovers(bgw, cuda, step, flags):
    """The fused FF kernel: at the stalled stage the MMA thread of both CTAs
    of every pair gives up; the pair's converters, producers and the drain
    then run out of their (short) budgets, every cluster barrier is still
    reached, and the call reports BGW_ERR_TIMEOUT.  The next call (per-iw
    outputs too: flags 8) is bitwise equal to one made before."""
    f = I.ff_seeded(200, 2, 4096, 256, 6, 3, seed=91)
    d = bgw.to_device(f, cuda)

    def call():
        return [x.cpu().numpy() for x in bgw.ff_sigma(d, precision="mixed", flags=flags)]
    before = call()
    _expect_timeout(bgw, call, step)
    for a, b in zip(call(), before):
        assert np.array_equal(a, b)


def test_stall_argument_checked(bgw):
    with pytest.raises(bgw.BgwError):
        bgw.inject_stall(-2)
    bgw.inject_stall(-1)
