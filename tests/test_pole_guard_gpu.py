"""GPU: the GPP near-pole guard (bgw_options.pole_guard; not in the
reference, which has no guard, GPP/gpp.cpp:273-274 only clamps wx): terms
with |wx - wtilde| < delta contribute zero.  Checked against the oracle with
the same guard on inputs with planted poles (parity unpinned, the oracle's
guard is itself checked against numpy in test_oracle.py).  Tolerance 1e-12
relative (FP64), 1e-9 (mixed band loop, whose elements near a pole or a cut
are summed in FP64)."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, MIXED_RTOL, rel_err
from test_oracle import near_pole_case

from bgwsigma import inputs as I

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
@pytest.mark.parametrize("delta", [1e-4, 3e-2])
def test_guard_vs_oracle(bgw, oracle, cuda, algorithm, delta):
    g = near_pole_case(seed=21, nb=40, nv=4, G=4096, npg=16)
    got = bgw.noflagOCC_solver(g, algorithm=algorithm, pole_guard=delta)
    assert rel_err(got, oracle.gpp(g, pole_guard=delta)) < FP64_RTOL
    d = bgw.to_device(g, cuda)
    dev = bgw.noflagOCC_solver(d, algorithm=algorithm, pole_guard=delta).cpu().numpy()
    assert rel_err(dev, oracle.gpp(g, pole_guard=delta)) < FP64_RTOL


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_guard_exchange_vs_oracle(bgw, oracle, cuda, algorithm):
    g = near_pole_case(seed=22, nb=24, nv=6, G=2048, npg=8)
    ach, asx = bgw.gpp_sigma(g, algorithm=algorithm, pole_guard=1e-3)
    assert rel_err(asx, oracle.gpp_sx(g, pole_guard=1e-3)) < FP64_RTOL
    assert rel_err(ach, oracle.gpp(g, pole_guard=1e-3)) < FP64_RTOL


def test_guard_band_dependent_wx(bgw, oracle, cuda):
    g = I.gpp_seeded(16, 2, 2048, 8, seed=23, wx_per_band=True)
    g.wx_array = np.ascontiguousarray(g.wx_array - 9.0)      # inside wtilde's range
    got = bgw.noflagOCC_solver(g, pole_guard=2e-2)
    assert rel_err(got, oracle.gpp(g, pole_guard=2e-2)) < FP64_RTOL


def test_guard_mixed(bgw, oracle, cuda):
    g = near_pole_case(seed=24, nb=40, nv=4, G=4096, npg=16)
    got = bgw.noflagOCC_solver(g, algorithm="bandloop", precision="mixed", pole_guard=1e-4)
    assert rel_err(got, oracle.gpp(g, pole_guard=1e-4)) < MIXED_RTOL


def test_mixed_near_poles_without_guard(bgw, oracle, cuda):
    """wx inside wtilde's range, no planted poles: the expansion would not
    converge there; the near elements are summed in FP64 instead."""
    g = I.gpp_seeded(40, 4, 4096, 16, seed=27)
    g.wx_array = np.array([1.0, 1.25, 1.5])
    got = bgw.noflagOCC_solver(g, algorithm="bandloop", precision="mixed")
    assert rel_err(got, oracle.gpp(g)) < MIXED_RTOL
    gb = I.gpp_seeded(24, 2, 2048, 8, seed=28, wx_per_band=True)
    gb.wx_array = np.ascontiguousarray(gb.wx_array - 9.0)
    assert rel_err(bgw.noflagOCC_solver(gb, precision="mixed"), oracle.gpp(gb)) < MIXED_RTOL


def test_batched_mixed_near_poles(bgw, oracle, cuda):
    insts = []
    for k, dims in enumerate([(40, 4, 4096, 16), (7, 2, 1000, 5)]):
        g = I.gpp_seeded(*dims, seed=30 + k)
        g.wx_array = np.array([1.0, 1.25, 1.5])
        insts.append(g)
    b = bgw.GppBatch([bgw.to_device(g, cuda) for g in insts], precision="mixed", algorithm="bandloop")
    out = b.execute().cpu().numpy()
    b.close()
    for k, g in enumerate(insts):
        assert rel_err(out[k], oracle.gpp(g)) < MIXED_RTOL


def test_guard_far_from_poles_changes_nothing(bgw, cuda):
    g = bgw.to_device(I.gpp_seeded(32, 2, 4096, 16, seed=25), cuda)
    for algorithm in ("bandloop", "factored"):
        a = bgw.noflagOCC_solver(g, algorithm=algorithm).cpu().numpy()
        b = bgw.noflagOCC_solver(g, algorithm=algorithm, pole_guard=1e-3).cpu().numpy()
        assert rel_err(b, a) < 1e-14


def test_guard_rejections(bgw, cuda):
    g = I.gpp_seeded(8, 2, 1024, 8, seed=26)
    for bad in (-1e-3, float("nan"), float("inf")):
        with pytest.raises(bgw.BgwError) as e:
            bgw.noflagOCC_solver(g, pole_guard=bad)
        assert e.value.status == -1
    with pytest.raises(bgw.BgwError) as e:
        bgw.noflagOCC_solver_backward(g, np.ones(3, np.complex128), pole_guard=1e-3)
    assert e.value.status == -7
    with pytest.raises(bgw.BgwError) as e:
        bgw.GppBatch([bgw.to_device(g, cuda)], pole_guard=1e-3)
    assert e.value.status == -7
