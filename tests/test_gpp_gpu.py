"""GPU parity of the GPP sum (noflagOCC_solver, GPP/gpp.cpp:307-402) through
the C ABI, against the reference's golden outputs, the long-double oracle and
closed-form known answers.  Tolerance: 1e-12 relative (plain FP64)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
from conftest import MIXED_RTOL, FP64_RTOL, l2c, rel_err

from bgwsigma import inputs as I
from cases import GPP_CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
@pytest.mark.parametrize("name", sorted(GPP_CASES))
def test_golden(bgw, golden, oracle, cuda, name, algorithm):
    g = GPP_CASES[name]()
    got = bgw.noflagOCC_solver(g, algorithm=algorithm)
    assert rel_err(got, l2c(golden["gpp"][name]["reference"])) < FP64_RTOL
    assert rel_err(got, l2c(golden["gpp"][name]["oracle"])) < FP64_RTOL


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_uniform_closed_form(bgw, cuda, algorithm):
    for nb, G, npg in [(64, 2048, 20), (7, 3000, 30)]:
        got = bgw.noflagOCC_solver(I.gpp_uniform(nb, 2, G, npg), algorithm=algorithm)
        assert rel_err(got, I.gpp_uniform_closed_form(nb, G, npg)) < FP64_RTOL


def test_band_dependent_wx(bgw, oracle, cuda):
    # General form: wx[n1][iw] with a band stride (not in the reference).
    for dims in [(40, 1500, 15), (600, 512, 16)]:
        g = I.gpp_seeded(dims[0], 2, dims[1], dims[2], seed=17, wx_per_band=True)
        assert g.wx_band_stride == 3
        got = bgw.noflagOCC_solver(g)
        assert rel_err(got, oracle.gpp(g)) < FP64_RTOL
    with pytest.raises(bgw.BgwError) as e:
        bgw.noflagOCC_solver(g, algorithm="factored")
    assert e.value.status == -7


def test_device_memory_matches_host_bitwise(bgw, cuda):
    import torch
    g = I.gpp_seeded(64, 2, 2048, 20, seed=1234)
    host = bgw.noflagOCC_solver(g)
    dev = bgw.noflagOCC_solver(bgw.to_device(g, cuda))
    torch.cuda.synchronize()
    assert np.array_equal(host, dev.cpu().numpy())


def test_deterministic_reruns(bgw, cuda):
    g = I.gpp_seeded(128, 2, 4096, 16, seed=5)
    a = bgw.noflagOCC_solver(g)
    for _ in range(3):
        assert np.array_equal(a, bgw.noflagOCC_solver(g))
    f = bgw.noflagOCC_solver(g, algorithm="factored")
    assert np.array_equal(f, bgw.noflagOCC_solver(g, algorithm="factored"))


def test_bad_index_reported_and_context_survives(bgw, cuda):
    g = I.gpp_seeded(8, 2, 400, 20, seed=2)
    bad = I.gpp_seeded(8, 2, 400, 20, seed=2)
    bad.inv_igp_index = bad.inv_igp_index.copy()
    bad.inv_igp_index[3] = len(bad.indinv) + 5          # past indinv
    with pytest.raises(bgw.BgwError) as e:
        bgw.noflagOCC_solver(bad)
    assert e.value.status == -2
    bad2 = I.gpp_seeded(8, 2, 400, 20, seed=2)
    bad2.indinv = bad2.indinv.copy()
    bad2.indinv[bad2.inv_igp_index[1]] = -4             # negative G index
    for algorithm in ("bandloop", "factored"):
        with pytest.raises(bgw.BgwError) as e:
            bgw.noflagOCC_solver(bad2, algorithm=algorithm)
        assert e.value.status == -2
    # The next call on the same context is unaffected.
    assert rel_err(bgw.noflagOCC_solver(g), bgw.noflagOCC_solver(g)) == 0.0


def test_empty_bands_and_columns(bgw, cuda):
    g = I.gpp_seeded(0, 0, 64, 8, seed=1)
    assert np.all(bgw.noflagOCC_solver(g) == 0)


@pytest.mark.parametrize("dims", [(0, 0, 512, 8), (5, 2, 64, 128)])   # no bands; no G' columns
@pytest.mark.parametrize("algorithm,precision", [("bandloop", "fp64"), ("factored", "fp64"), ("bandloop", "mixed")])
def test_empty_sums_every_path(bgw, cuda, dims, algorithm, precision):
    """An empty sum is exactly zero on every path, host and device memory,
    and in both outputs of bgw_gpp_sigma."""
    g = I.gpp_seeded(*dims, seed=2)
    for src in (g, bgw.to_device(g, cuda)):
        out = bgw.noflagOCC_solver(src, algorithm=algorithm, precision=precision)
        out = out.cpu().numpy() if hasattr(out, "cpu") else out
        assert np.all(out == 0)
        for o in bgw.gpp_sigma(src, algorithm=algorithm, precision=precision):
            o = o.cpu().numpy() if hasattr(o, "cpu") else o
            assert np.all(o == 0)


def test_async_flag_with_device_status(bgw, oracle, cuda):
    import torch
    g = I.gpp_seeded(16, 2, 1024, 16, seed=8)
    d = bgw.to_device(g, cuda)
    status = torch.full((1,), 99, dtype=torch.int32, device=cuda)
    out = torch.zeros(3, dtype=torch.complex128, device=cuda)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        bgw.noflagOCC_solver(d, out=out, stream=stream.cuda_stream, flags=bgw.FLAG_ASYNC,
                             device_status=status.data_ptr())
    stream.synchronize()
    assert int(status.item()) == 0
    assert rel_err(out.cpu().numpy(), oracle.gpp(g)) < FP64_RTOL


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_benchmark_size(bgw, oracle, golden, cuda, algorithm):
    """512 bands, ncouls 32768, nodes_per_group 20 (ngpown 1638): 2.7e10
    (band, G', G) terms, checked against the long-double oracle's factored
    evaluation (exact algebraic identity for the band-independent wx)."""
    g = I.gpp_seeded(512, 2, 32768, 20, seed=1234)
    ref = oracle.gpp(g, factored=True)
    got = bgw.noflagOCC_solver(bgw.to_device(g, cuda), algorithm=algorithm).cpu().numpy()
    assert rel_err(got, ref) < FP64_RTOL
    # ... and against the reference build's own output on the same inputs.
    assert rel_err(got, l2c(golden["full"]["gpp_benchmark"]["reference"])) < FP64_RTOL


def test_launch_counter_advances(bgw, cuda):
    n0 = bgw.launch_count()
    bgw.noflagOCC_solver(I.gpp_seeded(4, 2, 256, 16))
    assert bgw.launch_count() >= n0 + 3


def test_fp64_peak_probe(bgw, cuda):
    dfma, dmma = bgw.measure_fp64_peak()
    assert 5.0 < dfma < 100.0 and 5.0 < dmma < 100.0


def test_ctypes_invalid_option_struct(bgw, cuda):
    g = I.gpp_seeded(2, 1, 40, 20)
    o = bgw.make_options("host")
    o.struct_size = 4
    out = np.zeros(3, dtype=np.complex128)
    p = bgw._ptr
    st = bgw.load().bgw_noflagOCC_solver(2, 2, 40, p(g.inv_igp_index), p(g.indinv), 41, p(g.wx_array),
                                         p(g.wtilde_array), p(g.aqsmtemp), p(g.aqsntemp), p(g.I_eps_array),
                                         p(g.vcoul), p(out), ctypes.byref(o))
    assert st == -1


# Mixed precision: K = 3 Taylor terms of each step's expansion in FP64, the
# remainder quotients in FP32 (about 1e-7 |t|^3 of a term, |t| <= 1/8), the
# group sums TwoSum-compensated in FP64.  Bar: MIXED_RTOL = 1e-9 relative.


@pytest.mark.parametrize("order,bar", [(0, 2e-6), (1, 1e-7), (2, 1e-8), (3, MIXED_RTOL)])
def test_mixed_order_error_falls_with_k(bgw, oracle, cuda, order, bar):
    """mixed_order K: K hoisted Taylor terms; the FP32 remainder is |t|^K of
    a term.  Band-dependent wx (a shift U[-0.25, 0.25] per band)."""
    g = I.gpp_seeded(256, 2, 8192, 16, seed=19, wx_per_band=True)
    got = bgw.noflagOCC_solver(g, precision="mixed", mixed_order=order)
    assert rel_err(got, oracle.gpp(g)) < bar


def test_mixed_order_checked(bgw, cuda):
    for bad in (-1, 4):
        with pytest.raises(bgw.BgwError) as e:
            bgw.noflagOCC_solver(I.gpp_seeded(4, 2, 256, 16), precision="mixed", algorithm="bandloop",
                                 mixed_order=bad)
        assert e.value.status == -1


@pytest.mark.parametrize("name", ["gpp_small_seeded", "gpp_ragged", "gpp_many_bands", "gpp_small_uniform"])
def test_mixed_precision_golden(bgw, golden, cuda, name):
    g = GPP_CASES[name]()
    got = bgw.noflagOCC_solver(g, precision="mixed")
    assert rel_err(got, l2c(golden["gpp"][name]["reference"])) < MIXED_RTOL


def test_mixed_precision_band_dependent_wx(bgw, oracle, cuda):
    g = I.gpp_seeded(40, 2, 1500, 15, seed=17, wx_per_band=True)
    assert rel_err(bgw.noflagOCC_solver(g, precision="mixed"), oracle.gpp(g)) < MIXED_RTOL


def test_mixed_precision_factored_unsupported(bgw, cuda):
    with pytest.raises(bgw.BgwError) as e:
        bgw.noflagOCC_solver(I.gpp_seeded(4, 2, 256, 16), precision="mixed", algorithm="factored")
    assert e.value.status == -7


def test_mixed_precision_benchmark_size(bgw, oracle, cuda):
    g = I.gpp_seeded(512, 2, 32768, 20, seed=1234)
    got = bgw.noflagOCC_solver(bgw.to_device(g, cuda), precision="mixed").cpu().numpy()
    assert rel_err(got, oracle.gpp(g, factored=True)) < MIXED_RTOL
