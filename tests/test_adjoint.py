"""Adjoint of the GPP sum (bgw_noflagOCC_solver_backward).

CPU: the long-double oracle gradient is pinned by central finite differences
(h = 1e-6) of the long-double forward on 64 seeded entries of wtilde_array and
of I_eps_array (including every (p, igp) entry, where wtilde also enters
sch_store1) and on the frequencies.
GPU: the CUDA adjoint matches the oracle gradient to 1e-12 (normwise) at small
and benchmark sizes, and central differences to 1e-6 on 64 seeded entries.
A band-dependent wx takes the band-loop adjoint, checked the same way against
the oracle's band-loop gradient and long-double band-loop forward."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import rel_err

from bgwsigma import inputs as I

H = 1e-6
FD_RTOL = 1e-6


def _fwd(orc, g):
    """Long-double forward: factored for a shared wx, the band loop for a
    band-dependent one."""
    return orc.gpp_direct_ld(g) if g.wx_band_stride else orc.gpp_ld(g)


def _loss(orc, g, gcot) -> np.longdouble:
    s = _fwd(orc, g)
    gc = np.asarray(gcot, dtype=np.complex128)
    return np.longdouble(sum(np.longdouble(gc[i].real) * s[2 * i] + np.longdouble(gc[i].imag) * s[2 * i + 1]
                             for i in range(3)))


def _entries(g, n, rng):
    P, G = g.ngpown, g.ncouls
    igp = g.indinv[g.inv_igp_index]
    ent = [(p, int(igp[p])) for p in rng.choice(P, size=min(n // 4, P), replace=False)]
    while len(ent) < n:
        ent.append((int(rng.integers(P)), int(rng.integers(G))))
    return ent


def _fd(orc, g, gcot, name, p, ig):
    """(dL/dRe z, dL/dIm z) by central differences of the long-double forward."""
    arr = getattr(g, name)
    out = []
    for comp in (0, 1):
        v = arr.view(np.float64).reshape(arr.shape + (2,))
        x0 = v[p, ig, comp]
        v[p, ig, comp] = x0 + H
        xp = v[p, ig, comp]
        lp = _loss(orc, g, gcot)
        v[p, ig, comp] = x0 - H
        xm = v[p, ig, comp]
        lm = _loss(orc, g, gcot)
        v[p, ig, comp] = x0
        out.append(float((lp - lm) / (np.longdouble(xp) - np.longdouble(xm))))
    return complex(out[0], out[1])


def _fd_domega(orc, g, gcot):
    """d achtemp[iw] / d omega (complex) by central differences, omega
    shifting wx[iw] (every band's, for a band-dependent wx)."""
    wx0 = g.wx_array.copy()
    col = (lambda iw: (slice(None), iw)) if g.wx_band_stride else (lambda iw: iw)
    if g.wx_band_stride:
        assert g.wx_band_stride == 3 and wx0.ndim == 2
    res = []
    for iw in range(3):
        g.wx_array[...] = wx0
        g.wx_array[col(iw)] = wx0[col(iw)] + H
        sp = _fwd(orc, g)
        g.wx_array[col(iw)] = wx0[col(iw)] - H
        sm = _fwd(orc, g)
        g.wx_array[...] = wx0
        den = np.longdouble(2 * H)
        res.append(complex(float((sp[2 * iw] - sm[2 * iw]) / den), float((sp[2 * iw + 1] - sm[2 * iw + 1]) / den)))
    return np.array(res)


def _check_fd(orc, g, gcot, grads, entries):
    gw, gi, dw = grads
    for name, grad in (("wtilde_array", gw), ("I_eps_array", gi)):
        for p, ig in entries:
            fd = _fd(orc, g, gcot, name, p, ig)
            an = complex(grad[p, ig])
            assert abs(an - fd) <= FD_RTOL * abs(an) + 1e-300, (name, p, ig, an, fd)
    fdw = _fd_domega(orc, g, gcot)
    assert rel_err(dw, fdw) < FD_RTOL


def test_oracle_gradient_matches_finite_differences(oracle):
    rng = np.random.default_rng(7)
    g = I.gpp_seeded(16, 2, 512, 8, seed=41)           # ngpown 64
    gcot = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    grads = oracle.gpp_backward(g, gcot)
    _check_fd(oracle, g, gcot, grads, _entries(g, 64, rng))


def test_oracle_band_loop_gradient_matches_finite_differences(oracle):
    """Band-dependent wx: the oracle's band-loop gradient against central
    differences of its long-double band-loop forward."""
    rng = np.random.default_rng(8)
    g = I.gpp_seeded(8, 2, 256, 8, seed=43, wx_per_band=True)   # ngpown 32
    gcot = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    grads = oracle.gpp_backward(g, gcot)
    _check_fd(oracle, g, gcot, grads, _entries(g, 32, rng))


def test_oracle_band_loop_gradient_equals_factored_for_shared_wx(oracle):
    g = I.gpp_seeded(12, 2, 600, 6, seed=44)
    gcot = np.array([0.3 - 1.1j, 0.7 + 0.2j, -0.4 + 0.9j])
    for a, b in zip(oracle.gpp_backward(g, gcot), oracle.gpp_backward(g, gcot, direct=True)):
        assert rel_err(b, a) < 1e-15


def test_oracle_gradient_linear_in_cotangent(oracle):
    g = I.gpp_seeded(8, 2, 256, 8, seed=42)
    a = oracle.gpp_backward(g, [1, 0, 0])
    b = oracle.gpp_backward(g, [0, 1j, 0])
    c = oracle.gpp_backward(g, [1, 1j, 0])
    for x, y, z in zip(a[:2], b[:2], c[:2]):
        assert np.allclose(x + y, z, rtol=1e-13, atol=0)
    # d achtemp / d wx does not depend on the cotangent.
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[2], c[2])


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(16, 512, 8), (64, 2048, 20), (3, 1000, 7)])
def test_gpu_adjoint_matches_oracle(bgw, oracle, cuda, dims):
    rng = np.random.default_rng(dims[1])
    g = I.gpp_seeded(dims[0], 2, dims[1], dims[2], seed=dims[1] + 1)
    gcot = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    got = bgw.noflagOCC_solver_backward(g, gcot)
    ref = oracle.gpp_backward(g, gcot)
    for a, b in zip(got, ref):
        assert rel_err(a, b) < 1e-12


@pytest.mark.gpu
def test_gpu_adjoint_finite_differences(bgw, oracle, cuda):
    rng = np.random.default_rng(11)
    g = I.gpp_seeded(64, 2, 4096, 20, seed=12)         # ngpown 204
    gcot = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    grads = bgw.noflagOCC_solver_backward(g, gcot)
    _check_fd(oracle, g, gcot, grads, _entries(g, 64, rng))


@pytest.mark.gpu
def test_gpu_adjoint_device_matches_host_and_reruns(bgw, cuda):
    g = I.gpp_seeded(32, 2, 2048, 16, seed=13)
    gcot = np.array([1 + 2j, -0.5j, 0.25])
    h = bgw.noflagOCC_solver_backward(g, gcot)
    d = bgw.noflagOCC_solver_backward(bgw.to_device(g, cuda), gcot)
    for a, b in zip(h, d):
        assert np.array_equal(a, b.cpu().numpy())
    h2 = bgw.noflagOCC_solver_backward(g, gcot)
    for a, b in zip(h, h2):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_gpu_adjoint_benchmark_size(bgw, oracle, cuda):
    """512 bands, ncouls 32768, nodes_per_group 20: gradients over the full
    wtilde_array / I_eps_array [1638][32768] against the oracle."""
    g = I.gpp_seeded(512, 2, 32768, 20, seed=1234)
    gcot = np.array([0.3 - 1.1j, 0.7 + 0.2j, -0.4 + 0.9j])
    gw, gi, dw = (x.cpu().numpy() for x in bgw.noflagOCC_solver_backward(bgw.to_device(g, cuda), gcot))
    rw, ri, rd = oracle.gpp_backward(g, gcot)
    assert rel_err(gw, rw) < 1e-12
    assert rel_err(gi, ri) < 1e-12
    assert rel_err(dw, rd) < 1e-12


# ----------------------------------------------- band-loop adjoint (GPU) --

@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(16, 512, 8), (300, 1000, 10), (5, 777, 3)])
def test_gpu_band_loop_adjoint_matches_oracle(bgw, oracle, cuda, dims):
    """Band-dependent wx (the band-loop adjoint); 300 bands span two staged
    band chunks, ncouls not a multiple of the 512-element item."""
    rng = np.random.default_rng(dims[0])
    g = I.gpp_seeded(dims[0], 2, dims[1], dims[2], seed=dims[0] + 5, wx_per_band=True)
    gcot = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    got = bgw.noflagOCC_solver_backward(g, gcot)
    ref = oracle.gpp_backward(g, gcot)
    for a, b in zip(got, ref):
        assert rel_err(a, b) < 1e-12


@pytest.mark.gpu
def test_gpu_band_loop_adjoint_finite_differences(bgw, oracle, cuda):
    rng = np.random.default_rng(21)
    g = I.gpp_seeded(8, 2, 256, 8, seed=22, wx_per_band=True)
    gcot = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    grads = bgw.noflagOCC_solver_backward(g, gcot)
    _check_fd(oracle, g, gcot, grads, _entries(g, 32, rng))


@pytest.mark.gpu
def test_gpu_band_loop_adjoint_equals_factored_for_shared_wx(bgw, cuda):
    g = bgw.to_device(I.gpp_seeded(48, 2, 4096, 16, seed=23), cuda)
    gcot = np.array([0.3 - 1.1j, 0.7 + 0.2j, -0.4 + 0.9j])
    a = bgw.noflagOCC_solver_backward(g, gcot)
    b = bgw.noflagOCC_solver_backward(g, gcot, algorithm="bandloop")
    for x, y in zip(a, b):
        assert rel_err(y.cpu().numpy(), x.cpu().numpy()) < 1e-12


@pytest.mark.gpu
def test_gpu_band_loop_adjoint_host_device_and_reruns(bgw, cuda):
    g = I.gpp_seeded(20, 2, 2048, 16, seed=24, wx_per_band=True)
    gcot = np.array([1 + 2j, -0.5j, 0.25])
    h = bgw.noflagOCC_solver_backward(g, gcot)
    d = bgw.noflagOCC_solver_backward(bgw.to_device(g, cuda), gcot)
    for a, b in zip(h, d):
        assert np.array_equal(a, b.cpu().numpy())
    for a, b in zip(h, bgw.noflagOCC_solver_backward(g, gcot)):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_gpu_band_loop_adjoint_no_bands(bgw, cuda):
    g = I.gpp_seeded(4, 2, 512, 8, seed=25, wx_per_band=True)
    g.number_bands = 0
    g.aqsmtemp = g.aqsmtemp[:0]
    g.aqsntemp = g.aqsntemp[:0]
    g.wx_array = np.ascontiguousarray(g.wx_array[:1])
    gw, gi, dw = bgw.noflagOCC_solver_backward(g, [1, 1j, 0])
    assert not gw.any() and not gi.any() and not dw.any()
