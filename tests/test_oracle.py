"""CPU: the oracle is pinned against the reference's own outputs (golden
vectors made by tests/golden/make_golden.py from the reference build) and
against closed-form known answers of the reference's uniform fills."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, l2c, rel_err

from bgwsigma import inputs as I
from cases import FF_CASES, FULL_FF_CASES, FULL_GPP_CASES, GPP_CASES


@pytest.mark.parametrize("name", sorted(GPP_CASES))
def test_gpp_inputs_stable(golden, name):
    assert I.fingerprint(GPP_CASES[name]()) == golden["gpp"][name]["fingerprint"]


@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_ff_inputs_stable(golden, name):
    assert I.fingerprint(FF_CASES[name]()) == golden["ff"][name]["fingerprint"]


@pytest.mark.parametrize("name", sorted(GPP_CASES))
def test_gpp_oracle_vs_reference(golden, oracle, name):
    g = GPP_CASES[name]()
    ref = l2c(golden["gpp"][name]["reference"])
    assert rel_err(oracle.gpp(g), ref) < FP64_RTOL
    if g.wx_band_stride == 0:
        assert rel_err(oracle.gpp(g, factored=True), ref) < FP64_RTOL


@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_ff_oracle_vs_reference(golden, oracle, name):
    f = FF_CASES[name]()
    ref = golden["ff"][name]["reference"]
    assert rel_err(oracle.achs(f), l2c(ref["achs"])) < FP64_RTOL
    assert rel_err(oracle.asx(f), l2c(ref["asx"])) < FP64_RTOL
    assert rel_err(oracle.cor(f), l2c(ref["cor"])) < FP64_RTOL


def test_gpp_uniform_closed_form(oracle):
    # GPP/gpp.cpp fills: achtemp[iw] = N * 0.125i / (wx - 0.5 - 0.5i).
    for dims in [(64, 2048, 20), (8, 1000, 10), (1, 40, 20)]:
        nb, G, npg = dims
        g = I.gpp_uniform(nb, 2, G, npg)
        kat = I.gpp_uniform_closed_form(nb, G, npg)
        assert rel_err(oracle.gpp(g), kat) < 1e-14
        assert rel_err(oracle.gpp(g, factored=True), kat) < 1e-14


def test_gpp_default_size_closed_form_value():
    # The default GPP size (512 2 32768 20): achtemp(0) = (-264241152, 1321205760)
    # exactly; the reference OpenMP build gives (-264241151.999477,
    # 1321205760.003231).
    kat = I.gpp_uniform_closed_form(512, 32768, 20)
    assert kat[0] == complex(-264241152.0, 1321205760.0)


def test_ff_uniform_closed_forms(oracle):
    # FF/ff.cpp fills: a conj(am) = 0.5, R = 0.5+0.5i, A = 0.5-0.5i, R - A = i,
    # interpolation weights sum to 1.
    nb, nv, G, P, F, E = 64, 2, 512, 64, 15, 10
    f = I.ff_uniform(nb, nv, G, P, F, E)
    assert oracle.achs(f) == -0.125 * (1 + 1j) * nb * P * G
    assert np.all(oracle.asx(f) == 0.25 * (1 + 1j) * nv * P * G)
    # Kernel1 bands: wx = 10.5 - n1 > 0 and n1 >= nvband  ->  n1 = 2..10.
    assert np.all(oracle.cor(f) == -0.25j * 9 * P * G)


def test_compute_fact_quirks(oracle):
    grid = np.linspace(0.0, 2.0, 9)  # 0, 0.25, ..., 2
    # loop 1: a found ifreq == 0 is replaced by nFreq - 2 = 7 (ff.cpp:111).
    i, f1, f2 = oracle.compute_fact(0.1, grid, 1, False)
    assert i == 7 and f1 == pytest.approx((2.0 - 0.1) / 0.25) and f2 == pytest.approx((0.1 - 1.75) / 0.25)
    # loop 1 on a grid point: no strict bracket -> 0 -> 7.
    assert oracle.compute_fact(0.25, grid, 1, False)[0] == 7
    # loop 1, negative wx searches -wx (ff.cpp:116-126).
    i, f1, f2 = oracle.compute_fact(-0.6, grid, 1, False)
    assert i == 2 and f1 == pytest.approx((0.75 - 0.6) / 0.25) and f2 == pytest.approx((0.6 - 0.5) / 0.25)
    # loop 2, wx > 0: ifreq 0 is kept (the `== -1` test never fires), -0.5 factor.
    i, f1, f2 = oracle.compute_fact(0.1, grid, 2, False)
    assert i == 0 and f1 == pytest.approx(-0.5 * 0.15 / 0.25) and f2 == pytest.approx(-0.5 * 0.1 / 0.25)
    # loop 2, wx <= 0 and occupied: search -wx.
    i, f1, f2 = oracle.compute_fact(-0.3, grid, 2, True)
    assert i == 1 and f1 == pytest.approx(0.8) and f2 == pytest.approx(0.2)
    # loop 2, wx <= 0 and unoccupied: untouched.
    assert oracle.compute_fact(-0.3, grid, 2, False) == (0, 0.0, 0.0)


def test_compute_fact_golden(golden, oracle):
    """The probe table holds the reference's own compute_fact (FF/ff.cpp:103-152,
    compiled from ff.cpp by oracle/ref_fact.cpp): every branch and edge, bit for bit."""
    grid = np.array(golden["compute_fact_grid"])
    for wx, loop, occ, i, f1, f2 in golden["compute_fact"]:
        assert oracle.compute_fact(wx, grid, loop, bool(occ)) == (i, f1, f2)


def test_compute_fact_live_if_built(oracle):
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present on this machine")
    ref = Reference()
    rng = np.random.default_rng(12)
    for grid in (np.linspace(0.0, 2.0, 15), np.sort(rng.uniform(0.0, 3.0, 11))):
        for wx in rng.uniform(-4.0, 4.0, 200):
            for loop in (1, 2):
                for occ in (False, True):
                    assert oracle.compute_fact(wx, grid, loop, occ) == ref.compute_fact(wx, grid, loop, occ)


def test_reference_live_if_built(oracle):
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present on this machine")
    ref = Reference()
    g = I.gpp_seeded(16, 2, 512, 8, seed=99)
    assert rel_err(ref.gpp(g), oracle.gpp(g)) < FP64_RTOL
    f = I.ff_seeded(16, 3, 256, 32, 5, 2, seed=99)
    assert rel_err(ref.achs(f), oracle.achs(f)) < FP64_RTOL
    assert rel_err(ref.asx(f), oracle.asx(f)) < FP64_RTOL
    assert rel_err(ref.cor(f), oracle.cor(f)) < FP64_RTOL


@pytest.mark.parametrize("name", sorted(FF_CASES))
def test_ff_per_iw_oracle_pinned_at_iw1(golden, oracle, name):
    """With wx = freqevalmin - ekq + iw * freqevalstep per iw (an option the
    reference lacks), the iw = 1 entry is the reference's value (its single
    wx, FF/ff.cpp:245, 337); the other entries follow the same restatement."""
    f = FF_CASES[name]()
    if f.nfreqeval < 2:
        pytest.skip("needs two evaluation points")
    ref = golden["ff"][name]["reference"]
    asx, cor = oracle.asx(f, per_iw=True), oracle.cor(f, per_iw=True)
    assert rel_err(asx[1], l2c(ref["asx"])[1]) < 1e-14
    assert rel_err(cor[1], l2c(ref["cor"])[1]) < 1e-14


# ------------------------------------------------ GPP screened exchange --
# Specified from the GPP model (the reference has no flagOCC branch): parity
# unpinned; the oracle's product form is checked against the partial-fraction
# identity over the reference-pinned Coulomb-hole sum and a closed form.

def _occupied(g, nv, negate):
    import dataclasses
    stride = g.wx_band_stride
    wx = g.wx_array[: (nv - 1) * stride + 3] if stride and nv else g.wx_array
    return dataclasses.replace(g, number_bands=nv, aqsmtemp=g.aqsmtemp[:nv], aqsntemp=g.aqsntemp[:nv],
                               wx_array=np.ascontiguousarray(-wx if negate else wx))


@pytest.mark.parametrize("per_band", [False, True])
@pytest.mark.parametrize("nv", [1, 3, 7])
def test_gpp_sx_partial_fractions(oracle, nv, per_band):
    g = I.gpp_seeded(9, nv, 400, 8, seed=40 + nv, wx_per_band=per_band)
    sx = oracle.gpp_sx(g)
    pf = -(oracle.gpp(_occupied(g, nv, False)) + oracle.gpp(_occupied(g, nv, True)))
    assert rel_err(sx, pf) < 1e-14
    if not per_band:
        assert rel_err(oracle.gpp_sx(g, factored=True), sx) < 1e-13


def test_gpp_sx_uniform_closed_form(oracle):
    # gpp_uniform: s I_eps = 0.125i, wtilde = 0.5 + 0.5i, so each occupied
    # (band, p, ig) term is -0.125i (1/(wx - wt) - 1/(wx + wt)).
    nb, nv, G, npg = 8, 3, 400, 20
    g = I.gpp_uniform(nb, nv, G, npg)
    wt = 0.5 + 0.5j
    n = nv * (G // npg) * G
    kat = np.array([-n * 0.125j * (1 / (w - wt) - 1 / (w + wt)) for w in (3.0, 4.0, 5.0)])
    assert rel_err(oracle.gpp_sx(g), kat) < 1e-13
    assert np.all(oracle.gpp_sx(g, nvband=0) == 0)


# ------------------------------------------------------ near-pole guard --
# Not in the reference (it has no guard): terms with |wx - wtilde| < delta
# are left out.  Checked against an independent numpy evaluation and, for
# the exchange, against the partial-fraction identity with the guard on.

def near_pole_case(seed=3, nb=6, nv=2, G=300, npg=6):
    """Seeded inputs with wx inside wtilde's range and planted poles: some
    wtilde within 1e-7 of wx[1] and of -wx[0] (the exchange's -wx sum)."""
    g = I.gpp_seeded(nb, nv, G, npg, seed=seed)
    g.wx_array = np.array([1.0, 1.25, 1.5])
    wt = g.wtilde_array.copy()
    rng = np.random.default_rng(seed)
    P = wt.shape[0]
    for k in range(6):
        p, ig = int(rng.integers(P)), int(rng.integers(G))
        wt[p, ig] = (g.wx_array[1] if k % 2 == 0 else -g.wx_array[0]) + 1e-7 * (1 + 1j)
    g.wtilde_array = wt
    return g


def numpy_gpp(g, delta):
    igp = g.indinv[g.inv_igp_index]
    P = g.ngpown
    s = (np.conj(g.aqsmtemp[:, igp]) * g.aqsntemp[:, igp] * 0.5 * g.vcoul[igp]
         * g.wtilde_array[np.arange(P), igp]).sum(axis=0)                  # S(p)
    out = np.zeros(3, np.complex128)
    for iw, x in enumerate(g.wx_array):
        d = x - g.wtilde_array
        q = np.where(np.abs(d) ** 2 < delta ** 2, 0.0, g.I_eps_array / np.where(d == 0, 1, d))
        out[iw] = (s[:, None] * q).sum()
    return out


@pytest.mark.parametrize("delta", [1e-4, 3e-2, 0.2])
def test_gpp_pole_guard_vs_numpy(oracle, delta):
    g = near_pole_case()
    got = oracle.gpp(g, pole_guard=delta)
    assert rel_err(got, numpy_gpp(g, delta)) < 1e-12
    assert rel_err(oracle.gpp(g, factored=True, pole_guard=delta), got) < 1e-13
    # Unguarded, the planted poles dominate.
    assert np.abs(oracle.gpp(g)).max() > 50 * np.abs(got).max()
    # The guard is reset after the call.
    assert np.array_equal(oracle.gpp(g), oracle.gpp(g, pole_guard=0.0))


@pytest.mark.parametrize("delta", [1e-4, 3e-2])
def test_gpp_sx_pole_guard_partial_fractions(oracle, delta):
    g = near_pole_case(seed=5, nv=3)
    sx = oracle.gpp_sx(g, pole_guard=delta)
    pf = -(oracle.gpp(_occupied(g, 3, False), pole_guard=delta) + oracle.gpp(_occupied(g, 3, True), pole_guard=delta))
    assert rel_err(sx, pf) < 1e-13
    assert rel_err(oracle.gpp_sx(g, factored=True, pole_guard=delta), sx) < 1e-13


# ------------------------------------------------------ benchmark sizes --
# The reference build's own outputs at the benchmark sizes (golden "full",
# make_golden.py --full): the inputs regenerate bit for bit, and the oracle
# matches the reference there too.

def test_full_size_oracle_vs_reference(golden, oracle):
    full = golden["full"]
    g = FULL_GPP_CASES["gpp_benchmark"]()
    assert I.fingerprint(g) == full["gpp_benchmark"]["fingerprint"]
    assert rel_err(oracle.gpp(g, factored=True), l2c(full["gpp_benchmark"]["reference"])) < FP64_RTOL
    del g
    f = FULL_FF_CASES["ff_benchmark"]()
    assert I.fingerprint(f) == full["ff_benchmark"]["fingerprint"]
    ref = full["ff_benchmark"]["reference"]
    assert rel_err(oracle.achs(f), l2c(ref["achs"])) < FP64_RTOL
    assert rel_err(oracle.asx(f), l2c(ref["asx"])) < FP64_RTOL
    assert rel_err(oracle.cor(f), l2c(ref["cor"])) < FP64_RTOL
