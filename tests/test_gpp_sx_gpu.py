"""GPU: bgw_gpp_sigma -- the Coulomb-hole sum over all bands together with
the GPP screened exchange of the occupied bands (asxtemp).  The exchange has
no counterpart in the reference (GPP/gpp.cpp:307-402 has no flagOCC branch),
so it is checked against the oracle's product form, whose own CPU tests pin
it to the partial-fraction identity over the reference-pinned Coulomb-hole
sum and to a closed form.  Tolerance: 1e-12 relative (FP64); the mixed band
loop (1e-9 per sum) loses a factor of about wx / wtilde to the cancellation
between the +wx and -wx sums, hence 1e-8."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, MIXED_RTOL, rel_err

from bgwsigma import inputs as I

pytestmark = pytest.mark.gpu

MIXED_SX_RTOL = 1e-8


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_uniform_closed_form(bgw, cuda, algorithm):
    nb, nv, G, npg = 16, 3, 2000, 20
    g = I.gpp_uniform(nb, nv, G, npg)
    ach, asx = bgw.gpp_sigma(g, algorithm=algorithm)
    wt = 0.5 + 0.5j
    n = nv * (G // npg) * G
    kat = np.array([-n * 0.125j * (1 / (w - wt) - 1 / (w + wt)) for w in (3.0, 4.0, 5.0)])
    assert rel_err(asx, kat) < FP64_RTOL
    assert rel_err(ach, I.gpp_uniform_closed_form(nb, G, npg)) < FP64_RTOL


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
@pytest.mark.parametrize("dims", [(40, 4, 3000, 10), (7, 7, 1024, 8), (33, 1, 777, 3), (64, 16, 8192, 20)])
def test_seeded_vs_oracle(bgw, oracle, cuda, dims, algorithm):
    g = I.gpp_seeded(*dims, seed=sum(dims))
    ach, asx = bgw.gpp_sigma(g, algorithm=algorithm)
    assert rel_err(asx, oracle.gpp_sx(g)) < FP64_RTOL
    assert rel_err(ach, oracle.gpp(g)) < FP64_RTOL


def test_band_dependent_wx(bgw, oracle, cuda):
    g = I.gpp_seeded(24, 5, 2048, 16, seed=9, wx_per_band=True)
    ach, asx = bgw.gpp_sigma(g)
    assert rel_err(asx, oracle.gpp_sx(g)) < FP64_RTOL
    assert rel_err(ach, oracle.gpp(g)) < FP64_RTOL


@pytest.mark.parametrize("algorithm", ["bandloop", "factored"])
def test_achtemp_bitwise_equal_to_noflagOCC_solver(bgw, cuda, algorithm):
    g = bgw.to_device(I.gpp_seeded(48, 6, 4096, 20, seed=5), cuda)
    ach, _ = bgw.gpp_sigma(g, algorithm=algorithm)
    ref = bgw.noflagOCC_solver(g, algorithm=algorithm)
    assert np.array_equal(ach.cpu().numpy(), ref.cpu().numpy())


def test_host_and_device_agree(bgw, cuda):
    h = I.gpp_seeded(32, 4, 4096, 16, seed=6)
    ha, hs = bgw.gpp_sigma(h)
    da, ds = bgw.gpp_sigma(bgw.to_device(h, cuda))
    assert np.array_equal(ha, da.cpu().numpy())
    assert np.array_equal(hs, ds.cpu().numpy())


def test_one_output_only_and_nvband_limits(bgw, oracle, cuda):
    g = I.gpp_seeded(20, 4, 1024, 8, seed=7)
    ach, asx = bgw.gpp_sigma(g, want_ach=False)
    assert ach is None and rel_err(asx, oracle.gpp_sx(g)) < FP64_RTOL
    ach, asx = bgw.gpp_sigma(g, want_asx=False)
    assert asx is None and rel_err(ach, oracle.gpp(g)) < FP64_RTOL
    _, asx0 = bgw.gpp_sigma(g, nvband=0)
    assert np.all(asx0 == 0)
    _, asxn = bgw.gpp_sigma(g, nvband=20)
    assert rel_err(asxn, oracle.gpp_sx(g, nvband=20)) < FP64_RTOL
    for bad in (-1, 21):
        with pytest.raises(bgw.BgwError) as e:
            bgw.gpp_sigma(g, nvband=bad)
        assert e.value.status == -1
    with pytest.raises(bgw.BgwError):
        bgw.gpp_sigma(g, want_ach=False, want_asx=False)


def test_mixed_precision(bgw, oracle, cuda):
    g = I.gpp_seeded(64, 8, 8192, 20, seed=8)
    ach, asx = bgw.gpp_sigma(g, precision="mixed", algorithm="bandloop")
    assert rel_err(asx, oracle.gpp_sx(g)) < MIXED_SX_RTOL
    assert rel_err(ach, oracle.gpp(g)) < MIXED_RTOL


def test_default_size_factored(bgw, oracle, cuda):
    """512 bands (16 occupied) x 1638 x 32768, device-resident, factored."""
    g = I.gpp_seeded(512, 16, 32768, 20, seed=11)
    ach, asx = bgw.gpp_sigma(bgw.to_device(g, cuda), algorithm="factored")
    assert rel_err(asx.cpu().numpy(), oracle.gpp_sx(g, factored=True)) < FP64_RTOL
    assert rel_err(ach.cpu().numpy(), oracle.gpp(g, factored=True)) < FP64_RTOL
