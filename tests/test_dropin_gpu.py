"""GPU: the reference drivers' own `main` (GPP/gpp.cpp:133-305,
FF/ff.cpp:453-764), compiled unmodified and linked against the C++11 shim
(oracle/Makefile target `dropin`), run on the GPU through the shim and print
the closed-form answers of their uniform fills.  The executables are built
where the reference tree exists and travel with the working tree."""
from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest
from conftest import REPO

from bgwsigma import inputs as I

pytestmark = pytest.mark.gpu
REF = REPO / "oracle" / "_ref"


def _run(exe, args):
    if not exe.exists():
        pytest.skip(f"{exe.name} not built (needs the reference tree at build time)")
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _pairs(text):
    return [complex(float(a), float(b)) for a, b in re.findall(r"\(([-\d.eE+]+),([-\d.eE+]+)\)", text)]


def test_gpp_driver_through_shim(bgw, cuda):
    out = _run(REF / "gpp_dropin.ex", [64, 2, 2048, 20])
    got = _pairs(out.split("Final achtemp")[1])[0]
    kat = I.gpp_uniform_closed_form(64, 2048, 20)[0]
    assert abs(got - kat) / abs(kat) < 1e-11   # printed with 6 decimals


def test_ff_driver_through_shim(bgw, cuda):
    nb, nv, G, P, F, E = 64, 2, 512, 64, 15, 10
    out = _run(REF / "ff_dropin.ex", [nb, nv, G, P, F, E])
    vals = _pairs(out)
    achs, asx, cor = vals[-3], vals[-2], vals[-1]
    assert np.isclose(achs, -0.125 * (1 + 1j) * nb * P * G, rtol=1e-12)
    assert np.isclose(asx, 0.25 * (1 + 1j) * nv * P * G, rtol=1e-12)
    assert np.isclose(cor, -0.25j * 9 * P * G, rtol=1e-12)
