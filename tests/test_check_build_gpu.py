"""GPU: the small golden and oracle cases of every kernel family run under the
bounds-checked debug build (lib/libbgwsigma_check.so, compiled with
-DBGW_CHECK): the kernels check their staging ranges, shared-memory
capacities and tile / row / packed-buffer indices and would report
BGW_ERR_CHECK.  Every call must return BGW_OK and match the oracle at the
product build's tolerances.  The cases run in a child process that loads the
debug library through BGW_SIGMA_LIB."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

TESTS = Path(__file__).resolve().parent


def _run_all() -> None:
    import numpy as np
    import torch

    import bgwsigma as bgw
    from bgwsigma import inputs as I
    from conftest import FP64_RTOL, MIXED_RTOL, rel_err
    from cases import FF_CASES, GPP_CASES
    from oracle.oracle import Oracle

    assert Path(bgw.lib_path()).name == "libbgwsigma_check.so", bgw.lib_path()
    dev = torch.device("cuda:0")
    orc = Oracle()
    for name, make in GPP_CASES.items():
        g = make()
        ref = orc.gpp(g)
        for alg in ("bandloop", "factored"):
            assert rel_err(bgw.noflagOCC_solver(g, algorithm=alg), ref) < FP64_RTOL, (name, alg)
        assert rel_err(bgw.noflagOCC_solver(bgw.to_device(g, dev), algorithm="bandloop").cpu().numpy(),
                       ref) < FP64_RTOL, name
        assert rel_err(bgw.noflagOCC_solver(g, algorithm="bandloop", precision="mixed"), ref) < MIXED_RTOL, name
    gb = I.gpp_seeded(40, 2, 1500, 15, seed=17, wx_per_band=True)
    assert rel_err(bgw.noflagOCC_solver(gb, precision="mixed"), orc.gpp(gb)) < MIXED_RTOL
    d = bgw.to_device(I.gpp_seeded(48, 2, 2048, 16, seed=5), dev)
    gw, gi, dw = bgw.noflagOCC_solver_backward(d, [1, 1j, -1])
    h = I.gpp_seeded(48, 2, 2048, 16, seed=5)
    rw, ri, rd = orc.gpp_backward(h, [1, 1j, -1])
    assert rel_err(gw.cpu().numpy(), rw) < FP64_RTOL and rel_err(gi.cpu().numpy(), ri) < FP64_RTOL
    insts = [bgw.to_device(I.gpp_seeded(nb, 2, G, 16, seed=60 + k), dev)
             for k, (nb, G) in enumerate([(33, 2048), (7, 1000), (64, 4096)])]
    for prec, tol in (("fp64", FP64_RTOL), ("mixed", MIXED_RTOL)):
        b = bgw.GppBatch(insts, algorithm="bandloop", precision=prec)
        out = b.execute().cpu().numpy()
        b.close()
        for k, x in enumerate(insts):
            assert rel_err(out[k], orc.gpp(x.map_arrays(lambda t: t.cpu().numpy()))) < tol
    for name, make in FF_CASES.items():
        f = make()
        want = (orc.achs(f), orc.asx(f), orc.cor(f))
        want_iw = (want[0], orc.asx(f, per_iw=True), orc.cor(f, per_iw=True))
        for prec, fl, tol in (("fp64", 0, FP64_RTOL), ("mixed", bgw.FLAG_FF_SLICE_ALL, 1e-9),
                              ("fp64", bgw.FLAG_FF_WX_PER_IW, FP64_RTOL),
                              ("mixed", bgw.FLAG_FF_SLICE_ALL | bgw.FLAG_FF_WX_PER_IW, 1e-9)):
            got = bgw.ff_sigma(bgw.to_device(f, dev), precision=prec, flags=fl)
            ref = want_iw if fl & bgw.FLAG_FF_WX_PER_IW else want
            for a, w in zip(got, ref):
                assert rel_err(a.cpu().numpy(), w) < tol, (name, prec, fl)
    print("check build: all cases ok")


def test_golden_cases_under_the_bounds_checked_build():
    from bgwsigma import build as B
    lib = B.build_check()
    env = dict(os.environ, BGW_SIGMA_LIB=str(lib), BGW_SIGMA_NO_BUILD="1")
    code = ("import sys; sys.path[:0] = [%r, %r, %r, %r]; import test_check_build_gpu as t; t._run_all()"
            % (str(TESTS), str(TESTS.parent), str(TESTS.parent / "berkeleygw-kernels-cpp_b200"), str(TESTS / "golden")))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "all cases ok" in r.stdout
