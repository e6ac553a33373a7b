"""GPU: many uneven GPP instances in one persistent launch replayed from a
CUDA graph (bgw_gpp_batch_*), against per-instance calls and the oracle."""
from __future__ import annotations

import numpy as np
import pytest
from conftest import FP64_RTOL, MIXED_RTOL, rel_err

from bgwsigma import inputs as I

pytestmark = pytest.mark.gpu

# (number_bands, ncouls, nodes_per_group): uneven bands, ncouls not
# multiples of the chunk, an instance without bands, a long band list.
SHAPES = [(17, 1000, 7), (1, 512, 4), (64, 2048, 20), (0, 256, 8), (300, 1536, 16), (3, 700, 10),
          (130, 3000, 20), (600, 300, 6)]


def _batch_inputs(cuda, wx_per_band=False):
    import bgwsigma
    hosts = [I.gpp_seeded(nb, 2, G, npg, seed=100 + k, wx_per_band=wx_per_band)
             for k, (nb, G, npg) in enumerate(SHAPES)]
    return hosts, [bgwsigma.to_device(h, cuda) for h in hosts]


@pytest.mark.parametrize("algorithm,precision,rtol", [("bandloop", "fp64", FP64_RTOL), ("factored", "fp64", FP64_RTOL),
                                                      ("bandloop", "mixed", MIXED_RTOL)])
def test_batch_matches_oracle_and_single_calls(bgw, oracle, cuda, algorithm, precision, rtol):
    hosts, devs = _batch_inputs(cuda)
    b = bgw.GppBatch(devs, algorithm=algorithm, precision=precision)
    out = b.execute().cpu().numpy()
    for k, (h, d) in enumerate(zip(hosts, devs)):
        ref = oracle.gpp(h)
        if np.all(ref == 0):
            assert np.all(out[k] == 0)
            continue
        assert rel_err(out[k], ref) < rtol, (k, SHAPES[k])
        single = bgw.noflagOCC_solver(d, algorithm=algorithm, precision=precision).cpu().numpy()
        assert rel_err(out[k], single) < max(rtol, 1e-13)
    info = b.info()
    assert info["grid"] >= 1 and info["items"] > 0
    b.close()


def test_batch_replay_is_bitwise_identical(bgw, cuda):
    _, devs = _batch_inputs(cuda)
    b = bgw.GppBatch(devs, algorithm="bandloop")
    a = b.execute().cpu().numpy().copy()
    for _ in range(2):
        assert np.array_equal(a, b.execute().cpu().numpy())
    b.close()


def test_batch_band_dependent_wx(bgw, oracle, cuda):
    hosts, devs = _batch_inputs(cuda, wx_per_band=True)
    b = bgw.GppBatch(devs)                       # AUTO -> band loop
    out = b.execute().cpu().numpy()
    for k, h in enumerate(hosts):
        ref = oracle.gpp(h)
        if np.all(ref == 0):
            continue
        assert rel_err(out[k], ref) < FP64_RTOL
    with pytest.raises(bgw.BgwError) as e:
        bgw.GppBatch(devs, algorithm="factored")
    assert e.value.status == -7
    b.close()


def test_batch_reports_bad_index(bgw, cuda):
    hosts, devs = _batch_inputs(cuda)
    bad = devs[2]
    bad.inv_igp_index = bad.inv_igp_index.clone()
    bad.inv_igp_index[0] = 10 ** 6
    b = bgw.GppBatch(devs, algorithm="bandloop")
    with pytest.raises(bgw.BgwError) as e:
        b.execute()
    assert e.value.status == -2
    b.close()


def test_batch_requires_device_memory(bgw, cuda):
    hosts, _ = _batch_inputs(cuda)
    with pytest.raises(ValueError):
        bgw.GppBatch(hosts)


def test_64_instance_config_subset_vs_oracle(bgw, oracle, cuda):
    """The batched workload at its full size (64 uneven q-point instances,
    ~54 GB generated on the GPU by bgw_fill_uniform): the one persistent
    launch's results for a subset of the instances -- the smallest, the
    largest and two others -- match the oracle on the same inputs (the host
    twin of the fill), FP64 at 1e-12 and mixed at 1e-9."""
    import torch
    from bgwsigma import inputs as I
    shapes = I.batch_shapes()
    sizes = [nb * G for nb, G in shapes]
    pick = sorted({int(np.argmin(sizes)), int(np.argmax(sizes)), 17, 42})
    devs = I.batch_philox(device=cuda)
    want = {k: oracle.gpp(h, factored=True) for k, h in enumerate(I.batch_philox(only=pick)) if h is not None}
    for prec, tol in (("fp64", FP64_RTOL), ("mixed", MIXED_RTOL)):
        b = bgw.GppBatch(devs, algorithm="bandloop", precision=prec)
        out = b.execute().cpu().numpy()
        b.close()
        for k in pick:
            assert rel_err(out[k], want[k]) < tol, (prec, k, rel_err(out[k], want[k]))
    del devs
    torch.cuda.empty_cache()
