"""Golden cases: seeded (or fixed) inputs whose reference outputs are stored
in tests/golden/*.json by make_golden.py.  The inputs themselves are not
stored; they are regenerated from these definitions and checked against the
stored sha256 fingerprints."""
from __future__ import annotations

import numpy as np

from bgwsigma import inputs as I

# name -> (kind, builder)
GPP_CASES = {
    # The small configuration: 64 bands, ncouls 2048, nodes_per_group 20.
    "gpp_small_seeded": lambda: I.gpp_seeded(64, 2, 2048, 20, seed=1234),
    "gpp_small_uniform": lambda: I.gpp_uniform(64, 2, 2048, 20),
    # ncouls not a multiple of any tile, odd ngpown.
    "gpp_ragged": lambda: I.gpp_seeded(3, 1, 1000, 7, seed=7),
    # Smallest non-empty problem.
    "gpp_single": lambda: I.gpp_seeded(1, 1, 20, 20, seed=3),
    # Many bands (exercises band chunking of the staged sch_store1 table).
    "gpp_many_bands": lambda: I.gpp_seeded(1100, 2, 256, 16, seed=5),
}


def _ff_edges():
    """FF inputs whose band energies hit every branch of compute_fact
    (FF/ff.cpp:103-152): wx = 0.5 - ekq on a grid 0, 0.25, ..., 2."""
    f = I.ff_seeded(24, 12, 300, 40, 9, 4, seed=21)
    wx = np.array([0.1, 0.25, 3.0, -0.1, -0.3, 0.0, 1.3, -2.5, 0.6, -0.25, 1.99, 2.0,
                   0.1, 0.25, 3.0, -0.1, -0.3, 0.0, 1.3, -2.5, 0.6, -0.25, 1.99, 2.0])
    f.ekq = 0.5 - wx
    f.dFreqGrid = np.linspace(0.0, 2.0, 9)
    return f


FF_CASES = {
    "ff_small_seeded": lambda: I.ff_seeded(64, 2, 1024, 128, 15, 10, seed=1234),
    "ff_small_uniform": lambda: I.ff_uniform(64, 2, 512, 64, 15, 10),
    "ff_ragged": lambda: I.ff_seeded(37, 5, 777, 53, 7, 3, seed=11),
    "ff_many_occupied": lambda: I.ff_seeded(40, 20, 640, 70, 6, 2, seed=13),
    "ff_fact_edges": _ff_edges,
}


# The benchmark sizes (outputs only: the reference's own results at full size,
# regenerated by make_golden.py --full).
FULL_GPP_CASES = {
    "gpp_benchmark": lambda: I.gpp_seeded(512, 2, 32768, 20, seed=1234),
}
FULL_FF_CASES = {
    "ff_benchmark": lambda: I.ff_seeded(512, 2, 8192, 512, 15, 10, seed=1234),
}
