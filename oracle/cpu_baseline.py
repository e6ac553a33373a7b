"""Times the reference's own CPU build on the GPP benchmark workload
(TEST INFRASTRUCTURE: bench.py's cpu_baseline leg and reference arm only).

One timed repetition is one whole noflagOCC_solver call (GPP/gpp.cpp:282-289
times the same call) of the reference's OpenMP build, oracle/_ref/libbgwref.so
(GPP/gpp.cpp compiled unmodified), on every host thread OpenMP is given; where
that build is absent, the long-double restatement (oracle/_build/liboracle.so)
stands in ("kind": "port").  Inputs: bgwsigma.inputs.gpp_seeded with the
given sizes and seed (the bench's own inputs).  Warm-up calls run on the
first --warmup-bands bands (they warm the thread pool and fault in the
pages; the arrays they read are the full-size ones) and are not timed.

Run as its own process, so that no other runtime's threads (torch, the GPU
library's staging threads) share the cores:

  python -m oracle.cpu_baseline --bands 512 --ncouls 32768 --npg 20 --reps 3

prints one JSON line: {"kind", "cores", "times_s": [...], "achtemp": [...]}.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "berkeleygw-kernels-cpp_b200"))
sys.path.insert(0, str(REPO))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--bands", type=int, default=512)
    ap.add_argument("--nvband", type=int, default=2)
    ap.add_argument("--ncouls", type=int, default=32768)
    ap.add_argument("--npg", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--warmup-bands", type=int, default=16)
    args = ap.parse_args()

    import dataclasses

    import numpy as np

    from bgwsigma import inputs as I
    from oracle.oracle import Oracle, Reference

    g = I.gpp_seeded(args.bands, args.nvband, args.ncouls, args.npg, seed=args.seed)
    if Reference.available():
        impl, kind = Reference(), "reference"
        cores = impl.num_threads()
        run = impl.gpp
    else:
        import os
        impl, kind, cores = Oracle(), "port", os.cpu_count()
        run = lambda x: impl.gpp(x)  # noqa: E731
    wb = max(1, min(args.warmup_bands, args.bands))
    gw = dataclasses.replace(g, number_bands=wb, aqsmtemp=np.ascontiguousarray(g.aqsmtemp[:wb]),
                             aqsntemp=np.ascontiguousarray(g.aqsntemp[:wb]))
    for _ in range(args.warmup):
        run(gw)
    times, out = [], None
    for _ in range(args.reps):
        t0 = time.perf_counter()
        out = run(g)
        times.append(time.perf_counter() - t0)
    print(json.dumps({"kind": kind, "cores": cores, "times_s": times, "bands": args.bands,
                      "warmup_bands": wb, "achtemp": [[float(z.real), float(z.imag)] for z in np.atleast_1d(out)]}),
          flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
