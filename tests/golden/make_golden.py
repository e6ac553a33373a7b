"""Generates tests/golden/golden.json from the reference's own kernels.

Run where the reference tree is available (it builds oracle/_ref/libbgwref.so
from the reference sources, see oracle/Makefile):

    python tests/golden/make_golden.py          # every small case
    python tests/golden/make_golden.py --full   # adds the benchmark sizes

For every case of tests/golden/cases.py it records the input fingerprint,
the reference build's outputs (OpenMP 3.0 build, all host threads) and the
long-double oracle's outputs.  The benchmark-size cases (FULL_*_CASES) keep
the fingerprint and the reference's outputs only, in the "full" section,
which --full fills in place without recomputing the rest.  Complex numbers
are stored as [re, im].
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "berkeleygw-kernels-cpp_b200"))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

import numpy as np  # noqa: E402

from bgwsigma import inputs as I  # noqa: E402
from cases import FF_CASES, FULL_FF_CASES, FULL_GPP_CASES, GPP_CASES  # noqa: E402
from oracle.oracle import Oracle, Reference, build_oracle  # noqa: E402


def c2l(z):
    z = np.atleast_1d(np.asarray(z, dtype=np.complex128))
    return [[float(v.real), float(v.imag)] for v in z]


def main():
    build_oracle(ref=True)
    orc, ref = Oracle(), Reference()
    out = {"generator": "tests/golden/make_golden.py", "reference_threads": ref.num_threads(), "gpp": {}, "ff": {}}
    for name, mk in GPP_CASES.items():
        g = mk()
        out["gpp"][name] = {
            "fingerprint": I.fingerprint(g),
            "dims": [g.number_bands, g.ngpown, g.ncouls],
            "reference": c2l(ref.gpp(g)),
            "oracle": c2l(orc.gpp(g)),
        }
        print(name, out["gpp"][name]["reference"][0])
    for name, mk in FF_CASES.items():
        f = mk()
        out["ff"][name] = {
            "fingerprint": I.fingerprint(f),
            "dims": [f.number_bands, f.nvband, f.ncouls, f.ngpown, f.nFreq, f.nfreqeval],
            "reference": {"achs": c2l(ref.achs(f)), "asx": c2l(ref.asx(f)), "cor": c2l(ref.cor(f))},
            "oracle": {"achs": c2l(orc.achs(f)), "asx": c2l(orc.asx(f)), "cor": c2l(orc.cor(f))},
        }
        print(name, out["ff"][name]["reference"]["achs"][0])
    # compute_fact probes through the reference's own compute_fact (an inline
    # helper of ff.cpp, compiled from ff.cpp by oracle/ref_fact.cpp): every
    # branch, bracket edges and the grid ends.
    grid = np.linspace(0.0, 2.0, 9)
    probes = []
    for wx in [0.1, 0.25, 3.0, -0.1, -0.3, 0.0, 1.3, -2.5, 0.6, -0.25, 1.99, 2.0, 0.125, -0.125, 1e-9, -1e-9,
               1.75, -1.75, 2.5, -2.0]:
        for loop in (1, 2):
            for occ in (False, True):
                probes.append([wx, loop, int(occ), *ref.compute_fact(wx, grid, loop, occ)])
    # Mangled names of the reference kernels (the drop-in shim must export
    # exactly these), read from the objects built from the reference sources.
    import subprocess
    syms = []
    for obj in ("gpp_ref.o", "ff_ref.o"):
        nm = subprocess.run(["nm", str(REPO / "oracle" / "_ref" / obj)], capture_output=True, text=True, check=True)
        for line in nm.stdout.splitlines():
            parts = line.split()
            if len(parts) == 3 and parts[1] == "T" and any(k in parts[2] for k in (
                    "noflagOCC_solver", "achsDtemp_Kernel", "asxDtemp_Kernel", "achDtemp_cor_Kernel")):
                syms.append(parts[2])
    out["reference_symbols"] = sorted(syms)
    out["compute_fact_grid"] = grid.tolist()
    out["compute_fact"] = probes
    prev = HERE / "golden.json"
    if prev.exists():  # keep the benchmark-size section (make_golden.py --full)
        old = json.loads(prev.read_text())
        if "full" in old:
            out["full"] = old["full"]
    (HERE / "golden.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "golden.json")


def main_full():
    build_oracle(ref=True)
    ref = Reference()
    path = HERE / "golden.json"
    out = json.loads(path.read_text())
    full = {"reference_threads": ref.num_threads()}
    for name, mk in FULL_GPP_CASES.items():
        g = mk()
        full[name] = {"fingerprint": I.fingerprint(g), "dims": [g.number_bands, g.ngpown, g.ncouls],
                      "reference": c2l(ref.gpp(g))}
        print(name, full[name]["reference"][0])
        del g
    for name, mk in FULL_FF_CASES.items():
        f = mk()
        full[name] = {"fingerprint": I.fingerprint(f),
                      "dims": [f.number_bands, f.nvband, f.ncouls, f.ngpown, f.nFreq, f.nfreqeval],
                      "reference": {"achs": c2l(ref.achs(f)), "asx": c2l(ref.asx(f)), "cor": c2l(ref.cor(f))}}
        print(name, full[name]["reference"]["achs"][0])
        del f
    out["full"] = full
    path.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    if "--full" in sys.argv[1:]:
        main_full()
    else:
        main()
