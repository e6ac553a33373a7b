"""Synthetic inputs of the GPP and FF sums.

Two families:
  *_uniform  the reference drivers' own constant fills (GPP/gpp.cpp:246-275,
             FF/ff.cpp:585-633); their sums have closed forms (known-answer
             tests).
  *_seeded   seeded random inputs with the benchmark distributions:
             GPP  aqsmtemp/aqsntemp U[-1,1]^2, I_eps_array U[-0.5,0.5]^2,
                  wtilde_array Re U[0.5,2] Im U[-0.01,0.01], vcoul[ig] =
                  1/(1+ig), indinv a permutation of 0..ncouls-1 (plus the
                  reference's extra entry indinv[ncouls] = ncouls-1),
                  inv_igp_index[p] = p * nodes_per_group, wx = e_lk +
                  {-0.5, 0, 0.5} with e_lk = 10 (GPP/gpp.cpp:165);
             FF   aqsmtemp/aqsntemp U[-1,1]^2, I_epsR/I_epsA U[-0.5,0.5]^2,
                  ekq U[-1,1], dFreqGrid evenly spaced on [0, 2],
                  inv_igp_index[p] = p, indinv a permutation, vcoul[ig] =
                  1/(1+ig), freqevalmin 0, freqevalstep 0.5, occ 1
                  (FF/ff.cpp:465-467).
Random numbers come from numpy's PCG64 (np.random.default_rng(seed)), drawn
in the fixed order of the code below; fingerprint() hashes the arrays so a
change of stream is detected by the golden tests.
Complex arrays are complex128 (interleaved re/im doubles), row-major.
"""
from __future__ import annotations

import dataclasses
import hashlib
from typing import Any

import numpy as np


def _cuniform(rng: np.random.Generator, shape, lo: float, hi: float) -> np.ndarray:
    n = int(np.prod(shape))
    a = rng.random(2 * n)
    a *= hi - lo
    a += lo
    return a.view(np.complex128).reshape(shape)


@dataclasses.dataclass
class GppInputs:
    number_bands: int
    nvband: int
    ncouls: int
    ngpown: int
    inv_igp_index: Any        # int32 [ngpown]
    indinv: Any               # int32 [ncouls + 1]
    wx_array: Any             # float64 [3] or [number_bands][stride]
    wtilde_array: Any         # complex128 [ngpown][ncouls]
    aqsmtemp: Any             # complex128 [number_bands][ncouls]
    aqsntemp: Any             # complex128 [number_bands][ncouls]
    I_eps_array: Any          # complex128 [ngpown][ncouls]
    vcoul: Any                # float64 [ncouls]
    wx_band_stride: int = 0

    ARRAYS = ("inv_igp_index", "indinv", "wx_array", "wtilde_array", "aqsmtemp", "aqsntemp",
              "I_eps_array", "vcoul")

    def nbytes(self) -> int:
        return sum(int(getattr(self, k).nbytes if hasattr(getattr(self, k), "nbytes")
                       else getattr(self, k).numel() * getattr(self, k).element_size()) for k in self.ARRAYS)

    def map_arrays(self, fn) -> "GppInputs":
        return dataclasses.replace(self, **{k: fn(getattr(self, k)) for k in self.ARRAYS})


@dataclasses.dataclass
class FFInputs:
    number_bands: int
    nvband: int
    ncouls: int
    ngpown: int
    nFreq: int
    nfreqeval: int
    freqevalmin: float
    freqevalstep: float
    occ: float
    ekq: Any                  # float64 [number_bands]
    dFreqGrid: Any            # float64 [nFreq]
    inv_igp_index: Any        # int32 [ngpown]
    indinv: Any               # int32 [ncouls]
    aqsmtemp: Any             # complex128 [number_bands][ncouls]
    aqsntemp: Any             # complex128 [number_bands][ncouls]
    vcoul: Any                # float64 [ncouls]
    I_epsR_array: Any         # complex128 [nFreq][ngpown][ncouls]
    I_epsA_array: Any         # complex128 [nFreq][ngpown][ncouls]

    ARRAYS = ("ekq", "dFreqGrid", "inv_igp_index", "indinv", "aqsmtemp", "aqsntemp", "vcoul",
              "I_epsR_array", "I_epsA_array")

    def nbytes(self) -> int:
        return sum(int(getattr(self, k).nbytes if hasattr(getattr(self, k), "nbytes")
                       else getattr(self, k).numel() * getattr(self, k).element_size()) for k in self.ARRAYS)

    def map_arrays(self, fn) -> "FFInputs":
        return dataclasses.replace(self, **{k: fn(getattr(self, k)) for k in self.ARRAYS})


# ----------------------------------------------------------------- GPP --

def gpp_uniform(number_bands: int, nvband: int, ncouls: int, nodes_per_group: int) -> GppInputs:
    """The GPP driver's fills (GPP/gpp.cpp:143-162, 246-275)."""
    nb, G = number_bands, ncouls
    P = G // nodes_per_group
    e_lk, dw, to1, e_n1kq = 10.0, 1.0, 1e-6, 6.0
    expr = 0.5 + 0.5j
    wx = np.array([max(e_lk - e_n1kq + dw * ((iw + 1) - 2), to1) for iw in range(3)])
    return GppInputs(
        number_bands=nb, nvband=nvband, ncouls=G, ngpown=P,
        inv_igp_index=np.array([(ig + 1) * G // P for ig in range(P)], dtype=np.int32),
        indinv=np.concatenate([np.arange(G, dtype=np.int32), np.array([G - 1], dtype=np.int32)]),
        wx_array=wx,
        wtilde_array=np.full((P, G), expr, dtype=np.complex128),
        aqsmtemp=np.full((nb, G), expr, dtype=np.complex128),
        aqsntemp=np.full((nb, G), expr, dtype=np.complex128),
        I_eps_array=np.full((P, G), expr, dtype=np.complex128),
        vcoul=np.ones(G),
    )


def gpp_uniform_closed_form(number_bands: int, ncouls: int, nodes_per_group: int) -> np.ndarray:
    """achtemp of gpp_uniform: every term is 0.125i / (wx - 0.5 - 0.5i)
    (s = 0.125(1+i), s * I_eps = 0.125i), so achtemp[iw] = N * 0.125i /
    (wx_iw - 0.5 - 0.5i) with N = nb * ngpown * ncouls, wx = 3, 4, 5."""
    P = ncouls // nodes_per_group
    N = number_bands * P * ncouls
    return np.array([N * 0.125j / (wx - 0.5 - 0.5j) for wx in (3.0, 4.0, 5.0)])


def gpp_seeded(number_bands: int, nvband: int, ncouls: int, nodes_per_group: int, seed: int = 1234,
               wx_per_band: bool = False) -> GppInputs:
    nb, G = number_bands, ncouls
    P = G // nodes_per_group
    rng = np.random.default_rng(seed)
    aqsm = _cuniform(rng, (nb, G), -1.0, 1.0)
    aqsn = _cuniform(rng, (nb, G), -1.0, 1.0)
    I_eps = _cuniform(rng, (P, G), -0.5, 0.5)
    wt = np.empty((P, G), dtype=np.complex128)
    wv = wt.view(np.float64).reshape(P, G, 2)
    wv[..., 0] = rng.random((P, G)) * 1.5 + 0.5
    wv[..., 1] = rng.random((P, G)) * 0.02 - 0.01
    indinv = np.concatenate([rng.permutation(G).astype(np.int32), np.array([G - 1], dtype=np.int32)])
    inv = (np.arange(P, dtype=np.int64) * nodes_per_group).astype(np.int32)
    vcoul = 1.0 / (1.0 + np.arange(G, dtype=np.float64))
    e_lk = 10.0
    wx = e_lk + np.array([-0.5, 0.0, 0.5])
    stride = 0
    if wx_per_band:
        # Band-dependent frequencies (not in the reference; exercises the
        # general kernel): wx[n1] = e_lk + {-0.5, 0, 0.5} + U[-0.25, 0.25].
        shift = rng.random(nb) * 0.5 - 0.25
        wx = np.ascontiguousarray(wx[None, :] + shift[:, None])
        stride = 3
    return GppInputs(number_bands=nb, nvband=nvband, ncouls=G, ngpown=P, inv_igp_index=inv, indinv=indinv,
                     wx_array=wx, wtilde_array=wt, aqsmtemp=aqsm, aqsntemp=aqsn, I_eps_array=I_eps,
                     vcoul=vcoul, wx_band_stride=stride)


# ------------------------------------------------------------------ FF --

def ff_uniform(number_bands: int, nvband: int, ncouls: int, ngpown: int, nFreq: int, nfreqeval: int) -> FFInputs:
    """The FF driver's fills (FF/ff.cpp:465-469, 585-633)."""
    nb, G, P = number_bands, ncouls, ngpown
    return FFInputs(
        number_bands=nb, nvband=nvband, ncouls=G, ngpown=P, nFreq=nFreq, nfreqeval=nfreqeval,
        freqevalmin=0.0, freqevalstep=0.5, occ=1.0,
        ekq=-10.0 + np.arange(nb, dtype=np.float64),
        dFreqGrid=2.0 * np.arange(nFreq, dtype=np.float64),
        inv_igp_index=np.arange(P, dtype=np.int32),
        indinv=np.arange(G, dtype=np.int32),
        aqsmtemp=np.full((nb, G), 0.5 + 0.5j, dtype=np.complex128),
        aqsntemp=np.full((nb, G), 0.5 + 0.5j, dtype=np.complex128),
        vcoul=np.ones(G),
        I_epsR_array=np.full((nFreq, P, G), 0.5 + 0.5j, dtype=np.complex128),
        I_epsA_array=np.full((nFreq, P, G), 0.5 - 0.5j, dtype=np.complex128),
    )


def ff_seeded(number_bands: int, nvband: int, ncouls: int, ngpown: int, nFreq: int, nfreqeval: int,
              seed: int = 1234) -> FFInputs:
    nb, G, P = number_bands, ncouls, ngpown
    rng = np.random.default_rng(seed)
    aqsm = _cuniform(rng, (nb, G), -1.0, 1.0)
    aqsn = _cuniform(rng, (nb, G), -1.0, 1.0)
    R = _cuniform(rng, (nFreq, P, G), -0.5, 0.5)
    A = _cuniform(rng, (nFreq, P, G), -0.5, 0.5)
    ekq = rng.random(nb) * 2.0 - 1.0
    indinv = rng.permutation(G).astype(np.int32)
    return FFInputs(
        number_bands=nb, nvband=nvband, ncouls=G, ngpown=P, nFreq=nFreq, nfreqeval=nfreqeval,
        freqevalmin=0.0, freqevalstep=0.5, occ=1.0, ekq=ekq,
        dFreqGrid=np.linspace(0.0, 2.0, nFreq),
        inv_igp_index=np.arange(P, dtype=np.int32), indinv=indinv,
        aqsmtemp=aqsm, aqsntemp=aqsn, vcoul=1.0 / (1.0 + np.arange(G, dtype=np.float64)),
        I_epsR_array=R, I_epsA_array=A,
    )


def fingerprint(inp) -> str:
    """sha256 over the host arrays of a GppInputs / FFInputs (order fixed)."""
    h = hashlib.sha256()
    for k in inp.ARRAYS:
        a = np.ascontiguousarray(getattr(inp, k))
        h.update(k.encode())
        h.update(a.tobytes())
    return h.hexdigest()
