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


# ------------------------------------------- counter-based (Philox) family --
#
# The same distributions as gpp_seeded, drawn from Philox4x64-10 streams
# keyed by (seed, stream id), one stream per array, word w of an array being
# its w-th double (interleaved re/im).  Every value depends only on (seed,
# array, index), so a G' row block [p0, p1) of wtilde_array / I_eps_array is
# generated without the rest, on the host (numpy's Philox, below) or on the
# GPU (bgw_fill_uniform, bgwsigma.fill_uniform) with identical bits.
# indinv (a permutation of ncouls entries) is drawn on the host from PCG64.
PHILOX_STREAMS = {"aqsmtemp": 1, "aqsntemp": 2, "I_eps_array": 3, "wtilde_array": 4}
# (lo_even, hi_even, lo_odd, hi_odd): real and imaginary ranges per array.
GPP_RANGES = {"aqsmtemp": (-1.0, 1.0, -1.0, 1.0), "aqsntemp": (-1.0, 1.0, -1.0, 1.0),
              "I_eps_array": (-0.5, 0.5, -0.5, 0.5), "wtilde_array": (0.5, 2.0, -0.01, 0.01)}


def philox_uniform(n: int, seed: int, stream: int, offset: int, lo_even: float, hi_even: float, lo_odd: float,
                   hi_odd: float) -> np.ndarray:
    """Host twin of bgw_fill_uniform: words offset .. offset + n - 1 of
    numpy's Philox(key=seed + stream * 2**64) mapped to [lo, hi) by
    lo + (hi - lo) * ((word >> 11) * 2**-53) (even words: the real range,
    odd words: the imaginary range), in pieces of at most 2**22 words."""
    out = np.empty(n, dtype=np.float64)
    piece = 1 << 22
    for i in range(0, n, piece):
        m = min(piece, n - i)
        w0 = offset + i
        bg = np.random.Philox(key=int(seed) + (int(stream) << 64), counter=[w0 // 4, 0, 0, 0])
        skip = w0 % 4
        u = (bg.random_raw(m + skip)[skip:] >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
        even = ((w0 + np.arange(m)) & 1) == 0
        v = out[i:i + m]
        v[even] = u[even] * (hi_even - lo_even) + lo_even
        v[~even] = u[~even] * (hi_odd - lo_odd) + lo_odd
    return out


def gpp_philox(number_bands: int, nvband: int, ncouls: int, nodes_per_group: int, seed: int = 1234,
               rows: tuple[int, int] | None = None, device=None) -> GppInputs:
    """GPP inputs with the benchmark distributions from Philox streams.
    rows=(p0, p1): only G' rows [p0, p1) of the whole problem (ngpown =
    p1 - p0; inv_igp_index, wtilde_array and I_eps_array sliced), as one
    rank of a G'-sharded run holds them.  device (a torch device): the large
    arrays are generated there by bgw_fill_uniform; else on the host."""
    nb, G = number_bands, ncouls
    P_all = G // nodes_per_group
    p0, p1 = rows if rows is not None else (0, P_all)
    P = p1 - p0
    rng = np.random.default_rng(seed)
    indinv = np.concatenate([rng.permutation(G).astype(np.int32), np.array([G - 1], dtype=np.int32)])
    inv = (np.arange(p0, p1, dtype=np.int64) * nodes_per_group).astype(np.int32)
    vcoul = 1.0 / (1.0 + np.arange(G, dtype=np.float64))
    wx = 10.0 + np.array([-0.5, 0.0, 0.5])
    shapes = {"aqsmtemp": (nb, G, 0), "aqsntemp": (nb, G, 0), "I_eps_array": (P, G, p0), "wtilde_array": (P, G, p0)}
    big = {}
    for name, (r, c, r0) in shapes.items():
        n, off = 2 * r * c, 2 * r0 * c
        if device is None:
            big[name] = philox_uniform(n, seed, PHILOX_STREAMS[name], off, *GPP_RANGES[name]).view(
                np.complex128).reshape(r, c)
        else:
            import torch

            from . import fill_uniform
            t = torch.empty((r, c), dtype=torch.complex128, device=device)
            fill_uniform(torch.view_as_real(t), seed, PHILOX_STREAMS[name], off, *GPP_RANGES[name])
            big[name] = t
    small = dict(inv_igp_index=inv, indinv=indinv, wx_array=wx, vcoul=vcoul)
    if device is not None:
        import torch
        small = {k: torch.as_tensor(v).to(device) for k, v in small.items()}
    return GppInputs(number_bands=nb, nvband=nvband, ncouls=G, ngpown=P, wx_band_stride=0, **small, **big)


def batch_shapes(n: int = 64, seed: int = 4321) -> list[tuple[int, int]]:
    """(number_bands, ncouls) of the batched uneven q-point workload: ncouls
    uniform in {4096, 4608, ..., 32768}, number_bands uniform in [128, 512]
    (nodes_per_group 20), drawn from PCG64 in a fixed order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        G = int(rng.choice(np.arange(4096, 32768 + 1, 512)))
        nb = int(rng.integers(128, 513))
        out.append((nb, G))
    return out


def batch_philox(n: int = 64, seed: int = 4321, device=None, only=None) -> list[GppInputs]:
    """The batched workload's instances (batch_shapes), instance k drawn from
    gpp_philox with seed + k (on `device`, or on the host).  only: indices of
    the instances to generate (the others are None)."""
    shapes = batch_shapes(n, seed)
    return [gpp_philox(nb, 2, G, 20, seed=seed + k, device=device) if only is None or k in only else None
            for k, (nb, G) in enumerate(shapes)]


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
