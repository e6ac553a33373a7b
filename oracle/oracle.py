"""ctypes loaders of the CPU checkers (TEST INFRASTRUCTURE ONLY).

  Oracle      oracle/_build/liboracle.so -- long-double restatement
              (bgw_oracle.c) of the reference algorithms
  Reference   oracle/_ref/libbgwref.so   -- the reference's own GPP/FF kernels
              compiled unmodified (oracle/Makefile target `ref`); present
              only where it was built

Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and the
reference arm) may import this module; the product never does.
Both take the arrays of bgwsigma.inputs.GppInputs / FFInputs (host numpy).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libbgwref.so"
# The reference source tree: $BGW_REFERENCE_DIR, else the build container's mount.
REF_SRC = Path(os.environ.get("BGW_REFERENCE_DIR", "/root/reference"))

_P = ctypes.c_void_p
_L = ctypes.c_long
_D = ctypes.c_double


def build_oracle(ref: bool | None = None) -> None:
    """Builds liboracle.so, and libbgwref.so when the reference tree exists."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    if ref is None:
        ref = (REF_SRC / "GPP" / "gpp.cpp").exists()
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REF_SRC}"], check=True)


def _p(a) -> int:
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous, "host C-contiguous numpy array required"
    return a.ctypes.data


class Oracle:
    """Long-double CPU restatement of the reference (bgw_oracle.c)."""

    def __init__(self, path: Path = ORACLE_LIB):
        if not path.exists():
            build_oracle(ref=False)
        lib = ctypes.CDLL(str(path))
        lib.orc_gpp_direct.argtypes = [_L, _L, _L, _P, _P, _L, _P, _L, _P, _P, _P, _P, _P, _P]
        lib.orc_gpp_factored.argtypes = [_L, _L, _L, _P, _P, _L, _P, _P, _P, _P, _P, _P, _P]
        lib.orc_gpp_sx.argtypes = [_L, _L, _L, _L, _P, _P, _L, _P, _L, _P, _P, _P, _P, _P, _P, ctypes.c_int]
        lib.orc_set_pole_guard.argtypes = [_D]
        lib.orc_set_pole_guard.restype = None
        lib.orc_compute_fact.argtypes = [_D, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_D), ctypes.POINTER(_D)]
        lib.orc_compute_fact.restype = None
        lib.orc_gpp_backward.argtypes = [_L, _L, _L, _P, _P, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        lib.orc_gpp_backward_direct.argtypes = [_L, _L, _L, _P, _P, _L, _P, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        lib.orc_gpp_factored_ld.argtypes = [_L, _L, _L, _P, _P, _L, _P, _P, _P, _P, _P, _P, _P]
        lib.orc_gpp_direct_ld.argtypes = [_L, _L, _L, _P, _P, _L, _P, _L, _P, _P, _P, _P, _P, _P]
        lib.orc_ff_achs.argtypes = [_L, _L, _L, _L, _P, _P, _L, _P, _P, _P, _P, _P]
        lib.orc_ff_asx.argtypes = [_L, _L, _L, _L, _L, _D, _D, _D, _P, _P, _P, _P, _L, _P, _P, _P, _P, _P, _P]
        lib.orc_ff_cor.argtypes = [_L, _L, _L, _L, _L, _L, _D, _D, _P, _P, _P, _P, _L, _P, _P, _P, _P, _P, _P]
        lib.orc_ff_asx_iw.argtypes = lib.orc_ff_asx.argtypes
        lib.orc_ff_cor_iw.argtypes = lib.orc_ff_cor.argtypes
        self.lib = lib

    def _guarded(self, pole_guard, fn):
        """Runs fn() with the oracle's near-pole guard set to pole_guard."""
        self.lib.orc_set_pole_guard(float(pole_guard))
        try:
            return fn()
        finally:
            self.lib.orc_set_pole_guard(0.0)

    def gpp(self, g, factored: bool = False, pole_guard: float = 0.0) -> np.ndarray:
        if pole_guard:
            return self._guarded(pole_guard, lambda: self.gpp(g, factored))
        out = np.zeros(3, dtype=np.complex128)
        if factored:
            assert g.wx_band_stride == 0
            st = self.lib.orc_gpp_factored(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                           len(g.indinv), _p(g.wx_array), _p(g.wtilde_array), _p(g.aqsmtemp),
                                           _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul), _p(out))
        else:
            st = self.lib.orc_gpp_direct(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                         len(g.indinv), _p(g.wx_array), g.wx_band_stride, _p(g.wtilde_array),
                                         _p(g.aqsmtemp), _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul), _p(out))
        if st != 0:
            raise ValueError("oracle rejected the GPP inputs")
        return out

    def gpp_sx(self, g, nvband: int | None = None, factored: bool = False, pole_guard: float = 0.0) -> np.ndarray:
        """Screened exchange of the occupied bands (asxtemp), specified from
        the GPP model (not in the reference: parity unpinned)."""
        if pole_guard:
            return self._guarded(pole_guard, lambda: self.gpp_sx(g, nvband, factored))
        nv = g.nvband if nvband is None else nvband
        out = np.zeros(3, dtype=np.complex128)
        st = self.lib.orc_gpp_sx(g.number_bands, nv, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                 len(g.indinv), _p(g.wx_array), g.wx_band_stride if not factored else 0,
                                 _p(g.wtilde_array), _p(g.aqsmtemp), _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul),
                                 _p(out), int(factored))
        if st != 0:
            raise ValueError("oracle rejected the GPP inputs")
        return out

    def gpp_direct_ld(self, g) -> np.ndarray:
        """Band-loop GPP sum (any wx_band_stride) with long-double outputs:
        6 np.longdouble (re, im per iw)."""
        out = np.zeros(6, dtype=np.longdouble)
        st = self.lib.orc_gpp_direct_ld(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                        len(g.indinv), _p(g.wx_array), g.wx_band_stride, _p(g.wtilde_array),
                                        _p(g.aqsmtemp), _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul),
                                        out.ctypes.data)
        if st != 0:
            raise ValueError("oracle rejected the GPP inputs")
        return out

    def gpp_ld(self, g) -> np.ndarray:
        """Factored GPP sum with long-double outputs: 6 np.longdouble (re, im per iw)."""
        out = np.zeros(6, dtype=np.longdouble)
        st = self.lib.orc_gpp_factored_ld(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                          len(g.indinv), _p(g.wx_array), _p(g.wtilde_array), _p(g.aqsmtemp),
                                          _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul), out.ctypes.data)
        if st != 0:
            raise ValueError("oracle rejected the GPP inputs")
        return out

    def gpp_backward(self, g, gcot, direct: bool = False):
        """(grad_wtilde [P][G], grad_I_eps [P][G], dachtemp/domega [3]) complex128.
        direct (implied by a band-dependent wx): the band-loop form,
        O(nb P G), small sizes only."""
        gc = np.ascontiguousarray(np.asarray(gcot, dtype=np.complex128).reshape(3))
        gw = np.zeros((g.ngpown, g.ncouls), np.complex128)
        gi = np.zeros((g.ngpown, g.ncouls), np.complex128)
        dw = np.zeros(3, np.complex128)
        if direct or g.wx_band_stride:
            st = self.lib.orc_gpp_backward_direct(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index),
                                                  _p(g.indinv), len(g.indinv), _p(g.wx_array), g.wx_band_stride,
                                                  _p(g.wtilde_array), _p(g.aqsmtemp), _p(g.aqsntemp),
                                                  _p(g.I_eps_array), _p(g.vcoul), _p(gc), _p(gw), _p(gi), _p(dw))
            if st != 0:
                raise ValueError("oracle rejected the GPP inputs")
            return gw, gi, dw
        st = self.lib.orc_gpp_backward(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                       len(g.indinv), _p(g.wx_array), _p(g.wtilde_array), _p(g.aqsmtemp),
                                       _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul), _p(gc), _p(gw), _p(gi),
                                       _p(dw))
        if st != 0:
            raise ValueError("oracle rejected the GPP inputs")
        return gw, gi, dw

    def compute_fact(self, wx: float, grid: np.ndarray, loop: int, flag_occ: bool):
        i, f1, f2 = ctypes.c_int(0), _D(0.0), _D(0.0)
        self.lib.orc_compute_fact(wx, len(grid), _p(grid), loop, int(flag_occ), ctypes.byref(i), ctypes.byref(f1),
                                  ctypes.byref(f2))
        return i.value, f1.value, f2.value

    def achs(self, f) -> complex:
        out = np.zeros(1, dtype=np.complex128)
        st = self.lib.orc_ff_achs(f.number_bands, f.ngpown, f.ncouls, f.nFreq, _p(f.inv_igp_index), _p(f.indinv),
                                  len(f.indinv), _p(f.aqsntemp), _p(f.aqsmtemp), _p(f.I_epsR_array), _p(f.vcoul),
                                  _p(out))
        if st != 0:
            raise ValueError("oracle rejected the FF inputs")
        return complex(out[0])

    def asx(self, f, per_iw: bool = False) -> np.ndarray:
        """asxDtemp; per_iw: wx = freqevalmin - ekq + iw * freqevalstep per iw."""
        out = np.zeros(max(f.nfreqeval, 1), dtype=np.complex128)
        fn = self.lib.orc_ff_asx_iw if per_iw else self.lib.orc_ff_asx
        st = fn(f.nvband, f.nfreqeval, f.ncouls, f.ngpown, f.nFreq, f.freqevalmin, f.freqevalstep,
                f.occ, _p(f.ekq), _p(f.dFreqGrid), _p(f.inv_igp_index), _p(f.indinv),
                len(f.indinv), _p(f.aqsmtemp), _p(f.aqsntemp), _p(f.vcoul), _p(f.I_epsR_array),
                _p(f.I_epsA_array), _p(out))
        if st != 0:
            raise ValueError("oracle rejected the FF inputs")
        return out[:f.nfreqeval]

    def cor(self, f, per_iw: bool = False) -> np.ndarray:
        """achDtemp_cor; per_iw as in asx."""
        out = np.zeros(max(f.nfreqeval, 1), dtype=np.complex128)
        fn = self.lib.orc_ff_cor_iw if per_iw else self.lib.orc_ff_cor
        st = fn(f.number_bands, f.nvband, f.nfreqeval, f.ncouls, f.ngpown, f.nFreq, f.freqevalmin,
                f.freqevalstep, _p(f.ekq), _p(f.dFreqGrid), _p(f.inv_igp_index), _p(f.indinv),
                len(f.indinv), _p(f.aqsmtemp), _p(f.aqsntemp), _p(f.vcoul), _p(f.I_epsR_array),
                _p(f.I_epsA_array), _p(out))
        if st != 0:
            raise ValueError("oracle rejected the FF inputs")
        return out[:f.nfreqeval]


class Reference:
    """The reference's own kernels (compiled unmodified into libbgwref.so)."""

    def __init__(self, path: Path = REF_LIB):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (needs the reference tree; make -C oracle ref)")
        lib = ctypes.CDLL(str(path))
        lib.ref_gpp_noflagocc.argtypes = [_L, _L, _L, _P, _P, _L, _P, _P, _P, _P, _P, _P, _P]
        lib.ref_gpp_noflagocc.restype = None
        lib.ref_ff_achs.argtypes = [_L, _L, _L, _L, _P, _P, _L, _P, _P, _P, _P, _P]
        lib.ref_ff_achs.restype = None
        lib.ref_ff_asx.argtypes = [_L, _L, _L, _L, _L, _D, _D, _D, _P, _L, _P, _P, _P, _L, _P, _P, _P, _P, _P, _P]
        lib.ref_ff_asx.restype = None
        lib.ref_ff_cor.argtypes = [_L, _L, _L, _L, _L, _L, _D, _D, _P, _P, _P, _P, _L, _P, _P, _P, _P, _P, _P]
        lib.ref_ff_cor.restype = None
        lib.ref_num_threads.restype = ctypes.c_int
        lib.ref_compute_fact.argtypes = [_D, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_D), ctypes.POINTER(_D)]
        lib.ref_compute_fact.restype = None
        self.lib = lib

    def compute_fact(self, wx: float, grid: np.ndarray, loop: int, flag_occ: bool):
        """(ifreq, fact1, fact2) of the reference's own compute_fact (FF/ff.cpp:103-152)."""
        g = np.ascontiguousarray(grid, dtype=np.float64)
        i, f1, f2 = ctypes.c_int(0), _D(0.0), _D(0.0)
        self.lib.ref_compute_fact(wx, len(g), _p(g), loop, int(flag_occ), ctypes.byref(i), ctypes.byref(f1),
                                  ctypes.byref(f2))
        return i.value, f1.value, f2.value

    @staticmethod
    def available() -> bool:
        return REF_LIB.exists()

    def num_threads(self) -> int:
        return int(self.lib.ref_num_threads())

    def gpp(self, g) -> np.ndarray:
        assert g.wx_band_stride == 0, "the reference has a band-independent wx_array"
        out = np.zeros(3, dtype=np.complex128)
        self.lib.ref_gpp_noflagocc(g.number_bands, g.ngpown, g.ncouls, _p(g.inv_igp_index), _p(g.indinv),
                                   len(g.indinv), _p(g.wx_array), _p(g.wtilde_array), _p(g.aqsmtemp),
                                   _p(g.aqsntemp), _p(g.I_eps_array), _p(g.vcoul), _p(out))
        return out

    def achs(self, f) -> complex:
        out = np.zeros(1, dtype=np.complex128)
        self.lib.ref_ff_achs(f.number_bands, f.ngpown, f.ncouls, f.nFreq, _p(f.inv_igp_index), _p(f.indinv),
                             len(f.indinv), _p(f.aqsntemp), _p(f.aqsmtemp), _p(f.I_epsR_array), _p(f.vcoul), _p(out))
        return complex(out[0])

    def asx(self, f) -> np.ndarray:
        out = np.zeros(max(f.nfreqeval, 1), dtype=np.complex128)
        self.lib.ref_ff_asx(f.nvband, f.nfreqeval, f.ncouls, f.ngpown, f.nFreq, f.freqevalmin, f.freqevalstep, f.occ,
                            _p(f.ekq), f.number_bands, _p(f.dFreqGrid), _p(f.inv_igp_index), _p(f.indinv),
                            len(f.indinv), _p(f.aqsmtemp), _p(f.aqsntemp), _p(f.vcoul), _p(f.I_epsR_array),
                            _p(f.I_epsA_array), _p(out))
        return out[:f.nfreqeval]

    def cor(self, f) -> np.ndarray:
        out = np.zeros(max(f.nfreqeval, 1), dtype=np.complex128)
        self.lib.ref_ff_cor(f.number_bands, f.nvband, f.nfreqeval, f.ncouls, f.ngpown, f.nFreq, f.freqevalmin,
                            f.freqevalstep, _p(f.ekq), _p(f.dFreqGrid), _p(f.inv_igp_index), _p(f.indinv),
                            len(f.indinv), _p(f.aqsmtemp), _p(f.aqsntemp), _p(f.vcoul), _p(f.I_epsR_array),
                            _p(f.I_epsA_array), _p(out))
        return out[:f.nfreqeval]
