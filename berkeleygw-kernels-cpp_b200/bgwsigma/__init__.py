"""bgwsigma -- Python binding of libbgwsigma.so (include/bgw_sigma.h).

The product is the C ABI library; this module is the thin host-side mirror of
the reference's kernel interface used by tests and benchmarks:

  noflagOCC_solver(inp)      GPP/gpp.cpp:307-402     -> complex128[3]  (achtemp)
  achsDtemp_Kernel(inp)      FF/ff.cpp:171-209       -> complex        (achsDtemp)
  asxDtemp_Kernel(inp)       FF/ff.cpp:211-293       -> complex128[nfreqeval]
  achDtemp_cor_Kernel(inp)   FF/ff.cpp:295-379       -> complex128[nfreqeval]
  ff_sigma(inp)              the three FF sums in one call

Inputs are GppInputs / FFInputs (bgwsigma.inputs) holding either host
numpy arrays (BGW_MEMORY_HOST: the library copies them to the GPU) or CUDA
torch tensors (BGW_MEMORY_DEVICE).  Errors raise BgwError with the C status.
There is no CPU fallback: without the CUDA library or a GPU every call
raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from . import build as _build
from .inputs import FFInputs, GppInputs  # noqa: F401

BGW_OK = 0
STATUS = {0: "BGW_OK", -1: "BGW_ERR_INVALID_ARG", -2: "BGW_ERR_INDEX", -3: "BGW_ERR_CUDA",
          -4: "BGW_ERR_ALLOC", -5: "BGW_ERR_NO_DEVICE", -6: "BGW_ERR_TIMEOUT", -7: "BGW_ERR_UNSUPPORTED",
          -8: "BGW_ERR_CHECK"}
MEMORY = {"host": 0, "device": 1}
PRECISION = {"fp64": 0, "mixed": 1}
GPP_ALGO = {"bandloop": 0, "factored": 1, "auto": 2}
FLAG_ASYNC = 1
FLAG_PROFILE = 2
FLAG_FF_SLICE_ALL = 4
FLAG_FF_STAGED = 16
FLAG_FF_WX_PER_IW = 8

# Every extern "C" symbol include/bgw_sigma.h declares.
EXPORTS = ("bgw_options_init", "bgw_noflagOCC_solver", "bgw_achsDtemp_Kernel", "bgw_asxDtemp_Kernel",
           "bgw_achDtemp_cor_Kernel", "bgw_ff_sigma", "bgw_status_string", "bgw_abi_version",
           "bgw_launch_count", "bgw_measure_fp64_peak", "bgw_release_workspace", "bgw_last_profile",
           "bgw_noflagOCC_solver_noalloc", "bgw_noflagOCC_solver_backward", "bgw_gpp_batch_create",
           "bgw_gpp_batch_execute", "bgw_gpp_batch_info", "bgw_gpp_batch_destroy", "bgw_gpp_sigma",
           "bgw_debug_inject_stall", "bgw_fill_uniform", "bgw_debug_rcp_probe")


class BgwError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn}: {STATUS.get(status, status)} ({msg})")
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("memory", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("gpp_algorithm", ctypes.c_int32), ("wx_band_stride", ctypes.c_int64), ("device", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("stream", ctypes.c_void_p), ("device_status", ctypes.c_void_p),
                ("pole_guard", ctypes.c_double), ("mixed_order", ctypes.c_int32)]


class Profile(ctypes.Structure):
    _fields_ = [("main_kernel_ms", ctypes.c_double), ("device_ms", ctypes.c_double), ("flops", ctypes.c_double),
                ("main_bytes", ctypes.c_double), ("main_launches", ctypes.c_int32),
                ("total_launches", ctypes.c_int32), ("main_kernel", ctypes.c_char * 48)]

    def as_dict(self):
        return {"main_kernel": self.main_kernel.decode(), "main_kernel_ms": self.main_kernel_ms,
                "device_ms": self.device_ms, "flops": self.flops, "main_bytes": self.main_bytes,
                "main_launches": self.main_launches, "total_launches": self.total_launches}


class GppInstance(ctypes.Structure):
    _fields_ = [("number_bands", ctypes.c_int64), ("ngpown", ctypes.c_int64), ("ncouls", ctypes.c_int64),
                ("inv_igp_index", ctypes.c_void_p), ("indinv", ctypes.c_void_p), ("indinv_len", ctypes.c_int64),
                ("wx_array", ctypes.c_void_p), ("wx_band_stride", ctypes.c_int64), ("wtilde_array", ctypes.c_void_p),
                ("aqsmtemp", ctypes.c_void_p), ("aqsntemp", ctypes.c_void_p), ("I_eps_array", ctypes.c_void_p),
                ("vcoul", ctypes.c_void_p), ("achtemp", ctypes.c_void_p)]


_LIB = None
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double


def lib_path() -> Path:
    """The library to load: $BGW_SIGMA_LIB (e.g. the debug build
    lib/libbgwsigma_check.so) or lib/libbgwsigma.so."""
    env = os.environ.get("BGW_SIGMA_LIB")
    return Path(env) if env else _build.LIB


def load(build_if_needed: bool = True) -> ctypes.CDLL:
    """Loads libbgwsigma.so (building it first if its sources changed)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if build_if_needed and os.environ.get("BGW_SIGMA_NO_BUILD") != "1":
        if path == _build.CHECK_LIB:
            _build.build_check()
        elif path == _build.LIB:
            _build.build()
    if not path.exists():
        raise RuntimeError(f"libbgwsigma.so not built ({path}); run berkeleygw-kernels-cpp_b200/bgwsigma/build.py")
    lib = ctypes.CDLL(str(path))
    lib.bgw_options_init.argtypes = [ctypes.POINTER(Options)]
    lib.bgw_options_init.restype = None
    lib.bgw_status_string.argtypes = [ctypes.c_int]
    lib.bgw_status_string.restype = ctypes.c_char_p
    lib.bgw_abi_version.restype = ctypes.c_int
    lib.bgw_launch_count.restype = ctypes.c_uint64
    lib.bgw_measure_fp64_peak.argtypes = [ctypes.c_int32, ctypes.POINTER(_D), ctypes.POINTER(_D)]
    lib.bgw_release_workspace.argtypes = [ctypes.c_int32]
    lib.bgw_debug_inject_stall.argtypes = [ctypes.c_int64]
    lib.bgw_debug_rcp_probe.argtypes = [_P, _I64, _P, _P, _P, ctypes.c_int32]
    lib.bgw_last_profile.argtypes = [ctypes.POINTER(Profile)]
    opt = ctypes.POINTER(Options)
    lib.bgw_fill_uniform.argtypes = [_P, _I64, ctypes.c_uint64, ctypes.c_uint64, _I64, _D, _D, _D, _D, opt]
    lib.bgw_noflagOCC_solver.argtypes = [_I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, opt]
    lib.bgw_gpp_sigma.argtypes = [_I64, _I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, opt]
    lib.bgw_noflagOCC_solver_noalloc.argtypes = [_I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P,
                                                 ctypes.c_int32, _P]
    lib.bgw_noflagOCC_solver_backward.argtypes = [_I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P,
                                                  _P, _P, opt]
    lib.bgw_gpp_batch_create.argtypes = [ctypes.POINTER(GppInstance), _I64, opt, ctypes.POINTER(_P)]
    lib.bgw_gpp_batch_execute.argtypes = [_P, opt]
    lib.bgw_gpp_batch_info.argtypes = [_P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_int64)]
    lib.bgw_gpp_batch_destroy.argtypes = [_P]
    lib.bgw_achsDtemp_Kernel.argtypes = [_I64, _I64, _I64, _P, _P, _I64, _P, _P, _P, _I64, _P, _P, opt]
    lib.bgw_asxDtemp_Kernel.argtypes = [_I64, _I64, _I64, _I64, _I64, _D, _D, _D, _P, _P, _P, _P, _I64, _P, _P,
                                        _I64, _P, _P, _P, _P, opt]
    lib.bgw_achDtemp_cor_Kernel.argtypes = [_I64, _I64, _I64, _I64, _I64, _I64, _D, _D, _P, _P, _P, _P, _I64, _P,
                                            _P, _P, _P, _P, _P, opt]
    lib.bgw_ff_sigma.argtypes = [_I64, _I64, _I64, _I64, _I64, _I64, _D, _D, _D, _P, _P, _P, _P, _I64, _P, _P, _P,
                                 _P, _P, _P, _P, _P, opt]
    for fn in EXPORTS:
        if fn.startswith("bgw_") and fn not in ("bgw_options_init", "bgw_status_string", "bgw_launch_count"):
            getattr(lib, fn).restype = ctypes.c_int
    _LIB = lib
    return lib


def launch_count() -> int:
    return int(load().bgw_launch_count())


def measure_fp64_peak(device: int = -1):
    """(DFMA TFLOP/s, DMMA TFLOP/s) measured by the library's microkernels."""
    a, b = _D(), _D()
    _check("bgw_measure_fp64_peak", load().bgw_measure_fp64_peak(device, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def inject_stall(step: int = -1):
    """Test hook of the timeout path (bgw_debug_inject_stall): the staged
    kernels launched from now on let the wait of CTA-local step `step` run
    out, and their calls raise BgwError(BGW_ERR_TIMEOUT); -1 turns it off."""
    _check("bgw_debug_inject_stall", load().bgw_debug_inject_stall(int(step)))


def rcp_probe(values, device: int = -1):
    """(refined, seed, f32) reciprocals of `values` evaluated by the
    library's device code (bgw_debug_rcp_probe)."""
    x = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
    r, s, f = np.empty_like(x), np.empty_like(x), np.empty(x.shape, np.float32)
    _check("bgw_debug_rcp_probe", load().bgw_debug_rcp_probe(_ptr(x), x.size, _ptr(r), _ptr(s), _ptr(f), device))
    return r, s, f


def fill_uniform(out, seed: int, stream_id: int, offset: int, lo_even: float, hi_even: float, lo_odd: float,
                 hi_odd: float, *, stream=None):
    """Fills `out` (a float64 CUDA tensor or host numpy array, contiguous)
    with words offset .. offset + out.size - 1 of Philox stream (seed,
    stream_id), mapped to the given ranges (bgw_fill_uniform)."""
    lib = load()
    if _is_torch(out):
        n, mem = out.numel(), ("device" if out.is_cuda else "host")
        ok = out.dtype.is_floating_point and out.element_size() == 8
    else:
        n, mem, ok = out.size, "host", out.dtype == np.float64
    if not ok:
        raise ValueError("out must hold float64 values")
    dev = out.device.index if mem == "device" and out.device.index is not None else -1
    o = make_options(mem, device=dev, stream=_stream_handle(None, stream))
    _check("bgw_fill_uniform", lib.bgw_fill_uniform(_ptr(out), n, seed, stream_id, offset, lo_even, hi_even, lo_odd,
                                                    hi_odd, ctypes.byref(o)))
    return out


def last_profile() -> dict:
    """Profile of this thread's last synchronous call made with FLAG_PROFILE."""
    p = Profile()
    _check("bgw_last_profile", load().bgw_last_profile(ctypes.byref(p)))
    return p.as_dict()


def _check(fn: str, status: int):
    if status != BGW_OK:
        raise BgwError(fn, status, load().bgw_status_string(status).decode())


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x) -> int:
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    if not isinstance(x, np.ndarray) or not x.flags.c_contiguous:
        raise ValueError("array must be a C-contiguous numpy array")
    return x.ctypes.data


def _where(inp) -> str:
    kinds = set()
    for k in inp.ARRAYS:
        a = getattr(inp, k)
        kinds.add("device" if (_is_torch(a) and a.is_cuda) else "host")
    if len(kinds) != 1:
        raise ValueError("all arrays must be on the host or all on the GPU")
    return kinds.pop()


def make_options(memory="host", precision="fp64", algorithm="auto", wx_band_stride=0, device=-1, stream=None,
                 flags=0, device_status=None, pole_guard=0.0, mixed_order=None) -> Options:
    o = Options()
    load().bgw_options_init(ctypes.byref(o))
    o.memory = MEMORY[memory]
    o.precision = PRECISION[precision]
    o.gpp_algorithm = GPP_ALGO[algorithm]
    o.wx_band_stride = int(wx_band_stride)
    o.device = int(device)
    o.flags = int(flags)
    o.stream = stream
    o.device_status = device_status
    o.pole_guard = float(pole_guard)
    if mixed_order is not None:
        o.mixed_order = int(mixed_order)
    return o


def _stream_handle(inp, stream):
    if stream is not None:
        return int(stream)
    return None


def noflagOCC_solver(inp: GppInputs, *, precision="fp64", algorithm="auto", stream=None, out=None,
                     flags=0, device_status=None, pole_guard=0.0, mixed_order=None) -> np.ndarray:
    """achtemp[3] (complex128).  `out`: optional preallocated output (host
    numpy complex128[3] or a CUDA tensor for device-resident inputs).
    `pole_guard` > 0: terms with |wx - wtilde| below it contribute zero."""
    lib = load()
    mem = _where(inp)
    if out is None:
        if mem == "host":
            out = np.zeros(3, dtype=np.complex128)
        else:
            import torch
            out = torch.zeros(3, dtype=torch.complex128, device=inp.wtilde_array.device)
    o = make_options(mem, precision, algorithm, inp.wx_band_stride, stream=_stream_handle(inp, stream),
                     flags=flags, device_status=device_status, pole_guard=pole_guard, mixed_order=mixed_order)
    st = lib.bgw_noflagOCC_solver(inp.number_bands, inp.ngpown, inp.ncouls, _ptr(inp.inv_igp_index),
                                  _ptr(inp.indinv), len(inp.indinv), _ptr(inp.wx_array), _ptr(inp.wtilde_array),
                                  _ptr(inp.aqsmtemp), _ptr(inp.aqsntemp), _ptr(inp.I_eps_array), _ptr(inp.vcoul),
                                  _ptr(out), ctypes.byref(o))
    _check("bgw_noflagOCC_solver", st)
    return out


def gpp_sigma(inp: GppInputs, nvband=None, *, want_ach=True, want_asx=True, precision="fp64", algorithm="auto",
              stream=None, flags=0, device_status=None, pole_guard=0.0, mixed_order=None):
    """(achtemp[3], asxtemp[3]) complex128: the Coulomb-hole sum over all
    bands and the GPP screened exchange of the occupied bands n1 < nvband
    (default: inp.nvband).  A result not asked for is None."""
    lib = load()
    mem = _where(inp)
    nv = inp.nvband if nvband is None else int(nvband)

    def buf():
        if mem == "host":
            return np.zeros(3, dtype=np.complex128)
        import torch
        return torch.zeros(3, dtype=torch.complex128, device=inp.wtilde_array.device)

    ach = buf() if want_ach else None
    asx = buf() if want_asx else None
    o = make_options(mem, precision, algorithm, inp.wx_band_stride, stream=_stream_handle(inp, stream),
                     flags=flags, device_status=device_status, pole_guard=pole_guard, mixed_order=mixed_order)
    st = lib.bgw_gpp_sigma(inp.number_bands, nv, inp.ngpown, inp.ncouls, _ptr(inp.inv_igp_index),
                           _ptr(inp.indinv), len(inp.indinv), _ptr(inp.wx_array), _ptr(inp.wtilde_array),
                           _ptr(inp.aqsmtemp), _ptr(inp.aqsntemp), _ptr(inp.I_eps_array), _ptr(inp.vcoul),
                           _nz(ach), _nz(asx), ctypes.byref(o))
    _check("bgw_gpp_sigma", st)
    return ach, asx


def noflagOCC_solver_backward(inp: GppInputs, grad_achtemp, *, want_wtilde=True, want_I_eps=True,
                              want_domega=True, stream=None, flags=0, pole_guard=0.0, algorithm="auto"):
    """Adjoint of noflagOCC_solver.  grad_achtemp: 3 complex cotangents
    (dL/dRe + i dL/dIm of each achtemp entry).  Returns (grad_wtilde,
    grad_I_eps, dachtemp_domega) -- complex arrays [ngpown][ncouls],
    [ngpown][ncouls], [3] -- on the inputs' side (host or device)."""
    lib = load()
    mem = _where(inp)
    P, G = inp.ngpown, inp.ncouls
    if mem == "host":
        gc = np.ascontiguousarray(np.asarray(grad_achtemp, dtype=np.complex128).reshape(3))
        gw = np.zeros((P, G), np.complex128) if want_wtilde else None
        gi = np.zeros((P, G), np.complex128) if want_I_eps else None
        dw = np.zeros(3, np.complex128) if want_domega else None
    else:
        import torch
        dev = inp.wtilde_array.device
        gc = torch.as_tensor(np.asarray(grad_achtemp, dtype=np.complex128).reshape(3)).to(dev)
        gw = torch.zeros((P, G), dtype=torch.complex128, device=dev) if want_wtilde else None
        gi = torch.zeros((P, G), dtype=torch.complex128, device=dev) if want_I_eps else None
        dw = torch.zeros(3, dtype=torch.complex128, device=dev) if want_domega else None
    o = make_options(mem, "fp64", algorithm, inp.wx_band_stride, stream=_stream_handle(inp, stream), flags=flags,
                     pole_guard=pole_guard)
    st = lib.bgw_noflagOCC_solver_backward(inp.number_bands, P, G, _ptr(inp.inv_igp_index), _ptr(inp.indinv),
                                           len(inp.indinv), _ptr(inp.wx_array), _ptr(inp.wtilde_array),
                                           _ptr(inp.aqsmtemp), _ptr(inp.aqsntemp), _ptr(inp.I_eps_array),
                                           _ptr(inp.vcoul), _ptr(gc), _nz(gw), _nz(gi), _nz(dw), ctypes.byref(o))
    _check("bgw_noflagOCC_solver_backward", st)
    return gw, gi, dw


class GppBatch:
    """Many device-resident GPP instances in one persistent launch (a CUDA
    graph replayed by execute()).  `instances`: GppInputs with CUDA tensors."""

    def __init__(self, instances, *, precision="fp64", algorithm="auto", stream=None, pole_guard=0.0,
                 mixed_order=None):
        import torch
        lib = load()
        self.instances = list(instances)
        dev = self.instances[0].wtilde_array.device
        self.out = torch.zeros((len(self.instances), 3), dtype=torch.complex128, device=dev)
        arr = (GppInstance * len(self.instances))()
        for k, g in enumerate(self.instances):
            if _where(g) != "device":
                raise ValueError("batched instances must be CUDA tensors")
            arr[k] = GppInstance(g.number_bands, g.ngpown, g.ncouls, _ptr(g.inv_igp_index), _ptr(g.indinv),
                                 len(g.indinv), _ptr(g.wx_array), g.wx_band_stride, _ptr(g.wtilde_array),
                                 _ptr(g.aqsmtemp), _ptr(g.aqsntemp), _ptr(g.I_eps_array), _ptr(g.vcoul),
                                 self.out[k].data_ptr())
        self._arr = arr
        o = make_options("device", precision, algorithm, stream=_stream_handle(None, stream),
                         device=dev.index if dev.index is not None else -1, pole_guard=pole_guard,
                         mixed_order=mixed_order)
        h = _P()
        _check("bgw_gpp_batch_create", lib.bgw_gpp_batch_create(arr, len(self.instances), ctypes.byref(o),
                                                                ctypes.byref(h)))
        self.handle = h

    def execute(self, stream=None, flags=0):
        o = make_options("device", stream=_stream_handle(None, stream), flags=flags)
        _check("bgw_gpp_batch_execute", load().bgw_gpp_batch_execute(self.handle, ctypes.byref(o)))
        return self.out

    def info(self):
        ke, grid, items = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        _check("bgw_gpp_batch_info", load().bgw_gpp_batch_info(self.handle, ctypes.byref(ke), ctypes.byref(grid),
                                                                ctypes.byref(items)))
        return {"elems_per_thread": ke.value, "grid": grid.value, "items": items.value}

    def close(self):
        if getattr(self, "handle", None):
            load().bgw_gpp_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ff_out(inp: FFInputs, n: int, mem: str):
    if mem == "host":
        return np.zeros(n, dtype=np.complex128)
    import torch
    return torch.zeros(n, dtype=torch.complex128, device=inp.aqsmtemp.device)


def _nz(x):
    return None if x is None else _ptr(x)


def ff_sigma(inp: FFInputs, *, achs=True, asx=True, cor=True, precision="fp64", stream=None, flags=0):
    """(achsDtemp, asxDtemp[nfreqeval], achDtemp_cor[nfreqeval]); skipped sums are None."""
    lib = load()
    mem = _where(inp)
    o_achs = _ff_out(inp, 1, mem) if achs else None
    o_asx = _ff_out(inp, max(inp.nfreqeval, 1), mem) if asx else None
    o_cor = _ff_out(inp, max(inp.nfreqeval, 1), mem) if cor else None
    o = make_options(mem, precision, stream=_stream_handle(inp, stream), flags=flags)
    st = lib.bgw_ff_sigma(inp.number_bands, inp.nvband, inp.nfreqeval, inp.ncouls, inp.ngpown, inp.nFreq,
                          inp.freqevalmin, inp.freqevalstep, inp.occ, _ptr(inp.ekq), _ptr(inp.dFreqGrid),
                          _ptr(inp.inv_igp_index), _ptr(inp.indinv), len(inp.indinv), _ptr(inp.aqsmtemp),
                          _ptr(inp.aqsntemp), _ptr(inp.vcoul), _ptr(inp.I_epsR_array), _ptr(inp.I_epsA_array),
                          _nz(o_achs), _nz(o_asx), _nz(o_cor), ctypes.byref(o))
    _check("bgw_ff_sigma", st)
    return o_achs, o_asx, o_cor


def achsDtemp_Kernel(inp: FFInputs, *, precision="fp64", stream=None, flags=0):
    lib = load()
    mem = _where(inp)
    out = _ff_out(inp, 1, mem)
    o = make_options(mem, precision, stream=_stream_handle(inp, stream), flags=flags)
    st = lib.bgw_achsDtemp_Kernel(inp.number_bands, inp.ngpown, inp.ncouls, _ptr(inp.inv_igp_index),
                                  _ptr(inp.indinv), len(inp.indinv), _ptr(inp.aqsntemp), _ptr(inp.aqsmtemp),
                                  _ptr(inp.I_epsR_array), inp.nFreq, _ptr(inp.vcoul), _ptr(out), ctypes.byref(o))
    _check("bgw_achsDtemp_Kernel", st)
    return out


def asxDtemp_Kernel(inp: FFInputs, *, precision="fp64", stream=None, flags=0):
    lib = load()
    mem = _where(inp)
    out = _ff_out(inp, max(inp.nfreqeval, 1), mem)
    o = make_options(mem, precision, stream=_stream_handle(inp, stream), flags=flags)
    st = lib.bgw_asxDtemp_Kernel(inp.nvband, inp.nfreqeval, inp.ncouls, inp.ngpown, inp.nFreq, inp.freqevalmin,
                                 inp.freqevalstep, inp.occ, _ptr(inp.ekq), _ptr(inp.dFreqGrid),
                                 _ptr(inp.inv_igp_index), _ptr(inp.indinv), len(inp.indinv), _ptr(inp.aqsmtemp),
                                 _ptr(inp.aqsntemp), inp.number_bands, _ptr(inp.vcoul), _ptr(inp.I_epsR_array),
                                 _ptr(inp.I_epsA_array), _ptr(out), ctypes.byref(o))
    _check("bgw_asxDtemp_Kernel", st)
    return out


def achDtemp_cor_Kernel(inp: FFInputs, *, precision="fp64", stream=None, flags=0):
    lib = load()
    mem = _where(inp)
    out = _ff_out(inp, max(inp.nfreqeval, 1), mem)
    o = make_options(mem, precision, stream=_stream_handle(inp, stream), flags=flags)
    st = lib.bgw_achDtemp_cor_Kernel(inp.number_bands, inp.nvband, inp.nfreqeval, inp.ncouls, inp.ngpown,
                                     inp.nFreq, inp.freqevalmin, inp.freqevalstep, _ptr(inp.ekq),
                                     _ptr(inp.dFreqGrid), _ptr(inp.inv_igp_index), _ptr(inp.indinv),
                                     len(inp.indinv), _ptr(inp.aqsmtemp), _ptr(inp.aqsntemp), _ptr(inp.vcoul),
                                     _ptr(inp.I_epsR_array), _ptr(inp.I_epsA_array), _ptr(out), ctypes.byref(o))
    _check("bgw_achDtemp_cor_Kernel", st)
    return out


def to_device(inp, device="cuda"):
    """Copies every array of a GppInputs / FFInputs into CUDA torch tensors."""
    import torch

    def conv(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(device)
    return inp.map_arrays(conv)


def to_pinned(inp):
    """Copies every array into pinned host memory (numpy views on pinned
    torch storage), so host-memory calls copy at full DMA speed."""
    import torch

    def conv(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t.numpy()
    return inp.map_arrays(conv)
