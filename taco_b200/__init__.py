"""taco_b200 -- B200-native TCL4 generator engine.

Python mirror of the reference's C++ entry points for the L4(t) path, calling the
CUDA library through its C-ABI (include/taco_b200.h):

=================================  =====================================================
this module                        reference (cpp/include/taco/...)
=================================  =====================================================
System                             sys::System::build (system.hpp:201-226) + build_map
compute_triple_kernels             tcl4::compute_triple_kernels (tcl4.hpp:37-42), Exec{Cuda}
build_TCL4_generator               build_TCL4_generator_cuda_fused (backend/cuda/tcl4_fused_cuda.hpp:16-21)
build_TCL4_generator_batch         build_TCL4_generator_cuda_fused_batch (tcl4_fused_cuda.hpp:25-41)
build_correction_series            build_correction_series_cuda_fused (tcl4_fused_cuda.hpp:44-48)
propagate_rk4_dense                tcl::propagate_rk4_dense_* (rk4_dense.hpp:85-129), on the device
set_fcr_fft_pad_factor             tcl4::set_fcr_fft_pad_factor (tcl4_kernels.hpp:16-19)
=================================  =====================================================

Arrays: numpy arrays are host buffers (copied in and out inside the call); torch CUDA
tensors are device buffers (the call reads and writes them in place).  Gamma is
[nf, Nt] (row b = bucket b; the reference's column-major Nt x nf matrix).  L4 results
are returned as [T, N^2, N^2] arrays indexed [t, row, col].  Errors raise the
exception type the reference throws (ValueError for std::invalid_argument, IndexError
for std::out_of_range, OverflowError, RuntimeError).  There is no CPU fallback: every
call needs the CUDA library and a GPU.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _capi
from ._capi import (TacoError, TacoInvalidArgument, TacoOutOfRange, TacoOverflow,  # noqa: F401
                    TACO_PREC_FP32, TACO_PREC_FP64)
from .inputs import System, bcf_fft, gamma_trapz, spin_boson_system  # noqa: F401
from . import autotune as _autotune  # noqa: F401  (schedules load with the library)

__all__ = [
    "System", "bcf_fft", "gamma_trapz", "spin_boson_system", "compute_triple_kernels",
    "build_TCL4_generator", "build_TCL4_generator_batch", "build_correction_series", "build_instances",
    "propagate_rk4_dense", "l4_coefficients", "Tcl4Plan", "set_fcr_fft_pad_factor", "get_fcr_fft_pad_factor",
    "version", "device_count", "kernel_launches", "profile", "compute_triple_kernels_batch", "tcl2_generator_series", "gamma_trapz_device",
    "propagate_tcl", "gamma_trapz_device_batch", "set_work_budget", "fft_length", "build_mikx", "assemble_liouvillian", "gw_to_liouvillian",
    "set_fp32_guard", "fp32_guard", "fp32_guard_stats", "set_fused_conv", "fused_conv", "release_workspace",
    "set_guard_chunk_bytes",
]


def version() -> str:
    return _capi.lib().taco_version().decode()


def device_count() -> int:
    n = ct.c_int(0)
    _capi.check(_capi.lib().taco_device_count(ct.byref(n)))
    return n.value


def kernel_launches() -> int:
    """Kernels launched by the library since the process started."""
    n = ct.c_uint64(0)
    _capi.check(_capi.lib().taco_kernel_launches(ct.byref(n)))
    return int(n.value)


class profile:
    """Context manager: per-kernel device time (CUDA events around each launch).

    >>> with taco_b200.profile() as p: ...
    >>> p.entries  # {name: (launches, total_ms)}
    """

    def __enter__(self):
        L = _capi.lib()
        _capi.check(L.taco_profile_reset())
        _capi.check(L.taco_profile_enable(1))
        self.entries = {}
        return self

    def __exit__(self, *exc):
        L = _capi.lib()
        _capi.check(L.taco_profile_enable(0))
        count = ct.c_size_t(0)
        _capi.check(L.taco_profile_get(0, None, None, None, ct.byref(count)))
        for k in range(count.value):
            name = ct.c_char_p()
            n = ct.c_uint64(0)
            ms = ct.c_double(0.0)
            _capi.check(L.taco_profile_get(k, ct.byref(name), ct.byref(n), ct.byref(ms), None))
            self.entries[name.value.decode()] = (int(n.value), float(ms.value))
        return False


def set_work_budget(nbytes: int) -> None:
    """Transient device memory of one group of a build (0: automatic).  Larger instances
    are built in slices of their frequency triples."""
    _capi.check(_capi.lib().taco_set_work_budget(int(nbytes)))


def set_fp32_guard(tol: float) -> None:
    """Precision guard of the FP32 form: leading times whose FP32 result differs from an FP64
    head by more than `tol` (relative, on the head's upper half) are rebuilt in FP64, the
    head growing fourfold up to the whole instance.  0 turns it off; default 5e-7."""
    _capi.check(_capi.lib().taco_set_fp32_guard(float(tol)))


def fp32_guard() -> float:
    """The current tolerance of the FP32 form's precision guard (0: off)."""
    v = ct.c_double(0.0)
    _capi.check(_capi.lib().taco_get_fp32_guard(ct.byref(v)))
    return v.value


def set_guard_chunk_bytes(nbytes: int) -> None:
    """Bytes of FP64 head rows the precision guard builds and patches at a time (0: default,
    1 GiB); heads beyond it go in further chunks."""
    _capi.check(_capi.lib().taco_set_guard_chunk_bytes(int(nbytes)))


def set_fused_conv(on: bool) -> None:
    """The fused F/C/R path (transforms, scans and assembly of a triple in one CTA's shared
    memory) for the FFT lengths it fits; off (the default): the four-step passes everywhere."""
    _capi.check(_capi.lib().taco_set_fused_conv(1 if on else 0))


def fused_conv() -> bool:
    """Whether the fused F/C/R path is selected."""
    v = ct.c_int(0)
    _capi.check(_capi.lib().taco_get_fused_conv(ct.byref(v)))
    return bool(v.value)


def release_workspace() -> None:
    """Free this thread's grow-only device and pinned transient buffers (after its streams
    finish); the next build allocates them again.  Plans keep their own."""
    _capi.check(_capi.lib().taco_release_workspace())


def fp32_guard_stats() -> dict:
    """What the precision guard did in this thread's last FP32 build or plan creation."""
    v = (ct.c_uint64 * 6)()
    _capi.check(_capi.lib().taco_fp32_guard_stats(v))
    keys = ("instances", "instances_with_fp64_head", "fp64_head_rows", "rows_of_those_instances",
            "instances_fully_fp64", "rounds")
    return dict(zip(keys, (int(x) for x in v)))


def fft_length(n_in: int, precision: str = "fp32", full_length: bool = False):
    """(Nfft, schedule key) the build uses for n_in consumed Gamma samples."""
    n = ct.c_size_t(0)
    k = ct.c_int(0)
    prec = {"fp64": _capi.TACO_PREC_FP64, "fp32": _capi.TACO_PREC_FP32}[precision]
    _capi.check(_capi.lib().taco_fft_length(int(n_in), prec, _capi.TACO_FULL_LENGTH_FFT if full_length else 0,
                                            ct.byref(n), ct.byref(k)))
    return int(n.value), int(k.value)


def set_fcr_fft_pad_factor(factor: int) -> None:
    _capi.lib().taco_set_fcr_fft_pad_factor(int(factor))


def get_fcr_fft_pad_factor() -> int:
    return int(_capi.lib().taco_get_fcr_fft_pad_factor())


# ----------------------------------------------------------------- helpers --
def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _torch():
    import torch
    return torch


def _ptr(x):
    if x is None:
        return None
    if _is_torch(x):
        return ct.c_void_p(x.data_ptr())
    return x.ctypes.data_as(ct.c_void_p)


def _addr(x) -> int:
    """Integer address of a numpy array's or torch tensor's data (0 for None)."""
    if x is None:
        return 0
    if _is_torch(x):
        return x.data_ptr()
    if x.flags.writeable and x.flags.c_contiguous and x.size:
        return ct.addressof(ct.c_char.from_buffer(x))  # the cheapest route for writable buffers
    return x.__array_interface__["data"][0]


def _stream_ptr(x):
    if x is not None and _is_torch(x) and x.is_cuda:
        return ct.c_void_p(_torch().cuda.current_stream(x.device).cuda_stream)
    return None


def _c128_host(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _prep_gamma(gamma):
    """-> (array, on_device).  Device tensors must be contiguous complex128 [nf, Nt]."""
    if _is_torch(gamma):
        torch = _torch()
        if gamma.is_cuda:
            if gamma.dtype != torch.complex128:
                gamma = gamma.to(torch.complex128)
            return gamma.contiguous(), True
        gamma = gamma.numpy()
    return _c128_host(gamma), False


class _View:
    """Keeps the numpy buffers of a taco_system_view alive."""

    def __init__(self, system: System):
        self.omegas = np.ascontiguousarray(system.omegas, np.float64)
        self.mirror = np.ascontiguousarray(system.mirror, np.int32)
        self.p2f = np.ascontiguousarray(np.asarray(system.pair_to_freq).T, np.int32)  # column-major
        ops = system.A_eig
        self.ops = (np.ascontiguousarray(np.stack([np.asarray(A, np.complex128).T for A in ops]))
                    if len(ops) else np.zeros((0,), np.complex128))
        self.view = _capi.SystemView(int(system.N), int(system.nf), len(ops), _addr(self.omegas),
                                     _addr(self.mirror), _addr(self.p2f),
                                     _addr(self.ops) if len(ops) else None, float(system.tol))


def _out_array(like_device, shape, dtype, device=None):
    if like_device:
        torch = _torch()
        td = torch.complex128 if dtype == np.complex128 else torch.complex64
        return torch.empty(shape, dtype=td, device=device)
    return np.empty(shape, dtype=dtype)


def _system_view(system: System) -> _View:
    """The _View of `system`, reused while its arrays hold the same contents.

    Batched calls marshal hundreds of systems per call; the key (the bytes, types and shapes
    of the small arrays a view copies) costs a fraction of building the view again.
    Systems whose fields are not numpy arrays are marshalled every call.
    """
    om, mi, pf, ops = system.omegas, system.mirror, system.pair_to_freq, system.A_eig
    if not (type(om) is np.ndarray and type(mi) is np.ndarray and type(pf) is np.ndarray
            and all(type(A) is np.ndarray for A in ops)):
        return _View(system)
    key = (system.N, system.nf, system.tol, om.dtype.char, om.shape, om.tobytes(), mi.dtype.char, mi.shape,
           mi.tobytes(), pf.dtype.char, pf.shape, pf.tobytes(),
           tuple((A.dtype.char, A.shape, A.tobytes()) for A in ops))
    cached = getattr(system, "_taco_view", None)
    if cached is not None and cached[0] == key:
        return cached[1]
    v = _View(system)
    try:
        system._taco_view = (key, v)
    except AttributeError:  # objects without a __dict__ are marshalled every call
        pass
    return v


def _l4_view(buf, N2):
    """[T, N^2*N^2] column-major matrices -> [T, N^2, N^2] indexed [t, row, col]."""
    T = buf.shape[0]
    if _is_torch(buf):
        return buf.view(T, N2, N2).transpose(1, 2)
    return buf.reshape(T, N2, N2).transpose(0, 2, 1)


# --------------------------------------------------------------- entry points --
def compute_triple_kernels(system: System, gamma, dt: float, nmax: int = 2, method: int = 0):
    """F, C, R series of every frequency triple: arrays [nf, nf, nf, Nt] (complex128).

    ``nmax`` is accepted and ignored, as in the reference (tcl4.cpp:117).
    """
    del nmax
    g, dev = _prep_gamma(gamma)
    nf, Nt = g.shape
    v = _View(system)
    shape = (nf, nf, nf, Nt)
    outs = [_out_array(dev, shape, np.complex128, g.device if dev else None) for _ in range(3)]
    flags = (_capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE) if dev else 0
    _capi.check(_capi.lib().taco_compute_triple_kernels(ct.byref(v.view), _ptr(g), Nt, float(dt), int(method),
                                                        _ptr(outs[0]), _ptr(outs[1]), _ptr(outs[2]), flags,
                                                        _stream_ptr(g)))
    return tuple(outs)


def compute_triple_kernels_batch(systems, gammas, dts, method: int = 0):
    """compute_triple_kernels for many instances with CUDA tensors (batching form): one
    (F, C, R) tuple of [nf, nf, nf, Nt] complex128 tensors per instance."""
    if isinstance(dts, (int, float)):
        dts = [float(dts)] * len(systems)
    if not (len(systems) == len(gammas) == len(dts)):
        raise ValueError("systems, gammas and dts must have equal lengths")
    reqs = (_capi.FcrRequest * len(systems))()
    keep, results = [], []
    for k, (system, gamma, dt) in enumerate(zip(systems, gammas, dts)):
        g, dev = _prep_gamma(gamma)
        if not dev:
            raise ValueError("compute_triple_kernels_batch needs CUDA tensors for gamma")
        nf, Nt = g.shape
        v = _View(system)
        outs = [_out_array(True, (nf, nf, nf, Nt), np.complex128, g.device) for _ in range(3)]
        keep += [g, v]
        reqs[k].sys = v.view
        reqs[k].gamma = _addr(g)
        reqs[k].Nt = Nt
        reqs[k].dt = float(dt)
        reqs[k].F, reqs[k].C, reqs[k].R = _addr(outs[0]), _addr(outs[1]), _addr(outs[2])
        results.append(tuple(outs))
    if results:
        _capi.check(_capi.lib().taco_compute_triple_kernels_batch(reqs, len(results), int(method),
                                                                  _stream_ptr(keep[0])))
    return results


def build_TCL4_generator_batch(system: System, gamma, dt: float, time_indices=None, method: int = 0,
                               precision: str = "fp64", full_length: bool = False, out=None,
                               return_fcr_ms: bool = False):
    """L4 at each requested time index (all of [0, Nt) when ``time_indices`` is None/empty).

    precision "fp64": complex128 (the plain path); "fp32": FP32 FFT convolutions and
    contraction, FP64 phases and carries, complex64 results.  The FFT length follows
    max(time_indices)+1 (F/C/R(t) depend on gamma[0..t] only); ``full_length`` sizes it
    from Nt as the reference does (same results, more work).
    """
    g, dev = _prep_gamma(gamma)
    nf, Nt = g.shape
    prec = {"fp64": _capi.TACO_PREC_FP64, "fp32": _capi.TACO_PREC_FP32}[precision]
    tid = None if time_indices is None else np.ascontiguousarray(time_indices, dtype=np.uint32)
    if tid is not None and tid.size == 0:
        tid = None
    T = Nt if tid is None else tid.size
    N2 = int(system.N) ** 2
    dtype = np.complex128 if prec == _capi.TACO_PREC_FP64 else np.complex64
    if out is None:
        out = _out_array(dev, (T, N2 * N2), dtype, g.device if dev else None)
    flags = (_capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE) if dev else 0
    if full_length:
        flags |= _capi.TACO_FULL_LENGTH_FFT
    v = _View(system)
    ms = ct.c_double(0.0)
    _capi.check(_capi.lib().taco_tcl4_build_batch(ct.byref(v.view), _ptr(g), Nt, float(dt), _ptr(tid),
                                                  0 if tid is None else tid.size, int(method), prec, _ptr(out),
                                                  flags, _stream_ptr(g), ct.byref(ms)))
    res = _l4_view(out, N2)
    return (res, ms.value) if return_fcr_ms else res


def build_TCL4_generator(system: System, gamma, dt: float, time_index: int, method: int = 0):
    """L4 at one time index: [N^2, N^2] complex128."""
    g, dev = _prep_gamma(gamma)
    Nt = g.shape[1]
    if time_index < 0 or time_index >= Nt:
        raise TacoOutOfRange(_capi.TACO_ERR_OUT_OF_RANGE, "build_TCL4_generator: time_index out of range")
    return build_TCL4_generator_batch(system, g, dt, [time_index], method)[0]


def build_correction_series(system: System, gamma, dt: float, method: int = 0):
    return build_TCL4_generator_batch(system, gamma, dt, None, method)


def _instance_array(instances, prec, outs):
    dtype = np.complex128 if prec == _capi.TACO_PREC_FP64 else np.complex64
    arr = (_capi.Instance * len(instances))()
    keep = []
    results = []
    dev = None
    tid_of = {}  # one conversion per distinct time-index object (batches often share one)
    for k, (system, gamma, dt, tidx) in enumerate(instances):
        g, d = _prep_gamma(gamma)
        if dev is None:
            dev = d
        elif dev != d:
            raise ValueError("mix of host and device gamma")
        nf, Nt = g.shape
        if tidx is None or len(tidx) == 0:
            tid, tid_addr = None, None
        else:
            hit = tid_of.get(id(tidx))
            if hit is None or hit[0] is not tidx:
                t = np.ascontiguousarray(tidx, np.uint32)
                hit = tid_of[id(tidx)] = (tidx, t, _addr(t))
            tid, tid_addr = hit[1], hit[2]
        T = Nt if tid is None else tid.size
        N2 = int(system.N) ** 2
        o = outs[k] if outs is not None else _out_array(d, (T, N2 * N2), dtype, g.device if d else None)
        v = _system_view(system)
        keep += [g, tid, o, v]
        a = arr[k]
        a.sys = v.view
        a.gamma = _addr(g)
        a.Nt = Nt
        a.dt = float(dt)
        a.tidx = tid_addr
        a.T = 0 if tid is None else tid.size
        a.L4_out = _addr(o)
        results.append(_l4_view(o, N2))
    return arr, keep, results, bool(dev)


class Tcl4Plan:
    """A batched build prepared once and replayed as one CUDA graph (device tensors only).

    >>> plan = Tcl4Plan([(system, gamma_cuda, dt, tidx), ...], precision="fp32")
    >>> plan.run()          # asynchronous on the current torch stream
    >>> plan.results[k]     # [T, N^2, N^2] views of the output buffers
    """

    def __init__(self, instances, precision: str = "fp32", method: int = 0, outs=None, full_length: bool = False):
        prec = {"fp64": _capi.TACO_PREC_FP64, "fp32": _capi.TACO_PREC_FP32}[precision]
        arr, self._keep, self.results, dev = _instance_array(instances, prec, outs)
        if not dev:
            raise ValueError("Tcl4Plan needs CUDA tensors for gamma")
        flags = _capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE
        if full_length:
            flags |= _capi.TACO_FULL_LENGTH_FFT
        self._h = ct.c_void_p()
        _capi.check(_capi.lib().taco_tcl4_plan_create(arr, len(instances), int(method), prec, flags,
                                                      ct.byref(self._h)))
        self._stream_of = self._keep[0]

    def run(self, stream=None):
        """Replay on `stream` (a raw cudaStream_t handle) or torch's current stream."""
        if stream is None:
            stream = _torch().cuda.current_stream(self._stream_of.device).cuda_stream
        _capi.check(_capi.lib().taco_tcl4_plan_execute(self._h, ct.c_void_p(stream)))
        return self.results

    def close(self):
        if self._h and self._h.value:
            _capi.check(_capi.lib().taco_tcl4_plan_destroy(self._h))
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_instances(instances, precision: str = "fp64", method: int = 0, outs=None, full_length: bool = False):
    """Batching form: ``instances`` is a list of (system, gamma, dt, tidx); gammas all host
    (numpy) or all device (torch CUDA).  Returns one [T, N^2, N^2] result per instance."""
    prec = {"fp64": _capi.TACO_PREC_FP64, "fp32": _capi.TACO_PREC_FP32}[precision]
    arr, keep, results, dev = _instance_array(instances, prec, outs)
    flags = (_capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE) if dev else 0
    if full_length:
        flags |= _capi.TACO_FULL_LENGTH_FFT
    _capi.check(_capi.lib().taco_tcl4_build_instances(arr, len(instances), int(method), prec, flags,
                                                      _stream_ptr(keep[0]) if keep else None))
    return results


def propagate_rk4_dense(L_series, r0, dt: float, L_half=None, L_add=None, sample_every: int = 0, obs=None):
    """RK4 for r' = L(t) r on the device (rk4_dense.cpp:246-321).

    L_series: [steps+1, D, D] (indexed [step, row, col]); L_half: [steps, D, D] or None
    (midpoints by averaging); L_add: [steps+1, D, D] or None (added to L_series).
    Returns (r_final, samples or None, obs_values or None); samples every
    ``sample_every`` steps plus the final state.
    """
    dev = _is_torch(L_series) and L_series.is_cuda

    def prep_series(x):
        if x is None:
            return None
        if dev:
            return x.transpose(-1, -2).contiguous()  # column-major matrices
        a = np.asarray(x)
        dtype = np.complex64 if a.dtype == np.complex64 else np.complex128
        return np.ascontiguousarray(np.swapaxes(a, -1, -2), dtype=dtype)

    Ls = prep_series(L_series)
    Lh = prep_series(L_half)
    La = prep_series(L_add)
    is32 = (str(Ls.dtype).endswith("complex64"))
    for x in (Lh, La):
        if x is not None and str(x.dtype).endswith("complex64") != is32:
            raise ValueError("propagate_rk4_dense: all generator series must share one dtype")
    steps = Ls.shape[0] - 1
    D = Ls.shape[-1]
    if dev:
        torch = _torch()
        r = r0.to(torch.complex128).clone().contiguous()
        o = obs.to(torch.complex128).contiguous() if obs is not None else None
    else:
        r = _c128_host(r0).copy()
        o = _c128_host(obs) if obs is not None else None
    ns = 0 if sample_every <= 0 else (steps + sample_every - 1) // sample_every + 1
    samples = _out_array(dev, (ns, D), np.complex128, Ls.device if dev else None) if sample_every > 0 else None
    obs_out = _out_array(dev, (ns,), np.complex128, Ls.device if dev else None) if (sample_every > 0 and obs is not None) else None
    flags = _capi.TACO_IN_DEVICE if dev else 0
    _capi.check(_capi.lib().taco_rk4_propagate(_ptr(Ls), _ptr(Lh), _ptr(La), 1 if is32 else 0, steps, D, float(dt),
                                               _ptr(r), sample_every if sample_every > 0 else 0, _ptr(samples),
                                               _ptr(o), _ptr(obs_out), flags, _stream_ptr(Ls) if dev else None))
    return r, samples, obs_out


def tcl2_generator_series(system: System, gamma, time_indices=None):
    """L2(t) (TCL2 total(), generator.cpp:164-177) at the requested times: [T, N^2, N^2]."""
    if getattr(system, "eps", None) is None:
        raise ValueError("tcl2_generator_series needs the system eigenvalues (System.eps)")
    g, dev = _prep_gamma(gamma)
    nf, Nt = g.shape
    tid = None if time_indices is None else np.ascontiguousarray(time_indices, np.uint32)
    T = Nt if tid is None or tid.size == 0 else tid.size
    N2 = int(system.N) ** 2
    out = _out_array(dev, (T, N2 * N2), np.complex128, g.device if dev else None)
    eps = np.ascontiguousarray(system.eps, np.float64)
    v = _View(system)
    flags = (_capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE) if dev else 0
    _capi.check(_capi.lib().taco_tcl2_generator_series(ct.byref(v.view), _ptr(eps), _ptr(g), Nt, _ptr(tid),
                                                       0 if tid is None else tid.size, _ptr(out), flags,
                                                       _stream_ptr(g)))
    return _l4_view(out, N2)


def gamma_trapz_device(C, dt: float, omegas):
    """Gamma_b(t_k) by the trapezoid rule on the device (gamma.hpp:166-213): [nb, N]."""
    dev = _is_torch(C) and C.is_cuda
    if dev:
        torch = _torch()
        c = C.to(torch.complex128).contiguous()
    else:
        c = _c128_host(C)
    om = np.ascontiguousarray(omegas, np.float64)
    out = _out_array(dev, (om.size, c.shape[0]), np.complex128, c.device if dev else None)
    flags = (_capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE) if dev else 0
    _capi.check(_capi.lib().taco_gamma_trapz(_ptr(c), c.shape[0], float(dt), _ptr(om), om.size, _ptr(out), flags,
                                             _stream_ptr(c)))
    return out


def gamma_trapz_device_batch(Cs, dts, omegas_list):
    """gamma_trapz_device for many correlation functions in one pair of launches: Cs are
    complex128 CUDA tensors [N_k]; returns the list of [nb_k, N_k] tensors."""
    torch = _torch()
    cs = [c.to(torch.complex128).contiguous() for c in Cs]
    oms = [np.ascontiguousarray(o, np.float64) for o in omegas_list]
    outs = [torch.empty((o.size, c.shape[0]), dtype=torch.complex128, device=c.device) for c, o in zip(cs, oms)]
    reqs = (_capi.GammaRequest * len(cs))()
    for k, (c, dt, o, g) in enumerate(zip(cs, dts, oms, outs)):
        reqs[k].C = c.data_ptr()
        reqs[k].N = c.shape[0]
        reqs[k].dt = float(dt)
        reqs[k].omegas = o.ctypes.data
        reqs[k].M = o.size
        reqs[k].G = g.data_ptr()
    if cs:
        _capi.check(_capi.lib().taco_gamma_trapz_batch(reqs, len(cs), _stream_ptr(cs[0])))
    return outs


def propagate_tcl(system: System, gamma, dt: float, steps: int, rho0, obs=None, order: int = 4,
                  sample_every: int = 1, precision: str = "fp64"):
    """RK4 propagation of vec(rho) under L = L2 + L4 (order 4), L2 (order 2) or L0 (order 0)
    on the device (examples/TCL4_spin_boson_example.cpp:317-394).  rho0: [N^2] eigenbasis
    vec; obs: [N^2] weights with <O> = sum_l obs_l r_l.  Returns (obs_values or None, rho_final)."""
    g, dev = _prep_gamma(gamma)
    nf, Nt = g.shape
    D = int(system.N) ** 2
    eps = np.ascontiguousarray(system.eps, np.float64)
    prec = {"fp64": _capi.TACO_PREC_FP64, "fp32": _capi.TACO_PREC_FP32}[precision]
    if dev:
        torch = _torch()
        r0 = torch.as_tensor(rho0, dtype=torch.complex128, device=g.device).contiguous()
        o = torch.as_tensor(obs, dtype=torch.complex128, device=g.device).contiguous() if obs is not None else None
    else:
        r0 = _c128_host(rho0)
        o = _c128_host(obs) if obs is not None else None
    ns = (steps + sample_every - 1) // sample_every + 1
    obs_out = _out_array(dev, (ns,), np.complex128, g.device if dev else None) if obs is not None else None
    rho_out = _out_array(dev, (D,), np.complex128, g.device if dev else None)
    v = _View(system)
    flags = (_capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE) if dev else 0
    _capi.check(_capi.lib().taco_propagate_tcl(ct.byref(v.view), _ptr(eps), _ptr(g), Nt, float(dt), int(steps),
                                               int(order), prec, _ptr(r0), _ptr(o), int(sample_every), _ptr(obs_out),
                                               _ptr(rho_out), flags, _stream_ptr(g)))
    return obs_out, rho_out


def build_mikx(F, C, R, pair_to_freq, N):
    """M, I, K ([T, N^2, N^2] indexed [t, row, col]) and X ([T, N^6] flat6) from F, C, R
    ([T, nf^3] at (i*nf + j)*nf + k) on the device (build_mikx_cuda_batch)."""
    F, C, R = (_c128_host(np.atleast_2d(x)) for x in (F, C, R))
    T, nf3 = F.shape
    nf = round(nf3 ** (1 / 3))
    p2f = np.ascontiguousarray(np.asarray(pair_to_freq).T, np.int32)
    N2 = N * N
    M = np.empty((T, N2 * N2), np.complex128)
    I = np.empty_like(M)
    K = np.empty_like(M)
    X = np.empty((T, N2 ** 3), np.complex128)
    _capi.check(_capi.lib().taco_build_mikx(_ptr(F), _ptr(C), _ptr(R), _ptr(p2f), N, nf, T, _ptr(M), _ptr(I),
                                            _ptr(K), _ptr(X), 0, None))
    return _l4_view(M, N2), _l4_view(I, N2), _l4_view(K, N2), X


def assemble_liouvillian(M, I, K, X, coupling_ops, symmetrize: bool = True):
    """GW ([T, N^2, N^2]) by the NAKZWAN sums on the device (assemble_liouvillian_cuda)."""
    M, I, K = (np.asarray(x) for x in (M, I, K))
    T, N2 = M.shape[0], M.shape[1]
    N = round(N2 ** 0.5)
    cm = [_c128_host(np.swapaxes(x, -1, -2)) for x in (M, I, K)]  # column-major storage
    Xc = _c128_host(X)
    ops = _c128_host(np.stack([np.asarray(A, np.complex128).T for A in coupling_ops]))
    GW = np.empty((T, N2 * N2), np.complex128)
    _capi.check(_capi.lib().taco_assemble_liouvillian(_ptr(cm[0]), _ptr(cm[1]), _ptr(cm[2]), _ptr(Xc), _ptr(ops), N,
                                                      len(coupling_ops), T, 1 if symmetrize else 0, _ptr(GW), 0, None))
    return _l4_view(GW, N2)


def gw_to_liouvillian(GW):
    """L4 ([T, N^2, N^2]) from GW ([T, N^2, N^2]), L4(n+Nm, i+Nj) = GW(n+Ni, m+Nj)."""
    GW = np.asarray(GW)
    T, N2 = GW.shape[0], GW.shape[1]
    N = round(N2 ** 0.5)
    g = _c128_host(np.swapaxes(GW, -1, -2))
    L4 = np.empty((T, N2 * N2), np.complex128)
    _capi.check(_capi.lib().taco_gw_to_liouvillian(_ptr(g), N, T, _ptr(L4), 0, None))
    return _l4_view(L4, N2)


def l4_coefficients(system: System):
    """(rowptr [N^4+1], src [nnz], coef [nnz]) of the linear map F/C/R(t) -> L4(t)."""
    v = _View(system)
    N4 = int(system.N) ** 4
    rowptr = np.zeros(N4 + 1, np.int32)
    nnz = ct.c_size_t(0)
    _capi.check(_capi.lib().taco_l4_coefficients(ct.byref(v.view), _ptr(rowptr), None, None, 0, ct.byref(nnz)))
    src = np.zeros(max(1, nnz.value), np.uint32)
    coef = np.zeros(max(1, nnz.value), np.complex128)
    _capi.check(_capi.lib().taco_l4_coefficients(ct.byref(v.view), _ptr(rowptr), _ptr(src), _ptr(coef),
                                                 nnz.value, ct.byref(nnz)))
    return rowptr, src[: nnz.value], coef[: nnz.value]
