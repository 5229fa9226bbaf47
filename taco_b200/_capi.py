"""ctypes binding of libtaco_b200.so (the C-ABI declared in include/taco_b200.h)."""
from __future__ import annotations

import ctypes as ct
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libtaco_b200.so")

TACO_OK = 0
TACO_ERR_INVALID_ARGUMENT = 1
TACO_ERR_OUT_OF_RANGE = 2
TACO_ERR_RUNTIME = 3
TACO_ERR_OVERFLOW = 4
TACO_ERR_CUDA = 5
TACO_ERR_TIMEOUT = 6
TACO_ERR_NO_DEVICE = 7

TACO_FCR_CONVOLUTION = 0
TACO_FCR_DIRECT = 1
TACO_PREC_FP64 = 0
TACO_PREC_FP32 = 1
TACO_IN_DEVICE = 1
TACO_OUT_DEVICE = 2
TACO_CAUSAL_TRUNCATION = 4
TACO_FULL_LENGTH_FFT = 8
TACO_NOALLOC_SCRATCH_BYTES = 64 * 1024 * 1024

# every symbol the header declares
EXPORTED = [
    "taco_version", "taco_last_error", "taco_device_count", "taco_set_device",
    "taco_set_fcr_fft_pad_factor", "taco_get_fcr_fft_pad_factor", "taco_compute_triple_kernels",
    "taco_tcl4_build_batch", "taco_tcl4_build", "taco_tcl4_correction_series",
    "taco_tcl4_build_instances", "taco_rk4_propagate", "taco_l4_coefficients",
    "taco_kernel_launches", "taco_profile_enable", "taco_profile_reset", "taco_profile_get",
    "taco_set_tuning", "taco_get_tuning", "taco_clear_tuning", "taco_set_cluster_points",
    "taco_tcl4_plan_create", "taco_tcl4_plan_execute", "taco_tcl4_plan_destroy",
    "taco_tcl4_build_batch_noalloc", "taco_tcl2_generator_series", "taco_gamma_trapz", "taco_propagate_tcl",
    "taco_build_mikx", "taco_assemble_liouvillian", "taco_gw_to_liouvillian",
    "taco_bcf_fft", "taco_rk4_forward_checkpointed", "taco_rk4_adjoint", "taco_tcl4_adjoint",
    "taco_tcl2_adjoint", "taco_inner_re", "taco_set_work_budget", "taco_gamma_trapz_batch",
    "taco_fft_length", "taco_compute_triple_kernels_batch", "taco_set_fp32_guard", "taco_get_fp32_guard",
    "taco_fp32_guard_stats", "taco_set_fused_conv", "taco_get_fused_conv", "taco_set_guard_chunk_bytes",
    "taco_release_workspace", "taco_set_fft_length_enabled",
]


class SystemView(ct.Structure):
    _fields_ = [("N", ct.c_int), ("nf", ct.c_int), ("num_ops", ct.c_int),
                ("omegas", ct.c_void_p), ("mirror", ct.c_void_p), ("pair_to_freq", ct.c_void_p),
                ("ops", ct.c_void_p), ("tol", ct.c_double)]


class Instance(ct.Structure):
    _fields_ = [("sys", SystemView), ("gamma", ct.c_void_p), ("Nt", ct.c_size_t), ("dt", ct.c_double),
                ("tidx", ct.c_void_p), ("T", ct.c_size_t), ("L4_out", ct.c_void_p)]


class FcrRequest(ct.Structure):
    _fields_ = [("sys", SystemView), ("gamma", ct.c_void_p), ("Nt", ct.c_size_t), ("dt", ct.c_double),
                ("F", ct.c_void_p), ("C", ct.c_void_p), ("R", ct.c_void_p)]


class TacoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class TacoInvalidArgument(TacoError, ValueError):
    pass


class TacoOutOfRange(TacoError, IndexError):
    pass


class TacoOverflow(TacoError, OverflowError):
    pass


_ERRS = {TACO_ERR_INVALID_ARGUMENT: TacoInvalidArgument, TACO_ERR_OUT_OF_RANGE: TacoOutOfRange,
         TACO_ERR_OVERFLOW: TacoOverflow}


class BcfRequest(ct.Structure):
    _fields_ = [("model", ct.c_int), ("which", ct.c_int), ("alpha", ct.c_double), ("omega_c", ct.c_double),
                ("lam", ct.c_double), ("gam", ct.c_double), ("beta", ct.c_double), ("N", ct.c_size_t),
                ("dt", ct.c_double), ("out", ct.c_void_p), ("n_out", ct.c_size_t)]


class Rk4GradJob(ct.Structure):
    _fields_ = [("L", ct.c_void_p), ("L_add", ct.c_void_p), ("steps", ct.c_size_t), ("D", ct.c_int),
                ("dt", ct.c_double), ("r0", ct.c_void_p), ("obs", ct.c_void_p), ("sample_every", ct.c_size_t),
                ("ckpt", ct.c_void_p), ("obs_out", ct.c_void_p), ("r_out", ct.c_void_p), ("obs_bar", ct.c_void_p),
                ("r_final_bar", ct.c_void_p), ("L_bar", ct.c_void_p), ("r0_bar", ct.c_void_p),
                ("obs_vec_bar", ct.c_void_p)]


class Tcl4AdjointJob(ct.Structure):
    _fields_ = [("sys", ct.POINTER(SystemView)), ("gamma", ct.c_void_p), ("T", ct.c_size_t), ("dt", ct.c_double),
                ("L_bar", ct.c_void_p), ("F", ct.c_void_p), ("C", ct.c_void_p), ("R", ct.c_void_p),
                ("gamma_bar", ct.c_void_p), ("omega_bar", ct.c_void_p), ("ops_bar", ct.c_void_p)]


class Tcl2AdjointJob(ct.Structure):
    _fields_ = [("sys", ct.POINTER(SystemView)), ("eps", ct.c_void_p), ("gamma", ct.c_void_p), ("T", ct.c_size_t),
                ("L_bar", ct.c_void_p), ("gamma_bar", ct.c_void_p), ("ops_bar", ct.c_void_p),
                ("eps_bar", ct.c_void_p)]


class GammaRequest(ct.Structure):
    _fields_ = [("C", ct.c_void_p), ("N", ct.c_size_t), ("dt", ct.c_double), ("omegas", ct.c_void_p),
                ("M", ct.c_size_t), ("G", ct.c_void_p)]


class InnerJob(ct.Structure):
    _fields_ = [("a", ct.c_void_p), ("b", ct.c_void_p), ("n", ct.c_size_t)]


_lib = None


def lib():
    """Load libtaco_b200.so; raises if it was not built (there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m taco_b200.build` (nvcc, sm_100a)")
        L = ct.CDLL(LIB_PATH)
        L.taco_version.restype = ct.c_char_p
        L.taco_last_error.restype = ct.c_char_p
        L.taco_get_fcr_fft_pad_factor.restype = ct.c_size_t
        L.taco_set_fcr_fft_pad_factor.argtypes = [ct.c_size_t]
        L.taco_device_count.argtypes = [ct.POINTER(ct.c_int)]
        L.taco_set_device.argtypes = [ct.c_int]
        L.taco_compute_triple_kernels.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_size_t, ct.c_double,
                                                  ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int,
                                                  ct.c_void_p]
        L.taco_compute_triple_kernels_batch.argtypes = [ct.POINTER(FcrRequest), ct.c_size_t, ct.c_int, ct.c_void_p]
        L.taco_tcl4_build_batch.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_size_t, ct.c_double,
                                            ct.c_void_p, ct.c_size_t, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int,
                                            ct.c_void_p, ct.POINTER(ct.c_double)]
        L.taco_tcl4_build.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_size_t, ct.c_double, ct.c_size_t,
                                      ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p]
        L.taco_tcl4_correction_series.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_size_t, ct.c_double,
                                                  ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p]
        L.taco_tcl4_build_instances.argtypes = [ct.POINTER(Instance), ct.c_size_t, ct.c_int, ct.c_int, ct.c_int,
                                                ct.c_void_p]
        L.taco_rk4_propagate.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_size_t, ct.c_int,
                                         ct.c_double, ct.c_void_p, ct.c_size_t, ct.c_void_p, ct.c_void_p,
                                         ct.c_void_p, ct.c_int, ct.c_void_p]
        L.taco_l4_coefficients.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                           ct.c_size_t, ct.POINTER(ct.c_size_t)]
        L.taco_kernel_launches.argtypes = [ct.POINTER(ct.c_uint64)]
        L.taco_profile_enable.argtypes = [ct.c_int]
        L.taco_profile_get.argtypes = [ct.c_size_t, ct.POINTER(ct.c_char_p), ct.POINTER(ct.c_uint64),
                                       ct.POINTER(ct.c_double), ct.POINTER(ct.c_size_t)]
        L.taco_set_tuning.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_size_t, ct.c_int]
        L.taco_get_tuning.argtypes = [ct.c_int, ct.c_int, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                                      ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_int)]
        L.taco_set_cluster_points.argtypes = [ct.c_int, ct.c_int, ct.c_int]
        L.taco_tcl4_plan_create.argtypes = [ct.POINTER(Instance), ct.c_size_t, ct.c_int, ct.c_int, ct.c_int,
                                            ct.POINTER(ct.c_void_p)]
        L.taco_tcl4_plan_execute.argtypes = [ct.c_void_p, ct.c_void_p]
        L.taco_tcl4_plan_destroy.argtypes = [ct.c_void_p]
        L.taco_tcl2_generator_series.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_void_p, ct.c_size_t,
                                                 ct.c_void_p, ct.c_size_t, ct.c_void_p, ct.c_int, ct.c_void_p]
        L.taco_gamma_trapz.argtypes = [ct.c_void_p, ct.c_size_t, ct.c_double, ct.c_void_p, ct.c_size_t, ct.c_void_p,
                                       ct.c_int, ct.c_void_p]
        L.taco_propagate_tcl.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_void_p, ct.c_size_t, ct.c_double,
                                         ct.c_size_t, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_size_t,
                                         ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]
        L.taco_build_mikx.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int,
                                      ct.c_size_t, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int,
                                      ct.c_void_p]
        L.taco_assemble_liouvillian.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                                ct.c_int, ct.c_int, ct.c_size_t, ct.c_int, ct.c_void_p, ct.c_int,
                                                ct.c_void_p]
        L.taco_gw_to_liouvillian.argtypes = [ct.c_void_p, ct.c_int, ct.c_size_t, ct.c_void_p, ct.c_int, ct.c_void_p]
        L.taco_set_work_budget.argtypes = [ct.c_size_t]
        L.taco_set_fp32_guard.argtypes = [ct.c_double]
        L.taco_get_fp32_guard.argtypes = [ct.POINTER(ct.c_double)]
        L.taco_fp32_guard_stats.argtypes = [ct.POINTER(ct.c_uint64)]
        L.taco_set_fused_conv.argtypes = [ct.c_int]
        L.taco_get_fused_conv.argtypes = [ct.POINTER(ct.c_int)]
        L.taco_set_guard_chunk_bytes.argtypes = [ct.c_size_t]
        L.taco_release_workspace.argtypes = []
        L.taco_set_fft_length_enabled.argtypes = [ct.c_int, ct.c_int, ct.c_int]
        L.taco_fft_length.argtypes = [ct.c_size_t, ct.c_int, ct.c_int, ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_int)]
        L.taco_gamma_trapz_batch.argtypes = [ct.POINTER(GammaRequest), ct.c_size_t, ct.c_void_p]
        L.taco_bcf_fft.argtypes = [ct.POINTER(BcfRequest), ct.c_size_t, ct.c_int, ct.c_void_p]
        L.taco_rk4_forward_checkpointed.argtypes = [ct.POINTER(Rk4GradJob), ct.c_size_t, ct.c_size_t, ct.c_void_p]
        L.taco_rk4_adjoint.argtypes = [ct.POINTER(Rk4GradJob), ct.c_size_t, ct.c_size_t, ct.c_void_p]
        L.taco_tcl4_adjoint.argtypes = [ct.POINTER(Tcl4AdjointJob), ct.c_size_t, ct.c_void_p]
        L.taco_tcl2_adjoint.argtypes = [ct.POINTER(Tcl2AdjointJob), ct.c_size_t, ct.c_void_p]
        L.taco_inner_re.argtypes = [ct.POINTER(InnerJob), ct.c_size_t, ct.c_void_p, ct.c_void_p]
        L.taco_tcl4_build_batch_noalloc.argtypes = [ct.POINTER(SystemView), ct.c_void_p, ct.c_size_t,
                                                    ct.c_double, ct.c_void_p, ct.c_size_t, ct.c_int, ct.c_void_p,
                                                    ct.c_void_p]
        _lib = L
        _apply_tuning_table(L)
    return _lib


def _apply_tuning_table(L):
    """Apply the persisted launch schedules measured by the autotuner (taco_b200/tuning.json)."""
    import json

    path = os.path.join(_PKG, "tuning.json")
    if not os.path.exists(path):
        return
    with open(path) as f:
        table = json.load(f)
    for key, sch in table.items():
        if key.startswith("_"):
            continue
        L2, prec = key.split(":")
        pr = TACO_PREC_FP32 if prec == "fp32" else TACO_PREC_FP64
        if "col_tile" in sch:  # a tile schedule (entries may carry only the radix choice)
            L.taco_set_tuning(int(L2), pr, int(sch["col_tile"]), int(sch["row_tile"]), int(sch["chunk_bytes"]),
                              int(sch["inv_dft_rows"]))
            if "cluster_lm" in sch:
                L.taco_set_cluster_points(int(L2), pr, int(sch["cluster_lm"]))
        if int(L2) >= 64 and "enabled" in sch:  # 3 * 2^k and 5 * 2^k lengths the tuner measured slower
            L.taco_set_fft_length_enabled(int(L2), pr, 1 if sch["enabled"] else 0)


def check(rc: int) -> None:
    if rc != TACO_OK:
        msg = lib().taco_last_error().decode(errors="replace")
        raise _ERRS.get(rc, TacoError)(rc, msg)
