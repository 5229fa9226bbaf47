"""numpy/ctypes wrapper around libtaco_oracle.so (test infrastructure only)."""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtaco_oracle.so")
_lib = None

J_OHMIC = 0
J_OHMIC_DRUDE = 1
FCR_CONVOLUTION = 0
FCR_DIRECT = 1


def build(force: bool = False) -> str:
    """Compile libtaco_oracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "taco_oracle.cpp"))
    ):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ct.CDLL(_LIB_PATH)
        _lib.oracle_last_error.restype = ct.c_char_p
        _lib.oracle_next_pow2.restype = ct.c_size_t
        _lib.oracle_next_pow2.argtypes = [ct.c_size_t]
        _lib.oracle_get_fcr_fft_pad_factor.restype = ct.c_size_t
        _lib.oracle_set_fcr_fft_pad_factor.argtypes = [ct.c_size_t]
    return _lib


class OracleError(RuntimeError):
    pass


def _p(a):
    return a.ctypes.data_as(ct.c_void_p) if a is not None else None


def _check(rc):
    if rc != 0:
        raise OracleError(f"oracle error {rc}: {lib().oracle_last_error().decode()}")


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def set_threads(n: int) -> None:
    lib().oracle_set_threads(ct.c_int(n))


def next_pow2(n: int) -> int:
    return int(lib().oracle_next_pow2(n))


def set_fcr_fft_pad_factor(f: int) -> None:
    lib().oracle_set_fcr_fft_pad_factor(f)


def get_fcr_fft_pad_factor() -> int:
    return int(lib().oracle_get_fcr_fft_pad_factor())


def fft(a, forward=True):
    a = _c128(a).copy()
    _check(lib().oracle_fft(_p(a), ct.c_size_t(a.size), ct.c_int(1 if forward else 0)))
    return a


def bcf_fft(N, dt, model, params, beta):
    params = np.ascontiguousarray(params, dtype=np.float64)
    t = np.empty(N + 1, np.float64)
    C = np.empty(N + 1, np.complex128)
    _check(lib().oracle_bcf_fft(ct.c_size_t(N), ct.c_double(dt), ct.c_int(model), _p(params),
                                ct.c_double(beta), _p(t), _p(C)))
    return t, C


def gamma_trapz(C, dt, omegas):
    C = _c128(C)
    omegas = np.ascontiguousarray(omegas, dtype=np.float64)
    G = np.empty((omegas.size, C.size), np.complex128)  # bucket-major == [Nt x nf] col-major
    _check(lib().oracle_gamma_trapz(_p(C), ct.c_size_t(C.size), ct.c_double(dt), _p(omegas),
                                    ct.c_size_t(omegas.size), _p(G)))
    return G


def gamma_rect(C, dt, omegas):
    C = _c128(C)
    omegas = np.ascontiguousarray(omegas, dtype=np.float64)
    G = np.empty((omegas.size, C.size), np.complex128)
    _check(lib().oracle_gamma_rect(_p(C), ct.c_size_t(C.size), ct.c_double(dt), _p(omegas),
                                   ct.c_size_t(omegas.size), _p(G)))
    return G


class System:
    """Eigensystem + buckets; arrays are numpy, matrices column-major as (N, N) Fortran views."""

    def __init__(self, H, A_lab_list, tol=1e-9):
        H = np.asarray(H, np.complex128)
        d = H.shape[0]
        ops = [np.asarray(A, np.complex128) for A in A_lab_list]
        Hc = _c128(H.T)  # column-major
        Al = _c128(np.stack([A.T for A in ops])) if ops else np.zeros((0, d, d), np.complex128)
        eps = np.empty(d, np.float64)
        U = np.empty((d, d), np.complex128)
        nf = ct.c_int(0)
        om = np.empty(d * d, np.float64)
        p2f = np.full(d * d, -1, np.int32)
        Ae = np.empty((max(len(ops), 1), d, d), np.complex128)
        _check(lib().oracle_system_build(_p(Hc), ct.c_int(d), _p(Al), ct.c_int(len(ops)),
                                         ct.c_double(tol), _p(eps), _p(U), ct.byref(nf), _p(om),
                                         _p(p2f), _p(Ae)))
        self.N = d
        self.tol = tol
        self.eps = eps
        self.U = U.T.copy()  # back to row-major (d, d)
        self.nf = nf.value
        self.omegas = om[: self.nf].copy()
        self.pair_to_freq = p2f.reshape(d, d).T.copy()  # [a, b]
        self.A_eig = [Ae[k].T.copy() for k in range(len(ops))]
        self.mirror, self.zero_index = build_map(self.omegas, tol)

    def ops_colmajor(self):
        return _c128(np.stack([A.T for A in self.A_eig]))

    def p2f_colmajor(self):
        return np.ascontiguousarray(self.pair_to_freq.T, dtype=np.int32)


def build_map(omegas, tol=1e-9):
    omegas = np.ascontiguousarray(omegas, dtype=np.float64)
    mirror = np.empty(omegas.size, np.int32)
    zero = ct.c_int(-1)
    _check(lib().oracle_build_map(_p(omegas), ct.c_int(omegas.size), ct.c_double(tol), _p(mirror),
                                  ct.byref(zero)))
    return mirror, zero.value


def fcr_series(gamma, omegas, mirror, dt, method=FCR_CONVOLUTION):
    """gamma: [nf, Nt] complex (bucket-major).  Returns F, C, R as [nf^3, Nt]."""
    gamma = _c128(gamma)
    nf, Nt = gamma.shape
    omegas = np.ascontiguousarray(omegas, dtype=np.float64)
    mirror = np.ascontiguousarray(mirror, dtype=np.int32)
    F = np.empty((nf ** 3, Nt), np.complex128)
    Cc = np.empty_like(F)
    R = np.empty_like(F)
    _check(lib().oracle_fcr_series(_p(gamma), ct.c_size_t(Nt), ct.c_int(nf), _p(omegas), _p(mirror),
                                   ct.c_double(dt), ct.c_int(method), _p(F), _p(Cc), _p(R)))
    return F, Cc, R


def mikx(Ft, Ct, Rt, nf, p2f_colmajor, N):
    Ft, Ct, Rt = _c128(Ft), _c128(Ct), _c128(Rt)
    p2f = np.ascontiguousarray(p2f_colmajor, dtype=np.int32)
    N2 = N * N
    M = np.empty(N2 * N2, np.complex128)
    I = np.empty_like(M)
    K = np.empty_like(M)
    X = np.empty(N ** 6, np.complex128)
    _check(lib().oracle_mikx(_p(Ft), _p(Ct), _p(Rt), ct.c_int(nf), _p(p2f), ct.c_int(N), _p(M), _p(I),
                             _p(K), _p(X)))
    return M, I, K, X  # column-major flats


def assemble_gw(M, I, K, X, ops_colmajor, N):
    ops = _c128(ops_colmajor)
    GW = np.empty(N ** 4, np.complex128)
    _check(lib().oracle_assemble_gw(_p(_c128(M)), _p(_c128(I)), _p(_c128(K)), _p(_c128(X)), _p(ops),
                                    ct.c_int(ops.shape[0]), ct.c_int(N), _p(GW)))
    return GW


def gw_to_l4(GW, N):
    L4 = np.empty(N ** 4, np.complex128)
    _check(lib().oracle_gw_to_l4(_p(_c128(GW)), ct.c_int(N), _p(L4)))
    return L4


def tcl4_build_batch(N, nf, omegas, mirror, p2f_colmajor, ops_colmajor, gamma, dt, tidx=None,
                     method=FCR_CONVOLUTION, timings=False):
    """Returns L4 as [T, N^2, N^2] (row-major view of each column-major matrix is transposed back)."""
    gamma = _c128(gamma)
    Nt = gamma.shape[1]
    ops = _c128(ops_colmajor)
    if tidx is None:
        tid = np.zeros(0, np.uint32)
        T = Nt
    else:
        tid = np.ascontiguousarray(tidx, dtype=np.uint32)
        T = tid.size
    out = np.empty((T, N * N * N * N), np.complex128)
    fcr_ms = ct.c_double(0.0)
    pt_ms = ct.c_double(0.0)
    _check(lib().oracle_tcl4_build_batch(
        ct.c_int(N), ct.c_int(nf), _p(np.ascontiguousarray(omegas, np.float64)),
        _p(np.ascontiguousarray(mirror, np.int32)), _p(np.ascontiguousarray(p2f_colmajor, np.int32)),
        _p(ops), ct.c_int(ops.shape[0]), _p(gamma), ct.c_size_t(Nt), ct.c_double(dt),
        _p(tid) if tid.size else None, ct.c_size_t(tid.size), ct.c_int(method), _p(out),
        ct.byref(fcr_ms), ct.byref(pt_ms)))
    L4 = out.reshape(T, N * N, N * N).transpose(0, 2, 1)  # column-major -> [row, col]
    if timings:
        return L4, fcr_ms.value, pt_ms.value
    return L4


def unitary_superop(H_eff):
    H = np.asarray(H_eff, np.complex128)
    N = H.shape[0]
    L = np.empty(N ** 4, np.complex128)
    _check(lib().oracle_unitary_superop(ct.c_int(N), _p(_c128(H.T)), _p(L)))
    return L.reshape(N * N, N * N).T.copy()


def tcl2_total(system: System, gamma_b):
    N = system.N
    L = np.empty(N ** 4, np.complex128)
    Hls = np.empty(N * N, np.complex128)
    _check(lib().oracle_tcl2_total(ct.c_int(N), ct.c_int(system.nf), _p(system.eps),
                                   _p(system.p2f_colmajor()), _p(system.ops_colmajor()),
                                   ct.c_int(len(system.A_eig)), _p(_c128(gamma_b)), _p(L), _p(Hls)))
    return L.reshape(N * N, N * N).T.copy(), Hls.reshape(N, N).T.copy()


def rk4_propagate(L_series, r0, dt, L_half=None, sample_every=0):
    """L_series: [steps+1, D, D] (row-major matrices).  Returns (r_final, samples or None)."""
    Ls = _c128(np.transpose(np.asarray(L_series, np.complex128), (0, 2, 1)))
    steps = Ls.shape[0] - 1
    D = Ls.shape[1]
    Lh = _c128(np.transpose(np.asarray(L_half, np.complex128), (0, 2, 1))) if L_half is not None else None
    r = _c128(r0).copy()
    se = sample_every if sample_every > 0 else 1
    samples = np.empty((steps // se + 2, D), np.complex128) if sample_every > 0 else None
    ns = ct.c_size_t(0)
    _check(lib().oracle_rk4_propagate(_p(Ls), _p(Lh), ct.c_size_t(steps), ct.c_int(D), ct.c_double(dt),
                                      _p(r), ct.c_size_t(se), _p(samples), ct.byref(ns)))
    if samples is not None:
        samples = samples[: ns.value]
    return r, samples


def rk4_propagate_const(L, r0, t0, tf, dt):
    L = np.asarray(L, np.complex128)
    r = _c128(r0).copy()
    _check(lib().oracle_rk4_propagate_const(_p(_c128(L.T)), ct.c_int(L.shape[0]), ct.c_double(t0),
                                            ct.c_double(tf), ct.c_double(dt), _p(r)))
    return r


def spin_boson_trajectory(params, N, dt, steps, rho0=None, observable=None, sample_every=1):
    """<O(t)> (real) of the FP64 chain for one spin boson (eps, Delta, alpha, wc, beta):
    H = eps/2 sz + Delta/2 sx, A = sz, Ohmic bath by bcf_fft, trapezoid Gamma, L4 by the
    convolution method, L2 by tcl2_total, RK4 under L2 + L4 from rho0 (lab basis, |0><0|
    by default), O = sz by default (examples/TCL4_spin_boson_example.cpp:196-394)."""
    sx = np.array([[0, 1], [1, 0]], np.complex128)
    sz = np.array([[1, 0], [0, -1]], np.complex128)
    rho0 = np.array([[1, 0], [0, 0]], np.complex128) if rho0 is None else np.asarray(rho0, np.complex128)
    O = sz if observable is None else np.asarray(observable, np.complex128)
    eps, delta, alpha, wc, beta = params
    T = steps + 1
    osys = System(0.5 * eps * sz + 0.5 * delta * sx, [sz])
    _, C = bcf_fft(N, dt, J_OHMIC, [alpha, wc], beta)
    G = gamma_trapz(C[:T], dt, osys.omegas)
    L4 = tcl4_build_batch(osys.N, osys.nf, osys.omegas, osys.mirror, osys.p2f_colmajor(), osys.ops_colmajor(),
                          G, dt, tidx=np.arange(T))
    L2 = np.stack([tcl2_total(osys, G[:, t])[0] for t in range(T)])
    U = osys.U
    r0 = (U.conj().T @ rho0 @ U).reshape(-1, order="F")
    ov = (U.conj().T @ O @ U).T.reshape(-1, order="F")
    _, samp = rk4_propagate(L2 + L4, r0, dt, sample_every=sample_every)
    return np.real(samp @ ov)
