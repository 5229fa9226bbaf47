// common.cuh -- complex arithmetic, error plumbing and small device helpers shared by
// the TCL4 kernels.  All kernels are templated on the working real type R
// (double for the plain FP64 path, float for the FP32 precision form).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace taco {

template <class R> struct CplxT;
template <> struct CplxT<double> { using type = double2; };
template <> struct CplxT<float> { using type = float2; };
template <class R> using cplx_t = typename CplxT<R>::type;

template <class C> __host__ __device__ __forceinline__ C cmk(double re, double im) {
    C c;
    c.x = static_cast<decltype(c.x)>(re);
    c.y = static_cast<decltype(c.y)>(im);
    return c;
}
template <class C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <class C> __host__ __device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
template <class C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <class C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return C{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <class C> __host__ __device__ __forceinline__ C cconj(C a) { return C{a.x, -a.y}; }
template <class C, class S> __host__ __device__ __forceinline__ C cscale(C a, S s) {
    return C{a.x * s, a.y * s};
}
__host__ __device__ __forceinline__ float2 to_f2(double2 a) {
    return make_float2(static_cast<float>(a.x), static_cast<float>(a.y));
}
__host__ __device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__host__ __device__ __forceinline__ double2 to_d2(double2 a) { return a; }
template <class C> __host__ __device__ __forceinline__ C from_d2(double2 a);
template <> __host__ __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <> __host__ __device__ __forceinline__ float2 from_d2<float2>(double2 a) { return to_f2(a); }

// Status codes of the C-ABI (mirrored in include/taco_b200.h).
enum Status : int {
    kOk = 0,
    kInvalidArgument = 1,
    kOutOfRange = 2,
    kRuntime = 3,
    kOverflow = 4,
    kCuda = 5,
    kTimeout = 6,
    kNoDevice = 7,
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(kCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

inline std::size_t next_pow2(std::size_t n) {
    if (n <= 1) return 1;
    --n;
    for (std::size_t s = 1; s < sizeof(std::size_t) * 8; s <<= 1) n |= n >> s;
    return n + 1;
}

inline int ilog2(std::size_t n) {
    int l = 0;
    while ((std::size_t(1) << l) < n) ++l;
    return l;
}

#ifdef __CUDACC__
// Asynchronous 16-byte global -> shared copies (cp.async), their groups and waits.  Used
// by per-warp rings of shared-memory slots filled a few steps ahead of their use.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
#endif

}  // namespace taco
