// contract.cuh -- fused MIKX -> GW -> (T + T^H) -> L4 contraction for all requested times.
//
// Each L4 entry e is a sparse linear form in the F/C/R values at one time (see
// gw_coef.hpp).  A CTA takes a tile of OT output times; thread (e, o) walks the CSR
// row of e, gathers v_s at the time of output o (source-major layout v[s][u]: lanes
// with consecutive outputs read consecutive addresses) and accumulates in the working
// type.  Results are staged in shared memory and written as whole L4 matrices
// (column-major, output-major: out[o][e]).
#pragma once

#include "common.cuh"

namespace taco {

// Accumulator of one L4 entry: plain in FP64; compensated (Kahan, separately for the
// real and imaginary parts) in the FP32 form, where a sequential FP32 sum of the ~10^3
// terms per entry of d >= 6 systems would lose ~1e-6 relative accuracy.
template <class C>
struct EntryAcc;

template <>
struct EntryAcc<double2> {
    double2 s = make_double2(0.0, 0.0);
    __device__ __forceinline__ void add(double2 x) { s = cadd(s, x); }
    __device__ __forceinline__ double2 get() const { return s; }
};

template <>
struct EntryAcc<float2> {
    float2 s = make_float2(0.f, 0.f), c = make_float2(0.f, 0.f);
    __device__ __forceinline__ void add(float2 x) {
        const float yx = x.x - c.x, yy = x.y - c.y;
        const float tx = s.x + yx, ty = s.y + yy;
        c.x = (tx - s.x) - yx;
        c.y = (ty - s.y) - yy;
        s.x = tx;
        s.y = ty;
    }
    __device__ __forceinline__ float2 get() const { return s; }
};

struct ContractJob {
    const int32_t* rowptr;  // [E + 1]
    const uint32_t* src;    // [nnz] source | conj << 31
    const void* coef;       // [nnz] working complex type
    const void* v;          // [3 nf^3][U] working complex type
    const uint32_t* out_u;  // [T] unique-time position of each output
    void* out;              // [T][E] working complex type
    uint32_t T, U, E;
    uint32_t accumulate;    // 1: add into out (later slices of a sliced instance)
};

template <class R>
__global__ void k_contract(const ContractJob* __restrict__ jobs, int OT) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* res = reinterpret_cast<C*>(smem_raw);  // [OT][E]
    const ContractJob job = jobs[blockIdx.y];
    const uint32_t o0 = blockIdx.x * OT;
    if (o0 >= job.T) return;
    const uint32_t ot = min(static_cast<uint32_t>(OT), job.T - o0);
    const C* coef = static_cast<const C*>(job.coef);
    const C* v = static_cast<const C*>(job.v);
    const uint32_t work = job.E * OT;
    for (uint32_t idx = threadIdx.x; idx < work; idx += blockDim.x) {
        const uint32_t ol = idx % OT, e = idx / OT;
        if (ol >= ot) continue;
        const uint32_t u = __ldg(&job.out_u[o0 + ol]);
        EntryAcc<C> acc;
        const int32_t b = __ldg(&job.rowptr[e]), end = __ldg(&job.rowptr[e + 1]);
        for (int32_t k = b; k < end; ++k) {
            const uint32_t sk = __ldg(&job.src[k]);
            const C w = coef[k];
            C x = v[static_cast<size_t>(sk & 0x7fffffffu) * job.U + u];
            if (sk & 0x80000000u) x.y = -x.y;
            acc.add(cmul(w, x));
        }
        res[ol * job.E + e] = acc.get();
    }
    __syncthreads();
    C* out = static_cast<C*>(job.out) + static_cast<size_t>(o0) * job.E;
    const uint32_t total = ot * job.E;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x)
        out[idx] = job.accumulate ? cadd(out[idx], res[idx]) : res[idx];
}

// Shared-memory variant: the CTA stages v[s][u(o)] for its OT outputs and the CSR table,
// then every thread evaluates (entry, output) pairs from shared memory.  Used when the
// F/C/R tile fits (small systems: S = 3 nf^3 sources).
template <class R>
__global__ void k_contract_smem(const ContractJob* __restrict__ jobs, int OT, int S, int nnz_cap) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const ContractJob job = jobs[blockIdx.y];
    const uint32_t o0 = blockIdx.x * OT;
    if (o0 >= job.T) return;
    const uint32_t ot = min(static_cast<uint32_t>(OT), job.T - o0);
    C* vs = reinterpret_cast<C*>(smem_raw);           // [S][OT]
    C* res = vs + static_cast<size_t>(S) * OT;         // [OT][E]
    C* cf = res + static_cast<size_t>(OT) * job.E;     // [nnz]
    uint32_t* sr = reinterpret_cast<uint32_t*>(cf + nnz_cap);
    int32_t* rp = reinterpret_cast<int32_t*>(sr + nnz_cap);
    const int32_t nnz = __ldg(&job.rowptr[job.E]);
    const C* coef = static_cast<const C*>(job.coef);
    for (int32_t k = threadIdx.x; k < nnz; k += blockDim.x) {
        cf[k] = coef[k];
        sr[k] = __ldg(&job.src[k]);
    }
    for (uint32_t e = threadIdx.x; e <= job.E; e += blockDim.x) rp[e] = __ldg(&job.rowptr[e]);
    const C* v = static_cast<const C*>(job.v);
    const uint32_t nv = static_cast<uint32_t>(S) * OT;
    for (uint32_t idx = threadIdx.x; idx < nv; idx += blockDim.x) {
        const uint32_t sidx = idx / OT, ol = idx - sidx * OT;
        vs[idx] = ol < ot ? v[static_cast<size_t>(sidx) * job.U + __ldg(&job.out_u[o0 + ol])] : C{0, 0};
    }
    __syncthreads();
    const uint32_t work = job.E * OT;
    for (uint32_t idx = threadIdx.x; idx < work; idx += blockDim.x) {
        const uint32_t ol = idx % OT, e = idx / OT;
        EntryAcc<C> acc;
        const int32_t b = rp[e], end = rp[e + 1];
        for (int32_t k = b; k < end; ++k) {
            const uint32_t sk = sr[k];
            C x = vs[(sk & 0x7fffffffu) * OT + ol];
            if (sk & 0x80000000u) x.y = -x.y;
            acc.add(cmul(cf[k], x));
        }
        res[ol * job.E + e] = acc.get();
    }
    __syncthreads();
    C* out = static_cast<C*>(job.out) + static_cast<size_t>(o0) * job.E;
    const uint32_t total = ot * job.E;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x)
        out[idx] = job.accumulate ? cadd(out[idx], res[idx]) : res[idx];
}

// Output-per-thread variant: thread o evaluates every L4 entry at output time o, walking
// the CSR rows with warp-uniform (broadcast) coefficient loads while the lanes gather
// consecutive times of the same source (coalesced, L1-resident after the first touch).
// GW is assembled as T + T^H, so GW(c, r) = conj(GW(r, c)) exactly and
// L4[(n,m),(i,j)] = conj(L4[(m,n),(j,i)]): only entries with e <= partner(e) are summed,
// the others are their partners' conjugates.  Results are staged in shared memory
// ([threads][E + 1]) and written as whole matrices.
constexpr int CONTRACT_ROW_THREADS = 128;

__device__ __forceinline__ uint32_t l4_partner(uint32_t e, int N) {
    const uint32_t N2 = static_cast<uint32_t>(N) * N;
    const uint32_t row = e % N2, col = e / N2;
    const uint32_t n = row % N, m = row / N, i = col % N, j = col / N;
    return (m + N * n) + N2 * (j + N * i);
}

// Real coefficients of one term with the source conjugation folded in:
// c * x      = (a x.x + b x.y, c x.y + d x.x) with (a, b, c, d) = ( c.x, -c.y,  c.x, c.y)
// c * conj x                                    with (a, b, c, d) = ( c.x,  c.y, -c.x, c.y)
template <class R>
struct alignas(4 * sizeof(R)) Coef4 {
    R a, b, c, d;
};

template <class C, class R>
__device__ __forceinline__ void term_mac(C& p, const Coef4<R>& w, C x) {
    p.x = fma(w.a, x.x, p.x);
    p.x = fma(w.b, x.y, p.x);
    p.y = fma(w.c, x.y, p.y);
    p.y = fma(w.d, x.x, p.y);
}

// Shared-memory bytes of k_contract_rows_staged for `threads` times, E entries and a table
// of nnz terms.
template <class R>
inline std::size_t rows_staged_smem(int threads, int E, std::size_t nnz) {
    return static_cast<std::size_t>(threads) * (E + 1) * 2 * sizeof(R) + nnz * (sizeof(Coef4<R>) + 4) +
           static_cast<std::size_t>(E + 1) * 4 + 64;
}

// One thread per output time, as k_contract_rows, with the CSR table preprocessed into
// shared memory once per CTA: four real coefficients per term (conjugation folded in) and
// the source's element offset s * U (the host guarantees 3 nf^3 U < 2^32).  Terms are
// summed in groups of four by plain FMAs and each group is added with compensation.
template <class R>
__global__ void __launch_bounds__(CONTRACT_ROW_THREADS) k_contract_rows_staged(const ContractJob* __restrict__ jobs,
                                                                               int N, int nnz_cap) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const ContractJob job = jobs[blockIdx.y];
    const uint32_t o0 = blockIdx.x * CONTRACT_ROW_THREADS;
    if (o0 >= job.T) return;
    const uint32_t E = job.E, ld = E + 1;
    Coef4<R>* cf = reinterpret_cast<Coef4<R>*>(smem_raw);                      // [nnz_cap]
    C* res = reinterpret_cast<C*>(cf + nnz_cap);                               // [threads][E + 1]
    uint32_t* off = reinterpret_cast<uint32_t*>(res + CONTRACT_ROW_THREADS * ld);  // [nnz_cap]
    int32_t* rp = reinterpret_cast<int32_t*>(off + nnz_cap);                   // [E + 1]
    const int32_t nnz = __ldg(&job.rowptr[E]);
    const C* coef = static_cast<const C*>(job.coef);
    for (int32_t k = threadIdx.x; k < nnz; k += blockDim.x) {
        const uint32_t sk = __ldg(&job.src[k]);
        const C w = coef[k];
        const bool cj = (sk & 0x80000000u) != 0;
        cf[k] = Coef4<R>{w.x, cj ? w.y : -w.y, cj ? -w.x : w.x, w.y};
        off[k] = (sk & 0x7fffffffu) * job.U;
    }
    for (uint32_t e = threadIdx.x; e <= E; e += blockDim.x) rp[e] = __ldg(&job.rowptr[e]);
    __syncthreads();
    const uint32_t ot = min(static_cast<uint32_t>(CONTRACT_ROW_THREADS), job.T - o0);
    const uint32_t o = o0 + threadIdx.x;
    if (threadIdx.x < ot) {
        const C* v = static_cast<const C*>(job.v) + __ldg(&job.out_u[o]);
        for (uint32_t e = 0; e < E; ++e) {
            if (l4_partner(e, N) < e) continue;
            EntryAcc<C> acc;
            int32_t k = rp[e];
            const int32_t end = rp[e + 1];
            for (; k + 4 <= end; k += 4) {
                const C x0 = v[off[k]], x1 = v[off[k + 1]], x2 = v[off[k + 2]], x3 = v[off[k + 3]];
                C p{0, 0};
                term_mac(p, cf[k], x0);
                term_mac(p, cf[k + 1], x1);
                term_mac(p, cf[k + 2], x2);
                term_mac(p, cf[k + 3], x3);
                acc.add(p);
            }
            for (; k < end; ++k) {
                C p{0, 0};
                term_mac(p, cf[k], v[off[k]]);
                acc.add(p);
            }
            res[threadIdx.x * ld + e] = acc.get();
        }
        for (uint32_t e = 0; e < E; ++e) {
            const uint32_t p = l4_partner(e, N);
            if (p < e) res[threadIdx.x * ld + e] = cconj(res[threadIdx.x * ld + p]);
        }
    }
    __syncthreads();
    C* out = static_cast<C*>(job.out) + static_cast<size_t>(o0) * E;
    const uint32_t total = ot * E;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const uint32_t ol = idx / E, e = idx - ol * E;
        out[idx] = job.accumulate ? cadd(out[idx], res[ol * ld + e]) : res[ol * ld + e];
    }
}

// d = 2 (E = 16): k_contract_rows_staged with the 16 results of a time in registers and
// written as one 128-byte (FP32) or 256-byte (FP64) row by vector stores, so that shared
// memory holds only the table and more CTAs stay resident.  Unique entries (partner(e) >= e)
// are summed, the other six are conjugates.
__host__ __device__ constexpr int d2_partner_e(int e) {
    return (e % 4 / 2 + 2 * (e % 4 % 2)) + 4 * (e / 4 / 2 + 2 * (e / 4 % 2));
}

template <class R>
inline std::size_t rows_d2_smem(std::size_t nnz) {
    return nnz * (sizeof(Coef4<R>) + 4) + 17 * 4 + 64;
}

template <class R>
__global__ void __launch_bounds__(CONTRACT_ROW_THREADS) k_contract_rows_d2(const ContractJob* __restrict__ jobs,
                                                                           int nnz_cap) {
    using C = cplx_t<R>;
    constexpr int E = 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const ContractJob job = jobs[blockIdx.y];
    const uint32_t o0 = blockIdx.x * CONTRACT_ROW_THREADS;
    if (o0 >= job.T) return;
    Coef4<R>* cf = reinterpret_cast<Coef4<R>*>(smem_raw);          // [nnz_cap]
    uint32_t* off = reinterpret_cast<uint32_t*>(cf + nnz_cap);     // [nnz_cap]
    int32_t* rp = reinterpret_cast<int32_t*>(off + nnz_cap);       // [E + 1]
    const int32_t nnz = __ldg(&job.rowptr[E]);
    const C* coef = static_cast<const C*>(job.coef);
    for (int32_t k = threadIdx.x; k < nnz; k += blockDim.x) {
        const uint32_t sk = __ldg(&job.src[k]);
        const C w = coef[k];
        const bool cj = (sk & 0x80000000u) != 0;
        cf[k] = Coef4<R>{w.x, cj ? w.y : -w.y, cj ? -w.x : w.x, w.y};
        off[k] = (sk & 0x7fffffffu) * job.U;
    }
    for (uint32_t e = threadIdx.x; e <= E; e += blockDim.x) rp[e] = __ldg(&job.rowptr[e]);
    __syncthreads();
    const uint32_t o = o0 + threadIdx.x;
    if (o >= job.T) return;
    const C* v = static_cast<const C*>(job.v) + __ldg(&job.out_u[o]);
    C res[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        if (d2_partner_e(e) < e) continue;
        EntryAcc<C> acc;
        int32_t k = rp[e];
        const int32_t end = rp[e + 1];
        for (; k + 4 <= end; k += 4) {
            const C x0 = v[off[k]], x1 = v[off[k + 1]], x2 = v[off[k + 2]], x3 = v[off[k + 3]];
            C p{0, 0};
            term_mac(p, cf[k], x0);
            term_mac(p, cf[k + 1], x1);
            term_mac(p, cf[k + 2], x2);
            term_mac(p, cf[k + 3], x3);
            acc.add(p);
        }
        for (; k < end; ++k) {
            C p{0, 0};
            term_mac(p, cf[k], v[off[k]]);
            acc.add(p);
        }
        res[e] = acc.get();
    }
#pragma unroll
    for (int e = 0; e < E; ++e)
        if (d2_partner_e(e) < e) res[e] = cconj(res[d2_partner_e(e)]);
    C* out = static_cast<C*>(job.out) + static_cast<size_t>(o) * E;
    if (job.accumulate) {
#pragma unroll
        for (int e = 0; e < E; ++e) out[e] = cadd(out[e], res[e]);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) out[e] = res[e];
    }
}

template <class R>
__global__ void __launch_bounds__(CONTRACT_ROW_THREADS) k_contract_rows(const ContractJob* __restrict__ jobs, int N) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* res = reinterpret_cast<C*>(smem_raw);  // [threads][E + 1]
    const ContractJob job = jobs[blockIdx.y];
    const uint32_t o0 = blockIdx.x * CONTRACT_ROW_THREADS;
    if (o0 >= job.T) return;
    const uint32_t ot = min(static_cast<uint32_t>(CONTRACT_ROW_THREADS), job.T - o0);
    const uint32_t E = job.E, ld = E + 1;
    const uint32_t o = o0 + threadIdx.x;
    const C* coef = static_cast<const C*>(job.coef);
    const C* v = static_cast<const C*>(job.v);
    if (threadIdx.x < ot) {
        const uint32_t u = __ldg(&job.out_u[o]);
        for (uint32_t e = 0; e < E; ++e) {
            if (l4_partner(e, N) < e) continue;
            EntryAcc<C> acc;
            const int32_t b = __ldg(&job.rowptr[e]), end = __ldg(&job.rowptr[e + 1]);
            for (int32_t k = b; k < end; ++k) {
                const uint32_t sk = __ldg(&job.src[k]);
                C x = v[static_cast<size_t>(sk & 0x7fffffffu) * job.U + u];
                if (sk & 0x80000000u) x.y = -x.y;
                acc.add(cmul(coef[k], x));
            }
            res[threadIdx.x * ld + e] = acc.get();
        }
        for (uint32_t e = 0; e < E; ++e) {
            const uint32_t p = l4_partner(e, N);
            if (p < e) res[threadIdx.x * ld + e] = cconj(res[threadIdx.x * ld + p]);
        }
    }
    __syncthreads();
    C* out = static_cast<C*>(job.out) + static_cast<size_t>(o0) * E;
    const uint32_t total = ot * E;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const uint32_t ol = idx / E, e = idx - ol * E;
        out[idx] = job.accumulate ? cadd(out[idx], res[ol * ld + e]) : res[ol * ld + e];
    }
}

// Tiled variant for large L4 matrices: a CTA owns 32 consecutive entries x 32
// consecutive output times; each warp walks the CSR rows of some of its entries with
// warp-uniform (broadcast) coefficient loads while its lanes gather 32 consecutive times
// of the same source (one coalesced line per source), and the tile is written through
// shared memory as 32 contiguous entries per output time.
constexpr int CONTRACT_TILE = 32;
constexpr int CONTRACT_TILE_THREADS = 256;

template <class R>
__global__ void __launch_bounds__(CONTRACT_TILE_THREADS) k_contract_tiles(const ContractJob* __restrict__ jobs) {
    using C = cplx_t<R>;
    __shared__ C res[CONTRACT_TILE][CONTRACT_TILE + 1];  // [time][entry]
    const ContractJob job = jobs[blockIdx.z];
    const uint32_t o0 = blockIdx.x * CONTRACT_TILE, e0 = blockIdx.y * CONTRACT_TILE;
    if (o0 >= job.T || e0 >= job.E) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t o = o0 + lane;
    const uint32_t u = o < job.T ? __ldg(&job.out_u[o]) : 0u;
    const C* coef = static_cast<const C*>(job.coef);
    const C* v = static_cast<const C*>(job.v);
    for (int r = warp; r < CONTRACT_TILE; r += CONTRACT_TILE_THREADS / 32) {
        const uint32_t e = e0 + r;
        EntryAcc<C> acc;
        if (e < job.E) {
            const int32_t b = __ldg(&job.rowptr[e]), end = __ldg(&job.rowptr[e + 1]);
            for (int32_t k = b; k < end; ++k) {
                const uint32_t sk = __ldg(&job.src[k]);
                const C w = coef[k];
                C x = v[static_cast<size_t>(sk & 0x7fffffffu) * job.U + u];
                if (sk & 0x80000000u) x.y = -x.y;
                acc.add(cmul(w, x));
            }
        }
        res[lane][r] = acc.get();
    }
    __syncthreads();
    C* out = static_cast<C*>(job.out);
    for (int idx = threadIdx.x; idx < CONTRACT_TILE * CONTRACT_TILE; idx += CONTRACT_TILE_THREADS) {
        const int ol = idx / CONTRACT_TILE, el = idx % CONTRACT_TILE;
        const uint32_t oo = o0 + ol, e = e0 + el;
        if (oo >= job.T || e >= job.E) continue;
        C* p = out + static_cast<size_t>(oo) * job.E + e;
        *p = job.accumulate ? cadd(*p, res[ol][el]) : res[ol][el];
    }
}

}  // namespace taco
