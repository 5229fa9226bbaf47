// noalloc.cu -- L4(t) build for one instance that allocates no device or pinned memory.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree during their work -- code
// running inside a framework whose caching allocator already owns the device memory,
// latency-critical loops where an allocation would synchronise the device, and plugin
// hosts that forbid allocation after initialisation.  Every scratch buffer of the F/C/R
// pipeline and of the contraction (twiddle tables, partner spectra, FFT intermediates,
// convolutions, F/C/R values, coefficient table, job tables) is carved out of one fixed
// file-scope device array of TACO_NOALLOC_SCRATCH_BYTES.  The caller passes device
// pointers for gamma and for the L4 output, and a stream.
//
// The array exists once per GPU that loads the library and is held until the process
// exits.  Its host-side name is not a device address: host code only ever uses the
// address returned by cudaGetSymbolAddress, looked up once per device (with that device
// current) on the first call made on that device.  All calls share the array: calls whose
// work overlaps on the GPU (two host threads, or two streams) race on it.  Nothing in the
// array needs to start at zero: every buffer is written before it is read within a call.  Host-side metadata lives in
// ordinary heap vectors for the duration of the call and is copied with cudaMemcpyAsync
// from pageable memory, and the call synchronises its stream before it returns; a call on a
// stream that is being captured is rejected before any work.  gamma and the output must
// be device (or managed) memory of the current device, aligned for their complex type;
// anything else is rejected before any launch.  The FFT length is the power of two
// next_pow2(max(2 t_count - 1, pad * t_count)) (the allocating path also uses 3*2^k and
// 5*2^k lengths; the results agree to rounding).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "contract.cuh"
#include "engine.hpp"
#include "fcr_kernels.cuh"
#include "gw_coef.hpp"
#include "taco_b200.h"

// The fixed scratch (one per GPU that loads the library).
static __device__ __align__(256) unsigned char g_noalloc_scratch[TACO_NOALLOC_SCRATCH_BYTES];

namespace taco {

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
unsigned char* scratch_address() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw Error(kInvalidArgument, "no-alloc build: device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw Error(kCuda, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    return static_cast<unsigned char*>(g_addr[dev]);
}

template <class C>
__global__ void k_na_twiddle(C* out, uint32_t count, double denom) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= count) return;
    double s, c;
    sincospi(-2.0 * static_cast<double>(m) / denom, &s, &c);
    out[m] = from_d2<C>(make_double2(c, s));
}

std::size_t up256(std::size_t x) { return (x + 255) / 256 * 256; }

// Offsets inside the scratch; measure first, then place.
struct Carve {
    unsigned char* base;
    std::size_t off = 0;
    template <class T>
    T* take(std::size_t count) {
        off = up256(off);
        T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += count * sizeof(T);
        return p;
    }
};

template <class K>
void smem_attr(K kernel, std::size_t bytes) {
    raise_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}

template <class R>
void run(const SystemDesc& sys, const double2* gamma, std::size_t Nt, double dt, const std::vector<uint32_t>& tidx,
         std::size_t pad_factor, void* out, cudaStream_t st) {
    using C = cplx_t<R>;
    const int nf = sys.nf;
    const std::size_t nf3 = static_cast<std::size_t>(nf) * nf * nf;
    const std::size_t T = tidx.size();
    const std::size_t N2e = static_cast<std::size_t>(sys.N) * sys.N;
    const std::size_t E = N2e * N2e;
    // requested times
    uint32_t tmax = 0;
    for (uint32_t t : tidx) tmax = std::max(tmax, t);
    const std::size_t t_count = static_cast<std::size_t>(tmax) + 1;
    std::vector<uint32_t> uniq(tidx);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    const std::size_t U = uniq.size();
    std::vector<int> tmap(t_count, -1);
    for (std::size_t u = 0; u < U; ++u) tmap[uniq[u]] = static_cast<int>(u);
    std::vector<uint32_t> out_u(T);
    for (std::size_t o = 0; o < T; ++o) out_u[o] = static_cast<uint32_t>(tmap[tidx[o]]);
    // FFT length from max(tidx)+1 (F/C/R(t) depend on gamma[0..t] only)
    const std::size_t n_in = t_count;
    std::size_t target = 2 * n_in - 1;
    if (pad_factor > 0) target = std::max(target, pad_factor * n_in);
    const std::size_t Nfft = std::max<std::size_t>(8, next_pow2(target));
    if (Nfft > (std::size_t(1) << 22)) throw Error(kOverflow, "no-alloc build: FFT length above 2^22");
    const int L = ilog2(Nfft);
    const int L2 = (L + 1) / 2, L1 = L - L2, sfine = (L + 1) / 2;
    const int N1 = 1 << L1, N2 = 1 << L2;
    CoefTable coef;
    build_coef_table(sys.N, nf, sys.p2f.data(), sys.ops.data(), sys.num_ops, coef);
    const std::size_t nnz = coef.src.size();
    // schedule: the tuned tile sizes, shrunk like the allocating path's to fit shared memory
    const Tuning tune = get_tuning(L, std::is_same<R, float>::value);
    FftPlan<C> shape{};
    shape.L = L;
    shape.L1 = L1;
    shape.L2 = L2;
    shape.R = 1;
    const Geometry geo = geometry(shape, tune.col_tile, tune.row_tile);
    const int log2c = geo.log2c, col_threads = geo.col_threads, log2r = geo.log2r, row_threads = geo.row_threads;
    const std::size_t col_smem = geo.col_smem, row_smem = geo.row_smem;
    const unsigned col_grid = geo.col_grid, row_grid = geo.row_grid;
    const int inv_rows = static_cast<int>((t_count + N2 - 1) / N2);
    const bool inv_dft = inv_rows <= std::min(tune.inv_dft_rows, INV_DFT_MAXR);

    // layout: fixed part, then as many triples per chunk as fit
    const std::size_t n_spec = 2 * static_cast<std::size_t>(nf);
    auto place = [&](Carve& cv, std::size_t Q, C** tw, C** spec, C** scratch, C** conv, C** v, int** dtm,
                     uint32_t** dou, int32_t** drp, uint32_t** dsrc, C** dcoef, ColJob** cj, RowJob** rj,
                     InvJob** ij, ScanJob** sj, ContractJob** kj) {
        *tw = cv.take<C>(static_cast<std::size_t>(N1) + N2 + (Nfft >> sfine) + (std::size_t(1) << sfine));
        *spec = cv.take<C>(n_spec * Nfft);
        *conv = cv.take<C>(nf3 * 2 * t_count);
        *v = cv.take<C>(3 * nf3 * U);
        *dtm = cv.take<int>(t_count);
        *dou = cv.take<uint32_t>(T);
        *drp = cv.take<int32_t>(E + 1);
        *dsrc = cv.take<uint32_t>(std::max<std::size_t>(1, nnz));
        *dcoef = cv.take<C>(std::max<std::size_t>(1, nnz));
        *cj = cv.take<ColJob>(n_spec + nf3);
        *rj = cv.take<RowJob>(n_spec + nf3);
        *ij = cv.take<InvJob>(2 * nf3);
        *sj = cv.take<ScanJob>(nf3);
        *kj = cv.take<ContractJob>(1);
        *scratch = cv.take<C>(Q * 2 * Nfft);
    };
    C *tw, *spec, *scratch, *conv, *v, *dcoef;
    int* dtm;
    uint32_t *dou, *dsrc;
    int32_t* drp;
    ColJob* cjd;
    RowJob* rjd;
    InvJob* ijd;
    ScanJob* sjd;
    ContractJob* kjd;
    Carve m0{nullptr};
    place(m0, 0, &tw, &spec, &scratch, &conv, &v, &dtm, &dou, &drp, &dsrc, &dcoef, &cjd, &rjd, &ijd, &sjd, &kjd);
    const std::size_t fixed = up256(m0.off);
    const std::size_t per_tri = 2 * Nfft * sizeof(C);
    if (fixed + per_tri > TACO_NOALLOC_SCRATCH_BYTES)
        throw Error(kOverflow, "no-alloc build needs " + std::to_string(fixed + per_tri) +
                                   " bytes of scratch, above the fixed TACO_NOALLOC_SCRATCH_BYTES = " +
                                   std::to_string(static_cast<std::size_t>(TACO_NOALLOC_SCRATCH_BYTES)) +
                                   " (reduce max(tidx) or the number of requested times)");
    // the inverse pass launches 2 Q CTAs along y: Q <= 32767 keeps that within 65535
    const std::size_t Q = std::min<std::size_t>({(TACO_NOALLOC_SCRATCH_BYTES - fixed) / per_tri, nf3, 32767});
    Carve cv{scratch_address()};
    place(cv, Q, &tw, &spec, &scratch, &conv, &v, &dtm, &dou, &drp, &dsrc, &dcoef, &cjd, &rjd, &ijd, &sjd, &kjd);

    // twiddle tables (tw1 | tw2 | coarse | fine)
    FftPlan<C> plan;
    plan.L = L;
    plan.L1 = L1;
    plan.R = 1;
    plan.L2 = L2;
    plan.s = sfine;
    plan.tw1 = tw;
    plan.tw2 = tw + N1;
    plan.twc = tw + N1 + N2;
    plan.twf = tw + N1 + N2 + (Nfft >> sfine);
    auto fill = [&](const C* p, std::size_t count, double denom) {
        k_na_twiddle<C><<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(const_cast<C*>(p),
                                                                                    static_cast<uint32_t>(count), denom);
        cuda_check(cudaGetLastError(), "k_na_twiddle");
    };
    fill(plan.tw1, N1, static_cast<double>(N1));
    fill(plan.tw2, N2, static_cast<double>(N2));
    fill(plan.twc, Nfft >> sfine, static_cast<double>(Nfft >> sfine));
    fill(plan.twf, std::size_t(1) << sfine, static_cast<double>(Nfft));

    // job tables
    std::vector<ColJob> colj(n_spec + nf3);
    std::vector<RowJob> rowj(n_spec + nf3);
    std::vector<InvJob> invj(2 * nf3);
    std::vector<ScanJob> scanj(nf3);
    for (int half = 0; half < 2; ++half)
        for (int b = 0; b < nf; ++b) {
            const std::size_t k = static_cast<std::size_t>(half) * nf + b;
            ColJob& c = colj[k];
            c.g = gamma + static_cast<std::size_t>(b) * Nt;
            c.omega = 0.0;
            c.dt = dt;
            c.has_phase = 0;
            c.conj = half;
            c.n_in = static_cast<uint32_t>(n_in);
            c.out = spec + k * Nfft;
            rowj[k] = RowJob{c.out, nullptr, nullptr, nullptr};
        }
    const double scale = dt / static_cast<double>(Nfft);
    for (std::size_t q = 0; q < nf3; ++q) {
        const int tri = static_cast<int>(q);
        const int i = tri / (nf * nf), j = (tri / nf) % nf, k = tri % nf;
        const int jm = sys.mirror[j] >= 0 ? sys.mirror[j] : j;
        const double w = sys.omegas[i] + sys.omegas[j] + sys.omegas[k];
        C* z = scratch + (q % Q) * 2 * Nfft;
        C* wcb = z + Nfft;
        ColJob& c = colj[n_spec + q];
        c.g = gamma + static_cast<std::size_t>(i) * Nt;
        c.omega = w;
        c.dt = dt;
        c.has_phase = 1;
        c.conj = 0;
        c.n_in = static_cast<uint32_t>(n_in);
        c.out = z;
        rowj[n_spec + q] = RowJob{z, wcb, spec + static_cast<std::size_t>(jm) * Nfft,
                                  spec + static_cast<std::size_t>(nf + j) * Nfft};
        C* cf = conv + q * 2 * t_count;
        C* cc = cf + t_count;
        invj[2 * q] = InvJob{z, cf, static_cast<uint32_t>(t_count), scale};
        invj[2 * q + 1] = InvJob{wcb, cc, static_cast<uint32_t>(t_count), scale};
        ScanJob& s = scanj[q];
        s.gi = gamma + static_cast<std::size_t>(i) * Nt;
        s.gj = gamma + static_cast<std::size_t>(j) * Nt;
        s.gmj = gamma + static_cast<std::size_t>(jm) * Nt;
        s.omega = w;
        s.dt = dt;
        s.n_in = static_cast<uint32_t>(n_in);
        s.t_count = static_cast<uint32_t>(t_count);
        s.conv_f = cf;
        s.conv_c = cc;
        s.tmap = dtm;
        s.vf = v + q * U;
        s.vc = v + (nf3 + q) * U;
        s.vr = v + (2 * nf3 + q) * U;
    }
    ContractJob kjob{drp, dsrc, dcoef, v, dou, out, static_cast<uint32_t>(T), static_cast<uint32_t>(U),
                     static_cast<uint32_t>(E)};
    std::vector<C> coefc(std::max<std::size_t>(1, nnz));
    for (std::size_t e = 0; e < nnz; ++e) coefc[e] = from_d2<C>(coef.coef[e]);
    auto h2d = [&](void* dst, const void* src, std::size_t bytes) {
        if (bytes) cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(no-alloc meta)");
    };
    h2d(dtm, tmap.data(), tmap.size() * sizeof(int));
    h2d(dou, out_u.data(), out_u.size() * sizeof(uint32_t));
    h2d(drp, coef.rowptr.data(), coef.rowptr.size() * sizeof(int32_t));
    h2d(dsrc, coef.src.data(), nnz * sizeof(uint32_t));
    h2d(dcoef, coefc.data(), nnz * sizeof(C));
    h2d(cjd, colj.data(), colj.size() * sizeof(ColJob));
    h2d(rjd, rowj.data(), rowj.size() * sizeof(RowJob));
    h2d(ijd, invj.data(), invj.size() * sizeof(InvJob));
    h2d(sjd, scanj.data(), scanj.size() * sizeof(ScanJob));
    h2d(kjd, &kjob, sizeof(ContractJob));

    // launches (the same kernels as the allocating path)
    smem_attr(k_fwd_col<R>, col_smem);
    smem_attr(k_inv_col<R>, col_smem);
    smem_attr(k_row<R>, row_smem);
    k_fwd_col<R><<<dim3(col_grid, static_cast<unsigned>(n_spec)), col_threads, col_smem, st>>>(cjd, plan, log2c);
    cuda_check(cudaGetLastError(), "k_fwd_col(spectra)");
    k_row<R><<<dim3(row_grid, static_cast<unsigned>(n_spec)), row_threads, row_smem, st>>>(rjd, plan, log2r);
    cuda_check(cudaGetLastError(), "k_row(spectra)");
    for (std::size_t q0 = 0; q0 < nf3; q0 += Q) {
        const std::size_t nq = std::min(Q, nf3 - q0);
        k_fwd_col<R><<<dim3(col_grid, static_cast<unsigned>(nq)), col_threads, col_smem, st>>>(cjd + n_spec + q0,
                                                                                               plan, log2c);
        cuda_check(cudaGetLastError(), "k_fwd_col");
        k_row<R><<<dim3(row_grid, static_cast<unsigned>(nq)), row_threads, row_smem, st>>>(rjd + n_spec + q0, plan,
                                                                                           log2r);
        cuda_check(cudaGetLastError(), "k_row");
        if (inv_dft) {
            const unsigned g = static_cast<unsigned>((N2 + INV_DFT_THREADS - 1) / INV_DFT_THREADS);
            k_inv_col_dft<R><<<dim3(g, static_cast<unsigned>(2 * nq)), INV_DFT_THREADS, 0, st>>>(ijd + 2 * q0, plan,
                                                                                                 inv_rows);
        } else {
            k_inv_col<R><<<dim3(col_grid, static_cast<unsigned>(2 * nq)), col_threads, col_smem, st>>>(ijd + 2 * q0,
                                                                                                      plan, log2c);
        }
        cuda_check(cudaGetLastError(), "k_inv_col");
    }
    k_scan_assemble<R, SCAN_ITEMS, 3><<<static_cast<unsigned>(nf3), SCAN_THREADS, 0, st>>>(sjd);
    cuda_check(cudaGetLastError(), "k_scan_assemble");
    if (E * sizeof(C) <= 48 * 1024) {
        // several output times per CTA, their L4 matrices staged in shared memory
        const int OT = std::max(1, std::min(128, static_cast<int>((48 * 1024) / (E * sizeof(C)))));
        const std::size_t csmem = static_cast<std::size_t>(OT) * E * sizeof(C);
        k_contract<R><<<dim3(static_cast<unsigned>((T + OT - 1) / OT), 1), 256, csmem, st>>>(kjd, OT);
        cuda_check(cudaGetLastError(), "k_contract");
    } else {
        // large L4 matrices: 32 x 32 (time, entry) tiles in static shared memory
        const dim3 grid(static_cast<unsigned>((T + CONTRACT_TILE - 1) / CONTRACT_TILE),
                        static_cast<unsigned>((E + CONTRACT_TILE - 1) / CONTRACT_TILE), 1);
        k_contract_tiles<R><<<grid, CONTRACT_TILE_THREADS, 0, st>>>(kjd);
        cuda_check(cudaGetLastError(), "k_contract_tiles");
    }
    // the host vectors above are sources of the pending copies: finish before returning
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(no-alloc)");
}

// A caller's buffer must be device (or managed) memory of the current device, aligned for
// its complex type: a host address handed to the kernels would fault instead of failing.
void require_device_buffer(const void* p, std::size_t align, const char* what) {
    if (reinterpret_cast<std::uintptr_t>(p) % align != 0)
        throw Error(kInvalidArgument, std::string("no-alloc build: ") + what + " is not " + std::to_string(align) +
                                          "-byte aligned");
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();  // clear the sticky-free error state of the query
        throw Error(kInvalidArgument, std::string("no-alloc build: ") + what + " is not a CUDA allocation (" +
                                          cudaGetErrorString(e) + ")");
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        throw Error(kInvalidArgument, std::string("no-alloc build: ") + what + " must be device memory");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (a.type == cudaMemoryTypeDevice && a.device != dev)
        throw Error(kInvalidArgument, std::string("no-alloc build: ") + what + " is on device " +
                                          std::to_string(a.device) + ", not the current device " + std::to_string(dev));
}

}  // namespace

void noalloc_tcl4_build(const SystemDesc& sys, const double2* gamma, std::size_t Nt, double dt,
                        const std::vector<uint32_t>& tidx, bool fp32, std::size_t pad_factor, void* out,
                        cudaStream_t stream) {
    if (!gamma || !out) throw Error(kInvalidArgument, "no-alloc build: null gamma or output");
    // metadata is copied from pageable host memory and the stream is synchronised before
    // the call returns, neither of which a capturing stream accepts: checked before any
    // other CUDA call
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cuda_check(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
        throw Error(kInvalidArgument, "no-alloc build: the stream is being captured; call it outside stream capture");
    if (Nt == 0) throw Error(kInvalidArgument, "empty gamma_series");
    if (Nt >= (std::size_t(1) << 31)) throw Error(kOverflow, "Nt too large");
    if (!(dt > 0.0)) throw Error(kInvalidArgument, "dt must be > 0");
    if (sys.num_ops <= 0) throw Error(kInvalidArgument, "coupling_ops must be non-empty");
    if (static_cast<int>(sys.omegas.size()) != sys.nf || static_cast<int>(sys.mirror.size()) != sys.nf ||
        static_cast<int>(sys.p2f.size()) != sys.N * sys.N ||
        sys.ops.size() != static_cast<std::size_t>(sys.num_ops) * sys.N * sys.N)
        throw Error(kInvalidArgument, "system: metadata has wrong size");
    for (int b : sys.p2f) {
        if (b < 0) throw Error(kRuntime, "pair_to_freq contains -1 (missing frequency buckets)");
        if (b >= sys.nf) throw Error(kInvalidArgument, "pair_to_freq entry out of range");
    }
    for (int b : sys.mirror)
        if (b < 0 || b >= sys.nf) throw Error(kInvalidArgument, "mirror entry out of range");
    if (tidx.empty()) throw Error(kInvalidArgument, "no-alloc build: no time indices");
    for (uint32_t t : tidx)
        if (t >= Nt) throw Error(kOutOfRange, "time_index out of range");
    require_device_buffer(gamma, sizeof(double2), "gamma");
    require_device_buffer(out, fp32 ? sizeof(float2) : sizeof(double2), "L4_out");
    if (fp32) run<float>(sys, gamma, Nt, dt, tidx, pad_factor, out, stream);
    else run<double>(sys, gamma, Nt, dt, tidx, pad_factor, out, stream);
}

}  // namespace taco
