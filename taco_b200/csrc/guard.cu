// guard.cu -- precision guard of the FP32 form.
//
// L4(t) is a combination of the F/C/R values with heavy cancellation: at early times (before
// about one bath correlation time) L4 is orders of magnitude smaller than the values it is
// formed from, and for long, slowly decaying series the cancellation persists at all times.
// The FP32 FFT's round-off is spread evenly over the time axis, so the FP32 form's relative
// error is largest where L4 is smallest: measured FP32-vs-FP64 errors exceed 1e-3 in the
// first few hundred steps of long series, while the same series meet 1e-7 later on.  No
// FP32 evaluation of the F/C/R values can fix this (rounding exact values to FP32 alone
// gives 1e-4 at early times), so the guard measures the FP32 result against FP64 and
// recomputes in FP64 where it falls short:
//
//   1. the FP32 build of every instance (tcl4_build_direct / plan_create_direct);
//   2. per instance, a head [0, H) is built in FP64 (the causal rule makes its FFT length
//      follow H): H = max(512, t_count / 16) for direct calls, t_count / 4 for plans
//      (t_count = max(tidx)+1); its times below 2048 and below 256 are rebuilt by FP64 builds
//      of those times alone (FFTs of about 4096 and 512 points): at the earliest times L4 is
//      so small that the round-off of a long transform dominates it even in FP64 (the
//      reference's own FP64 convolution at FFT 2^19 misses the exact direct sums by a factor
//      of 100 at t < 64 on the batching form's longest series);
//   3. every head row is compared with the FP32 result; if the relative Frobenius difference
//      over the head's upper half [H/2, H) is within the tolerance (default 5e-7), the
//      instance is done -- the FP32 error decreases or stays flat with time after the early
//      transient in every measured series, so the rest keeps its FP32 values;
//   4. otherwise H grows fourfold (at most to t_count, which is a full FP64 build of the
//      instance) and step 2 repeats.
// The head an instance needs is the end of the latest dyadic window of times ([0, 64),
// [64, 128), [128, 256), ...) whose FP32 error misses the tolerance (none: no head).  A plan
// replays the FP32 graph followed by those FP64 heads and the row patch; a plan replayed on
// different inputs keeps the heads chosen at creation.  A direct call patches its whole
// accepted head and remembers, per gamma buffer, the accepted and the needed head and a
// fingerprint of the buffer's contents; a later call with the same fingerprint replays only
// the needed heads -- prepared FP64 plans, kept while consecutive calls have the same heads --
// on a side stream beside the FP32 pass, whose groups patch them on the device before their
// outputs are downloaded (no comparison), while a changed fingerprint is checked again from
// the accepted head.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iterator>
#include <map>
#include <string>
#include <tuple>
#include <memory>
#include <vector>

#include "common.cuh"
#include "engine.hpp"

namespace taco {

namespace {

std::atomic<double> g_guard_tol{5e-7};
thread_local GuardStats t_stats;
// What a direct call decided for a (gamma buffer, t_count): the head it accepted, the head
// the row profile requires, and a fingerprint of the buffer's contents.  A later call whose
// fingerprint matches builds the required head alone (no comparison round); one whose
// fingerprint differs starts from the accepted head and is checked as usual.
struct HeadMemory {
    uint32_t accepted = 0, required = 0;
    uint64_t fingerprint = 0;
};
thread_local std::map<std::pair<const void*, uint32_t>, HeadMemory> t_head_memory;


constexpr std::size_t kMinHead = 512;        // smallest head (samples)
constexpr std::size_t kWindowSamples = 256;  // requested times compared per check
// FP64 head rows per chunk of heads (a chunk's heads are built into one buffer and patched
// before the next chunk reuses it); settable for tests and tight memory
std::atomic<std::size_t> g_head_chunk_bytes{std::size_t(1) << 30};

struct GuardJob {
    const double2* h64;       // head rows [n][E], FP64
    float2* out32;            // patch destination rows (the output, or a device buffer for host outputs)
    const uint32_t* pos;      // [n] destination row of each head row
    const float2* cmp32;      // FP32 rows compared (the output, or the staged rows of a host output)
    const uint32_t* cmp_row;  // [nwin] row in cmp32 of each compared head row
    const uint32_t* win;      // [nwin] head rows compared
    double2* rowsum;          // [nwin] per compared row: (sum |cmp32 - h64|^2, sum |h64|^2)
    uint32_t n, nwin, E;
};

// Per compared row of job blockIdx.y (one warp per row): rowsum[q] = (sum |cmp32 - h64|^2,
// sum |h64|^2) over the row's entries.
__global__ void __launch_bounds__(256) k_guard_rows(const GuardJob* __restrict__ jobs) {
    const GuardJob job = jobs[blockIdx.y];
    const uint32_t q = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= job.nwin) return;
    const double2* r = job.h64 + static_cast<std::size_t>(job.win[q]) * job.E;
    const float2* f = job.cmp32 + static_cast<std::size_t>(job.cmp_row[q]) * job.E;
    double num = 0.0, den = 0.0;
    for (uint32_t e = lane; e < job.E; e += 32) {
        const double2 x = r[e];
        const float2 y = f[e];
        const double dx = static_cast<double>(y.x) - x.x, dy = static_cast<double>(y.y) - x.y;
        num += dx * dx + dy * dy;
        den += x.x * x.x + x.y * x.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    if (lane == 0) job.rowsum[q] = make_double2(num, den);
}

// out32[pos[k]][e] = h64[k][e] rounded to FP32, for every head row of job blockIdx.y.
__global__ void __launch_bounds__(256) k_guard_patch(const GuardJob* __restrict__ jobs) {
    const GuardJob job = jobs[blockIdx.y];
    const std::size_t total = static_cast<std::size_t>(job.n) * job.E;
    for (std::size_t idx = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const std::size_t k = idx / job.E, e = idx % job.E;
        const double2 r = job.h64[idx];
        job.out32[static_cast<std::size_t>(job.pos[k]) * job.E + e] =
            make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
    }
}

// Per row r < rows of a level and the head rows it would overwrite (E entries each; one warp
// per row): out[r] = (sum |l - h|^2, sum |l|^2).
__global__ void __launch_bounds__(256) k_level_rowsums(const double2* __restrict__ l, const double2* __restrict__ h,
                                                       uint32_t rows, uint32_t E, double2* __restrict__ out) {
    const uint32_t r = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    const double2* a = l + static_cast<std::size_t>(r) * E;
    const double2* b = h + static_cast<std::size_t>(r) * E;
    double num = 0.0, den = 0.0;
    for (uint32_t e = lane; e < E; e += 32) {
        const double2 x = a[e], y = b[e];
        const double dx = x.x - y.x, dy = x.y - y.y;
        num += dx * dx + dy * dy;
        den += x.x * x.x + x.y * x.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    if (lane == 0) out[r] = make_double2(num, den);
}

struct DevMem {
    void* p = nullptr;
    std::size_t cap = 0;
    void ensure(std::size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            std::size_t fr = 0, tot = 0;
            (void)cudaGetLastError();
            cudaMemGetInfo(&fr, &tot);
            throw Error(kCuda, "cudaMalloc(guard): " + std::string(cudaGetErrorString(e)) + " (" +
                                   std::to_string(bytes >> 20) + " MiB requested, " + std::to_string(fr >> 20) +
                                   " MiB free)");
        }
        cap = bytes;
    }
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() {
        if (p) cudaFree(p);
    }
};

// FNV-1a over bytes.
uint64_t fnv1a(uint64_t h, const void* p, std::size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (std::size_t k = 0; k < n; ++k) {
        h ^= b[k];
        h *= 1099511628211ull;
    }
    return h;
}

constexpr int kPrintSamples = 16;  // gamma samples per bucket in a fingerprint (first and last included)

__global__ void k_guard_gather(const double2* const* __restrict__ src, double2* __restrict__ out, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = *src[k];
}

// Fingerprints of the instances' gamma (the consumed samples of every bucket at 16 evenly
// spaced times, with the sizes and dt); device inputs are gathered by one launch.
std::vector<uint64_t> fingerprints(const std::vector<Tcl4Instance>& insts, const std::vector<uint32_t>& tcs,
                                   cudaStream_t st) {
    const std::size_t n = insts.size();
    std::vector<uint64_t> fp(n, 0);
    std::vector<const double2*> addr;
    std::vector<std::size_t> first(n, 0);
    std::vector<std::size_t> count(n, 0);
    for (std::size_t a = 0; a < n; ++a) {
        const Tcl4Instance& in = insts[a];
        if (in.tidx.empty()) continue;
        const uint32_t tc = tcs[a];
        const std::size_t n_in = std::min<std::size_t>(in.Nt, tc);
        first[a] = addr.size();
        for (int b = 0; b < in.sys.nf; ++b)
            for (int k = 0; k < kPrintSamples; ++k)
                addr.push_back(in.gamma + static_cast<std::size_t>(b) * in.Nt + (n_in - 1) * k / (kPrintSamples - 1));
        count[a] = addr.size() - first[a];
    }
    std::vector<double2> vals(addr.size());
    std::vector<const double2*> dev_addr;
    std::vector<std::size_t> dev_pos;
    for (std::size_t a = 0; a < n; ++a) {
        if (!count[a]) continue;
        if (insts[a].gamma_on_device) {
            for (std::size_t k = 0; k < count[a]; ++k) {
                dev_addr.push_back(addr[first[a] + k]);
                dev_pos.push_back(first[a] + k);
            }
        } else {
            for (std::size_t k = 0; k < count[a]; ++k) vals[first[a] + k] = *addr[first[a] + k];
        }
    }
    if (!dev_addr.empty()) {
        DevMem da, dv;
        da.ensure(dev_addr.size() * sizeof(double2*));
        dv.ensure(dev_addr.size() * sizeof(double2));
        std::vector<double2> got(dev_addr.size());
        cuda_check(cudaMemcpyAsync(da.p, dev_addr.data(), dev_addr.size() * sizeof(double2*), cudaMemcpyHostToDevice, st),
                   "cudaMemcpyAsync(fingerprint addresses)");
        k_guard_gather<<<static_cast<unsigned>((dev_addr.size() + 255) / 256), 256, 0, st>>>(
            static_cast<const double2* const*>(da.p), static_cast<double2*>(dv.p), static_cast<uint32_t>(dev_addr.size()));
        cuda_check(cudaGetLastError(), "k_guard_gather");
        count_launches(1);
        cuda_check(cudaMemcpyAsync(got.data(), dv.p, got.size() * sizeof(double2), cudaMemcpyDeviceToHost, st),
                   "cudaMemcpyAsync(fingerprint samples)");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(fingerprint)");
        for (std::size_t k = 0; k < dev_pos.size(); ++k) vals[dev_pos[k]] = got[k];
    }
    for (std::size_t a = 0; a < n; ++a) {
        if (!count[a]) continue;
        uint64_t h = 1469598103934665603ull;
        const uint64_t sizes[3] = {insts[a].Nt, static_cast<uint64_t>(insts[a].sys.nf), insts[a].tidx.size()};
        h = fnv1a(h, sizes, sizeof(sizes));
        h = fnv1a(h, &insts[a].dt, sizeof(double));
        h = fnv1a(h, vals.data() + first[a], count[a] * sizeof(double2));
        fp[a] = h;
    }
    return fp;
}

std::size_t entries(const Tcl4Instance& in) {
    const std::size_t N2 = static_cast<std::size_t>(in.sys.N) * in.sys.N;
    return N2 * N2;
}

uint32_t t_count_of(const Tcl4Instance& in) {
    uint32_t m = 0;
    for (uint32_t t : in.tidx) m = std::max(m, t);
    return m + 1;
}

// The head of one instance: its requested times below H (in request order), their output
// rows, and the head rows compared (times in [H/2, H), at most kWindowSamples evenly spaced;
// or every head row).
struct Head {
    std::size_t inst = 0;
    uint32_t H = 0, tc = 0;
    std::vector<uint32_t> times, pos, win;
    uint64_t rows_hash = 0;  // of times and pos
};

Head make_head(const std::vector<Tcl4Instance>& insts, std::size_t a, uint32_t H, uint32_t tc, bool all_rows = false) {
    Head h;
    h.inst = a;
    h.H = H;
    h.tc = tc;
    const Tcl4Instance& in = insts[a];
    std::vector<uint32_t> upper;
    for (std::size_t o = 0; o < in.tidx.size(); ++o) {
        const uint32_t t = in.tidx[o];
        if (t >= H) continue;
        if (2 * static_cast<std::size_t>(t) >= H) upper.push_back(static_cast<uint32_t>(h.times.size()));
        h.times.push_back(t);
        h.pos.push_back(static_cast<uint32_t>(o));
    }
    if (upper.empty() && !h.times.empty()) {
        // no requested time in the upper half: compare the latest quarter of the head rows
        std::vector<uint32_t> ord(h.times.size());
        for (std::size_t k = 0; k < ord.size(); ++k) ord[k] = static_cast<uint32_t>(k);
        std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return h.times[x] > h.times[y]; });
        upper.assign(ord.begin(), ord.begin() + std::max<std::size_t>(1, ord.size() / 4));
    }
    h.rows_hash = fnv1a(fnv1a(1469598103934665603ull, h.times.data(), h.times.size() * sizeof(uint32_t)), h.pos.data(),
                        h.pos.size() * sizeof(uint32_t));
    if (all_rows) {  // every head row (the row profile that sets a plan's final head)
        h.win.resize(h.times.size());
        for (std::size_t k = 0; k < h.win.size(); ++k) h.win[k] = static_cast<uint32_t>(k);
    } else if (upper.size() <= kWindowSamples) {
        h.win = upper;
    } else {
        for (std::size_t k = 0; k < kWindowSamples; ++k) h.win.push_back(upper[k * upper.size() / kWindowSamples]);
    }
    return h;
}

// Per call: the t_count and the head templates of each distinct time list (the instances of
// a call that name one caller array share one list, so each is scanned once).
class TimeCache {
public:
    uint32_t t_count(const Tcl4Instance& in) {
        if (in.tidx.empty()) return 0;
        auto it = tc_.find(in.tidx.identity());
        if (it == tc_.end()) it = tc_.emplace(in.tidx.identity(), t_count_of(in)).first;
        return it->second;
    }
    Head head(const std::vector<Tcl4Instance>& insts, std::size_t a, uint32_t H, uint32_t tc, bool all_rows = false) {
        const auto key = std::make_tuple(insts[a].tidx.identity(), H, all_rows);
        auto it = heads_.find(key);
        if (it == heads_.end()) it = heads_.emplace(key, make_head(insts, a, H, tc, all_rows)).first;
        Head h = it->second;
        h.inst = a;
        return h;
    }

private:
    std::map<const void*, uint32_t> tc_;
    std::map<std::tuple<const void*, uint32_t, bool>, Head> heads_;
};

// FP64 builds of the heads of `heads` (into one device buffer of head rows), chunked so
// that each chunk's rows fit the chunk size (a single head may exceed it).
template <class Fn>
void for_chunks(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads, Fn fn) {
    std::size_t k0 = 0;
    while (k0 < heads.size()) {
        std::size_t k1 = k0, bytes = 0;
        while (k1 < heads.size() && k1 - k0 < 32768) {  // jobs of one launch along grid y
            const std::size_t b = heads[k1].times.size() * entries(insts[heads[k1].inst]) * sizeof(double2);
            if (k1 > k0 && bytes + b > g_head_chunk_bytes.load()) break;
            bytes += b;
            ++k1;
        }
        fn(k0, k1, bytes);
        k0 = k1;
    }
}

// Head instances (FP64, device output rows at `base` + offsets) for heads [k0, k1).
std::vector<Tcl4Instance> head_instances(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads,
                                         std::size_t k0, std::size_t k1, double2* base, std::vector<std::size_t>& off) {
    std::vector<Tcl4Instance> hi;
    off.assign(k1 - k0, 0);
    std::size_t o = 0;
    for (std::size_t k = k0; k < k1; ++k) {
        const Tcl4Instance& in = insts[heads[k].inst];
        Tcl4Instance h;
        h.sys = in.sys;
        h.gamma = in.gamma;
        h.gamma_on_device = in.gamma_on_device;
        h.Nt = in.Nt;
        h.dt = in.dt;
        h.tidx = heads[k].times;
        h.out = base + o;
        h.out_on_device = true;
        h.internal = true;
        off[k - k0] = o;
        o += heads[k].times.size() * entries(in);
        hi.push_back(std::move(h));
    }
    return hi;
}

// Short-FFT levels of the heads [k0, k1): for a head longer than `bound` whose times are
// sorted, an FP64 build of its times below `bound` alone, written over the head's first rows.
// The causal rule gives such a build an FFT of about 2 bound points, whose round-off at the
// earliest, tiny L4 values is orders of magnitude below that of the head's own transform.
constexpr uint32_t kLevels[] = {2048, 256};

// Rows of head h that the level of `bound` rebuilds (0: the level does not apply).
std::size_t level_rows(const Head& h, uint32_t bound) {
    if (h.H <= bound || !std::is_sorted(h.times.begin(), h.times.end())) return 0;
    return static_cast<std::size_t>(std::lower_bound(h.times.begin(), h.times.end(), bound) - h.times.begin());
}

// keep (optional): per head of [k0, k1), whether this level is built at all.
std::vector<Tcl4Instance> level_instances(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads,
                                          std::size_t k0, std::size_t k1, double2* base,
                                          const std::vector<std::size_t>& off, uint32_t bound,
                                          const std::vector<char>* keep = nullptr) {
    std::vector<Tcl4Instance> li;
    for (std::size_t k = k0; k < k1; ++k) {
        const Head& h = heads[k];
        if (keep && !(*keep)[k - k0]) continue;
        const std::size_t n = level_rows(h, bound);
        if (n == 0) continue;
        const Tcl4Instance& in = insts[h.inst];
        Tcl4Instance l;
        l.sys = in.sys;
        l.gamma = in.gamma;
        l.gamma_on_device = in.gamma_on_device;
        l.Nt = in.Nt;
        l.dt = in.dt;
        l.tidx = std::vector<uint32_t>(h.times.begin(), h.times.begin() + n);
        l.out = base + off[k - k0];
        l.out_on_device = true;
        l.internal = true;
        li.push_back(std::move(l));
    }
    return li;
}

// The FP64 heads [k0, k1) into their rows at base + off: the head builds, then the short-FFT
// levels coarse to fine (each overwriting the rows below its bound).
void build_heads(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads, std::size_t k0, std::size_t k1,
                 double2* base, std::vector<std::size_t>& off, const BuildOptions& o64, cudaStream_t st) {
    std::vector<Tcl4Instance> hi = head_instances(insts, heads, k0, k1, base, off);
    tcl4_build_direct(hi, o64, st);  // synchronous
    for (uint32_t bound : kLevels) {
        std::vector<Tcl4Instance> li = level_instances(insts, heads, k0, k1, base, off, bound);
        if (!li.empty()) tcl4_build_direct(li, o64, st);
    }
}

// Which short-FFT levels of the heads [k0, k1) change their rows.  The heads and then each
// level (coarse to fine) are built once in FP64; a level is kept for a head when, in some
// window of times below its bound ([0, 64), [64, 128), ...), its rows differ from the rows it
// would overwrite (the head's, or a kept coarser level's) by more than tol / 8 (relative
// Frobenius); the others are left out of the replays.  keep[q][k - k0] for level q.
std::vector<std::vector<char>> needed_levels(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads,
                                             std::size_t k0, std::size_t k1, const BuildOptions& o64, double tol,
                                             cudaStream_t st) {
    if (!st) st = default_stream();  // builds, comparisons and copies in one stream's order
    const std::size_t n = k1 - k0;
    std::vector<std::vector<char>> keep(std::size(kLevels), std::vector<char>(n, 0));
    bool any = false;
    for (uint32_t bound : kLevels)
        for (std::size_t k = k0; k < k1; ++k) any = any || level_rows(heads[k], bound) > 0;
    if (!any) return keep;
    std::size_t bytes = 256;
    for (std::size_t k = k0; k < k1; ++k) bytes += heads[k].times.size() * entries(insts[heads[k].inst]) * sizeof(double2);
    DevMem hrows, lrows;
    hrows.ensure(bytes);
    lrows.ensure(bytes);
    std::vector<std::size_t> off;
    std::vector<Tcl4Instance> hi = head_instances(insts, heads, k0, k1, static_cast<double2*>(hrows.p), off);
    tcl4_build_direct(hi, o64, st);  // synchronous
    DevMem sums;
    std::vector<double2> rs;
    for (std::size_t q = 0; q < std::size(kLevels); ++q) {
        const uint32_t bound = kLevels[q];
        std::vector<char> all(n, 1);
        std::vector<Tcl4Instance> li =
            level_instances(insts, heads, k0, k1, static_cast<double2*>(lrows.p), off, bound, &all);
        if (li.empty()) continue;
        tcl4_build_direct(li, o64, st);
        for (std::size_t k = k0; k < k1; ++k) {
            const Head& h = heads[k];
            const std::size_t rows = level_rows(h, bound);
            if (!rows) continue;
            const std::size_t E = entries(insts[h.inst]);
            const double2* hp = static_cast<const double2*>(hrows.p) + off[k - k0];
            const double2* lp = static_cast<const double2*>(lrows.p) + off[k - k0];
            // per row on the device: (sum |level - head|^2, sum |level|^2) over the entries
            sums.ensure(rows * sizeof(double2));
            k_level_rowsums<<<static_cast<unsigned>((rows + 7) / 8), 256, 0, st>>>(
                lp, hp, static_cast<uint32_t>(rows), static_cast<uint32_t>(E), static_cast<double2*>(sums.p));
            cuda_check(cudaGetLastError(), "k_level_rowsums");
            count_launches(1);
            rs.resize(rows);
            cuda_check(cudaMemcpyAsync(rs.data(), sums.p, rows * sizeof(double2), cudaMemcpyDeviceToHost, st),
                       "cudaMemcpyAsync(levels)");
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(levels)");
            std::vector<double> num(40, 0.0), den(40, 0.0);
            for (std::size_t r = 0; r < rows; ++r) {
                int w = 0;
                while (w < 39 && (std::size_t(64) << w) <= h.times[r]) ++w;
                num[w] += rs[r].x;
                den[w] += rs[r].y;
            }
            bool need = false;
            for (int w = 0; w < 40 && !need; ++w)
                need = den[w] > 0.0 ? std::sqrt(num[w] / den[w]) > tol / 8 : num[w] > 0.0;
            keep[q][k - k0] = need ? 1 : 0;
            // a kept level's rows are what the next, finer level would overwrite
            if (need)
                cuda_check(cudaMemcpyAsync(const_cast<double2*>(hp), lp, rows * E * sizeof(double2),
                                           cudaMemcpyDeviceToDevice, st),
                           "cudaMemcpyAsync(levels)");
        }
    }
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(levels)");
    return keep;
}

// Device jobs of heads [k0, k1) and their index arrays, as one host image of the device
// layout at `dev` (null: measure only).  Host outputs compare against their window rows
// staged at `stage` (row offsets `stage_off`) and patch into `hpatch` (offsets `hpatch_off`).
struct JobImage {
    std::vector<unsigned char> host;
};

JobImage job_image(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads, std::size_t k0,
                   std::size_t k1, const double2* base, const std::vector<std::size_t>& off, unsigned char* dev,
                   const float2* stage = nullptr, const std::vector<std::size_t>* stage_off = nullptr,
                   float2* hpatch = nullptr, const std::vector<std::size_t>* hpatch_off = nullptr,
                   double2* rowsum = nullptr, const std::vector<std::size_t>* rowsum_off = nullptr) {
    const std::size_t n = k1 - k0;
    std::size_t bytes = n * sizeof(GuardJob);
    std::vector<std::size_t> pos_off(n), cmp_off(n), win_off(n);
    for (std::size_t k = 0; k < n; ++k) {
        pos_off[k] = bytes;
        bytes += heads[k0 + k].pos.size() * sizeof(uint32_t);
        cmp_off[k] = bytes;
        bytes += heads[k0 + k].win.size() * sizeof(uint32_t);
        win_off[k] = bytes;
        bytes += heads[k0 + k].win.size() * sizeof(uint32_t);
    }
    JobImage img;
    img.host.assign(bytes, 0);
    auto at = [&](std::size_t o) { return reinterpret_cast<const uint32_t*>(reinterpret_cast<std::uintptr_t>(dev) + o); };
    for (std::size_t k = 0; k < n; ++k) {
        const Head& h = heads[k0 + k];
        const Tcl4Instance& in = insts[h.inst];
        const bool host_out = !in.out_on_device;
        GuardJob j;
        j.h64 = base + off[k];
        j.pos = at(pos_off[k]);
        j.cmp_row = at(cmp_off[k]);
        j.win = at(win_off[k]);
        j.rowsum = rowsum ? rowsum + (*rowsum_off)[k] : nullptr;
        j.n = static_cast<uint32_t>(h.pos.size());
        j.nwin = static_cast<uint32_t>(h.win.size());
        j.E = static_cast<uint32_t>(entries(in));
        std::vector<uint32_t> pos(h.pos), cmp(h.win.size());
        if (host_out) {
            j.out32 = hpatch ? hpatch + (*hpatch_off)[k] : nullptr;
            j.cmp32 = stage ? stage + (*stage_off)[k] : nullptr;
            for (std::size_t q = 0; q < pos.size(); ++q) pos[q] = static_cast<uint32_t>(q);
            for (std::size_t q = 0; q < cmp.size(); ++q) cmp[q] = static_cast<uint32_t>(q);
        } else {
            j.out32 = static_cast<float2*>(in.out);
            j.cmp32 = static_cast<const float2*>(in.out);
            for (std::size_t q = 0; q < cmp.size(); ++q) cmp[q] = h.pos[h.win[q]];
        }
        std::memcpy(img.host.data() + k * sizeof(GuardJob), &j, sizeof(GuardJob));
        if (!pos.empty()) std::memcpy(img.host.data() + pos_off[k], pos.data(), pos.size() * sizeof(uint32_t));
        if (!cmp.empty()) std::memcpy(img.host.data() + cmp_off[k], cmp.data(), cmp.size() * sizeof(uint32_t));
        if (!h.win.empty()) std::memcpy(img.host.data() + win_off[k], h.win.data(), h.win.size() * sizeof(uint32_t));
    }
    return img;
}

unsigned patch_blocks(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads, std::size_t k0,
                      std::size_t k1) {
    std::size_t most = 1;
    for (std::size_t k = k0; k < k1; ++k) most = std::max(most, heads[k].pos.size() * entries(insts[heads[k].inst]));
    return static_cast<unsigned>(std::min<std::size_t>((most + 255) / 256, 592));
}

struct Decision {
    std::vector<Head> heads;  // final heads of the instances that need one
};

// Heads built before the guard loop starts (concurrently with the FP32 pass).
struct PreHeads {
    std::vector<Head> heads;
    DevMem* temp = nullptr;  // the calling thread's guard scratch
    std::vector<std::size_t> off;
};

// Grow-only pinned host memory (asynchronous uploads from it do not wait for the device).
struct PinnedMem {
    void* p = nullptr;
    std::size_t cap = 0;
    void ensure(std::size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        cuda_check(cudaHostAlloc(&p, bytes, cudaHostAllocDefault), "cudaHostAlloc(guard)");
        cap = bytes;
    }
    PinnedMem() = default;
    PinnedMem(const PinnedMem&) = delete;
    PinnedMem& operator=(const PinnedMem&) = delete;
    ~PinnedMem() {
        if (p) cudaFreeHost(p);
    }
};

// The guard's device buffers of the calling thread and device: grow-only and kept across calls
// (allocating and freeing them every call synchronised the device and cost milliseconds).
struct GuardScratch {
    DevMem temp, meta, rowsums, stage, hpatch, jobs;
    PinnedMem jobs_host;
    std::vector<float2> stage_host;
};
std::map<int, std::unique_ptr<GuardScratch>>& guard_scratch_map() {
    thread_local std::map<int, std::unique_ptr<GuardScratch>> m;
    return m;
}
GuardScratch& guard_scratch() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    auto& p = guard_scratch_map()[dev];
    if (!p) p = std::make_unique<GuardScratch>();
    return *p;
}

// Options of the FP64 head builds: the causal FFT length of each head (short transforms are
// both cheaper and more accurate at the first times) whatever length the FP32 pass uses.
BuildOptions head_options(const BuildOptions& opt) {
    BuildOptions o = opt;
    o.fp32 = false;
    o.fcr_ms = nullptr;
    o.out_hook = nullptr;
    o.causal_truncation = true;
    o.pad_factor = 0;
    return o;
}

// Runs the guard loop: FP64 heads, comparison, growth.  With `patch`, accepted heads are
// written into the outputs right away (direct calls); otherwise only the final heads are
// returned (plans).  The FP32 results must already be in the outputs.  Comparison and
// rounding run on the device; a host output stages its compared rows up and its patched
// rows down (one copy per run of consecutive output rows).
Decision run_guard(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, cudaStream_t st, bool patch,
                   PreHeads* pre = nullptr, bool trusted = false, const std::vector<uint64_t>* fps = nullptr) {
    const double tol = g_guard_tol.load();
    const BuildOptions o64 = head_options(opt);
    // every head row is compared: the row profile sets the head a plan replays, and the head
    // a direct call remembers for its next call on the same inputs; a plan's first head is a
    // quarter of the series, a direct call's a sixteenth
    auto profile = [&](std::size_t) { return true; };
    std::vector<Head> pending;
    for (std::size_t a = 0; a < insts.size(); ++a) {
        if (insts[a].tidx.empty()) continue;
        const uint32_t tc = t_count_of(insts[a]);
        const std::size_t frac = patch ? 16 : 4;
        uint32_t H = static_cast<uint32_t>(std::min<std::size_t>(tc, std::max<std::size_t>(kMinHead, (tc + frac - 1) / frac)));
        if (patch) {
            auto it = t_head_memory.find({insts[a].gamma, tc});
            if (it != t_head_memory.end() && it->second.accepted) H = it->second.accepted;
        }
        Head h = make_head(insts, a, H, tc, profile(a));
        if (!h.times.empty()) pending.push_back(std::move(h));
    }
    if (pre) pending = pre->heads;  // built already: the first round only evaluates them
    Decision dec;
    GuardScratch& gs = guard_scratch();
    DevMem &temp = gs.temp, &meta = gs.meta, &rowsums = gs.rowsums, &stage = gs.stage, &hpatch = gs.hpatch;
    std::vector<float2>& stage_host = gs.stage_host;
    t_stats = GuardStats{};
    t_stats.instances = insts.size();
    while (!pending.empty()) {
        ++t_stats.rounds;
        std::vector<Head> next;
        const bool prebuilt = pre && t_stats.rounds == 1;
        auto chunk = [&](std::size_t k0, std::size_t k1, std::size_t bytes) {
            const std::size_t n = k1 - k0;
            std::vector<std::size_t> off;
            double2* base = nullptr;
            if (prebuilt) {
                base = static_cast<double2*>(pre->temp->p);
                off = pre->off;
            } else {
                temp.ensure(std::max<std::size_t>(bytes, 256));
                base = static_cast<double2*>(temp.p);
                build_heads(insts, pending, k0, k1, base, off, o64, st);
            }
            // host outputs: their window rows staged up, their patched rows in a device buffer
            std::vector<std::size_t> soff(n, 0), poff(n, 0);
            std::size_t srows = 0, prows = 0;
            for (std::size_t k = k0; k < k1; ++k) {
                const Head& h = pending[k];
                const Tcl4Instance& in = insts[h.inst];
                if (in.out_on_device) continue;
                const std::size_t E = entries(in);
                soff[k - k0] = srows;
                poff[k - k0] = prows;
                if (!(prebuilt && trusted)) srows += h.win.size() * E;  // trusted heads compare nothing
                prows += h.pos.size() * E;
            }
            if (srows) {
                stage_host.resize(srows);
                for (std::size_t k = k0; k < k1; ++k) {
                    const Head& h = pending[k];
                    const Tcl4Instance& in = insts[h.inst];
                    if (in.out_on_device) continue;
                    const std::size_t E = entries(in);
                    const float2* f = static_cast<const float2*>(in.out);
                    for (std::size_t q = 0; q < h.win.size(); ++q)
                        std::memcpy(stage_host.data() + soff[k - k0] + q * E,
                                    f + static_cast<std::size_t>(h.pos[h.win[q]]) * E, E * sizeof(float2));
                }
                stage.ensure(srows * sizeof(float2));
                cuda_check(cudaMemcpyAsync(stage.p, stage_host.data(), srows * sizeof(float2), cudaMemcpyHostToDevice, st),
                           "cudaMemcpyAsync(guard stage)");
            }
            if (prows) hpatch.ensure(prows * sizeof(float2));
            const float2* stage_p = static_cast<const float2*>(stage.p);
            float2* hpatch_p = static_cast<float2*>(hpatch.p);
            if (prebuilt && trusted) {
                // heads that a matching fingerprint says suffice: patch them, no comparison
                std::vector<std::size_t> roff0(n, 0);
                meta.ensure(job_image(insts, pending, k0, k1, base, off, nullptr).host.size() + 256);
                JobImage img = job_image(insts, pending, k0, k1, base, off, static_cast<unsigned char*>(meta.p), stage_p,
                                         &soff, hpatch_p, &poff, nullptr, &roff0);
                cuda_check(cudaMemcpyAsync(meta.p, img.host.data(), img.host.size(), cudaMemcpyHostToDevice, st),
                           "cudaMemcpyAsync(guard jobs)");
                const dim3 grid(patch_blocks(insts, pending, k0, k1), static_cast<unsigned>(n));
                k_guard_patch<<<grid, 256, 0, st>>>(static_cast<const GuardJob*>(meta.p));
                cuda_check(cudaGetLastError(), "k_guard_patch");
                count_launches(1);
                for (std::size_t k = k0; k < k1; ++k) {
                    const Head& h = pending[k];
                    const Tcl4Instance& in = insts[h.inst];
                    ++t_stats.heads;
                    t_stats.head_rows += h.times.size();
                    t_stats.rows += in.tidx.size();
                    if (h.H >= h.tc) ++t_stats.full;
                    if (in.out_on_device) continue;
                    const std::size_t E = entries(in);
                    float2* f = static_cast<float2*>(in.out);
                    const float2* src = hpatch_p + poff[k - k0];
                    std::size_t q = 0;
                    while (q < h.pos.size()) {
                        std::size_t r = q + 1;
                        while (r < h.pos.size() && h.pos[r] == h.pos[r - 1] + 1) ++r;
                        cuda_check(cudaMemcpyAsync(f + static_cast<std::size_t>(h.pos[q]) * E, src + q * E,
                                                   (r - q) * E * sizeof(float2), cudaMemcpyDeviceToHost, st),
                                   "cudaMemcpyAsync(guard rows)");
                        q = r;
                    }
                }
                cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(guard patch)");
                return;
            }
            // per compared row: (squared difference, squared FP64 norm)
            std::vector<std::size_t> roff(n, 0);
            std::size_t nrows = 0, most_win = 1;
            for (std::size_t k = k0; k < k1; ++k) {
                roff[k - k0] = nrows;
                nrows += pending[k].win.size();
                most_win = std::max(most_win, pending[k].win.size());
            }
            rowsums.ensure(std::max<std::size_t>(1, nrows) * sizeof(double2));
            double2* rowsum_p = static_cast<double2*>(rowsums.p);
            meta.ensure(job_image(insts, pending, k0, k1, base, off, nullptr).host.size() + 256);
            JobImage img = job_image(insts, pending, k0, k1, base, off, static_cast<unsigned char*>(meta.p), stage_p, &soff,
                                     hpatch_p, &poff, rowsum_p, &roff);
            cuda_check(cudaMemcpyAsync(meta.p, img.host.data(), img.host.size(), cudaMemcpyHostToDevice, st),
                       "cudaMemcpyAsync(guard jobs)");
            k_guard_rows<<<dim3(static_cast<unsigned>((most_win + 7) / 8), static_cast<unsigned>(n)), 256, 0, st>>>(
                static_cast<const GuardJob*>(meta.p));
            cuda_check(cudaGetLastError(), "k_guard_rows");
            count_launches(1);
            std::vector<double2> rs(std::max<std::size_t>(1, nrows));
            if (nrows)
                cuda_check(cudaMemcpyAsync(rs.data(), rowsum_p, nrows * sizeof(double2), cudaMemcpyDeviceToHost, st),
                           "cudaMemcpyAsync(guard rows)");
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(guard)");
            // decide: the window [H/2, H) within the tolerance, or the whole series in FP64
            auto ok_of = [&](double num, double den) { return den > 0.0 ? std::sqrt(num / den) <= tol : num == 0.0; };
            std::vector<char> accept(n, 0);
            std::vector<uint32_t> final_h(n, 0);
            for (std::size_t k = k0; k < k1; ++k) {
                const Head& h = pending[k];
                const double2* r = rs.data() + roff[k - k0];
                double wn = 0.0, wd = 0.0;
                for (std::size_t q = 0; q < h.win.size(); ++q)
                    if (2 * static_cast<std::size_t>(h.times[h.win[q]]) >= h.H || !profile(h.inst)) {
                        wn += r[q].x;
                        wd += r[q].y;
                    }
                if (ok_of(wn, wd) || h.H >= h.tc) {
                    accept[k - k0] = 1;
                    final_h[k - k0] = h.H;
                    if (profile(h.inst)) {
                        // the head a plan replays: up to the end of the latest dyadic window
                        // ([0, 64), [64, 128), [128, 256), ...) that misses the tolerance
                        std::vector<double> num(40, 0.0), den(40, 0.0);
                        for (std::size_t q = 0; q < h.win.size(); ++q) {
                            const uint32_t t = h.times[h.win[q]];
                            int w = 0;
                            while (w < 39 && (std::size_t(64) << w) <= t) ++w;
                            num[w] += r[q].x;
                            den[w] += r[q].y;
                        }
                        uint32_t hf = 0;
                        for (int w = 39; w >= 0; --w)
                            if (den[w] > 0.0 || num[w] > 0.0) {
                                if (!ok_of(num[w], den[w])) {
                                    hf = static_cast<uint32_t>(std::min<std::size_t>(h.H, std::size_t(64) << w));
                                    break;
                                }
                            }
                        final_h[k - k0] = hf;
                    }
                } else {
                    const uint32_t H = static_cast<uint32_t>(std::min<std::size_t>(h.tc, 4 * static_cast<std::size_t>(h.H)));
                    next.push_back(make_head(insts, h.inst, H, h.tc, profile(h.inst)));
                }
            }
            if (patch) {
                // rejected heads patch nothing
                for (std::size_t k = 0; k < n; ++k)
                    if (!accept[k]) {
                        GuardJob j;
                        std::memcpy(&j, img.host.data() + k * sizeof(GuardJob), sizeof(GuardJob));
                        j.n = 0;
                        std::memcpy(img.host.data() + k * sizeof(GuardJob), &j, sizeof(GuardJob));
                    }
                cuda_check(cudaMemcpyAsync(meta.p, img.host.data(), n * sizeof(GuardJob), cudaMemcpyHostToDevice, st),
                           "cudaMemcpyAsync(guard jobs)");
                const dim3 grid(patch_blocks(insts, pending, k0, k1), static_cast<unsigned>(n));
                k_guard_patch<<<grid, 256, 0, st>>>(static_cast<const GuardJob*>(meta.p));
                cuda_check(cudaGetLastError(), "k_guard_patch");
                count_launches(1);
                // host outputs: one copy per run of consecutive output rows
                for (std::size_t k = k0; k < k1; ++k) {
                    const Head& h = pending[k];
                    const Tcl4Instance& in = insts[h.inst];
                    if (!accept[k - k0] || in.out_on_device) continue;
                    const std::size_t E = entries(in);
                    float2* f = static_cast<float2*>(in.out);
                    const float2* src = hpatch_p + poff[k - k0];
                    std::size_t q = 0;
                    while (q < h.pos.size()) {
                        std::size_t r = q + 1;
                        while (r < h.pos.size() && h.pos[r] == h.pos[r - 1] + 1) ++r;
                        cuda_check(cudaMemcpyAsync(f + static_cast<std::size_t>(h.pos[q]) * E, src + q * E,
                                                   (r - q) * E * sizeof(float2), cudaMemcpyDeviceToHost, st),
                                   "cudaMemcpyAsync(guard rows)");
                        q = r;
                    }
                }
                cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(guard patch)");
            }
            if (patch) {
                if (t_head_memory.size() > 65536) t_head_memory.clear();
                for (std::size_t k = k0; k < k1; ++k)
                    if (accept[k - k0]) {
                        HeadMemory& m = t_head_memory[{insts[pending[k].inst].gamma, pending[k].tc}];
                        m.accepted = pending[k].H;
                        m.required = final_h[k - k0];
                        m.fingerprint = fps ? (*fps)[pending[k].inst] : 0;
                    }
            }
            for (std::size_t k = k0; k < k1; ++k)
                if (accept[k - k0]) {
                    const Head& h0 = pending[k];
                    // a direct call has patched its whole accepted head; a plan replays the
                    // head the profile requires
                    const uint32_t keep = patch ? h0.H : final_h[k - k0];
                    if (keep == 0) continue;  // FP32 within the tolerance everywhere
                    Head h = keep == h0.H ? h0 : make_head(insts, h0.inst, keep, h0.tc);
                    if (h.times.empty()) continue;
                    ++t_stats.heads;
                    t_stats.head_rows += h.times.size();
                    t_stats.rows += insts[h.inst].tidx.size();
                    if (h.H >= h.tc) ++t_stats.full;
                    dec.heads.push_back(std::move(h));
                }
        };
        if (prebuilt) chunk(0, pending.size(), 0);
        else for_chunks(insts, pending, chunk);
        pending.swap(next);
    }
    return dec;
}

// A direct call's remembered heads as prepared FP64 plans -- the heads, then each short-FFT
// level over the heads' first rows -- replayed on a side stream while the FP32 pass runs; the
// pass's groups wait for them on the device and patch.  Host gamma is copied each call (from
// the caller's buffers, on the side stream) into a device buffer of the samples the heads
// consume.  One set per thread and device, kept while
// consecutive calls have the same heads (instances, systems, buffers, times, head lengths).
struct HeadPlans {
    uint64_t key = 0;
    std::vector<std::size_t> off;      // first element of each head's rows in `rows`
    std::vector<std::size_t> pos_off;  // first entry of each head's output positions in `pos`
    DevMem rows, work, gam, pos;
    struct Upload {
        const double2* src;
        std::size_t nf, stride, n, dst;  // buckets, source stride, samples per bucket, first element in gam
        uint32_t chunk;
    };
    std::vector<Upload> uploads;
    std::size_t gam_elems = 0;
    // The heads in chunks of the call's instance order (the FP32 pass downloads its first
    // instances first): each chunk's head and level plans, and the event after them.
    struct Chunk {
        std::vector<Tcl4Plan*> plans;
        cudaEvent_t ready = nullptr;
    };
    std::vector<Chunk> chunks;
    std::vector<uint32_t> chunk_of;  // per head
    cudaStream_t s = nullptr;
    cudaEvent_t start = nullptr;
    bool launched = false;
    bool empty() const { return chunks.empty(); }
    cudaEvent_t ready() const { return chunks.back().ready; }
    void drop() {
        for (auto& c : chunks) {
            for (Tcl4Plan* p : c.plans) plan_destroy(p);
            if (c.ready) cudaEventDestroy(c.ready);
        }
        chunks.clear();
        launched = false;
        key = 0;
    }
    HeadPlans() = default;
    HeadPlans(const HeadPlans&) = delete;
    HeadPlans& operator=(const HeadPlans&) = delete;
    ~HeadPlans() {
        drop();
        if (start) cudaEventDestroy(start);
        if (s) cudaStreamDestroy(s);
    }
};
// Instance-index bounds of the head chunks: the first 16 instances (the pass's short first
// sub-batch), the next 48, the rest.
constexpr std::size_t kChunkBounds[] = {16, 64};
std::map<int, std::unique_ptr<HeadPlans>>& head_plans_map() {
    thread_local std::map<int, std::unique_ptr<HeadPlans>> m;
    return m;
}
HeadPlans& head_plans() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    auto& p = head_plans_map()[dev];
    if (!p) p = std::make_unique<HeadPlans>();
    return *p;
}

uint64_t system_hash(uint64_t h, const SystemDesc& s) {
    const int head[3] = {s.N, s.nf, s.num_ops};
    h = fnv1a(h, head, sizeof(head));
    h = fnv1a(h, s.omegas.data(), s.omegas.size() * sizeof(double));
    h = fnv1a(h, s.mirror.data(), s.mirror.size() * sizeof(int));
    h = fnv1a(h, s.p2f.data(), s.p2f.size() * sizeof(int));
    return fnv1a(h, s.ops.data(), s.ops.size() * sizeof(double2));
}

// Identity of a call's heads: options, and per head its instance (position in the call,
// system, gamma buffer, sizes, dt) and its rows.
uint64_t heads_key(const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads, const BuildOptions& opt) {
    uint64_t h = 1469598103934665603ull;
    const uint64_t o[3] = {opt.causal_truncation ? 1u : 0u, opt.pad_factor, heads.size()};
    h = fnv1a(h, o, sizeof(o));
    for (const Head& hd : heads) {
        const Tcl4Instance& in = insts[hd.inst];
        const uint64_t v[8] = {hd.inst, static_cast<uint64_t>(reinterpret_cast<std::uintptr_t>(in.gamma)),
                               in.gamma_on_device ? 1u : 0u, in.Nt, hd.H, hd.tc, hd.rows_hash, in.tidx.size()};
        h = fnv1a(h, v, sizeof(v));
        h = fnv1a(h, &in.dt, sizeof(double));
        h = system_hash(h, in.sys);
    }
    return h;
}

// Prepares the plans of `heads` (their rows, positions and gamma copies) in `hp`.
void build_head_plans(HeadPlans& hp, const std::vector<Tcl4Instance>& insts, const std::vector<Head>& heads,
                      const BuildOptions& o64) {
    hp.drop();
    const std::size_t nh = heads.size();
    hp.off.assign(nh, 0);
    hp.pos_off.assign(nh, 0);
    std::size_t rows = 0, npos = 0;
    for (std::size_t k = 0; k < nh; ++k) {
        hp.off[k] = rows;
        rows += heads[k].times.size() * entries(insts[heads[k].inst]);
        hp.pos_off[k] = npos;
        npos += heads[k].pos.size();
    }
    hp.rows.ensure(std::max<std::size_t>(rows, 1) * sizeof(double2));
    hp.pos.ensure(std::max<std::size_t>(npos, 1) * sizeof(uint32_t));
    {
        std::vector<uint32_t> pos_h(std::max<std::size_t>(npos, 1));
        for (std::size_t k = 0; k < nh; ++k) std::copy(heads[k].pos.begin(), heads[k].pos.end(), pos_h.begin() + hp.pos_off[k]);
        cuda_check(cudaMemcpy(hp.pos.p, pos_h.data(), npos * sizeof(uint32_t), cudaMemcpyHostToDevice),
                   "cudaMemcpy(guard positions)");
    }
    // host gamma: the samples each head consumes (the causal rule reads up to its last time)
    hp.uploads.clear();
    hp.gam_elems = 0;
    std::vector<std::size_t> g_at(nh, 0), g_n(nh, 0);
    for (std::size_t k = 0; k < nh; ++k) {
        const Tcl4Instance& in = insts[heads[k].inst];
        if (in.gamma_on_device) continue;
        const std::size_t n =
            o64.causal_truncation ? static_cast<std::size_t>(*std::max_element(heads[k].times.begin(), heads[k].times.end())) + 1
                                  : in.Nt;
        g_at[k] = hp.gam_elems;
        g_n[k] = n;
        hp.uploads.push_back({in.gamma, static_cast<std::size_t>(in.sys.nf), in.Nt, n, hp.gam_elems, 0});
        hp.gam_elems += static_cast<std::size_t>(in.sys.nf) * n;
    }
    hp.gam.ensure(std::max<std::size_t>(hp.gam_elems, 1) * sizeof(double2));
    // the plans' instances; heads of one time list and length share one list of times
    std::map<std::tuple<const void*, uint32_t, uint32_t>, TimeList> lists;
    auto list_of = [&](const Head& h, uint32_t n) -> const TimeList& {
        const auto key = std::make_tuple(insts[h.inst].tidx.identity(), h.H, n);
        auto it = lists.find(key);
        if (it == lists.end()) {
            TimeList t;
            t.assign(h.times.data(), h.times.data() + n);
            it = lists.emplace(key, std::move(t)).first;
        }
        return it->second;
    };
    double2* rows_p = static_cast<double2*>(hp.rows.p);
    std::vector<Tcl4Instance> hi(nh);
    for (std::size_t k = 0; k < nh; ++k) {
        const Head& h = heads[k];
        const Tcl4Instance& in = insts[h.inst];
        Tcl4Instance& x = hi[k];
        x.sys = in.sys;
        x.gamma = in.gamma_on_device ? in.gamma : static_cast<const double2*>(hp.gam.p) + g_at[k];
        x.Nt = in.gamma_on_device ? in.Nt : g_n[k];
        x.gamma_on_device = true;
        x.dt = in.dt;
        x.tidx.share_with(list_of(h, static_cast<uint32_t>(h.times.size())));
        x.out = rows_p + hp.off[k];
        x.out_on_device = true;
        x.internal = true;
    }
    // chunks: per chunk the heads, then each level (instance lists; empty ones dropped)
    hp.chunk_of.assign(nh, 0);
    std::vector<std::vector<std::vector<Tcl4Instance>>> lists_of;
    for (std::size_t k = 0; k < nh; ++k) {
        uint32_t c = 0;
        while (c < 2 && heads[k].inst >= kChunkBounds[c]) ++c;
        hp.chunk_of[k] = c;
    }
    // the levels that change their heads' rows (measured once, for the kept set of heads)
    const std::vector<std::vector<char>> keep = needed_levels(insts, heads, 0, nh, o64, g_guard_tol.load(), nullptr);
    for (uint32_t c = 0; c < 3; ++c) {
        std::vector<std::vector<Tcl4Instance>> parts(1);
        for (std::size_t k = 0; k < nh; ++k)
            if (hp.chunk_of[k] == c) parts[0].push_back(hi[k]);
        if (parts[0].empty()) continue;
        for (std::size_t q = 0; q < std::size(kLevels); ++q) {
            std::vector<Tcl4Instance> li;
            for (std::size_t k = 0; k < nh; ++k) {
                const Head& h = heads[k];
                if (hp.chunk_of[k] != c || !keep[q][k]) continue;
                const std::size_t n = level_rows(h, kLevels[q]);
                if (n == 0) continue;
                Tcl4Instance l = hi[k];
                l.tidx.share_with(list_of(h, static_cast<uint32_t>(n)));
                li.push_back(std::move(l));
            }
            if (!li.empty()) parts.push_back(std::move(li));
        }
        lists_of.push_back(std::move(parts));
    }
    // chunks renumbered without the empty ones
    {
        std::vector<uint32_t> used;
        for (uint32_t c : hp.chunk_of)
            if (std::find(used.begin(), used.end(), c) == used.end()) used.push_back(c);
        std::sort(used.begin(), used.end());
        for (uint32_t& c : hp.chunk_of) c = static_cast<uint32_t>(std::find(used.begin(), used.end(), c) - used.begin());
        std::size_t u = 0;
        for (std::size_t k = 0; k < nh; ++k)
            if (!insts[heads[k].inst].gamma_on_device) hp.uploads[u++].chunk = hp.chunk_of[k];
    }
    const std::size_t budget = work_budget_now();
    std::size_t need = 256;
    for (auto& parts : lists_of)
        for (auto& li : parts) need = std::max(need, plan_work_bytes(li, o64, budget));
    hp.work.ensure(need + need / 8 + (std::size_t(1) << 20));
    for (auto& parts : lists_of) {
        hp.chunks.emplace_back();
        HeadPlans::Chunk& ch = hp.chunks.back();
        cuda_check(cudaEventCreateWithFlags(&ch.ready, cudaEventDisableTiming), "cudaEventCreate");
        for (auto& li : parts) ch.plans.push_back(plan_create_direct(li, o64, hp.work.p, hp.work.cap, budget));
    }
}

// Replays the head plans on their stream after the work queued on `st`; `ready` marks the end.
void launch_head_plans(HeadPlans& hp, cudaStream_t st) {
    if (!hp.s) {
        // high priority: the heads gate the downloads of the pass's groups, which are the
        // slowest part of a call with host outputs
        int lo = 0, hi = 0;
        cuda_check(cudaDeviceGetStreamPriorityRange(&lo, &hi), "cudaDeviceGetStreamPriorityRange");
        cuda_check(cudaStreamCreateWithPriority(&hp.s, cudaStreamNonBlocking, hi), "cudaStreamCreate(guard heads)");
    }
    if (!hp.start) cuda_check(cudaEventCreateWithFlags(&hp.start, cudaEventDisableTiming), "cudaEventCreate");
    if (hp.launched) cuda_check(cudaEventSynchronize(hp.ready()), "cudaEventSynchronize(guard heads)");
    cuda_check(cudaEventRecord(hp.start, st), "cudaEventRecord");
    cuda_check(cudaStreamWaitEvent(hp.s, hp.start, 0), "cudaStreamWaitEvent");
    for (uint32_t c = 0; c < hp.chunks.size(); ++c) {
        for (const auto& u : hp.uploads)
            if (u.chunk == c)
                cuda_check(cudaMemcpy2DAsync(static_cast<double2*>(hp.gam.p) + u.dst, u.n * sizeof(double2), u.src,
                                             u.stride * sizeof(double2), u.n * sizeof(double2), u.nf,
                                             cudaMemcpyHostToDevice, hp.s),
                           "cudaMemcpy2DAsync(guard gamma)");
        for (Tcl4Plan* p : hp.chunks[c].plans) plan_execute(p, hp.s);
        cuda_check(cudaEventRecord(hp.chunks[c].ready, hp.s), "cudaEventRecord");
    }
    hp.launched = true;
}

}  // namespace

void set_fp32_guard(double tol) { g_guard_tol.store(tol > 0.0 ? tol : 0.0); }
void set_guard_chunk_bytes(std::size_t bytes) { g_head_chunk_bytes.store(bytes ? bytes : std::size_t(1) << 30); }
void release_guard_scratch() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    guard_scratch_map().erase(dev);
    head_plans_map().erase(dev);
}
GuardStats fp32_guard_stats() { return t_stats; }
double fp32_guard() { return g_guard_tol.load(); }

void tcl4_build(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, cudaStream_t stream) {
    t_stats = GuardStats{};
    if (!opt.fp32 || g_guard_tol.load() <= 0.0) {
        tcl4_build_direct(insts, opt, stream);
        return;
    }
    cudaStream_t st = stream ? stream : default_stream();
    const auto t00 = std::chrono::steady_clock::now();
    // the FP32 pass on a copy: a direct build may point an instance at device copies of its
    // host input and output that it frees before returning; the guard needs the caller's
    std::vector<Tcl4Instance> pass(insts);
    TimeCache tcache;
    std::vector<uint32_t> tcs(insts.size(), 0);
    for (std::size_t a = 0; a < insts.size(); ++a) tcs[a] = tcache.t_count(insts[a]);
    const std::vector<uint64_t> fps = fingerprints(insts, tcs, st);
    const auto t01 = std::chrono::steady_clock::now();
    // every instance decided before on the same gamma contents: replay the FP64 heads it
    // requires (prepared plans) beside the FP32 pass, whose groups patch them on the device
    std::vector<Head> heads;
    bool trusted = true;
    for (std::size_t a = 0; a < insts.size() && trusted; ++a) {
        if (insts[a].tidx.empty()) continue;
        auto it = t_head_memory.find({insts[a].gamma, tcs[a]});
        if (it == t_head_memory.end() || it->second.fingerprint != fps[a] || it->second.accepted == 0) {
            trusted = false;
            break;
        }
        if (it->second.required == 0) continue;  // FP32 suffices everywhere
        Head h = tcache.head(insts, a, it->second.required, tcs[a]);
        if (!h.times.empty()) heads.push_back(std::move(h));
    }
    {
        // the prepared heads keep all their rows at once: within one chunk of head rows,
        // else the call is checked as usual (in chunks)
        std::size_t bytes = 0;
        for (const Head& h : heads) bytes += h.times.size() * entries(insts[h.inst]) * sizeof(double2);
        trusted = trusted && bytes <= g_head_chunk_bytes.load();
    }
    const auto t0 = std::chrono::steady_clock::now();
    auto t_key = t0;
    HeadPlans* hp = nullptr;
    bool rebuilt = false;
    if (trusted && !heads.empty()) {
        hp = &head_plans();
        const uint64_t key = heads_key(insts, heads, opt);
        t_key = std::chrono::steady_clock::now();
        if (key != hp->key || hp->empty()) {
            const BuildOptions o64 = head_options(opt);
            try {
                build_head_plans(*hp, insts, heads, o64);
                hp->key = key;
                rebuilt = true;
            } catch (const Error&) {
                // no room for the prepared heads (or no plan for them): check this call as usual
                hp->drop();
                trusted = false;
            }
        }
    }
    if (trusted) {
        const std::size_t nh = heads.size();
        if (nh) launch_head_plans(*hp, st);
        const auto t1 = std::chrono::steady_clock::now();
        // Each group of the FP32 pass patches the heads of its whole instances on the device,
        // after its contraction and the head plans, before its download (host outputs download
        // once, already patched).  One pinned job slot per head.
        GuardScratch& gs = guard_scratch();
        std::vector<int> head_of(insts.size(), -1);
        for (std::size_t k = 0; k < nh; ++k) head_of[heads[k].inst] = static_cast<int>(k);
        std::vector<char> patched(nh, 0);
        std::size_t used = 0;
        if (nh) {
            gs.jobs_host.ensure(nh * sizeof(GuardJob));
            gs.jobs.ensure(nh * sizeof(GuardJob));
        }
        const Tcl4Instance* pass0 = pass.data();
        BuildOptions po = opt;
        if (nh)
            po.out_hook = [&](const std::vector<std::pair<const Tcl4Instance*, void*>>& rows, cudaStream_t s) {
                GuardJob* jh = static_cast<GuardJob*>(gs.jobs_host.p) + used;
                std::size_t n = 0, most = 1;
                uint32_t last_chunk = 0;
                for (const auto& r : rows) {
                    const std::size_t a = static_cast<std::size_t>(r.first - pass0);
                    if (a >= head_of.size() || head_of[a] < 0 || patched[head_of[a]]) continue;
                    const std::size_t k = static_cast<std::size_t>(head_of[a]);
                    const Head& h = heads[k];
                    GuardJob j{};
                    j.h64 = static_cast<const double2*>(hp->rows.p) + hp->off[k];
                    j.out32 = static_cast<float2*>(r.second);
                    j.pos = static_cast<const uint32_t*>(hp->pos.p) + hp->pos_off[k];
                    j.n = static_cast<uint32_t>(h.pos.size());
                    j.E = static_cast<uint32_t>(entries(insts[a]));
                    jh[n++] = j;
                    patched[k] = 1;
                    last_chunk = std::max(last_chunk, hp->chunk_of[k]);
                    most = std::max(most, h.pos.size() * entries(insts[a]));
                }
                if (!n) return;
                GuardJob* jd = static_cast<GuardJob*>(gs.jobs.p) + used;
                used += n;
                // the chunks run in order: the last one these heads belong to covers them all
                cuda_check(cudaStreamWaitEvent(s, hp->chunks[last_chunk].ready, 0), "cudaStreamWaitEvent(guard heads)");
                cuda_check(cudaMemcpyAsync(jd, jh, n * sizeof(GuardJob), cudaMemcpyHostToDevice, s),
                           "cudaMemcpyAsync(guard jobs)");
                const unsigned bx = static_cast<unsigned>(std::min<std::size_t>((most + 255) / 256, 592));
                k_guard_patch<<<dim3(bx, static_cast<unsigned>(n)), 256, 0, s>>>(jd);
                cuda_check(cudaGetLastError(), "k_guard_patch");
                count_launches(1);
            };
        tcl4_build_direct(pass, po, stream);
        const auto t2 = std::chrono::steady_clock::now();
        t_stats = GuardStats{};
        t_stats.instances = insts.size();
        // heads of instances the pass built in slices: patched after it, as a separate step
        PreHeads rest;
        if (hp) rest.temp = &hp->rows;
        for (std::size_t k = 0; k < nh; ++k) {
            const Head& h = heads[k];
            if (!patched[k]) {
                rest.heads.push_back(h);
                rest.off.push_back(hp->off[k]);
                continue;
            }
            ++t_stats.heads;
            t_stats.head_rows += h.times.size();
            t_stats.rows += insts[h.inst].tidx.size();
            if (h.H >= h.tc) ++t_stats.full;
        }
        if (!rest.heads.empty()) {
            cuda_check(cudaEventSynchronize(hp->ready()), "cudaEventSynchronize(guard heads)");
            const GuardStats before = t_stats;
            run_guard(insts, opt, st, true, &rest, true, &fps);
            t_stats.heads += before.heads;
            t_stats.head_rows += before.head_rows;
            t_stats.rows += before.rows;
            t_stats.full += before.full;
        }
        t_stats.rounds = 1;
        if (host_trace_on())
            std::fprintf(stderr,
                         "taco guard (ms, heads from memory): setup %.3f (fingerprints %.3f), key %.3f, head plans %s "
                         "%.3f, fp32 pass with patches %.3f, rest %.3f (%zu of %zu heads patched in the pass)\n",
                         std::chrono::duration<double, std::milli>(t0 - t00).count(),
                         std::chrono::duration<double, std::milli>(t01 - t00).count(),
                         std::chrono::duration<double, std::milli>(t_key - t0).count(), rebuilt ? "built+launched" : "launched",
                         std::chrono::duration<double, std::milli>(t1 - t_key).count(),
                         std::chrono::duration<double, std::milli>(t2 - t1).count(),
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t2).count(),
                         nh - rest.heads.size(), nh);
        return;
    }
    const auto t3 = std::chrono::steady_clock::now();
    tcl4_build_direct(pass, opt, stream);
    const auto t4 = std::chrono::steady_clock::now();
    run_guard(insts, opt, st, true, nullptr, false, &fps);
    if (host_trace_on())
        std::fprintf(stderr, "taco guard (ms): setup %.3f, fp32 pass %.3f, guard rounds %.3f\n",
                     std::chrono::duration<double, std::milli>(t3 - t00).count(),
                     std::chrono::duration<double, std::milli>(t4 - t3).count(),
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t4).count());
}

Tcl4Plan* plan_create(std::vector<Tcl4Instance>& insts, const BuildOptions& opt) {
    Tcl4Plan* plan = plan_create_direct(insts, opt);
    t_stats = GuardStats{};
    if (!opt.fp32 || g_guard_tol.load() <= 0.0) return plan;
    try {
        // the FP32 results of the plan's inputs (written by the caller's streams: wait for the
        // device first), then the guard loop on them
        cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize(plan guard)");
        cudaStream_t st = default_stream();
        plan_execute(plan, st);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(plan guard)");
        Decision dec = run_guard(insts, opt, st, false);
        // the guard's direct builds grew this thread's transient buffers; the plans below
        // size theirs from the free memory
        release_workspace();
        release_guard_scratch();
        if (dec.heads.empty()) return plan;
        // the heads as FP64 plans over one shared buffer of head rows, each followed by its patch
        const BuildOptions o64 = head_options(opt);
        struct Part {
            Tcl4Plan* plan = nullptr;
            std::vector<Tcl4Plan*> levels;  // short-FFT levels, replayed after the head
            std::size_t jobs = 0;
            unsigned blocks = 0;
            std::size_t meta_off = 0;
        };
        struct TailState {
            DevMem rows, meta, work;
            std::vector<Part> parts;
            cudaStream_t side = nullptr;  // the heads run here, beside the FP32 graph
            cudaEvent_t start = nullptr, done = nullptr;
            ~TailState() {
                for (auto& p : parts) {
                    plan_destroy(p.plan);
                    for (Tcl4Plan* l : p.levels) plan_destroy(l);
                }
                if (start) cudaEventDestroy(start);
                if (done) cudaEventDestroy(done);
                if (side) cudaStreamDestroy(side);
            }
        };
        auto tail = std::make_shared<TailState>();
        cuda_check(cudaStreamCreateWithFlags(&tail->side, cudaStreamNonBlocking), "cudaStreamCreate(guard heads)");
        cuda_check(cudaEventCreateWithFlags(&tail->start, cudaEventDisableTiming), "cudaEventCreate");
        cuda_check(cudaEventCreateWithFlags(&tail->done, cudaEventDisableTiming), "cudaEventCreate");
        std::size_t most = 256, meta_total = 0;
        std::vector<JobImage> imgs;
        std::vector<std::pair<std::size_t, std::size_t>> ranges;
        for_chunks(insts, dec.heads, [&](std::size_t k0, std::size_t k1, std::size_t bytes) {
            most = std::max(most, bytes);
            ranges.emplace_back(k0, k1);
        });
        tail->rows.ensure(most);
        double2* base = static_cast<double2*>(tail->rows.p);
        // job images: measured first, then placed in one metadata buffer
        std::vector<std::vector<std::size_t>> offs(ranges.size());
        std::vector<std::vector<Tcl4Instance>> his(ranges.size());
        for (std::size_t c = 0; c < ranges.size(); ++c) {
            his[c] = head_instances(insts, dec.heads, ranges[c].first, ranges[c].second, base, offs[c]);
            JobImage im = job_image(insts, dec.heads, ranges[c].first, ranges[c].second, base, offs[c], nullptr);
            meta_total += (im.host.size() + 255) / 256 * 256;
        }
        tail->meta.ensure(meta_total + 256);
        // one transient buffer for every head plan (they run one after another)
        std::vector<std::vector<std::vector<Tcl4Instance>>> lis(ranges.size());
        for (std::size_t c = 0; c < ranges.size(); ++c) {
            const std::vector<std::vector<char>> keep =
                needed_levels(insts, dec.heads, ranges[c].first, ranges[c].second, o64, g_guard_tol.load(), st);
            for (std::size_t q = 0; q < std::size(kLevels); ++q)
                lis[c].push_back(level_instances(insts, dec.heads, ranges[c].first, ranges[c].second, base, offs[c],
                                                 kLevels[q], &keep[q]));
        }
        // measured under the current budget; the plans group by that same budget, and the
        // buffer has slack for the rounding of the slice sizes
        const std::size_t budget = work_budget_now();
        std::size_t work_need = 256;
        for (std::size_t c = 0; c < ranges.size(); ++c) {
            work_need = std::max(work_need, plan_work_bytes(his[c], o64, budget));
            for (auto& li : lis[c])
                if (!li.empty()) work_need = std::max(work_need, plan_work_bytes(li, o64, budget));
        }
        tail->work.ensure(work_need + work_need / 8 + (std::size_t(1) << 20));
        uint64_t kernels = 0;
        std::size_t moff = 0;
        for (std::size_t c = 0; c < ranges.size(); ++c) {
            unsigned char* dev = static_cast<unsigned char*>(tail->meta.p) + moff;
            JobImage im = job_image(insts, dec.heads, ranges[c].first, ranges[c].second, base, offs[c], dev);
            cuda_check(cudaMemcpy(dev, im.host.data(), im.host.size(), cudaMemcpyHostToDevice), "cudaMemcpy(guard jobs)");
            Part p;
            p.plan = plan_create_direct(his[c], o64, tail->work.p, tail->work.cap, budget);
            for (auto& li : lis[c])
                if (!li.empty()) {
                    p.levels.push_back(plan_create_direct(li, o64, tail->work.p, tail->work.cap, budget));
                    kernels += plan_kernels(p.levels.back());
                }
            p.jobs = ranges[c].second - ranges[c].first;
            p.blocks = patch_blocks(insts, dec.heads, ranges[c].first, ranges[c].second);
            p.meta_off = moff;
            tail->parts.push_back(p);
            kernels += plan_kernels(p.plan) + 1;
            moff += (im.host.size() + 255) / 256 * 256;
        }
        if (host_trace_on()) {
            std::map<uint32_t, std::size_t> hist;
            for (const Head& h : dec.heads) ++hist[h.H];
            std::string line = "taco guard plan: heads by length (H: count)";
            for (const auto& e : hist) line += " " + std::to_string(e.first) + ":" + std::to_string(e.second);
            std::size_t nl[2] = {0, 0};
            for (std::size_t c = 0; c < ranges.size(); ++c)
                for (std::size_t q = 0; q < lis[c].size() && q < 2; ++q) nl[q] += lis[c][q].size();
            std::fprintf(stderr, "%s; levels %zu (<%u) %zu (<%u); tail kernels %llu\n", line.c_str(), nl[0], kLevels[0], nl[1],
                         kLevels[1], static_cast<unsigned long long>(kernels));
        }
        // One chunk of heads: the FP64 heads (and their levels, in order) on the side stream,
        // after the work queued before the execute and beside the FP32 graph, the patch after
        // both.  Several chunks share one buffer of head rows: each chunk's heads, levels and
        // patch in turn after the graph.
        if (tail->parts.size() > 1) {
            plan_set_tail(
                plan, nullptr,
                [tail](cudaStream_t s) {
                    for (const Part& p : tail->parts) {
                        plan_execute(p.plan, s);
                        for (Tcl4Plan* l : p.levels) plan_execute(l, s);
                        const GuardJob* jobs =
                            reinterpret_cast<const GuardJob*>(static_cast<unsigned char*>(tail->meta.p) + p.meta_off);
                        k_guard_patch<<<dim3(p.blocks, static_cast<unsigned>(p.jobs)), 256, 0, s>>>(jobs);
                        cuda_check(cudaGetLastError(), "k_guard_patch");
                        count_launches(1);
                    }
                },
                kernels);
            return plan;
        }
        plan_set_tail(
            plan,
            [tail](cudaStream_t s) {
                cuda_check(cudaEventRecord(tail->start, s), "cudaEventRecord");
                cuda_check(cudaStreamWaitEvent(tail->side, tail->start, 0), "cudaStreamWaitEvent");
                for (const Part& p : tail->parts) {
                    plan_execute(p.plan, tail->side);
                    for (Tcl4Plan* l : p.levels) plan_execute(l, tail->side);
                }
                cuda_check(cudaEventRecord(tail->done, tail->side), "cudaEventRecord");
            },
            [tail](cudaStream_t s) {
                cuda_check(cudaStreamWaitEvent(s, tail->done, 0), "cudaStreamWaitEvent");
                for (const Part& p : tail->parts) {
                    const GuardJob* jobs =
                        reinterpret_cast<const GuardJob*>(static_cast<unsigned char*>(tail->meta.p) + p.meta_off);
                    k_guard_patch<<<dim3(p.blocks, static_cast<unsigned>(p.jobs)), 256, 0, s>>>(jobs);
                    cuda_check(cudaGetLastError(), "k_guard_patch");
                    count_launches(1);
                }
            },
            kernels);
        return plan;
    } catch (...) {
        plan_destroy(plan);
        throw;
    }
}

}  // namespace taco
