// gw_coef.cpp -- builds the merged linear map from F/C/R values to L4 entries.
#include "gw_coef.hpp"

#include <algorithm>
#include <array>
#include <complex>
#include <thread>
#include <unordered_map>

namespace taco {

namespace {

using cd = std::complex<double>;

// One factor of a term: entry (r, c) of coupling operator `op`.
struct Factor {
    int op, r, c;
};

// Walks the terms of the NAKZWAN sums (tcl4_assemble.cpp:108-185) for one entry of T and
// hands each (source, conjugation, sign, four operator factors) to `emit`.  MIKX
// (tcl4_mikx.cpp:87-177) turns every gathered tensor entry into one or two sources:
//   M(row=(j,k), col=(p,q)) = F[f(j,q), f(j,k), f(p,j)] - R[f(j,q), f(p,q), f(q,k)]
//   I(row=(j,k), col=(p,q)) = F[f(j,k), f(q,p), f(k,q)]
//   K(row=(j,k), col=(p,q)) = R[f(j,k), f(p,q), f(q,j)]
//   X(j,k,p,q,r,s)          = C[f(j,k), f(p,q), f(r,s)] + R[same]
struct TermWalker {
    int N, nf, num_ops;
    const int* p2f;
    std::size_t nf3;

    int f(int a, int b) const { return p2f[a + N * b]; }
    uint32_t tri(int a, int b, int c) const {
        return static_cast<uint32_t>((static_cast<std::size_t>(a) * nf + b) * nf + c);
    }
    uint32_t srcF(int a, int b, int c) const { return tri(a, b, c); }
    uint32_t srcC(int a, int b, int c) const { return static_cast<uint32_t>(nf3) + tri(a, b, c); }
    uint32_t srcR(int a, int b, int c) const { return static_cast<uint32_t>(2 * nf3) + tri(a, b, c); }

    template <class Emit>
    void walk(int n, int i, int m, int j, bool cj, Emit&& emit) const {
        using F4 = std::array<Factor, 4>;
        auto M = [&](int jj, int k, int p, int q, double sg, const F4& fs) {
            emit(srcF(f(jj, q), f(jj, k), f(p, jj)), cj, sg, fs);
            emit(srcR(f(jj, q), f(p, q), f(q, k)), cj, -sg, fs);
        };
        auto I = [&](int jj, int k, int p, int q, double sg, const F4& fs) {
            emit(srcF(f(jj, k), f(q, p), f(k, q)), cj, sg, fs);
        };
        auto K = [&](int jj, int k, int p, int q, double sg, const F4& fs) {
            emit(srcR(f(jj, k), f(p, q), f(q, jj)), cj, sg, fs);
        };
        auto X = [&](int jj, int k, int p, int q, int r, int s, double sg, const F4& fs) {
            emit(srcC(f(jj, k), f(p, q), f(r, s)), cj, sg, fs);
            emit(srcR(f(jj, k), f(p, q), f(r, s)), cj, sg, fs);
        };
        for (int iA = 0; iA < num_ops; ++iA)
            for (int iB = 0; iB < num_ops; ++iB) {
                auto A = [&](int r, int c) { return Factor{iA, r, c}; };
                auto B = [&](int r, int c) { return Factor{iB, r, c}; };
                for (int a = 0; a < N; ++a)
                    for (int b = 0; b < N; ++b) {
                        // res -= (t1 - t2 + t3 + t4 - t5 - t6 + t7)
                        M(b, i, n, a, -1.0, F4{B(n, a), A(a, b), B(b, i), A(j, m)});
                        I(a, n, i, b, +1.0, F4{A(n, a), B(a, b), B(b, i), A(j, m)});
                        K(i, b, n, a, -1.0, F4{B(n, a), B(a, b), A(b, i), A(j, m)});
                        X(a, n, j, b, n, i, -1.0, F4{A(n, a), B(a, i), B(j, b), A(b, m)});
                        X(i, a, j, b, n, i, +1.0, F4{B(n, a), A(a, i), B(j, b), A(b, m)});
                        X(b, a, j, m, a, i, +1.0, F4{A(n, a), A(a, b), B(b, i), B(j, m)});
                        X(i, b, j, m, a, i, -1.0, F4{A(n, a), B(a, b), A(b, i), B(j, m)});
                    }
                if (j == m) {
                    for (int a = 0; a < N; ++a)
                        for (int b = 0; b < N; ++b)
                            for (int c = 0; c < N; ++c) {
                                M(c, i, a, b, +1.0, F4{A(n, a), B(a, b), A(b, c), B(c, i)});
                                K(i, c, a, b, +1.0, F4{A(n, a), B(a, b), B(b, c), A(c, i)});
                                I(b, a, i, c, -1.0, F4{A(n, a), A(a, b), B(b, c), B(c, i)});
                            }
                }
            }
    }

    // Entry e of L4 (column-major, e = row + N^2 col):
    // L4(n + N m, i + N j) = GW(n + N i, m + N j) = T(n,i,m,j) + conj(T(m,j,n,i)).
    template <class Emit>
    void walk_entry(std::size_t e, Emit&& emit) const {
        const std::size_t N2 = static_cast<std::size_t>(N) * N;
        const int rowL = static_cast<int>(e % N2), colL = static_cast<int>(e / N2);
        const int n = rowL % N, m = rowL / N, i = colL % N, j = colL / N;
        walk(n, i, m, j, false, emit);
        walk(m, j, n, i, true, emit);
    }
};

}  // namespace

thread_local int g_coef_threads = 0;

void set_coef_table_threads(int n) { g_coef_threads = n; }

// Entries are independent: each is merged on its own (terms added in walk order, sources in
// ascending key order), on up to 16 host threads for large maps.  Per thread, a dense
// accumulator over (source, conjugation) with a list of the keys an entry touched replaces
// a hash map; the result is the same table.
void build_coef_table(int N, int nf, const int* p2f, const double2* ops, int num_ops, CoefTable& out, bool structural) {
    const TermWalker tw{N, nf, num_ops, p2f, static_cast<std::size_t>(nf) * nf * nf};
    const cd* op = reinterpret_cast<const cd*>(ops);
    const std::size_t N2 = static_cast<std::size_t>(N) * N;
    const std::size_t E = N2 * N2;
    const std::size_t S = 3 * tw.nf3;
    auto val = [&](const Factor& x) { return op[static_cast<std::size_t>(x.op) * N2 + x.r + N * x.c]; };
    std::vector<std::vector<uint32_t>> row_src(E);
    std::vector<std::vector<cd>> row_coef(E);
    const bool dense = 2 * S <= (std::size_t(1) << 26);
    const std::size_t per_thread = dense ? 2 * S * (sizeof(cd) + 1) : 0;
    unsigned nthreads = g_coef_threads > 0 ? static_cast<unsigned>(g_coef_threads)
                                           : std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (E < 256) nthreads = 1;
    if (per_thread) nthreads = std::max<unsigned>(1, std::min<std::size_t>(nthreads, (std::size_t(512) << 20) / per_thread));
    auto work = [&](std::size_t e0, std::size_t step) {
        std::vector<cd> dacc(dense ? 2 * S : 0);
        std::vector<uint8_t> seen(dense ? 2 * S : 0, 0);
        std::vector<uint32_t> keys;
        std::unordered_map<uint32_t, cd> macc;  // very large maps
        for (std::size_t e = e0; e < E; e += step) {
            keys.clear();
            macc.clear();
            tw.walk_entry(e, [&](uint32_t s, bool cj, double sg, const std::array<Factor, 4>& fs) {
                const cd w = sg * (val(fs[0]) * val(fs[1]) * val(fs[2]) * val(fs[3]));
                if (w == cd(0.0, 0.0) && !structural) return;
                const uint32_t key = s | (cj ? 0x80000000u : 0u);
                const cd add = cj ? std::conj(w) : w;
                if (dense) {
                    const std::size_t idx = 2 * static_cast<std::size_t>(s) + (cj ? 1 : 0);
                    if (!seen[idx]) {
                        seen[idx] = 1;
                        dacc[idx] = cd(0.0, 0.0);
                        keys.push_back(key);
                    }
                    dacc[idx] += add;
                } else {
                    auto it = macc.find(key);
                    if (it == macc.end()) {
                        macc.emplace(key, cd(0.0, 0.0) + add);
                        keys.push_back(key);
                    } else {
                        it->second += add;
                    }
                }
            });
            std::sort(keys.begin(), keys.end());
            for (uint32_t key : keys) {
                const uint32_t s = key & 0x7fffffffu;
                cd v;
                if (dense) {
                    const std::size_t idx = 2 * static_cast<std::size_t>(s) + (key >> 31);
                    v = dacc[idx];
                    seen[idx] = 0;
                } else {
                    v = macc[key];
                }
                if (v == cd(0.0, 0.0) && !structural) continue;
                row_src[e].push_back(key);
                row_coef[e].push_back(v);
            }
        }
    };
    if (nthreads <= 1) {
        work(0, 1);
    } else {
        std::vector<std::thread> pool;
        for (unsigned k = 0; k < nthreads; ++k) pool.emplace_back(work, k, nthreads);
        for (auto& th : pool) th.join();
    }
    out.N = N;
    out.nf = nf;
    out.rowptr.assign(E + 1, 0);
    std::size_t total = 0;
    for (std::size_t e = 0; e < E; ++e) {
        total += row_src[e].size();
        out.rowptr[e + 1] = static_cast<int32_t>(total);
    }
    out.src.resize(total);
    out.coef.resize(total);
    out.triple_fc_used.assign(tw.nf3, 0);
    out.triple_r_used.assign(tw.nf3, 0);
    for (std::size_t e = 0, k = 0; e < E; ++e) {
        for (std::size_t q = 0; q < row_src[e].size(); ++q, ++k) {
            const uint32_t key = row_src[e][q];
            out.src[k] = key;
            out.coef[k] = make_double2(row_coef[e][q].real(), row_coef[e][q].imag());
            const uint32_t s = key & 0x7fffffffu;
            const std::size_t kind = s / tw.nf3, t = s % tw.nf3;
            if (kind < 2) out.triple_fc_used[t] = 1;
            else out.triple_r_used[t] = 1;
        }
        std::vector<uint32_t>().swap(row_src[e]);
        std::vector<cd>().swap(row_coef[e]);
    }
}

void coef_table_ops_grad(int N, int nf, const int* p2f, const double2* ops, int num_ops, const CoefTable& table,
                         const double2* Z, double2* ops_bar) {
    const TermWalker tw{N, nf, num_ops, p2f, static_cast<std::size_t>(nf) * nf * nf};
    const cd* op = reinterpret_cast<const cd*>(ops);
    cd* g = reinterpret_cast<cd*>(ops_bar);
    const std::size_t N2 = static_cast<std::size_t>(N) * N;
    const std::size_t E = N2 * N2;
    auto idx = [&](const Factor& x) { return static_cast<std::size_t>(x.op) * N2 + x.r + N * x.c; };
    for (std::size_t e = 0; e < E; ++e) {
        const int32_t b = table.rowptr[e], nnz = table.rowptr[e + 1] - b;
        const uint32_t* keys = table.src.data() + b;
        tw.walk_entry(e, [&](uint32_t s, bool cj, double sg, const std::array<Factor, 4>& fs) {
            const uint32_t key = s | (cj ? 0x80000000u : 0u);
            const uint32_t* it = std::lower_bound(keys, keys + nnz, key);
            if (it == keys + nnz || *it != key) throw Error(kRuntime, "coef_table_ops_grad: table is not structural");
            const cd z = reinterpret_cast<const cd*>(Z)[b + (it - keys)];
            const cd v[4] = {op[idx(fs[0])], op[idx(fs[1])], op[idx(fs[2])], op[idx(fs[3])]};
            for (int q = 0; q < 4; ++q) {
                cd d = sg;  // dP / d factor q
                for (int o = 0; o < 4; ++o)
                    if (o != q) d *= v[o];
                // holomorphic term: G += conj(z dP); conjugated copy: G += z conj(dP)
                g[idx(fs[q])] += cj ? z * std::conj(d) : std::conj(z * d);
            }
        });
    }
}

}  // namespace taco
