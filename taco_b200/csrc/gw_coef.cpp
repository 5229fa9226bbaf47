// gw_coef.cpp -- builds the merged linear map from F/C/R values to L4 entries.
#include "gw_coef.hpp"

#include <algorithm>
#include <complex>
#include <unordered_map>

namespace taco {

namespace {

using cd = std::complex<double>;

struct Builder {
    int N, nf, num_ops;
    const int* p2f;
    const cd* ops;
    std::size_t nf3;
    std::unordered_map<uint32_t, cd> acc;  // key: source | conj << 31

    int f(int a, int b) const { return p2f[a + N * b]; }
    uint32_t tri(int a, int b, int c) const {
        return static_cast<uint32_t>((static_cast<std::size_t>(a) * nf + b) * nf + c);
    }
    uint32_t srcF(int a, int b, int c) const { return tri(a, b, c); }
    uint32_t srcC(int a, int b, int c) const { return static_cast<uint32_t>(nf3) + tri(a, b, c); }
    uint32_t srcR(int a, int b, int c) const { return static_cast<uint32_t>(2 * nf3) + tri(a, b, c); }
    cd op(int k, int r, int c) const { return ops[static_cast<std::size_t>(k) * N * N + r + N * c]; }

    void add(uint32_t s, cd w, bool cj) {
        if (w == cd(0.0, 0.0)) return;
        const uint32_t key = s | (cj ? 0x80000000u : 0u);
        acc[key] += cj ? std::conj(w) : w;
    }
    // M(row=(j,k), col=(p,q)) = F[f(j,q), f(j,k), f(p,j)] - R[f(j,q), f(p,q), f(q,k)]
    void addM(int j, int k, int p, int q, cd w, bool cj) {
        add(srcF(f(j, q), f(j, k), f(p, j)), w, cj);
        add(srcR(f(j, q), f(p, q), f(q, k)), -w, cj);
    }
    // I(row=(j,k), col=(p,q)) = F[f(j,k), f(q,p), f(k,q)]
    void addI(int j, int k, int p, int q, cd w, bool cj) { add(srcF(f(j, k), f(q, p), f(k, q)), w, cj); }
    // K(row=(j,k), col=(p,q)) = R[f(j,k), f(p,q), f(q,j)]
    void addK(int j, int k, int p, int q, cd w, bool cj) { add(srcR(f(j, k), f(p, q), f(q, j)), w, cj); }
    // X(j,k,p,q,r,s) = C[f(j,k), f(p,q), f(r,s)] + R[same]
    void addX(int j, int k, int p, int q, int r, int s, cd w, bool cj) {
        add(srcC(f(j, k), f(p, q), f(r, s)), w, cj);
        add(srcR(f(j, k), f(p, q), f(r, s)), w, cj);
    }

    // Terms of T(n,i,m,j) (tcl4_assemble.cpp:108-185); cj selects the conjugated copy.
    void emitT(int n, int i, int m, int j, bool cj) {
        for (int iA = 0; iA < num_ops; ++iA)
            for (int iB = 0; iB < num_ops; ++iB) {
                auto A = [&](int r, int c) { return op(iA, r, c); };
                auto B = [&](int r, int c) { return op(iB, r, c); };
                for (int a = 0; a < N; ++a)
                    for (int b = 0; b < N; ++b) {
                        // res -= (t1 - t2 + t3 + t4 - t5 - t6 + t7)
                        addM(b, i, n, a, -(B(n, a) * A(a, b) * B(b, i) * A(j, m)), cj);
                        addI(a, n, i, b, +(A(n, a) * B(a, b) * B(b, i) * A(j, m)), cj);
                        addK(i, b, n, a, -(B(n, a) * B(a, b) * A(b, i) * A(j, m)), cj);
                        addX(a, n, j, b, n, i, -(A(n, a) * B(a, i) * B(j, b) * A(b, m)), cj);
                        addX(i, a, j, b, n, i, +(B(n, a) * A(a, i) * B(j, b) * A(b, m)), cj);
                        addX(b, a, j, m, a, i, +(A(n, a) * A(a, b) * B(b, i) * B(j, m)), cj);
                        addX(i, b, j, m, a, i, -(A(n, a) * B(a, b) * A(b, i) * B(j, m)), cj);
                    }
                if (j == m) {
                    for (int a = 0; a < N; ++a)
                        for (int b = 0; b < N; ++b)
                            for (int c = 0; c < N; ++c) {
                                addM(c, i, a, b, A(n, a) * B(a, b) * A(b, c) * B(c, i), cj);
                                addK(i, c, a, b, A(n, a) * B(a, b) * B(b, c) * A(c, i), cj);
                                addI(b, a, i, c, -(A(n, a) * A(a, b) * B(b, c) * B(c, i)), cj);
                            }
                }
            }
    }
};

}  // namespace

void build_coef_table(int N, int nf, const int* p2f, const double2* ops, int num_ops, CoefTable& out) {
    Builder bld{N, nf, num_ops, p2f, reinterpret_cast<const cd*>(ops),
                static_cast<std::size_t>(nf) * nf * nf, {}};
    const std::size_t N2 = static_cast<std::size_t>(N) * N;
    const std::size_t E = N2 * N2;
    out.N = N;
    out.nf = nf;
    out.rowptr.assign(E + 1, 0);
    out.src.clear();
    out.coef.clear();
    out.triple_fc_used.assign(bld.nf3, 0);
    out.triple_r_used.assign(bld.nf3, 0);
    std::vector<std::pair<uint32_t, cd>> row;
    for (std::size_t e = 0; e < E; ++e) {
        const int rowL = static_cast<int>(e % N2), colL = static_cast<int>(e / N2);
        const int n = rowL % N, m = rowL / N, i = colL % N, j = colL / N;
        bld.acc.clear();
        // L4(n + N m, i + N j) = GW(n + N i, m + N j) = T(n,i,m,j) + conj(T(m,j,n,i))
        bld.emitT(n, i, m, j, false);
        bld.emitT(m, j, n, i, true);
        row.assign(bld.acc.begin(), bld.acc.end());
        std::sort(row.begin(), row.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (const auto& kv : row) {
            if (kv.second == cd(0.0, 0.0)) continue;
            out.src.push_back(kv.first);
            out.coef.push_back(make_double2(kv.second.real(), kv.second.imag()));
            const uint32_t s = kv.first & 0x7fffffffu;
            const std::size_t kind = s / bld.nf3, t = s % bld.nf3;
            if (kind < 2) out.triple_fc_used[t] = 1;
            else out.triple_r_used[t] = 1;
        }
        out.rowptr[e + 1] = static_cast<int32_t>(out.src.size());
    }
}

}  // namespace taco
