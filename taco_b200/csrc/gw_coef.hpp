// gw_coef.hpp -- time-independent coefficient table of the MIKX -> GW -> L4 chain.
//
// At one time t, L4 is linear in the F/C/R values of the nf^3 frequency triples:
//   MIKX (cpp/src/tcl/tcl4_mikx.cpp:87-177) gathers M = F - R, I = F, K = R, X = C + R;
//   NAKZWAN (cpp/src/tcl/tcl4_assemble.cpp:53-186) forms T(n,i,m,j) as a sum of
//   products of coupling-operator entries with those gathers;
//   GW = T + T^H (tcl4_assemble.cpp:188-200) and L4(n+Nm, i+Nj) = GW(n+Ni, m+Nj)
//   (tcl4_assemble.cpp:204-230).
// Walking those loops once with symbolic sources gives, for every L4 entry e,
//   L4_e(t) = sum_s w_es v_s(t) + sum_s w'_es conj(v_s(t)),
// with v_s the F (s < nf^3), C (nf^3 <= s < 2nf^3) or R (2nf^3 <= s) value of triple
// s mod nf^3 at time t.  Terms with equal (source, conjugation) are merged; exact
// zeros are dropped.  The table is stored in CSR form over the N^4 entries of L4
// (column-major entry index e = row + N^2 col).
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace taco {

struct CoefTable {
    int N = 0, nf = 0;
    std::vector<int32_t> rowptr;   // [N^4 + 1]
    std::vector<uint32_t> src;     // source index | (conj << 31)
    std::vector<double2> coef;
    std::vector<uint8_t> triple_fc_used;  // per triple: F or C referenced
    std::vector<uint8_t> triple_r_used;   // per triple: R referenced
};

// ops: num_ops matrices, column-major N x N (eigenbasis); p2f column-major N x N.
// structural: keep every (entry, source) pair the sums reach, zero coefficients included
// (the sparsity pattern of the map for all operator values, as the gradient needs).
// Host threads of build_coef_table on this thread (0: up to 16, as the map's size allows).
void set_coef_table_threads(int n);

void build_coef_table(int N, int nf, const int* p2f, const double2* ops, int num_ops, CoefTable& out,
                      bool structural = false);

// Gradient of a real loss with respect to the coupling operators through the table's
// coefficients (table built with structural = true).  Z[q] = sum_t conj(G(L4_e(t))) v~_q(t) for CSR entry q of row e (v~ the
// source value, conjugated for conjugated entries); ops_bar (num_ops x N x N) is
// accumulated with G(a) = dloss/dRe a + i dloss/dIm a for every operator entry a.
void coef_table_ops_grad(int N, int nf, const int* p2f, const double2* ops, int num_ops, const CoefTable& table,
                         const double2* Z, double2* ops_bar);

}  // namespace taco
