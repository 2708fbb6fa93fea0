// moves.cuh -- the particle-move enumeration shared by the H.C and density
// kernels and by the host code that packs coefficient tables.
//
// H.C (hamiltonian.c:7-406) is regrouped by the configuration it gathers
// from, so every distinct neighbour j of row i is loaded once:
//   diagonal   : h_kk n_k + 1/2 g_kkkk n_k(n_k-1) + 2 g_ksks n_k n_s (k<s)
//                (rules 1, 2 and the one-body diagonal)
//   single k->l: sqrt(n_k(n_l+1)) [h_kl + (n_k-1) g_kkkl + n_l g_klll
//                 + 2 sum_{s!=k,l} n_s g_kssl]          (one-body, rules 4,5,8)
//   double     : source pair k<=s, target pair q<=l, disjoint:
//                f g_ksql sqrt(n_k (n_s-[k=s]) (n_q+1) (n_l+1+[q=l])),
//                f = 1/2 (kk->qq, rule 3), 1 (kk->ql rule 6, ks->qq rule 7),
//                2 (ks->ql, rule 9);  g_ksql = hint[k + sM + qM^2 + lM^3].
// Table layout (double2), built by hc_prep_kernel:
//   [0, M)                 h_kk
//   [M, 2M)                1/2 g_kkkk
//   [2M, 2M + M(M-1)/2)    2 g_ksks, k<s
//   singles, (k,l) k!=l in row-major order, M+1 entries each:
//                          h_kl - g_kkkl, then W_s (s = 0..M-1) with
//                          W_k = g_kkkl, W_l = g_klll, W_s = 2 g_kssl
//   doubles, in enumeration order, the scaled f g_ksql.
#pragma once
#include <stdint.h>

namespace mctdhb {

__host__ __device__ constexpr int hc_ndiag(int M) { return 2 * M + M * (M - 1) / 2; }
__host__ __device__ constexpr int hc_nsingle(int M) { return M * (M - 1) * (M + 1); }
__host__ __device__ constexpr int hc_ndouble(int M) {
    return M * ((M - 1) * M / 2) + (M * (M - 1) / 2) * ((M - 2) * (M - 1) / 2);
}
__host__ __device__ constexpr int hc_table_size(int M) {
    return hc_ndiag(M) + hc_nsingle(M) + hc_ndouble(M);
}

// Density elements (density_matrices.c) in accumulation order:
//   rho1[k][k]; rho2[kkkk]; rho2[ksks] k<s;
//   per single move k<l: rho1[k][l], rho2[kkkl], rho2[klll], rho2[kssl] s asc;
//   doubles by source pair: (k,k) -> (q,q) q>k and (q,l) q<l with k not in
//   {q,l};  (k,s) k<s -> (q,l) q<l disjoint.
enum DensKind : int {
    D_R1_DIAG = 0,
    D_R2_KKKK = 1,
    D_R2_KSKS = 2,
    D_R1_OFF = 3,
    D_R2_KKKL = 4,
    D_R2_KLLL = 5,
    D_R2_KSSL = 6,
    D_R2_KKQQ = 7,
    D_R2_KKQL = 8,
    D_R2_KSQL = 9,
};

__host__ __device__ constexpr int dens_nelem(int M) {
    return M + M + M * (M - 1) / 2 + (M * (M - 1) / 2) * (M + 1) +
           M * (M - 1) / 2 +                          // kk -> qq, q > k
           M * ((M - 1) * (M - 2) / 2) +              // kk -> ql
           (M * (M - 1) / 2) * ((M - 2) * (M - 3) / 2);  // ks -> ql
}

// Enumerate the density elements in order, calling f(kind, k, s, q, l).
template <class Fn>
__host__ __device__ void for_each_density_element(int M, Fn&& f) {
    for (int k = 0; k < M; k++) f(D_R1_DIAG, k, k, k, k);
    for (int k = 0; k < M; k++) f(D_R2_KKKK, k, k, k, k);
    for (int k = 0; k < M; k++)
        for (int s = k + 1; s < M; s++) f(D_R2_KSKS, k, s, k, s);
    for (int k = 0; k < M; k++)
        for (int l = k + 1; l < M; l++) {
            f(D_R1_OFF, k, l, k, l);
            f(D_R2_KKKL, k, k, k, l);
            f(D_R2_KLLL, k, l, l, l);
            for (int s = 0; s < M; s++)
                if (s != k && s != l) f(D_R2_KSSL, k, s, s, l);
        }
    for (int k = 0; k < M; k++)
        for (int s = k; s < M; s++)
            for (int q = 0; q < M; q++)
                for (int l = q; l < M; l++) {
                    if (k == s) {
                        if (q == k || l == k) continue;
                        if (q == l) {
                            if (q > k) f(D_R2_KKQQ, k, k, q, q);
                        } else {
                            f(D_R2_KKQL, k, k, q, l);
                        }
                    } else {
                        if (q == l || q == k || q == s || l == k || l == s) continue;
                        f(D_R2_KSQL, k, s, q, l);
                    }
                }
}

}  // namespace mctdhb
