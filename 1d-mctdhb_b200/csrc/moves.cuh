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

#include "common.cuh"

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


// The same enumeration split into independent tasks, so many threads can
// write the element list at once: task t < M writes rho1[t][t] and
// rho2[tttt]; the next M(M-1)/2 tasks, one per pair k<l, write rho2[klkl]
// and the M+1 single-move elements of (k,l); the last M(M+1)/2 tasks, one
// per source pair k<=s, write that pair's doubles.  Every element lands at
// its index in for_each_density_element's order (offsets in closed form).
__host__ __device__ constexpr int dens_ntasks(int M) { return M + M * (M - 1) / 2 + M * (M + 1) / 2; }

template <class Fn>
__host__ __device__ void density_element_task(int M, int t, Fn&& f) {
    const int npair = M * (M - 1) / 2;
    if (t < M) {
        f(t, D_R1_DIAG, t, t, t, t);
        f(M + t, D_R2_KKKK, t, t, t, t);
        return;
    }
    t -= M;
    if (t < npair) {
        int k = 0, r = t;  // t-th pair k<l in lexicographic order
        while (r >= M - 1 - k) r -= M - 1 - k, k++;
        const int l = k + 1 + r;
        f(2 * M + t, D_R2_KSKS, k, l, k, l);
        int e = 2 * M + npair + t * (M + 1);
        f(e++, D_R1_OFF, k, l, k, l);
        f(e++, D_R2_KKKL, k, k, k, l);
        f(e++, D_R2_KLLL, k, l, l, l);
        for (int s = 0; s < M; s++)
            if (s != k && s != l) f(e++, D_R2_KSSL, k, s, s, l);
        return;
    }
    t -= npair;
    // t-th source pair k<=s; doubles of the pairs before it
    int e = 2 * M + npair + npair * (M + 1);
    int k = 0, s = 0;
    for (int u = 0;; u++) {
        if (u == t) break;
        e += (k == s) ? (M - 1 - k) + (M - 1) * (M - 2) / 2 : (M - 2) * (M - 3) / 2;
        if (++s == M) s = ++k;
    }
    for (int q = 0; q < M; q++)
        for (int l = q; l < M; l++) {
            if (k == s) {
                if (q == k || l == k) continue;
                if (q == l) {
                    if (q > k) f(e++, D_R2_KKQQ, k, k, q, q);
                } else {
                    f(e++, D_R2_KKQL, k, k, q, l);
                }
            } else {
                if (q == l || q == k || q == s || l == k || l == s) continue;
                f(e++, D_R2_KSQL, k, s, q, l);
            }
        }
}

// Packed H.C coefficient table (layout above) from h (M x M row-major) and
// g (hint[k + sM + qM^2 + lM^3]); the caller runs it on one thread.
__device__ inline void hc_pack_table(int M, const double2* __restrict__ hob,
                                     const double2* __restrict__ hint, double2* __restrict__ tab) {
    const int M2 = M * M, M3 = M2 * M;
    auto g = [&](int a, int b, int c, int d) { return hint[a + b * M + c * M2 + d * M3]; };
    int p = 0;
    for (int k = 0; k < M; k++) tab[p++] = hob[k * M + k];
    for (int k = 0; k < M; k++) tab[p++] = cscale(g(k, k, k, k), 0.5);
    for (int k = 0; k < M; k++)
        for (int s = k + 1; s < M; s++) tab[p++] = cscale(g(k, s, k, s), 2.0);
    for (int k = 0; k < M; k++)
        for (int l = 0; l < M; l++) {
            if (l == k) continue;
            double2 gk = g(k, k, k, l);
            double2 h = hob[k * M + l];
            tab[p++] = make_double2(h.x - gk.x, h.y - gk.y);
            for (int s = 0; s < M; s++) {
                if (s == k)
                    tab[p++] = gk;
                else if (s == l)
                    tab[p++] = g(k, l, l, l);
                else
                    tab[p++] = cscale(g(k, s, s, l), 2.0);
            }
        }
    for (int k = 0; k < M; k++)
        for (int s = k; s < M; s++)
            for (int q = 0; q < M; q++)
                for (int l = q; l < M; l++) {
                    if (q == k || q == s || l == k || l == s) continue;
                    double f = (k == s && q == l) ? 0.5 : ((k == s || q == l) ? 1.0 : 2.0);
                    tab[p++] = cscale(g(k, s, q, l), f);
                }
}

// Entry e = P * npairs + Q of the pair matrix W of H = sum W[P][Q] a+_P a_Q
// (pairhc_tmpl.cuh), P = {k <= s} created, Q = {q <= l} annihilated, with the g
// elements and factors of the reference's rules (the move coefficients of
// moves.cuh) and the one-body part spread over the spectator orbital x
// with weight 1/(N-1):
//   P = Q = {k,k}:    1/2 g_kkkk + h_kk/(N-1)
//   P = Q = {k,s}:    2 g_ksks + (h_kk + h_ss)/(N-1)
//   P = {a,x}, Q = {b,x}, a != b (one boson b -> a, spectator x):
//                     c + h_ab/(N-1),  c = g_aaab (x = a), g_abbb (x = b),
//                                          2 g_axxb otherwise
//   P, Q disjoint:    f g_ksql, f = 1/2 (k=s, q=l), 1 (one of them), 2
__device__ inline double2 pair_w_entry(int N, int M, const double2* __restrict__ hob,
                                       const double2* __restrict__ hint, int e) {
    const int P = M * (M + 1) / 2, M2 = M * M, M3 = M2 * M;
    const double inv = 1.0 / (double)(N - 1);
    auto g = [&](int a, int b, int c, int d) { return hint[a + b * M + c * M2 + d * M3]; };
    auto h = [&](int a, int b) { return hob[a * M + b]; };
    auto pair = [&](int p, int& a, int& b) {
        for (int u = 0, c = 0; u < M; u++)
            for (int v = u; v < M; v++, c++)
                if (c == p) a = u, b = v;
    };
    {
        const int pa = e / P, pb = e % P;
        int k = 0, s = 0, q = 0, l = 0;
        pair(pa, k, s);
        pair(pb, q, l);
        double2 w;
        if (pa == pb) {
            if (k == s) {
                w = cadd(cscale(g(k, k, k, k), 0.5), cscale(h(k, k), inv));
            } else {
                w = cadd(cscale(g(k, s, k, s), 2.0), cscale(cadd(h(k, k), h(s, s)), inv));
            }
        } else {
            int x = -1;
            if (k == q || k == l)
                x = k;
            else if (s == q || s == l)
                x = s;
            if (x >= 0) {
                const int a = (k == x) ? s : k, b = (q == x) ? l : q;
                double2 c;
                if (x == a)
                    c = g(a, a, a, b);
                else if (x == b)
                    c = g(a, b, b, b);
                else
                    c = cscale(g(a, x, x, b), 2.0);
                w = cadd(c, cscale(h(a, b), inv));
            } else {
                const double f = (k == s && q == l) ? 0.5 : ((k == s || q == l) ? 1.0 : 2.0);
                w = cscale(g(k, s, q, l), f);
            }
        }
        return w;
    }
}


// Store the summed density element v (descriptor kind, k, s, q, l) into
// rho1 (M x M row-major) / rho2 (M^4) with the reference's symmetric fill
// (density_matrices.c:33-50, 86-442).
__device__ inline void dens_fill(int kind, int k, int s, int q, int l, double2 v, int M,
                                 double2* __restrict__ rho1, double2* __restrict__ rho2) {
    const double2 c = make_double2(v.x, -v.y);
    const int M2 = M * M, M3 = M2 * M;
    auto R = [&](int a, int b, int cc, int d) -> double2& { return rho2[a + b * M + cc * M2 + d * M3]; };
    switch (kind) {
        case D_R1_DIAG: rho1[k * M + k] = v; break;
        case D_R2_KKKK: R(k, k, k, k) = v; break;
        case D_R2_KSKS:
            R(k, s, k, s) = v; R(s, k, k, s) = v; R(s, k, s, k) = v; R(k, s, s, k) = v;
            break;
        case D_R1_OFF:  // (k, l) stored as (k, s=l)
            rho1[k * M + s] = v;
            rho1[s * M + k] = c;
            break;
        case D_R2_KKKL:
            R(k, k, k, l) = v; R(k, k, l, k) = v; R(l, k, k, k) = c; R(k, l, k, k) = c;
            break;
        case D_R2_KLLL:  // (k, l, l, l) stored as (k, s=l, q=l, l)
            R(k, l, l, l) = v; R(l, k, l, l) = v; R(l, l, l, k) = c; R(l, l, k, l) = c;
            break;
        case D_R2_KSSL:
            R(k, s, s, l) = v; R(s, k, s, l) = v; R(s, k, l, s) = v; R(k, s, l, s) = v;
            R(l, s, s, k) = c; R(s, l, s, k) = c; R(s, l, k, s) = c; R(l, s, k, s) = c;
            break;
        case D_R2_KKQQ:
            R(k, k, q, q) = v; R(q, q, k, k) = c;
            break;
        case D_R2_KKQL:
            R(k, k, q, l) = v; R(k, k, l, q) = v; R(l, q, k, k) = c; R(q, l, k, k) = c;
            break;
        case D_R2_KSQL:
            R(k, s, q, l) = v; R(s, k, q, l) = v; R(k, s, l, q) = v; R(s, k, l, q) = v;
            break;
    }
}

}  // namespace mctdhb
