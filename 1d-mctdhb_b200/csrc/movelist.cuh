// movelist.cuh -- compile-time move / element lists for the register-resident
// kernels (M <= 8).  Every loop over moves is a fold over an index sequence,
// so occupations, rank offsets and accumulator slots are indexed with
// constants and stay in registers.
#pragma once
#include <utility>

#include "moves.cuh"

namespace mctdhb {

template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- H.C: single moves (k -> l) then double moves (k,s -> q,l) ----------
struct HcMove {
    int k, s, q, l;     // s = -1 / l = ... for single moves: k -> q, s = l = -1
    int first, last;    // first / last target of a source pair (doubles)
    int tab;            // table offset (single: start of its M+1 block)
};

template <int M>
struct HcMoveList {
    static constexpr int NS = M * (M - 1);
    static constexpr int ND = hc_ndouble(M);
    static constexpr int N = NS + ND;
    HcMove m[N > 0 ? N : 1];
    constexpr HcMoveList() : m{} {
        int e = 0;
        int p = hc_ndiag(M);
        for (int k = 0; k < M; k++)
            for (int l = 0; l < M; l++) {
                if (l == k) continue;
                m[e] = HcMove{k, -1, l, -1, 0, 0, p};
                p += M + 1;
                e++;
            }
        for (int k = 0; k < M; k++)
            for (int s = k; s < M; s++) {
                int first = e;
                for (int q = 0; q < M; q++)
                    for (int l = q; l < M; l++) {
                        if (q == k || q == s || l == k || l == s) continue;
                        m[e] = HcMove{k, s, q, l, e == first, 0, p};
                        p++;
                        e++;
                    }
                if (e > first) m[e - 1].last = 1;
            }
    }
};
template <int M>
inline constexpr HcMoveList<M> kHcMoves{};

// ---- density elements (moves.cuh order) -----------------------------------
struct DensElem {
    int kind, k, s, q, l;
};

template <int M>
struct DensElemList {
    static constexpr int N = dens_nelem(M);
    DensElem e[N > 0 ? N : 1];
    constexpr DensElemList() : e{} {
        int n = 0;
        for (int k = 0; k < M; k++) e[n++] = DensElem{D_R1_DIAG, k, k, k, k};
        for (int k = 0; k < M; k++) e[n++] = DensElem{D_R2_KKKK, k, k, k, k};
        for (int k = 0; k < M; k++)
            for (int s = k + 1; s < M; s++) e[n++] = DensElem{D_R2_KSKS, k, s, k, s};
        for (int k = 0; k < M; k++)
            for (int l = k + 1; l < M; l++) {
                e[n++] = DensElem{D_R1_OFF, k, l, k, l};
                e[n++] = DensElem{D_R2_KKKL, k, k, k, l};
                e[n++] = DensElem{D_R2_KLLL, k, l, l, l};
                for (int s = 0; s < M; s++)
                    if (s != k && s != l) e[n++] = DensElem{D_R2_KSSL, k, s, s, l};
            }
        for (int k = 0; k < M; k++)
            for (int s = k; s < M; s++)
                for (int q = 0; q < M; q++)
                    for (int l = q; l < M; l++) {
                        if (k == s) {
                            if (q == k || l == k) continue;
                            if (q == l) {
                                if (q > k) e[n++] = DensElem{D_R2_KKQQ, k, k, q, q};
                            } else {
                                e[n++] = DensElem{D_R2_KKQL, k, k, q, l};
                            }
                        } else {
                            if (q == l || q == k || q == s || l == k || l == s) continue;
                            e[n++] = DensElem{D_R2_KSQL, k, s, q, l};
                        }
                    }
    }
};
template <int M>
inline constexpr DensElemList<M> kDensElems{};

}  // namespace mctdhb
