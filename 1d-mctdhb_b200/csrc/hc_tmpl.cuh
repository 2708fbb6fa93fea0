// hc_tmpl.cuh -- register-resident H.C kernel for M <= 8 orbitals, one
// explicit instantiation per translation unit (hc_m*.cu).  See
// hamiltonian.cu for the design notes and moves.cuh for the coefficient
// folding.
//
// Instruction supply.  The fully unrolled move list is the lowest
// instruction count per row (every orbital index, rank offset and table
// offset is an immediate), but at M = 8 it is ~180 KB of code: warps that
// drift apart stream different parts of it and stall on instruction fetch.
// SYNC > 0 puts a block barrier every SYNC moves so the warps of a block
// walk the code together and share instruction-cache lines; BLOCK and SYNC
// are picked per (N, M) by the autotuner (hamiltonian.cu).
#pragma once
#include "common.cuh"
#include "kernels.h"
#include "movelist.cuh"

namespace mctdhb {

// jump target with compile-time orbitals (k, s removed; q, l added; -1 none)
template <int M, int k, int s, int q, int l>
__device__ __forceinline__ uint32_t jumpc(const RowState<M>& st, uint32_t row) {
    uint32_t d = 0;
    static_for<M - 1>([&](auto mi) {
        constexpr int m = decltype(mi)::value;
        constexpr int dl = (q >= 0 && m >= q) + (l >= 0 && m >= l) - (k >= 0 && m >= k) -
                           (s >= 0 && m >= s);
        if constexpr (dl != 0) d += st.F[m][dl_index(dl)];
    });
    return row - d;
}

template <int M>
__device__ __forceinline__ void zero_row(RowState<M>& st) {
    static_for<M>([&](auto mi) { st.n[decltype(mi)::value] = 0; });
    static_for<(M > 1 ? M - 1 : 1)>([&](auto mi) {
        constexpr int m = decltype(mi)::value;
        st.F[m][0] = st.F[m][1] = st.F[m][2] = st.F[m][3] = 0;
    });
}

// H.C of one row: the diagonal plus every distinct neighbour reached by one
// or two moves.  Called by all threads of a block together (the SYNC
// barriers inside); `live` is false for padding threads past the last row.
template <int M, int SYNC>
__device__ __forceinline__ double2 hc_row(const SpaceView& sp, uint32_t row, bool live,
                                          const double2* __restrict__ C,
                                          const double2* __restrict__ tab) {
    constexpr int NMOVE = HcMoveList<M>::N;
    RowState<M> st;
    if (live)
        load_row<M>(sp, row, st);
    else
        zero_row<M>(st);
    double sq0[M], sq1[M];
    static_for<M>([&](auto mi) {
        constexpr int m = decltype(mi)::value;
        sq0[m] = __ldg(sp.sq + st.n[m]);
        sq1[m] = __ldg(sp.sq + st.n[m] + 1);
    });
    const double2 ci = live ? __ldg(C + row) : make_double2(0.0, 0.0);

    // diagonal: h_kk n_k + 1/2 g_kkkk n_k (n_k - 1) + 2 g_ksks n_k n_s
    double2 dg = make_double2(0.0, 0.0);
    static_for<M>([&](auto ki) {
        constexpr int k = decltype(ki)::value;
        dg = cadd(dg, cscale(tab[k], (double)st.n[k]));
        dg = cadd(dg, cscale(tab[M + k], (double)(st.n[k] * (st.n[k] - 1))));
        static_for<M>([&](auto si) {
            constexpr int s = decltype(si)::value;
            if constexpr (s > k) {
                constexpr int p = 2 * M + k * M - k * (k + 1) / 2 + (s - k - 1);
                dg = cadd(dg, cscale(tab[p], (double)(st.n[k] * st.n[s])));
            }
        });
    });
    double2 acc = cmul(dg, ci);

    bool vs = false;
    double sa = 0.0;
    double2 as = make_double2(0.0, 0.0);
    static_for<NMOVE>([&](auto ei) {
        constexpr int e = decltype(ei)::value;
        constexpr HcMove mv = kHcMoves<M>.m[e];
        constexpr int k = mv.k, s = mv.s, q = mv.q, l = mv.l;
        if constexpr (s < 0) {
            // single move k -> q
            if (st.n[k] > 0) {
                const uint32_t j = jumpc<M, k, -1, q, -1>(st, row);
                const double2 cj = __ldg(C + j);
                double2 c = tab[mv.tab];
                static_for<M>([&](auto xi) {
                    constexpr int x = decltype(xi)::value;
                    c = cadd(c, cscale(tab[mv.tab + 1 + x], (double)st.n[x]));
                });
                acc = cfma(cscale(c, sq0[k] * sq1[q]), cj, acc);
            }
        } else {
            // double move (k, s) -> (q, l), accumulated per source pair
            if constexpr (mv.first) {
                if constexpr (k == s) {
                    vs = st.n[k] >= 2;
                    sa = vs ? sq0[k] * __ldg(sp.sq + st.n[k] - 1) : 0.0;
                } else {
                    vs = st.n[k] >= 1 && st.n[s] >= 1;
                    sa = sq0[k] * sq0[s];
                }
                as = make_double2(0.0, 0.0);
            }
            if (vs) {
                const uint32_t j = jumpc<M, k, s, q, l>(st, row);
                const double2 cj = __ldg(C + j);
                double sb;
                if constexpr (q == l)
                    sb = sq1[q] * __ldg(sp.sq + st.n[q] + 2);
                else
                    sb = sq1[q] * sq1[l];
                as = cfma(tab[mv.tab], cscale(cj, sb), as);
            }
            if constexpr (mv.last) acc = cadd(acc, cscale(as, sa));
        }
        if constexpr (SYNC > 0 && e % SYNC == SYNC - 1) __syncthreads();
    });
    return acc;
}

template <int M, int BLOCK, int SYNC>
__global__ void __launch_bounds__(BLOCK, (BLOCK <= 256 ? 2 : 1))
    hc_kernel(SpaceView sp, const double2* __restrict__ C, double2* __restrict__ HC,
              const double2* __restrict__ tab_g, HcEpilogue ep) {
    constexpr int TAB = hc_table_size(M);
    __shared__ double2 tab[TAB];
    for (int i = threadIdx.x; i < TAB; i += BLOCK) tab[i] = tab_g[i];
    __syncthreads();
    if (ep.flag != nullptr && *ep.flag != 0) return;  // Lanczos breakdown: no-op

    // block-uniform trip count: every thread reaches every barrier
    for (uint32_t base = blockIdx.x * BLOCK; base < sp.dim; base += gridDim.x * BLOCK) {
        const uint32_t row = base + threadIdx.x;
        const bool live = row < sp.dim;
        double2 acc = hc_row<M, SYNC>(sp, row, live, C, tab);
        // Lanczos epilogue: out = HC - beta * prev
        if (ep.prev != nullptr && live) {
            const double2 pv = __ldg(ep.prev + row);
            const double b = *ep.beta;
            acc.x -= b * pv.x;
            acc.y -= b * pv.y;
        }
        if (live) HC[row] = acc;
    }
}

template <int M, int BLOCK, int SYNC>
int hc_launch_variant(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
                      const HcEpilogue& ep, int blocks_per_sm, cudaStream_t st) {
    const uint64_t need = ((uint64_t)sp.dim + BLOCK - 1) / BLOCK;
    const uint64_t cap = (uint64_t)num_sms() * blocks_per_sm;
    const int grid = (int)(need < cap ? (need ? need : 1) : cap);
    hc_kernel<M, BLOCK, SYNC><<<grid, BLOCK, 0, st>>>(sp, C, HC, tab, ep);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

// the tuned variants (kHcVariants of them, kernels.h), in autotuner order
template <int M>
int hc_launch_tmpl(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
                   const HcEpilogue& ep, int variant, cudaStream_t st) {
    // variant 0 is the default outside the tuner (best measured at N=30, M=8)
    switch (variant) {
        case 1: return hc_launch_variant<M, 512, 32>(sp, C, HC, tab, ep, 1, st);
        case 2: return hc_launch_variant<M, 512, 128>(sp, C, HC, tab, ep, 1, st);
        case 3: return hc_launch_variant<M, 256, 32>(sp, C, HC, tab, ep, 2, st);
        case 4: return hc_launch_variant<M, 256, 0>(sp, C, HC, tab, ep, 2, st);
        default: return hc_launch_variant<M, 512, 64>(sp, C, HC, tab, ep, 1, st);
    }
}

}  // namespace mctdhb
