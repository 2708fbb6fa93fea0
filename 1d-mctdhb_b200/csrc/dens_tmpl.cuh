// dens_tmpl.cuh -- register-resident density-matrix kernel for M <= 8
// orbitals, one explicit instantiation per translation unit (dens_m*.cu).
// See density.cu for the design notes.
#pragma once
#include <algorithm>

#include "common.cuh"
#include "hc_tmpl.cuh"
#include "kernels.h"
#include "movelist.cuh"

namespace mctdhb {

// transposed reduction of v[0..7] over the 32 lanes; lane l with (l & 3) == 0
// adds the warp sum of element (l >> 2) to acc[l >> 2].
__device__ __forceinline__ void flush8(double2 (&v)[8], double2* acc, int lane) {
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    double2 w[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        double2 send = b4 ? v[j] : v[j + 4];
        double2 keep = b4 ? v[j + 4] : v[j];
        keep.x += __shfl_xor_sync(0xffffffffu, send.x, 16);
        keep.y += __shfl_xor_sync(0xffffffffu, send.y, 16);
        w[j] = keep;
    }
    double2 x[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        double2 send = b3 ? w[j] : w[j + 2];
        double2 keep = b3 ? w[j + 2] : w[j];
        keep.x += __shfl_xor_sync(0xffffffffu, send.x, 8);
        keep.y += __shfl_xor_sync(0xffffffffu, send.y, 8);
        x[j] = keep;
    }
    double2 send = b2 ? x[0] : x[1];
    double2 y = b2 ? x[1] : x[0];
    y.x += __shfl_xor_sync(0xffffffffu, send.x, 4);
    y.y += __shfl_xor_sync(0xffffffffu, send.y, 4);
    y.x += __shfl_xor_sync(0xffffffffu, y.x, 2);
    y.y += __shfl_xor_sync(0xffffffffu, y.y, 2);
    y.x += __shfl_xor_sync(0xffffffffu, y.x, 1);
    y.y += __shfl_xor_sync(0xffffffffu, y.y, 1);
    if ((lane & 3) == 0) {
        double2 a = acc[lane >> 2];
        a.x += y.x;
        a.y += y.y;
        acc[lane >> 2] = a;
    }
}

// Contributions of one row to every density element, reduced across the
// warp and added to the warp's accumulators wacc[0..EP).  Called by all
// threads of a block together (the SYNC barriers inside); `live` is false
// for padding threads past the last row.
template <int M, int SYNC>
__device__ __forceinline__ void dens_row(const SpaceView& sp, uint32_t row, bool live,
                                         const double2* __restrict__ C, double2* wacc,
                                         int lane) {
    constexpr int E = dens_nelem(M);
    constexpr int EP = (E + 7) / 8 * 8;
    RowState<M> st;
    double2 ci = make_double2(0.0, 0.0);
    if (live) {
        load_row<M>(sp, row, st);
        ci = __ldg(C + row);
    } else {
        static_for<M>([&](auto mi) { st.n[decltype(mi)::value] = 0; });
        static_for<(M > 1 ? M - 1 : 1)>([&](auto mi) {
            constexpr int m = decltype(mi)::value;
            st.F[m][0] = st.F[m][1] = st.F[m][2] = st.F[m][3] = 0;
        });
    }
    double sq0[M], sq1[M];
    static_for<M>([&](auto mi) {
        constexpr int m = decltype(mi)::value;
        sq0[m] = __ldg(sp.sq + st.n[m]);
        sq1[m] = __ldg(sp.sq + st.n[m] + 1);
    });
    const double m2 = ci.x * ci.x + ci.y * ci.y;
    double2 v[8];
    double2 t = make_double2(0.0, 0.0);  // current single-move product

    static_for<EP>([&](auto ei) {
        constexpr int e = decltype(ei)::value;
        double2 x = make_double2(0.0, 0.0);
        if constexpr (e < E) {
            constexpr DensElem d = kDensElems<M>.e[e];
            constexpr int k = d.k, s = d.s, q = d.q, l = d.l;
            if constexpr (d.kind == D_R1_DIAG) {
                x.x = m2 * st.n[k];
            } else if constexpr (d.kind == D_R2_KKKK) {
                x.x = m2 * (st.n[k] * (st.n[k] - 1));
            } else if constexpr (d.kind == D_R2_KSKS) {
                x.x = m2 * (st.n[k] * st.n[s]);
            } else if constexpr (d.kind == D_R1_OFF) {  // move k -> s
                t = make_double2(0.0, 0.0);
                if (st.n[k] > 0) {
                    const uint32_t j = jumpc<M, k, -1, s, -1>(st, row);
                    const double2 cj = __ldg(C + j);
                    t = cscale(cfma_conj(ci, cj, make_double2(0.0, 0.0)), sq0[k] * sq1[s]);
                }
                x = t;
            } else if constexpr (d.kind == D_R2_KKKL) {
                x = cscale(t, (double)(st.n[k] - 1));
            } else if constexpr (d.kind == D_R2_KLLL || d.kind == D_R2_KSSL) {
                x = cscale(t, (double)st.n[s]);
            } else {
                bool valid;
                double sa;
                if constexpr (k == s) {
                    valid = st.n[k] >= 2;
                    sa = valid ? sq0[k] * __ldg(sp.sq + st.n[k] - 1) : 0.0;
                } else {
                    valid = st.n[k] >= 1 && st.n[s] >= 1;
                    sa = sq0[k] * sq0[s];
                }
                if (valid) {
                    const uint32_t j = jumpc<M, k, s, q, l>(st, row);
                    const double2 cj = __ldg(C + j);
                    double sb;
                    if constexpr (q == l)
                        sb = sq1[q] * __ldg(sp.sq + st.n[q] + 2);
                    else
                        sb = sq1[q] * sq1[l];
                    x = cscale(cfma_conj(ci, cj, make_double2(0.0, 0.0)), sa * sb);
                }
            }
        }
        v[e % 8] = x;
        if constexpr (e % 8 == 7) flush8(v, wacc + (e / 8) * 8, lane);
        if constexpr (SYNC > 0 && e % SYNC == SYNC - 1) __syncthreads();
    });
}

// Rows are dealt to blocks of DENS_BLOCK threads in a block-uniform loop, so
// SYNC > 0 can put a block barrier every SYNC elements (the warps then walk
// the unrolled code together and share instruction-cache lines, as in the
// H.C kernel).  The barrier changes no arithmetic: every SYNC variant sums
// in the same order and gives the same bits.
constexpr int DENS_BLOCK = 128;

// The reduction layout is fixed by the grid, which is a function of the space
// size only (min(888, dim/128) blocks; 888 = 6 x 148 runs in whole waves at
// two or three resident blocks per SM): block b owns rows
// b*128 + k*grid*128 + t and one partial slice, so the sums do not depend on
// the launch variant.
template <int M, int SYNC, int MINB>
__global__ void __launch_bounds__(DENS_BLOCK, MINB)
    dens_kernel(SpaceView sp, const double2* __restrict__ C, double2* __restrict__ partial) {
    constexpr int E = dens_nelem(M);
    constexpr int EP = (E + 7) / 8 * 8;
    extern __shared__ double2 sacc[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = DENS_BLOCK >> 5;
    double2* wacc = sacc + warp * EP;
    for (int i = lane; i < EP; i += 32) wacc[i] = make_double2(0.0, 0.0);
    __syncwarp();

    for (uint32_t bbase = blockIdx.x * DENS_BLOCK; bbase < sp.dim;
         bbase += gridDim.x * DENS_BLOCK) {
        const uint32_t row = bbase + threadIdx.x;
        const bool live = row < sp.dim;
        dens_row<M, SYNC>(sp, row, live, C, wacc, lane);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < EP; e += DENS_BLOCK) {
        double2 s = sacc[e];
        for (int w = 1; w < nwarps; w++) {
            s.x += sacc[w * EP + e].x;
            s.y += sacc[w * EP + e].y;
        }
        partial[(size_t)blockIdx.x * EP + e] = s;
    }
}

template <int M, int SYNC, int MINB>
int dens_launch_variant(const SpaceView& sp, const double2* C, double2* partial, int grid,
                        cudaStream_t st) {
    constexpr int EP = (dens_nelem(M) + 7) / 8 * 8;
    const size_t smem = (size_t)(DENS_BLOCK / 32) * EP * sizeof(double2);
    static std::atomic<uint64_t> attr{0};
    if (set_attributes_once(attr, [&]() -> int {
            MCTDHB_CUDA_TRY(cudaFuncSetAttribute(dens_kernel<M, SYNC, MINB>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem));
            return 0;
        }))
        return -1;
    if (grid == 0) return 0;  // attributes only (before graph capture)
    dens_kernel<M, SYNC, MINB><<<grid, DENS_BLOCK, smem, st>>>(sp, C, partial);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

// kDensVariants (kernels.h): barrier interval x register budget (MINB
// resident blocks per SM); variant 0 is the default
template <int M>
int dens_launch_tmpl(const SpaceView& sp, const double2* C, double2* partial, int grid,
                     int variant, cudaStream_t st) {
    switch (variant) {
        case 1: return dens_launch_variant<M, 32, 0>(sp, C, partial, grid, st);
        case 2: return dens_launch_variant<M, 64, 3>(sp, C, partial, grid, st);
        case 3: return dens_launch_variant<M, 128, 0>(sp, C, partial, grid, st);
        default: return dens_launch_variant<M, 64, 0>(sp, C, partial, grid, st);
    }
}

}  // namespace mctdhb
