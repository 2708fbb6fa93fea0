// batch_tmpl.cuh -- per-M H.C and density kernels of the batched engine:
// persistent blocks walk the tile list of one orbital count M, each tile a
// run of rows of one slot, with the row bodies of the single-system kernels
// (hc_row, dens_row).  One explicit instantiation per M (batch_m*.cu).
#pragma once
#include "batch.h"
#include "dens_tmpl.cuh"
#include "hc_tmpl.cuh"

namespace mctdhb {

// Lanczos H.C of step iteration `iter` for every slot of the list:
//   out = H V[iter] - beta_{iter-1} V[iter-1]   (iter > 0)
//   out = H V[0]                                (iter == 0)
// Slots that stopped, or whose Lanczos recurrence broke down in this step,
// are skipped (multiconfig_lanczos.c:70-71).
template <int M, int SYNC>
__global__ void __launch_bounds__(kBatchHcRows, 2)
    hc_batch_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                    const int* __restrict__ off, const int* __restrict__ cnt, int iter) {
    constexpr int TAB = hc_table_size(M);
    __shared__ double2 tab[TAB];
    const int nt = cnt[M];
    const BatchTile* list = tiles + off[M];
    int cur = -1;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const BatchTile tl = list[t];
        const BatchSlot& S = slots[tl.slot];
        if (S.flags[BF_STATE] != SLOT_RUNNING || S.flags[BF_BREAK]) continue;
        if (tl.slot != cur) {
            __syncthreads();
            for (int i = threadIdx.x; i < TAB; i += kBatchHcRows) tab[i] = S.tab[i];
            __syncthreads();
            cur = tl.slot;
        }
        const uint32_t nc = S.nc;
        const uint32_t row = tl.idx + threadIdx.x;
        const bool live = row < nc;
        double2 acc = hc_row<M, SYNC>(S.sp, row, live, S.V + (size_t)iter * nc, tab);
        if (iter > 0 && live) {
            const double2 pv = S.V[(size_t)(iter - 1) * nc + row];
            const double b = S.scal[BS_OFFD + iter - 1].x;
            acc.x -= b * pv.x;
            acc.y -= b * pv.y;
        }
        if (live) S.out[row] = acc;
    }
}

// rho1/rho2 partial sums of V[0]: slice `idx` of a slot covers dchunks runs
// of 128 rows; its block writes the slice's sums to dpart[idx * EP ...].
template <int M, int SYNC>
__global__ void __launch_bounds__(kBatchDensThreads)
    dens_batch_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                      const int* __restrict__ off, const int* __restrict__ cnt) {
    constexpr int E = dens_nelem(M);
    constexpr int EP = (E + 7) / 8 * 8;
    constexpr int NW = kBatchDensThreads / 32;
    extern __shared__ double2 sacc[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2* wacc = sacc + warp * EP;
    const int nt = cnt[M];
    const BatchTile* list = tiles + off[M];
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const BatchTile tl = list[t];
        const BatchSlot& S = slots[tl.slot];
        if (S.flags[BF_STATE] != SLOT_RUNNING) continue;
        for (int i = lane; i < EP; i += 32) wacc[i] = make_double2(0.0, 0.0);
        __syncwarp();
        const uint32_t nc = S.nc;
        const uint32_t r0 = tl.idx * (uint32_t)S.dchunks * kBatchDensThreads;
        for (int c = 0; c < S.dchunks; c++) {
            const uint32_t base = r0 + (uint32_t)c * kBatchDensThreads;
            if (base >= nc) break;  // block-uniform
            const uint32_t row = base + threadIdx.x;
            dens_row<M, SYNC>(S.sp, row, row < nc, S.V, wacc, lane);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < EP; e += kBatchDensThreads) {
            double2 s = sacc[e];
            for (int w = 1; w < NW; w++) {
                s.x += sacc[w * EP + e].x;
                s.y += sacc[w * EP + e].y;
            }
            S.dpart[(size_t)tl.idx * EP + e] = s;
        }
        __syncthreads();
    }
}

// barrier interval of the unrolled row bodies: the larger move lists need
// the warps of a block to walk the code together (hc_tmpl.cuh)
template <int M>
constexpr int batch_sync() {
    return M >= 6 ? 64 : 0;
}

template <int M>
int hc_batch_launch(const BatchSlot* slots, const BatchTile* tiles, const int* off,
                    const int* cnt, int iter, cudaStream_t st) {
    hc_batch_kernel<M, batch_sync<M>()><<<num_sms() * 2, kBatchHcRows, 0, st>>>(slots, tiles, off,
                                                                              cnt, iter);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int M>
int dens_batch_launch(const BatchSlot* slots, const BatchTile* tiles, const int* off,
                      const int* cnt, cudaStream_t st) {
    constexpr int EP = (dens_nelem(M) + 7) / 8 * 8;
    const size_t smem = (size_t)(kBatchDensThreads / 32) * EP * sizeof(double2);
    if (slots == nullptr) {  // launch attributes only (before graph capture)
        MCTDHB_CUDA_TRY(cudaFuncSetAttribute(dens_batch_kernel<M, batch_sync<M>()>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
        return 0;
    }
    dens_batch_kernel<M, batch_sync<M>()><<<num_sms() * 3, kBatchDensThreads, smem, st>>>(
        slots, tiles, off, cnt);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mctdhb
