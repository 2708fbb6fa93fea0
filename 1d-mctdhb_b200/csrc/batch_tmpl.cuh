// batch_tmpl.cuh -- per-M H.C and density kernels of the batched engine:
// persistent blocks walk the tile lists of one orbital count M (batch.h),
// each tile a run of rows of one slot, with the building blocks of the
// single-system kernels (pairhc_tmpl.cuh, gram_tmpl.cuh).  One explicit
// instantiation per M (batch_m*.cu).
//
// Every value of a slot is computed by one thread, or summed over the
// slot's own slices in a fixed order, so a slot's result does not depend on
// the other slots of the batch.
#pragma once
#include <algorithm>

#include "batch.h"
#include "gram_tmpl.cuh"
#include "pairhc_tmpl.cuh"

namespace mctdhb {

// H.C of this step's Lanczos iteration runs for the slot; the monitor's
// H.C (iter == kBatchMonIter) for the slots whose eigen residual is due
__device__ __forceinline__ bool bt_hc_active(const BatchSlot& S, int iter) {
    if (iter == kBatchMonIter) return S.flags[BF_MON] != 0;
    return S.flags[BF_STATE] == SLOT_RUNNING && !S.flags[BF_BREAK];
}

// Pair contraction Y = A W^T of V[iter] for every tile of list LIST_HY:
// warp-specialised and double-buffered as hcp_y_kernel.  Consecutive tiles
// may belong to different slots, so the producer warps stage a tile's W with
// its A (skipped when the buffer already holds that slot's W) and publish
// the tile's output row, size, Y plane and real-W flag in shared memory; the
// consumers start on the tensor cores without a chain of global loads.  The
// next tile's descriptor is loaded one tile ahead.
struct PairTileMeta {
    double2* Y;
    uint32_t row0, D2;
    int active, real;
};

template <int M, int V>
__global__ void __launch_bounds__(PairHcShape<M, V>::THREADS, 1)
    bhcp_y_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                  const int* __restrict__ cnt, int iter) {
    using PS_ = PairHcShape<M, V>;
    constexpr int P = PS_::P, PS = PS_::PS, ROWS = PS_::ROWS;
    static_assert(ROWS == batch_pair_rows(M), "tile rows of the host lists");
    extern __shared__ double2 smem[];
    __shared__ PairTileMeta meta[2];
    constexpr int WS = PS_::WS;
    double2* Wb = smem;               // two buffers of P x WS
    double2* Ab = smem + 2 * P * WS;  // two buffers of ROWS x PS
    if (iter == kBatchMonIter && batch_mon(cnt)[M] == 0) return;  // no residual due
    const int nt = batch_cnt(cnt, LIST_HY, M);
    const BatchTile* list = tiles + batch_off(cnt, LIST_HY, M);
    const int t = threadIdx.x;
    __shared__ uint64_t bar_full[2], bar_empty[2];  // variant 3's handover
    if constexpr (PS_::MBAR) {
        if (t == 0) {
            mbar_init(&bar_full[0], PS_::PRODUCERS);
            mbar_init(&bar_full[1], PS_::PRODUCERS);
            mbar_init(&bar_empty[0], PS_::CONSUMERS);
            mbar_init(&bar_empty[1], PS_::CONSUMERS);
        }
        __syncthreads();
    }
    // Producers and consumers run their own loops and meet at one block
    // barrier per tile (named barrier 1 over all threads): the producers
    // fill buffer buf ^ 1 while the consumers contract buffer buf.
    if (t >= PS_::CONSUMERS) {
        const int pt = t - PS_::CONSUMERS;
        const int vin = iter < 0 ? 0 : iter;  // input vector V[vin]
        int wslot[2] = {-1, -1};  // slot whose W each buffer holds (same in every producer)
        int tslot = -1;           // slot whose tables the shared table area holds
        void* tab = Ab + 2 * ROWS * PS;
        auto fill = [&](const BatchTile tl, int buf) {
            const BatchSlot& S = slots[tl.slot];
            const bool active = bt_hc_active(S, iter);
            if (pt == 0)
                meta[buf] = PairTileMeta{S.sp.pair_y, tl.idx * (uint32_t)ROWS, S.sp.dim2, active,
                                         active && S.sp.pair_w[P * P].x != 0.0};
            if (!active) return;
            if (wslot[buf] != tl.slot) {
                pair_stage_w<M, V>(S.sp.pair_w, Wb + buf * P * WS, pt, PS_::PRODUCERS);
                wslot[buf] = tl.slot;
            }
            // the slot's rank tables: the previous fill's reads ended at the
            // last block barrier; the producers meet before the new reads
            SpaceView tv = S.sp;
            if (tslot != tl.slot) {
                tv = pair_stage_tab(S.sp, tab, pt, PS_::PRODUCERS);
                pair_producer_barrier<PS_::PRODUCERS>();
                tslot = tl.slot;
            } else if (pair_tab_fits(S.sp.N, M)) {
                tv.sq = (const double*)tab;
                tv.T = (const uint32_t*)((const double*)tab + S.sp.N + 3);
            }
            pair_gather<M, V>(tv, S.V + (size_t)vin * S.nc, tl.idx,
                              Ab + (size_t)buf * ROWS * PS, pt, PS_::PRODUCERS);
        };
        if constexpr (PS_::MBAR) {
            // item i goes to buffer i & 1 once the consumers released it
            // (their item i - 2), then the buffer is marked full
            int i = 0;
            for (int k = blockIdx.x; k < nt; k += gridDim.x, i++) {
                const int buf = i & 1;
                if (i >= 2 && !mbar_wait(&bar_empty[buf], ((i >> 1) - 1) & 1)) {
                    slots[list[k].slot].flags[BF_STATE] = SLOT_ABORTED;  // handover lost
                    return;
                }
                fill(list[k], buf);
                mbar_arrive(&bar_full[buf]);
            }
            return;
        }
        BatchTile next{};
        if ((int)blockIdx.x < nt) fill(list[blockIdx.x], 0);
        if ((int)(blockIdx.x + gridDim.x) < nt) next = list[blockIdx.x + gridDim.x];
        pair_tile_barrier<PS_::THREADS>();
        int buf = 0;
        for (int k = blockIdx.x; k < nt; k += gridDim.x, buf ^= 1) {
            if (k + (int)gridDim.x < nt) {
                const BatchTile cur = next;
                if (k + 2 * (int)gridDim.x < nt) next = list[k + 2 * gridDim.x];
                fill(cur, buf ^ 1);
            }
            pair_tile_barrier<PS_::THREADS>();
        }
    } else {
        if constexpr (PS_::MBAR) {
            int i = 0;
            for (int k = blockIdx.x; k < nt; k += gridDim.x, i++) {
                const int buf = i & 1;
                if (!mbar_wait(&bar_full[buf], (i >> 1) & 1)) {
                    slots[list[k].slot].flags[BF_STATE] = SLOT_ABORTED;  // handover lost
                    return;
                }
                const PairTileMeta tm = meta[buf];
                if (tm.active)
                    pair_consume<M, V>(Ab + (size_t)buf * ROWS * PS, Wb + buf * P * WS, t,
                                       tm.row0, tm.D2, tm.Y, tm.real != 0);
                mbar_arrive(&bar_empty[buf]);
            }
            return;
        }
        pair_tile_barrier<PS_::THREADS>();
        int buf = 0;
        for (int k = blockIdx.x; k < nt; k += gridDim.x, buf ^= 1) {
            const PairTileMeta tm = meta[buf];
            if (tm.active)
                pair_consume<M, V>(Ab + (size_t)buf * ROWS * PS, Wb + buf * P * WS, t, tm.row0,
                                   tm.D2, tm.Y, tm.real != 0);
            pair_tile_barrier<PS_::THREADS>();
        }
    }
}

// Lanczos H.C of step iteration `iter`, gathered back from Y:
//   out = H V[iter] - beta_{iter-1} V[iter-1]   (iter > 0)
//   out = H V[0]                                (iter == 0, kBatchMonIter)
// Slots that stopped, or whose Lanczos recurrence broke down in this step,
// are skipped (multiconfig_lanczos.c:70-71); the monitor's launch
// (kBatchMonIter) takes only the slots whose eigen residual is due.
template <int M>
__global__ void __launch_bounds__(kBatchHcRows)
    bhcp_g_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                  const int* __restrict__ cnt, int iter) {
    if (iter == kBatchMonIter && batch_mon(cnt)[M] == 0) return;
    const int nt = batch_cnt(cnt, LIST_HG, M);
    const BatchTile* list = tiles + batch_off(cnt, LIST_HG, M);
    for (int k = blockIdx.x; k < nt; k += gridDim.x) {
        const BatchTile tl = list[k];
        const BatchSlot& S = slots[tl.slot];
        if (!bt_hc_active(S, iter)) continue;
        const uint32_t nc = S.nc;
        const uint32_t row = tl.idx + threadIdx.x;
        if (row >= nc) continue;
        double2 acc = pair_gather_back<M>(S.sp, S.sp.pair_y, row);
        if (iter > 0) {
            const double2 pv = S.V[(size_t)(iter - 1) * nc + row];
            const double b = S.scal[BS_OFFD + iter - 1].x;
            acc.x -= b * pv.x;
            acc.y -= b * pv.y;
        }
        S.out[row] = acc;
    }
}

// rho2 Gram partial of slice `idx` of a slot: its gk[2] consecutive row
// tiles of the (N-2)-boson space, summed into gpart (gram_tmpl.cuh building
// blocks); rho1 follows from rho2 in bgram_finalize_kernel
template <int M>
__global__ void __launch_bounds__(kGramThreads, 2)
    bgram_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                 const int* __restrict__ cnt) {
    constexpr int R = 2;
    using GS = GramShape<M, R>;
    extern __shared__ double2 As[];
    const int nt = batch_cnt(cnt, LIST_G2, M);
    const BatchTile* list = tiles + batch_off(cnt, LIST_G2, M);
    const GramRole<M, R> role(threadIdx.x);
    for (int k = blockIdx.x; k < nt; k += gridDim.x) {
        const BatchTile tl = list[k];
        const BatchSlot& S = slots[tl.slot];
        if (S.flags[BF_STATE] != SLOT_RUNNING) continue;  // block-uniform
        const uint32_t Dp = S.sp.dim2;
        const uint32_t ntr = (Dp + GS::ROWS - 1) / GS::ROWS;
        const uint32_t t0 = tl.idx * (uint32_t)S.gk[R];
        const uint32_t t1 = min(t0 + (uint32_t)S.gk[R], ntr);
        double2 acc[GS::RT][GS::RT];
#pragma unroll
        for (int a = 0; a < GS::RT; a++)
#pragma unroll
            for (int b = 0; b < GS::RT; b++) acc[a][b] = make_double2(0.0, 0.0);
        for (uint32_t tr = t0; tr < t1; tr++) {
            gram_gather<M, R>(S.sp, Dp, S.V, tr, As, threadIdx.x);
            __syncthreads();
            gram_accumulate<M, R>(As, role, acc);
            __syncthreads();
        }
        gram_store<M, R>(role, acc, As, S.gpart + (size_t)tl.idx * gram_entries(M, 2));
    }
}

// rho2 of every running slot of orbital count M: fixed-order sum of the
// slot's slices and the reference's symmetric fill (gram_fill); then rho1
// from rho2 (rho1_from_rho2: every batched job has two or more bosons)
template <int M>
__global__ void __launch_bounds__(kBatchVecThreads)
    bgram_finalize_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                          const int* __restrict__ nlist) {
    if ((int)blockIdx.x >= *nlist) return;
    const BatchSlot& S = slots[list[blockIdx.x]];
    if (S.M != M || S.flags[BF_STATE] != SLOT_RUNNING) return;  // block-uniform
    constexpr int ENT2 = gram_entries(M, 2);
    const int ns = S.gs[2];
    for (int e = threadIdx.x; e < ENT2; e += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int q = 0; q < ns; q++) v = cadd(v, S.gpart[(size_t)q * ENT2 + e]);
        gram_fill<M>(2, e, v, S.rho1, S.rho2);
    }
    __syncthreads();  // the block's rho2 stores are visible to the whole block
    rho1_from_rho2<M>(S.sp.N, S.rho2, S.rho1, threadIdx.x, blockDim.x);
}

template <int M, int V>
constexpr size_t batch_y_smem() {
    using PS_ = PairHcShape<M, V>;
    return (2 * (size_t)PS_::P * PS_::WS + 2 * (size_t)PS_::ROWS * PS_::PS) * sizeof(double2) +
           kPairTabBytes;
}

// the batched tile lists fix the rows per tile: variants 0, 2 and 3
__host__ __device__ constexpr bool batch_variant_ok(int M, int V) {
    return V == 3 || ((V == 0 || V == 2) && pair_variant_ok(M, V));
}

template <int M, int V>
int batch_y_attr() {
    static_assert(batch_y_smem<M, V>() <= 227 * 1024, "shared memory of one block (227 KB)");
    if constexpr (batch_variant_ok(M, V))
        MCTDHB_CUDA_TRY(cudaFuncSetAttribute(bhcp_y_kernel<M, V>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)batch_y_smem<M, V>()));
    return 0;
}

template <int M>
int batch_prepare() {
    static std::atomic<uint64_t> done{0};
    return set_attributes_once(done, []() -> int {
        if (batch_y_attr<M, 0>() || batch_y_attr<M, 2>() || batch_y_attr<M, 3>()) return -1;
        MCTDHB_CUDA_TRY(cudaFuncSetAttribute(bgram_kernel<M>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             gram_smem(M, 2)));
        return 0;
    });
}

template <int M, int V>
int bhcp_y_launch(const BatchSlot* slots, const BatchTile* hy, const int* cnt, int iter,
                  cudaStream_t st) {
    if constexpr (!batch_variant_ok(M, V)) {
        set_error("batched pair contraction variant %d does not exist for %d orbitals", V, M);
        return -1;
    } else {
        bhcp_y_kernel<M, V><<<num_sms(), PairHcShape<M, V>::THREADS, batch_y_smem<M, V>(), st>>>(
            slots, hy, cnt, iter);
        MCTDHB_CUDA_TRY(cudaGetLastError());
        return 0;
    }
}

template <int M>
int hcp_batch_launch(const BatchSlot* slots, const BatchTile* hy, const BatchTile* hg,
                     const int* cnt, int iter, int parts, int variant, cudaStream_t st) {
    if (parts & 1) {
        const int rc = variant == 3   ? bhcp_y_launch<M, 3>(slots, hy, cnt, iter, st)
                       : variant == 2 ? bhcp_y_launch<M, 2>(slots, hy, cnt, iter, st)
                                      : bhcp_y_launch<M, 0>(slots, hy, cnt, iter, st);
        if (rc) return -1;
    }
    if (parts & 2) {
        bhcp_g_kernel<M><<<num_sms() * 8, kBatchHcRows, 0, st>>>(slots, hg, cnt, iter);
        MCTDHB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

template <int M>
int gram_batch_launch(const BatchSlot* slots, const BatchTile* g2, const int* cnt,
                      const int* list, const int* nlist, int nblocks, cudaStream_t st) {
    bgram_kernel<M><<<num_sms() * 2, kGramThreads, gram_smem(M, 2), st>>>(slots, g2, cnt);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    bgram_finalize_kernel<M><<<std::max(nblocks, 1), kBatchVecThreads, 0, st>>>(slots, list, nlist);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mctdhb
