// batch_kernels.h -- launch interface of batch_kernels.cu (slot and vector
// kernels of the batched engine).  Tile kernels take a tile list and its
// device count; slot kernels a slot list and its device count.
#pragma once
#include "batch.h"

namespace mctdhb {

// mon: the count block's monitor flags, cleared at the start of a step
// (mode 0); nullptr for the admission set-up (mode 1)
__global__ void bt_orbital_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                                  const int* __restrict__ nlist, int mode, int* __restrict__ mon);
__global__ void bt_dot_kernel(const BatchSlot* __restrict__ slots,
                              const BatchTile* __restrict__ tiles, const int* __restrict__ ntiles,
                              int i);
// out -= alpha_i V[i] and the dots <V[k], out>, k <= i (one launch)
void bt_subdots(int i, int grid, cudaStream_t st, const BatchSlot* slots, const BatchTile* tiles,
                const int* ntiles);
__global__ void bt_orth_kernel(const BatchSlot* __restrict__ slots,
                               const BatchTile* __restrict__ tiles, const int* __restrict__ ntiles,
                               int i);
__global__ void bt_scale_kernel(const BatchSlot* __restrict__ slots,
                                const BatchTile* __restrict__ tiles,
                                const int* __restrict__ ntiles, int i);
__global__ void bt_combine_kernel(const BatchSlot* __restrict__ slots,
                                  const BatchTile* __restrict__ tiles,
                                  const int* __restrict__ ntiles);
__global__ void bt_norm2_kernel(const BatchSlot* __restrict__ slots,
                                const BatchTile* __restrict__ tiles,
                                const int* __restrict__ ntiles);
__global__ void bt_renorm_kernel(const BatchSlot* __restrict__ slots,
                                 const BatchTile* __restrict__ tiles,
                                 const int* __restrict__ ntiles);
__global__ void bt_reduce_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                                 const int* __restrict__ nlist, int nvals, int dst, int skip_break);
__global__ void bt_norm_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                               const int* __restrict__ nlist, int i);
__global__ void bt_small_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                                const int* __restrict__ nlist);
__global__ void bt_tail_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                               const int* __restrict__ nlist, int prologue, int* __restrict__ mon);
// the monitor's eigen residual: per-tile maxima, then the per-slot decision
__global__ void bt_resid_kernel(const BatchSlot* __restrict__ slots,
                                const BatchTile* __restrict__ tiles,
                                const int* __restrict__ ntiles);
__global__ void bt_monitor_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                                  const int* __restrict__ nlist);

}  // namespace mctdhb
