// kernels.h -- internal launch interface between the kernel files and the
// host runtime (space.cu, capi.cu).  Not part of the public C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace mctdhb {

// Optional fused epilogue of the H.C kernel, used by the Lanczos recurrence
// (multiconfig_lanczos.c:78-82): out = H v - beta * prev.  `flag` != 0 turns
// the launch into a no-op (a breakdown detected on the device earlier in the
// same step).
struct HcEpilogue {
    const int* flag = nullptr;
    const double2* prev = nullptr;
    const double* beta = nullptr;
};

// Deterministic block reduction of one complex value per thread; thread 0
// writes the block's sum to out[blockIdx.x].  Every thread must call it.
__device__ __forceinline__ void block_reduce_store(double2 v, double2* out) {
    __shared__ double2 red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 s = red[0];
        for (int i = 1; i < nw; i++) {
            s.x += red[i].x;
            s.y += red[i].y;
        }
        out[blockIdx.x] = s;
    }
}

// per-M register-resident kernels (hc_tmpl.cuh / dens_tmpl.cuh, explicit
// instantiations in hc_m*.cu / dens_m*.cu); H.C has kHcVariants launch
// variants (block size x barrier interval) chosen by the autotuner
constexpr int kHcVariants = 5;
constexpr int kDensVariants = 4;
template <int M>
int hc_launch_tmpl(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
                   const HcEpilogue& ep, int variant, cudaStream_t st);
template <int M>
int dens_launch_tmpl(const SpaceView& sp, const double2* C, double2* partial, int grid,
                     int variant, cudaStream_t st);
// rho1/rho2 as Gram matrices of the one- and two-boson-annihilated states
// (gram_tmpl.cuh): D2 = D(N-2, M), D1 = D(N-1, M) rows; partial holds
// gram_partial_elems(M, D2, D1) complex
template <int M>
int gram_apply_tmpl(const SpaceView& sp, uint32_t D2, uint32_t D1, const double2* C,
                    double2* partial, double2* rho1, double2* rho2, cudaStream_t st);
template <int M>
int gram_prepare_tmpl();

// Launch variants of the pair contraction (pairhc_tmpl.cuh, PairHcShape):
// 0 the default tile, 1 half the rows per tile (up to 6 orbitals), 2 the
// other output-tile grouping per pass (6 orbitals and more; below, it is
// the default grouping), 3 variant 0's tiles handed over through mbarriers
__host__ __device__ constexpr bool pair_variant_ok(int M, int V) {
    return V == 0 || V == 3 || (V == 1 && M * (M + 1) / 2 <= 21) ||
           (V == 2 && M * (M + 1) / 2 > 16);
}
constexpr int kPairVariants = 4;       // single-system kernel: 0, 1, 2, 3
constexpr int kBatchPairVariants = 4;  // batched kernel: 0, 2, 3

// H.C through the two-boson-annihilated space (pairhc_tmpl.cuh), M <= 8,
// N >= 2: launch attributes (before any capture) and the launches
// (parts & 1 the contraction, parts & 2 the gather-back) of a variant
template <int M>
int hcp_prepare_tmpl();
template <int M>
int hcp_apply_tmpl(const SpaceView& sp, const double2* C, double2* HC, const HcEpilogue& ep,
                   int variant, int parts, cudaStream_t st);

// tune.cu: autotuner.  The launch variant of `kernel` for (current device,
// N, M): the cached choice, else -- outside a stream capture -- each variant
// is timed on the caller's own data with `launch(v)` and the fastest kept;
// inside a capture (no timing possible) variant 0.  MCTDHB_TUNE_CACHE names
// an optional text file persisting choices across processes.
int tune_pick(const char* kernel, int N, int M, int nvariants, cudaStream_t st,
              int (*launch)(void* ctx, int v, cudaStream_t st), void* ctx);
int tune_lookup(const char* kernel, int N, int M);  // -1 when not tuned
void tune_set(const char* kernel, int N, int M, int variant);  // a caller's choice

// hamiltonian.cu
// the packed coefficient table of h, g (and the pair matrix when sp has one)
int hc_prep(const SpaceView& sp, const double2* d_hob, const double2* d_hint, double2* d_tab,
            cudaStream_t st);
// whether the pair-space H.C applies to (N, M), and its scratch size in bytes
bool hcp_eligible(int N, int M);
size_t hcp_scratch_bytes(int N, int M);
int hcp_prepare(int M);
int hc_variant(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
               const HcEpilogue& ep, cudaStream_t st);
int hc_apply(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
             const HcEpilogue& ep, cudaStream_t st);

// density.cu
int dens_grid(const SpaceView& sp);
size_t dens_partial_elems(const SpaceView& sp);  // doubles2 in the partial buffer
size_t gram_partial_elems(const SpaceView& sp);  // those of the Gram kernels (M <= 8)
int dens_apply(const SpaceView& sp, const double2* C, double2* partial, double2* rho1,
               double2* rho2, const int* d_desc, cudaStream_t st);
int dens_descriptors(int M, int* host_desc);  // returns count; desc = 5 ints/elem
// rho1/rho2 by the per-row pass (dens_tmpl.cuh, generic kernel) and its
// one-time launch attributes and tuned variant, before any capture
int dens_apply_rows(const SpaceView& sp, const double2* C, double2* partial, double2* rho1,
                    double2* rho2, const int* d_desc, cudaStream_t st);
int dens_prepare_rows(const SpaceView& sp, const double2* C, double2* partial, cudaStream_t st);
// set-up of dens_apply before any capture (launch attributes)
int dens_prepare(const SpaceView& sp, const double2* C, double2* partial, cudaStream_t st);
// kernels of density.cu also launched by noalloc.cu on its own scratch
__global__ void dens_generic_kernel(SpaceView sp, const double2* __restrict__ C,
                                    double2* __restrict__ partial, int EP);
__global__ void dens_finalize_kernel(int M, int E, int EP, int nblocks,
                                     const double2* __restrict__ partial,
                                     const int* __restrict__ desc, double2* __restrict__ rho1,
                                     double2* __restrict__ rho2);

// space.cu (map kernels)
int build_hash_table(const SpaceView& sp, uint16_t* d_ht, cudaStream_t st);
int build_single_map(const SpaceView& sp, uint32_t* d_map, cudaStream_t st);
int count_double_chunks(const SpaceView& sp, int diff, uint64_t* d_cnt, cudaStream_t st);
int exclusive_scan_u64(uint64_t* d_data, uint64_t n, uint64_t* d_total, void* d_tmp,
                       size_t tmp_bytes, cudaStream_t st);
size_t exclusive_scan_tmp_bytes(uint64_t n);
int build_double_map(const SpaceView& sp, int diff, const uint64_t* d_offsets,
                     uint32_t* d_map, cudaStream_t st);
int scale_offsets(uint64_t* d_off, uint64_t n, uint64_t factor, cudaStream_t st);

// lanczos.cu
struct LanczosDev;
}  // namespace mctdhb
