// gram.h -- sizes of the Gram-matrix density kernels (gram_tmpl.cuh), shared
// with the host code that allocates their partial sums.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mctdhb {

__host__ __device__ constexpr int gram_p(int M, int R) { return R == 1 ? M : M * (M + 1) / 2; }
__host__ __device__ constexpr int gram_rt(int P) {
    return (P % 4 == 0 && P >= 16) ? 4 : (P % 3 == 0 && P >= 9) ? 3 : (P % 2 == 0 && P >= 4) ? 2 : 1;
}
__host__ __device__ constexpr int gram_nt(int M, int R) { return gram_p(M, R) / gram_rt(gram_p(M, R)); }
__host__ __device__ constexpr int gram_ntiles(int M, int R) {
    return gram_nt(M, R) * (gram_nt(M, R) + 1) / 2;
}
// complex entries of one block partial: the upper-triangle tiles, RT x RT each
__host__ __device__ constexpr int gram_entries(int M, int R) {
    return gram_ntiles(M, R) * gram_rt(gram_p(M, R)) * gram_rt(gram_p(M, R));
}
constexpr int kGramThreads = 256;
constexpr int kGramRows = 64;        // rows of A per tile
constexpr int kGramMaxBlocks = 296;  // 2 x 148: fixed, so the sums depend on (N, M) only

// blocks (= partial slices) for Dp rows: a function of the space size only
inline int gram_blocks(uint32_t Dp) {
    const uint32_t need = (Dp + kGramRows - 1) / kGramRows;
    return (int)(need < (uint32_t)kGramMaxBlocks ? need : (uint32_t)kGramMaxBlocks);
}

}  // namespace mctdhb
