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
constexpr int kGramMaxBlocks = 296;  // 2 x 148: fixed, so the sums depend on (N, M) only
constexpr int kGramSmemBudget = 96 * 1024;  // A tile bytes: two blocks per SM

// A tile layout: the RT-wide column chunks of a row sit an odd number of
// 16-byte words apart (RT for odd RT, RT + 1 for even RT) and so do the
// rows, so the chunk reads of a warp (different chunks of one row, or one
// column of consecutive rows) fall in different shared-memory banks
__host__ __device__ constexpr int gram_chunk_stride(int RT) { return RT % 2 ? RT : RT + 1; }
__host__ __device__ constexpr int gram_row_stride(int M, int R) {
    return (gram_nt(M, R) * gram_chunk_stride(gram_rt(gram_p(M, R)))) | 1;
}
// rows per tile: the largest of 256 / 128 / 64 whose tile fits the budget
__host__ __device__ constexpr int gram_rows(int M, int R) {
    return (256 * gram_row_stride(M, R) * 16 <= kGramSmemBudget) ? 256
           : (128 * gram_row_stride(M, R) * 16 <= kGramSmemBudget) ? 128 : 64;
}
__host__ __device__ constexpr int gram_smem(int M, int R) {
    return gram_rows(M, R) * gram_row_stride(M, R) * 16;
}

// blocks (= partial slices) for Dp rows: a function of (N, M) only
inline int gram_blocks_rows(uint32_t Dp, int rows) {
    const uint32_t need = (Dp + rows - 1) / rows;
    return (int)(need < (uint32_t)kGramMaxBlocks ? need : (uint32_t)kGramMaxBlocks);
}
inline int gram_blocks(int M, int R, uint32_t Dp) { return gram_blocks_rows(Dp, gram_rows(M, R)); }

}  // namespace mctdhb
