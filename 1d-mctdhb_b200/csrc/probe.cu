// probe.cu -- throughput probe of the FP64 tensor cores, the roofline
// denominator of the pair contraction (pairhc_tmpl.cuh): every warp runs
// `iters` rounds of four independent mma.sync m16n8k8 f64 chains, the
// instruction of the contraction (enough in flight to cover the MMA
// latency).  FLOPs of one launch: blocks x 8 warps x iters x 4 x 1024 x 2.
#include <cuda_runtime.h>

#include "common.cuh"
#include "pairhc_tmpl.cuh"

namespace mctdhb {

__global__ void __launch_bounds__(256) fp64_mma_probe_kernel(int iters, double* __restrict__ out) {
    double d[4][4];
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
        for (int j = 0; j < 4; j++) d[c][j] = 0.0;
    const double a = 1e-3 * (threadIdx.x + 1), b = 1e-3 * (blockIdx.x + 1);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < 4; c++) dmma1688(d[c], a, 2.0 * a, 3.0 * a, 4.0 * a, b, 2.0 * b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 4; c++) s += d[c][0] + d[c][1] + d[c][2] + d[c][3];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace mctdhb

using namespace mctdhb;

extern "C" int mctdhb_fp64_mma_probe(int blocks, int iters, void* d_out, void* stream) {
    if (blocks < 1 || iters < 1 || !d_out) {
        set_error("mctdhb_fp64_mma_probe: invalid argument");
        return -1;
    }
    fp64_mma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, (double*)d_out);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}
