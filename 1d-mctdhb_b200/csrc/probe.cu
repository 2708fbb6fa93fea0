// probe.cu -- throughput probe of the FP64 tensor cores, the roofline
// denominator of the pair contraction (pairhc_tmpl.cuh): every warp runs
// `iters` rounds of eight independent mma.sync m8n8k4 f64 chains (enough
// in flight to cover the MMA latency).  FLOPs of one launch:
// blocks x 8 warps x iters x 8 x 256 x 2.
#include <cuda_runtime.h>

#include "common.cuh"
#include "pairhc_tmpl.cuh"

namespace mctdhb {

__global__ void __launch_bounds__(256) fp64_mma_probe_kernel(int iters, double* __restrict__ out) {
    double d[8][2];
#pragma unroll
    for (int c = 0; c < 8; c++) d[c][0] = d[c][1] = 0.0;
    const double a = 1e-3 * (threadIdx.x + 1), b = 1e-3 * (blockIdx.x + 1);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < 8; c++) dmma84(d[c][0], d[c][1], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 8; c++) s += d[c][0] + d[c][1];
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
