// noalloc.cu -- rho1 and rho2 without any device allocation
// (mctdhb_dev_density_matrices_noalloc, include/mctdhb_gpu.h).
//
// Some callers cannot let a library call cudaMalloc or cudaFree: a process
// whose device memory belongs to its own pool allocator (PyTorch's caching
// allocator, an arena reserved at start-up), or a loop that cannot afford
// the device-wide synchronisation cudaMalloc/cudaFree imply.  This entry
// point serves them.  It needs no mctdhb_space (whose creation allocates):
// the Fock space is named by (npar, norb), and the rank table, the sqrt
// table, the element descriptors and the per-block partial sums all live in
// one file-scope device array of kScratchBytes, which every GPU that loads
// the library holds until the process exits.
//
// The kernels are the ones mctdhb_dev_density_matrices runs: for norb <= 8
// the Gram-matrix kernels (gram_tmpl.cuh; their block count is a function
// of (npar, norb) alone, at most 296 partial sums of rho2 -- and of rho1 for
// one boson; with more, rho1 is rho2's partial trace -- so the result is the
// same as that entry point's, bit for bit), above that
// dens_generic_kernel and dens_finalize_kernel with the grid capped so the
// partial sums fit.  Only their scratch comes from here.  Layout of the
// array for one call (each part 256-byte aligned):
//   T     (norb-1) x (npar+1) uint32   rank table T_m(L) = C(L+m, m+1)
//   sq    npar+3 doubles               sqrt(0..npar+2)
//   desc  5 ints per density element  (kind, k, s, q, l; generic kernel)
//   part  partial sums                (Gram blocks, or slices x EP complex)
// Every call rewrites the parts it reads before the kernels read them; the
// kernels store (do not accumulate) their partial sums, or zero their own
// slices first, so nothing has to start at zero and nothing carries over
// from the previous call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/mctdhb_gpu.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "moves.cuh"

namespace mctdhb {
namespace {

constexpr size_t kScratchBytes = MCTDHB_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char* g_dev_scratch[kMaxDevices] = {};  // device address of g_scratch per device

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Once per device, with that device current: the device address of
// g_scratch.  In host code `g_scratch` only names the symbol.
int scratch_address(unsigned char** out) {
    int dev = 0;
    MCTDHB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("mctdhb_dev_density_matrices_noalloc: device %d beyond the %d supported", dev,
                  kMaxDevices);
        return -1;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_scratch[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            set_error("mctdhb_dev_density_matrices_noalloc: device address of the scratch array "
                      "on device %d: %s", dev, cudaGetErrorString(e));
            return -1;
        }
        g_dev_scratch[dev] = (unsigned char*)p;
    }
    *out = g_dev_scratch[dev];
    return 0;
}

// T_m(L) = C(L+m, m+1) by the multiplicative formula; with the space's
// dimension below 2^32 every intermediate C(n-k+i, i) (i <= k) is at most
// the final value, so the products stay below 2^32 * (npar + norb) and the
// divisions are exact.  Same integers as the host table of space_init.
__device__ uint32_t binom_u32(uint32_t n, uint32_t k) {
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    uint64_t r = 1;
    for (uint32_t i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return (uint32_t)r;
}

__global__ void noalloc_tables_kernel(int N, int M, uint32_t* __restrict__ T,
                                      double* __restrict__ sq, int* __restrict__ desc) {
    const int rows = M > 1 ? M - 1 : 1;
    const int nT = rows * (N + 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nT + N + 3;
         i += gridDim.x * blockDim.x) {
        if (i < nT) {
            const int m = i / (N + 1), L = i % (N + 1);
            T[i] = (M > 1) ? binom_u32((uint32_t)(L + m), (uint32_t)(m + 1)) : 0u;
        } else {
            sq[i - nT] = sqrt((double)(i - nT));
        }
    }
    // element descriptors: independent tasks (one per orbital, per pair
    // k<l and per source pair k<=s), so the list is written in parallel
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < dens_ntasks(M);
         t += gridDim.x * blockDim.x) {
        density_element_task(M, t, [&](int e, int kind, int k, int s, int q, int l) {
            desc[5 * e] = kind;
            desc[5 * e + 1] = k;
            desc[5 * e + 2] = s;
            desc[5 * e + 3] = q;
            desc[5 * e + 4] = l;
        });
    }
}

}  // namespace
}  // namespace mctdhb

using namespace mctdhb;

extern "C" int mctdhb_dev_density_matrices_noalloc(uint16_t npar, uint16_t norb,
                                                   const void* d_coef, void* d_rho1,
                                                   void* d_rho2, void* stream) {
    const char* fn = "mctdhb_dev_density_matrices_noalloc";
    if (!d_coef || !d_rho1 || !d_rho2) {
        set_error("%s: null argument", fn);
        return -1;
    }
    const int N = npar, M = norb;
    if (N < 1 || M < 1 || M > kMaxOrb || N > 10000) {
        set_error("%s: invalid Fock space: %d particles, %d orbitals (need 1..10000, 1..%d)", fn,
                  N, M, kMaxOrb);
        return -1;
    }
    const uint64_t dim = fock_dimension(N, M);
    if (dim == 0 || dim >= (uint64_t)UINT32_MAX) {
        set_error("%s: %d particles in %d orbitals exceed 32-bit configuration indices", fn, N,
                  M);
        return -1;
    }
    SpaceView sp{};
    sp.N = N;
    sp.M = M;
    sp.dim = (uint32_t)dim;
    const int rows = M > 1 ? M - 1 : 1;
    const int E = dens_nelem(M);
    const int EP = (E + 7) / 8 * 8;
    const bool templ = M >= 2 && M <= kMaxTemplOrb;
    const size_t off_sq = align256((size_t)rows * (N + 1) * sizeof(uint32_t));
    const size_t off_desc = off_sq + align256((size_t)(N + 3) * sizeof(double));
    const size_t off_part = off_desc + align256((size_t)5 * E * sizeof(int));
    const size_t slice = (size_t)EP * sizeof(double2);
    const size_t fit = off_part < kScratchBytes ? (kScratchBytes - off_part) / slice : 0;
    // generic kernel: one slice per warp, 4 per block
    const int grid = templ ? 1 : (int)std::min<size_t>((size_t)dens_grid(sp), fit / 4);
    const size_t need = templ ? off_part + gram_partial_elems(sp) * sizeof(double2)
                              : off_part + 4 * slice;
    if (grid < 1 || need > kScratchBytes) {
        set_error("%s: %d particles in %d orbitals need %zu bytes of scratch; the fixed scratch "
                  "array holds %zu (MCTDHB_NOALLOC_SCRATCH_BYTES)", fn, N, M, need,
                  kScratchBytes);
        return -1;
    }
    unsigned char* base = nullptr;
    if (scratch_address(&base)) return -1;
    uint32_t* T = (uint32_t*)base;
    double* sq = (double*)(base + off_sq);
    int* desc = (int*)(base + off_desc);
    double2* part = (double2*)(base + off_part);
    sp.T = T;
    sp.sq = sq;
    cudaStream_t st = (cudaStream_t)stream;

    const int ntab = std::max(rows * (N + 1) + N + 3, dens_ntasks(M));
    noalloc_tables_kernel<<<std::max(1, std::min(64, (ntab + 255) / 256)), 256, 0, st>>>(
        N, M, T, sq, desc);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    const double2* C = (const double2*)d_coef;
    if (templ) {
        // the Gram kernels (launch attributes set once per device, then the
        // two Gram passes and their fixed-order finalisation)
        if (dens_prepare(sp, C, part, st)) return -1;
        return dens_apply(sp, C, part, (double2*)d_rho1, (double2*)d_rho2, desc, st);
    }
    dens_generic_kernel<<<grid, 128, 0, st>>>(sp, C, part, EP);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    dens_finalize_kernel<<<(E + 127) / 128, 128, 0, st>>>(M, E, EP, grid * 4, part, desc,
                                                          (double2*)d_rho1, (double2*)d_rho2);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}
