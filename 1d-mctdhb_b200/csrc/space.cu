// space.cu -- Fock-space runtime: rank tables, and the reference's index
// tables built on the GPU, bit-exact with space.c:
//   hash table      (get_hash_table,          space.c:181-199)
//   single map      (get_single_jump_map,     space.c:202-251)
//   double maps     (get_double_diffjump_map / get_double_equaljump_map,
//                    space.c:255-451): per-row chunk counts, an exclusive
//                    scan for the strides, then the M^2-entry chunks.
// None of these tables is read by the H.C / density kernels (they rank on
// the fly); they exist for drop-in callers that read the reference's
// MultiConfiguration fields.
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "moves.cuh"

namespace mctdhb {

static uint64_t binom_u64(uint64_t n, uint64_t k) {
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (uint64_t i = 1; i <= k; i++) {
        r = r * (n - k + i) / i;
        if (r > (unsigned __int128)UINT64_MAX) return UINT64_MAX;
    }
    return (uint64_t)r;
}

uint64_t fock_dimension(int npar, int norb) {
    if (norb < 1) return 0;
    return binom_u64((uint64_t)npar + norb - 1, (uint64_t)norb - 1);
}

int space_init(SpaceCtx& s, int N, int M) {
    if (N < 1 || M < 1 || M > kMaxOrb || N > 10000) {
        set_error("invalid Fock space: %d particles, %d orbitals (need 1..10000, 1..%d)", N, M,
                  kMaxOrb);
        return -1;
    }
    const uint64_t dim = fock_dimension(N, M);
    if (dim == 0 || dim >= (uint64_t)UINT32_MAX) {
        set_error("Fock space of %d particles in %d orbitals has %llu configurations; "
                  "32-bit configuration indices (as in the reference) are exceeded",
                  N, M, (unsigned long long)dim);
        return -1;
    }
    s.N = N;
    s.M = M;
    s.dim = (uint32_t)dim;
    const int rows = M > 1 ? M - 1 : 1;
    std::vector<uint32_t> T((size_t)rows * (N + 1), 0);
    for (int m = 0; m < M - 1; m++)
        for (int L = 0; L <= N; L++) T[(size_t)m * (N + 1) + L] = (uint32_t)binom_u64(L + m, m + 1);
    std::vector<double> sq(N + 3);
    for (int x = 0; x < N + 3; x++) sq[x] = std::sqrt((double)x);
    MCTDHB_CUDA_TRY(cudaMalloc(&s.d_T, T.size() * sizeof(uint32_t)));
    MCTDHB_CUDA_TRY(cudaMemcpy(s.d_T, T.data(), T.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    MCTDHB_CUDA_TRY(cudaMalloc(&s.d_sq, sq.size() * sizeof(double)));
    MCTDHB_CUDA_TRY(cudaMemcpy(s.d_sq, sq.data(), sq.size() * sizeof(double), cudaMemcpyHostToDevice));
    s.view.N = N;
    s.view.M = M;
    s.view.dim = s.dim;
    s.view.T = s.d_T;
    s.view.sq = s.d_sq;
    // H.C coefficient table
    MCTDHB_CUDA_TRY(cudaMalloc(&s.d_tab, (size_t)hc_table_size(M) * sizeof(double2)));
    // density descriptors + partials
    const int E = dens_descriptors(M, nullptr);
    std::vector<int> desc((size_t)5 * E);
    dens_descriptors(M, desc.data());
    MCTDHB_CUDA_TRY(cudaMalloc(&s.d_dens_desc, desc.size() * sizeof(int)));
    MCTDHB_CUDA_TRY(cudaMemcpy(s.d_dens_desc, desc.data(), desc.size() * sizeof(int),
                               cudaMemcpyHostToDevice));
    MCTDHB_CUDA_TRY(cudaMalloc(&s.d_dens_part, dens_partial_elems(s.view) * sizeof(double2)));
    if (dens_prepare(s.view, nullptr, nullptr, nullptr)) return -1;
    // pair-space H.C: the pair matrix and its D(N-2, M) x P scratch; when the
    // scratch cannot be had the space keeps the per-row kernel
    if (hcp_eligible(N, M)) {
        const size_t P = (size_t)M * (M + 1) / 2;
        double2 *w = nullptr, *y = nullptr;
        if (cudaMalloc(&w, (P * P + 1) * sizeof(double2)) == cudaSuccess &&
            cudaMalloc(&y, hcp_scratch_bytes(N, M)) == cudaSuccess && hcp_prepare(M) == 0) {
            s.view.dim2 = (uint32_t)fock_dimension(N - 2, M);
            s.view.pair_w = w;
            s.view.pair_y = y;
        } else {
            cudaGetLastError();  // clear the allocation failure
            cudaFree(w);
            cudaFree(y);
        }
    }
    return 0;
}

void space_release(SpaceCtx& s) {
    cudaFree(s.d_T);
    cudaFree(s.d_sq);
    cudaFree(s.d_tab);
    cudaFree(s.d_dens_desc);
    cudaFree(s.d_dens_part);
    cudaFree(s.view.pair_w);
    cudaFree(s.view.pair_y);
    s = SpaceCtx();
}

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------
__device__ __forceinline__ void unrank_generic(const SpaceView& sp, uint32_t row, int* n, int* L) {
    const int M = sp.M, N = sp.N;
    uint32_t S = sp.dim - 1u - row;
    int Lnext = N;
    for (int m = M - 2; m >= 0; m--) {
        const uint32_t* Tm = sp.T + m * (N + 1);
        int lo = 0, hi = Lnext;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (Tm[mid] <= S)
                lo = mid;
            else
                hi = mid - 1;
        }
        S -= Tm[lo];
        n[m + 1] = Lnext - lo;
        L[m] = lo;
        Lnext = lo;
    }
    n[0] = Lnext;
}

__device__ __forceinline__ uint32_t move_rank(const SpaceView& sp, uint32_t row, const int* L,
                                              int k, int s, int q, int l) {
    uint32_t d = 0;
    for (int m = 0; m < sp.M - 1; m++) {
        int dl = (q >= 0 && m >= q) + (l >= 0 && m >= l) - (k >= 0 && m >= k) - (s >= 0 && m >= s);
        if (dl != 0) {
            const uint32_t* Tm = sp.T + m * (sp.N + 1);
            d += Tm[L[m] + dl] - Tm[L[m]];
        }
    }
    return row - d;
}

__global__ void hash_table_kernel(SpaceView sp, uint16_t* __restrict__ ht) {
    int n[kMaxOrb], L[kMaxOrb];
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < sp.dim;
         row += gridDim.x * blockDim.x) {
        unrank_generic(sp, row, n, L);
        for (int m = 0; m < sp.M; m++) ht[(size_t)row * sp.M + m] = (uint16_t)n[m];
    }
}

// map[i + k dim + l M dim]: coalesced over i for every (k, l)
__global__ void single_map_kernel(SpaceView sp, uint32_t* __restrict__ map) {
    int n[kMaxOrb], L[kMaxOrb];
    const size_t dim = sp.dim;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < sp.dim;
         row += gridDim.x * blockDim.x) {
        unrank_generic(sp, row, n, L);
        for (int k = 0; k < sp.M; k++)
            for (int l = 0; l < sp.M; l++) {
                uint32_t v = 0;
                if (n[k] > 0) v = (k == l) ? row : move_rank(sp, row, L, k, -1, l, -1);
                map[row + k * dim + (size_t)l * sp.M * dim] = v;
            }
    }
}

__global__ void chunk_count_kernel(SpaceView sp, int diff, uint64_t* __restrict__ cnt) {
    int n[kMaxOrb], L[kMaxOrb];
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < sp.dim;
         row += gridDim.x * blockDim.x) {
        unrank_generic(sp, row, n, L);
        uint64_t c = 0;
        if (diff) {
            int nz = 0;
            for (int k = 0; k < sp.M; k++) nz += n[k] > 0;
            c = (uint64_t)nz * (nz - 1) / 2;
        } else {
            for (int k = 0; k < sp.M; k++) c += n[k] > 1;
        }
        cnt[row] = c;
    }
}

// chunk c of row i covers map[off[i] + c M^2 + l + q M]  (off = chunks * M^2)
__global__ void double_map_kernel(SpaceView sp, int diff, const uint64_t* __restrict__ off,
                                  uint32_t* __restrict__ map) {
    int n[kMaxOrb], L[kMaxOrb];
    const int M = sp.M;
    const uint64_t M2 = (uint64_t)M * M;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < sp.dim;
         row += gridDim.x * blockDim.x) {
        unrank_generic(sp, row, n, L);
        uint64_t base = off[row] * M2;
        for (int k = 0; k < M; k++) {
            if (diff) {
                if (n[k] < 1) continue;
                for (int s = k + 1; s < M; s++) {
                    if (n[s] < 1) continue;
                    for (int q = 0; q < M; q++)
                        for (int l = 0; l < M; l++)
                            map[base + l + (uint64_t)q * M] = move_rank(sp, row, L, k, s, l, q);
                    base += M2;
                }
            } else {
                if (n[k] < 2) continue;
                for (int q = 0; q < M; q++)
                    for (int l = 0; l < M; l++)
                        map[base + l + (uint64_t)q * M] = move_rank(sp, row, L, k, k, l, q);
                base += M2;
            }
        }
    }
}

static int table_grid(uint32_t dim) {
    uint64_t need = ((uint64_t)dim + 255) / 256;
    uint64_t cap = (uint64_t)num_sms() * 16;
    return (int)(need < cap ? (need ? need : 1) : cap);
}

int build_hash_table(const SpaceView& sp, uint16_t* d_ht, cudaStream_t st) {
    hash_table_kernel<<<table_grid(sp.dim), 256, 0, st>>>(sp, d_ht);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int build_single_map(const SpaceView& sp, uint32_t* d_map, cudaStream_t st) {
    single_map_kernel<<<table_grid(sp.dim), 256, 0, st>>>(sp, d_map);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int count_double_chunks(const SpaceView& sp, int diff, uint64_t* d_cnt, cudaStream_t st) {
    chunk_count_kernel<<<table_grid(sp.dim), 256, 0, st>>>(sp, diff, d_cnt);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int build_double_map(const SpaceView& sp, int diff, const uint64_t* d_off, uint32_t* d_map,
                     cudaStream_t st) {
    double_map_kernel<<<table_grid(sp.dim), 256, 0, st>>>(sp, diff, d_off, d_map);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

__global__ void scale_offsets_kernel(uint64_t* off, uint64_t n, uint64_t f) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        off[i] *= f;
}

int scale_offsets(uint64_t* d_off, uint64_t n, uint64_t factor, cudaStream_t st) {
    scale_offsets_kernel<<<table_grid((uint32_t)n), 256, 0, st>>>(d_off, n, factor);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// exclusive scan of uint64 (three-phase: tile sums, scan of sums, apply)
// ---------------------------------------------------------------------------
constexpr int kScanTile = 1024;

__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* total) {
    __shared__ uint64_t warp_sums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        uint64_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    const uint64_t before = (w > 0 ? warp_sums[w - 1] : 0) + x - v;
    if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__global__ void scan_tiles_kernel(uint64_t* data, uint64_t n, uint64_t* tile_sums) {
    const uint64_t i = (uint64_t)blockIdx.x * kScanTile + threadIdx.x;
    uint64_t v = i < n ? data[i] : 0;
    uint64_t tot;
    uint64_t ex = block_exclusive_scan(v, &tot);
    if (i < n) data[i] = ex;
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// single block, sequential over chunks of 1024 tile sums
__global__ void scan_sums_kernel(uint64_t* sums, uint64_t ntiles, uint64_t* total) {
    uint64_t carry = 0;
    for (uint64_t base = 0; base < ntiles; base += kScanTile) {
        const uint64_t i = base + threadIdx.x;
        uint64_t v = i < ntiles ? sums[i] : 0;
        uint64_t tot;
        uint64_t ex = block_exclusive_scan(v, &tot);
        if (i < ntiles) sums[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_apply_kernel(uint64_t* data, uint64_t n, const uint64_t* tile_offsets) {
    const uint64_t i = (uint64_t)blockIdx.x * kScanTile + threadIdx.x;
    if (i < n) data[i] += tile_offsets[blockIdx.x];
}

size_t exclusive_scan_tmp_bytes(uint64_t n) {
    return ((n + kScanTile - 1) / kScanTile + 1) * sizeof(uint64_t);
}

int exclusive_scan_u64(uint64_t* d_data, uint64_t n, uint64_t* d_total, void* d_tmp,
                       size_t tmp_bytes, cudaStream_t st) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (tmp_bytes < exclusive_scan_tmp_bytes(n)) {
        set_error("scan workspace too small");
        return -1;
    }
    uint64_t* sums = (uint64_t*)d_tmp;
    scan_tiles_kernel<<<(unsigned)ntiles, kScanTile, 0, st>>>(d_data, n, sums);
    scan_sums_kernel<<<1, kScanTile, 0, st>>>(sums, ntiles, d_total);
    scan_apply_kernel<<<(unsigned)ntiles, kScanTile, 0, st>>>(d_data, n, sums);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mctdhb
