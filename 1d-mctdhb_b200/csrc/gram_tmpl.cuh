// gram_tmpl.cuh -- density matrices as Gram matrices of annihilated states,
// register-tiled for M <= 8 orbitals (explicit instantiations in dens_m*.cu).
//
// rho2[k,s,q,l] = <a+_k a+_s a_q a_l> and rho1[k][l] = <a+_k a_l>
// (density_matrices.c:9-443) are inner products of states with one or two
// bosons removed.  Inserting the identity of the (N-R)-boson space,
//     rho2[k,s,q,l] = sum_m conj(A_m(k,s)) A_m(q,l),  A_m(q,l) = <m|a_q a_l|C>,
//     rho1[k][l]    = sum_m conj(B_m(k))   B_m(l),    B_m(l)   = <m|a_l|C>,
// with m over the D(N-2, M) (resp. D(N-1, M)) configurations.  With two or
// more bosons only the rho2 Gram matrix is formed: rho1[k][l] =
// sum_s rho2[k,s,s,l] / (N-1) (rho1_from_rho2); the rho1 Gram pass runs for
// one boson, where rho2 vanishes.  Each A value
// is one scaled coefficient, A_m(q,l) = sqrt((m_q+1)(m_l+1+[q=l])) C[m+e_q+e_l]:
// at N=30, M=8 that is 6.7 M rows x 36 pairs = 242 M gathers (against the
// ~3 G coupling gathers of a per-row pass) and a 36 x 36 Hermitian Gram
// matrix, FP64-FMA bound instead of gather and shuffle bound.
//
// Ranking.  With the cumulative occupations L_x of m and the rank-weight
// table T_x(L) = C(L+x, x+1) (common.cuh), the rank of m + e_q + e_l in the
// N-boson space is
//     j = (D_N - D_{N-R}) + rank(m) - (U1[q] - U1[l]) - U2[l],
//     U_d[x] = sum_{y=x}^{M-2} (T_y(L_y + d) - T_y(L_y)),
// two subtractions per pair once U1, U2 are formed per row.
//
// Work split.  A block takes tiles of ROWS rows (as many as a 96 KB tile
// holds): every thread unranks its row and gathers its share of the row's
// A values into shared memory (gram.h gives the bank-spread layout); then
// thread groups accumulate the upper triangle of the P x P Gram matrix in
// RT x RT complex register tiles, each group over an interleaved subset of
// the tile's rows.  At the end the groups are added in a fixed order and the
// block writes one partial; gram_finalize_kernel adds the partials in block
// order.  The grid is a function of (N, M) only, so the result is
// deterministic and the same in any launch context.
#pragma once
#include "common.cuh"
#include "kernels.h"
#include "gram.h"
#include "movelist.cuh"

namespace mctdhb {

// pair p <-> (q, l), q <= l, in row-major order of the upper triangle
template <int M>
struct PairList {
    int q[M * (M + 1) / 2], l[M * (M + 1) / 2];
    constexpr PairList() : q{}, l{} {
        int p = 0;
        for (int a = 0; a < M; a++)
            for (int b = a; b < M; b++) {
                q[p] = a;
                l[p] = b;
                p++;
            }
    }
};
template <int M>
inline constexpr PairList<M> kPairs{};

// Unrank `row` of the space of Np bosons (dimension Dp) with the rank table
// of a space of N >= Np bosons (row stride N + 1): occupations n[] and the
// suffix sums U1, U2 of the rank offsets of adding one / two bosons.
// GEN: generic table loads (the table may be staged in shared memory).
template <int M, int R, bool GEN = false>
__device__ __forceinline__ void gram_unrank(const uint32_t* __restrict__ T, int N, int Np,
                                            uint32_t Dp, uint32_t row, int (&n)[M],
                                            uint32_t (&U1)[M], uint32_t (&U2)[M]) {
    uint32_t S = Dp - 1u - row;
    int Lnext = Np;
    int L[M > 1 ? M - 1 : 1];
#pragma unroll
    for (int x = M - 2; x >= 0; x--) {
        const uint32_t* Tx = T + x * (N + 1);
        const int lo = cns_level<GEN>(Tx, x, Lnext, S);
        S -= tab_ld<GEN>(Tx + lo);
        n[x + 1] = Lnext - lo;
        L[x] = lo;
        Lnext = lo;
    }
    n[0] = Lnext;
    U1[M - 1] = 0u;
    U2[M - 1] = 0u;
#pragma unroll
    for (int x = M - 2; x >= 0; x--) {
        const uint32_t* Tx = T + x * (N + 1);
        const uint32_t t0 = tab_ld<GEN>(Tx + L[x]);
        U1[x] = U1[x + 1] + (tab_ld<GEN>(Tx + L[x] + 1) - t0);
        if constexpr (R == 2) U2[x] = U2[x + 1] + (tab_ld<GEN>(Tx + L[x] + 2) - t0);
    }
}

// ---------------------------------------------------------------------------
// building blocks (shared with the batched engine, batch_tmpl.cuh)
// ---------------------------------------------------------------------------
template <int M, int R>
struct GramShape {
    static constexpr int P = gram_p(M, R);
    static constexpr int RT = gram_rt(P);
    static constexpr int NT = P / RT;
    static constexpr int NTILES = NT * (NT + 1) / 2;
    static constexpr int ENT = NTILES * RT * RT;
    static constexpr int ROWS = gram_rows(M, R);
    static constexpr int PS = gram_row_stride(M, R);
    static constexpr int PARTS = kGramThreads / ROWS;  // threads per row in the gather
    static constexpr int GROUPS = (kGramThreads / NTILES) < ROWS ? (kGramThreads / NTILES) : ROWS;
    static_assert(ENT <= ROWS * PS, "the group reduction reuses the A tile");
    // word of column p in a row of the A tile
    static constexpr int CS = gram_chunk_stride(RT);
    __host__ __device__ static constexpr int col(int p) { return (p / RT) * CS + p % RT; }
};

// Per-thread role in the Gram accumulation: group and upper-triangle tile.
template <int M, int R>
struct GramRole {
    int grp, tile, ti, tj;
    bool accum;
    __device__ explicit GramRole(int t) {
        using S = GramShape<M, R>;
        grp = t / S::NTILES;
        tile = t % S::NTILES;
        accum = grp < S::GROUPS;
        ti = 0;
        tj = 0;
        for (int a = 0, c = 0; a < S::NT; a++)
            for (int b = a; b < S::NT; b++, c++)
                if (c == tile) ti = a, tj = b;
    }
};

// Gather tile `tr` (ROWS rows of the (N-R)-boson space, Dp rows in all):
// thread t fills the values p = part, part + PARTS, ... of row t % ROWS.
template <int M, int R>
__device__ __forceinline__ void gram_gather(const SpaceView& sp, uint32_t Dp,
                                            const double2* __restrict__ C, uint32_t tr,
                                            double2* As, int t) {
    using S = GramShape<M, R>;
    constexpr int P = S::P, PS = S::PS, ROWS = S::ROWS, PARTS = S::PARTS;
    const int N = sp.N;
    const int r = t % ROWS, part = t / ROWS;  // part is warp-uniform (ROWS >= 64)
    const uint32_t row = tr * ROWS + r;
    const bool live = row < Dp;
    int n[M];
    uint32_t U1[M], U2[M];
    if (live) {
        gram_unrank<M, R>(sp.T, N, N - R, Dp, row, n, U1, U2);
    } else {
#pragma unroll
        for (int x = 0; x < M; x++) n[x] = 0, U1[x] = 0u, U2[x] = 0u;
    }
    const uint32_t j0 = sp.dim - Dp + row;
    // pairs: sqrt(n_x + 1), sqrt(n_x + 2) loaded once per orbital when a
    // thread takes at least half of a row's pairs
    constexpr bool HOIST = R == 2 && PARTS <= 2;
    double s1[HOIST ? M : 1], s2[HOIST ? M : 1];
    if constexpr (HOIST) {
#pragma unroll
        for (int x = 0; x < M; x++) {
            s1[x] = __ldg(sp.sq + n[x] + 1);
            s2[x] = __ldg(sp.sq + n[x] + 2);
        }
    }
    // coefficient gathers through L2 only (ld.global.cg), leaving L1 to the
    // rank and square-root tables
    static_for<P>([&](auto pi) {
        constexpr int p = decltype(pi)::value;
        if (p % PARTS == part) {
            double2 v = make_double2(0.0, 0.0);
            if (live) {
                if constexpr (R == 1) {
                    const uint32_t j = j0 - U1[p];
                    v = cscale(__ldcg(C + j), __ldg(sp.sq + n[p] + 1));
                } else {
                    constexpr int q = kPairs<M>.q[p], l = kPairs<M>.l[p];
                    const uint32_t j = j0 - (U1[q] - U1[l]) - U2[l];
                    double f;
                    if constexpr (HOIST)
                        f = q == l ? s1[q] * s2[q] : s1[q] * s1[l];
                    else if constexpr (q == l)
                        f = __ldg(sp.sq + n[q] + 1) * __ldg(sp.sq + n[q] + 2);
                    else
                        f = __ldg(sp.sq + n[q] + 1) * __ldg(sp.sq + n[l] + 1);
                    v = cscale(__ldcg(C + j), f);
                }
            }
            As[r * PS + S::col(p)] = v;
        }
    });
}

// acc += conj(A[:, ti-chunk])^T A[:, tj-chunk] over rows grp, grp + GROUPS, ...
template <int M, int R>
__device__ __forceinline__ void gram_accumulate(const double2* As, const GramRole<M, R>& role,
                                                double2 (&acc)[gram_rt(gram_p(M, R))]
                                                              [gram_rt(gram_p(M, R))]) {
    using S = GramShape<M, R>;
    constexpr int RT = S::RT, PS = S::PS;
    if (!role.accum) return;
    for (int r = role.grp; r < S::ROWS; r += S::GROUPS) {
        double2 a[RT], b[RT];
#pragma unroll
        for (int x = 0; x < RT; x++) {
            a[x] = As[r * PS + role.ti * S::CS + x];
            b[x] = As[r * PS + role.tj * S::CS + x];
        }
#pragma unroll
        for (int x = 0; x < RT; x++)
#pragma unroll
            for (int y = 0; y < RT; y++) acc[x][y] = cfma_conj(a[x], b[y], acc[x][y]);
    }
}

// groups added in order 0, 1, ... in shared memory `red` (ENT entries), then
// stored to out[0..ENT); every thread of the block calls it
template <int M, int R>
__device__ __forceinline__ void gram_store(const GramRole<M, R>& role,
                                           const double2 (&acc)[gram_rt(gram_p(M, R))]
                                                               [gram_rt(gram_p(M, R))],
                                           double2* red, double2* __restrict__ out) {
    using S = GramShape<M, R>;
    constexpr int RT = S::RT;
    for (int g = 0; g < S::GROUPS; g++) {
        if (role.accum && role.grp == g) {
#pragma unroll
            for (int x = 0; x < RT; x++)
#pragma unroll
                for (int y = 0; y < RT; y++) {
                    const int e = (role.tile * RT + x) * RT + y;
                    red[e] = g == 0 ? acc[x][y] : cadd(red[e], acc[x][y]);
                }
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < S::ENT; e += blockDim.x) out[e] = red[e];
    __syncthreads();
}

// Summed Gram entry `ee` (packed upper-triangle tiles) written to rho1
// (R = 1, M x M row-major) or rho2 (R = 2, M^4, (k,s,q,l) at k + sM + qM^2
// + lM^3): every ordering of a pair reads the same entry, the lower
// triangle is the conjugate of the upper, diagonal entries are real.
template <int M>
__device__ inline void gram_fill(int R, int ee, double2 v, double2* __restrict__ rho1,
                                 double2* __restrict__ rho2) {
    const int P = R == 2 ? gram_p(M, 2) : gram_p(M, 1);
    const int RT = gram_rt(P), NT = P / RT;
    const int tile = ee / (RT * RT), x = (ee / RT) % RT, y = ee % RT;
    int ti = 0, tj = 0;
    for (int a = 0, c = 0; a < NT; a++)
        for (int b = a; b < NT; b++, c++)
            if (c == tile) ti = a, tj = b;
    const int pa = ti * RT + x, pb = tj * RT + y;
    if (pa > pb) return;  // lower part of a diagonal tile: written by (pb, pa)
    if (pa == pb) v.y = 0.0;
    const double2 vc = make_double2(v.x, -v.y);
    if (R == 1) {
        rho1[pa * M + pb] = v;
        rho1[pb * M + pa] = vc;
        return;
    }
    int k = 0, s = 0, q = 0, l = 0;
    for (int a = 0, c = 0; a < M; a++)
        for (int b = a; b < M; b++, c++) {
            if (c == pa) k = a, s = b;
            if (c == pb) q = a, l = b;
        }
    constexpr int M2 = M * M, M3 = M2 * M;
    const int ks[2][2] = {{k, s}, {s, k}}, ql[2][2] = {{q, l}, {l, q}};
    for (int u = 0; u < (k == s ? 1 : 2); u++)
        for (int w = 0; w < (q == l ? 1 : 2); w++) {
            rho2[ks[u][0] + ks[u][1] * M + ql[w][0] * M2 + ql[w][1] * M3] = v;
            rho2[ql[w][0] + ql[w][1] * M + ks[u][0] * M2 + ks[u][1] * M3] = vc;
        }
}

// rho1 from the filled rho2 (N >= 2 bosons): sum_s a+_s a_s counts the N - 1
// bosons left after a_l, so rho1[k][l] = sum_s rho2[k,s,s,l] / (N - 1).  The
// sum runs over s in order; rho2[l,s,s,k] is the exact conjugate of
// rho2[k,s,s,l] (gram_fill), so rho1 comes out exactly Hermitian with a
// real diagonal.  Threads t, t + nt, ... take one entry each.  rho2 may have
// been written earlier in the same kernel (the batched finalize), so it is
// read through a plain pointer: no read-only (non-coherent) cache path.
template <int M>
__device__ __forceinline__ void rho1_from_rho2(int N, const double2* rho2, double2* rho1, int t,
                                               int nt) {
    constexpr int M2 = M * M, M3 = M2 * M;
    const double d = (double)(N - 1);
    for (int e = t; e < M2; e += nt) {
        const int k = e / M, l = e % M;
        double2 v = make_double2(0.0, 0.0);
#pragma unroll
        for (int s = 0; s < M; s++) v = cadd(v, rho2[k + s * M + s * M2 + l * M3]);
        rho1[e] = make_double2(v.x / d, v.y / d);
    }
}

// ---------------------------------------------------------------------------
// single-system kernels
// ---------------------------------------------------------------------------
// One block's share of the Gram matrix of the R-annihilated states of C:
// tiles blockIdx.x, blockIdx.x + gridDim.x, ...; partial: gridDim.x x ENT.
template <int M, int R>
__global__ void __launch_bounds__(kGramThreads, 2)
    gram_kernel(SpaceView sp, uint32_t Dp, const double2* __restrict__ C,
                double2* __restrict__ partial) {
    using S = GramShape<M, R>;
    extern __shared__ double2 As[];
    const GramRole<M, R> role(threadIdx.x);
    double2 acc[S::RT][S::RT];
#pragma unroll
    for (int a = 0; a < S::RT; a++)
#pragma unroll
        for (int b = 0; b < S::RT; b++) acc[a][b] = make_double2(0.0, 0.0);
    const uint32_t ntile_rows = (Dp + S::ROWS - 1) / S::ROWS;
    for (uint32_t tr = blockIdx.x; tr < ntile_rows; tr += gridDim.x) {
        gram_gather<M, R>(sp, Dp, C, tr, As, threadIdx.x);
        __syncthreads();
        gram_accumulate<M, R>(As, role, acc);
        __syncthreads();
    }
    gram_store<M, R>(role, acc, As, partial + (size_t)blockIdx.x * S::ENT);
}

// Sum of the block partials (block order) and the fill of rho1 / rho2; one
// thread per packed entry, rho2's first.  nent = ENT2 fills rho2 alone
// (rho1 then follows from rho2: gram_rho1_kernel).
template <int M>
__global__ void gram_finalize_kernel(int nent, int blocks2, int blocks1,
                                     const double2* __restrict__ part2,
                                     const double2* __restrict__ part1, double2* __restrict__ rho1,
                                     double2* __restrict__ rho2) {
    constexpr int ENT2 = gram_entries(M, 2), ENT1 = gram_entries(M, 1);
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nent) return;
    const bool two = e < ENT2;
    const int ee = two ? e : e - ENT2;
    const int nb = two ? blocks2 : blocks1, ent = two ? ENT2 : ENT1;
    const double2* part = two ? part2 : part1;
    double2 v = make_double2(0.0, 0.0);
    for (int b = 0; b < nb; b++) v = cadd(v, part[(size_t)b * ent + ee]);
    gram_fill<M>(two ? 2 : 1, ee, v, rho1, rho2);
}

template <int M>
__global__ void __launch_bounds__(64) gram_rho1_kernel(int N, const double2* __restrict__ rho2,
                                                      double2* __restrict__ rho1) {
    rho1_from_rho2<M>(N, rho2, rho1, threadIdx.x, blockDim.x);
}

template <int M, int R>
int gram_launch(const SpaceView& sp, uint32_t Dp, const double2* C, double2* partial, int blocks,
                cudaStream_t st) {
    if (blocks <= 0) return 0;
    gram_kernel<M, R><<<blocks, kGramThreads, gram_smem(M, R), st>>>(sp, Dp, C, partial);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

// launch attributes (dynamic shared memory beyond 48 KB), before any capture
template <int M>
int gram_prepare_tmpl() {
    static std::atomic<uint64_t> done{0};
    return set_attributes_once(done, []() -> int {
        MCTDHB_CUDA_TRY(cudaFuncSetAttribute(gram_kernel<M, 2>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             gram_smem(M, 2)));
        MCTDHB_CUDA_TRY(cudaFuncSetAttribute(gram_kernel<M, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             gram_smem(M, 1)));
        return 0;
    });
}

template <int M>
int gram_apply_tmpl(const SpaceView& sp, uint32_t D2, uint32_t D1, const double2* C,
                    double2* partial, double2* rho1, double2* rho2, cudaStream_t st) {
    // two or more bosons: rho1 from rho2 (rho1_from_rho2), no rho1 Gram pass
    const bool derive = sp.N >= 2;
    const int b2 = gram_blocks(M, 2, D2), b1 = derive ? 0 : gram_blocks(M, 1, D1);
    double2* part2 = partial;
    double2* part1 = partial + (size_t)b2 * gram_entries(M, 2);
    if (gram_launch<M, 2>(sp, D2, C, part2, b2, st)) return -1;
    if (gram_launch<M, 1>(sp, D1, C, part1, b1, st)) return -1;
    const int ent = gram_entries(M, 2) + (derive ? 0 : gram_entries(M, 1));
    gram_finalize_kernel<M><<<(ent + 127) / 128, 128, 0, st>>>(ent, b2, b1, part2, part1, rho1,
                                                               rho2);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    if (derive) {
        gram_rho1_kernel<M><<<1, 64, 0, st>>>(sp.N, rho2, rho1);
        MCTDHB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

}  // namespace mctdhb
