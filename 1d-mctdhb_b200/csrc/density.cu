// density.cu -- one- and two-body density matrices rho1 (M x M) and rho2
// (M^4) in one pass over the configurations (replaces set_onebody_dm and
// set_twobody_dm, density_matrices.c:9-443, which make one full pass over
// the coefficients per unique element).
//
// Every unique element of the reference (its rules 1-8 for rho2 plus rho1)
// is a sum over rows i of conj(C_i) C_j b(n_i) for one particle move; the
// kernel visits each row once, computes all its element contributions in
// registers (moves.cuh order) and reduces them across the warp in groups of
// eight with a transposed butterfly (4.5 shuffles per element instead of
// 20), accumulating into warp-private shared memory.  Blocks write partial
// sums; dens_finalize adds them in a fixed order and fills rho1/rho2 with
// the reference's symmetric pattern.  The result is deterministic for a
// given launch geometry, which depends only on the Fock-space size.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "gram.h"
#include "kernels.h"
#include "moves.cuh"

namespace mctdhb {

// generic M (<= 30): runtime loops, contributions reduced naively across the
// warp and accumulated into the warp's own slice of the global partial buffer
// (the element count grows as M^4/4, too large for shared memory).
// Correctness path for orbital counts without a register-resident kernel.
__global__ void __launch_bounds__(128)
    dens_generic_kernel(SpaceView sp, const double2* __restrict__ C, double2* __restrict__ partial,
                        int EP) {
    const int M = sp.M, N = sp.N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t gwarp = blockIdx.x * nwarps + warp;
    double2* wacc = partial + (size_t)gwarp * EP;
    for (int i = lane; i < EP; i += 32) wacc[i] = make_double2(0.0, 0.0);
    __syncwarp();
    const uint32_t twarps = gridDim.x * nwarps;
    for (uint32_t base = gwarp * 32u; base < sp.dim; base += twarps * 32u) {
        const uint32_t row = base + lane;
        const bool live = row < sp.dim;
        int n[kMaxOrb], L[kMaxOrb];
        for (int m = 0; m < M; m++) n[m] = 0, L[m] = 0;
        double2 ci = make_double2(0.0, 0.0);
        if (live) {
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
            ci = C[row];
        }
        auto target = [&](int k, int s, int q, int l) -> uint32_t {
            uint32_t d = 0;
            for (int m = 0; m < M - 1; m++) {
                int dl = (q >= 0 && m >= q) + (l >= 0 && m >= l) - (k >= 0 && m >= k) -
                         (s >= 0 && m >= s);
                if (dl != 0) {
                    const uint32_t* Tm = sp.T + m * (N + 1);
                    d += Tm[L[m] + dl] - Tm[L[m]];
                }
            }
            return row - d;
        };
        const double m2 = ci.x * ci.x + ci.y * ci.y;
        int e = 0;
        double2 t1 = make_double2(0.0, 0.0);
        for_each_density_element(M, [&](int kind, int k, int s, int q, int l) {
            double2 x = make_double2(0.0, 0.0);
            switch (kind) {
                case D_R1_DIAG: x.x = m2 * n[k]; break;
                case D_R2_KKKK: x.x = m2 * (n[k] * (n[k] - 1)); break;
                case D_R2_KSKS: x.x = m2 * (n[k] * n[s]); break;
                case D_R1_OFF:  // k -> l single move, l stored in s
                    t1 = make_double2(0.0, 0.0);
                    if (live && n[k] > 0) {
                        const uint32_t j = target(k, -1, s, -1);
                        t1 = cscale(cfma_conj(ci, C[j], make_double2(0.0, 0.0)),
                                    sp.sq[n[k]] * sp.sq[n[s] + 1]);
                    }
                    x = t1;
                    break;
                case D_R2_KKKL: x = cscale(t1, (double)(n[k] - 1)); break;
                case D_R2_KLLL: x = cscale(t1, (double)n[s]); break;
                case D_R2_KSSL: x = cscale(t1, (double)n[s]); break;
                default: {
                    const bool valid = (k == s) ? (n[k] >= 2) : (n[k] >= 1 && n[s] >= 1);
                    if (live && valid) {
                        const uint32_t j = target(k, s, q, l);
                        double sa = (k == s) ? sp.sq[n[k]] * sp.sq[n[k] - 1] : sp.sq[n[k]] * sp.sq[n[s]];
                        double sb = (q == l) ? sp.sq[n[q] + 1] * sp.sq[n[q] + 2]
                                             : sp.sq[n[q] + 1] * sp.sq[n[l] + 1];
                        x = cscale(cfma_conj(ci, C[j], make_double2(0.0, 0.0)), sa * sb);
                    }
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                x.x += __shfl_xor_sync(0xffffffffu, x.x, o);
                x.y += __shfl_xor_sync(0xffffffffu, x.y, o);
            }
            if (lane == 0) {
                wacc[e].x += x.x;
                wacc[e].y += x.y;
            }
            e++;
        });
    }
}

// one thread per element: fixed-order sum over block partials, then the
// reference's symmetric fill (density_matrices.c:33-50, 86-442)
__global__ void dens_finalize_kernel(int M, int E, int EP, int nblocks,
                                     const double2* __restrict__ partial,
                                     const int* __restrict__ desc, double2* __restrict__ rho1,
                                     double2* __restrict__ rho2) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double2 v = partial[e];
    for (int b = 1; b < nblocks; b++) {
        double2 p = partial[(size_t)b * EP + e];
        v.x += p.x;
        v.y += p.y;
    }
    const int kind = desc[5 * e], k = desc[5 * e + 1], s = desc[5 * e + 2], q = desc[5 * e + 3],
              l = desc[5 * e + 4];
    dens_fill(kind, k, s, q, l, v, M, rho1, rho2);
}

int dens_descriptors(int M, int* desc) {
    int e = 0;
    for_each_density_element(M, [&](int kind, int k, int s, int q, int l) {
        if (desc) {
            desc[5 * e] = kind;
            desc[5 * e + 1] = k;
            desc[5 * e + 2] = s;
            desc[5 * e + 3] = q;
            desc[5 * e + 4] = l;
        }
        e++;
    });
    return e;
}

static int dens_ep(int M) { return (dens_nelem(M) + 7) / 8 * 8; }

static bool dens_templated(int M) { return M >= 2 && M <= kMaxTemplOrb; }

// templated kernels: the number of virtual blocks (partial slices), a
// function of the space size only; generic kernel: its (small) grid
int dens_grid(const SpaceView& sp) {
    uint64_t need = ((uint64_t)sp.dim + 127) / 128;
    uint64_t cap = dens_templated(sp.M) ? 888 : 16;
    return (int)std::max<uint64_t>(1, std::min(need, cap));
}

// number of partial slices the finalize pass adds: blocks for the templated
// kernels, warps for the generic one
static int dens_slices(const SpaceView& sp) {
    return dens_templated(sp.M) ? dens_grid(sp) : dens_grid(sp) * 4;
}

// rows of the one- and two-boson-annihilated spaces (0 when empty)
static uint32_t annihilated_dim(const SpaceView& sp, int R) {
    return sp.N >= R ? (uint32_t)fock_dimension(sp.N - R, sp.M) : 0u;
}

size_t gram_partial_elems(const SpaceView& sp) {
    return (size_t)gram_blocks(sp.M, 2, annihilated_dim(sp, 2)) * gram_entries(sp.M, 2) +
           (size_t)gram_blocks(sp.M, 1, annihilated_dim(sp, 1)) * gram_entries(sp.M, 1);
}

size_t dens_partial_elems(const SpaceView& sp) {
    const size_t per_row = (size_t)dens_slices(sp) * dens_ep(sp.M);
    return dens_templated(sp.M) ? std::max(per_row, gram_partial_elems(sp)) : per_row;
}

// M <= 8: the Gram-matrix kernels (gram_tmpl.cuh)
static int gram_apply(const SpaceView& sp, const double2* C, double2* partial, double2* rho1,
                      double2* rho2, cudaStream_t st) {
    const uint32_t D2 = annihilated_dim(sp, 2), D1 = annihilated_dim(sp, 1);
    switch (sp.M) {
        case 2: return gram_apply_tmpl<2>(sp, D2, D1, C, partial, rho1, rho2, st);
        case 3: return gram_apply_tmpl<3>(sp, D2, D1, C, partial, rho1, rho2, st);
        case 4: return gram_apply_tmpl<4>(sp, D2, D1, C, partial, rho1, rho2, st);
        case 5: return gram_apply_tmpl<5>(sp, D2, D1, C, partial, rho1, rho2, st);
        case 6: return gram_apply_tmpl<6>(sp, D2, D1, C, partial, rho1, rho2, st);
        case 7: return gram_apply_tmpl<7>(sp, D2, D1, C, partial, rho1, rho2, st);
        case 8: return gram_apply_tmpl<8>(sp, D2, D1, C, partial, rho1, rho2, st);
    }
    set_error("gram_apply: %d orbitals outside 2..8", sp.M);
    return -1;
}

static int dens_launch_v(const SpaceView& sp, const double2* C, double2* partial, int grid,
                         int v, cudaStream_t st) {
    switch (sp.M) {
        case 2: return dens_launch_tmpl<2>(sp, C, partial, grid, v, st);
        case 3: return dens_launch_tmpl<3>(sp, C, partial, grid, v, st);
        case 4: return dens_launch_tmpl<4>(sp, C, partial, grid, v, st);
        case 5: return dens_launch_tmpl<5>(sp, C, partial, grid, v, st);
        case 6: return dens_launch_tmpl<6>(sp, C, partial, grid, v, st);
        case 7: return dens_launch_tmpl<7>(sp, C, partial, grid, v, st);
        case 8: return dens_launch_tmpl<8>(sp, C, partial, grid, v, st);
        default:
            dens_generic_kernel<<<grid, 128, 0, st>>>(sp, C, partial, dens_ep(sp.M));
            MCTDHB_CUDA_TRY(cudaGetLastError());
            return 0;
    }
}

// the variants differ only in the barrier interval (dens_tmpl.cuh): same
// blocks, same row order, same sums -- the tuner changes speed, not bits
namespace {
struct DensTuneCtx {
    const SpaceView* sp;
    const double2* C;
    double2* partial;
    int grid;
};
int dens_tune_launch(void* p, int v, cudaStream_t st) {
    auto* c = (DensTuneCtx*)p;
    return dens_launch_v(*c->sp, c->C, c->partial, c->grid, v, st);
}
int dens_variant(const SpaceView& sp, const double2* C, double2* partial, cudaStream_t st) {
    if (!dens_templated(sp.M) || sp.dim < 4096) return 0;
    DensTuneCtx ctx{&sp, C, partial, dens_grid(sp)};
    return tune_pick("dens", sp.N, sp.M, kDensVariants, st, dens_tune_launch, &ctx);
}
}  // namespace

int dens_prepare(const SpaceView& sp, const double2* C, double2* partial, cudaStream_t st) {
    (void)C;
    (void)partial;
    (void)st;
    switch (sp.M) {  // launch attributes of the Gram kernels (M <= 8)
        case 2: return gram_prepare_tmpl<2>();
        case 3: return gram_prepare_tmpl<3>();
        case 4: return gram_prepare_tmpl<4>();
        case 5: return gram_prepare_tmpl<5>();
        case 6: return gram_prepare_tmpl<6>();
        case 7: return gram_prepare_tmpl<7>();
        case 8: return gram_prepare_tmpl<8>();
    }
    return 0;
}

// Set-up of the per-row kernels (dens_tmpl.cuh): launch attributes and the
// tuned variant, before any capture.
int dens_prepare_rows(const SpaceView& sp, const double2* C, double2* partial, cudaStream_t st) {
    if (!dens_templated(sp.M)) return 0;
    for (int v = 0; v < kDensVariants; v++)
        if (dens_launch_v(sp, nullptr, nullptr, 0, v, st)) return -1;  // attributes only
    dens_variant(sp, C, partial, st);
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
}

int dens_apply(const SpaceView& sp, const double2* C, double2* partial, double2* rho1,
               double2* rho2, const int* d_desc, cudaStream_t st) {
    if (dens_templated(sp.M)) return gram_apply(sp, C, partial, rho1, rho2, st);
    return dens_apply_rows(sp, C, partial, rho1, rho2, d_desc, st);
}

// The per-row pass: every row's contributions to every unique element,
// reduced across the warp (dens_tmpl.cuh for M <= 8, the generic kernel
// beyond).
int dens_apply_rows(const SpaceView& sp, const double2* C, double2* partial, double2* rho1,
                    double2* rho2, const int* d_desc, cudaStream_t st) {
    const int grid = dens_grid(sp);
    const int M = sp.M;
    const int EP = dens_ep(M);
    const int v = dens_variant(sp, C, partial, st);
    if (int rc = dens_launch_v(sp, C, partial, grid, v, st)) return rc;
    const int E = dens_nelem(M);
    dens_finalize_kernel<<<(E + 127) / 128, 128, 0, st>>>(M, E, EP, dens_slices(sp), partial,
                                                          d_desc, rho1, rho2);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mctdhb
