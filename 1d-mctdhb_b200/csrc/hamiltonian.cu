// hamiltonian.cu -- the many-body Hamiltonian action HC = H C in complex128
// (replaces apply_hamiltonian, hamiltonian.c:7-406 of the reference).
//
// Design (B200): H.C is a gather-bound sparse action (~0.5 flop/byte), so
// the kernel is organised around the gathers, not around arithmetic:
//   * one thread per configuration (row); consecutive rows of a warp reach
//     consecutive neighbours for every move (the rank offset of a move is
//     constant over runs of rows that differ only in orbitals 0 and 1), so
//     each gather of the warp is a coalesced 16-byte-per-lane load;
//   * jump targets come from the rank offsets F[m][d] held in registers --
//     no map table is read (the reference's maps would cost 4 bytes of
//     index per 16 bytes of coefficient, and do not fit at N=30, M=8);
//   * every distinct neighbour is gathered once, with all rules that reach
//     it folded into one coefficient (moves.cuh);
//   * h_kl / g_ksql enter through a packed coefficient table staged in
//     shared memory (uniform broadcast loads);
//   * for M <= 8 the move loops are fully unrolled so occupations, rank
//     offsets and sqrt factors stay in registers;  larger M use a generic
//     runtime-loop kernel.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "moves.cuh"

namespace mctdhb {

// ---------------------------------------------------------------------------
// coefficient table (hob row-major M*M, hint M^4) -> packed table
// ---------------------------------------------------------------------------
__global__ void hc_prep_kernel(int M, const double2* __restrict__ hob,
                               const double2* __restrict__ hint,
                               double2* __restrict__ tab) {
    // one thread does the (tiny) enumeration in order; the table is a few KB
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    hc_pack_table(M, hob, hint, tab);
}

// ---------------------------------------------------------------------------
// generic kernel, any M <= 30 (runtime loops, local arrays)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    hc_generic_kernel(SpaceView sp, const double2* __restrict__ C, double2* __restrict__ HC,
                      const double2* __restrict__ tab, HcEpilogue ep) {
    if (ep.flag != nullptr && *ep.flag != 0) return;
    const int M = sp.M, N = sp.N;
    const int ND = hc_ndiag(M), NS = hc_nsingle(M);
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < sp.dim;
         row += gridDim.x * blockDim.x) {
        int n[kMaxOrb], L[kMaxOrb];
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
        auto rank_delta = [&](int k, int s, int q, int l) -> uint32_t {
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
        const double2 ci = C[row];
        double2 dg = make_double2(0.0, 0.0);
        for (int k = 0; k < M; k++) {
            dg = cadd(dg, cscale(tab[k], (double)n[k]));
            dg = cadd(dg, cscale(tab[M + k], (double)(n[k] * (n[k] - 1))));
        }
        int p = 2 * M;
        for (int k = 0; k < M; k++)
            for (int s = k + 1; s < M; s++, p++) dg = cadd(dg, cscale(tab[p], (double)(n[k] * n[s])));
        double2 acc = cmul(dg, ci);
        p = ND;
        for (int k = 0; k < M; k++)
            for (int l = 0; l < M; l++) {
                if (l == k) continue;
                if (n[k] > 0) {
                    const uint32_t j = rank_delta(k, -1, l, -1);
                    double2 c = tab[p];
                    for (int s = 0; s < M; s++) c = cadd(c, cscale(tab[p + 1 + s], (double)n[s]));
                    acc = cfma(cscale(c, sp.sq[n[k]] * sp.sq[n[l] + 1]), C[j], acc);
                }
                p += M + 1;
            }
        p = ND + NS;
        for (int k = 0; k < M; k++)
            for (int s = k; s < M; s++) {
                const bool valid = (k == s) ? (n[k] >= 2) : (n[k] >= 1 && n[s] >= 1);
                const double sa = valid ? ((k == s) ? sp.sq[n[k]] * sp.sq[n[k] - 1]
                                                    : sp.sq[n[k]] * sp.sq[n[s]])
                                        : 0.0;
                for (int q = 0; q < M; q++)
                    for (int l = q; l < M; l++) {
                        if (q == k || q == s || l == k || l == s) continue;
                        if (valid) {
                            const uint32_t j = rank_delta(k, s, q, l);
                            const double sb = (q == l) ? sp.sq[n[q] + 1] * sp.sq[n[q] + 2]
                                                       : sp.sq[n[q] + 1] * sp.sq[n[l] + 1];
                            acc = cfma(tab[p], cscale(C[j], sa * sb), acc);
                        }
                        p++;
                    }
            }
        if (ep.prev != nullptr) {
            const double2 pv = ep.prev[row];
            const double b = *ep.beta;
            acc.x -= b * pv.x;
            acc.y -= b * pv.y;
        }
        HC[row] = acc;
    }
}

// ---------------------------------------------------------------------------
// launchers and autotuner
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// pair matrix W of H = sum_{P,Q} W[P][Q] a+_P a_Q (pairhc_tmpl.cuh)
// ---------------------------------------------------------------------------
// one block; W[P*P].x = 1 when every entry is real (the contraction then
// runs two real products instead of three)
__global__ void hcp_w_kernel(int N, int M, const double2* __restrict__ hob,
                             const double2* __restrict__ hint, double2* __restrict__ W) {
    const int P = M * (M + 1) / 2;
    bool real = true;
    for (int e = threadIdx.x; e < P * P; e += blockDim.x) {
        const double2 w = pair_w_entry(N, M, hob, hint, e);
        real = real && w.y == 0.0;
        W[e] = w;
    }
    real = __syncthreads_and(real);
    if (threadIdx.x == 0) W[P * P] = make_double2(real ? 1.0 : 0.0, 0.0);
}

bool hcp_eligible(int N, int M) { return N >= 2 && M >= 2 && M <= kMaxTemplOrb; }

size_t hcp_scratch_bytes(int N, int M) {
    if (!hcp_eligible(N, M)) return 0;
    return (size_t)fock_dimension(N - 2, M) * (size_t)(M * (M + 1) / 2) * sizeof(double2);
}

int hcp_prepare(int M) {
    switch (M) {
        case 2: return hcp_prepare_tmpl<2>();
        case 3: return hcp_prepare_tmpl<3>();
        case 4: return hcp_prepare_tmpl<4>();
        case 5: return hcp_prepare_tmpl<5>();
        case 6: return hcp_prepare_tmpl<6>();
        case 7: return hcp_prepare_tmpl<7>();
        case 8: return hcp_prepare_tmpl<8>();
    }
    return 0;
}

int hc_prep(const SpaceView& sp, const double2* d_hob, const double2* d_hint, double2* d_tab,
            cudaStream_t st) {
    hc_prep_kernel<<<1, 32, 0, st>>>(sp.M, d_hob, d_hint, d_tab);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    if (sp.pair_y != nullptr) {
        hcp_w_kernel<<<1, 256, 0, st>>>(sp.N, sp.M, d_hob, d_hint, sp.pair_w);
        MCTDHB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

static bool hc_templated(int M) { return M >= 2 && M <= kMaxTemplOrb; }

static int hcp_apply_v(const SpaceView& sp, const double2* C, double2* HC, const HcEpilogue& ep,
                       int v, int parts, cudaStream_t st) {
    switch (sp.M) {
        case 2: return hcp_apply_tmpl<2>(sp, C, HC, ep, v, parts, st);
        case 3: return hcp_apply_tmpl<3>(sp, C, HC, ep, v, parts, st);
        case 4: return hcp_apply_tmpl<4>(sp, C, HC, ep, v, parts, st);
        case 5: return hcp_apply_tmpl<5>(sp, C, HC, ep, v, parts, st);
        case 6: return hcp_apply_tmpl<6>(sp, C, HC, ep, v, parts, st);
        case 7: return hcp_apply_tmpl<7>(sp, C, HC, ep, v, parts, st);
        case 8: return hcp_apply_tmpl<8>(sp, C, HC, ep, v, parts, st);
    }
    set_error("hcp_apply: %d orbitals outside 2..8", sp.M);
    return -1;
}

// the pair contraction's launch variant for (N, M) (pairhc_tmpl.cuh): the
// tuned choice, timed on the caller's data (the contraction alone) outside
// a capture; variants that do not exist for M are skipped
namespace {
struct PairTuneCtx {
    const SpaceView* sp;
    const double2* C;
    double2* HC;
    const HcEpilogue* ep;
};
int pair_tune_launch(void* p, int v, cudaStream_t st) {
    auto* c = (PairTuneCtx*)p;
    if (!pair_variant_ok(c->sp->M, v)) return 1;  // no such variant: skipped
    return hcp_apply_v(*c->sp, c->C, c->HC, *c->ep, v, 1, st);
}
}  // namespace

static int pair_variant(const SpaceView& sp, const double2* C, double2* HC, const HcEpilogue& ep,
                        cudaStream_t st) {
    PairTuneCtx ctx{&sp, C, HC, &ep};
    const int v = tune_pick("hcp_y", sp.N, sp.M, kPairVariants, st, pair_tune_launch, &ctx);
    return v >= 0 && v < kPairVariants && pair_variant_ok(sp.M, v) ? v : 0;
}

static int hcp_apply(const SpaceView& sp, const double2* C, double2* HC, const HcEpilogue& ep,
                     cudaStream_t st) {
    return hcp_apply_v(sp, C, HC, ep, pair_variant(sp, C, HC, ep, st), 3, st);
}

static int hc_launch_v(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
                       const HcEpilogue& ep, int v, cudaStream_t st) {
    switch (sp.M) {
        case 2: return hc_launch_tmpl<2>(sp, C, HC, tab, ep, v, st);
        case 3: return hc_launch_tmpl<3>(sp, C, HC, tab, ep, v, st);
        case 4: return hc_launch_tmpl<4>(sp, C, HC, tab, ep, v, st);
        case 5: return hc_launch_tmpl<5>(sp, C, HC, tab, ep, v, st);
        case 6: return hc_launch_tmpl<6>(sp, C, HC, tab, ep, v, st);
        case 7: return hc_launch_tmpl<7>(sp, C, HC, tab, ep, v, st);
        case 8: return hc_launch_tmpl<8>(sp, C, HC, tab, ep, v, st);
        default: {
            uint64_t need = ((uint64_t)sp.dim + 127) / 128;
            uint64_t cap = (uint64_t)num_sms() * 8;
            const int grid = (int)(need < cap ? (need ? need : 1) : cap);
            hc_generic_kernel<<<grid, 128, 0, st>>>(sp, C, HC, tab, ep);
            MCTDHB_CUDA_TRY(cudaGetLastError());
            return 0;
        }
    }
}

// launch variant (block size x barrier interval, hc_tmpl.cuh) chosen by the
// autotuner (tune.cu) on the caller's own data; small spaces use variant 0
namespace {
struct HcTuneCtx {
    const SpaceView* sp;
    const double2* C;
    double2* HC;
    const double2* tab;
    const HcEpilogue* ep;
};
int hc_tune_launch(void* p, int v, cudaStream_t st) {
    auto* c = (HcTuneCtx*)p;
    return hc_launch_v(*c->sp, c->C, c->HC, c->tab, *c->ep, v, st);
}
}  // namespace

int hc_variant(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
               const HcEpilogue& ep, cudaStream_t st) {
    if (sp.pair_y != nullptr) return pair_variant(sp, C, HC, ep, st);
    if (!hc_templated(sp.M) || sp.dim < 4096) return 0;
    HcTuneCtx ctx{&sp, C, HC, tab, &ep};
    return tune_pick("hc", sp.N, sp.M, kHcVariants, st, hc_tune_launch, &ctx);
}

int hc_apply(const SpaceView& sp, const double2* C, double2* HC, const double2* tab,
             const HcEpilogue& ep, cudaStream_t st) {
    if (sp.pair_y != nullptr) return hcp_apply(sp, C, HC, ep, st);
    const int v = hc_variant(sp, C, HC, tab, ep, st);
    return hc_launch_v(sp, C, HC, tab, ep, v, st);
}

}  // namespace mctdhb
