// batch_kernels.cu -- the slot-level and vector kernels of the batched engine
// (batch.h).  Per slot, one step is the full step of the single-system
// solver (driver.c:159-201):
//   bt_orbital_kernel   one block per slot: Runge-Kutta step of the orbital
//                       equation with the slot's rho1^{-1} and rho2,
//                       Gram-Schmidt in imaginary time, h_kl and g_ksql of the
//                       new orbitals, the pair matrix of H.C, Lanczos set-up
//   Lanczos             the pair-space H.C (per M, batch_tmpl.cuh) and the
//                       vector kernels below, multiconfig_lanczos.c:12-90
//                       operation for operation
//   SIL                 tridiagonal eigenproblem, C = V U exp(-i D dt) U^T e1,
//                       renormalisation in imaginary time
//                       (coefficients_integration.c:59-160)
//   densities           Gram-matrix rho1 / rho2 (per M, batch_tmpl.cuh)
//   bt_tail_kernel      rho1 regularisation and inverse (synchronize.c:42-57),
//                       energy (integrator_monitor.c:56-88), step count and
//                       the imaginary-time stop rule (driver.c:47-67)
// Vector kernels walk tiles of kBatchVecRows rows; every per-slot sum is
// formed from per-tile partials in tile order.
#include <cuda_runtime.h>

#include "batch.h"
#include "batch_kernels.h"
#include "common.cuh"
#include "moves.cuh"
#include "orbital_dev.cuh"
#include "small_linalg.cuh"

namespace mctdhb {

namespace {

__device__ __forceinline__ bool slot_running(const BatchSlot& S) {
    return S.flags[BF_STATE] == SLOT_RUNNING;
}

// ---------------------------------------------------------------------------
// orbital side, one block per slot
// ---------------------------------------------------------------------------

// <y_s|y_l> (Simpson) for every s, l into out[s * M + l], one warp per entry
__device__ void bt_overlaps(const BatchSlot& S, const double2* __restrict__ y, double2* out) {
    const OrbView& o = S.ov;
    const int M = o.M, G = o.G;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int p = warp; p < M * M; p += nw) {
        const int a = p / M, b = p % M;
        double2 acc = make_double2(0.0, 0.0);
        for (int x = lane; x < G; x += 32) {
            const double2 t = cfma_conj(y[(size_t)a * G + x], y[(size_t)b * G + x],
                                        make_double2(0.0, 0.0));
            acc.x += o.w[x] * t.x;
            acc.y += o.w[x] * t.y;
        }
        acc = warp_sum(acc);
        if (lane == 0) out[p] = acc;
    }
    __syncthreads();
}

// robust projector (orbital_integration.c:22-92): P <- S^{-1} P with the
// full overlap matrix S_sl = <y_s|y_l> of the stage orbitals, as the
// single-system solver does; a singular S keeps the simple projector's P
// and flags the slot (BF_ROBFAIL)
__device__ void bt_robust(const BatchSlot& S, const double2* __restrict__ y, double2* sP) {
    __shared__ double2 sS[kBatchMaxOrb * kBatchMaxOrb], sI[kBatchMaxOrb * kBatchMaxOrb];
    const int M = S.ov.M;
    bt_overlaps(S, y, sS);
    if (threadIdx.x == 0) {
        if (herm_inverse(M, sS, sI)) {
            S.flags[BF_ROBFAIL] = 1;
        } else {
            double2 t[kBatchMaxOrb * kBatchMaxOrb];
            for (int a = 0; a < M; a++)
                for (int k = 0; k < M; k++) {
                    double2 z = make_double2(0.0, 0.0);
                    for (int l = 0; l < M; l++) z = cfma(sI[a * M + l], sP[l * M + k], z);
                    t[a * M + k] = z;
                }
            for (int i = 0; i < M * M; i++) sP[i] = t[i];
        }
    }
    __syncthreads();
}

// overlap residual sum_{k<l} |<f_k|f_l>| / M of the slot's orbitals
// (integrator_monitor.c:31-42) into scal[BS_MISC + 5], summed in the
// reference's (k, l) order
__device__ void bt_overlap_residual(const BatchSlot& S) {
    __shared__ double2 sS[kBatchMaxOrb * kBatchMaxOrb];
    const int M = S.ov.M;
    bt_overlaps(S, S.orb, sS);
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int k = 0; k < M; k++)
            for (int l = k + 1; l < M; l++) sum += hypot(sS[k * M + l].x, sS[k * M + l].y);
        S.scal[BS_MISC + 5] = make_double2(sum / M, 0.0);
    }
    __syncthreads();
}

// dy/dt of the orbital equation (orbital_integration.c:179-240) for all
// orbitals y (M x G): H = linear part + interacting part, overlaps
// P[s][k] = <y_s|H_k> (simple projector, :95-131), out = -i tf (H - sum_s y_s P[s][k]).
__device__ void bt_rhs(const BatchSlot& S, const double2* __restrict__ y, double2* __restrict__ out,
                       double2* sP) {
    const OrbView& o = S.ov;
    const int M = o.M, G = o.G, n = M * G;
    double2* H = S.H;
    const double2* Q = S.Q;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = t / G, x = t % G;
        const double2 lin = o.lin_t ? toeplitz_at(o, y + (size_t)k * G, x)
                                    : linear_at(o, y + (size_t)k * G, x);
        double2 fx[kBatchMaxOrb];
        for (int a = 0; a < M; a++) fx[a] = y[(size_t)a * G + x];
        const double2* Qk = Q + (size_t)k * M * M * M;
        double2 red = make_double2(0.0, 0.0);
        for (int s = 0; s < M; s++) {
            double2 ts = make_double2(0.0, 0.0);
            for (int l = 0; l < M; l++) {
                double2 tl = make_double2(0.0, 0.0);
                for (int q = 0; q < M; q++) tl = cfma(Qk[s + q * M + l * M * M], fx[q], tl);
                ts = cfma(tl, fx[l], ts);
            }
            red = cfma(make_double2(fx[s].x, -fx[s].y), ts, red);
        }
        H[t] = cadd(red, lin);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int p = warp; p < M * M; p += nw) {
        const int s = p / M, k = p % M;
        double2 acc = make_double2(0.0, 0.0);
        for (int x = lane; x < G; x += 32) {
            const double2 t = cfma_conj(y[(size_t)s * G + x], H[(size_t)k * G + x],
                                        make_double2(0.0, 0.0));
            acc.x += o.w[x] * t.x;
            acc.y += o.w[x] * t.y;
        }
        acc = warp_sum(acc);
        if (lane == 0) sP[p] = acc;
    }
    __syncthreads();
    if (S.flags[BF_ROBUST]) bt_robust(S, y, sP);
    const double2 mi_tf = make_double2(o.tf.y, -o.tf.x);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = t / G, x = t % G;
        double2 proj = make_double2(0.0, 0.0);
        for (int s = 0; s < M; s++) proj = cfma(y[(size_t)s * G + x], sP[s * M + k], proj);
        const double2 d = make_double2(H[t].x - proj.x, H[t].y - proj.y);
        out[t] = cmul(mi_tf, d);
    }
    __syncthreads();
}

// the split step's nonlinear right-hand side (orbital_integration.c:
// 243-281), as orb_split_rhs_kernel: -i tf (interacting - sum_j (h[j][k] +
// B[k][j]) f_j + V f_k), h of the half-stepped orbitals
__device__ void bt_split_rhs(const BatchSlot& S, const double2* __restrict__ y,
                             double2* __restrict__ out) {
    const OrbView& o = S.ov;
    const int M = o.M, G = o.G, n = M * G;
    const double2* Q = S.Q;
    const double2 mi_tf = make_double2(o.tf.y, -o.tf.x);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = t / G, x = t % G;
        double2 fx[kBatchMaxOrb];
        for (int a = 0; a < M; a++) fx[a] = y[(size_t)a * G + x];
        const double2* Qk = Q + (size_t)k * M * M * M;
        double2 red = make_double2(0.0, 0.0);
        for (int s = 0; s < M; s++) {
            double2 ts = make_double2(0.0, 0.0);
            for (int l = 0; l < M; l++) {
                double2 tl = make_double2(0.0, 0.0);
                for (int q = 0; q < M; q++) tl = cfma(Qk[s + q * M + l * M * M], fx[q], tl);
                ts = cfma(tl, fx[l], ts);
            }
            red = cfma(make_double2(fx[s].x, -fx[s].y), ts, red);
        }
        for (int j = 0; j < M; j++) {
            const double2 c = cadd(S.hob[j * M + k], S.B[k * M + j]);
            red.x -= c.x * fx[j].x - c.y * fx[j].y;
            red.y -= c.x * fx[j].y + c.y * fx[j].x;
        }
        red = cadd(red, cscale(fx[k], o.pot[x]));
        out[t] = cmul(mi_tf, red);
    }
    __syncthreads();
}

// linear half step of the split step, y <- Op y for every orbital, through
// the spare stage buffer (orb_half_kernel: the same sums in the same order)
__device__ void bt_half_step(const BatchSlot& S, double2* y) {
    const int M = S.ov.M, G = S.ov.G, n = M * G;
    const int dense = S.half_dense, nn = dense ? G : G - 1;
    double2* w = S.stage + (size_t)7 * n - n;  // stage[6], the stage input of RK
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = t / G, x = t % G;
        const double2* f = y + (size_t)k * G;
        double2 acc = make_double2(0.0, 0.0);
        if (dense) {
            for (int j = 0; j < nn; j++) acc = cfma(S.half[(size_t)j * G + x], f[j], acc);
        } else {
            const double2* tk = S.half + (nn - 1 - (x == nn ? 0 : x));
            for (int j = 0; j < nn; j++) acc = cfma(tk[j], f[j], acc);
        }
        w[t] = acc;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) y[t] = w[t];
    __syncthreads();
}

// B[k][j] = sum_a rinv[k][a] sum_{s,q,l} rho2[a + sM + qM^2 + lM^3]
//           hint[j + sM + lM^2 + qM^3] (orb_bmat_kernel, same order)
__device__ void bt_bmat(const BatchSlot& S) {
    const int M = S.M, M2 = M * M, M3 = M2 * M;
    for (int e = threadIdx.x; e < M2; e += blockDim.x) {
        const int k = e / M, j = e % M;
        double2 acc = make_double2(0.0, 0.0);
        for (int a = 0; a < M; a++) {
            double2 inner = make_double2(0.0, 0.0);
            for (int s = 0; s < M; s++)
                for (int q = 0; q < M; q++)
                    for (int l = 0; l < M; l++)
                        inner = cfma(S.rho2[a + s * M + q * M2 + l * M3],
                                     S.hint[j + s * M + l * M2 + q * M3], inner);
            acc = cfma(S.rinv[k * M + a], inner, acc);
        }
        S.B[e] = acc;
    }
    __syncthreads();
}

// out = y + dt sum_j c_j k_j
struct Combo {
    int n;
    int j[5];
    double c[5];
};

// (out may be y itself: each point is read before it is written)
__device__ void bt_combo(const BatchSlot& S, const double2* y, const Combo& cb, double2* out) {
    const int n = S.ov.M * S.ov.G;
    const double dt = S.dt;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int q = 0; q < cb.n; q++) {
            const double2 kv = S.stage[(size_t)cb.j[q] * n + t];
            s.x += cb.c[q] * kv.x;
            s.y += cb.c[q] * kv.y;
        }
        out[t] = make_double2(y[t].x + dt * s.x, y[t].y + dt * s.y);
    }
    __syncthreads();
}

// Runge-Kutta step of the orbitals in place (orbital_integration.c:284-349)
// with the named tableaux Heun (2), classical RK4 (4) and Butcher RK5 (5);
// split: the split step's nonlinear right-hand side (orbital_integration.c:
// 387-415) in place of the full one.  Stage j lives in stage[j], the stage
// input in stage[6].
__device__ void bt_rk_step(const BatchSlot& S, double2* sP, bool split) {
    const int n = S.ov.M * S.ov.G;
    double2* y = S.orb;
    double2* w = S.stage + (size_t)6 * n;
    auto k = [&](int j) { return S.stage + (size_t)j * n; };
    auto rhs = [&](const double2* in, double2* out) {
        if (split)
            bt_split_rhs(S, in, out);
        else
            bt_rhs(S, in, out, sP);
    };
    auto C1 = [](int a, double ca) { Combo c{1, {a}, {ca}}; return c; };
    switch (S.rk) {
        case 2:
            rhs(y, k(0));
            bt_combo(S, y, C1(0, 1.0), w);
            rhs(w, k(1));
            bt_combo(S, y, Combo{2, {0, 1}, {0.5, 0.5}}, y);
            break;
        case 4:
            rhs(y, k(0));
            bt_combo(S, y, C1(0, 0.5), w);
            rhs(w, k(1));
            bt_combo(S, y, C1(1, 0.5), w);
            rhs(w, k(2));
            bt_combo(S, y, C1(2, 1.0), w);
            rhs(w, k(3));
            bt_combo(S, y, Combo{4, {0, 1, 2, 3}, {1.0 / 6, 2.0 / 6, 2.0 / 6, 1.0 / 6}}, y);
            break;
        default:  // 5
            rhs(y, k(0));
            bt_combo(S, y, C1(0, 0.25), w);
            rhs(w, k(1));
            bt_combo(S, y, Combo{2, {0, 1}, {0.125, 0.125}}, w);
            rhs(w, k(2));
            bt_combo(S, y, Combo{2, {1, 2}, {-0.5, 1.0}}, w);
            rhs(w, k(3));
            bt_combo(S, y, Combo{2, {0, 3}, {3.0 / 16, 9.0 / 16}}, w);
            rhs(w, k(4));
            bt_combo(S, y,
                     Combo{5, {0, 1, 2, 3, 4}, {-3.0 / 7, 2.0 / 7, 12.0 / 7, -12.0 / 7, 8.0 / 7}},
                     w);
            rhs(w, k(5));
            bt_combo(S, y,
                     Combo{5, {0, 2, 3, 4, 5}, {7.0 / 90, 32.0 / 90, 12.0 / 90, 32.0 / 90, 7.0 / 90}},
                     y);
            break;
    }
}

__device__ void bt_periodic(const BatchSlot& S) {
    const int M = S.ov.M, G = S.ov.G;
    if (S.ov.periodic && threadIdx.x < M) S.orb[(size_t)threadIdx.x * G + G - 1] = S.orb[(size_t)threadIdx.x * G];
    __syncthreads();
}

// h_kl (orbital_matrices.c:22-70): one warp per pair k <= l;
// g_ksql: one warp per 8 x 8 tensor-core tile (hint_tile)
__device__ void bt_matrices(const BatchSlot& S) {
    const OrbView& o = S.ov;
    const int M = o.M, G = o.G;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const double r = 1.0 / (12 * o.dx);
    const int npair = M * (M + 1) / 2;
    for (int p = warp; p < npair; p += nw) {
        int q = p, k = 0;
        while (q >= M - k) {
            q -= M - k;
            k++;
        }
        const int l = k + q;
        const double2* fk = S.orb + (size_t)k * G;
        const double2* fl = S.orb + (size_t)l * G;
        double2 acc = make_double2(0.0, 0.0);
        for (int x = lane; x < G; x += 32) {
            const double2 t = hob_integrand(o, fk, fl, x, r);
            acc.x += o.w[x] * t.x;
            acc.y += o.w[x] * t.y;
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            if (k == l) {
                S.hob[k * M + k] = make_double2(acc.x, 0.0);
            } else {
                S.hob[k * M + l] = acc;
                S.hob[l * M + k] = make_double2(acc.x, -acc.y);
            }
        }
    }
    const int tiles = (M * M + 7) / 8;
    for (int t = warp; t < tiles * tiles; t += nw) hint_tile(o, S.orb, S.g, S.hint, t, lane);
    __syncthreads();
}

}  // namespace

// mode 0: one full orbital step (periodic copy, Runge-Kutta, Gram-Schmidt,
// periodic copy), then the matrices of the new orbitals;
// mode 1: the matrices of the orbitals as given (set-up of a new slot)
__global__ void __launch_bounds__(kBatchOrbThreads)
    bt_orbital_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                      const int* __restrict__ nlist, int mode, int* __restrict__ mon) {
    // a new step: no monitor H.C due yet in any orbital count
    if (mon != nullptr && blockIdx.x == 0 && threadIdx.x < kBatchNumM) mon[threadIdx.x] = 0;
    if ((int)blockIdx.x >= *nlist) return;
    const BatchSlot& S = slots[list[blockIdx.x]];
    if (!slot_running(S)) return;
    extern __shared__ double scan[];  // G doubles (Gram-Schmidt)
    __shared__ double2 sP[kBatchMaxOrb * kBatchMaxOrb];
    const int M = S.M;
    if (mode == 0) {
        bt_periodic(S);
        // Q[k][s + qM + lM^2] = g sum_a rinv[k][a] rho2[a, s, q, l]
        const int M3 = M * M * M, M4 = M3 * M;
        const double g = *S.g;
        for (int e = threadIdx.x; e < M4; e += blockDim.x) {
            const int k = e / M3, sql = e % M3;
            double2 acc = make_double2(0.0, 0.0);
            for (int a = 0; a < M; a++) acc = cfma(S.rinv[k * M + a], S.rho2[a + M * sql], acc);
            S.Q[e] = cscale(acc, g);
        }
        __syncthreads();
        if (S.split) {
            // orbital_integration.c:352-434: half step, h and g of the
            // half-stepped orbitals, B, RK of the nonlinear part, half step
            bt_half_step(S, S.orb);
            bt_matrices(S);
            bt_bmat(S);
            bt_rk_step(S, sP, true);
            bt_half_step(S, S.orb);
        } else {
            bt_rk_step(S, sP, false);
        }
        if (S.imag) {
            orthonormalize_block(S.ov, S.orb, scan);
            __syncthreads();
        }
        bt_periodic(S);
        // real time: the orbitals' drift from orthonormality, for the
        // monitor of the tail kernel (driver.c:69-96)
        if (!S.imag) bt_overlap_residual(S);
    }
    bt_matrices(S);
    __syncthreads();
    // the pair matrix of H.C for the new h and g, and its real flag
    // (pairhc_tmpl.cuh)
    const int P2 = M * (M + 1) / 2 * (M * (M + 1) / 2);
    bool real = true;
    for (int e = threadIdx.x; e < P2; e += blockDim.x) {
        const double2 w = pair_w_entry(S.N, M, S.hob, S.hint, e);
        real = real && w.y == 0.0;
        S.sp.pair_w[e] = w;
    }
    real = __syncthreads_and(real);
    if (threadIdx.x == 0) {
        S.sp.pair_w[P2] = make_double2(real ? 1.0 : 0.0, 0.0);
        // Lanczos set-up of this step (multiconfig_lanczos.c:30-41)
        S.flags[BF_BREAK] = 0;
        S.flags[BF_ITERS] = S.lz;
        S.flags[BF_QL] = 0;
        S.scal[BS_MISC + 0] = make_double2(0.0, 0.0);
        S.scal[BS_OFFD + S.lz - 1] = make_double2(0.0, 0.0);
    }
}

// ---------------------------------------------------------------------------
// vector kernels over tiles of kBatchVecRows rows
// ---------------------------------------------------------------------------
#define BT_TILE_LOOP                                                              \
    const int nt = *ntiles;                                                       \
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {                            \
        const BatchTile tl = tiles[t];                                            \
        const BatchSlot& S = slots[tl.slot];                                      \
        const uint32_t nc = S.nc;                                                 \
        const uint32_t r0 = tl.idx * (uint32_t)kBatchVecRows;
#define BT_ROWS(r)                                                                \
    for (uint32_t r = r0 + threadIdx.x; r < nc && r < r0 + kBatchVecRows; r += kBatchVecThreads)

// part[tile] = <V[i], out>   (alpha_i, multiconfig_lanczos.c:40-41, :83)
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_dot_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                  const int* __restrict__ ntiles, int i) {
    BT_TILE_LOOP
    if (!slot_running(S) || S.flags[BF_BREAK]) continue;
    const double2* v = S.V + (size_t)i * nc;
    double2 acc = make_double2(0.0, 0.0);
    BT_ROWS(r) acc = cfma_conj(v[r], S.out[r], acc);
    const double2 s = block_sum(acc);
    if (threadIdx.x == 0) S.part[tl.idx] = s;
    }
}

// out -= alpha_i V[i]; part[k * vtiles + tile] = <V[k], out>, k <= i
// (multiconfig_lanczos.c:46, :57-62)
// (the iteration is a template parameter: only the i + 1 accumulators in
// use take registers, which keeps enough warps resident)
template <int I>
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_subdots_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                      const int* __restrict__ ntiles) {
    BT_TILE_LOOP
    if (!slot_running(S) || S.flags[BF_BREAK]) continue;
    const double2 alpha = S.scal[BS_DIAG + I];
    double2 acc[I + 1];
#pragma unroll
    for (int k = 0; k <= I; k++) acc[k] = make_double2(0.0, 0.0);
    BT_ROWS(r) {
        // every Krylov value is loaded before the store to out (which may
        // alias V as far as the compiler knows), V[I] once
        double2 v[I + 1];
#pragma unroll
        for (int k = 0; k <= I; k++) v[k] = S.V[(size_t)k * nc + r];
        double2 o = S.out[r];
        const double2 av = cmul(alpha, v[I]);
        o.x -= av.x;
        o.y -= av.y;
        S.out[r] = o;
#pragma unroll
        for (int k = 0; k <= I; k++) acc[k] = cfma_conj(v[k], o, acc[k]);
    }
#pragma unroll
    for (int k = 0; k <= I; k++) {
        const double2 s = block_sum(acc[k]);
        if (threadIdx.x == 0) S.part[(size_t)k * S.vtiles + tl.idx] = s;
    }
    }
}

template <int I>
static void subdots_launch(int i, int grid, cudaStream_t st, const BatchSlot* slots,
                           const BatchTile* tiles, const int* ntiles) {
    if (i == I)
        bt_subdots_kernel<I><<<grid, kBatchVecThreads, 0, st>>>(slots, tiles, ntiles);
    else if constexpr (I > 0)
        subdots_launch<I - 1>(i, grid, st, slots, tiles, ntiles);
}

// out -= sum_{k<=i} o_k V[k]; part[tile] = |out|^2 (multiconfig_lanczos.c:57-64)
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_orth_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                   const int* __restrict__ ntiles, int i) {
    BT_TILE_LOOP
    if (!slot_running(S) || S.flags[BF_BREAK]) continue;
    double acc = 0.0;
    BT_ROWS(r) {
        double2 o = S.out[r];
        for (int k = 0; k <= i; k++) {
            const double2 tv = cmul(S.V[(size_t)k * nc + r], S.scal[BS_ORTHO + k]);
            o.x -= tv.x;
            o.y -= tv.y;
        }
        S.out[r] = o;
        acc += o.x * o.x + o.y * o.y;
    }
    const double2 s = block_sum(make_double2(acc, 0.0));
    if (threadIdx.x == 0) S.part[tl.idx] = s;
    }
}

// V[i+1] = out / beta_i (multiconfig_lanczos.c:74)
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_scale_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                    const int* __restrict__ ntiles, int i) {
    BT_TILE_LOOP
    if (!slot_running(S) || S.flags[BF_BREAK]) continue;
    const double inv = S.scal[BS_MISC + 1].x;
    BT_ROWS(r) {
        const double2 o = S.out[r];
        S.V[(size_t)(i + 1) * nc + r] = make_double2(o.x * inv, o.y * inv);
    }
    }
}

// C = sum_j y_j V[j] over the vectors built (coefficients_integration.c:127-154);
// C is V[0], overwritten row by row after its own rows are read
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_combine_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                      const int* __restrict__ ntiles) {
    BT_TILE_LOOP
    if (!slot_running(S)) continue;
    const int it = S.flags[BF_ITERS];
    BT_ROWS(r) {
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < it; j++) s = cfma(S.V[(size_t)j * nc + r], S.scal[BS_Y + j], s);
        S.V[r] = s;
    }
    }
}

// part[tile] = |C|^2
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_norm2_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                    const int* __restrict__ ntiles) {
    BT_TILE_LOOP
    if (!slot_running(S) || !S.imag) continue;
    double acc = 0.0;
    BT_ROWS(r) acc += S.V[r].x * S.V[r].x + S.V[r].y * S.V[r].y;
    const double2 s = block_sum(make_double2(acc, 0.0));
    if (threadIdx.x == 0) S.part[tl.idx] = s;
    }
}

// C /= |C| (imaginary time, coefficients_integration.c:156-159)
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_renorm_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                     const int* __restrict__ ntiles) {
    BT_TILE_LOOP
    if (!slot_running(S) || !S.imag) continue;
    const double rn = 1.0 / sqrt(S.scal[BS_MISC + 2].x);
    BT_ROWS(r) {
        S.V[r].x *= rn;
        S.V[r].y *= rn;
    }
    }
}

#undef BT_TILE_LOOP
#undef BT_ROWS

// ---------------------------------------------------------------------------
// slot kernels: one block per slot of the list
// ---------------------------------------------------------------------------
#define BT_SLOT                                                                   \
    if ((int)blockIdx.x >= *nlist) return;                                        \
    const BatchSlot& S = slots[list[blockIdx.x]];                                 \
    if (!slot_running(S)) return;

// fixed-order sum of part[k * vtiles + t] over t, for k < nvals, into
// scal[dst + k]: threads take strided partial sums, then a tree (256 threads)
__device__ double2 bt_sum_parts(const double2* part, int ntile) {
    __shared__ double2 sh[kBatchVecThreads];
    double2 s = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < ntile; b += blockDim.x) {
        s.x += part[b].x;
        s.y += part[b].y;
    }
    __syncthreads();
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[threadIdx.x].x += sh[threadIdx.x + o].x;
            sh[threadIdx.x].y += sh[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    return sh[0];
}

// scal[dst + k] = sum_t part[k * vtiles + t], k < nvals.  skip_break: the
// value belongs to a Lanczos iteration a breakdown has cancelled.
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_reduce_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                     const int* __restrict__ nlist, int nvals, int dst, int skip_break) {
    BT_SLOT
    if (skip_break && S.flags[BF_BREAK]) return;
    for (int k = 0; k < nvals; k++) {
        const double2 s = bt_sum_parts(S.part + (size_t)k * S.vtiles, S.vtiles);
        if (threadIdx.x == 0) S.scal[dst + k] = s;
        __syncthreads();
    }
}

// beta_i = |out|; breakdown when beta_i / max beta < 1e-14 (or beta_i = 0);
// 1/beta_i for the scaling (multiconfig_lanczos.c:64-74)
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_norm_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                   const int* __restrict__ nlist, int i) {
    BT_SLOT
    if (S.flags[BF_BREAK]) return;
    const double2 s = bt_sum_parts(S.part, S.vtiles);
    if (threadIdx.x != 0) return;
    const double beta = sqrt(s.x);
    S.scal[BS_OFFD + i] = make_double2(beta, 0.0);
    double mx = S.scal[BS_MISC + 0].x;
    if (mx < beta) mx = beta;
    S.scal[BS_MISC + 0].x = mx;
    if (beta == 0.0 || beta / mx < 1e-14) {
        S.flags[BF_BREAK] = 1;
        S.flags[BF_ITERS] = i + 1;
        return;
    }
    S.scal[BS_MISC + 1] = make_double2(1.0 / beta, 0.0);
}

// y = U exp(-i D pdt) U^T e1 of the tridiagonal (alpha, beta) (implicit QL)
__global__ void bt_small_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                                const int* __restrict__ nlist) {
    BT_SLOT
    if (threadIdx.x != 0) return;
    const int n = S.flags[BF_ITERS];
    double d[kBatchMaxLz], e[kBatchMaxLz];
    for (int k = 0; k < n; k++) {
        d[k] = S.scal[BS_DIAG + k].x;
        e[k] = S.scal[BS_OFFD + k].x;
    }
    double* z = (double*)(S.scal + BS_Z);
    S.flags[BF_QL] = tridiag_ql(n, d, e, z);
    const double2 pdt = S.pdt;
    // imaginary time: exponents shifted by their maximum (a constant factor
    // the renormalisation at the end of the step removes), so exp cannot
    // overflow at |E| dt > 709; real time: no shift, unchanged bits
    double shift = 0.0;
    if (pdt.y != 0.0)
        for (int k = 0; k < n; k++) shift = k == 0 ? d[k] * pdt.y : fmax(shift, d[k] * pdt.y);
    double2 aux[kBatchMaxLz];
    for (int k = 0; k < n; k++) {
        const double re = d[k] * pdt.y, im = -d[k] * pdt.x;
        const double mag = exp(re - shift);
        double sn, cs;
        sincos(im, &sn, &cs);
        const double u = z[0 * n + k];
        aux[k] = make_double2(u * mag * cs, u * mag * sn);
    }
    for (int k = 0; k < n; k++) {
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < n; j++) {
            s.x += z[k * n + j] * aux[j].x;
            s.y += z[k * n + j] * aux[j].y;
        }
        S.scal[BS_Y + k] = s;
    }
}

// rho1 regularisation and inverse, energy, step count, stop rules.
// prologue: set-up of a new slot (no step counted; the energy seeds the
// imaginary-time stop rule as driver.c:229 does).
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_tail_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                   const int* __restrict__ nlist, int prologue, int* __restrict__ mon) {
    BT_SLOT
    const int M = S.M;
    if (threadIdx.x == 0) {
        // staged in shared memory: the routine's dependent accesses stay on
        // the SM (same operations and bits as on the arena's copies)
        __shared__ double2 r1[kBatchMaxOrb * kBatchMaxOrb], ri[kBatchMaxOrb * kBatchMaxOrb];
        __shared__ double2 w[3 * kBatchMaxOrb * kBatchMaxOrb + kBatchMaxOrb / 2 + 1];
        const int M2 = M * M;
        for (int i = 0; i < M2; i++) r1[i] = S.rho1[i];
        S.flags[BF_INFO] = sync_rho1(M, r1, ri, S.reg_fac, w, (double*)(w + 3 * M2));
        for (int i = 0; i < M2; i++) {
            S.rho1[i] = r1[i];
            S.rinv[i] = ri[i];
        }
    }
    __syncthreads();
    const double2 E = energy_block(M, S.rho1, S.rho2, S.hob, S.hint);
    if (threadIdx.x != 0) return;
    S.scal[BS_MISC + 3] = E;
    if (prologue) {
        S.scal[BS_MISC + 4] = make_double2(E.x / S.N, 0.0);
        S.scal[BS_MISC + 6] = make_double2(-1.0, 0.0);  // no eigen residual yet
        return;
    }
    const int steps = S.flags[BF_STEPS] + 1;
    S.flags[BF_STEPS] = steps;
    int state = SLOT_RUNNING;
    const bool check = S.check_every > 0 && steps % S.check_every == 0;
    if (S.imag && check) {
        // driver.c:47-67: |E/N - prev| < tol * prev, and with eig_tol set the
        // eigen residual below it: that half is decided by bt_monitor_kernel
        // after the monitor's H.C of this step
        const double curr = E.x / S.N, prev = S.scal[BS_MISC + 4].x;
        if (fabs(curr - prev) < S.etol * prev) {
            if (S.eig_tol > 0.0) {
                S.flags[BF_MON] = 1;
                mon[S.M] = 1;
            } else {
                state = SLOT_DONE;
                S.flags[BF_CONV] = 1;
            }
        }
        S.scal[BS_MISC + 4] = make_double2(curr, 0.0);
    }
    if (!S.imag && check) {
        // driver.c:69-96: switch the robust projector on above the
        // threshold; above the critical residual the reference exits, the
        // engine stops this job
        const double o = S.scal[BS_MISC + 5].x;
        if (o > S.ortho_tol && !S.flags[BF_ROBUST]) S.flags[BF_ROBUST] = 1;
        if (o > kOverlapAbort) state = SLOT_ABORTED;
    }
    if ((uint32_t)steps >= S.max_steps && state == SLOT_RUNNING) state = SLOT_DONE;
    S.flags[BF_STATE] = state;
}

// max_i |E C_i - (H C)_i| over a vector tile of the slots whose eigen
// residual is due (integrator_monitor.c:9-28), into part[tile].x
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_resid_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                    const int* __restrict__ ntiles) {
    __shared__ double sh[kBatchVecThreads];
    const int nt = *ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const BatchTile tl = tiles[t];
        const BatchSlot& S = slots[tl.slot];
        if (!S.flags[BF_MON]) continue;  // block-uniform
        const uint32_t nc = S.nc;
        const uint32_t r0 = tl.idx * (uint32_t)kBatchVecRows;
        const double e = S.scal[BS_MISC + 3].x;
        double m = 0.0;
        for (uint32_t r = r0 + threadIdx.x; r < nc && r < r0 + kBatchVecRows;
             r += kBatchVecThreads) {
            const double2 c = S.V[r], h = S.out[r];
            m = fmax(m, hypot(e * c.x - h.x, e * c.y - h.y));
        }
        sh[threadIdx.x] = m;
        __syncthreads();
        for (int o = kBatchVecThreads / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
            __syncthreads();
        }
        if (threadIdx.x == 0) S.part[tl.idx] = make_double2(sh[0], 0.0);
        __syncthreads();
    }
}

// the eigen-residual half of the imaginary-time stop rule (driver.c:47-67):
// res = max over the tiles / N; the slot stops (converged) when res is
// below eig_tol
__global__ void __launch_bounds__(kBatchVecThreads)
    bt_monitor_kernel(const BatchSlot* __restrict__ slots, const int* __restrict__ list,
                      const int* __restrict__ nlist) {
    __shared__ double sh[kBatchVecThreads];
    if ((int)blockIdx.x >= *nlist) return;
    const BatchSlot& S = slots[list[blockIdx.x]];
    if (!S.flags[BF_MON]) return;
    double m = 0.0;
    for (int t = threadIdx.x; t < S.vtiles; t += blockDim.x) m = fmax(m, S.part[t].x);
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double res = sh[0] / S.N;
    S.scal[BS_MISC + 6] = make_double2(res, 0.0);
    if (res < S.eig_tol) {
        S.flags[BF_STATE] = SLOT_DONE;
        S.flags[BF_CONV] = 1;
    }
    S.flags[BF_MON] = 0;
}

#undef BT_SLOT

void bt_subdots(int i, int grid, cudaStream_t st, const BatchSlot* slots, const BatchTile* tiles,
                const int* ntiles) {
    subdots_launch<kBatchMaxLz - 2>(i, grid, st, slots, tiles, ntiles);
}

}  // namespace mctdhb
