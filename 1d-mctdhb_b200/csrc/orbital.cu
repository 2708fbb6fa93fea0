// orbital.cu -- the orbital side of one MCTDHB step on the device:
//   h_kl                 set_orbital_hob     (orbital_matrices.c:22-70)
//   g_ksql               set_orbital_hint    (orbital_matrices.c:73-287),
//                        as one (M^2 x G)(G x M^2) complex contraction on the
//                        FP64 tensor cores (mma.sync m8n8k4 f64)
//   orbital equation     dodt_fullstep_interface (orbital_integration.c:179-240)
//                        with the linear part of orbital_integration.c:137-176:
//                        finite differences (split_linear_orbitals.c:210-255),
//                        or the DVR matrix (:83-166) / spectral derivative
//                        (:257-287) as one Toeplitz product, the interacting
//                        part (split_nonlinear_orbitals.c:4-61) and the simple
//                        projector (orbital_integration.c:95-131) or, once
//                        the orbitals drift from orthonormality, the robust
//                        one (orbital_integration.c:22-92)
//   Runge-Kutta step     propagate_fullstep_orb_rk (orbital_integration.c:284)
//                        with the named tableaux Heun / classical RK4 /
//                        Butcher RK5
//   split step           propagate_splitstep_orb (orbital_integration.c:352):
//                        Crank-Nicolson or FFT-exponential half steps as one
//                        precomputed operator product (circulant on periodic
//                        grids, dense with zero bounds), RK of the full
//                        nonlinear term (split_nonlinear_orbitals.c:63-160)
//   Gram-Schmidt         orthonormalize (calculus.c:171-191)
//   rho1 synchronisation sync_density_matrices (synchronize.c:42-57)
// Grid functions are row-major M x G complex128; integrals use the composite
// Simpson weights of calculus.c:9-40 (3/8 rule on the last four points for
// an even number of points).
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "orbital.h"
#include "orbital_dev.cuh"
#include "small_linalg.cuh"

namespace mctdhb {

std::vector<double> simpson_weights(int n, double h) {
    std::vector<double> w(n, 0.0);
    if (n % 2 == 0) {
        for (int i = 0; i < n - 4; i += 2) {
            w[i] += 1;
            w[i + 1] += 4;
            w[i + 2] += 1;
        }
        for (int i = 0; i < n - 3; i++) w[i] *= h / 3;
        w[n - 4] += 3 * h / 8;
        w[n - 3] += 9 * h / 8;
        w[n - 2] += 9 * h / 8;
        w[n - 1] += 3 * h / 8;
    } else {
        for (int i = 0; i < n - 2; i += 2) {
            w[i] += 1;
            w[i + 1] += 4;
            w[i + 2] += 1;
        }
        for (int i = 0; i < n; i++) w[i] *= h / 3;
    }
    return w;
}

// h_kl, one block per pair k <= l (orbital_matrices.c:22-70)
__global__ void hob_kernel(OrbView o, const double2* __restrict__ orb, double2* __restrict__ hob) {
    const int M = o.M, G = o.G;
    int p = blockIdx.x, k = 0;
    while (p >= M - k) {
        p -= M - k;
        k++;
    }
    const int l = k + p;
    const double2* fk = orb + (size_t)k * G;
    const double2* fl = orb + (size_t)l * G;
    const double r = 1.0 / (12 * o.dx);
    double2 acc = make_double2(0.0, 0.0);
    for (int x = threadIdx.x; x < G; x += blockDim.x) {
        const double2 t = hob_integrand(o, fk, fl, x, r);
        acc.x += o.w[x] * t.x;
        acc.y += o.w[x] * t.y;
    }
    const double2 s = block_sum(acc);
    if (threadIdx.x == 0) {
        if (k == l) {
            hob[k * M + k] = make_double2(s.x, 0.0);
        } else {
            hob[k * M + l] = s;
            hob[l * M + k] = make_double2(s.x, -s.y);
        }
    }
}

// g_ksql on the FP64 tensor cores, one warp per 8 x 8 tile (hint_tile)
__global__ void hint_dmma_kernel(OrbView o, const double2* __restrict__ orb,
                                 const double* __restrict__ g_dev, double2* __restrict__ hint) {
    const int M2 = o.M * o.M;
    const int tiles = (M2 + 7) / 8;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= tiles * tiles) return;
    hint_tile(o, orb, g_dev, hint, warp, threadIdx.x & 31);
}

// Q[k,s,q,l] = g sum_a rinv[k][a] rho2[a,s,q,l]
__global__ void orb_q_kernel(int M, const double* __restrict__ g_dev,
                             const double2* __restrict__ rinv, const double2* __restrict__ rho2,
                             double2* __restrict__ Q) {
    const int M3 = M * M * M, M4 = M3 * M;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M4) return;
    const int k = e / M3, sql = e % M3;  // Q stored as [k][s + qM + lM^2]
    double2 acc = make_double2(0.0, 0.0);
    for (int a = 0; a < M; a++) acc = cfma(rinv[k * M + a], rho2[a + M * sql], acc);
    Q[e] = cscale(acc, *g_dev);
}

// DVR / spectral linear part (orbital_integration.c:137-176):
// L_k(x) = sum_j lin_t[j - x + n - 1] f_k(j) + V(x) f_k(x) on the n = G - 1
// periodic points, L_k(n) = L_k(0).  Block (k, chunk) stages f_k in shared
// memory; thread x sums over j, reading the kernel at consecutive addresses.
__global__ void __launch_bounds__(256) orb_toeplitz_kernel(OrbView o, const double2* __restrict__ y,
                                                           double2* __restrict__ L) {
    extern __shared__ double2 fs[];  // n values
    const int G = o.G, n = G - 1;
    const int k = blockIdx.y;
    const double2* f = y + (size_t)k * G;
    for (int j = threadIdx.x; j < n; j += blockDim.x) fs[j] = f[j];
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x > n) return;
    const int xr = x == n ? 0 : x;
    const double2* t = o.lin_t + (n - 1 - xr);
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < n; j++) acc = cfma(__ldg(t + j), fs[j], acc);
    L[(size_t)k * G + x] = cadd(acc, cscale(fs[xr], o.pot[xr]));
}

// Linear half step of the split-step integrator: out_k = Op f_k.  Circulant
// Op on the n = G - 1 periodic points (kernel t, (Op f)_x =
// sum_j t[j - x + n - 1] f_j, out(n) = out(0)), or dense on all G points
// (zero bounds; stored column-major, Op[x][j] = D[j G + x]).
__global__ void __launch_bounds__(256) orb_half_kernel(OrbView o, const double2* __restrict__ op,
                                                       int dense, const double2* __restrict__ y,
                                                       double2* __restrict__ out) {
    extern __shared__ double2 fs[];
    const int G = o.G, n = dense ? G : G - 1;
    const int k = blockIdx.y;
    const double2* f = y + (size_t)k * G;
    for (int j = threadIdx.x; j < n; j += blockDim.x) fs[j] = f[j];
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= G) return;
    double2 acc = make_double2(0.0, 0.0);
    if (dense) {
        for (int j = 0; j < n; j++) acc = cfma(__ldg(op + (size_t)j * G + x), fs[j], acc);
    } else {
        const double2* t = op + (n - 1 - (x == n ? 0 : x));
        for (int j = 0; j < n; j++) acc = cfma(__ldg(t + j), fs[j], acc);
    }
    out[(size_t)k * G + x] = acc;
}

// B[k][j] = sum_{a,s,q,l} rinv[k][a] rho2[a + sM + qM^2 + lM^3]
//           hint[j + sM + lM^2 + qM^3]: the projection of the interacting
// part through g in orb_full_nonlinear (split_nonlinear_orbitals.c:63-160),
// summed over all index orders (rho2 and g are symmetric in the pairs)
__global__ void orb_bmat_kernel(int M, const double2* __restrict__ rinv,
                                const double2* __restrict__ rho2,
                                const double2* __restrict__ hint, double2* __restrict__ B) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * M) return;
    const int k = e / M, j = e % M, M2 = M * M, M3 = M2 * M;
    double2 acc = make_double2(0.0, 0.0);
    for (int a = 0; a < M; a++) {
        double2 inner = make_double2(0.0, 0.0);
        for (int s = 0; s < M; s++)
            for (int q = 0; q < M; q++)
                for (int l = 0; l < M; l++)
                    inner = cfma(rho2[a + s * M + q * M2 + l * M3],
                                 hint[j + s * M + l * M2 + q * M3], inner);
        acc = cfma(rinv[k * M + a], inner, acc);
    }
    B[e] = acc;
}

// nonlinear right-hand side of the split step (orbital_integration.c:
// 243-281): -i tf (interacting - sum_j (h[j][k] + B[k][j]) f_j + V f_k)
__global__ void orb_split_rhs_kernel(OrbView o, const double2* __restrict__ y,
                                     const double2* __restrict__ Q,
                                     const double2* __restrict__ hob,
                                     const double2* __restrict__ B, double2* __restrict__ out) {
    const int M = o.M, G = o.G;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * G) return;
    const int k = t / G, x = t % G;
    double2 fx[kMaxOrb];
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
        const double2 c = cadd(hob[j * M + k], B[k * M + j]);
        red.x -= c.x * fx[j].x - c.y * fx[j].y;
        red.y -= c.x * fx[j].y + c.y * fx[j].x;
    }
    red = cadd(red, cscale(fx[k], o.pot[x]));
    const double2 mi_tf = make_double2(o.tf.y, -o.tf.x);
    out[t] = cmul(mi_tf, red);
}

// H phi_k at every grid point: linear part (finite differences, or the
// precomputed L of DVR / spectral derivatives) plus the interacting part
// sum_s conj(f_s) sum_{q,l} Q[k,s,q,l] f_q f_l
__global__ void orb_haction_kernel(OrbView o, const double2* __restrict__ y,
                                   const double2* __restrict__ Q, const double2* __restrict__ L,
                                   double2* __restrict__ H) {
    const int M = o.M, G = o.G;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * G) return;
    const int k = t / G, x = t % G;
    const double2* f = y + (size_t)k * G;
    const double2 lin = L ? L[t] : linear_at(o, f, x);  // split_linear_orbitals.c:210-255
    // interacting part
    double2 fx[kMaxOrb];
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

// proj[s][k] = <f_s | H_k> (Simpson), one block per (s, k)
__global__ void orb_overlap_kernel(OrbView o, const double2* __restrict__ y,
                                   const double2* __restrict__ H, double2* __restrict__ P) {
    const int M = o.M, G = o.G;
    const int s = blockIdx.x / M, k = blockIdx.x % M;
    double2 acc = make_double2(0.0, 0.0);
    for (int x = threadIdx.x; x < G; x += blockDim.x) {
        const double2 t = cfma_conj(y[(size_t)s * G + x], H[(size_t)k * G + x],
                                    make_double2(0.0, 0.0));
        acc.x += o.w[x] * t.x;
        acc.y += o.w[x] * t.y;
    }
    const double2 r = block_sum(acc);
    if (threadIdx.x == 0) P[s * M + k] = r;
}

// robust projector (orbital_integration.c:22-92): P <- S^{-1} P with the full
// overlap matrix S_sl = <f_s|f_l> (the reference's set_overlap_matrix,
// orbital_matrices.c:7-19, starts its inner loop at 2 and leaves S_01 and
// S_10 unset; the full matrix is its evident intent).  One thread: M <= 30.
// A singular S sets *fail and leaves P as the simple projector's.
__global__ void orb_robust_kernel(int M, const double2* __restrict__ S, double2* __restrict__ P,
                                  double2* __restrict__ work, int* __restrict__ fail) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int M2 = M * M;
    double2 *a = work, *inv = work + M2, *t = work + 2 * M2;
    for (int i = 0; i < M2; i++) a[i] = S[i];
    if (herm_inverse(M, a, inv)) {
        *fail = 1;
        return;
    }
    for (int s = 0; s < M; s++)
        for (int k = 0; k < M; k++) {
            double2 z = make_double2(0.0, 0.0);
            for (int l = 0; l < M; l++) z = cfma(inv[s * M + l], P[l * M + k], z);
            t[s * M + k] = z;
        }
    for (int i = 0; i < M2; i++) P[i] = t[i];
}

// dy/dt = -i tf (H_k - sum_s f_s <f_s|H_k>)
__global__ void orb_rhs_finish_kernel(OrbView o, const double2* __restrict__ y,
                                      const double2* __restrict__ H,
                                      const double2* __restrict__ P, double2* __restrict__ out) {
    const int M = o.M, G = o.G;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * G) return;
    const int k = t / G, x = t % G;
    double2 proj = make_double2(0.0, 0.0);
    for (int s = 0; s < M; s++) proj = cfma(y[(size_t)s * G + x], P[s * M + k], proj);
    const double2 d = make_double2(H[t].x - proj.x, H[t].y - proj.y);
    // -i * tf * d
    const double2 mi_tf = make_double2(o.tf.y, -o.tf.x);
    out[t] = cmul(mi_tf, d);
}

// y_out = y + dt sum_j c_j k_j
struct RkCombo {
    const double2* k[6];
    double c[6];
    int n;
};
__global__ void rk_combo_kernel(int total, const double2* __restrict__ y, RkCombo cb, double dt,
                                double2* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    double2 s = make_double2(0.0, 0.0);
    for (int j = 0; j < cb.n; j++) {
        s.x += cb.c[j] * cb.k[j][t].x;
        s.y += cb.c[j] * cb.k[j][t].y;
    }
    out[t] = make_double2(y[t].x + dt * s.x, y[t].y + dt * s.y);
}

__global__ void periodic_kernel(int M, int G, double2* orb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < M) orb[(size_t)k * G + G - 1] = orb[(size_t)k * G];
}

// orthonormalize (calculus.c:171-191) in one block (orthonormalize_block)
__global__ void orthonormalize_kernel(OrbView o, double2* __restrict__ F) {
    extern __shared__ double scan[];  // G doubles
    orthonormalize_block(o, F, scan);
}

// rho1 <- regularised rho1, rinv = rho1^{-1} (one thread; M <= 30).  With
// dynamic shared memory (smem > 0) the matrices are staged there: the
// routine's thousands of dependent accesses then stay on the SM instead of
// going to L2 (about 1 ms at M = 8 in global memory); same operations, same
// bits.
__global__ void sync_rho1_kernel(int M, double2* rho1, double2* rinv, double reg_fac,
                                 double2* work, int* info, int smem) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int M2 = M * M;
    if (smem > 0) {
        extern __shared__ double2 sh[];
        double2 *r1 = sh, *ri = sh + M2, *w = sh + 2 * M2;
        for (int i = 0; i < M2; i++) r1[i] = rho1[i];
        const int r = sync_rho1(M, r1, ri, reg_fac, w, (double*)(w + 3 * M2));
        for (int i = 0; i < M2; i++) {
            rho1[i] = r1[i];
            rinv[i] = ri[i];
        }
        if (info) *info = r;
        return;
    }
    double* wd = (double*)(work + 3 * M2);
    const int r = sync_rho1(M, rho1, rinv, reg_fac, work, wd);
    if (info) *info = r;
}

// total energy (integrator_monitor.c:56-88) in one block (energy_block)
__global__ void energy_kernel(int M, const double2* __restrict__ rho1,
                              const double2* __restrict__ rho2, const double2* __restrict__ hob,
                              const double2* __restrict__ hint, double2* __restrict__ E) {
    const double2 s = energy_block(M, rho1, rho2, hob, hint);
    if (threadIdx.x == 0) *E = s;
}

// ---------------------------------------------------------------------------
int orb_init(OrbCtx& c, int M, int G, double xi, double xf, double a2, double2 a1, int periodic,
             int imagtime) {
    if (M < 1 || M > kMaxOrb || G < 5) {
        set_error("orbital grid: %d orbitals, %d points (need 1..%d, >= 5)", M, G, kMaxOrb);
        return -1;
    }
    c.M = M;
    c.G = G;
    const double dx = (xf - xi) / (G - 1);
    const size_t n = (size_t)M * G;
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_w, G * sizeof(double)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_pot, G * sizeof(double)));
    MCTDHB_CUDA_TRY(cudaMemset(c.d_pot, 0, G * sizeof(double)));
    const std::vector<double> w = simpson_weights(G, dx);
    MCTDHB_CUDA_TRY(cudaMemcpy(c.d_w, w.data(), G * sizeof(double), cudaMemcpyHostToDevice));
    for (int i = 0; i < 8; i++) MCTDHB_CUDA_TRY(cudaMalloc(&c.d_k[i], n * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_H, n * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_P, (size_t)M * M * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_Q, (size_t)M * M * M * M * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_g, sizeof(double)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_work, (3 * (size_t)M * M + M + 2) * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_S, (size_t)M * M * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_fail, sizeof(int)));
    MCTDHB_CUDA_TRY(cudaMemset(c.d_fail, 0, sizeof(int)));
    c.view.M = M;
    c.view.G = G;
    c.view.dx = dx;
    c.view.a2 = a2;
    c.view.a1 = a1;
    c.view.periodic = periodic;
    c.view.tf = imagtime ? make_double2(0.0, -1.0) : make_double2(1.0, 0.0);
    c.view.w = c.d_w;
    c.view.pot = c.d_pot;
    return 0;
}

void orb_release(OrbCtx& c) {
    cudaFree(c.d_w);
    cudaFree(c.d_pot);
    for (int i = 0; i < 8; i++) cudaFree(c.d_k[i]);
    cudaFree(c.d_H);
    cudaFree(c.d_P);
    cudaFree(c.d_Q);
    cudaFree(c.d_g);
    cudaFree(c.d_work);
    cudaFree(c.d_S);
    cudaFree(c.d_fail);
    cudaFree(c.d_lin_t);
    cudaFree(c.d_L);
    cudaFree(c.d_half);
    cudaFree(c.d_B);
    c = OrbCtx();
}

int orb_matrices(const OrbCtx& c, const double2* orb, double2* hob, double2* hint,
                 cudaStream_t st) {
    const int M = c.M;
    hob_kernel<<<M * (M + 1) / 2, 256, 0, st>>>(c.view, orb, hob);
    const int tiles = (M * M + 7) / 8;
    const int warps = tiles * tiles;
    hint_dmma_kernel<<<(warps + 3) / 4, 128, 0, st>>>(c.view, orb, c.d_g, hint);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int orb_rhs(const OrbCtx& c, const double2* y, double2* out, cudaStream_t st) {
    const int n = c.M * c.G;
    const double2* L = nullptr;
    if (c.view.lin_t) {
        const dim3 grid((c.G + 255) / 256, c.M);
        orb_toeplitz_kernel<<<grid, 256, (size_t)(c.G - 1) * sizeof(double2), st>>>(c.view, y,
                                                                                   c.d_L);
        L = c.d_L;
    }
    orb_haction_kernel<<<(n + 127) / 128, 128, 0, st>>>(c.view, y, c.d_Q, L, c.d_H);
    orb_overlap_kernel<<<c.M * c.M, 256, 0, st>>>(c.view, y, c.d_H, c.d_P);
    if (c.robust) {
        orb_overlap_kernel<<<c.M * c.M, 256, 0, st>>>(c.view, y, y, c.d_S);
        orb_robust_kernel<<<1, 32, 0, st>>>(c.M, c.d_S, c.d_P, c.d_work, c.d_fail);
    }
    orb_rhs_finish_kernel<<<(n + 255) / 256, 256, 0, st>>>(c.view, y, c.d_H, c.d_P, out);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int combo(const OrbCtx& c, const double2* y, std::initializer_list<std::pair<int, double>> t,
                 double dt, double2* out, cudaStream_t st) {
    RkCombo cb{};
    cb.n = 0;
    for (auto& p : t) {
        cb.k[cb.n] = c.d_k[p.first];
        cb.c[cb.n] = p.second;
        cb.n++;
    }
    const int n = c.M * c.G;
    rk_combo_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, y, cb, dt, out);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

// right-hand side of one RK stage: full step (orb_rhs) or the split step's
// nonlinear part (Q, c.split_hob and c.d_B prepared)
static int stage_rhs(const OrbCtx& c, bool split, const double2* y, double2* out,
                     cudaStream_t st) {
    if (!split) return orb_rhs(c, y, out, st);
    const int n = c.M * c.G;
    orb_split_rhs_kernel<<<(n + 127) / 128, 128, 0, st>>>(c.view, y, c.d_Q, c.split_hob, c.d_B,
                                                          out);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int rk_stages(const OrbCtx& c, bool split, int order, double dt, const double2* y,
                     double2* ynext, cudaStream_t st) {
    auto orb_rhs = [&](const OrbCtx& cc, const double2* yy, double2* out, cudaStream_t s2) {
        return stage_rhs(cc, split, yy, out, s2);
    };
    double2* const* k = c.d_k;
    double2* w = c.d_k[6];
    int rc = 0;
    if (order == 2) {
        rc |= orb_rhs(c, y, k[0], st);
        rc |= combo(c, y, {{0, 1.0}}, dt, w, st);
        rc |= orb_rhs(c, w, k[1], st);
        rc |= combo(c, y, {{0, 0.5}, {1, 0.5}}, dt, ynext, st);
    } else if (order == 4) {
        rc |= orb_rhs(c, y, k[0], st);
        rc |= combo(c, y, {{0, 0.5}}, dt, w, st);
        rc |= orb_rhs(c, w, k[1], st);
        rc |= combo(c, y, {{1, 0.5}}, dt, w, st);
        rc |= orb_rhs(c, w, k[2], st);
        rc |= combo(c, y, {{2, 1.0}}, dt, w, st);
        rc |= orb_rhs(c, w, k[3], st);
        rc |= combo(c, y, {{0, 1.0 / 6}, {1, 2.0 / 6}, {2, 2.0 / 6}, {3, 1.0 / 6}}, dt, ynext, st);
    } else if (order == 5) {
        rc |= orb_rhs(c, y, k[0], st);
        rc |= combo(c, y, {{0, 0.25}}, dt, w, st);
        rc |= orb_rhs(c, w, k[1], st);
        rc |= combo(c, y, {{0, 0.125}, {1, 0.125}}, dt, w, st);
        rc |= orb_rhs(c, w, k[2], st);
        rc |= combo(c, y, {{1, -0.5}, {2, 1.0}}, dt, w, st);
        rc |= orb_rhs(c, w, k[3], st);
        rc |= combo(c, y, {{0, 3.0 / 16}, {3, 9.0 / 16}}, dt, w, st);
        rc |= orb_rhs(c, w, k[4], st);
        rc |= combo(c, y, {{0, -3.0 / 7}, {1, 2.0 / 7}, {2, 12.0 / 7}, {3, -12.0 / 7}, {4, 8.0 / 7}},
                    dt, w, st);
        rc |= orb_rhs(c, w, k[5], st);
        rc |= combo(c, y,
                    {{0, 7.0 / 90}, {2, 32.0 / 90}, {3, 12.0 / 90}, {4, 32.0 / 90}, {5, 7.0 / 90}},
                    dt, ynext, st);
    } else {
        set_error("Runge-Kutta order %d not in {2, 4, 5}", order);
        return -1;
    }
    return rc ? -1 : 0;
}

int orb_rk_step(const OrbCtx& c, int order, double dt, const double2* rinv, const double2* rho2,
                const double2* y, double2* ynext, cudaStream_t st) {
    const int M = c.M, M4 = M * M * M * M;
    orb_q_kernel<<<(M4 + 127) / 128, 128, 0, st>>>(M, c.d_g, rinv, rho2, c.d_Q);
    return rk_stages(c, false, order, dt, y, ynext, st);
}

// apply the half-step operator to every orbital of y (in place, through
// the spare stage buffer)
static int half_step(const OrbCtx& c, double2* y, cudaStream_t st) {
    const int G = c.G;
    const int nn = c.half_dense ? G : G - 1;
    const dim3 grid((G + 255) / 256, c.M);
    orb_half_kernel<<<grid, 256, (size_t)nn * sizeof(double2), st>>>(c.view, c.d_half,
                                                                      c.half_dense, y, c.d_k[7]);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(y, c.d_k[7], (size_t)c.M * G * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, st));
    return 0;
}

int orb_split_step(OrbCtx& c, int order, double dt, const double2* rinv, const double2* rho2,
                   double2* y, double2* ynext, double2* hob, double2* hint, cudaStream_t st) {
    if (!c.split || !c.d_half) {
        set_error("orb_split_step: split-step operator not set up");
        return -1;
    }
    const int M = c.M, M4 = M * M * M * M;
    if (half_step(c, y, st)) return -1;
    // h and g of the half-stepped orbitals (the reference's
    // sync_orbital_matrices inside propagate_splitstep_orb)
    if (orb_matrices(c, y, hob, hint, st)) return -1;
    orb_q_kernel<<<(M4 + 127) / 128, 128, 0, st>>>(M, c.d_g, rinv, rho2, c.d_Q);
    orb_bmat_kernel<<<(M * M + 63) / 64, 64, 0, st>>>(M, rinv, rho2, hint, c.d_B);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    c.split_hob = hob;
    if (rk_stages(c, true, order, dt, y, ynext, st)) return -1;
    return half_step(c, ynext, st);
}

int orb_rhs_eval(const OrbCtx& c, const double2* rinv, const double2* rho2, const double2* y,
                 double2* out, cudaStream_t st) {
    const int M = c.M, M4 = M * M * M * M;
    orb_q_kernel<<<(M4 + 127) / 128, 128, 0, st>>>(M, c.d_g, rinv, rho2, c.d_Q);
    return orb_rhs(c, y, out, st);
}

int orb_periodic(const OrbCtx& c, double2* orb, cudaStream_t st) {
    periodic_kernel<<<1, 32, 0, st>>>(c.M, c.G, orb);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Toeplitz kernel of the DVR / spectral derivative part on n = G - 1 points,
// t[d + n - 1] for d = j - i in (-n, n), with a2, a1 folded in.
//   DVR (split_linear_orbitals.c:83-166): first and second derivatives in the
//     exponential basis, kmom = k - n/2; for d > 0 the element is
//     sum_k g(kmom) e^{2 pi i kmom d / n} / n, for d < 0 the conjugate
//     (second derivative) or minus the conjugate (first), on the diagonal
//     sum_k g(kmom) / n, with g1 = -2 pi i kmom / L, g2 = -(2 pi kmom / L)^2.
//   spectral (split_linear_orbitals.c:257-287, calculus.c:272-285): the
//     circulant of FFT -> (i freq a1 - freq^2 a2) -> inverse FFT with
//     1/sqrt(n) both ways: t[d + n - 1] = c[(-d) mod n],
//     c[e] = sum_m mult_m e^{2 pi i m e / n} / n.
std::vector<double2> derivative_toeplitz(int der, int G, double dx, double a2,
                                         std::complex<double> a1) {
    using cd = std::complex<double>;
    const int n = G - 1;
    const double pi = 3.14159265358979323846, len = n * dx;
    // e^{2 pi i m / n}, m = 0 .. n-1
    std::vector<cd> ex(n);
    for (int m = 0; m < n; m++) ex[m] = std::polar(1.0, 2.0 * pi * m / n);
    std::vector<double2> t(2 * (size_t)n - 1);
    auto put = [&](int d, cd v) { t[d + n - 1] = make_double2(v.real(), v.imag()); };
    if (der == kDerDVR) {
        for (int d = 0; d < n; d++) {
            cd s1 = 0.0, s2 = 0.0;
            for (int k = 0; k < n; k++) {
                const int kmom = k - n / 2;
                const cd g1 = cd(0.0, -2.0 * pi * kmom / len);
                const double g2 = -(2.0 * pi * kmom / len) * (2.0 * pi * kmom / len);
                const long ph = (((long)kmom * d) % n + n) % n;
                s1 += g1 * ex[ph] / (double)n;
                s2 += g2 * ex[ph] / (double)n;
            }
            if (d == 0) {
                put(0, a2 * s2 + a1 * s1);
            } else {
                put(d, a2 * s2 + a1 * s1);
                put(-d, a2 * std::conj(s2) - a1 * std::conj(s1));
            }
        }
    } else {
        std::vector<cd> mult(n), c(n);
        for (int m = 0; m < n; m++) {
            const double freq = m <= (n - 1) / 2 ? 2.0 * pi * m / len : 2.0 * pi * (m - n) / len;
            mult[m] = freq * cd(0.0, 1.0) * a1 - freq * freq * a2;
        }
        for (int e = 0; e < n; e++) {
            cd z = 0.0;
            for (int m = 0; m < n; m++) z += mult[m] * ex[((long)m * e) % n];
            c[e] = z / (double)n;
        }
        for (int d = -(n - 1); d < n; d++) put(d, c[((-d) % n + n) % n]);
    }
    return t;
}

int orb_set_derivative(OrbCtx& c, int der) {
    if (der == c.der) return 0;
    if (der != kDerFiniteDiff && der != kDerDVR && der != kDerSpectral) {
        set_error("orbital derivative method %d not in {300 DVR, 301 SPECTRAL, 302 FINITEDIFF}",
                  der);
        return -1;
    }
    if (der != kDerFiniteDiff && !c.view.periodic) {
        set_error("DVR and spectral derivatives need periodic boundaries");
        return -1;
    }
    if (der != kDerFiniteDiff && c.G - 1 > 8191) {
        set_error("DVR / spectral derivatives: grid of %d points above 8192", c.G);
        return -1;
    }
    cudaFree(c.d_lin_t);
    cudaFree(c.d_L);
    c.d_lin_t = c.d_L = nullptr;
    c.view.lin_t = nullptr;
    c.der = kDerFiniteDiff;
    if (der == kDerFiniteDiff) return 0;
    const std::vector<double2> t = derivative_toeplitz(
        der, c.G, c.view.dx, c.view.a2, std::complex<double>(c.view.a1.x, c.view.a1.y));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_lin_t, t.size() * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_L, (size_t)c.M * c.G * sizeof(double2)));
    MCTDHB_CUDA_TRY(
        cudaMemcpy(c.d_lin_t, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice));
    MCTDHB_CUDA_TRY(cudaFuncSetAttribute(orb_toeplitz_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)((size_t)(c.G - 1) * sizeof(double2))));
    c.view.lin_t = c.d_lin_t;
    c.der = der;
    return 0;
}

// Half-step operator of the split-step integrator for dth = prop_dt / 2
// (LINEAR_TSTEP_FRAC of split_linear_orbitals.h):
//   finite differences, Crank-Nicolson (split_linear_orbitals.c:23-56,
//     289-373): Op = A^{-1} B with A = i + dth (a2 D2 + a1 D1),
//     B = i - dth (a2 D2 + a1 D1) in the reference's tridiagonal entries;
//     periodic grids: A and B are circulant on the G - 1 distinct points, so
//     Op is the circulant with eigenvalues lambda_B / lambda_A; zero bounds:
//     Op dense, column by column by the Thomas algorithm
//   DVR / spectral, FFT exponential (:57-82, 375-402): the circulant with
//     eigenvalues exp(-i dth (i freq a1 - freq^2 a2)) at the FFT frequencies
int split_half_operator(int G, double dx, double a2, double2 a1v, int periodic, int der,
                        double dt, int imagtime, std::vector<double2>& op, int* dense) {
    using cd = std::complex<double>;
    const bool fd = der == kDerFiniteDiff;
    if (!periodic && !fd) {
        set_error("split step: the FFT exponential needs periodic boundaries");
        return -1;
    }
    if ((periodic && G - 1 > 8191) || (!periodic && G > 2048)) {
        set_error("split step: grid of %d points above the operator's limit", G);
        return -1;
    }
    const double pi = 3.14159265358979323846;
    const cd a1(a1v.x, a1v.y), I(0.0, 1.0);
    const cd dth = 0.5 * (imagtime ? cd(0.0, -dt) : cd(dt, 0.0));
    const cd mid = I + a2 * dth / dx / dx, up = -a2 * dth / dx / dx / 2.0 - a1 * dth / dx / 4.0,
             lo = -a2 * dth / dx / dx / 2.0 + a1 * dth / dx / 4.0;
    const cd rmid = I - a2 * dth / dx / dx;
    op.clear();
    if (periodic) {
        const int n = G - 1;
        std::vector<cd> ex(n), mu(n), cop(n);
        for (int m = 0; m < n; m++) ex[m] = std::polar(1.0, 2.0 * pi * m / n);
        for (int m = 0; m < n; m++) {
            if (fd) {
                const cd w = ex[m], wi = std::conj(ex[m]);
                mu[m] = (rmid - up * w - lo * wi) / (mid + up * w + lo * wi);
            } else {
                const double freq = m <= (n - 1) / 2 ? 2.0 * pi * m / (n * dx)
                                                     : 2.0 * pi * (m - n) / (n * dx);
                mu[m] = std::exp(-I * dth * (I * a1 * freq - a2 * freq * freq));
            }
        }
        // c_op[d] = (1/n) sum_m mu_m e^{-2 pi i m d / n}
        for (int d = 0; d < n; d++) {
            cd z = 0.0;
            for (int m = 0; m < n; m++) z += mu[m] * std::conj(ex[((long)m * d) % n]);
            cop[d] = z / (double)n;
        }
        op.resize(2 * (size_t)n - 1);
        for (int d = -(n - 1); d < n; d++) {
            const cd v = cop[((d % n) + n) % n];
            op[d + n - 1] = make_double2(v.real(), v.imag());
        }
    } else {
        // zero bounds: columns of A^{-1} B (A, B tridiagonal on all G points)
        op.resize((size_t)G * G);
        std::vector<cd> cc(G), dd(G), b(G), x(G);
        for (int j = 0; j < G; j++) {
            for (int i = 0; i < G; i++) b[i] = 0.0;
            b[j] = rmid;
            if (j > 0) b[j - 1] = -up;  // B[j-1][j]
            if (j + 1 < G) b[j + 1] = -lo;  // B[j+1][j]
            cc[0] = up / mid;
            dd[0] = b[0] / mid;
            for (int i = 1; i < G; i++) {
                const cd den = mid - lo * cc[i - 1];
                cc[i] = up / den;
                dd[i] = (b[i] - lo * dd[i - 1]) / den;
            }
            x[G - 1] = dd[G - 1];
            for (int i = G - 2; i >= 0; i--) x[i] = dd[i] - cc[i] * x[i + 1];
            for (int i = 0; i < G; i++)
                op[(size_t)j * G + i] = make_double2(x[i].real(), x[i].imag());
        }
    }
    *dense = periodic ? 0 : 1;
    return 0;
}

int orb_set_split(OrbCtx& c, int split, double dt, int imagtime) {
    cudaFree(c.d_half);
    cudaFree(c.d_B);
    c.d_half = nullptr;
    c.d_B = nullptr;
    c.split = 0;
    if (!split) return 0;
    const int G = c.G;
    std::vector<double2> op;
    int dense = 0;
    if (split_half_operator(G, c.view.dx, c.view.a2, c.view.a1, c.view.periodic, c.der, dt,
                            imagtime, op, &dense))
        return -1;
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_half, op.size() * sizeof(double2)));
    MCTDHB_CUDA_TRY(
        cudaMemcpy(c.d_half, op.data(), op.size() * sizeof(double2), cudaMemcpyHostToDevice));
    MCTDHB_CUDA_TRY(cudaMalloc(&c.d_B, (size_t)c.M * c.M * sizeof(double2)));
    const int nn = dense ? G : G - 1;
    MCTDHB_CUDA_TRY(cudaFuncSetAttribute(orb_half_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)((size_t)nn * sizeof(double2))));
    c.half_dense = dense;
    c.split = 1;
    return 0;
}

int orb_overlap_matrix(const OrbCtx& c, const double2* orb, cudaStream_t st) {
    orb_overlap_kernel<<<c.M * c.M, 256, 0, st>>>(c.view, orb, orb, c.d_S);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int orb_orthonormalize(const OrbCtx& c, double2* orb, cudaStream_t st) {
    const size_t smem = (size_t)c.G * sizeof(double);
    if (smem > 48 * 1024) {
        set_error("orthonormalize: grid of %d points exceeds the block scan", c.G);
        return -1;
    }
    orthonormalize_kernel<<<1, 256, smem, st>>>(c.view, orb);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int orb_sync_rho1(const OrbCtx& c, double2* rho1, double2* rinv, double reg_fac, int* d_info,
                  cudaStream_t st) {
    // rho1, rinv and the 3 M^2 + M work values in shared memory up to 48 KB
    const size_t sm = (size_t)(5 * c.M * c.M) * sizeof(double2) + (size_t)c.M * sizeof(double);
    const int smem = sm <= 48 * 1024 ? (int)sm : 0;
    sync_rho1_kernel<<<1, 32, smem, st>>>(c.M, rho1, rinv, reg_fac, c.d_work, d_info, smem);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int orb_energy(int M, const double2* rho1, const double2* rho2, const double2* hob,
               const double2* hint, double2* E, cudaStream_t st) {
    energy_kernel<<<1, 256, 0, st>>>(M, rho1, rho2, hob, hint, E);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mctdhb
