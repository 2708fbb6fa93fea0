// orbital.cu -- the orbital side of one MCTDHB step on the device:
//   h_kl                 set_orbital_hob     (orbital_matrices.c:22-70)
//   g_ksql               set_orbital_hint    (orbital_matrices.c:73-287),
//                        as one (M^2 x G)(G x M^2) complex contraction on the
//                        FP64 tensor cores (mma.sync m8n8k4 f64)
//   orbital equation     dodt_fullstep_interface (orbital_integration.c:179-240)
//                        with the finite-difference linear part
//                        (split_linear_orbitals.c:210-255), the interacting
//                        part (split_nonlinear_orbitals.c:4-61) and the simple
//                        projector (orbital_integration.c:95-131)
//   Runge-Kutta step     propagate_fullstep_orb_rk (orbital_integration.c:284)
//                        with the named tableaux Heun / classical RK4 /
//                        Butcher RK5
//   Gram-Schmidt         orthonormalize (calculus.c:171-191)
//   rho1 synchronisation sync_density_matrices (synchronize.c:42-57)
// Grid functions are row-major M x G complex128; integrals use the composite
// Simpson weights of calculus.c:9-40 (3/8 rule on the last four points for
// an even number of points).
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "orbital.h"
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

// periodic fourth-order first derivative (calculus.c:288-305): the grid has
// P = G - 1 distinct points, f[G-1] is the copy of f[0]
__device__ __forceinline__ double2 dxfd_at(const double2* f, int G, int i, double r) {
    const int P = G - 1;
    if (i == G - 1) i = 0;
    const double2 a = f[(i - 2 + P) % P], b = f[(i + 2) % P], c = f[(i + 1) % P],
                  d = f[(i - 1 + P) % P];
    return make_double2((a.x - b.x + 8 * (c.x - d.x)) * r, (a.y - b.y + 8 * (c.y - d.y)) * r);
}

__device__ __forceinline__ double2 block_sum(double2 v) {
    __shared__ double2 red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double2 s = make_double2(0.0, 0.0);
    for (int i = 0; i < nw; i++) {
        s.x += red[i].x;
        s.y += red[i].y;
    }
    return s;  // every thread gets the block sum
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
    const double a2 = o.a2;
    const double2 a1 = o.a1;
    double2 acc = make_double2(0.0, 0.0);
    for (int x = threadIdx.x; x < G; x += blockDim.x) {
        const double2 dk = dxfd_at(fk, G, x, r), dl = dxfd_at(fl, G, x, r);
        const double2 ck = make_double2(fk[x].x, -fk[x].y);
        // -a2 conj(dk) dl + a1 conj(fk) dl + V conj(fk) fl
        double2 t = cmul(make_double2(-a2 * dk.x, a2 * dk.y), dl);
        t = cadd(t, cmul(cmul(a1, ck), dl));
        t = cadd(t, cscale(cmul(ck, fl[x]), o.pot[x]));
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

// g_ksql = g sum_x w_x conj(f_k f_s) f_q f_l as a complex GEMM
//   Out[r][c] = sum_x A[r][x] B[x][c],  A = w conj(P), B = P,
//   P_r(x) = f_a(x) f_b(x), r = a + b M  -> hint[r + M^2 c]
// on the FP64 tensor cores: one warp per 8 x 8 tile, mma.sync m8n8k4 f64.
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void hint_dmma_kernel(OrbView o, const double2* __restrict__ orb,
                                 const double* __restrict__ g_dev, double2* __restrict__ hint) {
    const int M = o.M, G = o.G, M2 = M * M;
    const int tiles = (M2 + 7) / 8;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= tiles * tiles) return;
    const int R0 = (warp / tiles) * 8, C0 = (warp % tiles) * 8;
    const int ra = R0 + (lane >> 2);  // A row held by this lane
    const int cb = C0 + (lane >> 2);  // B column held by this lane
    const int kk = lane & 3;          // k offset within the 4-wide step
    const bool rv = ra < M2, cv = cb < M2;
    const double2* fa1 = orb + (size_t)(rv ? ra % M : 0) * G;
    const double2* fa2 = orb + (size_t)(rv ? ra / M : 0) * G;
    const double2* fb1 = orb + (size_t)(cv ? cb % M : 0) * G;
    const double2* fb2 = orb + (size_t)(cv ? cb / M : 0) * G;
    double rr0 = 0, rr1 = 0, ii0 = 0, ii1 = 0, im0 = 0, im1 = 0;
    for (int x0 = 0; x0 < G; x0 += 4) {
        const int x = x0 + kk;
        double ar = 0, ai = 0, br = 0, bi = 0;
        if (x < G) {
            if (rv) {
                const double2 p = cmul(fa1[x], fa2[x]);
                ar = o.w[x] * p.x;  // w conj(P)
                ai = -o.w[x] * p.y;
            }
            if (cv) {
                const double2 p = cmul(fb1[x], fb2[x]);
                br = p.x;
                bi = p.y;
            }
        }
        dmma(rr0, rr1, ar, br);  // sum Ar Br
        dmma(ii0, ii1, ai, bi);  // sum Ai Bi
        dmma(im0, im1, ar, bi);  // sum Ar Bi + Ai Br
        dmma(im0, im1, ai, br);
    }
    const double g = *g_dev;
    const int row = R0 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int col = C0 + (lane & 3) * 2 + j;
        if (row < M2 && col < M2) {
            const double re = j ? rr1 - ii1 : rr0 - ii0;
            const double im = j ? im1 : im0;
            hint[row + (size_t)M2 * col] = make_double2(g * re, g * im);
        }
    }
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

// H phi_k at every grid point: linear part (finite differences) plus the
// interacting part sum_s conj(f_s) sum_{q,l} Q[k,s,q,l] f_q f_l
__global__ void orb_haction_kernel(OrbView o, const double2* __restrict__ y,
                                   const double2* __restrict__ Q, double2* __restrict__ H) {
    const int M = o.M, G = o.G;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * G) return;
    const int k = t / G, x = t % G;
    const double2* f = y + (size_t)k * G;
    // split_linear_orbitals.c:210-255
    const double a2 = o.a2, dx = o.dx;
    const double2 a1 = o.a1;
    const double2 up = make_double2(a2 / dx / dx + a1.x / dx / 2, a1.y / dx / 2);
    const double2 lo = make_double2(a2 / dx / dx - a1.x / dx / 2, -a1.y / dx / 2);
    double2 lin;
    if (o.periodic) {
        if (x == G - 1) {
            // out[G-1] = out[0]
            const double mid = -2 * a2 / dx / dx + o.pot[0];
            lin = cadd(cadd(cscale(f[0], mid), cmul(up, f[1])), cmul(lo, f[G - 2]));
        } else if (x == 0) {
            const double mid = -2 * a2 / dx / dx + o.pot[0];
            lin = cadd(cadd(cscale(f[0], mid), cmul(up, f[1])), cmul(lo, f[G - 2]));
        } else if (x == G - 2) {
            const double mid = -2 * a2 / dx / dx + o.pot[G - 2];
            lin = cadd(cadd(cscale(f[G - 2], mid), cmul(up, f[0])), cmul(lo, f[G - 3]));
        } else {
            const double mid = -2 * a2 / dx / dx + o.pot[x];
            lin = cadd(cadd(cscale(f[x], mid), cmul(up, f[x + 1])), cmul(lo, f[x - 1]));
        }
    } else {
        const double mid = -2 * a2 / dx / dx + o.pot[x];
        if (x == 0)
            lin = cadd(cscale(f[0], mid), cmul(up, f[1]));
        else if (x == G - 1)
            lin = cadd(cscale(f[G - 1], mid), cmul(lo, f[G - 2]));
        else
            lin = cadd(cadd(cscale(f[x], mid), cmul(up, f[x + 1])), cmul(lo, f[x - 1]));
    }
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

// orthonormalize (calculus.c:171-191) in one block.  The reference
// re-evaluates <F_j|F_i> for every grid point k while F_i is being updated;
// that overlap obeys ov_{k+1} = ov_k (1 - w_k |F_j[k]|^2), so the update is a
// prefix product, evaluated here with a block scan.
__global__ void orthonormalize_kernel(OrbView o, double2* __restrict__ F) {
    const int M = o.M, G = o.G;
    __shared__ double2 ovs;
    __shared__ double carry;
    extern __shared__ double scan[];  // G doubles
    auto renorm = [&](double2* f) {
        double acc = 0.0;
        for (int x = threadIdx.x; x < G; x += blockDim.x) acc += o.w[x] * (f[x].x * f[x].x + f[x].y * f[x].y);
        const double s = block_sum(make_double2(acc, 0.0)).x;
        const double r = sqrt(1.0 / s);
        __syncthreads();
        for (int x = threadIdx.x; x < G; x += blockDim.x) f[x] = cscale(f[x], r);
        __syncthreads();
    };
    renorm(F);
    for (int i = 1; i < M; i++) {
        double2* fi = F + (size_t)i * G;
        for (int j = 0; j < i; j++) {
            const double2* fj = F + (size_t)j * G;
            double2 acc = make_double2(0.0, 0.0);
            for (int x = threadIdx.x; x < G; x += blockDim.x) {
                const double2 t = cfma_conj(fj[x], fi[x], make_double2(0.0, 0.0));
                acc.x += o.w[x] * t.x;
                acc.y += o.w[x] * t.y;
            }
            const double2 ov0 = block_sum(acc);
            if (threadIdx.x == 0) ovs = ov0;
            // factors (1 - w_x |F_j[x]|^2), exclusive prefix product
            for (int x = threadIdx.x; x < G; x += blockDim.x)
                scan[x] = 1.0 - o.w[x] * (fj[x].x * fj[x].x + fj[x].y * fj[x].y);
            __syncthreads();
            if (threadIdx.x == 0) {
                double p = 1.0;
                for (int x = 0; x < G; x++) {
                    const double f = scan[x];
                    scan[x] = p;
                    p *= f;
                }
                carry = p;
            }
            __syncthreads();
            const double2 ov = ovs;
            for (int x = threadIdx.x; x < G; x += blockDim.x) {
                const double2 c = cscale(ov, scan[x]);
                const double2 t = cmul(c, fj[x]);
                fi[x].x -= t.x;
                fi[x].y -= t.y;
            }
            __syncthreads();
        }
        renorm(fi);
    }
}

// rho1 <- regularised rho1, rinv = rho1^{-1} (one thread; M <= 30)
__global__ void sync_rho1_kernel(int M, double2* rho1, double2* rinv, double reg_fac,
                                 double2* work, int* info) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double* wd = (double*)(work + 3 * M * M);
    const int r = sync_rho1(M, rho1, rinv, reg_fac, work, wd);
    if (info) *info = r;
}

// E = sum_kl rho1[k][l] h[k][l] + 1/2 sum rho2[k,l,s,q] g[k,l,q,s]
// (integrator_monitor.c:56-88)
__global__ void energy_kernel(int M, const double2* __restrict__ rho1,
                              const double2* __restrict__ rho2, const double2* __restrict__ hob,
                              const double2* __restrict__ hint, double2* __restrict__ E) {
    const int M2 = M * M, M3 = M2 * M, M4 = M3 * M;
    double2 acc = make_double2(0.0, 0.0);
    for (int e = threadIdx.x; e < M4; e += blockDim.x) {
        const int k = e % M, l = (e / M) % M, s = (e / M2) % M, q = e / M3;
        acc = cfma(rho2[k + l * M + s * M2 + q * M3], hint[k + l * M + q * M2 + s * M3], acc);
    }
    acc = cscale(acc, 0.5);
    for (int e = threadIdx.x; e < M2; e += blockDim.x) acc = cfma(rho1[e], hob[e], acc);
    const double2 s = block_sum(acc);
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
    orb_haction_kernel<<<(n + 127) / 128, 128, 0, st>>>(c.view, y, c.d_Q, c.d_H);
    orb_overlap_kernel<<<c.M * c.M, 256, 0, st>>>(c.view, y, c.d_H, c.d_P);
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

int orb_rk_step(const OrbCtx& c, int order, double dt, const double2* rinv, const double2* rho2,
                const double2* y, double2* ynext, cudaStream_t st) {
    const int M = c.M, M4 = M * M * M * M;
    orb_q_kernel<<<(M4 + 127) / 128, 128, 0, st>>>(M, c.d_g, rinv, rho2, c.d_Q);
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
    sync_rho1_kernel<<<1, 32, 0, st>>>(c.M, rho1, rinv, reg_fac, c.d_work, d_info);
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
