// orbital_dev.cuh -- device math of the orbital side, shared by the
// single-system kernels (orbital.cu) and the batched engine (batch.cu):
// finite-difference derivatives and the linear part of the orbital
// equation, block and warp reductions, the g_ksql tensor-core tile,
// Gram-Schmidt, the energy.
#pragma once
#include "common.cuh"
#include "orbital.h"

namespace mctdhb {

// periodic fourth-order first derivative (calculus.c:288-305): the grid has
// P = G - 1 distinct points, f[G-1] is the copy of f[0]
__device__ __forceinline__ double2 dxfd_at(const double2* f, int G, int i, double r) {
    const int P = G - 1;
    if (i == G - 1) i = 0;
    const double2 a = f[(i - 2 + P) % P], b = f[(i + 2) % P], c = f[(i + 1) % P],
                  d = f[(i - 1 + P) % P];
    return make_double2((a.x - b.x + 8 * (c.x - d.x)) * r, (a.y - b.y + 8 * (c.y - d.y)) * r);
}

// every thread gets the block sum (fixed order); all threads must call it
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
    return s;
}

// every lane gets the warp sum
__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// Linear part of the orbital equation at grid point x of orbital f
// (split_linear_orbitals.c:210-255): a2 f'' + a1 f' + V f by second-order
// central differences; periodic grids wrap through the copy f[G-1] = f[0].
__device__ __forceinline__ double2 linear_at(const OrbView& o, const double2* f, int x) {
    const int G = o.G;
    const double a2 = o.a2, dx = o.dx;
    const double2 a1 = o.a1;
    const double2 up = make_double2(a2 / dx / dx + a1.x / dx / 2, a1.y / dx / 2);
    const double2 lo = make_double2(a2 / dx / dx - a1.x / dx / 2, -a1.y / dx / 2);
    double2 lin;
    if (o.periodic) {
        if (x == G - 1 || x == 0) {
            // out[G-1] = out[0]
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
    return lin;
}

// DVR / spectral linear part at point x of orbital f (orbital_integration.c:
// 137-176): sum_j lin_t[j - x + n - 1] f_j + V(x) f(x) on the n = G - 1
// periodic points, the last point repeating the first
__device__ __forceinline__ double2 toeplitz_at(const OrbView& o, const double2* f, int x) {
    const int n = o.G - 1, xr = x == n ? 0 : x;
    const double2* t = o.lin_t + (n - 1 - xr);
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < n; j++) acc = cfma(__ldg(t + j), f[j], acc);
    return cadd(acc, cscale(f[xr], o.pot[xr]));
}

// h_kl integrand at x (orbital_matrices.c:22-70):
//   -a2 conj(f_k') f_l' + a1 conj(f_k) f_l' + V conj(f_k) f_l
__device__ __forceinline__ double2 hob_integrand(const OrbView& o, const double2* fk,
                                                 const double2* fl, int x, double r) {
    const int G = o.G;
    const double2 dk = dxfd_at(fk, G, x, r), dl = dxfd_at(fl, G, x, r);
    const double2 ck = make_double2(fk[x].x, -fk[x].y);
    double2 t = cmul(make_double2(-o.a2 * dk.x, o.a2 * dk.y), dl);
    t = cadd(t, cmul(cmul(o.a1, ck), dl));
    t = cadd(t, cscale(cmul(ck, fl[x]), o.pot[x]));
    return t;
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

// one 8 x 8 tile (index `tile` of ((M^2+7)/8)^2) computed by the calling warp
__device__ __forceinline__ void hint_tile(const OrbView& o, const double2* __restrict__ orb,
                                          const double* __restrict__ g_dev,
                                          double2* __restrict__ hint, int tile, int lane) {
    const int M = o.M, G = o.G, M2 = M * M;
    const int tiles = (M2 + 7) / 8;
    const int R0 = (tile / tiles) * 8, C0 = (tile % tiles) * 8;
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

// orthonormalize (calculus.c:171-191) by the calling block.  The reference
// re-evaluates <F_j|F_i> for every grid point k while F_i is being updated;
// that overlap obeys ov_{k+1} = ov_k (1 - w_k |F_j[k]|^2), so the update is a
// prefix product.  `scan` holds G doubles (shared memory).
__device__ __forceinline__ void orthonormalize_block(const OrbView& o, double2* __restrict__ F,
                                                     double* scan) {
    const int M = o.M, G = o.G;
    __shared__ double2 ovs;
    auto renorm = [&](double2* f) {
        double acc = 0.0;
        for (int x = threadIdx.x; x < G; x += blockDim.x)
            acc += o.w[x] * (f[x].x * f[x].x + f[x].y * f[x].y);
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

// E = sum_kl rho1[k][l] h[k][l] + 1/2 sum rho2[k,l,s,q] g[k,l,q,s]
// (integrator_monitor.c:56-88), summed by the calling block
__device__ __forceinline__ double2 energy_block(int M, const double2* __restrict__ rho1,
                                                const double2* __restrict__ rho2,
                                                const double2* __restrict__ hob,
                                                const double2* __restrict__ hint) {
    const int M2 = M * M, M3 = M2 * M, M4 = M3 * M;
    double2 acc = make_double2(0.0, 0.0);
    for (int e = threadIdx.x; e < M4; e += blockDim.x) {
        const int k = e % M, l = (e / M) % M, s = (e / M2) % M, q = e / M3;
        acc = cfma(rho2[k + l * M + s * M2 + q * M3], hint[k + l * M + q * M2 + s * M3], acc);
    }
    acc = cscale(acc, 0.5);
    for (int e = threadIdx.x; e < M2; e += blockDim.x) acc = cfma(rho1[e], hob[e], acc);
    return block_sum(acc);
}

}  // namespace mctdhb
