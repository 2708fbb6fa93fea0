// lanczos.cu -- Lanczos recurrence with full reorthogonalisation and the
// short-iterative-Lanczos (SIL) step, entirely on the device.
//
// Follows multiconfig_lanczos.c:12-90 (lanczos), :93-172
// (lowest_state_lanczos) and coefficients_integration.c:59-160
// (propagate_coef_sil) operation for operation:
//   out = H v0;  a0 = <v0, out>
//   for i < m-1:  out -= a_i v_i;  o_k = <v_k, out> (k <= i);
//                 out -= sum_k o_k v_k;  b_i = |out|;  breakdown if
//                 b_i / max b < 1e-14;  v_{i+1} = out / b_i;
//                 out = H v_{i+1} - b_i v_i;  a_{i+1} = <v_{i+1}, out>
// then the m x m tridiagonal eigenproblem (implicit QL with Wilkinson
// shifts, the EISPACK tql2 scheme, in place of LAPACK dstev), the
// propagator y = U exp(-i D dt) U^T e1 and C = sum_j y_j v_j.
// Every scalar (a, b, o, y, the breakdown flag and iteration count) lives
// in device memory, so a step is a fixed launch sequence with no host
// round trip: it can be captured into a CUDA graph.  All reductions are
// fixed-order (per-block partials, then one ordered pass), so results are
// reproducible bit for bit.
#include <algorithm>
#include <initializer_list>
#include <utility>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "small_linalg.cuh"

namespace mctdhb {

// device scalar layout (double2 slots)
constexpr int kSlots = 64;
constexpr int S_DIAG = 0;
constexpr int S_OFFD = kSlots;
constexpr int S_ORTHO = 2 * kSlots;
constexpr int S_Y = 3 * kSlots;
constexpr int S_MISC = 4 * kSlots;  // [0] maxCheck, [1] 1/b, [2] energy, [3] |C|
constexpr int S_TOTAL = 4 * kSlots + 8;
constexpr int kDotChunk = 16;  // dots per pass of the reorthogonalisation

int vec_grid_for(uint32_t n) {
    uint64_t need = ((uint64_t)n + 255) / 256;
    uint64_t cap = (uint64_t)num_sms() * 8;
    return (int)std::max<uint64_t>(1, std::min(need, cap));
}

// part[r * ncols + b] -> out[r], fixed order
__global__ void reduce_rows_kernel(const double2* __restrict__ part, int ncols,
                                   double2* __restrict__ out) {
    const int r = blockIdx.x;
    double2 s = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < ncols; b += blockDim.x) {
        s.x += part[(size_t)r * ncols + b].x;
        s.y += part[(size_t)r * ncols + b].y;
    }
    __shared__ double2 sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[threadIdx.x].x += sh[threadIdx.x + o].x;
            sh[threadIdx.x].y += sh[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[r] = sh[0];
}

static int reduce_rows(const double2* part, int nrows, int ncols, double2* out, cudaStream_t st) {
    reduce_rows_kernel<<<nrows, 256, 0, st>>>(part, ncols, out);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

__global__ void dot_kernel(const double2* __restrict__ a, const double2* __restrict__ b,
                           uint32_t n, double2* __restrict__ part) {
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc = cfma_conj(a[i], b[i], acc);
    block_reduce_store(acc, part);
}

int vec_dot(const double2* a, const double2* b, uint32_t n, double2* part, int grid,
            double2* d_out, cudaStream_t st) {
    dot_kernel<<<grid, 256, 0, st>>>(a, b, n, part);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return reduce_rows(part, 1, grid, d_out, st);
}

// out -= a_i v_i (when k0 == 0), and partial dots <v_k, out> for k in [k0, k1]
// NK = k1 - k0 + 1 dots (compile time: only the accumulators in use take
// registers, which keeps enough warps resident for a memory-bound pass)
template <int NK>
__global__ void __launch_bounds__(256)
    lz_sub_dots_kernel(int i, int k0, const double2* __restrict__ V, uint32_t n,
                       double2* __restrict__ out, const double2* __restrict__ scal,
                       const int* __restrict__ iflag, double2* __restrict__ part) {
    if (iflag[0]) return;
    const double2 alpha = scal[S_DIAG + i];
    double2 acc[NK];
#pragma unroll
    for (int k = 0; k < NK; k++) acc[k] = make_double2(0.0, 0.0);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double2 o = out[r];
        if (k0 == 0) {
            const double2 av = cmul(alpha, V[(size_t)i * n + r]);
            o.x -= av.x;
            o.y -= av.y;
            out[r] = o;
        }
#pragma unroll
        for (int k = 0; k < NK; k++) acc[k] = cfma_conj(V[(size_t)(k0 + k) * n + r], o, acc[k]);
    }
#pragma unroll
    for (int k = 0; k < NK; k++) block_reduce_store(acc[k], part + (size_t)k * gridDim.x);
}

template <int NK>
static void sub_dots_launch(int nk, int vg, cudaStream_t st, int i, int k0, const double2* V,
                            uint32_t n, double2* out, const double2* scal, const int* iflag,
                            double2* part) {
    if (nk == NK)
        lz_sub_dots_kernel<NK><<<vg, 256, 0, st>>>(i, k0, V, n, out, scal, iflag, part);
    else if constexpr (NK > 1)
        sub_dots_launch<NK - 1>(nk, vg, st, i, k0, V, n, out, scal, iflag, part);
}

// out -= sum_{k<=i} o_k v_k; partial |out|^2
__global__ void __launch_bounds__(256)
    lz_orth_kernel(int i, const double2* __restrict__ V, uint32_t n, double2* __restrict__ out,
                   const double2* __restrict__ scal, const int* __restrict__ iflag,
                   double2* __restrict__ part) {
    if (iflag[0]) return;
    double acc = 0.0;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double2 o = out[r];
        for (int k = 0; k <= i; k++) {
            const double2 t = cmul(V[(size_t)k * n + r], scal[S_ORTHO + k]);
            o.x -= t.x;
            o.y -= t.y;
        }
        out[r] = o;
        acc += o.x * o.x + o.y * o.y;
    }
    block_reduce_store(make_double2(acc, 0.0), part);
}

// b_i = sqrt(sum part); breakdown test; 1/b_i
__global__ void lz_norm_kernel(int i, const double2* __restrict__ part, int np,
                               double2* __restrict__ scal, int* __restrict__ iflag) {
    __shared__ double sh[256];
    double s = 0.0;
    for (int b = threadIdx.x; b < np; b += blockDim.x) s += part[b].x;
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x != 0 || iflag[0]) return;
    const double beta = sqrt(sh[0]);
    scal[S_OFFD + i] = make_double2(beta, 0.0);
    double mx = scal[S_MISC + 0].x;
    if (mx < beta) mx = beta;
    scal[S_MISC + 0].x = mx;
    if (beta == 0.0 || beta / mx < 1e-14) {
        iflag[0] = 1;
        iflag[1] = i + 1;
        return;
    }
    scal[S_MISC + 1] = make_double2(1.0 / beta, 0.0);
}

__global__ void lz_scale_kernel(int i, const double2* __restrict__ out, double2* __restrict__ V,
                                uint32_t n, const double2* __restrict__ scal,
                                const int* __restrict__ iflag) {
    if (iflag[0]) return;
    const double inv = scal[S_MISC + 1].x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double2 o = out[r];
        V[(size_t)(i + 1) * n + r] = make_double2(o.x * inv, o.y * inv);
    }
}

__global__ void lz_init_kernel(double2* scal, int* iflag, int m) {
    if (threadIdx.x == 0) {
        scal[S_MISC + 0] = make_double2(0.0, 0.0);
        scal[S_OFFD + m - 1] = make_double2(0.0, 0.0);
        iflag[0] = 0;
        iflag[1] = m;
        iflag[2] = 0;
    }
}

// mode 0: SIL propagator y = U exp(-i D prop_dt) U^T e1
// mode 2: the same up to a positive constant factor, for a step that
//         renormalises y (imaginary time)
// mode 1: lowest Ritz vector y = U[:, argmin D], energy -> scal[S_MISC+2]
__global__ void lz_small_kernel(int mode, double2 prop_dt, double2* __restrict__ scal,
                                int* __restrict__ iflag, double* __restrict__ z,
                                double* __restrict__ energy) {
    if (threadIdx.x != 0) return;
    const int n = iflag[1];
    double d[kSlots], e[kSlots];
    for (int k = 0; k < n; k++) {
        d[k] = scal[S_DIAG + k].x;
        e[k] = scal[S_OFFD + k].x;
    }
    iflag[2] = tridiag_ql(n, d, e, z);
    if (mode != 1) {
        // mode 2: exponents shifted by their maximum (a constant factor the
        // renormalisation at the end of the step removes), so exp cannot
        // overflow at |E| dt > 709; a real prop_dt has no shift either way
        double shift = 0.0;
        if (mode == 2 && prop_dt.y != 0.0)
            for (int k = 0; k < n; k++)
                shift = k == 0 ? d[k] * prop_dt.y : fmax(shift, d[k] * prop_dt.y);
        double2 aux[kSlots];
        for (int k = 0; k < n; k++) {
            // exp(-i d_k prop_dt), prop_dt complex
            const double re = d[k] * prop_dt.y, im = -d[k] * prop_dt.x;
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
            scal[S_Y + k] = s;
        }
    } else {
        double sentinel = 1e15;
        int jm = 0;
        for (int k = 0; k < n; k++)
            if (sentinel > d[k]) {
                sentinel = d[k];
                jm = k;
            }
        for (int k = 0; k < n; k++) scal[S_Y + k] = make_double2(z[k * n + jm], 0.0);
        scal[S_MISC + 2] = make_double2(sentinel, 0.0);
        if (energy) *energy = sentinel;
    }
}

// C = sum_j V_j y_j
__global__ void lz_combine_kernel(const double2* __restrict__ V, uint32_t n,
                                  const double2* __restrict__ scal, const int* __restrict__ iflag,
                                  double2* __restrict__ C) {
    const int it = iflag[1];
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < it; j++) s = cfma(V[(size_t)j * n + r], scal[S_Y + j], s);
        C[r] = s;
    }
}

__global__ void norm2_kernel(const double2* __restrict__ a, uint32_t n, double2* __restrict__ part) {
    double acc = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += a[i].x * a[i].x + a[i].y * a[i].y;
    block_reduce_store(make_double2(acc, 0.0), part);
}

__global__ void renorm_kernel(double2* __restrict__ a, uint32_t n, const double2* __restrict__ nrm2) {
    const double r = 1.0 / sqrt(nrm2->x);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a[i].x *= r;
        a[i].y *= r;
    }
}

// ---------------------------------------------------------------------------
int lanczos_alloc(LanczosWork& w, const SpaceCtx& s, int mmax) {
    if (mmax < 1 || mmax > kSlots) {
        set_error("Lanczos dimension %d outside 1..%d", mmax, kSlots);
        return -1;
    }
    w.mmax = mmax;
    w.dim = s.dim;
    w.vec_grid = vec_grid_for(s.dim);
    const size_t part_elems = (size_t)kDotChunk * w.vec_grid;
    MCTDHB_CUDA_TRY(cudaMalloc(&w.V, (size_t)mmax * s.dim * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&w.out, (size_t)s.dim * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&w.part, part_elems * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&w.scal, (S_TOTAL + kSlots * kSlots / 2 + 8) * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMemset(w.scal, 0, (S_TOTAL + kSlots * kSlots / 2 + 8) * sizeof(double2)));
    MCTDHB_CUDA_TRY(cudaMalloc(&w.iflag, 4 * sizeof(int)));
    return 0;
}

void lanczos_free(LanczosWork& w) {
    cudaFree(w.V);
    cudaFree(w.out);
    cudaFree(w.part);
    cudaFree(w.scal);
    cudaFree(w.iflag);
    w = LanczosWork();
}

static double* zbuf(const LanczosWork& w) { return (double*)(w.scal + S_TOTAL); }

int lanczos_run(const SpaceCtx& s, LanczosWork& w, int m, cudaStream_t st) {
    if (m < 1 || m > w.mmax) {
        set_error("Lanczos dimension %d outside 1..%d", m, w.mmax);
        return -1;
    }
    const uint32_t n = s.dim;
    const int vg = w.vec_grid;
    lz_init_kernel<<<1, 32, 0, st>>>(w.scal, w.iflag, m);
    HcEpilogue ep;
    ep.flag = w.iflag;
    if (hc_apply(s.view, w.V, w.out, s.d_tab, ep, st)) return -1;
    // a_0 = <v0, H v0>: fixed-geometry reduction, independent of the H.C
    // launch variant
    if (vec_dot(w.V, w.out, n, w.part, vg, w.scal + S_DIAG, st)) return -1;
    for (int i = 0; i < m - 1; i++) {
        for (int k0 = 0; k0 <= i; k0 += kDotChunk) {
            const int k1 = std::min(i, k0 + kDotChunk - 1);
            sub_dots_launch<kDotChunk>(k1 - k0 + 1, vg, st, i, k0, w.V, n, w.out, w.scal,
                                       w.iflag, w.part);
            MCTDHB_CUDA_TRY(cudaGetLastError());
            if (reduce_rows(w.part, k1 - k0 + 1, vg, w.scal + S_ORTHO + k0, st)) return -1;
        }
        lz_orth_kernel<<<vg, 256, 0, st>>>(i, w.V, n, w.out, w.scal, w.iflag, w.part);
        lz_norm_kernel<<<1, 256, 0, st>>>(i, w.part, vg, w.scal, w.iflag);
        lz_scale_kernel<<<vg, 256, 0, st>>>(i, w.out, w.V, n, w.scal, w.iflag);
        MCTDHB_CUDA_TRY(cudaGetLastError());
        HcEpilogue e2;
        e2.flag = w.iflag;
        e2.prev = w.V + (size_t)i * n;
        e2.beta = &(w.scal + S_OFFD + i)->x;
        if (hc_apply(s.view, w.V + (size_t)(i + 1) * n, w.out, s.d_tab, e2, st)) return -1;
        // a_{i+1}; after a breakdown the value is never read (iterations < i+2)
        if (vec_dot(w.V + (size_t)(i + 1) * n, w.out, n, w.part, vg, w.scal + S_DIAG + i + 1, st))
            return -1;
    }
    return 0;
}

// diag[0..it-1] and offd[0..min(it, m-1)-1] as the reference leaves them
int lanczos_fetch(const LanczosWork& w, int m, int* iters, double2* diag, double2* offd,
                  cudaStream_t st) {
    int fl[4];
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(fl, w.iflag, sizeof(fl), cudaMemcpyDeviceToHost, st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int it = fl[1];
    const int nofd = std::min(it, m - 1);
    if (diag && it > 0)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(diag, w.scal + S_DIAG, it * sizeof(double2),
                                        cudaMemcpyDeviceToHost, st));
    if (offd && nofd > 0)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(offd, w.scal + S_OFFD, nofd * sizeof(double2),
                                        cudaMemcpyDeviceToHost, st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(st));
    if (iters) *iters = it;
    return 0;
}

int sil_step(const SpaceCtx& s, LanczosWork& w, double2* d_C, int m, double2 prop_dt,
             int imagtime, cudaStream_t st) {
    const uint32_t n = s.dim;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(w.V, d_C, (size_t)n * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, st));
    if (lanczos_run(s, w, m, st)) return -1;
    lz_small_kernel<<<1, 32, 0, st>>>(imagtime ? 2 : 0, prop_dt, w.scal, w.iflag, zbuf(w),
                                      nullptr);
    lz_combine_kernel<<<w.vec_grid, 256, 0, st>>>(w.V, n, w.scal, w.iflag, d_C);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    if (imagtime) {
        norm2_kernel<<<w.vec_grid, 256, 0, st>>>(d_C, n, w.part);
        if (reduce_rows(w.part, 1, w.vec_grid, w.scal + S_MISC + 3, st)) return -1;
        renorm_kernel<<<w.vec_grid, 256, 0, st>>>(d_C, n, w.scal + S_MISC + 3);
        MCTDHB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

// out = y + sum_j c_j V_j (complex c_j), up to 6 terms
struct CoefCombo {
    double2 c[6];
    int n;
};
__global__ void coef_combo_kernel(const double2* __restrict__ y, const double2* __restrict__ V,
                                  uint32_t n, CoefCombo cb, double2* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double2 acc = y[i];
        for (int j = 0; j < cb.n; j++) acc = cfma(cb.c[j], V[(size_t)j * n + i], acc);
        out[i] = acc;
    }
}

// One Runge-Kutta step of the coefficients (coefficients_integration.c:15-57):
// dC/dt = -i tf H C with the named tableaux (classical RK4, Butcher's RK5;
// order 2 takes the RK5 tableau as there, :44-47).  Stage H.C products go to
// V[0..5], the stage input to V[6]; in imaginary time C is renormalised and
// |C|^2 before it kept for sil_norm2.
int coef_rk_step(const SpaceCtx& s, LanczosWork& w, double2* d_C, int order, double dt,
                 int imagtime, cudaStream_t st) {
    const uint32_t n = s.dim;
    if (w.mmax < 7) {
        set_error("coef_rk_step: workspace of %d vectors, 7 needed", w.mmax);
        return -1;
    }
    double2* V = w.V;
    double2* tmp = w.V + (size_t)6 * n;
    // -i tf dt: tf = 1 (real time) or -i (imaginary time)
    const double2 f = imagtime ? make_double2(-dt, 0.0) : make_double2(0.0, -dt);
    HcEpilogue ep;
    auto H = [&](const double2* in, int j) {
        return hc_apply(s.view, in, V + (size_t)j * n, s.d_tab, ep, st);
    };
    auto combo = [&](std::initializer_list<std::pair<int, double>> t, double2* out) {
        CoefCombo cb{};
        cb.n = 0;
        for (auto& p : t) {
            // terms j index V rows in order 0..n-1; absent rows get weight 0
            while (cb.n < p.first) cb.c[cb.n++] = make_double2(0.0, 0.0);
            cb.c[cb.n++] = make_double2(f.x * p.second, f.y * p.second);
        }
        coef_combo_kernel<<<w.vec_grid, 256, 0, st>>>(d_C, V, n, cb, out);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    };
    int rc = 0;
    if (order == 4) {
        rc |= H(d_C, 0);
        rc |= combo({{0, 0.5}}, tmp);
        rc |= H(tmp, 1);
        rc |= combo({{1, 0.5}}, tmp);
        rc |= H(tmp, 2);
        rc |= combo({{2, 1.0}}, tmp);
        rc |= H(tmp, 3);
        rc |= combo({{0, 1.0 / 6}, {1, 2.0 / 6}, {2, 2.0 / 6}, {3, 1.0 / 6}}, d_C);
    } else if (order == 5 || order == 2) {
        rc |= H(d_C, 0);
        rc |= combo({{0, 0.25}}, tmp);
        rc |= H(tmp, 1);
        rc |= combo({{0, 0.125}, {1, 0.125}}, tmp);
        rc |= H(tmp, 2);
        rc |= combo({{1, -0.5}, {2, 1.0}}, tmp);
        rc |= H(tmp, 3);
        rc |= combo({{0, 3.0 / 16}, {3, 9.0 / 16}}, tmp);
        rc |= H(tmp, 4);
        rc |= combo({{0, -3.0 / 7}, {1, 2.0 / 7}, {2, 12.0 / 7}, {3, -12.0 / 7}, {4, 8.0 / 7}},
                    tmp);
        rc |= H(tmp, 5);
        rc |= combo({{0, 7.0 / 90}, {2, 32.0 / 90}, {3, 12.0 / 90}, {4, 32.0 / 90}, {5, 7.0 / 90}},
                    d_C);
    } else {
        set_error("coefficient Runge-Kutta order %d not in {2, 4, 5}", order);
        return -1;
    }
    if (rc) {
        set_error("coef_rk_step: launch failed");
        return -1;
    }
    if (imagtime) {
        norm2_kernel<<<w.vec_grid, 256, 0, st>>>(d_C, n, w.part);
        if (reduce_rows(w.part, 1, w.vec_grid, w.scal + S_MISC + 3, st)) return -1;
        renorm_kernel<<<w.vec_grid, 256, 0, st>>>(d_C, n, w.scal + S_MISC + 3);
        MCTDHB_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

int sil_norm2(const LanczosWork& w, double* out) {
    double2 v;
    MCTDHB_CUDA_TRY(cudaDeviceSynchronize());
    MCTDHB_CUDA_TRY(cudaMemcpy(&v, w.scal + S_MISC + 3, sizeof(v), cudaMemcpyDeviceToHost));
    *out = v.x;
    return 0;
}

int lowest_state(const SpaceCtx& s, LanczosWork& w, double2* d_C, int m, double* d_energy,
                 cudaStream_t st) {
    const uint32_t n = s.dim;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(w.V, d_C, (size_t)n * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, st));
    if (lanczos_run(s, w, m, st)) return -1;
    lz_small_kernel<<<1, 32, 0, st>>>(1, make_double2(0.0, 0.0), w.scal, w.iflag, zbuf(w),
                                      d_energy);
    lz_combine_kernel<<<w.vec_grid, 256, 0, st>>>(w.V, n, w.scal, w.iflag, d_C);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mctdhb
