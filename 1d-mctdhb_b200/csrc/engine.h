// engine.h -- device-resident runtime objects behind the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace mctdhb {

uint64_t fock_dimension(int npar, int norb);

// One Fock space on one device: rank tables, the packed H.C coefficient
// table of the current orbital matrices, and reduction scratch.
struct SpaceCtx {
    int N = 0, M = 0;
    uint32_t dim = 0;
    SpaceView view{};
    uint32_t* d_T = nullptr;
    double* d_sq = nullptr;
    double2* d_tab = nullptr;       // H.C coefficient table (moves.cuh layout)
    int* d_dens_desc = nullptr;     // density element descriptors
    double2* d_dens_part = nullptr; // density partial sums
};

int space_init(SpaceCtx& s, int N, int M);
void space_release(SpaceCtx& s);

// Short-iterative-Lanczos workspace (multiconfig_lanczos.c:12-90,
// coefficients_integration.c:59-160) with every scalar kept on the device,
// so one step is a fixed launch sequence (CUDA-graph capturable).
struct LanczosWork {
    int mmax = 0;
    uint32_t dim = 0;
    double2* V = nullptr;      // mmax x dim Krylov vectors
    double2* out = nullptr;    // dim
    double2* part = nullptr;   // reduction partials
    double2* scal = nullptr;   // device scalars (see lanczos.cu)
    int* iflag = nullptr;      // [0] breakdown flag, [1] iterations done, [2] eigensolver info
    int vec_grid = 0;
};

int lanczos_alloc(LanczosWork& w, const SpaceCtx& s, int mmax);
void lanczos_free(LanczosWork& w);

// Builds the Krylov basis of V[0] (already in w.V) with `m` vectors;
// the tridiagonal coefficients stay in w.scal.  Returns 0 or -1.
int lanczos_run(const SpaceCtx& s, LanczosWork& w, int m, cudaStream_t st);
// Host-visible copies of the Lanczos results (synchronises the stream).
int lanczos_fetch(const LanczosWork& w, int m, int* iters, double2* diag, double2* offd,
                  cudaStream_t st);
// One SIL step on C (device, in/out): C <- V U exp(-i D prop_dt) U^T e1,
// renormalised in imaginary time.
int sil_step(const SpaceCtx& s, LanczosWork& w, double2* d_C, int m, double2 prop_dt,
             int imagtime, cudaStream_t st);
// One Runge-Kutta step of C (device, in/out) with dC/dt = -i tf H C
// (coefficients_integration.c:15-57), renormalised in imaginary time; the
// workspace needs 7 vectors.
int coef_rk_step(const SpaceCtx& s, LanczosWork& w, double2* d_C, int order, double dt,
                 int imagtime, cudaStream_t st);
// |C|^2 of the last imaginary-time SIL (or coefficient RK) step before its
// renormalisation
int sil_norm2(const LanczosWork& w, double* out);
// Lowest Ritz pair of an m-step Lanczos started from C (in/out); the Ritz
// value is written to *d_energy (device).
int lowest_state(const SpaceCtx& s, LanczosWork& w, double2* d_C, int m, double* d_energy,
                 cudaStream_t st);

// Fixed-order vector reductions used by the C ABI (device in/out)
int vec_dot(const double2* a, const double2* b, uint32_t n, double2* part, int grid,
            double2* d_out, cudaStream_t st);
int vec_grid_for(uint32_t n);

}  // namespace mctdhb

#include <mutex>

// handle behind the public `mctdhb_space` (include/mctdhb_gpu.h)
struct mctdhb_space_s {
    mctdhb::SpaceCtx sp;
    mctdhb::LanczosWork lw;
    std::mutex mu;
};
