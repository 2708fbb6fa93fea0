// orbital.h -- device objects of the orbital side (orbital.cu) and of the
// full MCTDHB step (solver.cu).
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace mctdhb {

// grid, equation coefficients and Simpson weights (device pointers)
struct OrbView {
    int M, G, periodic;
    double dx, a2;  // a2: coefficient of d^2/dx^2 (d2coef), a1: of d/dx (d1coef)
    double2 a1, tf;  // tf: time factor, 1 (real time) or -i (imaginary time)
    const double* w;
    const double* pot;
    // DVR / spectral derivatives: Toeplitz kernel on the n = G - 1 periodic
    // points, (D f)_i = sum_j lin_t[j - i + n - 1] f_j; null: finite
    // differences
    const double2* lin_t;
};

// derivative methods of the orbital equation (mctdhb_types.h OrbDerivative)
constexpr int kDerDVR = 300, kDerSpectral = 301, kDerFiniteDiff = 302;

// Toeplitz kernel (2(G-1) - 1 values, a2 and a1 folded in) of the DVR or
// spectral linear part on the G - 1 periodic points (orbital.cu)
std::vector<double2> derivative_toeplitz(int der, int G, double dx, double a2,
                                         std::complex<double> a1);

struct OrbCtx {
    int M = 0, G = 0;
    OrbView view{};
    double* d_w = nullptr;
    double* d_pot = nullptr;
    double* d_g = nullptr;         // contact interaction strength (device scalar)
    double2* d_k[8] = {};          // Runge-Kutta stages + stage input
    double2* d_H = nullptr;        // H phi
    double2* d_P = nullptr;        // projector overlaps
    double2* d_Q = nullptr;        // g rho1^{-1} rho2
    double2* d_work = nullptr;     // small dense work (rho1 synchronisation, projector)
    double2* d_S = nullptr;        // orbital overlap matrix <f_s|f_l>
    int* d_fail = nullptr;         // set when the robust projector met a singular overlap
    int robust = 0;                // robust projector (orbital_integration.c:22-92)
    int der = kDerFiniteDiff;      // derivative method of the linear part
    double2* d_lin_t = nullptr;    // Toeplitz kernel of DVR / spectral derivatives
    double2* d_L = nullptr;        // linear part of every orbital (DVR / spectral)
    // split-step integrator (orbital_integration.c:352-434)
    int split = 0;
    int half_dense = 0;            // half-step operator: 0 circulant kernel, 1 dense
    double2* d_half = nullptr;     // circulant: 2n - 1 kernel; dense: G x G, column-major
    double2* d_B = nullptr;        // M x M projection through g of the nonlinear part
    const double2* split_hob = nullptr;  // h of the half-stepped orbitals (caller's buffer)
};

std::vector<double> simpson_weights(int n, double h);
int orb_init(OrbCtx& c, int M, int G, double xi, double xf, double a2, double2 a1, int periodic,
             int imagtime);
void orb_release(OrbCtx& c);
int orb_matrices(const OrbCtx& c, const double2* orb, double2* hob, double2* hint,
                 cudaStream_t st);
int orb_rhs_eval(const OrbCtx& c, const double2* rinv, const double2* rho2, const double2* y,
                 double2* out, cudaStream_t st);
int orb_rk_step(const OrbCtx& c, int order, double dt, const double2* rinv, const double2* rho2,
                const double2* y, double2* ynext, cudaStream_t st);
int orb_periodic(const OrbCtx& c, double2* orb, cudaStream_t st);
// derivative method: kDerFiniteDiff, or kDerDVR / kDerSpectral on a
// periodic grid (the Toeplitz kernel is set up on the host)
int orb_set_derivative(OrbCtx& c, int der);
// split-step integrator on or off; builds the linear half-step operator
// for time step dt (Crank-Nicolson for finite differences, the FFT
// exponential for DVR / spectral), again whenever the method changes
int orb_set_split(OrbCtx& c, int split, double dt, int imagtime);
// the split step's half-step operator on the host (split_linear_orbitals.c
// 23-82, 289-402): periodic grids, the circulant kernel of Crank-Nicolson
// A^{-1} B (finite differences) or of the FFT exponential (DVR, spectral) on
// the n = G - 1 periodic points (2n - 1 values, *dense = 0); zero bounds
// (finite differences only), A^{-1} B on all G points column-major
// (*dense = 1)
int split_half_operator(int G, double dx, double a2, double2 a1, int periodic, int der,
                        double dt, int imagtime, std::vector<double2>& op, int* dense);
// one split step of the orbitals: y -> ynext through the half steps, h and
// g of the half-stepped orbitals into hob / hint, and RK of the nonlinear part
int orb_split_step(OrbCtx& c, int order, double dt, const double2* rinv, const double2* rho2,
                   double2* y, double2* ynext, double2* hob, double2* hint, cudaStream_t st);
// S_sl = <f_s|f_l> (Simpson) into c.d_S
int orb_overlap_matrix(const OrbCtx& c, const double2* orb, cudaStream_t st);
int orb_orthonormalize(const OrbCtx& c, double2* orb, cudaStream_t st);
int orb_sync_rho1(const OrbCtx& c, double2* rho1, double2* rinv, double reg_fac, int* d_info,
                  cudaStream_t st);
int orb_energy(int M, const double2* rho1, const double2* rho2, const double2* hob,
               const double2* hint, double2* E, cudaStream_t st);

}  // namespace mctdhb
