// dropin_orbital.cu -- the reference's orbital-side entry points backed by
// the GPU: set_orbital_hob, set_orbital_hint, sync_orbital_matrices and the
// full step mctdhb_propagate_step (names and conventions of
// andriati-alex/1d-mctdhb; see include/mctdhb_gpu.h).
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/mctdhb_gpu.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "orbital.h"

using namespace mctdhb;

// solver.cu internals used by the drop-in step
int mctdhb_solver_phase(mctdhb_solver s, int phase, cudaStream_t st);
double2* mctdhb_solver_orb_next(mctdhb_solver s);
mctdhb_space mctdhb_solver_space(mctdhb_solver s);

namespace {

using OrbKey = std::tuple<int, int, double, double, double, double, double, int>;

struct OrbDrop {
    OrbCtx c;
    double2 *d_orb = nullptr, *d_hob = nullptr, *d_hint = nullptr;
    cudaStream_t st = nullptr;
    std::mutex mu;
};

std::mutex g_mu;
std::map<OrbKey, std::unique_ptr<OrbDrop>> g_orb;

OrbDrop* orb_ctx(OrbitalEquation eq, int M) {
    const int G = eq->grid_size;
    const OrbKey key{M, G, eq->xi, eq->xf, eq->d2coef, std::real(eq->d1coef), std::imag(eq->d1coef),
                     eq->bounds == PERIODIC_BOUNDS};
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_orb.find(key);
    if (it != g_orb.end()) return it->second.get();
    auto d = std::make_unique<OrbDrop>();
    const double2 a1 = make_double2(std::real(eq->d1coef), std::imag(eq->d1coef));
    if (orb_init(d->c, M, G, eq->xi, eq->xf, eq->d2coef, a1, eq->bounds == PERIODIC_BOUNDS, 0))
        return nullptr;
    const size_t n = (size_t)M * G, M2 = (size_t)M * M;
    if (cudaMalloc(&d->d_orb, n * sizeof(double2)) || cudaMalloc(&d->d_hob, M2 * sizeof(double2)) ||
        cudaMalloc(&d->d_hint, M2 * M2 * sizeof(double2)) ||
        cudaStreamCreateWithFlags(&d->st, cudaStreamNonBlocking)) {
        set_error("orbital matrices: device allocation failed");
        return nullptr;
    }
    OrbDrop* p = d.get();
    g_orb[key] = std::move(d);
    return p;
}

// orbitals (row pointers) -> device, trap and interaction of eq
int upload_orbitals(OrbDrop& d, OrbitalEquation eq, int M, Cmatrix orb) {
    const int G = eq->grid_size;
    for (int k = 0; k < M; k++)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(d.d_orb + (size_t)k * G, orb[k], G * sizeof(double2),
                                        cudaMemcpyHostToDevice, d.st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(d.c.d_pot, eq->pot_grid, G * sizeof(double),
                                    cudaMemcpyHostToDevice, d.st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(d.c.d_g, &eq->g, sizeof(double), cudaMemcpyHostToDevice, d.st));
    return 0;
}

int orbital_matrices_host(OrbitalEquation eq, int M, Cmatrix orb, Cmatrix hob, Carray hint) {
    if (!eq || !orb) {
        set_error("orbital matrices: null argument");
        return -1;
    }
    OrbDrop* d = orb_ctx(eq, M);
    if (!d) return -1;
    std::lock_guard<std::mutex> lk(d->mu);
    if (upload_orbitals(*d, eq, M, orb) || orb_matrices(d->c, d->d_orb, d->d_hob, d->d_hint, d->st))
        return -1;
    if (hob)
        for (int k = 0; k < M; k++)
            MCTDHB_CUDA_TRY(cudaMemcpyAsync(hob[k], d->d_hob + (size_t)k * M, M * sizeof(double2),
                                            cudaMemcpyDeviceToHost, d->st));
    if (hint)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(hint, d->d_hint, (size_t)M * M * M * M * sizeof(double2),
                                        cudaMemcpyDeviceToHost, d->st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(d->st));
    return 0;
}

// ---- full step --------------------------------------------------------------
struct StepKey {
    int N, M, G, periodic, imag, rk, lz;
    double xi, xf, a2, a1r, a1i, dt;
    bool operator==(const StepKey& o) const {
        return N == o.N && M == o.M && G == o.G && periodic == o.periodic && imag == o.imag &&
               rk == o.rk && lz == o.lz && xi == o.xi && xf == o.xf && a2 == o.a2 &&
               a1r == o.a1r && a1i == o.a1i && dt == o.dt;
    }
};

struct StepCtx {
    StepKey key{};
    mctdhb_solver s = nullptr;
    std::vector<double2> stage;  // contiguous staging of row-pointer matrices
    std::mutex mu;
};

std::map<const void*, std::unique_ptr<StepCtx>> g_steps;

}  // namespace

extern "C" {

void set_orbital_hob(OrbitalEquation eq_desc, uint16_t norb, Cmatrix orb, Cmatrix hob) {
    orbital_matrices_host(eq_desc, norb, orb, hob, nullptr);
}

void set_orbital_hint(OrbitalEquation eq_desc, uint16_t norb, Cmatrix orb, Carray hint) {
    orbital_matrices_host(eq_desc, norb, orb, nullptr, hint);
}

void sync_orbital_matrices(OrbitalEquation eq_desc, ManyBodyState psi) {
    if (!psi) {
        set_error("sync_orbital_matrices: null state");
        return;
    }
    orbital_matrices_host(eq_desc, psi->norb, psi->orbitals, psi->hob, psi->hint);
}

void mctdhb_propagate_step(MCTDHBDataStruct mctdhb, Carray orb_works, Carray coef_works,
                           uint32_t curr_step) {
    if (!mctdhb || !mctdhb->state || !mctdhb->orb_eq || !mctdhb->multiconfig_space) {
        set_error("mctdhb_propagate_step: incomplete MCTDHBDataStruct");
        return;
    }
    if (mctdhb->orb_integ_method != FULLSTEP_RUNGEKUTTA && mctdhb->orb_integ_method != SPLITSTEP) {
        set_error("mctdhb_propagate_step: orbital method %d not FULLSTEP_RUNGEKUTTA or SPLITSTEP",
                  (int)mctdhb->orb_integ_method);
        return;
    }
    const bool sil = mctdhb->coef_integ_method == LANCZOS;
    if ((!sil && mctdhb->coef_integ_method != RUNGEKUTTA) ||
        (sil && (!mctdhb->coef_workspace || !mctdhb->coef_workspace->lan_work))) {
        set_error("mctdhb_propagate_step: coefficients by LANCZOS (with its workspace) or "
                  "RUNGEKUTTA (got %d)", (int)mctdhb->coef_integ_method);
        return;
    }
    // Lanczos dimension of the SIL step (unused by Runge-Kutta coefficients)
    const int lz = sil ? (int)mctdhb->coef_workspace->lan_work->iter : 5;
    ManyBodyState psi = mctdhb->state;
    OrbitalEquation eq = mctdhb->orb_eq;
    const int N = psi->npar, M = psi->norb, G = psi->grid_size;
    StepKey key{N, M, G, eq->bounds == PERIODIC_BOUNDS, mctdhb->integ_type == IMAGTIME,
                (int)mctdhb->rk_order, lz, eq->xi, eq->xf,
                eq->d2coef, std::real(eq->d1coef), std::imag(eq->d1coef), eq->tstep};
    StepCtx* c;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto& slot = g_steps[mctdhb];
        if (!slot) slot = std::make_unique<StepCtx>();
        c = slot.get();
    }
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->s || !(c->key == key)) {
        mctdhb_solver_destroy(c->s);
        c->s = nullptr;
        if (mctdhb_solver_create(N, M, G, eq->xi, eq->xf, eq->d2coef, key.a1r, key.a1i,
                                 key.periodic, key.imag, key.rk, key.lz, eq->tstep, &c->s))
            return;
        c->key = key;
    }
    mctdhb_solver s = c->s;
    const size_t n = (size_t)M * G, M2 = (size_t)M * M;
    const size_t nc = psi->space_dim;
    c->stage.resize(std::max(n, M2));
    // state in: orbitals, coefficients, rho2, rho1^{-1}; trap, g, factor
    for (int k = 0; k < M; k++)
        std::memcpy(c->stage.data() + (size_t)k * G, psi->orbitals[k], G * sizeof(double2));
    std::vector<double2> rinv(M2);
    for (int k = 0; k < M; k++)
        std::memcpy(rinv.data() + (size_t)k * M, psi->inv_ob_denmat[k], M * sizeof(double2));
    if (mctdhb_solver_put(s, c->stage.data(), psi->coef, psi->tb_denmat, rinv.data()) ||
        mctdhb_solver_set_potential(s, eq->pot_grid) || mctdhb_solver_set_interaction(s, eq->g) ||
        mctdhb_solver_set_regularization(s, get_current_regularization_factor()))
        return;
    // the projector the reference's driver selected (orbital_integration.c:219-227)
    // and the derivative method of the linear part (:137-176)
    if (mctdhb->orb_workspace &&
        mctdhb_solver_set_orthogonality(s, mctdhb->orb_workspace->impr_ortho ? 1 : 0))
        return;
    if (mctdhb_solver_set_derivative(s, (int)mctdhb->orb_der_method) ||
        mctdhb_solver_set_coef_method(s, (int)mctdhb->coef_integ_method) ||
        mctdhb_solver_set_orb_method(s, (int)mctdhb->orb_integ_method))
        return;
    cudaStream_t st = 0;
    if (mctdhb_solver_phase(s, 0, st)) return;
    // driver.c:175-177: time advances, trap and interaction follow in real time
    eq->t = (curr_step + 1) * eq->tstep;
    if (mctdhb->integ_type == REALTIME && eq->pot_func && eq->inter_param) {
        eq->g = eq->inter_param(eq->t, eq->inter_extra_args);
        eq->pot_func(eq->t, eq->grid_size, eq->grid_pts, eq->pot_extra_args, eq->pot_grid);
        if (mctdhb_solver_set_potential(s, eq->pot_grid) || mctdhb_solver_set_interaction(s, eq->g))
            return;
    }
    if (mctdhb_solver_phase(s, 1, st)) return;
    // state out
    std::vector<double2> orbh(n), hob(M2), rho1(M2);
    if (mctdhb_solver_get(s, orbh.data(), psi->coef, hob.data(), psi->hint, rho1.data(),
                          psi->tb_denmat, rinv.data()))
        return;
    // std::complex<double> is laid out as two doubles, like double2
    for (int k = 0; k < M; k++) {
        std::memcpy(static_cast<void*>(psi->orbitals[k]), orbh.data() + (size_t)k * G,
                    G * sizeof(double2));
        std::memcpy(static_cast<void*>(psi->hob[k]), hob.data() + (size_t)k * M,
                    M * sizeof(double2));
        std::memcpy(static_cast<void*>(psi->ob_denmat[k]), rho1.data() + (size_t)k * M,
                    M * sizeof(double2));
        std::memcpy(static_cast<void*>(psi->inv_ob_denmat[k]), rinv.data() + (size_t)k * M,
                    M * sizeof(double2));
    }
    if (orb_works &&
        cudaMemcpy(orb_works, mctdhb_solver_orb_next(s), n * sizeof(double2),
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("mctdhb_propagate_step: copy of the Runge-Kutta orbitals failed");
        return;
    }
    if (coef_works && M > 1) {
        if (cudaMemcpy(coef_works, mctdhb_solver_device_coef(s), nc * sizeof(double2),
                       cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error("mctdhb_propagate_step: copy of the coefficients failed");
            return;
        }
        if (mctdhb->integ_type == IMAGTIME) {  // the step's result before renormalisation
            double nrm2 = 1.0;
            if (sil_norm2(mctdhb_solver_space(s)->lw, &nrm2)) return;
            const double scale = std::sqrt(nrm2);
            for (size_t i = 0; i < nc; i++) coef_works[i] *= scale;
        }
    }
}

}  // extern "C"
