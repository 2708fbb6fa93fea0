// solver.cu -- one full MCTDHB time step on the device (driver.c:159-201):
//   orbitals:  Runge-Kutta step of the orbital equation with the current
//              rho1^{-1} and rho2; Gram-Schmidt in imaginary time
//   matrices:  h_kl and g_ksql of the new orbitals
//   coefficients: short-iterative-Lanczos step with the new h, g
//   densities: rho1, rho2 of the new coefficients; regularised rho1^{-1}
// Everything stays in HBM; the step is captured once into a CUDA graph and
// replayed, so a step costs one graph launch and no host round trip.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/mctdhb_gpu.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "orbital.h"

using namespace mctdhb;

struct mctdhb_solver_s {
    mctdhb_space sp = nullptr;
    OrbCtx orb;
    int N = 0, M = 0, G = 0, imagtime = 0, rk_order = 5, lanczos_m = 5;
    int coef_method = 20;  // 20 LANCZOS (SIL), 21 RUNGEKUTTA
    double dt = 0.0, reg_fac = 1e-9, t = 0.0;
    double2 *d_orb = nullptr, *d_orb_next = nullptr, *d_coef = nullptr, *d_hob = nullptr,
            *d_hint = nullptr, *d_rho1 = nullptr, *d_rho2 = nullptr, *d_rinv = nullptr,
            *d_E = nullptr;
    int* d_info = nullptr;
    cudaStream_t cs = nullptr;
    // recorded on the caller's stream after each step or phase launch; reads
    // of the state on `cs` wait for it
    cudaEvent_t ev_step = nullptr;
    // phase 0: orbital step; phase 1: matrices, SIL, densities
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    // mctdhb_solver_relax: the step inside a conditional WHILE node
    cudaGraph_t relax_graph = nullptr;
    cudaGraphExec_t relax_exec = nullptr;
    struct RelaxCtl* d_ctl = nullptr;
    struct RelaxCtl* h_ctl = nullptr;  // pinned
    bool relax_pending = false;
    int kernels = 0;
    bool has_state = false;
    std::mutex mu;
};

// device state of mctdhb_solver_relax: the parameters of a run (written
// before each launch) and its counters
struct RelaxCtl {
    uint32_t max_steps, steps;
    int check_every, conv;
    double tol, prev;
};

namespace {

constexpr uint32_t kRelaxHardCap = 100000000u;  // no run passes this many steps

// E of the state before the first step seeds the energy rule (driver.c:229)
__global__ void relax_init_kernel(RelaxCtl* __restrict__ c, const double2* __restrict__ E,
                                  int N) {
    c->steps = 0;
    c->conv = 0;
    c->prev = E->x / N;
}

// after every step: the imaginary-time energy rule of driver.c:47-67 (every
// check_every steps) and the step limit; the WHILE node repeats the step
// while this sets 1
__global__ void relax_rule_kernel(RelaxCtl* __restrict__ c, const double2* __restrict__ E,
                                  int N, int imag, cudaGraphConditionalHandle h) {
    const uint32_t steps = ++c->steps;
    bool stop = steps >= c->max_steps || steps >= kRelaxHardCap;
    if (imag && c->check_every > 0 && steps % (uint32_t)c->check_every == 0) {
        const double curr = E->x / N;
        if (fabs(curr - c->prev) < c->tol * c->prev) {
            c->conv = 1;
            stop = true;
        }
        c->prev = curr;
    }
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// phase 0 (orbital_integration.c:284-349): orbitals advanced with the
// current rho1^{-1} and rho2
int phase_orbitals(mctdhb_solver_s* s, cudaStream_t st) {
    OrbCtx& o = s->orb;
    const size_t n = (size_t)s->M * s->G;
    if (o.view.periodic && orb_periodic(o, s->d_orb, st)) return -1;
    if (o.split) {
        // orbital_integration.c:352-434 (h and g of the half-stepped
        // orbitals are rebuilt in phase 1 from the new orbitals)
        if (orb_split_step(o, s->rk_order, s->dt, s->d_rinv, s->d_rho2, s->d_orb, s->d_orb_next,
                           s->d_hob, s->d_hint, st))
            return -1;
    } else if (orb_rk_step(o, s->rk_order, s->dt, s->d_rinv, s->d_rho2, s->d_orb,
                           s->d_orb_next, st)) {
        return -1;
    }
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(s->d_orb, s->d_orb_next, n * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, st));
    if (s->imagtime && orb_orthonormalize(o, s->d_orb, st)) return -1;
    return 0;
}

// phase 1 (driver.c:179-200): matrices of the new orbitals (with the trap
// and interaction of the new time), SIL step, density matrices
int phase_coefficients(mctdhb_solver_s* s, cudaStream_t st) {
    const OrbCtx& o = s->orb;
    if (o.view.periodic && orb_periodic(o, s->d_orb, st)) return -1;
    if (orb_matrices(o, s->d_orb, s->d_hob, s->d_hint, st)) return -1;
    if (s->M == 1) return 0;  // Gross-Pitaevskii: the coefficient is trivial
    SpaceCtx& sc = s->sp->sp;
    if (hc_prep(sc.view, s->d_hob, s->d_hint, sc.d_tab, st)) return -1;
    if (s->coef_method == 21) {
        if (coef_rk_step(sc, s->sp->lw, s->d_coef, s->rk_order, s->dt, s->imagtime, st))
            return -1;
    } else {
        const double2 pdt = s->imagtime ? make_double2(0.0, -s->dt) : make_double2(s->dt, 0.0);
        if (sil_step(sc, s->sp->lw, s->d_coef, s->lanczos_m, pdt, s->imagtime, st)) return -1;
    }
    if (dens_apply(sc.view, s->d_coef, sc.d_dens_part, s->d_rho1, s->d_rho2, sc.d_dens_desc, st))
        return -1;
    return orb_sync_rho1(o, s->d_rho1, s->d_rinv, s->reg_fac, s->d_info, st);
}

int count_kernels(cudaGraph_t g) {
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(g, nodes.data(), &nn);
    int k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        cudaGraphNodeGetType(nd, &t);
        if (t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

int build_graphs(mctdhb_solver_s* s) {
    if (s->exec[0] && s->exec[1]) return 0;
    s->kernels = 0;
    for (int p = 0; p < 2; p++) {
        cudaError_t e = cudaStreamBeginCapture(s->cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            set_error("solver: capture: %s", cudaGetErrorString(e));
            return -1;
        }
        const int rc = p == 0 ? phase_orbitals(s, s->cs) : phase_coefficients(s, s->cs);
        e = cudaStreamEndCapture(s->cs, &s->graph[p]);
        if (rc) return -1;
        if (e != cudaSuccess || cudaGraphInstantiate(&s->exec[p], s->graph[p], 0) != cudaSuccess) {
            set_error("solver: graph capture failed: %s", cudaGetErrorString(e));
            return -1;
        }
        s->kernels += count_kernels(s->graph[p]);
    }
    return 0;
}

void drop_graphs(mctdhb_solver_s* s) {
    for (int p = 0; p < 2; p++) {
        if (s->exec[p]) cudaGraphExecDestroy(s->exec[p]);
        if (s->graph[p]) cudaGraphDestroy(s->graph[p]);
        s->exec[p] = nullptr;
        s->graph[p] = nullptr;
    }
    if (s->relax_exec) cudaGraphExecDestroy(s->relax_exec);
    if (s->relax_graph) cudaGraphDestroy(s->relax_graph);
    s->relax_exec = nullptr;
    s->relax_graph = nullptr;
}

// The relaxation graph: the energy of the current state and the rule's
// initial state, then a conditional WHILE node whose body is one step
// (both phases), the energy of the new state and the rule kernel.
int build_relax_graph(mctdhb_solver_s* s) {
    if (s->relax_exec) return 0;
    cudaStream_t st = s->cs;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        set_error("solver relax: capture: %s", cudaGetErrorString(e));
        return -1;
    }
    cudaGraph_t g = nullptr;
    cudaGraphConditionalHandle h = 0;
    cudaGraphNode_t cnode = nullptr;
    cudaGraph_t body = nullptr;
    int rc = orb_energy(s->M, s->d_rho1, s->d_rho2, s->d_hob, s->d_hint, s->d_E, st);
    if (!rc) {
        relax_init_kernel<<<1, 1, 0, st>>>(s->d_ctl, s->d_E, s->N);
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaStreamCaptureStatus cs;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp);
            if (e == cudaSuccess) body = cp.conditional.phGraph_out[0];
        }
        if (e == cudaSuccess)
            e = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) {
            set_error("solver relax: conditional node: %s", cudaGetErrorString(e));
            rc = -1;
        }
    }
    e = cudaStreamEndCapture(st, &s->relax_graph);
    if (rc || e != cudaSuccess) {
        if (!rc) set_error("solver relax: capture: %s", cudaGetErrorString(e));
        drop_graphs(s);
        return -1;
    }
    // the body: one step, the energy, the rule
    e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        set_error("solver relax: body capture: %s", cudaGetErrorString(e));
        drop_graphs(s);
        return -1;
    }
    rc = phase_orbitals(s, st) || phase_coefficients(s, st) ||
         orb_energy(s->M, s->d_rho1, s->d_rho2, s->d_hob, s->d_hint, s->d_E, st);
    if (!rc) {
        relax_rule_kernel<<<1, 1, 0, st>>>(s->d_ctl, s->d_E, s->N, s->imagtime, h);
        if (cudaGetLastError() != cudaSuccess) rc = -1;
    }
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(st, &out);
    if (rc || e != cudaSuccess) {
        if (!rc) set_error("solver relax: body capture: %s", cudaGetErrorString(e));
        drop_graphs(s);
        return -1;
    }
    e = cudaGraphInstantiate(&s->relax_exec, s->relax_graph, 0);
    if (e != cudaSuccess) {
        set_error("solver relax: instantiate: %s", cudaGetErrorString(e));
        drop_graphs(s);
        return -1;
    }
    return 0;
}

}  // namespace

// one phase of a step, for callers that change the trap or the interaction
// between the two phases (the reference's sync_equation_params)
int mctdhb_solver_phase(mctdhb_solver s, int phase, cudaStream_t st) {
    if (build_graphs(s)) return -1;
    MCTDHB_CUDA_TRY(cudaGraphLaunch(s->exec[phase], st));
    MCTDHB_CUDA_TRY(cudaEventRecord(s->ev_step, st));
    return 0;
}

double2* mctdhb_solver_orb_next(mctdhb_solver s) { return s->d_orb_next; }
mctdhb_space mctdhb_solver_space(mctdhb_solver s) { return s->sp; }

extern "C" {

int mctdhb_solver_create(uint16_t npar, uint16_t norb, uint16_t grid_size, double xi, double xf,
                         double d2coef, double d1coef_re, double d1coef_im, int periodic,
                         int imagtime, int rk_order, int lanczos_iter, double dt,
                         mctdhb_solver* out) {
    if (!out) {
        set_error("mctdhb_solver_create: null output");
        return -1;
    }
    *out = nullptr;
    if (rk_order != 2 && rk_order != 4 && rk_order != 5) {
        set_error("mctdhb_solver_create: Runge-Kutta order %d not in {2, 4, 5}", rk_order);
        return -1;
    }
    if (lanczos_iter < 2 || lanczos_iter > 64) {
        set_error("mctdhb_solver_create: Lanczos dimension %d outside 2..64", lanczos_iter);
        return -1;
    }
    auto* s = new mctdhb_solver_s();
    s->N = npar;
    s->M = norb;
    s->G = grid_size;
    s->imagtime = imagtime ? 1 : 0;
    s->rk_order = rk_order;
    s->lanczos_m = lanczos_iter;
    s->dt = dt;
    auto fail = [&]() {
        mctdhb_solver_destroy(s);
        return -1;
    };
    if (mctdhb_space_create(npar, norb, &s->sp)) return fail();
    if (orb_init(s->orb, norb, grid_size, xi, xf, d2coef, make_double2(d1coef_re, d1coef_im),
                 periodic, imagtime))
        return fail();
    const size_t n = (size_t)norb * grid_size, M2 = (size_t)norb * norb, M4 = M2 * M2;
    const size_t nc = mctdhb_space_dim(s->sp);
    if (cudaMalloc(&s->d_orb, n * sizeof(double2)) || cudaMalloc(&s->d_orb_next, n * sizeof(double2)) ||
        cudaMalloc(&s->d_coef, nc * sizeof(double2)) || cudaMalloc(&s->d_hob, M2 * sizeof(double2)) ||
        cudaMalloc(&s->d_hint, M4 * sizeof(double2)) || cudaMalloc(&s->d_rho1, M2 * sizeof(double2)) ||
        cudaMalloc(&s->d_rho2, M4 * sizeof(double2)) || cudaMalloc(&s->d_rinv, M2 * sizeof(double2)) ||
        cudaMalloc(&s->d_E, sizeof(double2)) || cudaMalloc(&s->d_info, sizeof(int)) ||
        cudaStreamCreateWithFlags(&s->cs, cudaStreamNonBlocking) ||
        cudaEventCreateWithFlags(&s->ev_step, cudaEventDisableTiming)) {
        set_error("mctdhb_solver_create: device allocation failed");
        return fail();
    }
    int rc = 0;
    {
        std::lock_guard<std::mutex> lk(s->sp->mu);
        if (s->sp->lw.mmax < lanczos_iter) {
            lanczos_free(s->sp->lw);
            rc = lanczos_alloc(s->sp->lw, s->sp->sp, std::max(lanczos_iter, 16));
        }
    }
    if (rc) return fail();
    *out = s;
    return 0;
}

void mctdhb_solver_destroy(mctdhb_solver s) {
    if (!s) return;
    drop_graphs(s);
    cudaFree(s->d_orb);
    cudaFree(s->d_orb_next);
    cudaFree(s->d_coef);
    cudaFree(s->d_hob);
    cudaFree(s->d_hint);
    cudaFree(s->d_rho1);
    cudaFree(s->d_rho2);
    cudaFree(s->d_rinv);
    cudaFree(s->d_E);
    cudaFree(s->d_info);
    cudaFree(s->d_ctl);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->cs) cudaStreamDestroy(s->cs);
    if (s->ev_step) cudaEventDestroy(s->ev_step);
    orb_release(s->orb);
    mctdhb_space_destroy(s->sp);
    delete s;
}

int mctdhb_solver_set_potential(mctdhb_solver s, const double* pot) {
    if (!s || !pot) {
        set_error("mctdhb_solver_set_potential: null argument");
        return -1;
    }
    // the steps may still run on a caller stream that this copy does not order with
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    MCTDHB_CUDA_TRY(cudaMemcpy(s->orb.d_pot, pot, s->G * sizeof(double), cudaMemcpyHostToDevice));
    return 0;
}

int mctdhb_solver_set_interaction(mctdhb_solver s, double g) {
    if (!s) {
        set_error("mctdhb_solver_set_interaction: null solver");
        return -1;
    }
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    MCTDHB_CUDA_TRY(cudaMemcpy(s->orb.d_g, &g, sizeof(double), cudaMemcpyHostToDevice));
    return 0;
}

int mctdhb_solver_set_regularization(mctdhb_solver s, double reg_fac) {
    if (!s || reg_fac > 1e-6 || reg_fac < 1e-13) {
        set_error("mctdhb_solver_set_regularization: factor outside [1E-13, 1E-6]");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (reg_fac == s->reg_fac) return 0;
    s->reg_fac = reg_fac;
    drop_graphs(s);  // the factor is a launch argument: capture again
    return 0;
}

// Coefficient integrator (driver.c:190-198): 20 LANCZOS (short iterative
// Lanczos, the default) or 21 RUNGEKUTTA (coefficients_integration.c:29-57,
// the solver's Runge-Kutta order).
int mctdhb_solver_set_coef_method(mctdhb_solver s, int coef_method) {
    if (!s || (coef_method != 20 && coef_method != 21)) {
        set_error("mctdhb_solver_set_coef_method: method not in {20 LANCZOS, 21 RUNGEKUTTA}");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (coef_method == s->coef_method) return 0;
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    drop_graphs(s);
    s->coef_method = coef_method;
    return 0;
}

// Derivative method of the orbital equation's linear part
// (orbital_integration.c:137-176): 302 finite differences (the default),
// 300 DVR, 301 spectral; the last two need periodic boundaries.
int mctdhb_solver_set_derivative(mctdhb_solver s, int der_method) {
    if (!s) {
        set_error("mctdhb_solver_set_derivative: null solver");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (der_method == s->orb.der) return 0;
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    drop_graphs(s);  // the linear part is part of the captured step
    if (orb_set_derivative(s->orb, der_method)) return -1;
    return s->orb.split ? orb_set_split(s->orb, 1, s->dt, s->imagtime) : 0;
}

// Orbital integrator (driver.c:165-173): 30 FULLSTEP_RUNGEKUTTA (default),
// 31 SPLITSTEP (orbital_integration.c:352-434: Crank-Nicolson half steps of
// the linear part for finite differences, the FFT exponential for DVR and
// spectral derivatives, around a Runge-Kutta step of the nonlinear part)
int mctdhb_solver_set_orb_method(mctdhb_solver s, int orb_method) {
    if (!s || (orb_method != 30 && orb_method != 31)) {
        set_error("mctdhb_solver_set_orb_method: method not in {30 FULLSTEP_RUNGEKUTTA, "
                  "31 SPLITSTEP}");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    const int split = orb_method == 31;
    if (split == s->orb.split) return 0;
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    drop_graphs(s);
    return orb_set_split(s->orb, split, s->dt, s->imagtime);
}

// The projector of the orbital equation: 0 the simple one, 1 the robust one
// with the inverse overlap matrix (orbital_integration.c:22-131; the
// reference switches when impr_ortho is set, driver.c:70-96).
int mctdhb_solver_set_orthogonality(mctdhb_solver s, int robust) {
    if (!s) {
        set_error("mctdhb_solver_set_orthogonality: null solver");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    robust = robust ? 1 : 0;
    if (robust == s->orb.robust) return 0;
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    s->orb.robust = robust;
    drop_graphs(s);  // the projector is part of the captured step
    return 0;
}

// Initial state: orbitals (M x G row-major) and coefficients (host), then the
// synchronisation the reference performs before integrating
// (dataio.c full_setup: sync_density_matrices + sync_orbital_matrices).
int mctdhb_solver_set_state(mctdhb_solver s, const void* orb, const void* coef) {
    if (!s || !orb || !coef) {
        set_error("mctdhb_solver_set_state: null argument");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    const size_t n = (size_t)s->M * s->G;
    const size_t nc = mctdhb_space_dim(s->sp);
    cudaStream_t st = s->cs;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(s->d_orb, orb, n * sizeof(double2), cudaMemcpyHostToDevice, st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(s->d_coef, coef, nc * sizeof(double2), cudaMemcpyHostToDevice, st));
    SpaceCtx& sc = s->sp->sp;
    if (dens_prepare(sc.view, s->d_coef, sc.d_dens_part, st)) return -1;
    if (dens_apply(sc.view, s->d_coef, sc.d_dens_part, s->d_rho1, s->d_rho2, sc.d_dens_desc, st))
        return -1;
    if (orb_sync_rho1(s->orb, s->d_rho1, s->d_rinv, s->reg_fac, s->d_info, st)) return -1;
    if (orb_matrices(s->orb, s->d_orb, s->d_hob, s->d_hint, st)) return -1;
    if (s->M > 1) {
        if (hc_prep(sc.view, s->d_hob, s->d_hint, sc.d_tab, st)) return -1;
        HcEpilogue ep;  // tune H.C on this state before the graph is captured
        hc_variant(sc.view, s->d_coef, s->sp->lw.out, sc.d_tab, ep, st);
    }
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(st));
    s->has_state = true;
    s->t = 0.0;
    return 0;
}

int mctdhb_solver_step(mctdhb_solver s, int nsteps, void* stream) {
    if (!s || !s->has_state) {
        set_error("mctdhb_solver_step: solver without state");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (build_graphs(s)) return -1;
    for (int i = 0; i < nsteps; i++) {
        MCTDHB_CUDA_TRY(cudaGraphLaunch(s->exec[0], (cudaStream_t)stream));
        MCTDHB_CUDA_TRY(cudaGraphLaunch(s->exec[1], (cudaStream_t)stream));
        s->t += s->dt;
    }
    MCTDHB_CUDA_TRY(cudaEventRecord(s->ev_step, (cudaStream_t)stream));
    return 0;
}

// Steps on the device until the imaginary-time energy rule or max_steps,
// with no host round trip: one launch of the relaxation graph.
int mctdhb_solver_relax(mctdhb_solver s, uint32_t max_steps, double energy_tol, int check_every,
                        void* stream) {
    if (!s || !s->has_state || max_steps < 1 || max_steps > kRelaxHardCap || check_every < 0 ||
        !(energy_tol >= 0.0)) {
        set_error("mctdhb_solver_relax: invalid argument or solver without state");
        return -1;
    }
    if (s->M == 1) {
        set_error("mctdhb_solver_relax: one orbital (no coefficients to relax); use step");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->d_ctl) {
        if (cudaMalloc(&s->d_ctl, sizeof(RelaxCtl)) != cudaSuccess ||
            cudaMallocHost(&s->h_ctl, sizeof(RelaxCtl)) != cudaSuccess) {
            set_error("mctdhb_solver_relax: allocation failed");
            return -1;
        }
    }
    if (build_relax_graph(s)) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    // the previous run's counters may still be read: order after it
    MCTDHB_CUDA_TRY(cudaStreamWaitEvent(st, s->ev_step, 0));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(st));
    *s->h_ctl = RelaxCtl{max_steps, 0u, check_every, 0, energy_tol, 0.0};
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(s->d_ctl, s->h_ctl, sizeof(RelaxCtl), cudaMemcpyHostToDevice,
                                    st));
    MCTDHB_CUDA_TRY(cudaGraphLaunch(s->relax_exec, st));
    MCTDHB_CUDA_TRY(cudaEventRecord(s->ev_step, st));
    s->relax_pending = true;
    return 0;
}

int mctdhb_solver_query(mctdhb_solver s) {
    if (!s) {
        set_error("mctdhb_solver_query: null solver");
        return -1;
    }
    const cudaError_t e = cudaEventQuery(s->ev_step);
    if (e == cudaErrorNotReady) return 0;
    MCTDHB_CUDA_TRY(e);
    return 1;
}

int mctdhb_solver_relax_result(mctdhb_solver s, uint32_t* steps, int* converged) {
    if (!s || !s->d_ctl) {
        set_error("mctdhb_solver_relax_result: no relaxation run");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    RelaxCtl c;
    MCTDHB_CUDA_TRY(cudaMemcpy(&c, s->d_ctl, sizeof(c), cudaMemcpyDeviceToHost));
    if (s->relax_pending) {
        s->t += c.steps * s->dt;
        s->relax_pending = false;
    }
    if (steps) *steps = c.steps;
    if (converged) *converged = c.conv;
    return 0;
}

// One phase of a step (0: orbitals at the current trap and interaction;
// 1: matrices of the new orbitals, SIL, densities), for callers that change
// the trap or the interaction between the two (driver.c:176-177)
int mctdhb_solver_step_phase(mctdhb_solver s, int phase, void* stream) {
    if (!s || !s->has_state || phase < 0 || phase > 1) {
        set_error("mctdhb_solver_step_phase: invalid argument or solver without state");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (mctdhb_solver_phase(s, phase, (cudaStream_t)stream)) return -1;
    if (phase == 1) s->t += s->dt;
    return 0;
}

int mctdhb_solver_kernel_count(mctdhb_solver s) {
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    if (build_graphs(s)) return -1;
    return s->kernels;
}

// Copies the state to host buffers (NULL skips a field); synchronises.
int mctdhb_solver_get(mctdhb_solver s, void* orb, void* coef, void* hob, void* hint, void* rho1,
                      void* rho2, void* rinv) {
    if (!s) {
        set_error("mctdhb_solver_get: null solver");
        return -1;
    }
    const size_t n = (size_t)s->M * s->G, M2 = (size_t)s->M * s->M, M4 = M2 * M2;
    const size_t nc = mctdhb_space_dim(s->sp);
    MCTDHB_CUDA_TRY(cudaDeviceSynchronize());
    struct {
        void* h;
        const void* d;
        size_t b;
    } cp[] = {{orb, s->d_orb, n}, {coef, s->d_coef, nc}, {hob, s->d_hob, M2},
              {hint, s->d_hint, M4}, {rho1, s->d_rho1, M2}, {rho2, s->d_rho2, M4},
              {rinv, s->d_rinv, M2}};
    for (auto& c : cp)
        if (c.h) MCTDHB_CUDA_TRY(cudaMemcpy(c.h, c.d, c.b * sizeof(double2), cudaMemcpyDeviceToHost));
    return 0;
}

// Replaces the parts of the state a caller may change between steps
// (NULL keeps a field): orbitals, coefficients, rho2, rho1^{-1}.
int mctdhb_solver_put(mctdhb_solver s, const void* orb, const void* coef, const void* rho2,
                      const void* rinv) {
    if (!s) {
        set_error("mctdhb_solver_put: null solver");
        return -1;
    }
    const size_t n = (size_t)s->M * s->G, M2 = (size_t)s->M * s->M, M4 = M2 * M2;
    const size_t nc = mctdhb_space_dim(s->sp);
    MCTDHB_CUDA_TRY(cudaDeviceSynchronize());
    struct {
        void* d;
        const void* h;
        size_t b;
    } cp[] = {{s->d_orb, orb, n}, {s->d_coef, coef, nc}, {s->d_rho2, rho2, M4},
              {s->d_rinv, rinv, M2}};
    for (auto& c : cp)
        if (c.h) MCTDHB_CUDA_TRY(cudaMemcpy(c.d, c.h, c.b * sizeof(double2), cudaMemcpyHostToDevice));
    s->has_state = true;
    return 0;
}

// E = Tr(rho1 h) + 1/2 sum rho2 g of the current state (integrator_monitor.c:56)
int mctdhb_solver_energy(mctdhb_solver s, double* e) {
    if (!s || !e) {
        set_error("mctdhb_solver_energy: null argument");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    // the steps may run on any caller stream: order after the last one
    MCTDHB_CUDA_TRY(cudaStreamWaitEvent(s->cs, s->ev_step, 0));
    if (orb_energy(s->M, s->d_rho1, s->d_rho2, s->d_hob, s->d_hint, s->d_E, s->cs)) return -1;
    double2 v;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(&v, s->d_E, sizeof(v), cudaMemcpyDeviceToHost, s->cs));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(s->cs));
    e[0] = v.x;
    e[1] = v.y;
    return 0;
}

// sum_{k<l} |<f_k|f_l>| / M of the current orbitals (integrator_monitor.c:31-42);
// fails when a step met a singular overlap matrix in the robust projector
int mctdhb_solver_overlap_residual(mctdhb_solver s, double* res) {
    if (!s || !res) {
        set_error("mctdhb_solver_overlap_residual: null argument");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    const int M = s->M;
    std::vector<double2> S((size_t)M * M);
    int fail = 0;
    MCTDHB_CUDA_TRY(cudaStreamWaitEvent(s->cs, s->ev_step, 0));
    if (orb_overlap_matrix(s->orb, s->d_orb, s->cs)) return -1;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(S.data(), s->orb.d_S, S.size() * sizeof(double2),
                                    cudaMemcpyDeviceToHost, s->cs));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(&fail, s->orb.d_fail, sizeof(int), cudaMemcpyDeviceToHost,
                                    s->cs));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(s->cs));
    if (fail) {
        set_error("mctdhb_solver: singular orbital overlap matrix in the robust projector");
        return -1;
    }
    double sum = 0.0;
    for (int k = 0; k < M; k++)
        for (int l = k + 1; l < M; l++) sum += std::hypot(S[k * M + l].x, S[k * M + l].y);
    *res = sum / M;
    return 0;
}

namespace {
// max_i |e c_i - (Hc)_i| over the grid, as the bits of a non-negative double
__global__ void resid_max_kernel(size_t n, double e, const double2* __restrict__ c,
                                 const double2* __restrict__ hc,
                                 unsigned long long* __restrict__ out) {
    double m = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, hypot(e * c[i].x - hc[i].x, e * c[i].y - hc[i].y));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
}  // namespace

// max_i |e c_i - (H c)_i| / N with the current h, g (integrator_monitor.c:9-28)
int mctdhb_solver_eig_residual(mctdhb_solver s, double e, double* res) {
    if (!s || !res || !s->has_state) {
        set_error("mctdhb_solver_eig_residual: null argument or solver without state");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    const size_t nc = mctdhb_space_dim(s->sp);
    if (s->M == 1) {  // one configuration: H c = E_gp c exactly
        *res = 0.0;
        return 0;
    }
    std::lock_guard<std::mutex> lk2(s->sp->mu);
    SpaceCtx& sc = s->sp->sp;
    unsigned long long bits = 0;
    auto* d_bits = reinterpret_cast<unsigned long long*>(s->d_E);
    MCTDHB_CUDA_TRY(cudaStreamWaitEvent(s->cs, s->ev_step, 0));
    // the step leaves h, g of the current orbitals in the H.C tables
    HcEpilogue ep;
    if (hc_apply(sc.view, s->d_coef, s->sp->lw.out, sc.d_tab, ep, s->cs)) return -1;
    MCTDHB_CUDA_TRY(cudaMemsetAsync(d_bits, 0, sizeof(bits), s->cs));
    resid_max_kernel<<<592, 256, 0, s->cs>>>(nc, e, s->d_coef, s->sp->lw.out, d_bits);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(&bits, d_bits, sizeof(bits), cudaMemcpyDeviceToHost, s->cs));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(s->cs));
    double m;
    std::memcpy(&m, &bits, sizeof(m));
    *res = m / s->N;
    return 0;
}

// Replaces the coefficients by the lowest eigenvector of H in the current
// orbitals after `niter` Lanczos iterations (multiconfig_lanczos.c,
// lowest_state_lanczos; the final diagonalisation of driver.c:296-306).  The
// density matrices are not recomputed, as there; *e is the Lanczos energy.
int mctdhb_solver_lowest_state(mctdhb_solver s, int niter, double* e) {
    if (!s || !s->has_state || niter < 1 || niter > 64) {
        set_error("mctdhb_solver_lowest_state: invalid argument or solver without state");
        return -1;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->M == 1) {
        if (e) *e = NAN;
        return 0;
    }
    std::lock_guard<std::mutex> lk2(s->sp->mu);
    MCTDHB_CUDA_TRY(cudaEventSynchronize(s->ev_step));
    if (s->sp->lw.mmax < niter) {  // the step graphs hold the old Lanczos buffers
        drop_graphs(s);
        lanczos_free(s->sp->lw);
        if (lanczos_alloc(s->sp->lw, s->sp->sp, niter)) return -1;
    }
    double* d_e = reinterpret_cast<double*>(s->d_E);
    if (lowest_state(s->sp->sp, s->sp->lw, s->d_coef, niter, d_e, s->cs)) return -1;
    double v = NAN;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(&v, d_e, sizeof(v), cudaMemcpyDeviceToHost, s->cs));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(s->cs));
    if (e) *e = v;
    return 0;
}

void* mctdhb_solver_device_coef(mctdhb_solver s) { return s ? s->d_coef : nullptr; }
void* mctdhb_solver_device_orbitals(mctdhb_solver s) { return s ? s->d_orb : nullptr; }
double mctdhb_solver_time(mctdhb_solver s) { return s ? s->t : NAN; }

}  // extern "C"
