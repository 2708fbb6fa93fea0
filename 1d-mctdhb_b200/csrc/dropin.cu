// dropin.cu -- the reference's own entry points (names, signatures and
// host-memory conventions of andriati-alex/1d-mctdhb) backed by the GPU
// kernels.  See include/mctdhb_gpu.h for the list and the reference
// declarations each one replaces.
//
// A device context is kept per Fock space (npar, norb): rank tables,
// coefficient/output buffers, the Lanczos workspace and a stream.  Host
// `Cmatrix` arguments (row-pointer matrices) are gathered row by row.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/mctdhb_gpu.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "small_linalg.cuh"

using namespace mctdhb;

namespace {

struct DropCtx {
    mctdhb_space h = nullptr;
    cudaStream_t st = nullptr;
    double2 *d_c = nullptr, *d_hc = nullptr, *d_hob = nullptr, *d_hint = nullptr;
    double2 *d_rho1 = nullptr, *d_rho2 = nullptr;
    double* d_scal = nullptr;
    std::mutex mu;
};

std::mutex g_ctx_mu;
std::map<std::pair<int, int>, std::unique_ptr<DropCtx>> g_ctx;

#define DROP_TRY(call)                                                                  \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
            return -1;                                                                  \
        }                                                                               \
    } while (0)

int ctx_alloc(DropCtx& c, int N, int M) {
    if (mctdhb_space_create((uint16_t)N, (uint16_t)M, &c.h)) return -1;
    const size_t dim = mctdhb_space_dim(c.h);
    const size_t M2 = (size_t)M * M, M4 = M2 * M2;
    DROP_TRY(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
    DROP_TRY(cudaMalloc(&c.d_c, dim * sizeof(double2)));
    DROP_TRY(cudaMalloc(&c.d_hc, dim * sizeof(double2)));
    DROP_TRY(cudaMalloc(&c.d_hob, M2 * sizeof(double2)));
    DROP_TRY(cudaMalloc(&c.d_hint, M4 * sizeof(double2)));
    DROP_TRY(cudaMalloc(&c.d_rho1, M2 * sizeof(double2)));
    DROP_TRY(cudaMalloc(&c.d_rho2, M4 * sizeof(double2)));
    DROP_TRY(cudaMalloc(&c.d_scal, 16 * sizeof(double)));
    return 0;
}

DropCtx* get_ctx(int N, int M) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto key = std::make_pair(N, M);
    auto it = g_ctx.find(key);
    if (it != g_ctx.end()) return it->second.get();
    auto c = std::make_unique<DropCtx>();
    if (ctx_alloc(*c, N, M)) return nullptr;
    DropCtx* p = c.get();
    g_ctx[key] = std::move(c);
    return p;
}

// host Cmatrix (rows) -> device row-major
int upload_rows(double2* d, Cmatrix m, int rows, int cols, cudaStream_t st) {
    for (int r = 0; r < rows; r++)
        DROP_TRY(cudaMemcpyAsync(d + (size_t)r * cols, m[r], cols * sizeof(double2),
                                 cudaMemcpyHostToDevice, st));
    return 0;
}

int download_rows(Cmatrix m, const double2* d, int rows, int cols, cudaStream_t st) {
    for (int r = 0; r < rows; r++)
        DROP_TRY(cudaMemcpyAsync(m[r], d + (size_t)r * cols, cols * sizeof(double2),
                                 cudaMemcpyDeviceToHost, st));
    return 0;
}

int set_matrices_from_host(DropCtx& c, int M, Cmatrix hob, Carray hint) {
    if (upload_rows(c.d_hob, hob, M, M, c.st)) return -1;
    DROP_TRY(cudaMemcpyAsync(c.d_hint, hint, (size_t)M * M * M * M * sizeof(double2),
                             cudaMemcpyHostToDevice, c.st));
    return mctdhb_dev_set_matrices(c.h, c.d_hob, c.d_hint, c.st);
}

bool check_mc(MultiConfiguration mc, const char* fn) {
    if (mc == nullptr) {
        set_error("%s: null MultiConfiguration", fn);
        return false;
    }
    return true;
}

// Rank tables for the host helpers (set_config, hash_index)
uint64_t binom_host(uint64_t n, uint64_t k) {
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (uint64_t i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return (uint64_t)r;
}

// ---- double-jump tables in the reference's 32-bit layout ----
uint32_t* double_map_host(int N, int M, int diff, uint32_t* strides) {
    mctdhb_space h = nullptr;
    if (mctdhb_space_create((uint16_t)N, (uint16_t)M, &h)) return nullptr;
    uint64_t chunks = 0;
    uint32_t* out = nullptr;
    const uint64_t M2 = (uint64_t)M * M;
    const uint32_t dim = mctdhb_space_dim(h);
    if (mctdhb_dev_double_jump_chunks(h, diff, &chunks) == 0) {
        if (chunks > UINT32_MAX / M2) {
            set_error("%s jump map of %d particles in %d orbitals needs %llu entries; it "
                      "cannot be indexed by 32-bit integers (the GPU path does not need it)",
                      diff ? "double (different orbitals)" : "double (same orbital)", N, M,
                      (unsigned long long)(chunks * M2));
        } else {
            uint64_t* d_str = nullptr;
            uint32_t* d_map = nullptr;
            const size_t entries = std::max<uint64_t>(chunks * M2, 1);
            bool ok = cudaMalloc(&d_str, ((size_t)dim + 1) * sizeof(uint64_t)) == cudaSuccess &&
                      cudaMalloc(&d_map, entries * sizeof(uint32_t)) == cudaSuccess;
            if (ok && mctdhb_dev_double_jump_map(h, diff, d_str, d_map, nullptr) == 0) {
                out = (uint32_t*)malloc(entries * sizeof(uint32_t));
                std::vector<uint64_t> st64(dim);
                if (out && cudaMemcpy(out, d_map, entries * sizeof(uint32_t),
                                      cudaMemcpyDeviceToHost) == cudaSuccess &&
                    cudaMemcpy(st64.data(), d_str, (size_t)dim * sizeof(uint64_t),
                               cudaMemcpyDeviceToHost) == cudaSuccess) {
                    if (strides)
                        for (uint32_t i = 0; i < dim; i++) strides[i] = (uint32_t)st64[i];
                } else {
                    set_error("double jump map: device copy failed");
                    free(out);
                    out = nullptr;
                }
            } else if (!ok) {
                set_error("double jump map: device allocation of %llu entries failed",
                          (unsigned long long)entries);
            }
            cudaFree(d_str);
            cudaFree(d_map);
        }
    }
    mctdhb_space_destroy(h);
    return out;
}

}  // namespace

extern "C" {

uint32_t space_dimension(uint16_t npar, uint16_t norb) {
    const uint64_t d = fock_dimension(npar, norb);
    if (d >= (uint64_t)UINT32_MAX) {
        set_error("space_dimension: %u particles in %u orbitals overflow 32-bit indices", npar,
                  norb);
        return 0;
    }
    return (uint32_t)d;
}

uint32_t* get_subspaces_dim(uint16_t npar, uint16_t norb) {
    uint32_t* s = (uint32_t*)malloc((size_t)(norb + 1) * (npar + 1) * sizeof(uint32_t));
    if (!s) {
        set_error("get_subspaces_dim: out of host memory");
        return nullptr;
    }
    for (int i = 0; i <= npar; i++) {
        s[i] = 0;
        if (norb >= 1) s[i + (npar + 1)] = 1;
        for (int j = 2; j <= norb; j++) s[i + (npar + 1) * j] = (uint32_t)fock_dimension(i, j);
    }
    return s;
}

// combinatorial-number-system decode: S = D-1-hash = sum_m C(L_m+m, m+1)
void set_config(uint32_t hash_i, uint16_t npar, uint16_t norb, uint16_t* conf) {
    const int N = npar, M = norb;
    uint64_t S = fock_dimension(N, M) - 1 - hash_i;
    int Lnext = N;
    for (int m = M - 2; m >= 0; m--) {
        int lo = 0, hi = Lnext;
        while (lo < hi) {
            int mid = (lo + hi + 1) / 2;
            if (binom_host(mid + m, m + 1) <= S)
                lo = mid;
            else
                hi = mid - 1;
        }
        S -= binom_host(lo + m, m + 1);
        conf[m + 1] = (uint16_t)(Lnext - lo);
        Lnext = lo;
    }
    conf[0] = (uint16_t)Lnext;
}

uint32_t hash_index(uint16_t npar, uint16_t norb, uint32_t* subsdim, uint16_t* conf) {
    (void)subsdim;  // the rank is computed from binomials directly
    uint64_t S = 0;
    int L = 0;
    for (int m = 0; m < norb - 1; m++) {
        L += conf[m];
        S += binom_host(L + m, m + 1);
    }
    return (uint32_t)(fock_dimension(npar, norb) - 1 - S);
}

uint16_t* get_hash_table(uint16_t npar, uint16_t norb) {
    mctdhb_space h = nullptr;
    if (mctdhb_space_create(npar, norb, &h)) return nullptr;
    const size_t n = (size_t)mctdhb_space_dim(h) * norb;
    uint16_t *d = nullptr, *out = nullptr;
    if (cudaMalloc(&d, n * sizeof(uint16_t)) == cudaSuccess &&
        mctdhb_dev_hash_table(h, d, nullptr) == 0) {
        out = (uint16_t*)malloc(n * sizeof(uint16_t));
        if (out && cudaMemcpy(out, d, n * sizeof(uint16_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
            free(out);
            out = nullptr;
        }
    }
    if (!out) set_error("get_hash_table failed: %s", last_error());
    cudaFree(d);
    mctdhb_space_destroy(h);
    return out;
}

uint32_t* get_single_jump_map(uint16_t npar, uint16_t norb, uint32_t* subsdim,
                              uint16_t* hash_table) {
    (void)subsdim;
    (void)hash_table;
    mctdhb_space h = nullptr;
    if (mctdhb_space_create(npar, norb, &h)) return nullptr;
    const uint64_t n = (uint64_t)mctdhb_space_dim(h) * norb * norb;
    uint32_t *d = nullptr, *out = nullptr;
    if (n > UINT32_MAX) {
        set_error("get_single_jump_map: %llu entries cannot be indexed by 32-bit integers",
                  (unsigned long long)n);
    } else if (cudaMalloc(&d, n * sizeof(uint32_t)) == cudaSuccess &&
               mctdhb_dev_single_jump_map(h, d, nullptr) == 0) {
        out = (uint32_t*)malloc(n * sizeof(uint32_t));
        if (out && cudaMemcpy(out, d, n * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
            free(out);
            out = nullptr;
        }
    }
    cudaFree(d);
    mctdhb_space_destroy(h);
    return out;
}

uint32_t* get_double_diffjump_map(uint16_t npar, uint16_t norb, uint32_t* subsdim,
                                  uint16_t* hash_table, uint32_t* strides) {
    (void)subsdim;
    (void)hash_table;
    return double_map_host(npar, norb, 1, strides);
}

uint32_t* get_double_equaljump_map(uint16_t npar, uint16_t norb, uint32_t* subsdim,
                                   uint16_t* hash_table, uint32_t* strides) {
    (void)subsdim;
    (void)hash_table;
    return double_map_host(npar, norb, 0, strides);
}

MultiConfiguration get_multiconf_struct(uint16_t npar, uint16_t norb) {
    if (npar == 0 || norb == 0 || norb > MAX_ORBITALS || npar > MAX_PARTICLES) {
        set_error("get_multiconf_struct: invalid %u particles / %u orbitals", npar, norb);
        return nullptr;
    }
    const uint32_t dim = space_dimension(npar, norb);
    if (dim == 0) return nullptr;
    auto* mc = (MultiConfiguration)calloc(1, sizeof(_MultiConfiguration));
    auto* om = (OperatorMappings)calloc(1, sizeof(_OperatorMappings));
    mc->npar = npar;
    mc->norb = norb;
    mc->dim = dim;
    mc->op_maps = om;
    mc->subspaces_dim = get_subspaces_dim(npar, norb);
    mc->hash_table = get_hash_table(npar, norb);
    if (!mc->hash_table) {
        destroy_multiconf_struct(mc);
        return nullptr;
    }
    om->map = get_single_jump_map(npar, norb, mc->subspaces_dim, mc->hash_table);
    om->stridett = (uint32_t*)malloc((size_t)dim * sizeof(uint32_t));
    om->strideot = (uint32_t*)malloc((size_t)dim * sizeof(uint32_t));
    om->maptt = get_double_diffjump_map(npar, norb, nullptr, nullptr, om->stridett);
    if (!om->maptt) {
        free(om->stridett);
        om->stridett = nullptr;
    }
    om->mapot = get_double_equaljump_map(npar, norb, nullptr, nullptr, om->strideot);
    if (!om->mapot) {
        free(om->strideot);
        om->strideot = nullptr;
    }
    mctdhb_gpu_clear_error();  // missing optional tables are not failures
    return mc;
}

void destroy_multiconf_struct(MultiConfiguration mc) {
    if (!mc) return;
    free(mc->subspaces_dim);
    free(mc->hash_table);
    if (mc->op_maps) {
        free(mc->op_maps->strideot);
        free(mc->op_maps->stridett);
        free(mc->op_maps->map);
        free(mc->op_maps->mapot);
        free(mc->op_maps->maptt);
        free(mc->op_maps);
    }
    free(mc);
}

void apply_hamiltonian(MultiConfiguration mc, Carray coef, Cmatrix hob, Carray hint,
                       Carray hcoef) {
    if (!check_mc(mc, "apply_hamiltonian")) return;
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t dim = mc->dim;
    if (cudaMemcpyAsync(c->d_c, coef, dim * sizeof(double2), cudaMemcpyHostToDevice, c->st) !=
            cudaSuccess ||
        set_matrices_from_host(*c, mc->norb, hob, hint) ||
        mctdhb_dev_apply_hamiltonian(c->h, c->d_c, c->d_hc, c->st) ||
        cudaMemcpyAsync(hcoef, c->d_hc, dim * sizeof(double2), cudaMemcpyDeviceToHost, c->st) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
        if (!*mctdhb_gpu_last_error()) set_error("apply_hamiltonian: CUDA failure");
    }
}

static int density_host(MultiConfiguration mc, Carray coef, DropCtx** out) {
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return -1;
    *out = c;
    if (cudaMemcpyAsync(c->d_c, coef, (size_t)mc->dim * sizeof(double2), cudaMemcpyHostToDevice,
                        c->st) != cudaSuccess)
        return -1;
    return mctdhb_dev_density_matrices(c->h, c->d_c, c->d_rho1, c->d_rho2, c->st);
}

void set_onebody_dm(MultiConfiguration mc, Carray coef, Cmatrix rho) {
    if (!check_mc(mc, "set_onebody_dm")) return;
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->mu);
    DropCtx* cc;
    if (density_host(mc, coef, &cc) || download_rows(rho, c->d_rho1, mc->norb, mc->norb, c->st) ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
        if (!*mctdhb_gpu_last_error()) set_error("set_onebody_dm: CUDA failure");
    }
}

void set_twobody_dm(MultiConfiguration mc, Carray coef, Carray rho) {
    if (!check_mc(mc, "set_twobody_dm")) return;
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t M4 = (size_t)mc->norb * mc->norb * mc->norb * mc->norb;
    DropCtx* cc;
    if (density_host(mc, coef, &cc) ||
        cudaMemcpyAsync(rho, c->d_rho2, M4 * sizeof(double2), cudaMemcpyDeviceToHost, c->st) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
        if (!*mctdhb_gpu_last_error()) set_error("set_twobody_dm: CUDA failure");
    }
}

int lanczos(MultiConfiguration mc, Cmatrix Ho, Carray Hint, int lm, Carray diag, Carray offdiag,
            Cmatrix lvec) {
    if (!check_mc(mc, "lanczos")) return -1;
    if (lm < 1 || lm > 64) {
        set_error("lanczos: %d iterations outside 1..64", lm);
        return -1;
    }
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return -1;
    std::lock_guard<std::mutex> lk(c->mu);
    mctdhb_space h = c->h;
    std::lock_guard<std::mutex> lk2(h->mu);
    if (h->lw.mmax < lm) {
        lanczos_free(h->lw);
        if (lanczos_alloc(h->lw, h->sp, std::max(lm, 16))) return -1;
    }
    const size_t dim = mc->dim;
    int iters = 0;
    if (cudaMemcpyAsync(h->lw.V, lvec[0], dim * sizeof(double2), cudaMemcpyHostToDevice, c->st) !=
            cudaSuccess ||
        set_matrices_from_host(*c, mc->norb, Ho, Hint) || lanczos_run(h->sp, h->lw, lm, c->st) ||
        lanczos_fetch(h->lw, lm, &iters, (double2*)diag, (double2*)offdiag, c->st))
        return -1;
    if (download_rows(lvec, h->lw.V, iters, (int)dim, c->st) ||
        cudaStreamSynchronize(c->st) != cudaSuccess)
        return -1;
    return iters;
}

double lowest_state_lanczos(uint16_t niter, MultiConfiguration mc, Cmatrix Ho, Carray Hint,
                            Carray C) {
    if (!check_mc(mc, "lowest_state_lanczos")) return NAN;
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return NAN;
    std::lock_guard<std::mutex> lk(c->mu);
    mctdhb_space h = c->h;
    std::lock_guard<std::mutex> lk2(h->mu);
    if (niter < 1 || niter > 64) {
        set_error("lowest_state_lanczos: %u iterations outside 1..64", niter);
        return NAN;
    }
    if (h->lw.mmax < niter) {
        lanczos_free(h->lw);
        if (lanczos_alloc(h->lw, h->sp, std::max<int>(niter, 16))) return NAN;
    }
    const size_t dim = mc->dim;
    double e = NAN;
    if (cudaMemcpyAsync(c->d_c, C, dim * sizeof(double2), cudaMemcpyHostToDevice, c->st) !=
            cudaSuccess ||
        set_matrices_from_host(*c, mc->norb, Ho, Hint) ||
        lowest_state(h->sp, h->lw, c->d_c, niter, c->d_scal, c->st) ||
        cudaMemcpyAsync(C, c->d_c, dim * sizeof(double2), cudaMemcpyDeviceToHost, c->st) !=
            cudaSuccess ||
        cudaMemcpyAsync(&e, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->st) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess)
        return NAN;
    return e;
}

void propagate_coef_sil(MCTDHBDataStruct mctdhb, Carray cnext) {
    if (!mctdhb || !mctdhb->multiconfig_space || !mctdhb->state || !mctdhb->orb_eq ||
        !mctdhb->coef_workspace || !mctdhb->coef_workspace->lan_work) {
        set_error("propagate_coef_sil: incomplete MCTDHBDataStruct");
        return;
    }
    MultiConfiguration mc = mctdhb->multiconfig_space;
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->mu);
    mctdhb_space h = c->h;
    std::lock_guard<std::mutex> lk2(h->mu);
    WorkspaceLanczos lw = mctdhb->coef_workspace->lan_work;
    const int m = lw->iter;
    if (m < 1 || m > 64) {
        set_error("propagate_coef_sil: %d Lanczos iterations outside 1..64", m);
        return;
    }
    if (h->lw.mmax < m) {
        lanczos_free(h->lw);
        if (lanczos_alloc(h->lw, h->sp, std::max(m, 16))) return;
    }
    const size_t dim = mc->dim;
    const dcomplex pdt = mctdhb->orb_eq->prop_dt;
    const double2 prop_dt = make_double2(std::real(pdt), std::imag(pdt));
    const bool imag = mctdhb->integ_type == IMAGTIME;
    int iters = 0;
    // cnext receives the Lanczos combination, state->coef the same vector
    // renormalised in imaginary time (coefficients_integration.c:152-159)
    if (cudaMemcpyAsync(c->d_c, mctdhb->state->coef, dim * sizeof(double2),
                        cudaMemcpyHostToDevice, c->st) != cudaSuccess ||
        set_matrices_from_host(*c, mc->norb, mctdhb->state->hob, mctdhb->state->hint) ||
        sil_step(h->sp, h->lw, c->d_c, m, prop_dt, 0, c->st) ||
        cudaMemcpyAsync(cnext, c->d_c, dim * sizeof(double2), cudaMemcpyDeviceToHost, c->st) !=
            cudaSuccess)
        return;
    if (imag) {
        double2 nrm;
        if (vec_dot(c->d_c, c->d_c, (uint32_t)dim, h->lw.part, h->lw.vec_grid,
                    (double2*)c->d_scal, c->st) ||
            cudaMemcpyAsync(&nrm, c->d_scal, sizeof(double2), cudaMemcpyDeviceToHost, c->st) !=
                cudaSuccess ||
            cudaStreamSynchronize(c->st) != cudaSuccess)
            return;
        const double r = 1.0 / std::sqrt(nrm.x);
        for (size_t i = 0; i < dim; i++) mctdhb->state->coef[i] = cnext[i] * r;
    } else {
        if (cudaStreamSynchronize(c->st) != cudaSuccess) return;
        std::memcpy(mctdhb->state->coef, cnext, dim * sizeof(double2));
    }
    lanczos_fetch(h->lw, m, &iters, (double2*)lw->decomp_diag, (double2*)lw->decomp_offd, c->st);
}

// synchronize.c:10-33: the regularisation factor of sync_density_matrices,
// process-wide as in the reference (atomic: callers on other threads read it)
static std::atomic<double> g_reg_fac{1e-9};

void set_regulatization_factor(double reg_fac) {
    if (reg_fac > 1e-6 || reg_fac < 1e-13) {
        set_error("set_regulatization_factor: %.1E outside [1E-13, 1E-6]", reg_fac);
        return;
    }
    g_reg_fac.store(reg_fac);
}

double get_current_regularization_factor(void) { return g_reg_fac.load(); }

void sync_density_matrices(MultiConfiguration mc, ManyBodyState psi) {
    if (!check_mc(mc, "sync_density_matrices") || !psi) return;
    DropCtx* c = get_ctx(mc->npar, mc->norb);
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->mu);
    const int M = mc->norb;
    const size_t M4 = (size_t)M * M * M * M;
    std::vector<double2> r1((size_t)M * M), rinv((size_t)M * M), work(3 * (size_t)M * M);
    std::vector<double> wd(M);
    DropCtx* cc;
    if (density_host(mc, psi->coef, &cc) ||
        cudaMemcpyAsync(r1.data(), c->d_rho1, (size_t)M * M * sizeof(double2),
                        cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaMemcpyAsync(psi->tb_denmat, c->d_rho2, M4 * sizeof(double2), cudaMemcpyDeviceToHost,
                        c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
        if (!*mctdhb_gpu_last_error()) set_error("sync_density_matrices: CUDA failure");
        return;
    }
    if (sync_rho1(M, r1.data(), rinv.data(), g_reg_fac.load(), work.data(), wd.data()) != 0)
        set_error("sync_density_matrices: one-body density matrix is singular");
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) {
            psi->ob_denmat[i][j] = dcomplex(r1[i * M + j].x, r1[i * M + j].y);
            psi->inv_ob_denmat[i][j] = dcomplex(rinv[i * M + j].x, rinv[i * M + j].y);
        }
}

dcomplex total_energy(ManyBodyState psi) {
    const int M = psi->norb, M2 = M * M, M3 = M2 * M;
    dcomplex w = 0, z = 0;
    for (int k = 0; k < M; k++)
        for (int l = 0; l < M; l++) {
            w += psi->ob_denmat[k][l] * psi->hob[k][l];
            for (int s = 0; s < M; s++)
                for (int q = 0; q < M; q++)
                    z += psi->tb_denmat[k + l * M + s * M2 + q * M3] *
                         psi->hint[k + l * M + q * M2 + s * M3];
        }
    return w + z / 2.0;
}

double eig_residual(MultiConfiguration mc, Carray cvec, Cmatrix hob, Carray hint, double e) {
    if (!check_mc(mc, "eig_residual")) return NAN;
    std::vector<dcomplex> hc(mc->dim);
    apply_hamiltonian(mc, cvec, hob, hint, hc.data());
    double mx = 0;
    for (uint32_t i = 0; i < mc->dim; i++) mx = std::max(mx, std::abs(e * cvec[i] - hc[i]));
    return mx / mc->npar;
}

}  // extern "C"
