// capi.cu -- the C ABI of libmctdhb_b200 (include/mctdhb_gpu.h).
//
// Drop-in entry points keep the reference's names, argument meanings and
// host-memory conventions; each call stages its inputs into a device
// context cached per Fock space (npar, norb), runs the kernels and copies
// the outputs back.  The device-resident API exposes the same kernels on
// device pointers and caller streams.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mctdhb_gpu.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "moves.cuh"

namespace mctdhb {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}
const char* last_error() { return g_err.c_str(); }
void clear_error() { g_err.clear(); }

std::mutex& attr_mutex() {
    static std::mutex mu;
    return mu;
}

}  // namespace mctdhb

using namespace mctdhb;

static int ensure_lanczos(mctdhb_space_s* h, int m) {
    if (h->lw.mmax >= m) return 0;
    lanczos_free(h->lw);
    return lanczos_alloc(h->lw, h->sp, std::max(m, 16));
}

// ---------------------------------------------------------------------------
// device-resident API
// ---------------------------------------------------------------------------
extern "C" {

const char* mctdhb_gpu_last_error(void) { return last_error(); }
void mctdhb_gpu_clear_error(void) { clear_error(); }

int mctdhb_space_create(uint16_t npar, uint16_t norb, mctdhb_space* out) {
    if (!out) {
        set_error("mctdhb_space_create: null output handle");
        return -1;
    }
    *out = nullptr;
    auto* h = new mctdhb_space_s();
    if (space_init(h->sp, npar, norb)) {
        delete h;
        return -1;
    }
    *out = h;
    return 0;
}

void mctdhb_space_destroy(mctdhb_space h) {
    if (!h) return;
    lanczos_free(h->lw);
    space_release(h->sp);
    delete h;
}

uint32_t mctdhb_space_dim(mctdhb_space h) { return h ? h->sp.dim : 0; }

int mctdhb_dev_set_matrices(mctdhb_space h, const void* d_hob, const void* d_hint, void* stream) {
    if (!h || !d_hob || !d_hint) {
        set_error("mctdhb_dev_set_matrices: null argument");
        return -1;
    }
    return hc_prep(h->sp.view, (const double2*)d_hob, (const double2*)d_hint, h->sp.d_tab,
                   (cudaStream_t)stream);
}

int mctdhb_dev_apply_hamiltonian(mctdhb_space h, const void* d_coef, void* d_hc, void* stream) {
    if (!h || !d_coef || !d_hc) {
        set_error("mctdhb_dev_apply_hamiltonian: null argument");
        return -1;
    }
    HcEpilogue ep;
    return hc_apply(h->sp.view, (const double2*)d_coef, (double2*)d_hc, h->sp.d_tab, ep,
                    (cudaStream_t)stream);
}

int mctdhb_dev_density_matrices(mctdhb_space h, const void* d_coef, void* d_rho1, void* d_rho2,
                                void* stream) {
    if (!h || !d_coef || !d_rho1 || !d_rho2) {
        set_error("mctdhb_dev_density_matrices: null argument");
        return -1;
    }
    return dens_apply(h->sp.view, (const double2*)d_coef, h->sp.d_dens_part, (double2*)d_rho1,
                      (double2*)d_rho2, h->sp.d_dens_desc, (cudaStream_t)stream);
}

int mctdhb_dev_sil_step(mctdhb_space h, void* d_coef, int m, double dt, int imagtime,
                        void* stream) {
    if (!h || !d_coef) {
        set_error("mctdhb_dev_sil_step: null argument");
        return -1;
    }
    if (m < 2 || m > 64) {
        set_error("mctdhb_dev_sil_step: Lanczos dimension %d outside 2..64", m);
        return -1;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    if (ensure_lanczos(h, m)) return -1;
    const double2 pdt = imagtime ? make_double2(0.0, -dt) : make_double2(dt, 0.0);
    return sil_step(h->sp, h->lw, (double2*)d_coef, m, pdt, imagtime, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// one configurational step captured as a CUDA graph
// ---------------------------------------------------------------------------
struct mctdhb_step_s {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
};

int mctdhb_step_create(mctdhb_space h, void* d_coef, void* d_rho1, void* d_rho2, int m,
                       double dt, int imagtime, mctdhb_step* out) {
    if (!h || !d_coef || !d_rho1 || !d_rho2 || !out) {
        set_error("mctdhb_step_create: null argument");
        return -1;
    }
    if (m < 2 || m > 64) {
        set_error("mctdhb_step_create: Lanczos dimension %d outside 2..64", m);
        return -1;
    }
    *out = nullptr;
    std::lock_guard<std::mutex> lk(h->mu);
    if (ensure_lanczos(h, m)) return -1;
    cudaStream_t cs;
    MCTDHB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    {
        // pick the launch variants now: a capture cannot time launches
        HcEpilogue ep;
        hc_variant(h->sp.view, (const double2*)d_coef, h->lw.out, h->sp.d_tab, ep, cs);
        if (dens_prepare(h->sp.view, (const double2*)d_coef, h->sp.d_dens_part, cs)) {
            cudaStreamDestroy(cs);
            return -1;
        }
        MCTDHB_CUDA_TRY(cudaStreamSynchronize(cs));
    }
    auto* s = new mctdhb_step_s();
    const double2 pdt = imagtime ? make_double2(0.0, -dt) : make_double2(dt, 0.0);
    int rc = 0;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = sil_step(h->sp, h->lw, (double2*)d_coef, m, pdt, imagtime, cs);
        if (!rc)
            rc = dens_apply(h->sp.view, (const double2*)d_coef, h->sp.d_dens_part,
                            (double2*)d_rho1, (double2*)d_rho2, h->sp.d_dens_desc, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &s->graph);
        if (e2 != cudaSuccess && !rc) {
            set_error("mctdhb_step_create: capture failed: %s", cudaGetErrorString(e2));
            rc = -1;
        }
    } else {
        set_error("mctdhb_step_create: %s", cudaGetErrorString(e));
        rc = -1;
    }
    cudaStreamDestroy(cs);
    if (!rc && cudaGraphInstantiate(&s->exec, s->graph, 0) != cudaSuccess) {
        set_error("mctdhb_step_create: graph instantiation failed");
        rc = -1;
    }
    if (!rc) {
        size_t n = 0;
        cudaGraphGetNodes(s->graph, nullptr, &n);
        std::vector<cudaGraphNode_t> nodes(n);
        cudaGraphGetNodes(s->graph, nodes.data(), &n);
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            cudaGraphNodeGetType(nd, &t);
            if (t == cudaGraphNodeTypeKernel) s->kernels++;
        }
    }
    if (rc) {
        if (s->exec) cudaGraphExecDestroy(s->exec);
        if (s->graph) cudaGraphDestroy(s->graph);
        delete s;
        return -1;
    }
    *out = s;
    return 0;
}

int mctdhb_step_launch(mctdhb_step s, void* stream) {
    if (!s) {
        set_error("mctdhb_step_launch: null step");
        return -1;
    }
    MCTDHB_CUDA_TRY(cudaGraphLaunch(s->exec, (cudaStream_t)stream));
    return 0;
}

int mctdhb_step_kernel_count(mctdhb_step s) { return s ? s->kernels : -1; }

void mctdhb_step_destroy(mctdhb_step s) {
    if (!s) return;
    cudaGraphExecDestroy(s->exec);
    cudaGraphDestroy(s->graph);
    delete s;
}

int mctdhb_dev_hash_table(mctdhb_space h, void* d_ht, void* stream) {
    if (!h || !d_ht) {
        set_error("mctdhb_dev_hash_table: null argument");
        return -1;
    }
    return build_hash_table(h->sp.view, (uint16_t*)d_ht, (cudaStream_t)stream);
}

int mctdhb_dev_single_jump_map(mctdhb_space h, void* d_map, void* stream) {
    if (!h || !d_map) {
        set_error("mctdhb_dev_single_jump_map: null argument");
        return -1;
    }
    return build_single_map(h->sp.view, (uint32_t*)d_map, (cudaStream_t)stream);
}

int mctdhb_dev_double_jump_chunks(mctdhb_space h, int diff, uint64_t* n_chunks) {
    if (!h || !n_chunks) {
        set_error("mctdhb_dev_double_jump_chunks: null argument");
        return -1;
    }
    uint64_t* d_cnt = nullptr;
    void* d_tmp = nullptr;
    const size_t tb = exclusive_scan_tmp_bytes(h->sp.dim);
    MCTDHB_CUDA_TRY(cudaMalloc(&d_cnt, ((size_t)h->sp.dim + 1) * sizeof(uint64_t)));
    MCTDHB_CUDA_TRY(cudaMalloc(&d_tmp, tb));
    int rc = count_double_chunks(h->sp.view, diff, d_cnt, 0);
    if (!rc) rc = exclusive_scan_u64(d_cnt, h->sp.dim, d_cnt + h->sp.dim, d_tmp, tb, 0);
    if (!rc) {
        cudaError_t e = cudaMemcpy(n_chunks, d_cnt + h->sp.dim, sizeof(uint64_t),
                                   cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            set_error("mctdhb_dev_double_jump_chunks: %s", cudaGetErrorString(e));
            rc = -1;
        }
    }
    cudaFree(d_cnt);
    cudaFree(d_tmp);
    return rc;
}

int mctdhb_dev_double_jump_map(mctdhb_space h, int diff, void* d_strides, void* d_map,
                               void* stream) {
    if (!h || !d_strides || !d_map) {
        set_error("mctdhb_dev_double_jump_map: null argument");
        return -1;
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t* off = (uint64_t*)d_strides;  // chunk offsets, then scaled in place
    void* d_tmp = nullptr;
    uint64_t* d_total = nullptr;
    const size_t tb = exclusive_scan_tmp_bytes(h->sp.dim);
    MCTDHB_CUDA_TRY(cudaMalloc(&d_tmp, tb));
    MCTDHB_CUDA_TRY(cudaMalloc(&d_total, sizeof(uint64_t)));
    int rc = count_double_chunks(h->sp.view, diff, off, st);
    if (!rc) rc = exclusive_scan_u64(off, h->sp.dim, d_total, d_tmp, tb, st);
    if (!rc) rc = build_double_map(h->sp.view, diff, off, (uint32_t*)d_map, st);
    if (!rc) rc = scale_offsets(off, h->sp.dim, (uint64_t)h->sp.M * h->sp.M, st);
    cudaStreamSynchronize(st);
    cudaFree(d_tmp);
    cudaFree(d_total);
    return rc;
}

}  // extern "C"
