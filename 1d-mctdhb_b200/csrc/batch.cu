// batch.cu -- host side of the batched engine (include/mctdhb_gpu.h, part 3):
// many independent MCTDHB systems of uneven (N, M, grid) resident in one HBM
// arena and advanced together, one CUDA graph launch per step of the whole
// batch.
//
//   admission   a job's exact footprint (mctdhb_batch_job_bytes) is carved
//               from the arena (first fit); the job is refused (not queued)
//               when no free slot or range is left, so a serving loop admits
//               by memory footprint.  Admission uploads the state and runs
//               the set-up the single-system solver runs before integrating
//               (rho1, rho2, regularised rho1^{-1}, h, g, energy).
//   work lists  per-slot tiles (vector rows, H.C rows and density slices per
//               orbital count, whole slots) live in device memory; the step
//               graph's persistent kernels read them at run time, so the
//               graph is captured once per set of orbital counts present and
//               systems join and leave between launches without a capture.
//   stopping    each slot stops on the device (step limit, or the
//               imaginary-time energy rule of driver.c:47-67) and is then
//               skipped by every kernel; poll/fetch/release hand it back.
// Every slot's arithmetic depends only on that slot's data and sizes, so a
// system gives the same bits alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <complex>
#include <vector>

#include "../../include/mctdhb_gpu.h"
#include "batch.h"
#include "batch_kernels.h"
#include "common.cuh"
#include "engine.h"
#include "gram.h"
#include "kernels.h"
#include "moves.cuh"
#include "orbital.h"

using namespace mctdhb;

namespace {

size_t al256(size_t b) { return (b + 255) / 256 * 256; }

// sizes of one job's parts, in the arena order
struct JobLayout {
    uint32_t nc = 0, D1 = 0, D2 = 0;
    int vtiles = 0, ytiles = 0, gs[3] = {0, 0, 0}, gk[3] = {0, 0, 0};
    size_t o_orb, o_stage, o_H, o_pot, o_w, o_Q, o_hob, o_hint, o_pw, o_lint, o_rho1, o_rho2,
        o_rinv,
        o_work, o_T, o_sq, o_g, o_V, o_out, o_part, o_py, o_gpart, o_half, o_B, total;
};

// der: 0 / 302 finite differences, 300 DVR, 301 spectral (periodic only);
// split: the split step's half-step operator and B in the arena
int job_layout(int N, int M, int G, int lz, int der, int periodic, int split, JobLayout& L) {
    if (der != 0 && der != kDerFiniteDiff && der != kDerDVR && der != kDerSpectral) {
        set_error("batch: derivative method %d not in {302, 300, 301}", der);
        return -1;
    }
    const bool toeplitz = der == kDerDVR || der == kDerSpectral;
    if (toeplitz && !periodic) {
        set_error("batch: DVR and spectral derivatives need periodic boundaries");
        return -1;
    }
    if (M < kBatchMinOrb || M > kBatchMaxOrb) {
        set_error("batch: %d orbitals outside %d..%d", M, kBatchMinOrb, kBatchMaxOrb);
        return -1;
    }
    if (N < 2 || N > 10000) {
        set_error("batch: %d particles outside 2..10000 (one boson: the single-system solver)",
                  N);
        return -1;
    }
    if (G < 5 || G > kBatchMaxGrid) {
        set_error("batch: grid of %d points outside 5..%d", G, kBatchMaxGrid);
        return -1;
    }
    const uint64_t dim = fock_dimension(N, M);
    if (dim == 0 || dim >= (uint64_t)UINT32_MAX) {
        set_error("batch: %d particles in %d orbitals exceed 32-bit configuration indices", N, M);
        return -1;
    }
    L.nc = (uint32_t)dim;
    L.D1 = (uint32_t)fock_dimension(N - 1, M);
    L.D2 = (uint32_t)fock_dimension(N - 2, M);
    L.vtiles = (int)((dim + kBatchVecRows - 1) / kBatchVecRows);
    L.ytiles = (int)((L.D2 + batch_pair_rows(M) - 1) / batch_pair_rows(M));
    // rho2 Gram slices: consecutive row tiles, at most kBatchMaxSlices (rho1
    // follows from rho2: no rho1 Gram pass)
    {
        const uint64_t ntr = (L.D2 + gram_rows(M, 2) - 1) / gram_rows(M, 2);
        L.gk[2] = (int)std::max<uint64_t>(1, (ntr + kBatchMaxSlices - 1) / kBatchMaxSlices);
        L.gs[2] = (int)((ntr + L.gk[2] - 1) / L.gk[2]);
    }
    const size_t n = (size_t)M * G, M2 = (size_t)M * M, M4 = M2 * M2, z = sizeof(double2);
    const size_t P = (size_t)M * (M + 1) / 2;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += al256(bytes);
        return at;
    };
    L.o_orb = take(n * z);
    L.o_stage = take(7 * n * z);
    L.o_H = take(n * z);
    L.o_pot = take((size_t)G * sizeof(double));
    L.o_w = take((size_t)G * sizeof(double));
    L.o_Q = take(M4 * z);
    L.o_hob = take(M2 * z);
    L.o_hint = take(M4 * z);
    L.o_pw = take((P * P + 1) * z);  // + the real-W flag (pairhc_tmpl.cuh)
    L.o_lint = take(toeplitz ? (2 * (size_t)(G - 1) - 1) * z : 0);
    L.o_rho1 = take(M2 * z);
    L.o_rho2 = take(M4 * z);
    L.o_rinv = take(M2 * z);
    L.o_work = take((3 * M2 + M + 2) * z);
    L.o_T = take((size_t)(M - 1) * (N + 1) * sizeof(uint32_t));
    L.o_sq = take((size_t)(N + 3) * sizeof(double));
    L.o_g = take(sizeof(double));
    L.o_V = take((size_t)lz * dim * z);
    L.o_out = take((size_t)dim * z);
    L.o_part = take((size_t)kBatchMaxLz * L.vtiles * z);
    L.o_py = take((size_t)L.D2 * P * z);
    L.o_gpart = take((size_t)L.gs[2] * gram_entries(M, 2) * z);
    if (split && !periodic && der != 0 && der != kDerFiniteDiff) {
        set_error("batch: the split step's FFT exponential needs periodic boundaries");
        return -1;
    }
    if (split && !periodic && G > 2048) {
        set_error("batch: split step on zero bounds limited to 2048 points");
        return -1;
    }
    L.o_half = take(split ? (periodic ? 2 * (size_t)(G - 1) - 1 : (size_t)G * G) * z : 0);
    L.o_B = take(split ? M2 * z : 0);
    L.total = o;
    return 0;
}

struct HostSlot {
    bool used = false;
    bool running = false;
    size_t off = 0, bytes = 0;
    BatchSlot d{};
    JobLayout L{};
};

constexpr int kNumM = kBatchMaxOrb + 1;  // lists indexed by M

}  // namespace

struct mctdhb_batch_s {
    int max_slots = 0, lz = 0;
    size_t arena_bytes = 0;
    char* arena = nullptr;
    std::map<size_t, size_t> free_ranges;  // offset -> bytes
    std::vector<HostSlot> hs;
    BatchSlot* d_slots = nullptr;
    double2* d_scal = nullptr;  // max_slots x BS_TOTAL
    int* d_flags = nullptr;     // max_slots x BF_TOTAL
    // work lists (device) and their pinned host images: vector tiles, and the
    // per-M lists LIST_HG, LIST_HY, LIST_G2 (batch.h)
    size_t cap_vec = 0, cap[kBatchLists] = {};
    int* d_list = nullptr;  // [0] count, [1..] slots
    BatchTile* d_vec = nullptr;
    BatchTile* d_tl[kBatchLists] = {};
    int* d_cnt = nullptr;  // count block (batch.h)
    int* h_list = nullptr;
    BatchTile* h_vec = nullptr;
    BatchTile* h_tl[kBatchLists] = {};
    int* h_cnt = nullptr;
    // single-slot lists of the admission set-up: [0] 1, [1] slot, then a
    // count block; its rho2 Gram slices at d_pro_g
    int* d_pro = nullptr;
    BatchTile* d_pro_g = nullptr;
    int* h_pro = nullptr;
    BatchTile* h_pro_g = nullptr;
    int* h_flags = nullptr;
    double2* h_scal = nullptr;
    unsigned present_mask = 0;  // orbital counts present in the lists
    bool lists_dirty = true;
    cudaStream_t st = nullptr;
    cudaStream_t side[kNumM] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kNumM] = {};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned graph_mask = 0;
    int kernels = 0;
    // the pair contraction's launch variant per orbital count, chosen by the
    // autotuner when the step graph is captured (or set by the caller)
    int pair_v[kNumM] = {};
    bool pair_v_forced[kNumM] = {};
    std::mutex mu;
};

namespace {

int* cnt_vec(int* c) { return c; }
constexpr int kCntInts = kBatchCntAll;  // with the monitor flags

void drop_graph(mctdhb_batch_s* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// arena first fit
bool arena_take(mctdhb_batch_s* b, size_t bytes, size_t* off) {
    for (auto it = b->free_ranges.begin(); it != b->free_ranges.end(); ++it) {
        if (it->second >= bytes) {
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t at = it->first + bytes;
            b->free_ranges.erase(it);
            if (rest) b->free_ranges[at] = rest;
            return true;
        }
    }
    return false;
}

void arena_give(mctdhb_batch_s* b, size_t off, size_t bytes) {
    auto it = b->free_ranges.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != b->free_ranges.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        b->free_ranges.erase(nx);
    }
    if (it != b->free_ranges.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            b->free_ranges.erase(it);
        }
    }
}

// the step's work lists from the running slots, uploaded on the engine stream
int rebuild_lists(mctdhb_batch_s* b) {
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(b->st));  // the pinned images are free to rewrite
    int ns = 0;
    size_t nv = 0;
    std::memset(b->h_cnt, 0, kCntInts * sizeof(int));
    unsigned mask = 0;
    for (int s = 0; s < b->max_slots; s++) {
        const HostSlot& h = b->hs[s];
        if (!h.used || !h.running) continue;
        b->h_list[1 + ns++] = s;
        for (int t = 0; t < h.L.vtiles; t++) b->h_vec[nv++] = BatchTile{s, (uint32_t)t};
        mask |= 1u << h.d.M;
    }
    b->h_list[0] = ns;
    cnt_vec(b->h_cnt)[0] = (int)nv;
    size_t n[kBatchLists] = {};
    for (int M = kBatchMinOrb; M <= kBatchMaxOrb; M++) {
        for (int li = 0; li < kBatchLists; li++) batch_offs(b->h_cnt, li)[M] = (int)n[li];
        for (int q = 0; q < ns; q++) {
            const int s = b->h_list[1 + q];
            const HostSlot& h = b->hs[s];
            if (h.d.M != M) continue;
            BatchTile* const* tl = b->h_tl;
            auto push = [&](int li, uint32_t idx) {
                if (n[li] < b->cap[li]) tl[li][n[li]] = BatchTile{s, idx};
                n[li]++;
            };
            for (uint32_t r = 0; r < h.L.nc; r += kBatchHcRows) push(LIST_HG, r);
            for (int t = 0; t < h.L.ytiles; t++) push(LIST_HY, (uint32_t)t);
            for (int g = 0; g < h.L.gs[2]; g++) push(LIST_G2, (uint32_t)g);
        }
        for (int li = 0; li < kBatchLists; li++)
            batch_cnts(b->h_cnt, li)[M] = (int)n[li] - batch_offs(b->h_cnt, li)[M];
    }
    bool over = nv > b->cap_vec;
    for (int li = 0; li < kBatchLists; li++) over = over || n[li] > b->cap[li];
    if (over) {
        set_error("batch: work lists exceed their capacity");
        return -1;
    }
    cudaStream_t st = b->st;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(b->d_list, b->h_list, (1 + ns) * sizeof(int),
                                    cudaMemcpyHostToDevice, st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(b->d_cnt, b->h_cnt, kCntInts * sizeof(int),
                                    cudaMemcpyHostToDevice, st));
    if (nv)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(b->d_vec, b->h_vec, nv * sizeof(BatchTile),
                                        cudaMemcpyHostToDevice, st));
    for (int li = 0; li < kBatchLists; li++)
        if (n[li])
            MCTDHB_CUDA_TRY(cudaMemcpyAsync(b->d_tl[li], b->h_tl[li], n[li] * sizeof(BatchTile),
                                            cudaMemcpyHostToDevice, st));
    b->present_mask = mask;
    b->lists_dirty = false;
    return 0;
}

// H.C of Lanczos iteration `iter` of the slots of orbital count M
int hc_group(int M, const BatchSlot* slots, const BatchTile* hy, const BatchTile* hg,
             const int* cnt, int iter, cudaStream_t st, int parts = 3, int v = 0) {
    switch (M) {
        case 2: return hcp_batch_launch<2>(slots, hy, hg, cnt, iter, parts, v, st);
        case 3: return hcp_batch_launch<3>(slots, hy, hg, cnt, iter, parts, v, st);
        case 4: return hcp_batch_launch<4>(slots, hy, hg, cnt, iter, parts, v, st);
        case 5: return hcp_batch_launch<5>(slots, hy, hg, cnt, iter, parts, v, st);
        case 6: return hcp_batch_launch<6>(slots, hy, hg, cnt, iter, parts, v, st);
        case 7: return hcp_batch_launch<7>(slots, hy, hg, cnt, iter, parts, v, st);
        case 8: return hcp_batch_launch<8>(slots, hy, hg, cnt, iter, parts, v, st);
    }
    return 0;
}

// the batched contraction variants (0 and 2, pairhc_tmpl.cuh)
bool batch_v_ok(int M, int v) {
    return M >= kBatchMinOrb && M <= kBatchMaxOrb &&
           (v == 3 || ((v == 0 || v == 2) && pair_variant_ok(M, v)));
}

// rho1 / rho2 of the slots of orbital count M (the slot list gives the
// finalize blocks)
int dens_group(int M, const BatchSlot* slots, const BatchTile* g2, const int* cnt,
               const int* list, const int* nlist, int nblocks, cudaStream_t st) {
    switch (M) {
        case 2: return gram_batch_launch<2>(slots, g2, cnt, list, nlist, nblocks, st);
        case 3: return gram_batch_launch<3>(slots, g2, cnt, list, nlist, nblocks, st);
        case 4: return gram_batch_launch<4>(slots, g2, cnt, list, nlist, nblocks, st);
        case 5: return gram_batch_launch<5>(slots, g2, cnt, list, nlist, nblocks, st);
        case 6: return gram_batch_launch<6>(slots, g2, cnt, list, nlist, nblocks, st);
        case 7: return gram_batch_launch<7>(slots, g2, cnt, list, nlist, nblocks, st);
        case 8: return gram_batch_launch<8>(slots, g2, cnt, list, nlist, nblocks, st);
    }
    return 0;
}

// launch attributes of the per-M kernels (before any capture)
int prepare_group(int M) {
    switch (M) {
        case 2: return batch_prepare<2>();
        case 3: return batch_prepare<3>();
        case 4: return batch_prepare<4>();
        case 5: return batch_prepare<5>();
        case 6: return batch_prepare<6>();
        case 7: return batch_prepare<7>();
        case 8: return batch_prepare<8>();
    }
    return 0;
}

// one launch per orbital count present, on parallel branches of the graph
template <class F>
int per_group(mctdhb_batch_s* b, unsigned mask, F&& launch) {
    int groups = 0;
    for (int M = kBatchMinOrb; M <= kBatchMaxOrb; M++)
        if (mask >> M & 1) groups++;
    if (groups <= 1) {
        for (int M = kBatchMinOrb; M <= kBatchMaxOrb; M++)
            if (mask >> M & 1)
                if (launch(M, b->st)) return -1;
        return 0;
    }
    MCTDHB_CUDA_TRY(cudaEventRecord(b->ev_fork, b->st));
    for (int M = kBatchMinOrb; M <= kBatchMaxOrb; M++) {
        if (!(mask >> M & 1)) continue;
        MCTDHB_CUDA_TRY(cudaStreamWaitEvent(b->side[M], b->ev_fork, 0));
        if (launch(M, b->side[M])) return -1;
        MCTDHB_CUDA_TRY(cudaEventRecord(b->ev_join[M], b->side[M]));
    }
    for (int M = kBatchMinOrb; M <= kBatchMaxOrb; M++)
        if (mask >> M & 1) MCTDHB_CUDA_TRY(cudaStreamWaitEvent(b->st, b->ev_join[M], 0));
    return 0;
}

// the launch sequence of one batch step (captured into the step graph)
int enqueue_step(mctdhb_batch_s* b, unsigned mask) {
    cudaStream_t st = b->st;
    const BatchSlot* S = b->d_slots;
    const int* nL = b->d_list;  // count in element 0, slots from element 1
    const int* sl = b->d_list + 1;
    const BatchTile* V = b->d_vec;
    const int* nV = cnt_vec(b->d_cnt);
    const int vgrid = num_sms() * 8, sgrid = b->max_slots;
    const int lz = b->lz;
    int* mon = batch_mon(b->d_cnt);
    bt_orbital_kernel<<<sgrid, kBatchOrbThreads, kBatchMaxGrid * sizeof(double), st>>>(S, sl, nL, 0,
                                                                                       mon);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    auto hc = [&](int iter) {
        return per_group(b, mask, [&](int M, cudaStream_t s) {
            return hc_group(M, S, b->d_tl[LIST_HY], b->d_tl[LIST_HG], b->d_cnt, iter, s, 3,
                            b->pair_v[M]);
        });
    };
    // Lanczos (multiconfig_lanczos.c:12-90)
    if (hc(0)) return -1;
    bt_dot_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV, 0);
    bt_reduce_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL, 1, BS_DIAG, 0);
    for (int i = 0; i < lz - 1; i++) {
        bt_subdots(i, vgrid, st, S, V, nV);
        bt_reduce_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL, i + 1, BS_ORTHO, 1);
        bt_orth_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV, i);
        bt_norm_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL, i);
        bt_scale_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV, i);
        MCTDHB_CUDA_TRY(cudaGetLastError());
        if (hc(i + 1)) return -1;
        bt_dot_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV, i + 1);
        bt_reduce_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL, 1, BS_DIAG + i + 1, 1);
    }
    // SIL combination and renormalisation (coefficients_integration.c:59-160)
    bt_small_kernel<<<sgrid, 32, 0, st>>>(S, sl, nL);
    bt_combine_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV);
    bt_norm2_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV);
    bt_reduce_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL, 1, BS_MISC + 2, 0);
    bt_renorm_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    // densities, rho1 synchronisation, energy, stop rules
    if (per_group(b, mask, [&](int M, cudaStream_t s) {
            return dens_group(M, S, b->d_tl[LIST_G2], b->d_cnt, sl, nL, sgrid, s);
        }))
        return -1;
    bt_tail_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL, 0, mon);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    // the monitor: the eigen residual of the slots whose energy rule passed
    // in this step with eig_tol set (driver.c:47-67); every launch returns at
    // once when no slot of its orbital count needs it
    if (hc(kBatchMonIter)) return -1;
    bt_resid_kernel<<<vgrid, kBatchVecThreads, 0, st>>>(S, V, nV);
    bt_monitor_kernel<<<sgrid, kBatchVecThreads, 0, st>>>(S, sl, nL);
    MCTDHB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int count_graph_kernels(cudaGraph_t g) {
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

// the autotuner's choice of the contraction variant of orbital count M for
// the current jobs (key: M and the group's (N-2)-space rows, to a factor of
// 2), timed on the jobs' own coefficients before the capture
struct BatchTuneCtx {
    mctdhb_batch_s* b;
    int M;
};
int batch_tune_launch(void* p, int v, cudaStream_t st) {
    auto* c = (BatchTuneCtx*)p;
    if (!batch_v_ok(c->M, v)) return 1;
    return hc_group(c->M, c->b->d_slots, c->b->d_tl[LIST_HY], c->b->d_tl[LIST_HG], c->b->d_cnt,
                    0, st, 1, v);
}

int tune_group(mctdhb_batch_s* b, int M) {
    if (b->pair_v_forced[M]) return 0;
    uint64_t rows = 0;
    for (const HostSlot& h : b->hs)
        if (h.used && h.running && h.d.M == M) rows += h.L.D2;
    int bucket = 0;
    while ((1ull << bucket) < rows) bucket++;
    BatchTuneCtx ctx{b, M};
    const int v = tune_pick("bhcp_y", bucket, M, kBatchPairVariants, b->st, batch_tune_launch,
                            &ctx);
    b->pair_v[M] = batch_v_ok(M, v) ? v : 0;
    return 0;
}

int ensure_graph(mctdhb_batch_s* b) {
    if (b->exec && b->graph_mask == b->present_mask) return 0;
    drop_graph(b);
    for (int M = kBatchMinOrb; M <= kBatchMaxOrb; M++)
        if (b->present_mask >> M & 1)
            if (prepare_group(M) || tune_group(b, M)) return -1;
    cudaError_t e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        set_error("batch: capture: %s", cudaGetErrorString(e));
        return -1;
    }
    const int rc = enqueue_step(b, b->present_mask);
    e = cudaStreamEndCapture(b->st, &b->graph);
    if (rc) {
        if (b->graph) cudaGraphDestroy(b->graph);
        b->graph = nullptr;
        return -1;
    }
    if (e != cudaSuccess || cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
        set_error("batch: graph capture failed: %s", cudaGetErrorString(e));
        drop_graph(b);
        return -1;
    }
    b->graph_mask = b->present_mask;
    b->kernels = count_graph_kernels(b->graph);
    return 0;
}

uint32_t binom_u32(int n, int k) {
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    uint64_t r = 1;
    for (int i = 1; i <= k; i++) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
    return (uint32_t)r;
}

}  // namespace

extern "C" {

size_t mctdhb_batch_job_bytes(const mctdhb_job* job, int lanczos_iter) {
    if (!job) return 0;
    JobLayout L;
    if (job_layout(job->npar, job->norb, job->grid_size, lanczos_iter, job->der_method,
                   job->periodic, job->orb_method == 31, L))
        return 0;
    return L.total;
}

int mctdhb_batch_create(int max_slots, size_t arena_bytes, int lanczos_iter, mctdhb_batch* out) {
    if (!out) {
        set_error("mctdhb_batch_create: null output");
        return -1;
    }
    *out = nullptr;
    if (max_slots < 1 || max_slots > 65536) {
        set_error("mctdhb_batch_create: %d slots outside 1..65536", max_slots);
        return -1;
    }
    if (lanczos_iter < 2 || lanczos_iter > kBatchMaxLz) {
        set_error("mctdhb_batch_create: Lanczos dimension %d outside 2..%d", lanczos_iter,
                  kBatchMaxLz);
        return -1;
    }
    auto* b = new mctdhb_batch_s();
    b->max_slots = max_slots;
    b->lz = lanczos_iter;
    b->arena_bytes = arena_bytes / 256 * 256;
    b->hs.resize(max_slots);
    auto fail = [&]() {
        mctdhb_batch_destroy(b);
        return -1;
    };
    // every job holds at least (lz + 1) nc complex numbers: bounds the tiles
    const size_t max_rows = b->arena_bytes / ((size_t)(lanczos_iter + 1) * sizeof(double2));
    // (the Y tiles and Gram row tiles have at least 64 rows each)
    b->cap_vec = max_rows / kBatchVecRows + max_slots;
    b->cap[LIST_HG] = max_rows / kBatchHcRows + max_slots;
    b->cap[LIST_HY] = max_rows / 64 + max_slots;
    b->cap[LIST_G2] = max_rows / 64 + max_slots;
    bool bad = cudaMalloc(&b->arena, std::max<size_t>(b->arena_bytes, 256)) ||
               cudaMalloc(&b->d_slots, max_slots * sizeof(BatchSlot)) ||
               cudaMalloc(&b->d_scal, (size_t)max_slots * BS_TOTAL * sizeof(double2)) ||
               cudaMalloc(&b->d_flags, (size_t)max_slots * BF_TOTAL * sizeof(int)) ||
               cudaMalloc(&b->d_list, (max_slots + 1) * sizeof(int)) ||
               cudaMalloc(&b->d_vec, b->cap_vec * sizeof(BatchTile)) ||
               cudaMalloc(&b->d_cnt, kCntInts * sizeof(int)) ||
               cudaMalloc(&b->d_pro, (2 + kCntInts) * sizeof(int)) ||
               cudaMalloc(&b->d_pro_g, kBatchMaxSlices * sizeof(BatchTile)) ||
               cudaMallocHost(&b->h_list, (max_slots + 1) * sizeof(int)) ||
               cudaMallocHost(&b->h_vec, b->cap_vec * sizeof(BatchTile)) ||
               cudaMallocHost(&b->h_cnt, kCntInts * sizeof(int)) ||
               cudaMallocHost(&b->h_pro, (2 + kCntInts) * sizeof(int)) ||
               cudaMallocHost(&b->h_pro_g, kBatchMaxSlices * sizeof(BatchTile));
    for (int li = 0; li < kBatchLists && !bad; li++)
        bad = cudaMalloc(&b->d_tl[li], b->cap[li] * sizeof(BatchTile)) ||
              cudaMallocHost(&b->h_tl[li], b->cap[li] * sizeof(BatchTile));
    // the engine's stream (and with it every launch of its step graph) takes
    // the device's highest priority: a batch of many small jobs shares the
    // GPU with work on other streams (a serving loop's one-at-a-time lane for
    // jobs that fill the GPU alone) and its short kernels go first whenever
    // SMs free up
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (bad ||
        cudaMallocHost(&b->h_flags, (size_t)max_slots * BF_TOTAL * sizeof(int)) ||
        cudaMallocHost(&b->h_scal, (size_t)max_slots * BS_TOTAL * sizeof(double2)) ||
        cudaStreamCreateWithPriority(&b->st, cudaStreamNonBlocking, prio_hi) ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming)) {
        set_error("mctdhb_batch_create: device allocation of %zu bytes failed", b->arena_bytes);
        return fail();
    }
    for (int M = 0; M < kNumM; M++)
        if (cudaStreamCreateWithPriority(&b->side[M], cudaStreamNonBlocking, prio_hi) ||
            cudaEventCreateWithFlags(&b->ev_join[M], cudaEventDisableTiming)) {
            set_error("mctdhb_batch_create: stream creation failed");
            return fail();
        }
    if (cudaMemset(b->d_flags, 0, (size_t)max_slots * BF_TOTAL * sizeof(int)) ||
        cudaMemset(b->d_scal, 0, (size_t)max_slots * BS_TOTAL * sizeof(double2)) ||
        cudaMemset(b->d_slots, 0, max_slots * sizeof(BatchSlot))) {
        set_error("mctdhb_batch_create: initialisation failed");
        return fail();
    }
    if (b->arena_bytes) b->free_ranges[0] = b->arena_bytes;
    if (rebuild_lists(b)) return fail();
    *out = b;
    return 0;
}

void mctdhb_batch_destroy(mctdhb_batch b) {
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    drop_graph(b);
    cudaFree(b->arena);
    cudaFree(b->d_slots);
    cudaFree(b->d_scal);
    cudaFree(b->d_flags);
    cudaFree(b->d_list);
    cudaFree(b->d_vec);
    cudaFree(b->d_cnt);
    cudaFree(b->d_pro);
    cudaFree(b->d_pro_g);
    for (int li = 0; li < kBatchLists; li++) {
        cudaFree(b->d_tl[li]);
        cudaFreeHost(b->h_tl[li]);
    }
    for (int M = 0; M < kNumM; M++) {
        if (b->side[M]) cudaStreamDestroy(b->side[M]);
        if (b->ev_join[M]) cudaEventDestroy(b->ev_join[M]);
    }
    cudaFreeHost(b->h_list);
    cudaFreeHost(b->h_vec);
    cudaFreeHost(b->h_cnt);
    cudaFreeHost(b->h_pro);
    cudaFreeHost(b->h_pro_g);
    cudaFreeHost(b->h_flags);
    cudaFreeHost(b->h_scal);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

int mctdhb_batch_admit(mctdhb_batch b, const mctdhb_job* job, int* slot) {
    if (!b || !job || !slot || !job->pot || !job->orbitals || !job->coef) {
        set_error("mctdhb_batch_admit: null argument");
        return -1;
    }
    *slot = -1;
    if (job->rk_order != 2 && job->rk_order != 4 && job->rk_order != 5) {
        set_error("mctdhb_batch_admit: Runge-Kutta order %d not in {2, 4, 5}", job->rk_order);
        return -1;
    }
    if (!(job->dt > 0) || job->max_steps < 1) {
        set_error("mctdhb_batch_admit: need dt > 0 and at least one step");
        return -1;
    }
    if (job->eig_tol < 0 || job->ortho_tol < 0 || job->ortho_tol > kOverlapAbort) {
        set_error("mctdhb_batch_admit: need eig_tol >= 0 and 0 <= ortho_tol <= %g", kOverlapAbort);
        return -1;
    }
    const double reg = job->reg_fac > 0 ? job->reg_fac : 1e-9;
    std::lock_guard<std::mutex> lk(b->mu);
    JobLayout L;
    const int split = job->orb_method == 31;
    if (job->orb_method != 0 && job->orb_method != 30 && !split) {
        set_error("mctdhb_batch_admit: orbital method %d not in {30 FULLSTEP_RUNGEKUTTA, "
                  "31 SPLITSTEP}", job->orb_method);
        return -1;
    }
    if (job_layout(job->npar, job->norb, job->grid_size, b->lz, job->der_method, job->periodic,
                   split, L))
        return -1;
    int s = -1;
    for (int i = 0; i < b->max_slots; i++)
        if (!b->hs[i].used) {
            s = i;
            break;
        }
    size_t off = 0;
    if (s < 0 || !arena_take(b, L.total, &off)) return 1;  // no room now
    HostSlot& h = b->hs[s];
    h = HostSlot();
    h.used = true;
    h.running = true;
    h.off = off;
    h.bytes = L.total;
    h.L = L;
    const int N = job->npar, M = job->norb, G = job->grid_size;
    const size_t n = (size_t)M * G;
    char* base = b->arena + off;
    auto P = [&](size_t o) { return (void*)(base + o); };
    BatchSlot& d = h.d;
    d.N = N;
    d.M = M;
    d.G = G;
    d.imag = job->imagtime ? 1 : 0;
    d.rk = job->rk_order;
    d.check_every = job->check_every;
    d.lz = b->lz;
    d.nc = L.nc;
    d.max_steps = job->max_steps;
    d.vtiles = L.vtiles;
    d.ytiles = L.ytiles;
    for (int R = 0; R < 3; R++) {
        d.gs[R] = L.gs[R];
        d.gk[R] = L.gk[R];
    }
    d.D1 = L.D1;
    d.dt = job->dt;
    d.etol = job->energy_tol;
    d.reg_fac = reg;
    d.eig_tol = job->eig_tol > 0 ? job->eig_tol : 0.0;
    d.ortho_tol = job->ortho_tol > 0 ? job->ortho_tol : kOrthoSwitch;
    d.pdt = d.imag ? make_double2(0.0, -job->dt) : make_double2(job->dt, 0.0);
    d.ov.M = M;
    d.ov.G = G;
    d.ov.periodic = job->periodic ? 1 : 0;
    d.ov.dx = (job->xf - job->xi) / (G - 1);
    d.ov.a2 = job->d2coef;
    d.ov.a1 = make_double2(job->d1coef_re, job->d1coef_im);
    d.ov.tf = d.imag ? make_double2(0.0, -1.0) : make_double2(1.0, 0.0);
    d.ov.w = (const double*)P(L.o_w);
    d.ov.pot = (const double*)P(L.o_pot);
    const bool toeplitz = job->der_method == kDerDVR || job->der_method == kDerSpectral;
    d.ov.lin_t = toeplitz ? (const double2*)P(L.o_lint) : nullptr;
    d.sp.N = N;
    d.sp.M = M;
    d.sp.dim = L.nc;
    d.sp.T = (const uint32_t*)P(L.o_T);
    d.sp.sq = (const double*)P(L.o_sq);
    d.sp.dim2 = L.D2;
    d.sp.pair_w = (double2*)P(L.o_pw);
    d.sp.pair_y = (double2*)P(L.o_py);
    d.g = (const double*)P(L.o_g);
    d.orb = (double2*)P(L.o_orb);
    d.stage = (double2*)P(L.o_stage);
    d.H = (double2*)P(L.o_H);
    d.Q = (double2*)P(L.o_Q);
    d.hob = (double2*)P(L.o_hob);
    d.hint = (double2*)P(L.o_hint);
    d.rho1 = (double2*)P(L.o_rho1);
    d.rho2 = (double2*)P(L.o_rho2);
    d.rinv = (double2*)P(L.o_rinv);
    d.work = (double2*)P(L.o_work);
    d.V = (double2*)P(L.o_V);
    d.out = (double2*)P(L.o_out);
    d.part = (double2*)P(L.o_part);
    d.gpart = (double2*)P(L.o_gpart);
    d.scal = b->d_scal + (size_t)s * BS_TOTAL;
    d.flags = b->d_flags + (size_t)s * BF_TOTAL;
    // host-side tables (the rank table of space_init, Simpson weights)
    std::vector<uint32_t> T((size_t)(M - 1) * (N + 1));
    for (int m = 0; m < M - 1; m++)
        for (int l = 0; l <= N; l++) T[(size_t)m * (N + 1) + l] = binom_u32(l + m, m + 1);
    std::vector<double> sq(N + 3);
    for (int x = 0; x < N + 3; x++) sq[x] = std::sqrt((double)x);
    const std::vector<double> w = simpson_weights(G, d.ov.dx);
    // DVR / spectral: the Toeplitz kernel of the solver's orbital step
    const std::vector<double2> lint =
        toeplitz ? derivative_toeplitz(job->der_method, G, d.ov.dx, d.ov.a2,
                                       std::complex<double>(d.ov.a1.x, d.ov.a1.y))
                 : std::vector<double2>();
    // the split step's half-step operator (the single-system solver's own)
    std::vector<double2> half;
    d.split = split;
    d.half_dense = 0;
    d.half = split ? (const double2*)P(L.o_half) : nullptr;
    d.B = split ? (double2*)P(L.o_B) : nullptr;
    if (split && split_half_operator(G, d.ov.dx, d.ov.a2, d.ov.a1, d.ov.periodic,
                                     job->der_method == 0 ? kDerFiniteDiff : job->der_method,
                                     job->dt, d.imag, half, &d.half_dense)) {
        arena_give(b, h.off, h.bytes);
        h = HostSlot();
        return -1;
    }
    int fl[BF_TOTAL] = {0};
    fl[BF_STATE] = SLOT_RUNNING;
    fl[BF_ROBUST] = job->impr_ortho ? 1 : 0;
    cudaStream_t st = b->st;
    auto undo = [&]() {
        arena_give(b, h.off, h.bytes);
        h = HostSlot();
        return -1;
    };
    if (cudaStreamSynchronize(st) ||
        cudaMemcpyAsync(d.orb, job->orbitals, n * sizeof(double2), cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(d.V, job->coef, (size_t)L.nc * sizeof(double2), cudaMemcpyHostToDevice,
                        st) ||
        cudaMemcpyAsync((void*)d.ov.pot, job->pot, G * sizeof(double), cudaMemcpyHostToDevice,
                        st) ||
        cudaMemcpyAsync((void*)d.ov.w, w.data(), G * sizeof(double), cudaMemcpyHostToDevice, st) ||
        (toeplitz && cudaMemcpyAsync((void*)d.ov.lin_t, lint.data(), lint.size() * sizeof(double2),
                                     cudaMemcpyHostToDevice, st)) ||
        (split && cudaMemcpyAsync((void*)d.half, half.data(), half.size() * sizeof(double2),
                                  cudaMemcpyHostToDevice, st)) ||
        cudaMemcpyAsync((void*)d.sp.T, T.data(), T.size() * sizeof(uint32_t),
                        cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync((void*)d.sp.sq, sq.data(), sq.size() * sizeof(double),
                        cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync((void*)d.g, &job->g, sizeof(double), cudaMemcpyHostToDevice, st) ||
        cudaMemsetAsync(d.scal, 0, BS_TOTAL * sizeof(double2), st) ||
        cudaMemcpyAsync(d.flags, fl, sizeof(fl), cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(b->d_slots + s, &d, sizeof(BatchSlot), cudaMemcpyHostToDevice, st)) {
        set_error("mctdhb_batch_admit: upload failed");
        return undo();
    }
    // set-up (mctdhb_solver_set_state): rho1, rho2 and rho1^{-1} of the
    // initial coefficients, h and g of the initial orbitals, the energy
    int* hp = b->h_pro;
    std::memset(hp, 0, (2 + kCntInts) * sizeof(int));
    hp[0] = 1;
    hp[1] = s;
    int* pc = hp + 2;
    batch_offs(pc, LIST_G2)[M] = 0;
    batch_cnts(pc, LIST_G2)[M] = L.gs[2];
    for (int q = 0; q < L.gs[2]; q++) b->h_pro_g[q] = BatchTile{s, (uint32_t)q};
    const int* pl = b->d_pro;
    const int* dpc = b->d_pro + 2;
    if (cudaMemcpyAsync(b->d_pro, hp, (2 + kCntInts) * sizeof(int), cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(b->d_pro_g, b->h_pro_g, kBatchMaxSlices * sizeof(BatchTile),
                        cudaMemcpyHostToDevice, st)) {
        set_error("mctdhb_batch_admit: upload failed");
        return undo();
    }
    bt_orbital_kernel<<<1, kBatchOrbThreads, kBatchMaxGrid * sizeof(double), st>>>(
        b->d_slots, pl + 1, pl, 1, nullptr);
    if (prepare_group(M) ||
        dens_group(M, b->d_slots, b->d_pro_g, dpc, pl + 1, pl, 1, st))
        return undo();
    bt_tail_kernel<<<1, kBatchVecThreads, 0, st>>>(b->d_slots, pl + 1, pl, 1, nullptr);
    const cudaError_t e = cudaGetLastError();
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        set_error("mctdhb_batch_admit: set-up failed: %s",
                  cudaGetErrorString(e != cudaSuccess ? e : e2));
        return undo();
    }
    b->lists_dirty = true;
    *slot = s;
    return 0;
}

int mctdhb_batch_step(mctdhb_batch b, int nsteps) {
    if (!b || nsteps < 0) {
        set_error("mctdhb_batch_step: invalid argument");
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    if (b->lists_dirty && rebuild_lists(b)) return -1;
    if (b->present_mask == 0) return 0;  // nothing running
    if (ensure_graph(b)) return -1;
    for (int i = 0; i < nsteps; i++) MCTDHB_CUDA_TRY(cudaGraphLaunch(b->exec, b->st));
    return 0;
}

int mctdhb_batch_sync(mctdhb_batch b) {
    if (!b) {
        set_error("mctdhb_batch_sync: null batch");
        return -1;
    }
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(b->st));
    return 0;
}

int mctdhb_batch_poll(mctdhb_batch b, int* state, uint32_t* steps, double* energy) {
    if (!b) {
        set_error("mctdhb_batch_poll: null batch");
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    const int S = b->max_slots;
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(b->h_flags, b->d_flags, (size_t)S * BF_TOTAL * sizeof(int),
                                    cudaMemcpyDeviceToHost, b->st));
    if (energy)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(b->h_scal, b->d_scal,
                                        (size_t)S * BS_TOTAL * sizeof(double2),
                                        cudaMemcpyDeviceToHost, b->st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(b->st));
    int running = 0;
    for (int s = 0; s < S; s++) {
        HostSlot& h = b->hs[s];
        const int* f = b->h_flags + (size_t)s * BF_TOTAL;
        const int stt = h.used ? f[BF_STATE] : SLOT_EMPTY;
        if (h.used && h.running && stt != SLOT_RUNNING) {
            h.running = false;
            b->lists_dirty = true;  // drop the stopped slot's tiles
        }
        if (stt == SLOT_RUNNING) running++;
        if (state) state[s] = stt;
        if (steps) steps[s] = h.used ? (uint32_t)f[BF_STEPS] : 0u;
        if (energy) energy[s] = h.used ? b->h_scal[(size_t)s * BS_TOTAL + BS_MISC + 3].x : 0.0;
    }
    return running;
}

int mctdhb_batch_fetch(mctdhb_batch b, int slot, void* orbitals, void* coef, void* rho1,
                       void* rho2, double* energy, uint32_t* steps, int* converged) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->hs[slot].used) {
        set_error("mctdhb_batch_fetch: no job in slot %d", slot);
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    const HostSlot& h = b->hs[slot];
    const BatchSlot& d = h.d;
    cudaStream_t st = b->st;
    const size_t n = (size_t)d.M * d.G, M2 = (size_t)d.M * d.M;
    int fl[BF_TOTAL];
    double2 sc[BS_TOTAL];
    if (orbitals)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(orbitals, d.orb, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
    if (coef)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(coef, d.V, (size_t)d.nc * sizeof(double2),
                                        cudaMemcpyDeviceToHost, st));
    if (rho1)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(rho1, d.rho1, M2 * sizeof(double2), cudaMemcpyDeviceToHost, st));
    if (rho2)
        MCTDHB_CUDA_TRY(cudaMemcpyAsync(rho2, d.rho2, M2 * M2 * sizeof(double2),
                                        cudaMemcpyDeviceToHost, st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(fl, d.flags, sizeof(fl), cudaMemcpyDeviceToHost, st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(sc, d.scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(st));
    if (energy) *energy = sc[BS_MISC + 3].x;
    if (steps) *steps = (uint32_t)fl[BF_STEPS];
    if (converged) *converged = fl[BF_CONV];
    return 0;
}

int mctdhb_batch_release(mctdhb_batch b, int slot) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->hs[slot].used) {
        set_error("mctdhb_batch_release: no job in slot %d", slot);
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    HostSlot& h = b->hs[slot];
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(b->st));  // no step in flight reads the region
    const int fl[BF_TOTAL] = {0};
    MCTDHB_CUDA_TRY(cudaMemcpy(b->d_flags + (size_t)slot * BF_TOTAL, fl, sizeof(fl),
                               cudaMemcpyHostToDevice));
    arena_give(b, h.off, h.bytes);
    h = HostSlot();
    b->lists_dirty = true;
    return 0;
}

int mctdhb_batch_monitor(mctdhb_batch b, int slot, double* overlap_res, double* eig_res,
                         int* robust) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->hs[slot].used) {
        set_error("mctdhb_batch_monitor: no job in slot %d", slot);
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    const BatchSlot& d = b->hs[slot].d;
    int fl[BF_TOTAL];
    double2 sc[BS_TOTAL];
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(fl, d.flags, sizeof(fl), cudaMemcpyDeviceToHost, b->st));
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(sc, d.scal, sizeof(sc), cudaMemcpyDeviceToHost, b->st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(b->st));
    if (overlap_res) *overlap_res = sc[BS_MISC + 5].x;
    if (eig_res) *eig_res = sc[BS_MISC + 6].x;
    if (robust) *robust = fl[BF_ROBUST] | (fl[BF_ROBFAIL] << 1);
    return 0;
}

int mctdhb_batch_lowest_state(mctdhb_batch b, int slot, int niter, double* energy) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->hs[slot].used || niter < 0 ||
        niter > 64) {
        set_error("mctdhb_batch_lowest_state: no job in slot %d or niter %d outside 0..64", slot,
                  niter);
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    HostSlot& h = b->hs[slot];
    const BatchSlot& d = h.d;
    int fl[BF_TOTAL];
    MCTDHB_CUDA_TRY(cudaMemcpyAsync(fl, d.flags, sizeof(fl), cudaMemcpyDeviceToHost, b->st));
    MCTDHB_CUDA_TRY(cudaStreamSynchronize(b->st));
    if (fl[BF_STATE] == SLOT_RUNNING) {
        set_error("mctdhb_batch_lowest_state: the job in slot %d is still running", slot);
        return -1;
    }
    // driver.c:41-46: min(nc / 2, 50) iterations, none below 4 configurations
    int it = niter;
    if (it == 0) it = d.nc < 4 ? 0 : (int)std::min<uint32_t>(d.nc / 2, 50u);
    double e = 0.0;
    if (it > 0) {
        SpaceCtx sc;
        sc.N = d.N;
        sc.M = d.M;
        sc.dim = d.nc;
        sc.view = d.sp;
        LanczosWork w;
        double* d_e = nullptr;
        int rc = hcp_prepare(d.M) || lanczos_alloc(w, sc, it);
        if (!rc && cudaMalloc(&d_e, sizeof(double)) != cudaSuccess) {
            set_error("mctdhb_batch_lowest_state: cudaMalloc failed");
            rc = -1;
        }
        if (!rc) rc = lowest_state(sc, w, d.V, it, d_e, b->st);
        if (!rc && (cudaMemcpyAsync(&e, d_e, sizeof(double), cudaMemcpyDeviceToHost, b->st) ||
                    cudaStreamSynchronize(b->st))) {
            set_error("mctdhb_batch_lowest_state: %s", cudaGetErrorString(cudaGetLastError()));
            rc = -1;
        }
        lanczos_free(w);
        if (d_e) cudaFree(d_e);
        if (rc) return -1;
    } else {
        double2 sc[BS_TOTAL];
        MCTDHB_CUDA_TRY(cudaMemcpy(sc, d.scal, sizeof(sc), cudaMemcpyDeviceToHost));
        e = sc[BS_MISC + 3].x;
    }
    if (energy) *energy = e;
    return 0;
}

size_t mctdhb_batch_free_bytes(mctdhb_batch b) {
    if (!b) return 0;
    std::lock_guard<std::mutex> lk(b->mu);
    size_t best = 0;
    for (auto& r : b->free_ranges) best = std::max(best, r.second);
    return best;
}

int mctdhb_batch_kernel_count(mctdhb_batch b) { return b ? b->kernels : 0; }

int mctdhb_batch_launch_hc(mctdhb_batch b, int norb, int parts) {
    if (!b || norb < kBatchMinOrb || norb > kBatchMaxOrb || parts < 1 || parts > 3) {
        set_error("mctdhb_batch_launch_hc: invalid argument");
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    if (b->lists_dirty && rebuild_lists(b)) return -1;
    if (prepare_group(norb)) return -1;
    return hc_group(norb, b->d_slots, b->d_tl[LIST_HY], b->d_tl[LIST_HG], b->d_cnt, 0, b->st,
                    parts, b->pair_v[norb]);
}

int mctdhb_batch_variant(mctdhb_batch b, int norb) {
    if (!b || norb < kBatchMinOrb || norb > kBatchMaxOrb) {
        set_error("mctdhb_batch_variant: invalid argument");
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    return b->pair_v[norb];
}

int mctdhb_batch_set_variant(mctdhb_batch b, int norb, int variant) {
    if (!b || norb < kBatchMinOrb || norb > kBatchMaxOrb ||
        (variant >= 0 && !batch_v_ok(norb, variant))) {
        set_error("mctdhb_batch_set_variant: no variant %d of the batched contraction for %d "
                  "orbitals", variant, norb);
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    b->pair_v_forced[norb] = variant >= 0;
    b->pair_v[norb] = variant >= 0 ? variant : 0;
    drop_graph(b);  // captured with the old variant
    return 0;
}

void* mctdhb_batch_stream(mctdhb_batch b) { return b ? (void*)b->st : nullptr; }

}  // extern "C"
