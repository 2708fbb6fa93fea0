// batch.h -- device layout of the batched engine (batch.cu, batch_tmpl.cuh):
// many independent MCTDHB systems of uneven (N, M, grid) advanced together.
//
// Every system (a "slot") keeps its whole state in one region of the
// engine's HBM arena.  A step of the batch is a fixed sequence of launches,
// captured once into a CUDA graph, whose kernels are persistent: they walk
// work lists (tiles of rows of one slot, or whole slots) that the host
// rewrites in device memory when systems join or leave, so one graph serves
// every mix.  All per-slot reductions use a layout fixed by the slot's own
// sizes (partials per tile, summed in tile order), which makes each
// system's result independent of the other systems in the batch, bit for
// bit.
#pragma once
#include <stdint.h>

#include "common.cuh"
#include "orbital.h"

namespace mctdhb {

constexpr int kBatchVecRows = 4096;  // rows of one vector tile (256 threads x 16)
constexpr int kBatchVecThreads = 256;
constexpr int kBatchHcRows = 256;    // rows of one H.C gather-back tile (one 256-thread block)
constexpr int kBatchMaxSlices = 1024;  // Gram slices per slot and annihilation order
constexpr int kBatchMaxLz = 16;        // Lanczos vectors per step
constexpr int kBatchMinOrb = 2, kBatchMaxOrb = 8;
constexpr int kBatchMaxGrid = 4096;
constexpr int kBatchMonIter = -1;  // H.C launch of the monitor (eigen residual)
constexpr int kBatchOrbThreads = 512;

// per-slot device scalars (double2 units)
constexpr int BS_DIAG = 0;
constexpr int BS_OFFD = kBatchMaxLz;
constexpr int BS_ORTHO = 2 * kBatchMaxLz;
constexpr int BS_Y = 3 * kBatchMaxLz;
// [0] max beta, [1] 1/beta, [2] |C|^2, [3] energy, [4] previous E/N (stop rule),
// [5] overlap residual of the orbitals (real time), [6] eigen residual
// max_i |E C_i - (H C)_i| / N at its last evaluation (imaginary time)
constexpr int BS_MISC = 4 * kBatchMaxLz;
constexpr int BS_Z = BS_MISC + 8;  // kBatchMaxLz^2 doubles of eigenvectors
constexpr int BS_TOTAL = BS_Z + kBatchMaxLz * kBatchMaxLz / 2;

// per-slot device flags (ints)
constexpr int BF_BREAK = 0;  // Lanczos breakdown in this step
constexpr int BF_ITERS = 1;  // Lanczos vectors built in this step
constexpr int BF_QL = 2;     // tridiagonal eigensolver status
constexpr int BF_STATE = 3;  // SLOT_*
constexpr int BF_STEPS = 4;  // steps done
constexpr int BF_CONV = 5;   // 1: stopped by the energy rule
constexpr int BF_INFO = 6;   // rho1 inverse status
constexpr int BF_ROBUST = 7; // robust projector of the orbital equation on
constexpr int BF_MON = 8;    // eigen residual due in this step (monitor H.C)
constexpr int BF_ROBFAIL = 9;  // singular overlap matrix met by the robust projector
constexpr int BF_TOTAL = 10;

// SLOT_ABORTED: real time, overlap residual above the reference's critical
// value (REALTIME_OVERLAP_RESIDUE_TOL, driver.c:89-95, where the reference
// exits; the engine stops that job alone)
constexpr int SLOT_EMPTY = 0, SLOT_RUNNING = 1, SLOT_DONE = 2, SLOT_ABORTED = 3;
constexpr double kOverlapAbort = 1e-3;     // REALTIME_OVERLAP_RESIDUE_TOL (driver.h:7)
constexpr double kOrthoSwitch = 1e-8;      // threshold_impr_ortho (driver.c:19)

struct BatchSlot {
    int N, M, G, imag, rk, check_every, lz, pad0;
    uint32_t nc, max_steps;
    int vtiles;   // ceil(nc / kBatchVecRows)
    int ytiles;   // tiles of the (N-2)-boson space of the pair-space H.C
    int gs[3];    // rho2 Gram slices of the (N-2)-boson space at index 2 (1 unused)
    int gk[3];    // row tiles per Gram slice, index 2
    uint32_t D1;  // D(N-1, M); D(N-2, M) is sp.dim2
    int pad1;
    double dt, etol, reg_fac;
    double eig_tol;    // eigen-residual half of the imaginary-time stop rule (0: off)
    double ortho_tol;  // real time: overlap residual that switches the robust projector on
    double2 pdt;  // SIL time step: dt (real time) or -i dt (imaginary time)
    OrbView ov;   // grid, equation coefficients, Simpson weights, trap
    SpaceView sp; // with the pair matrix sp.pair_w and its scratch sp.pair_y
    const double* g;     // contact interaction (device scalar)
    double2 *orb, *stage, *H, *Q, *hob, *hint, *rho1, *rho2, *rinv, *work;
    double2 *V;          // lz x nc Krylov vectors; V[0] holds the coefficients
    // split step (split: 1): the half-step operator (orbital.h,
    // split_half_operator; dense: column-major G x G, else the circulant
    // kernel of the G - 1 periodic points) and the M x M projection B
    int split, half_dense;
    const double2* half;
    double2* B;
    double2 *out, *part;
    double2* gpart;      // rho2 Gram partials: gs[2] slices
    double2* scal;       // BS_TOTAL
    int* flags;          // BF_TOTAL
};

// a unit of work of a persistent kernel: `idx` is the first row (H.C),
// the tile number (vector kernels) or the slice number (density)
struct BatchTile {
    int slot;
    uint32_t idx;
};

// Tile lists of the per-M kernels.  The count block c (device) holds, after
// c[0] (the vector-tile count), the offset and the count of every list for
// every orbital count: the list `list` of orbital count M is
// tiles_list[batch_off(c, list, M) ...] with batch_cnt(c, list, M) tiles.
constexpr int kBatchNumM = kBatchMaxOrb + 1;
constexpr int LIST_HG = 0;  // H.C gather-back: idx = first row (kBatchHcRows rows)
constexpr int LIST_HY = 1;  // H.C pair contraction: idx = tile of the (N-2)-space
constexpr int LIST_G2 = 2;  // rho2 Gram: idx = slice (rho1 follows from rho2)
constexpr int kBatchLists = 3;
constexpr int kBatchCntInts = 1 + 2 * kBatchLists * kBatchNumM;
// after the count block: one flag per orbital count, set in a step when a
// slot of that count needs the monitor H.C (eigen residual), cleared at the
// start of every step
constexpr int kBatchCntAll = kBatchCntInts + kBatchNumM;
__host__ __device__ inline int* batch_mon(int* c) { return c + kBatchCntInts; }
__host__ __device__ inline const int* batch_mon(const int* c) { return c + kBatchCntInts; }
__host__ __device__ inline int* batch_offs(int* c, int list) { return c + 1 + 2 * list * kBatchNumM; }
__host__ __device__ inline int* batch_cnts(int* c, int list) {
    return c + 1 + (2 * list + 1) * kBatchNumM;
}
__host__ __device__ inline int batch_off(const int* c, int list, int M) {
    return c[1 + 2 * list * kBatchNumM + M];
}
__host__ __device__ inline int batch_cnt(const int* c, int list, int M) {
    return c[1 + (2 * list + 1) * kBatchNumM + M];
}

// rows per tile of the pair contraction (pairhc_tmpl.cuh, PairHcShape)
__host__ __device__ constexpr int batch_pair_rows(int M) {
    return M * (M + 1) / 2 <= 21 ? 256 : 128;
}

// batch_m*.cu: per-M kernels over the tile lists.
//   hcp_batch_launch   out = H V[iter] (- beta V[iter-1]) of every running
//                      slot of orbital count M: pair contraction (parts & 1),
//                      gather-back (parts & 2); iter = kBatchMonIter: out =
//                      H V[0] of the slots whose eigen residual is due;
//                      variant: the contraction's launch variant (0 or 2,
//                      pairhc_tmpl.cuh)
//   gram_batch_launch  rho1 / rho2 of V[0] of the slots of orbital count M
//                      (`list` / `nlist`: the slots, one finalize block each)
//   batch_prepare      launch attributes (call before any stream capture)
template <int M>
int hcp_batch_launch(const BatchSlot* slots, const BatchTile* hy, const BatchTile* hg,
                     const int* cnt, int iter, int parts, int variant, cudaStream_t st);
template <int M>
int gram_batch_launch(const BatchSlot* slots, const BatchTile* g2, const int* cnt,
                      const int* list, const int* nlist, int nblocks, cudaStream_t st);
template <int M>
int batch_prepare();

}  // namespace mctdhb
