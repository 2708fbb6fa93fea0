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

constexpr int kBatchVecRows = 1024;  // rows of one vector tile (256 threads x 4)
constexpr int kBatchVecThreads = 256;
constexpr int kBatchHcRows = 256;    // rows of one H.C tile (one 256-thread block)
constexpr int kBatchDensThreads = 128;
constexpr int kBatchMaxSlices = 1024;  // density slices per slot
constexpr int kBatchMaxLz = 16;        // Lanczos vectors per step
constexpr int kBatchMinOrb = 2, kBatchMaxOrb = 8;
constexpr int kBatchMaxGrid = 4096;
constexpr int kBatchOrbThreads = 512;

// per-slot device scalars (double2 units)
constexpr int BS_DIAG = 0;
constexpr int BS_OFFD = kBatchMaxLz;
constexpr int BS_ORTHO = 2 * kBatchMaxLz;
constexpr int BS_Y = 3 * kBatchMaxLz;
// [0] max beta, [1] 1/beta, [2] |C|^2, [3] energy, [4] previous E/N (stop rule)
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
constexpr int BF_TOTAL = 8;

constexpr int SLOT_EMPTY = 0, SLOT_RUNNING = 1, SLOT_DONE = 2;

struct BatchSlot {
    int N, M, G, imag, rk, check_every, lz, pad0;
    uint32_t nc, max_steps;
    int vtiles;   // ceil(nc / kBatchVecRows)
    int dslices;  // density slices; each covers dchunks x 128 rows
    int dchunks;
    int pad1;
    double dt, etol, reg_fac;
    double2 pdt;  // SIL time step: dt (real time) or -i dt (imaginary time)
    OrbView ov;   // grid, equation coefficients, Simpson weights, trap
    SpaceView sp;
    const double* g;     // contact interaction (device scalar)
    const int* desc;     // density element descriptors for M
    double2 *orb, *stage, *H, *Q, *hob, *hint, *tab, *rho1, *rho2, *rinv, *work;
    double2 *V;          // lz x nc Krylov vectors; V[0] holds the coefficients
    double2 *out, *part, *dpart;
    double2* scal;       // BS_TOTAL
    int* flags;          // BF_TOTAL
};

// a unit of work of a persistent kernel: `idx` is the first row (H.C),
// the tile number (vector kernels) or the slice number (density)
struct BatchTile {
    int slot;
    uint32_t idx;
};

// batch_m*.cu: per-M H.C and density kernels over a tile list.  `off` and
// `cnt` are device arrays indexed by M (the list of orbital count M starts
// at tiles + off[M]).  dens_batch_launch with slots == nullptr only sets the
// kernel's launch attributes (call it before any stream capture).
template <int M>
int hc_batch_launch(const BatchSlot* slots, const BatchTile* tiles, const int* off,
                    const int* cnt, int iter, cudaStream_t st);
template <int M>
int dens_batch_launch(const BatchSlot* slots, const BatchTile* tiles, const int* off,
                      const int* cnt, cudaStream_t st);

}  // namespace mctdhb
