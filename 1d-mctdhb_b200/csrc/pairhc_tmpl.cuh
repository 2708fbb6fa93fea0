// pairhc_tmpl.cuh -- H.C through the two-boson-annihilated space, for
// 2 <= M <= 8 orbitals and N >= 2 bosons (explicit instantiations in
// hc_m*.cu).
//
// The Hamiltonian of hamiltonian.c:7-406 is a pair operator.  On the N-boson
// space a+_k a_q = (1/(N-1)) sum_x a+_k a+_x a_x a_q (sum_x a+_x a_x counts
// the N-1 bosons left after a_q), so
//     H = sum_{P,Q} W[P][Q] a+_P a_Q,     P = {k <= s}, Q = {q <= l},
// with a+_P = a+_k a+_s, a_Q = a_q a_l and W built from h and g with the
// same g elements and combinatorial factors as the reference's rules
// (hcp_w_kernel).  With A_m(Q) = <m|a_Q|C> over the D(N-2, M) configurations
// m of N-2 bosons,
//     Y_m(P) = sum_Q W[P][Q] A_m(Q)                 (hcp_y_kernel)
//     (HC)_i = sum_{P in i} <i|a+_P|i-P> Y_{i-P}(P)  (hcp_g_kernel)
// At N=30, M=8 this is 6.7 M x 36 gathers, a 36 x 36 complex matrix-vector
// product per m (FP64 tensor cores, W staged in shared memory; gather and
// contraction overlapped by warp specialisation) and 10.3 M x 36
// coalesced reads of Y, instead of ~576 scattered coefficient gathers per
// row.  Y (D(N-2, M) x P complex, pair-major so that both kernels access it
// with consecutive lanes on consecutive m) is scratch owned by the Fock
// space.  Every value is computed by one thread in a fixed order, so the
// result does not depend on the launch geometry.
#pragma once
#include <algorithm>

#include "common.cuh"
#include "gram_tmpl.cuh"
#include "kernels.h"
#include "movelist.cuh"

namespace mctdhb {

__host__ __device__ constexpr int pair_stride4(int x) { return x + ((12 - x % 8) % 8); }

// shared memory for the producers' rank and square-root tables
constexpr int kPairTabBytes = 8192;

// Launch variants of the pair contraction (the autotuner's choices, tune.cu):
// every variant computes each Y value with the same instructions in the
// same order, so a choice changes speed, never results.
//   0  the default tile (below)
//   1  tiles of half as many rows (up to 6 orbitals): twice the tiles, for
//      spaces with fewer tiles than SMs
//   2  the other output-tile grouping per pass (6 orbitals: one pass over
//      all three output tiles; 7: four at once; 8: two; below 6 orbitals
//      the default already takes all tiles in one pass)
// pair_variant_ok says which exist for M; the batched engine, whose tile
// lists fix the rows per tile, takes 0 and 2.
// (pair_variant_ok and kPairVariants: kernels.h)

template <int M, int V = 0>
struct PairHcShape {
    static constexpr int P = M * (M + 1) / 2;
    static constexpr int CONSUMERS = 256;  // 8 warps: the contraction on the tensor cores
    // Rows of A per tile, one producer thread per row (unrank and gather).
    // Up to 6 orbitals a row carries little contraction, so a tile must
    // keep 256 rows of gathers in flight for the tensor cores; at 7 and 8
    // orbitals 128 rows do.  Measured alternatives at six orbitals (mix
    // contraction 14.3 ms): 128-row tiles 16.9-18.7 ms; two rows per
    // producer thread with half the producers (freeing registers for one
    // output pass and W in registers) 16.8 ms; one output pass at 128
    // registers (spills) 14.7 ms.  The gathers want threads.
    static constexpr bool WIDE = P <= 21;
    static constexpr int ROWS = (WIDE ? 256 : 128) / (V == 1 ? 2 : 1);
    static constexpr int PRODUCERS = ROWS;
    static constexpr int THREADS = CONSUMERS + PRODUCERS;
    // W fragments held in registers by the consumers (up to 5 orbitals; at 6
    // they would spill under the 128-register budget of a 512-thread block)
    static constexpr bool WREG = P <= 15;
    // contraction depth on the tensor cores: P rounded up to 4, in KB8
    // blocks of 8 and KB4 (0 or 1) block of 4 (mma.sync m16n8k8 / m16n8k4);
    // 8-wide output tiles.  When P is one above a multiple of 4 (21 pairs,
    // six orbitals) the last input pair is added by FP64 FMAs on the
    // accumulator fragments after the MMAs (KTAIL) instead of a padded
    // block: 20 columns on the tensor cores instead of 24.
    static constexpr bool KTAIL = P % 4 == 1 && P > 4;
    static constexpr int KP = KTAIL ? P - 1 : (P + 3) / 4 * 4;
    static constexpr int KB8 = KP / 8;
    static constexpr int KB4 = (KP % 8) / 4;
    static constexpr int NN = (P + 7) / 8;
    // output tiles per pass over a strip: two (three at 8 orbitals) keep
    // the accumulators of the three products within the register budget
    static constexpr int NG0 = NN <= 2 ? NN : (NN == 5 ? 3 : 2);
    static constexpr int NG = V != 2 ? NG0 : (NN <= 4 ? NN : 2);
    // variant 3: the tiles handed over through a full and an empty
    // mbarrier per buffer instead of a block barrier per tile, so each warp
    // moves on as soon as its buffer is ready
    static constexpr bool MBAR = V == 3;
    // Shared memory, in 16-byte words.  A row of the A tile takes PS = KP
    // rounded up to 8 words, and element q of row r sits at
    // r * PS + (q ^ swz(r)): the 8 rows stored by 8 consecutive producer
    // lanes fall in 8 different bank groups, and so do the 8 lanes (rows g,
    // g + 1, columns t = 0..3) of each phase of a fragment load.  W rows take
    // WS = 4 (mod 8) words.
    static constexpr int PS = ((KTAIL ? P : KP) + 7) / 8 * 8;
    static constexpr int WS = pair_stride4(P);
    static constexpr size_t SMEM =
        (2 * (size_t)ROWS * PS + (size_t)P * WS) * sizeof(double2) + kPairTabBytes;
    __host__ __device__ static constexpr int swz(int r) { return ((r & 1) << 2) | ((r >> 1) & 3); }
    __host__ __device__ static constexpr int at(int r, int q) { return r * PS + (q ^ swz(r)); }
};

// mbarriers in shared memory (CTA scope): init by one thread before a block
// barrier; arrive (release) by every thread of a role; a wait (acquire)
// that gives up after about two seconds of clock cycles and returns false,
// so a handover that never comes cannot hold the GPU
__device__ __forceinline__ unsigned mbar_addr(const uint64_t* bar) {
    return (unsigned)__cvta_generic_to_shared(bar);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar_addr(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(
                     mbar_addr(bar))
                 : "memory");
}
constexpr long long kMbarWaitCycles = 4000000000LL;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const long long t0 = clock64();
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mbar_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kMbarWaitCycles) return false;
    }
}

// barrier 1 over the block's NT threads (producer and consumer loops meet
// here from their own code paths)
template <int NT>
__device__ __forceinline__ void pair_tile_barrier() {
    asm volatile("bar.sync 1, %0;\n" ::"n"(NT) : "memory");
}

// barrier 2 over the NP producer threads (table staging in the batched
// kernel)
template <int NP>
__device__ __forceinline__ void pair_producer_barrier() {
    asm volatile("bar.sync 2, %0;\n" ::"n"(NP) : "memory");
}

// FP64 mma.sync m16n8k8: D(16x8) += A(16x8) B(8x8).  With g = lane / 4 and
// t = lane % 4, lane l holds A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4];
// B[t][g], B[t+4][g]; D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]
__device__ __forceinline__ void dmma1688(double (&d)[4], double a0, double a1, double a2,
                                         double a3, double b0, double b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// m16n8k4: lane l holds A[g][t], A[g+8][t]; B[t][g]; D as m16n8k8
__device__ __forceinline__ void dmma1684(double (&d)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
        "{%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// The rank table (M - 1 rows of N + 1) and the square-root table (N + 3)
// of a space staged in shared memory for the producers' unranking, when
// they fit kPairTabBytes (else the view keeps the global tables): the
// unrank is a chain of dependent table reads, and the L1 left beside the
// contraction's shared memory does not hold them against the gathers.
__host__ __device__ constexpr bool pair_tab_fits(int N, int M) {
    return (N + 3) * 8 + (M - 1) * (N + 1) * 4 <= kPairTabBytes;
}
// tab: kPairTabBytes of shared memory (8-byte aligned); threads t, t + nt, ...
// copy; the caller synchronises its threads before the view is used
__device__ __forceinline__ SpaceView pair_stage_tab(const SpaceView& sp, void* tab, int t,
                                                    int nt) {
    SpaceView v = sp;
    if (!pair_tab_fits(sp.N, sp.M)) return v;
    double* sq = (double*)tab;
    uint32_t* T = (uint32_t*)(sq + sp.N + 3);
    const int nsq = sp.N + 3, nT = (sp.M - 1) * (sp.N + 1);
    for (int i = t; i < nsq; i += nt) sq[i] = sp.sq[i];
    for (int i = t; i < nT; i += nt) T[i] = sp.T[i];
    v.sq = sq;
    v.T = T;
    return v;
}

// W (P x P, global) staged into Ws[p * WS + q] by threads t, t + nt, ...
template <int M, int V = 0>
__device__ __forceinline__ void pair_stage_w(const double2* __restrict__ W, double2* Ws, int t,
                                             int nt) {
    using S = PairHcShape<M, V>;
    for (int i = t; i < S::P * S::P; i += nt) Ws[(i / S::P) * S::WS + i % S::P] = W[i];
}

// ---------------------------------------------------------------------------
// building blocks (shared with the batched engine, batch_tmpl.cuh)
// ---------------------------------------------------------------------------
// Rows r = r0, r0 + rstep, ... < ROWS of tile `tr` of the (N-2)-boson space
// into As[at(r, p)]: A_m(Q) = sqrt((m_q+1)(m_l+1+[q=l])) C[m + e_q + e_l].
template <int M, int V = 0>
__device__ __forceinline__ void pair_gather(const SpaceView& sp, const double2* __restrict__ C,
                                            uint32_t tr, double2* As, int r0, int rstep) {
    using S = PairHcShape<M, V>;
    constexpr int P = S::P, ROWS = S::ROWS;
    const int N = sp.N;
    const uint32_t D2 = sp.dim2;
    const uint32_t jbase = sp.dim - D2;
    for (int r = r0; r < ROWS; r += rstep) {
        const uint32_t row = tr * ROWS + r;
        const bool live = row < D2;
        int n[M];
        uint32_t U1[M], U2[M];
        if (live) {
            gram_unrank<M, 2, true>(sp.T, N, N - 2, D2, row, n, U1, U2);
        } else {
#pragma unroll
            for (int x = 0; x < M; x++) n[x] = 0, U1[x] = 0u, U2[x] = 0u;
        }
        const uint32_t j0 = jbase + row;
        // sqrt(n_x + 1), sqrt(n_x + 2) once per orbital
        double s1[M], s2[M];
#pragma unroll
        for (int x = 0; x < M; x++) {
            s1[x] = sp.sq[n[x] + 1];
            s2[x] = sp.sq[n[x] + 2];
        }
        static_for<P>([&](auto pi) {
            constexpr int p = decltype(pi)::value;
            constexpr int q = kPairs<M>.q[p], l = kPairs<M>.l[p];
            double2 v = make_double2(0.0, 0.0);
            if (live) {
                const uint32_t j = j0 - (U1[q] - U1[l]) - U2[l];
                const double f = q == l ? s1[q] * s2[q] : s1[q] * s1[l];
                v = cscale(__ldg(C + j), f);
            }
            As[S::at(r, p)] = v;
        });
    }
}

// Y_m(P) = sum_Q W[P][Q] A_m(Q) for a whole tile by the consumer warps on
// the FP64 tensor cores, with three real products per complex product (Gauss):
// T1 = Ar Wr^T, T2 = Ai Wi^T, T3 = (Ar + Ai)(Wr + Wi)^T, then Yr = T1 - T2,
// Yi = T3 - T1 - T2.  When W is real (REAL: real orbitals and coefficients)
// two products do: Yr = Ar Wr^T, Yi = Ai Wr^T.  Warp cw takes the 16-row
// strips cw, cw + 8, ... of the tile and, per pass over NG output tiles of
// 8 pairs, runs m16n8k8 products over the depth (an m16n8k4 one for the
// last 4 when P rounds to an odd number of 4s).  A fragments hold the real
// and imaginary part of an element in one 16-byte load.  Columns q >= P
// read as zero; outputs p >= P and rows m >= D2 are not stored.
template <int M, int V, bool REAL>
__device__ __forceinline__ void pair_contract_mma(const double2* As, const double2* Ws, int cw,
                                                  int lane, uint32_t row0, uint32_t D2,
                                                  double2* __restrict__ Y) {
    using S = PairHcShape<M, V>;
    constexpr int P = S::P, WS = S::WS, PS = S::PS, NN = S::NN, NG = S::NG;
    constexpr int KB8 = S::KB8, KB4 = S::KB4, NPASS = (NN + NG - 1) / NG;
    constexpr int STRIPS = S::ROWS / 16, CW = S::CONSUMERS / 32;
    const int g = lane >> 2, t = lane & 3;
    const int sw = S::swz(g);  // rows g and g + 8 of every strip
    auto wat = [&](int p, int q) {
        return (p < P && q < P) ? Ws[p * WS + q] : make_double2(0.0, 0.0);
    };
    // up to 5 orbitals the W fragments stay in registers: [k step][tile][2]
    constexpr int KS = KB8 + KB4;
    double2 wf[S::WREG ? KS : 1][S::WREG ? NN : 1][2];
    if constexpr (S::WREG) {
#pragma unroll
        for (int k = 0; k < KS; k++)
#pragma unroll
            for (int n = 0; n < NN; n++) {
                const int p = n * 8 + g, q = k * 8 + t;
                wf[k][n][0] = wat(p, q);
                wf[k][n][1] = k < KB8 ? wat(p, q + 4) : make_double2(0.0, 0.0);
            }
    }
    for (int st = cw; st < STRIPS; st += CW) {
        const double2* a_g = As + (size_t)(st * 16 + g) * PS;
        const double2* a_h = a_g + 8 * PS;
        const uint32_t m0 = row0 + st * 16 + g, m1 = m0 + 8;
        auto aat = [&](const double2* row, int q) {
            return q < P ? row[q ^ sw] : make_double2(0.0, 0.0);
        };
#pragma unroll
        for (int pass = 0; pass < NPASS; pass++) {
            const int n0 = pass * NG;
            double t1[NG][4], t2[NG][4], t3[REAL ? 1 : NG][4];
#pragma unroll
            for (int n = 0; n < NG; n++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    t1[n][j] = t2[n][j] = 0.0;
                    if constexpr (!REAL) t3[n][j] = 0.0;
                }
#pragma unroll
            for (int k = 0; k < KS; k++) {
                const bool deep = k < KB8;  // an 8-deep step (else the last 4)
                const int q = k * 8 + t;
                const double2 a0 = aat(a_g, q), a1 = aat(a_h, q);
                const double2 a2 = deep ? aat(a_g, q + 4) : make_double2(0.0, 0.0);
                const double2 a3 = deep ? aat(a_h, q + 4) : make_double2(0.0, 0.0);
#pragma unroll
                for (int n = 0; n < NG; n++) {
                    const int nt = n0 + n;
                    if (nt >= NN) continue;
                    double2 b0, b1;
                    if constexpr (S::WREG) {
                        b0 = wf[k][nt][0];
                        b1 = wf[k][nt][1];
                    } else {
                        const int p = nt * 8 + g;
                        b0 = wat(p, q);
                        b1 = deep ? wat(p, q + 4) : make_double2(0.0, 0.0);
                    }
                    if (deep) {
                        dmma1688(t1[n], a0.x, a1.x, a2.x, a3.x, b0.x, b1.x);
                        if constexpr (REAL) {
                            dmma1688(t2[n], a0.y, a1.y, a2.y, a3.y, b0.x, b1.x);
                        } else {
                            dmma1688(t2[n], a0.y, a1.y, a2.y, a3.y, b0.y, b1.y);
                            dmma1688(t3[n], a0.x + a0.y, a1.x + a1.y, a2.x + a2.y, a3.x + a3.y,
                                     b0.x + b0.y, b1.x + b1.y);
                        }
                    } else {
                        dmma1684(t1[n], a0.x, a1.x, b0.x);
                        if constexpr (REAL) {
                            dmma1684(t2[n], a0.y, a1.y, b0.x);
                        } else {
                            dmma1684(t2[n], a0.y, a1.y, b0.y);
                            dmma1684(t3[n], a0.x + a0.y, a1.x + a1.y, b0.x + b0.y);
                        }
                    }
                }
            }
            if constexpr (S::KTAIL) {
                // input pair P - 1: D[g][2t + j] += A[g][P-1] W[2t + j][P-1]
                // (rows g + 8 alike), after the tensor-core columns
                const double2 e0 = aat(a_g, P - 1), e1 = aat(a_h, P - 1);
#pragma unroll
                for (int n = 0; n < NG; n++) {
                    const int nt = n0 + n;
                    if (nt >= NN) continue;
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        const double2 w = wat(nt * 8 + 2 * t + j, P - 1);
                        t1[n][j] = fma(e0.x, w.x, t1[n][j]);
                        t1[n][j + 2] = fma(e1.x, w.x, t1[n][j + 2]);
                        if constexpr (REAL) {
                            t2[n][j] = fma(e0.y, w.x, t2[n][j]);
                            t2[n][j + 2] = fma(e1.y, w.x, t2[n][j + 2]);
                        } else {
                            t2[n][j] = fma(e0.y, w.y, t2[n][j]);
                            t2[n][j + 2] = fma(e1.y, w.y, t2[n][j + 2]);
                            t3[n][j] = fma(e0.x + e0.y, w.x + w.y, t3[n][j]);
                            t3[n][j + 2] = fma(e1.x + e1.y, w.x + w.y, t3[n][j + 2]);
                        }
                    }
                }
            }
#pragma unroll
            for (int n = 0; n < NG; n++) {
                const int nt = n0 + n;
                if (nt >= NN) continue;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int p = nt * 8 + 2 * t + j;
                    if (p >= P) continue;
                    double2 y0, y1;
                    if constexpr (REAL) {
                        y0 = make_double2(t1[n][j], t2[n][j]);
                        y1 = make_double2(t1[n][j + 2], t2[n][j + 2]);
                    } else {
                        y0 = make_double2(t1[n][j] - t2[n][j], t3[n][j] - t1[n][j] - t2[n][j]);
                        y1 = make_double2(t1[n][j + 2] - t2[n][j + 2],
                                          t3[n][j + 2] - t1[n][j + 2] - t2[n][j + 2]);
                    }
                    if (m0 < D2) Y[(size_t)p * D2 + m0] = y0;
                    if (m1 < D2) Y[(size_t)p * D2 + m1] = y1;
                }
            }
        }
    }
}

// consumer thread t (0 .. CONSUMERS-1) of a tile whose first row is row0;
// `real`: the flag stored after the P x P entries of W
template <int M, int V = 0>
__device__ __forceinline__ void pair_consume(const double2* As, const double2* Ws, int t,
                                             uint32_t row0, uint32_t D2, double2* __restrict__ Y,
                                             bool real) {
    if (real)
        pair_contract_mma<M, V, true>(As, Ws, t >> 5, t & 31, row0, D2, Y);
    else
        pair_contract_mma<M, V, false>(As, Ws, t >> 5, t & 31, row0, D2, Y);
}

// (HC)_row = sum over pairs P = {k <= s} present in the row of
// sqrt(n_k (n_s - [k=s])) Y_{row - e_k - e_s}(P)
template <int M>
__device__ __forceinline__ double2 pair_gather_back(const SpaceView& sp,
                                                    const double2* __restrict__ Y,
                                                    uint32_t row) {
    constexpr int P = M * (M + 1) / 2;
    const int N = sp.N;
    const uint32_t D2 = sp.dim2;
    // occupations and the suffix sums of the rank offsets of removing one /
    // two bosons: V_d[x] = sum_{y >= x} T_y(L_y) - T_y(L_y - d)
    int n[M];
    uint32_t V1[M], V2[M];
    {
        uint32_t S = sp.dim - 1u - row;
        int Lnext = N;
        int L[M - 1];
#pragma unroll
        for (int x = M - 2; x >= 0; x--) {
            const uint32_t* Tx = sp.T + x * (N + 1);
            const int lo = cns_level(Tx, x, Lnext, S);
            S -= __ldg(Tx + lo);
            n[x + 1] = Lnext - lo;
            L[x] = lo;
            Lnext = lo;
        }
        n[0] = Lnext;
        V1[M - 1] = 0u;
        V2[M - 1] = 0u;
        // an L_y below d only occurs for y below the orbitals of a pair that
        // cannot be removed; those sums are never used
#pragma unroll
        for (int x = M - 2; x >= 0; x--) {
            const uint32_t* Tx = sp.T + x * (N + 1);
            const uint32_t t0 = __ldg(Tx + L[x]);
            V1[x] = V1[x + 1] + (t0 - __ldg(Tx + (L[x] >= 1 ? L[x] - 1 : 0)));
            V2[x] = V2[x + 1] + (t0 - __ldg(Tx + (L[x] >= 2 ? L[x] - 2 : 0)));
        }
    }
    const uint32_t base = D2 - sp.dim + row;
    double2 acc = make_double2(0.0, 0.0);
    // every pair is loaded (row 0 of its plane where the pair is absent, with
    // weight f = 0), so the loads do not wait on branches
    static_for<P>([&](auto pi) {
        constexpr int p = decltype(pi)::value;
        constexpr int k = kPairs<M>.q[p], s = kPairs<M>.l[p];
        bool valid;
        double f;
        if constexpr (k == s) {
            valid = n[k] >= 2;
            f = __ldg(sp.sq + n[k]) * __ldg(sp.sq + (n[k] >= 1 ? n[k] - 1 : 0));
        } else {
            valid = n[k] >= 1 && n[s] >= 1;
            f = __ldg(sp.sq + n[k]) * __ldg(sp.sq + n[s]);
        }
        const uint32_t m = valid ? base + (V1[k] - V1[s]) + V2[s] : 0u;
        const double2 y = __ldg(Y + (size_t)p * D2 + m);
        acc.x = fma(f, y.x, acc.x);
        acc.y = fma(f, y.y, acc.y);
    });
    return acc;
}

// ---------------------------------------------------------------------------
// single-system kernels
// ---------------------------------------------------------------------------
// Y = A W^T for the rows m of the (N-2)-boson space; Y[p * D2 + m].
// Warp-specialised and double-buffered: while the consumer warps contract
// tile k from one A buffer, the producer warps unrank and gather tile k + 1
// into the other; one block barrier per tile hands the buffers over.
template <int M, int V>
__global__ void __launch_bounds__(PairHcShape<M, V>::THREADS, 1)
    hcp_y_kernel(SpaceView sp, const double2* __restrict__ C, const double2* __restrict__ W,
                 double2* __restrict__ Y, HcEpilogue ep) {
    using S = PairHcShape<M, V>;
    constexpr int P = S::P, PS = S::PS, ROWS = S::ROWS;
    extern __shared__ double2 smem[];
    double2* Ws = smem;               // Ws[p * WS + q]
    double2* Ab = smem + P * S::WS;   // two buffers of ROWS x PS
    if (ep.flag != nullptr && *ep.flag != 0) return;  // Lanczos breakdown: no-op
    const int t = threadIdx.x;
    pair_stage_w<M, V>(W, Ws, t, S::THREADS);
    const SpaceView tv = pair_stage_tab(sp, Ab + 2 * ROWS * PS, t, S::THREADS);
    __shared__ uint64_t bar_full[2], bar_empty[2];  // variant 3's handover
    if constexpr (S::MBAR) {
        if (t == 0) {
            mbar_init(&bar_full[0], S::PRODUCERS);
            mbar_init(&bar_full[1], S::PRODUCERS);
            mbar_init(&bar_empty[0], S::CONSUMERS);
            mbar_init(&bar_empty[1], S::CONSUMERS);
        }
    }
    __syncthreads();
    const uint32_t ntiles = (sp.dim2 + ROWS - 1) / ROWS;
    const bool producer = t >= S::CONSUMERS;
    const int pt = t - S::CONSUMERS;
    if (producer && blockIdx.x < ntiles)
        pair_gather<M, V>(tv, C, blockIdx.x, Ab, pt, S::PRODUCERS);
    __syncthreads();
    const bool real = W[P * P].x != 0.0;
    if constexpr (S::MBAR) {
        // variant 3: the same tiles handed over through mbarriers.  A lost
        // handover (a wait that ran out) leaves NaN in Y, so the H.C and
        // everything after it come out NaN instead of silently wrong.
        int i = 0;
        for (uint32_t tr = blockIdx.x; tr < ntiles; tr += gridDim.x, i++) {
            const int buf = i & 1;
            if (producer) {
                if (i >= 1 && !mbar_wait(&bar_empty[buf ^ 1], ((i - 1) >> 1) & 1)) {
                    Y[0] = make_double2(__longlong_as_double(0x7ff8000000000000LL), 0.0);
                    return;
                }
                const uint32_t nx = tr + gridDim.x;
                if (nx < ntiles)
                    pair_gather<M, V>(tv, C, nx, Ab + (size_t)(buf ^ 1) * ROWS * PS, pt,
                                      S::PRODUCERS);
                mbar_arrive(&bar_full[buf ^ 1]);
            } else {
                if (i >= 1 && !mbar_wait(&bar_full[buf], ((i - 1) >> 1) & 1)) {
                    Y[0] = make_double2(__longlong_as_double(0x7ff8000000000000LL), 0.0);
                    return;
                }
                pair_consume<M, V>(Ab + (size_t)buf * ROWS * PS, Ws, t, tr * ROWS, sp.dim2, Y,
                                   real);
                mbar_arrive(&bar_empty[buf]);
            }
        }
        return;
    }
    int buf = 0;
    for (uint32_t tr = blockIdx.x; tr < ntiles; tr += gridDim.x, buf ^= 1) {
        if (producer) {
            const uint32_t nx = tr + gridDim.x;
            if (nx < ntiles)
                pair_gather<M, V>(tv, C, nx, Ab + (size_t)(buf ^ 1) * ROWS * PS, pt,
                                  S::PRODUCERS);
        } else {
            pair_consume<M, V>(Ab + (size_t)buf * ROWS * PS, Ws, t, tr * ROWS, sp.dim2, Y, real);
        }
        __syncthreads();
    }
}

// (HC)_i gathered back from Y, then the Lanczos epilogue
template <int M>
__global__ void __launch_bounds__(256)
    hcp_g_kernel(SpaceView sp, const double2* __restrict__ Y, double2* __restrict__ HC,
                 HcEpilogue ep) {
    if (ep.flag != nullptr && *ep.flag != 0) return;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < sp.dim;
         row += gridDim.x * blockDim.x) {
        double2 acc = pair_gather_back<M>(sp, Y, row);
        if (ep.prev != nullptr) {
            const double2 pv = __ldg(ep.prev + row);
            const double b = *ep.beta;
            acc.x -= b * pv.x;
            acc.y -= b * pv.y;
        }
        HC[row] = acc;
    }
}

template <int M, int V>
int hcp_set_attr() {
    static_assert(PairHcShape<M, V>::SMEM <= 227 * 1024, "shared memory of one block (227 KB)");
    if constexpr (pair_variant_ok(M, V))
        MCTDHB_CUDA_TRY(cudaFuncSetAttribute(hcp_y_kernel<M, V>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)PairHcShape<M, V>::SMEM));
    return 0;
}

template <int M>
int hcp_prepare_tmpl() {
    static std::atomic<uint64_t> done{0};
    return set_attributes_once(done, []() -> int {
        return hcp_set_attr<M, 0>() || hcp_set_attr<M, 1>() || hcp_set_attr<M, 2>() ||
               hcp_set_attr<M, 3>();
    });
}

// parts & 1: the contraction; parts & 2: the gather-back (with the epilogue)
template <int M, int V>
int hcp_launch_v(const SpaceView& sp, const double2* C, double2* HC, const HcEpilogue& ep,
                 int parts, cudaStream_t st) {
    if constexpr (!pair_variant_ok(M, V)) {
        set_error("pair contraction variant %d does not exist for %d orbitals", V, M);
        return -1;
    } else {
        using S = PairHcShape<M, V>;
        if (parts & 1) {
            const uint32_t ntiles = (sp.dim2 + S::ROWS - 1) / S::ROWS;
            const int gy = (int)std::min<uint32_t>(ntiles, (uint32_t)num_sms());
            if (gy > 0) {
                hcp_y_kernel<M, V><<<gy, S::THREADS, S::SMEM, st>>>(sp, C, sp.pair_w, sp.pair_y,
                                                                    ep);
                MCTDHB_CUDA_TRY(cudaGetLastError());
            }
        }
        if (parts & 2) {
            const uint32_t need = (sp.dim + 255) / 256;
            const int gg =
                (int)std::max<uint32_t>(1u, std::min<uint32_t>(need, (uint32_t)num_sms() * 8));
            hcp_g_kernel<M><<<gg, 256, 0, st>>>(sp, sp.pair_y, HC, ep);
            MCTDHB_CUDA_TRY(cudaGetLastError());
        }
        return 0;
    }
}

template <int M>
int hcp_apply_tmpl(const SpaceView& sp, const double2* C, double2* HC, const HcEpilogue& ep,
                   int variant, int parts, cudaStream_t st) {
    switch (variant) {
        case 1: return hcp_launch_v<M, 1>(sp, C, HC, ep, parts, st);
        case 2: return hcp_launch_v<M, 2>(sp, C, HC, ep, parts, st);
        case 3: return hcp_launch_v<M, 3>(sp, C, HC, ep, parts, st);
        default: return hcp_launch_v<M, 0>(sp, C, HC, ep, parts, st);
    }
}

}  // namespace mctdhb
