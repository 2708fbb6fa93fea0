// common.cuh -- shared device infrastructure of libmctdhb_b200.
//
// Configuration ranking.  The reference ranks an occupation vector n of N
// bosons in M orbitals with (space.c:159-178)
//     hash(n) = sum_{m=M-1..1} sum_{t<n_m} dim(N_basket - t, m)
// which telescopes into a combinatorial-number-system rank over the
// cumulative occupations L_m = n_0 + ... + n_m:
//     hash(n) = D - 1 - sum_{m=0}^{M-2} T_m(L_m),   T_m(L) = C(L+m, m+1),
// D = C(N+M-1, M-1).  Every jump map entry of the reference (space.c:202,
// 297, 399) is therefore a sum over the few m whose L_m a particle move
// shifts: moving bosons changes L_m by dL_m in {-2..2} and
//     j = i - sum_m [T_m(L_m + dL_m) - T_m(L_m)].
// Each thread precomputes F[m][d] = T_m(L_m + d) - T_m(L_m) for its row, so a
// jump costs a handful of register adds and the 2.6-48 GB map tables of the
// reference never have to be read (or even built) on the hot path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <string>

namespace mctdhb {

constexpr int kMaxOrb = 30;      // MAX_ORBITALS of the reference
constexpr int kMaxTemplOrb = 8;  // orbital counts with a register-resident kernel

// thread-local error record of the C ABI (the reference calls exit(); this
// library reports instead)
void set_error(const char* fmt, ...);
const char* last_error();
void clear_error();

#define MCTDHB_CUDA_TRY(call)                                                  \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess) {                                               \
            ::mctdhb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,     \
                                cudaGetErrorString(_e));                       \
            return -1;                                                         \
        }                                                                      \
    } while (0)

// Device view of one Fock space.  T is the (M-1) x (N+1) rank-weight table,
// sq the sqrt table sqrt(x), x = 0..N+2.  The pair-space H.C
// (pairhc_tmpl.cuh) uses dim2 = D(N-2, M), the pair matrix pair_w (P x P)
// and its scratch pair_y (P x dim2); pair_y is null where that path is off.
struct SpaceView {
    int N, M;
    uint32_t dim;
    const uint32_t* T;
    const double* sq;
    uint32_t dim2 = 0;
    double2* pair_w = nullptr;
    double2* pair_y = nullptr;
};

__host__ __device__ constexpr int dl_index(int d) { return d < 0 ? d + 2 : d + 1; }

// Register-resident state of one configuration (row) of the Fock space.
template <int M>
struct RowState {
    int n[M];                 // occupations
    uint32_t F[M > 1 ? M - 1 : 1][4];  // T_m(L_m+d) - T_m(L_m), d = -2,-1,+1,+2
};

// One level of the greedy CNS decode: the largest L in [0, Lmax] with
// T_x(L) = C(L+x, x+1) <= S.  A closed-form estimate -- exact for x = 0, the
// root of the quadratic for x = 1, the (x+1)-th root of (x+1)! S less x/2
// (T_x(L) ~ (L + x/2)^(x+1) / (x+1)!) for x >= 2 -- then corrected against
// the table; the estimate (the root by the fast hardware power, __powf) is
// within a step or two for every S < 2^32 and x <= 6 (M <= 8, the templated
// kernels; the runtime-M kernels keep a binary search), so a level costs a
// few table loads instead of a binary search.  The corrections make the
// result exact whatever the estimate.
// Table reads: read-only global loads (__ldg), or plain (generic) loads
// when GEN is set -- the table may then sit in shared memory.
template <bool GEN, typename T>
__device__ __forceinline__ T tab_ld(const T* p) {
    if constexpr (GEN)
        return *p;
    else
        return __ldg(p);
}

template <bool GEN = false>
__device__ __forceinline__ int cns_level(const uint32_t* __restrict__ Tx, int x, int Lmax,
                                         uint32_t S) {
    if (x == 0) return S < (uint32_t)Lmax ? (int)S : Lmax;
    float est;
    if (x == 1) {
        est = (sqrtf(8.0f * (float)S + 1.0f) - 1.0f) * 0.5f;
    } else {
        float f = 1.0f;  // (x+1)!
        for (int k = 2; k <= x + 1; k++) f *= (float)k;
        est = __powf(f * (float)S, 1.0f / (float)(x + 1)) - 0.5f * (float)x;
    }
    int L = est > 0.0f ? (int)est : 0;
    L = L < Lmax ? L : Lmax;
    while (L < Lmax && tab_ld<GEN>(Tx + L + 1) <= S) L++;
    while (L > 0 && tab_ld<GEN>(Tx + L) > S) L--;
    return L;
}

// Unrank `row` (greedy CNS decode, identical to set_config of space.c:138)
// and fill the jump offsets.
template <int M>
__device__ __forceinline__ void load_row(const SpaceView& sp, uint32_t row,
                                         RowState<M>& st) {
    const int N = sp.N;
    uint32_t S = sp.dim - 1u - row;
    int Lnext = N;
    int L[M > 1 ? M - 1 : 1];
#pragma unroll
    for (int m = M - 2; m >= 0; m--) {
        const uint32_t* Tm = sp.T + m * (N + 1);
        const int lo = cns_level(Tm, m, Lnext, S);
        S -= __ldg(Tm + lo);
        st.n[m + 1] = Lnext - lo;
        L[m] = lo;
        Lnext = lo;
    }
    st.n[0] = Lnext;
#pragma unroll
    for (int m = 0; m < M - 1; m++) {
        const uint32_t* Tm = sp.T + m * (N + 1);
        uint32_t t0 = __ldg(Tm + L[m]);
#pragma unroll
        for (int di = 0; di < 4; di++) {
            int d = di < 2 ? di - 2 : di - 1;
            int x = L[m] + d;
            x = x < 0 ? 0 : (x > N ? N : x);  // only reached by invalid moves
            st.F[m][di] = __ldg(Tm + x) - t0;
        }
    }
}

// Rank of the configuration reached from `row` by removing bosons from
// orbitals k and s and adding them to q and l (k==s, q==l allowed; a single
// move k->l is jump(k, -1, l, -1) with -1 meaning "none").  All orbital
// indices are compile-time constants after unrolling.
template <int M>
__device__ __forceinline__ uint32_t jump(const RowState<M>& st, uint32_t row,
                                         int k, int s, int q, int l) {
    uint32_t d = 0;
#pragma unroll
    for (int m = 0; m < M - 1; m++) {
        int dl = (q >= 0 && m >= q) + (l >= 0 && m >= l) -
                 (k >= 0 && m >= k) - (s >= 0 && m >= s);
        if (dl != 0) d += st.F[m][dl_index(dl)];
    }
    return row - d;
}

// complex helpers on double2
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc += conj(a) * b
__device__ __forceinline__ double2 cfma_conj(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ double2 cscale(double2 a, double r) {
    return make_double2(a.x * r, a.y * r);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}

// Function attributes such as the dynamic shared-memory limit above 48 KB
// belong to one device: a set-once guard keeps one bit per device (the
// device current at the call) and takes a process-wide lock, so the first
// call on every device sets them and host threads calling at once do not
// race on the flag.  `set` returns 0 on success.
std::mutex& attr_mutex();
template <class F>
int set_attributes_once(std::atomic<uint64_t>& done, F&& set) {
    int dev = 0;
    MCTDHB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(attr_mutex());
    if (dev < 0 || dev >= 64) return set();  // no bit for it: set on every call
    const uint64_t bit = 1ull << dev;
    if (done.load(std::memory_order_acquire) & bit) return 0;
    if (set()) return -1;
    done.fetch_or(bit, std::memory_order_release);
    return 0;
}

// SM count of the current device, read once per device (an atomic slot per
// device ordinal, so host threads on different devices neither race nor
// share a count)
inline int num_sms() {
    static std::atomic<int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    const bool slot = dev >= 0 && dev < 64;
    int n = slot ? cache[dev].load(std::memory_order_relaxed) : 0;
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            n <= 0)
            n = 148;
        if (slot) cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

}  // namespace mctdhb
