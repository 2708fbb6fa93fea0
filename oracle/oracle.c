/* oracle.c -- CPU restatement of the reference's configurational path.
 *
 * TEST INFRASTRUCTURE (see oracle.h): the checker for the GPU library and the
 * timed CPU baseline.  Each function cites the reference file:line it
 * follows (paths relative to the reference project root).
 *
 * Configuration ranking.  The reference ranks an occupation vector n with
 *   hash = sum_{m=M-1..1} sum_{t<n_m} dim(N_basket - t, m)      (space.c:159)
 * which telescopes (hockey-stick identity) into a combinatorial-number-system
 * rank over the cumulative occupations L_m = n_0 + ... + n_m:
 *   hash = D - 1 - sum_{m=0}^{M-2} C(L_m + m, m + 1),   D = C(N+M-1, M-1).
 * T[m][L] = C(L + m, m + 1) is tabulated once; ranking is O(M) and unranking
 * is a greedy CNS decode, identical in result to set_config (space.c:138).
 */
#include "oracle.h"
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* combinatorics                                                       */
/* ------------------------------------------------------------------ */

static uint64_t
binom(uint64_t n, uint64_t k)
{
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (uint64_t i = 1; i <= k; i++)
    {
        r = r * (n - k + i) / i;
        if (r > (unsigned __int128) UINT64_MAX) return UINT64_MAX;
    }
    return (uint64_t) r;
}

uint64_t
orc_space_dimension(int npar, int norb)
{
    return binom((uint64_t) npar + norb - 1, (uint64_t) norb - 1);
}

typedef struct
{
    int       npar, norb;
    uint64_t  dim;
    uint64_t* T; /* T[m*(N+1)+L] = C(L+m, m+1), m = 0..M-2 */
} space_t;

static space_t
space_make(int npar, int norb)
{
    space_t s;
    s.npar = npar;
    s.norb = norb;
    s.dim = orc_space_dimension(npar, norb);
    int rows = norb > 1 ? norb - 1 : 1;
    s.T = malloc(sizeof(uint64_t) * rows * (npar + 1));
    for (int m = 0; m < norb - 1; m++)
        for (int L = 0; L <= npar; L++)
            s.T[m * (npar + 1) + L] = binom((uint64_t) L + m, (uint64_t) m + 1);
    return s;
}

static void
space_free(space_t* s)
{
    free(s->T);
}

static inline uint64_t
rank_occ(const space_t* s, const uint16_t* occ)
{
    uint64_t S = 0;
    int      L = 0;
    for (int m = 0; m < s->norb - 1; m++)
    {
        L += occ[m];
        S += s->T[m * (s->npar + 1) + L];
    }
    return s->dim - 1 - S;
}

static void
unrank_occ(const space_t* s, uint64_t idx, uint16_t* occ)
{
    int      M = s->norb, N = s->npar;
    uint64_t S = s->dim - 1 - idx;
    int      Lnext = N;
    for (int m = M - 2; m >= 0; m--)
    {
        const uint64_t* Tm = s->T + m * (N + 1);
        int             lo = 0, hi = Lnext; /* largest L in [0,Lnext], Tm[L]<=S */
        while (lo < hi)
        {
            int mid = (lo + hi + 1) / 2;
            if (Tm[mid] <= S)
                lo = mid;
            else
                hi = mid - 1;
        }
        S -= Tm[lo];
        occ[m + 1] = (uint16_t) (Lnext - lo);
        Lnext = lo;
    }
    occ[0] = (uint16_t) Lnext;
}

uint64_t
orc_rank(int npar, int norb, const uint16_t* occ)
{
    space_t  s = space_make(npar, norb);
    uint64_t r = rank_occ(&s, occ);
    space_free(&s);
    return r;
}

void
orc_unrank(int npar, int norb, uint64_t idx, uint16_t* occ)
{
    space_t s = space_make(npar, norb);
    unrank_occ(&s, idx, occ);
    space_free(&s);
}

/* space.c:120-135: S[n + (N+1) m] = dim(n particles, m orbitals), m=0 -> 0 */
void
orc_subspaces_dim(int npar, int norb, uint32_t* out)
{
    for (int i = 0; i <= npar; i++)
    {
        out[i] = 0;
        if (norb >= 1) out[i + (npar + 1)] = 1;
        for (int j = 2; j <= norb; j++)
            out[i + (npar + 1) * j] = (uint32_t) orc_space_dimension(i, j);
    }
}

/* space.c:181-199 */
void
orc_hash_table(int npar, int norb, uint16_t* ht)
{
    space_t s = space_make(npar, norb);
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < s.dim; i++) unrank_occ(&s, i, ht + i * norb);
    space_free(&s);
}

/* space.c:202-251 */
void
orc_single_jump_map(int npar, int norb, uint32_t* map)
{
    space_t  s = space_make(npar, norb);
    uint64_t dim = s.dim;
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < dim; i++)
    {
        uint16_t occ[64];
        unrank_occ(&s, i, occ);
        for (int k = 0; k < norb; k++)
        {
            for (int l = 0; l < norb; l++)
            {
                uint64_t idx = i + k * dim + (uint64_t) l * norb * dim;
                if (occ[k] < 1)
                {
                    map[idx] = 0;
                    continue;
                }
                occ[k]--;
                occ[l]++;
                map[idx] = (uint32_t) rank_occ(&s, occ);
                occ[k]++;
                occ[l]--;
            }
        }
    }
    space_free(&s);
}

static uint64_t
count_pairs(const uint16_t* occ, int M)
{
    int nz = 0;
    for (int k = 0; k < M; k++) nz += occ[k] > 0;
    return (uint64_t) nz * (nz - 1) / 2;
}

static uint64_t
count_doubles(const uint16_t* occ, int M)
{
    uint64_t c = 0;
    for (int k = 0; k < M; k++) c += occ[k] > 1;
    return c;
}

static uint64_t
chunk_offsets(int npar, int norb, int diff, uint64_t* strides)
{
    space_t   s = space_make(npar, norb);
    uint64_t  dim = s.dim, M2 = (uint64_t) norb * norb;
    uint64_t* cnt = malloc(sizeof(uint64_t) * dim);
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < dim; i++)
    {
        uint16_t occ[64];
        unrank_occ(&s, i, occ);
        cnt[i] = diff ? count_pairs(occ, norb) : count_doubles(occ, norb);
    }
    uint64_t total = 0;
    for (uint64_t i = 0; i < dim; i++)
    {
        if (strides) strides[i] = total * M2;
        total += cnt[i];
    }
    free(cnt);
    space_free(&s);
    return total;
}

uint64_t
orc_double_diffjump_chunks(int npar, int norb)
{
    return chunk_offsets(npar, norb, 1, NULL);
}

uint64_t
orc_double_equaljump_chunks(int npar, int norb)
{
    return chunk_offsets(npar, norb, 0, NULL);
}

/* space.c:297-358 */
void
orc_double_diffjump_map(int npar, int norb, uint64_t* strides, uint32_t* map)
{
    chunk_offsets(npar, norb, 1, strides);
    space_t s = space_make(npar, norb);
    int     M = norb;
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < s.dim; i++)
    {
        uint16_t occ[64];
        unrank_occ(&s, i, occ);
        uint64_t chunk = 0;
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            for (int q = k + 1; q < M; q++)
            {
                if (occ[q] < 1) continue;
                uint64_t base = strides[i] + chunk * M * M;
                for (int l = 0; l < M; l++)
                    for (int p = 0; p < M; p++)
                    {
                        occ[k]--;
                        occ[q]--;
                        occ[l]++;
                        occ[p]++;
                        map[base + l + p * M] = (uint32_t) rank_occ(&s, occ);
                        occ[k]++;
                        occ[q]++;
                        occ[l]--;
                        occ[p]--;
                    }
                chunk++;
            }
        }
    }
    space_free(&s);
}

/* space.c:399-451 */
void
orc_double_equaljump_map(int npar, int norb, uint64_t* strides, uint32_t* map)
{
    chunk_offsets(npar, norb, 0, strides);
    space_t s = space_make(npar, norb);
    int     M = norb;
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < s.dim; i++)
    {
        uint16_t occ[64];
        unrank_occ(&s, i, occ);
        uint64_t chunk = 0;
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 2) continue;
            uint64_t base = strides[i] + chunk * M * M;
            for (int l = 0; l < M; l++)
                for (int p = 0; p < M; p++)
                {
                    occ[k] -= 2;
                    occ[l]++;
                    occ[p]++;
                    map[base + l + p * M] = (uint32_t) rank_occ(&s, occ);
                    occ[k] += 2;
                    occ[l]--;
                    occ[p]--;
                }
            chunk++;
        }
    }
    space_free(&s);
}

/* ------------------------------------------------------------------ */
/* H.C  (hamiltonian.c:7-406), rule for rule, maps -> on-the-fly rank  */
/* ------------------------------------------------------------------ */

static inline uint64_t
jump1(const space_t* s, uint16_t* o, int k, int l)
{
    o[k]--;
    o[l]++;
    uint64_t j = rank_occ(s, o);
    o[k]++;
    o[l]--;
    return j;
}

static inline uint64_t
jump2(const space_t* s, uint16_t* o, int k, int t, int q, int l)
{
    o[k]--;
    o[t]--;
    o[q]++;
    o[l]++;
    uint64_t j = rank_occ(s, o);
    o[k]++;
    o[t]++;
    o[q]--;
    o[l]--;
    return j;
}

static void
hc_rows(const space_t* sp, const ocplx* coef, const ocplx* hob,
        const ocplx* hint, ocplx* hc, uint64_t r0, uint64_t r1)
{
    const int M = sp->norb, M2 = M * M, M3 = M * M * M;
#pragma omp parallel for schedule(static)
    for (uint64_t i = r0; i < r1; i++)
    {
        uint16_t occ[64];
        ocplx    w = 0, z = 0;
        double   bf;
        uint64_t j;
        unrank_occ(sp, i, occ);

        /* one-body (hamiltonian.c:44-55) */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            w = w + hob[k * M + k] * occ[k] * coef[i];
            for (int l = 0; l < M; l++)
            {
                if (l == k) continue;
                bf = sqrt((double) occ[k] * (occ[l] + 1));
                j = jump1(sp, occ, k, l);
                w = w + hob[k * M + l] * bf * coef[j];
            }
        }
        /* rule 1 (:57-63) */
        for (int k = 0; k < M; k++)
        {
            bf = occ[k] * (occ[k] - 1);
            z += hint[k + M * k + M2 * k + M3 * k] * coef[i] * bf;
        }
        /* rule 2 (:65-79) */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            for (int s = k + 1; s < M; s++)
            {
                bf = occ[k] * occ[s];
                z += 4 * hint[k + s * M + k * M2 + s * M3] * bf * coef[i];
            }
        }
        /* rule 3 (:81-104) */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 2) continue;
            for (int q = 0; q < M; q++)
            {
                if (q == k) continue;
                bf = sqrt((double) (occ[k] - 1) * occ[k] * (occ[q] + 1) *
                          (occ[q] + 2));
                j = jump2(sp, occ, k, k, q, q);
                z += hint[k + k * M + q * M2 + q * M3] * coef[j] * bf;
            }
        }
        /* rule 4 (:106-121) */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 2) continue;
            for (int l = 0; l < M; l++)
            {
                if (l == k) continue;
                bf = (occ[k] - 1) * sqrt((double) occ[k] * (occ[l] + 1));
                j = jump1(sp, occ, k, l);
                z += 2 * hint[k + k * M + k * M2 + l * M3] * coef[j] * bf;
            }
        }
        /* rule 5 (:123-138) */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            for (int s = 0; s < M; s++)
            {
                if (s == k || occ[s] < 1) continue;
                bf = occ[s] * sqrt((double) occ[k] * (occ[s] + 1));
                j = jump1(sp, occ, k, s);
                z += 2 * hint[k + s * M + s * M2 + s * M3] * coef[j] * bf;
            }
        }
        /* rules 6.0, 6.1, 6.2 (:140-223): k k -> q l, q < l, k not in {q,l},
         * visited in the reference's three loop orders */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 2) continue;
            for (int q = k + 1; q < M; q++)
                for (int l = q + 1; l < M; l++)
                {
                    bf = sqrt((double) occ[k] * (occ[k] - 1) * (occ[q] + 1) *
                              (occ[l] + 1));
                    j = jump2(sp, occ, k, k, q, l);
                    z += 2 * hint[k + k * M + q * M2 + l * M3] * coef[j] * bf;
                }
        }
        for (int q = 0; q < M; q++)
            for (int k = q + 1; k < M; k++)
            {
                if (occ[k] < 2) continue;
                for (int l = k + 1; l < M; l++)
                {
                    bf = sqrt((double) occ[k] * (occ[k] - 1) * (occ[q] + 1) *
                              (occ[l] + 1));
                    j = jump2(sp, occ, k, k, q, l);
                    z += 2 * hint[k + k * M + q * M2 + l * M3] * coef[j] * bf;
                }
            }
        for (int q = 0; q < M; q++)
            for (int l = q + 1; l < M; l++)
                for (int k = l + 1; k < M; k++)
                {
                    if (occ[k] < 2) continue;
                    bf = sqrt((double) occ[k] * (occ[k] - 1) * (occ[q] + 1) *
                              (occ[l] + 1));
                    j = jump2(sp, occ, k, k, q, l);
                    z += 2 * hint[k + k * M + q * M2 + l * M3] * coef[j] * bf;
                }
        /* rules 7.0, 7.1, 7.2 (:225-334): k s -> q q, k < s, q not in {k,s} */
        for (int q = 0; q < M; q++)
            for (int k = q + 1; k < M; k++)
            {
                if (occ[k] < 1) continue;
                for (int s = k + 1; s < M; s++)
                {
                    if (occ[s] < 1) continue;
                    bf = sqrt((double) occ[k] * occ[s] * (occ[q] + 1) *
                              (occ[q] + 2));
                    j = jump2(sp, occ, k, s, q, q);
                    z += 2 * hint[k + s * M + q * M2 + q * M3] * coef[j] * bf;
                }
            }
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            for (int q = k + 1; q < M; q++)
                for (int s = q + 1; s < M; s++)
                {
                    if (occ[s] < 1) continue;
                    bf = sqrt((double) occ[k] * occ[s] * (occ[q] + 1) *
                              (occ[q] + 2));
                    j = jump2(sp, occ, k, s, q, q);
                    z += 2 * hint[k + s * M + q * M2 + q * M3] * coef[j] * bf;
                }
        }
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            for (int s = k + 1; s < M; s++)
            {
                if (occ[s] < 1) continue;
                for (int q = s + 1; q < M; q++)
                {
                    bf = sqrt((double) occ[k] * occ[s] * (occ[q] + 1) *
                              (occ[q] + 2));
                    j = jump2(sp, occ, k, s, q, q);
                    z += 2 * hint[k + s * M + q * M2 + q * M3] * coef[j] * bf;
                }
            }
        }
        /* rule 8 (:336-360): k s -> s l, l not in {k,s} */
        for (int s = 0; s < M; s++)
        {
            if (occ[s] < 1) continue;
            for (int k = 0; k < M; k++)
            {
                if (occ[k] < 1 || k == s) continue;
                for (int l = 0; l < M; l++)
                {
                    if (l == k || l == s) continue;
                    bf = occ[s] * sqrt((double) occ[k] * (occ[l] + 1));
                    j = jump1(sp, occ, k, l);
                    z += 4 * hint[k + s * M + s * M2 + l * M3] * coef[j] * bf;
                }
            }
        }
        /* rule 9 (:362-398): k s -> q l, k < s, q < l, all distinct */
        for (int k = 0; k < M; k++)
        {
            if (occ[k] < 1) continue;
            for (int s = k + 1; s < M; s++)
            {
                if (occ[s] < 1) continue;
                for (int q = 0; q < M; q++)
                {
                    if (q == s || q == k) continue;
                    for (int l = q + 1; l < M; l++)
                    {
                        if (l == k || l == s) continue;
                        bf = sqrt((double) occ[k] * occ[s] * (occ[q] + 1) *
                                  (occ[l] + 1));
                        j = jump2(sp, occ, k, s, q, l);
                        z += 4 * hint[k + s * M + q * M2 + l * M3] * coef[j] *
                             bf;
                    }
                }
            }
        }
        hc[i] = w + 0.5 * z;
    }
}

void
orc_apply_hamiltonian(int npar, int norb, const ocplx* coef, const ocplx* hob,
                      const ocplx* hint, ocplx* hc)
{
    space_t s = space_make(npar, norb);
    hc_rows(&s, coef, hob, hint, hc, 0, s.dim);
    space_free(&s);
}

void
orc_apply_hamiltonian_rows(int npar, int norb, const ocplx* coef,
                           const ocplx* hob, const ocplx* hint, ocplx* hc,
                           uint64_t row0, uint64_t row1)
{
    space_t s = space_make(npar, norb);
    if (row1 > s.dim) row1 = s.dim;
    hc_rows(&s, coef, hob, hint, hc, row0, row1);
    space_free(&s);
}

/* ------------------------------------------------------------------ */
/* density matrices (density_matrices.c)                               */
/* ------------------------------------------------------------------ */

/* density_matrices.c:9-52 */
void
orc_onebody_dm(int npar, int norb, const ocplx* coef, ocplx* rho)
{
    space_t s = space_make(npar, norb);
    int     M = norb;
    int     nt = omp_get_max_threads();
    ocplx*  part = calloc((size_t) nt * M * M, sizeof(ocplx));
#pragma omp parallel
    {
        ocplx*   acc = part + (size_t) omp_get_thread_num() * M * M;
        uint16_t occ[64];
#pragma omp for schedule(static)
        for (uint64_t i = 0; i < s.dim; i++)
        {
            unrank_occ(&s, i, occ);
            double m2 = creal(coef[i]) * creal(coef[i]) +
                        cimag(coef[i]) * cimag(coef[i]);
            for (int k = 0; k < M; k++)
            {
                acc[k * M + k] += m2 * occ[k];
                if (occ[k] < 1) continue;
                for (int l = k + 1; l < M; l++)
                {
                    uint64_t j = jump1(&s, occ, k, l);
                    acc[k * M + l] += conj(coef[i]) * coef[j] *
                                      sqrt((double) (occ[l] + 1) * occ[k]);
                }
            }
        }
    }
    for (int k = 0; k < M; k++)
    {
        for (int l = k; l < M; l++)
        {
            ocplx v = 0;
            for (int t = 0; t < nt; t++) v += part[(size_t) t * M * M + k * M + l];
            rho[k * M + l] = v;
            if (l > k) rho[l * M + k] = conj(v);
        }
    }
    free(part);
    space_free(&s);
}

#define IX(a, b, c, d) ((a) + M * (b) + M2 * (c) + M3 * (d))

static void
tb_rows(const space_t* sp, const ocplx* coef, ocplx* rho, uint64_t r0,
        uint64_t r1)
{
    const int M = sp->norb, M2 = M * M, M3 = M2 * M, M4 = M3 * M;
    int       nt = omp_get_max_threads();
    ocplx*    part = calloc((size_t) nt * M4, sizeof(ocplx));
#pragma omp parallel
    {
        ocplx*   acc = part + (size_t) omp_get_thread_num() * M4;
        uint16_t o[64];
#pragma omp for schedule(static)
        for (uint64_t i = r0; i < r1; i++)
        {
            unrank_occ(sp, i, o);
            ocplx  ci = coef[i], cc = conj(ci);
            double m2 = creal(ci) * creal(ci) + cimag(ci) * cimag(ci);
            uint64_t j;
            /* rule 1 (:76-90) */
            for (int k = 0; k < M; k++)
                if (o[k] >= 2) acc[IX(k, k, k, k)] += m2 * (o[k] * (o[k] - 1));
            /* rule 2 (:92-112) */
            for (int k = 0; k < M; k++)
                for (int s = k + 1; s < M; s++)
                    acc[IX(k, s, k, s)] += m2 * (o[k] * o[s]);
            /* rule 3 (:114-143): k < q */
            for (int k = 0; k < M; k++)
            {
                if (o[k] < 2) continue;
                for (int q = k + 1; q < M; q++)
                {
                    j = jump2(sp, o, k, k, q, q);
                    acc[IX(k, k, q, q)] +=
                        cc * coef[j] *
                        sqrt((double) (o[k] - 1) * o[k] * (o[q] + 1) *
                             (o[q] + 2));
                }
            }
            /* rule 4 (:145-166): k < l */
            for (int k = 0; k < M; k++)
            {
                if (o[k] < 2) continue;
                for (int l = k + 1; l < M; l++)
                {
                    j = jump1(sp, o, k, l);
                    acc[IX(k, k, k, l)] += cc * coef[j] * ((o[k] - 1) *
                                           sqrt((double) o[k] * (o[l] + 1)));
                }
            }
            /* rule 5 (:168-189): k < s */
            for (int k = 0; k < M; k++)
            {
                if (o[k] < 1) continue;
                for (int s = k + 1; s < M; s++)
                {
                    if (o[s] < 1) continue;
                    j = jump1(sp, o, k, s);
                    acc[IX(k, s, s, s)] +=
                        cc * coef[j] * (o[s] * sqrt((double) o[k] * (o[s] + 1)));
                }
            }
            /* rules 6.0-6.2 (:191-298): k k -> q l, q < l, k not in {q,l} */
            for (int k = 0; k < M; k++)
            {
                if (o[k] < 2) continue;
                for (int q = 0; q < M; q++)
                {
                    if (q == k) continue;
                    for (int l = q + 1; l < M; l++)
                    {
                        if (l == k) continue;
                        j = jump2(sp, o, k, k, q, l);
                        acc[IX(k, k, q, l)] +=
                            cc * coef[j] *
                            sqrt((double) o[k] * (o[k] - 1) * (o[q] + 1) *
                                 (o[l] + 1));
                    }
                }
            }
            /* rules 7.0-7.2 (:300-403): k -> l with spectator s, k < l */
            for (int k = 0; k < M; k++)
            {
                if (o[k] < 1) continue;
                for (int l = k + 1; l < M; l++)
                {
                    j = jump1(sp, o, k, l);
                    ocplx t = cc * coef[j];
                    for (int s = 0; s < M; s++)
                    {
                        if (s == k || s == l || o[s] < 1) continue;
                        acc[IX(k, s, s, l)] +=
                            t * (o[s] * sqrt((double) o[k] * (o[l] + 1)));
                    }
                }
            }
            /* rule 8 (:405-442): k s -> q l, k < s, q < l, disjoint */
            for (int k = 0; k < M; k++)
            {
                if (o[k] < 1) continue;
                for (int s = k + 1; s < M; s++)
                {
                    if (o[s] < 1) continue;
                    for (int q = 0; q < M; q++)
                    {
                        if (q == s || q == k) continue;
                        for (int l = q + 1; l < M; l++)
                        {
                            if (l == k || l == s) continue;
                            j = jump2(sp, o, k, s, q, l);
                            acc[IX(k, s, q, l)] +=
                                cc * coef[j] *
                                sqrt((double) o[k] * o[s] * (o[q] + 1) *
                                     (o[l] + 1));
                        }
                    }
                }
            }
        }
    }
    ocplx* a = calloc(M4, sizeof(ocplx));
    for (int t = 0; t < nt; t++)
        for (int e = 0; e < M4; e++) a[e] += part[(size_t) t * M4 + e];
    free(part);

    /* symmetric fill in the reference's rule order */
    for (int k = 0; k < M; k++) rho[IX(k, k, k, k)] = a[IX(k, k, k, k)];
    for (int k = 0; k < M; k++)
        for (int s = k + 1; s < M; s++)
        {
            ocplx v = a[IX(k, s, k, s)];
            rho[IX(k, s, k, s)] = v;
            rho[IX(s, k, k, s)] = v;
            rho[IX(s, k, s, k)] = v;
            rho[IX(k, s, s, k)] = v;
        }
    for (int k = 0; k < M; k++)
        for (int q = k + 1; q < M; q++)
        {
            ocplx v = a[IX(k, k, q, q)];
            rho[IX(k, k, q, q)] = v;
            rho[IX(q, q, k, k)] = conj(v);
        }
    for (int k = 0; k < M; k++)
        for (int l = k + 1; l < M; l++)
        {
            ocplx v = a[IX(k, k, k, l)];
            rho[IX(k, k, k, l)] = v;
            rho[IX(k, k, l, k)] = v;
            rho[IX(l, k, k, k)] = conj(v);
            rho[IX(k, l, k, k)] = conj(v);
        }
    for (int k = 0; k < M; k++)
        for (int s = k + 1; s < M; s++)
        {
            ocplx v = a[IX(k, s, s, s)];
            rho[IX(k, s, s, s)] = v;
            rho[IX(s, k, s, s)] = v;
            rho[IX(s, s, s, k)] = conj(v);
            rho[IX(s, s, k, s)] = conj(v);
        }
    for (int k = 0; k < M; k++)
        for (int q = 0; q < M; q++)
        {
            if (q == k) continue;
            for (int l = q + 1; l < M; l++)
            {
                if (l == k) continue;
                ocplx v = a[IX(k, k, q, l)];
                rho[IX(k, k, q, l)] = v;
                rho[IX(k, k, l, q)] = v;
                rho[IX(l, q, k, k)] = conj(v);
                rho[IX(q, l, k, k)] = conj(v);
            }
        }
    for (int k = 0; k < M; k++)
        for (int l = k + 1; l < M; l++)
            for (int s = 0; s < M; s++)
            {
                if (s == k || s == l) continue;
                ocplx v = a[IX(k, s, s, l)];
                rho[IX(k, s, s, l)] = v;
                rho[IX(s, k, s, l)] = v;
                rho[IX(s, k, l, s)] = v;
                rho[IX(k, s, l, s)] = v;
                rho[IX(l, s, s, k)] = conj(v);
                rho[IX(s, l, s, k)] = conj(v);
                rho[IX(s, l, k, s)] = conj(v);
                rho[IX(l, s, k, s)] = conj(v);
            }
    for (int k = 0; k < M; k++)
        for (int s = k + 1; s < M; s++)
            for (int q = 0; q < M; q++)
            {
                if (q == s || q == k) continue;
                for (int l = q + 1; l < M; l++)
                {
                    if (l == k || l == s) continue;
                    ocplx v = a[IX(k, s, q, l)];
                    rho[IX(k, s, q, l)] = v;
                    rho[IX(s, k, q, l)] = v;
                    rho[IX(k, s, l, q)] = v;
                    rho[IX(s, k, l, q)] = v;
                }
            }
    free(a);
}

void
orc_twobody_dm(int npar, int norb, const ocplx* coef, ocplx* rho)
{
    space_t s = space_make(npar, norb);
    tb_rows(&s, coef, rho, 0, s.dim);
    space_free(&s);
}

void
orc_twobody_dm_rows(int npar, int norb, const ocplx* coef, ocplx* rho,
                    uint64_t row0, uint64_t row1)
{
    space_t s = space_make(npar, norb);
    if (row1 > s.dim) row1 = s.dim;
    tb_rows(&s, coef, rho, row0, row1);
    space_free(&s);
}

/* ------------------------------------------------------------------ */
/* dense helpers                                                       */
/* ------------------------------------------------------------------ */

/* Implicit QL with Wilkinson shifts on a symmetric tridiagonal matrix
 * (the EISPACK tql2 scheme).  Eigenvectors accumulate into the columns of
 * the row-major z. */
int
orc_tridiag_eig(int n, double* d, double* e, double* z)
{
    for (int i = 0; i < n * n; i++) z[i] = 0;
    for (int i = 0; i < n; i++) z[i * n + i] = 1;
    if (n < 1) return 0;
    e[n - 1] = 0;
    for (int l = 0; l < n; l++)
    {
        int iter = 0, m;
        for (;;)
        {
            for (m = l; m < n - 1; m++)
            {
                double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) <= 2.220446049250313e-16 * dd) break;
            }
            if (m == l) break;
            if (++iter > 60) return l + 1;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
            double s = 1.0, c = 1.0, p = 0.0;
            int    i;
            int    deflated = 0;
            for (i = m - 1; i >= l; i--)
            {
                double f = s * e[i], b = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0)
                {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = 1;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; k++)
                {
                    f = z[k * n + i + 1];
                    z[k * n + i + 1] = s * z[k * n + i] + c * f;
                    z[k * n + i] = c * z[k * n + i] - s * f;
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

static ocplx
cdot(uint64_t n, const ocplx* a, const ocplx* b)
{
    double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
    for (uint64_t i = 0; i < n; i++)
    {
        ocplx z = conj(a[i]) * b[i];
        re += creal(z);
        im += cimag(z);
    }
    return re + I * im;
}

static double
cnorm(uint64_t n, const ocplx* a)
{
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (uint64_t i = 0; i < n; i++)
        s += creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]);
    return sqrt(s);
}

/* multiconfig_lanczos.c:12-90 */
int
orc_lanczos(int npar, int norb, const ocplx* hob, const ocplx* hint, int lm,
            ocplx* diag, ocplx* offd, ocplx* lvec)
{
    space_t  sp = space_make(npar, norb);
    uint64_t nc = sp.dim;
    ocplx*   out = malloc(sizeof(ocplx) * nc);
    ocplx    ortho[64];
    double   maxCheck = 0, tol = 1e-14;
    int      done = lm;

    hc_rows(&sp, lvec, hob, hint, out, 0, nc);
    diag[0] = cdot(nc, lvec, out);
    for (int i = 0; i < lm - 1; i++)
    {
        ocplx* vi = lvec + (uint64_t) i * nc;
#pragma omp parallel for schedule(static)
        for (uint64_t j = 0; j < nc; j++) out[j] = out[j] - diag[i] * vi[j];
        for (int k = 0; k < i + 1; k++)
            ortho[k] = cdot(nc, lvec + (uint64_t) k * nc, out);
#pragma omp parallel for schedule(static)
        for (uint64_t j = 0; j < nc; j++)
            for (int k = 0; k < i + 1; k++)
                out[j] -= lvec[(uint64_t) k * nc + j] * ortho[k];
        offd[i] = cnorm(nc, out);
        if (maxCheck < creal(offd[i])) maxCheck = creal(offd[i]);
        if (creal(offd[i]) == 0.0 || creal(offd[i]) / maxCheck < tol)
        {
            done = i + 1;
            break;
        }
        ocplx* vn = lvec + (uint64_t) (i + 1) * nc;
        ocplx  sc = 1.0 / offd[i];
#pragma omp parallel for schedule(static)
        for (uint64_t j = 0; j < nc; j++) vn[j] = out[j] * sc;
        hc_rows(&sp, vn, hob, hint, out, 0, nc);
#pragma omp parallel for schedule(static)
        for (uint64_t j = 0; j < nc; j++) out[j] = out[j] - offd[i] * vi[j];
        diag[i + 1] = cdot(nc, vn, out);
    }
    free(out);
    space_free(&sp);
    return done;
}

/* coefficients_integration.c:59-160 */
int
orc_sil_step(int npar, int norb, const ocplx* hob, const ocplx* hint, int m,
             ocplx prop_dt, int imagtime, ocplx* coef, ocplx* lvec)
{
    uint64_t nc = orc_space_dimension(npar, norb);
    ocplx    diag[64], offd[64], aux[64], cl[64];
    double   d[64], e[64], z[64 * 64];
    memcpy(lvec, coef, sizeof(ocplx) * nc);
    offd[m - 1] = 0;
    int it = orc_lanczos(npar, norb, hob, hint, m, diag, offd, lvec);
    for (int k = 0; k < it; k++)
    {
        d[k] = creal(diag[k]);
        e[k] = creal(offd[k]);
    }
    if (orc_tridiag_eig(it, d, e, z) != 0) return -1;
    for (int k = 0; k < it; k++) cl[k] = 0;
    cl[0] = 1.0;
    for (int k = 0; k < it; k++)
    {
        aux[k] = 0;
        for (int j = 0; j < it; j++) aux[k] += z[j * it + k] * cl[j];
        aux[k] = aux[k] * cexp(-I * d[k] * prop_dt);
    }
    for (int k = 0; k < it; k++)
    {
        cl[k] = 0;
        for (int j = 0; j < it; j++) cl[k] += z[k * it + j] * aux[j];
    }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < nc; i++)
    {
        ocplx s = 0;
        for (int j = 0; j < it; j++) s += lvec[(uint64_t) j * nc + i] * cl[j];
        coef[i] = s;
    }
    if (imagtime)
    {
        double r = 1.0 / cnorm(nc, coef);
#pragma omp parallel for schedule(static)
        for (uint64_t i = 0; i < nc; i++) coef[i] = coef[i] * r;
    }
    return it;
}

/* multiconfig_lanczos.c:93-172 */
double
orc_lowest_state_lanczos(int npar, int norb, const ocplx* hob,
                         const ocplx* hint, int m, ocplx* coef, ocplx* lvec)
{
    uint64_t nc = orc_space_dimension(npar, norb);
    ocplx*   diag = malloc(sizeof(ocplx) * m);
    ocplx*   offd = malloc(sizeof(ocplx) * m);
    double * d = malloc(sizeof(double) * m), *e = malloc(sizeof(double) * m);
    double*  z = malloc(sizeof(double) * m * m);
    memcpy(lvec, coef, sizeof(ocplx) * nc);
    offd[m - 1] = 0;
    int it = orc_lanczos(npar, norb, hob, hint, m, diag, offd, lvec);
    for (int k = 0; k < it; k++)
    {
        d[k] = creal(diag[k]);
        e[k] = creal(offd[k]);
    }
    orc_tridiag_eig(it, d, e, z);
    double sentinel = 1e15;
    int    jm = 0;
    for (int k = 0; k < it; k++)
        if (sentinel > d[k])
        {
            sentinel = d[k];
            jm = k;
        }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < nc; i++)
    {
        ocplx s = 0;
        for (int k = 0; k < it; k++) s += lvec[(uint64_t) k * nc + i] * z[k * it + jm];
        coef[i] = s;
    }
    free(diag);
    free(offd);
    free(d);
    free(e);
    free(z);
    return sentinel;
}

/* integrator_monitor.c:56-88 */
ocplx
orc_total_energy(int M, const ocplx* rho1, const ocplx* rho2, const ocplx* hob,
                 const ocplx* hint)
{
    ocplx z = 0, w = 0;
    int   M2 = M * M, M3 = M2 * M;
    for (int k = 0; k < M; k++)
        for (int l = 0; l < M; l++)
        {
            w = w + rho1[k * M + l] * hob[k * M + l];
            for (int s = 0; s < M; s++)
                for (int q = 0; q < M; q++)
                    z = z + rho2[k + l * M + s * M2 + q * M3] *
                                hint[k + l * M + q * M2 + s * M3];
        }
    return w + z / 2;
}

/* integrator_monitor.c:10-28 */
double
orc_eig_residual(int npar, int norb, const ocplx* c, const ocplx* hob,
                 const ocplx* hint, double e)
{
    uint64_t nc = orc_space_dimension(npar, norb);
    ocplx*   hc = malloc(sizeof(ocplx) * nc);
    orc_apply_hamiltonian(npar, norb, c, hob, hint, hc);
    double mx = 0;
    for (uint64_t i = 0; i < nc; i++)
    {
        double a = cabs(e * c[i] - hc[i]);
        if (a > mx) mx = a;
    }
    free(hc);
    return mx / npar;
}

/* ------------------------------------------------------------------ */
/* orbital side                                                        */
/* ------------------------------------------------------------------ */

/* calculus.c:9-40 */
ocplx
orc_simpson(int n, double h, const ocplx* f)
{
    ocplx sum = 0;
    if (n % 2 == 0)
    {
        for (int i = 0; i < n - 4; i += 2) sum += f[i] + 4 * f[i + 1] + f[i + 2];
        sum *= h / 3;
        sum += (f[n - 4] + 3 * (f[n - 3] + f[n - 2]) + f[n - 1]) * 3 * h / 8;
        return sum;
    }
    for (int i = 0; i < n - 2; i += 2) sum += f[i] + 4 * f[i + 1] + f[i + 2];
    sum *= h / 3;
    return sum;
}

static double
rsimpson(int n, double h, const double* f)
{
    double sum = 0;
    if (n % 2 == 0)
    {
        for (int i = 0; i < n - 4; i += 2) sum += f[i] + 4 * f[i + 1] + f[i + 2];
        sum *= h / 3;
        sum += (f[n - 4] + 3 * (f[n - 3] + f[n - 2]) + f[n - 1]) * 3 * h / 8;
        return sum;
    }
    for (int i = 0; i < n - 2; i += 2) sum += f[i] + 4 * f[i + 1] + f[i + 2];
    sum *= h / 3;
    return sum;
}

/* calculus.c:288-305 */
void
orc_dxfd(int n, double dx, const ocplx* f, ocplx* d)
{
    double r = 1.0 / (12 * dx);
    d[0] = (f[n - 3] - f[2] + 8 * (f[1] - f[n - 2])) * r;
    d[1] = (f[n - 2] - f[3] + 8 * (f[2] - f[0])) * r;
    d[n - 3] = (f[n - 5] - f[0] + 8 * (f[n - 2] - f[n - 4])) * r;
    d[n - 2] = (f[n - 4] - f[1] + 8 * (f[0] - f[n - 3])) * r;
    d[n - 1] = d[0];
    for (int i = 2; i < n - 3; i++)
        d[i] = (f[i - 2] - f[i + 2] + 8 * (f[i + 1] - f[i - 1])) * r;
}

/* orbital_matrices.c:22-70 */
void
orc_orbital_hob(int M, int G, double dx, double a2, ocplx a1, const double* V,
                const ocplx* orb, ocplx* hob)
{
    ocplx* di = malloc(sizeof(ocplx) * G);
    ocplx* dj = malloc(sizeof(ocplx) * G);
    ocplx* in = malloc(sizeof(ocplx) * G);
    for (int i = 0; i < M; i++)
    {
        const ocplx* oi = orb + (size_t) i * G;
        orc_dxfd(G, dx, oi, di);
        for (int j = i + 1; j < M; j++)
        {
            const ocplx* oj = orb + (size_t) j * G;
            orc_dxfd(G, dx, oj, dj);
            for (int k = 0; k < G; k++)
            {
                ocplx part = -a2 * conj(di[k]) * dj[k];
                part = part + a1 * conj(oi[k]) * dj[k];
                part = part + V[k] * conj(oi[k]) * oj[k];
                in[k] = part;
            }
            ocplx p = orc_simpson(G, dx, in);
            hob[i * M + j] = p;
            hob[j * M + i] = conj(p);
        }
        for (int k = 0; k < G; k++)
        {
            ocplx part = -a2 * conj(di[k]) * di[k];
            part = part + a1 * conj(oi[k]) * di[k];
            part = part + V[k] * conj(oi[k]) * oi[k];
            in[k] = part;
        }
        hob[i * M + i] = creal(orc_simpson(G, dx, in));
    }
    free(di);
    free(dj);
    free(in);
}

/* orbital_matrices.c:73-287: every element of
 *   hint[a + b M + c M^2 + d M^3] = g * Simpson( conj(phi_a phi_b) phi_c phi_d )
 * (the reference evaluates the unique classes and fills the rest by the
 * exchange and conjugation symmetries; the values agree to rounding). */
void
orc_orbital_hint(int M, int G, double dx, double g, const ocplx* orb,
                 ocplx* hint)
{
    ocplx* in = malloc(sizeof(ocplx) * G);
    for (int a = 0; a < M; a++)
        for (int b = 0; b < M; b++)
            for (int c = 0; c < M; c++)
                for (int d = 0; d < M; d++)
                {
                    for (int x = 0; x < G; x++)
                        in[x] = conj(orb[a * G + x] * orb[b * G + x]) *
                                orb[c * G + x] * orb[d * G + x];
                    hint[a + b * M + c * M * M + d * M * M * M] =
                        g * orc_simpson(G, dx, in);
                }
    free(in);
}

/* calculus.c:117-129 */
static void
renormalize(int n, double dx, ocplx* f)
{
    double* m2 = malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++)
        m2[i] = creal(f[i]) * creal(f[i]) + cimag(f[i]) * cimag(f[i]);
    double r = sqrt(1.0 / rsimpson(n, dx, m2));
    for (int i = 0; i < n; i++) f[i] = f[i] * r;
    free(m2);
}

static ocplx
sprod(int n, double h, const ocplx* a, const ocplx* b, ocplx* work)
{
    for (int i = 0; i < n; i++) work[i] = conj(a[i]) * b[i];
    return orc_simpson(n, h, work);
}

/* calculus.c:171-191.  Note the reference re-evaluates the overlap for every
 * grid point k while F[i] is being updated (calculus.c:181-184); that is
 * restated literally. */
void
orc_orthonormalize(int G, double dx, int nf, ocplx* F)
{
    ocplx* w = malloc(sizeof(ocplx) * G);
    renormalize(G, dx, F);
    for (int i = 1; i < nf; i++)
    {
        for (int j = 0; j < i; j++)
            for (int k = 0; k < G; k++)
                F[i * G + k] -= sprod(G, dx, F + j * G, F + i * G, w) * F[j * G + k];
        renormalize(G, dx, F + i * G);
    }
    free(w);
}

/* Cyclic Jacobi for an n x n Hermitian matrix (row-major); eigenvalues
 * ascending in w, eigenvectors in the columns of vec. */
int
orc_herm_eig(int n, const ocplx* a0, double* w, ocplx* vec)
{
    ocplx* a = malloc(sizeof(ocplx) * n * n);
    ocplx* v = malloc(sizeof(ocplx) * n * n);
    memcpy(a, a0, sizeof(ocplx) * n * n);
    for (int i = 0; i < n * n; i++) v[i] = 0;
    for (int i = 0; i < n; i++) v[i * n + i] = 1;
    for (int sweep = 0; sweep < 100; sweep++)
    {
        double off = 0, tot = 0;
        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++)
            {
                double m = cabs(a[p * n + q]);
                tot += m * m;
                if (p != q) off += m * m;
            }
        if (off <= 1e-30 * tot || off == 0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++)
            {
                ocplx  apq = a[p * n + q];
                double mag = cabs(apq);
                if (mag == 0) continue;
                double app = creal(a[p * n + p]), aqq = creal(a[q * n + q]);
                ocplx  ph = apq / mag; /* a_pq = |a_pq| e^{i phi} */
                double theta = 0.5 * atan2(2 * mag, aqq - app);
                double c = cos(theta), s = sin(theta);
                /* rotation J: columns p,q -> p' = c p - s conj(ph) q ... */
                for (int k = 0; k < n; k++)
                {
                    ocplx akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = c * akp - s * conj(ph) * akq;
                    a[k * n + q] = s * ph * akp + c * akq;
                }
                for (int k = 0; k < n; k++)
                {
                    ocplx apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = c * apk - s * ph * aqk;
                    a[q * n + k] = s * conj(ph) * apk + c * aqk;
                }
                for (int k = 0; k < n; k++)
                {
                    ocplx vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = c * vkp - s * conj(ph) * vkq;
                    v[k * n + q] = s * ph * vkp + c * vkq;
                }
            }
    }
    /* sort ascending */
    int idx[64];
    for (int i = 0; i < n; i++) idx[i] = i;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (creal(a[idx[j] * n + idx[j]]) < creal(a[idx[i] * n + idx[i]]))
            {
                int t = idx[i];
                idx[i] = idx[j];
                idx[j] = t;
            }
    for (int i = 0; i < n; i++)
    {
        w[i] = creal(a[idx[i] * n + idx[i]]);
        if (vec)
            for (int k = 0; k < n; k++) vec[k * n + i] = v[k * n + idx[i]];
    }
    free(a);
    free(v);
    return 0;
}

/* Gauss-Jordan inverse with partial pivoting */
int
orc_herm_inverse(int n, const ocplx* a0, ocplx* inv)
{
    ocplx* a = malloc(sizeof(ocplx) * n * n);
    memcpy(a, a0, sizeof(ocplx) * n * n);
    for (int i = 0; i < n * n; i++) inv[i] = 0;
    for (int i = 0; i < n; i++) inv[i * n + i] = 1;
    for (int c = 0; c < n; c++)
    {
        int    piv = c;
        double best = cabs(a[c * n + c]);
        for (int r = c + 1; r < n; r++)
            if (cabs(a[r * n + c]) > best)
            {
                best = cabs(a[r * n + c]);
                piv = r;
            }
        if (best == 0)
        {
            free(a);
            return c + 1;
        }
        if (piv != c)
            for (int k = 0; k < n; k++)
            {
                ocplx t = a[c * n + k];
                a[c * n + k] = a[piv * n + k];
                a[piv * n + k] = t;
                t = inv[c * n + k];
                inv[c * n + k] = inv[piv * n + k];
                inv[piv * n + k] = t;
            }
        ocplx p = 1.0 / a[c * n + c];
        for (int k = 0; k < n; k++)
        {
            a[c * n + k] *= p;
            inv[c * n + k] *= p;
        }
        for (int r = 0; r < n; r++)
        {
            if (r == c) continue;
            ocplx f = a[r * n + c];
            if (f == 0) continue;
            for (int k = 0; k < n; k++)
            {
                a[r * n + k] -= f * a[c * n + k];
                inv[r * n + k] -= f * inv[c * n + k];
            }
        }
    }
    free(a);
    return 0;
}

/* synchronize.c:42-57 with lapack_interface.c:100-163 */
void
orc_sync_density_matrices(int npar, int M, const ocplx* coef, double reg_fac,
                          ocplx* rho1, ocplx* rho2, ocplx* rinv)
{
    double w[64];
    orc_onebody_dm(npar, M, coef, rho1);
    orc_twobody_dm(npar, M, coef, rho2);
    orc_herm_eig(M, rho1, w, NULL);
    if (w[0] / w[M - 1] < reg_fac)
    {
        double x = w[M - 1] * reg_fac;
        ocplx* vec = malloc(sizeof(ocplx) * M * M);
        double ev[64];
        orc_herm_eig(M, rho1, ev, vec);
        for (int i = 0; i < M; i++)
            for (int j = 0; j < M; j++)
            {
                ocplx z = 0;
                for (int k = 0; k < M; k++)
                    z += vec[i * M + k] * (x * exp(-ev[k] / x)) * conj(vec[j * M + k]);
                rho1[i * M + j] = rho1[i * M + j] + z;
            }
        free(vec);
    }
    orc_herm_inverse(M, rho1, rinv);
}

/* split_nonlinear_orbitals.c:4-61 */
static ocplx
interacting_part(int k, int n, int M, int G, double g, const ocplx* rho,
                 const ocplx* rinv, const ocplx* orb)
{
    int   mm = M * M, mmm = M * M * M;
    ocplx red = 0, grho, swap;
#define O(a, x) orb[(a) * G + (x)]
    for (int a = 0; a < M; a++)
    {
        for (int q = 0; q < M; q++)
        {
            grho = g * rinv[k * M + a] * rho[a + M * a + mm * q + mmm * q];
            red = red + grho * conj(O(a, n)) * O(q, n) * O(q, n);
            for (int l = q + 1; l < M; l++)
            {
                grho = 2 * g * rinv[k * M + a] * rho[a + M * a + mm * q + mmm * l];
                red = red + grho * conj(O(a, n)) * O(l, n) * O(q, n);
            }
        }
        for (int s = a + 1; s < M; s++)
        {
            for (int q = 0; q < M; q++)
            {
                grho = g * rinv[k * M + a] * rho[a + M * s + mm * q + mmm * q];
                swap = g * rinv[k * M + s] * rho[a + M * s + mm * q + mmm * q];
                red = red + (grho * conj(O(s, n)) + swap * conj(O(a, n))) *
                                O(q, n) * O(q, n);
                for (int l = q + 1; l < M; l++)
                {
                    grho = 2 * g * rinv[k * M + a] * rho[a + M * s + mm * q + mmm * l];
                    swap = 2 * g * rinv[k * M + s] * rho[a + M * s + mm * q + mmm * l];
                    red = red + (grho * conj(O(s, n)) + swap * conj(O(a, n))) *
                                    O(l, n) * O(q, n);
                }
            }
        }
    }
#undef O
    return red;
}

/* split_linear_orbitals.c:210-255 */
static void
linear_fd(int G, double dx, double a2, ocplx a1, int periodic, const double* pot,
          const ocplx* f, ocplx* out)
{
    ocplx upper = a2 / dx / dx + a1 / dx / 2;
    ocplx lower = a2 / dx / dx - a1 / dx / 2;
    ocplx mid = -2 * a2 / dx / dx + pot[0];
    if (!periodic)
        out[0] = mid * f[0] + upper * f[1];
    else
        out[0] = mid * f[0] + upper * f[1] + lower * f[G - 2];
    for (int i = 1; i < G - 1; i++)
    {
        mid = -2 * a2 / dx / dx + pot[i];
        out[i] = mid * f[i] + upper * f[i + 1] + lower * f[i - 1];
    }
    if (!periodic)
    {
        mid = -2 * a2 / dx / dx + pot[G - 1];
        out[G - 1] = mid * f[G - 1] + lower * f[G - 2];
    }
    else
    {
        mid = -2 * a2 / dx / dx + pot[G - 2];
        out[G - 2] = mid * f[G - 2] + upper * f[0] + lower * f[G - 3];
        out[G - 1] = out[0];
    }
}

/* The DVR matrix of split_linear_orbitals.c:83-166 on the n = G - 1
 * periodic points (row-major n x n): first and second derivatives in the
 * exponential basis, kmom = k - n/2, each element summed over k in order,
 * with d1coef / d2coef applied as there. */
static ocplx*
dvr_matrix(int n, double dx, double a2, ocplx a1)
{
    const double pi = 3.14159265358979323846, length = n * dx;
    ocplx*       d1 = malloc(sizeof(ocplx) * n * n);
    ocplx*       d2 = malloc(sizeof(ocplx) * n * n);
    ocplx*       out = malloc(sizeof(ocplx) * n * n);
    for (int i = 0; i < n; i++)
    {
        for (int j = i + 1; j < n; j++)
        {
            ocplx s1 = 0, s2 = 0;
            for (int k = 0; k < n; k++)
            {
                const int    kmom = k - n / 2;
                const ocplx  e = cexp(2 * I * kmom * (j - i) * pi / n);
                const ocplx  g1 = -(2 * I * pi * kmom / length);
                const double g2 = -(2 * pi * kmom / length) * (2 * pi * kmom / length);
                s1 += g1 * e / n;
                s2 += g2 * e / n;
            }
            d1[i * n + j] = s1;
            d1[j * n + i] = -conj(s1);
            d2[i * n + j] = s2;
            d2[j * n + i] = conj(s2);
        }
        ocplx s1 = 0, s2 = 0;
        for (int k = 0; k < n; k++)
        {
            const int kmom = k - n / 2;
            s1 = s1 + (-(2 * I * pi * kmom / length)) / n;
            s2 = s2 + (-(2 * pi * kmom / length) * (2 * pi * kmom / length)) / n;
        }
        d1[i * n + i] = s1;
        d2[i * n + i] = s2;
    }
    for (int i = 0; i < n * n; i++) out[i] = a2 * d2[i] + a1 * d1[i];
    free(d1);
    free(d2);
    return out;
}

/* linear part a2 f'' + a1 f' + V f (orbital_integration.c:137-176):
 * der = 302 finite differences (split_linear_orbitals.c:210-255); 300 the
 * DVR matrix; 301 spectral (split_linear_orbitals.c:257-287): forward DFT
 * with 1/sqrt(n) scaling, multiplication by freq i d1coef - freq^2 d2coef
 * (calculus.c:272-285), backward DFT with 1/sqrt(n), restated here as the
 * direct transform sums.  The last point repeats the first. */
static void
linear_part(int der, int G, double dx, double a2, ocplx a1, int periodic,
            const double* pot, const ocplx* dvr, const ocplx* f, ocplx* out)
{
    const int n = G - 1;
    if (der == 300)
    {
        for (int i = 0; i < n; i++)
        {
            ocplx z = 0;
            for (int j = 0; j < n; j++) z += dvr[i * n + j] * f[j];
            out[i] = z + pot[i] * f[i];
        }
        out[n] = out[0];
    }
    else if (der == 301)
    {
        const double pi = 3.14159265358979323846, sc = 1.0 / sqrt((double) n);
        ocplx*       F = malloc(sizeof(ocplx) * n);
        for (int k = 0; k < n; k++)
        {
            ocplx z = 0;
            for (int x = 0; x < n; x++)
                z += f[x] * cexp(-2 * I * pi * (double) (((long) k * x) % n) / n);
            const double freq = k <= (n - 1) / 2 ? 2 * pi * k / (n * dx)
                                                 : 2 * pi * (k - n) / (n * dx);
            F[k] = z * sc * (freq * I * a1 - freq * freq * a2);
        }
        for (int x = 0; x < n; x++)
        {
            ocplx z = 0;
            for (int k = 0; k < n; k++)
                z += F[k] * cexp(2 * I * pi * (double) (((long) k * x) % n) / n);
            out[x] = z * sc + pot[x] * f[x];
        }
        out[n] = out[0];
        free(F);
    }
    else
        linear_fd(G, dx, a2, a1, periodic, pot, f, out);
}

/* orbital_integration.c:179-240 (FINITEDIFF).  robust = 0: the simple
 * projector (:95-131), P_k = sum_s f_s <f_s|H f_k>; robust = 1: the robust
 * projector (:22-92), P_k = sum_{s,l} f_s (S^-1)_{sl} <f_l|H f_k> with the
 * overlap matrix S_{sl} = <f_s|f_l> (orbital_matrices.c:7-19, all entries:
 * that loop starts its inner index at 2, which leaves S_01 and S_10 as
 * uninitialised heap memory in the reference; the full matrix is its
 * evident intent).  Returns 0, or the inversion's error code with dodt
 * untouched. */
int
orc_orbital_rhs(int M, int G, double dx, double a2, ocplx a1, double g,
                int periodic, ocplx time_fac, const double* pot,
                const ocplx* rinv, const ocplx* rho2, const ocplx* orb,
                ocplx* dodt, int robust, int der)
{
    ocplx* lin = malloc(sizeof(ocplx) * M * G);
    ocplx* ha = malloc(sizeof(ocplx) * M * G);
    ocplx* po = malloc(sizeof(ocplx) * M * M);
    ocplx* w = malloc(sizeof(ocplx) * G);
    ocplx* dvr = der == 300 ? dvr_matrix(G - 1, dx, a2, a1) : NULL;
    for (int k = 0; k < M; k++)
        linear_part(der, G, dx, a2, a1, periodic, pot, dvr, orb + k * G, lin + k * G);
    free(dvr);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < M; k++)
        for (int j = 0; j < G; j++)
            ha[k * G + j] =
                interacting_part(k, j, M, G, g, rho2, rinv, orb) + lin[k * G + j];
    for (int k = 0; k < M; k++)
        for (int s = 0; s < M; s++)
            po[s * M + k] = sprod(G, dx, orb + s * G, ha + k * G, w);
    int info = 0;
    if (robust)
    {
        ocplx* ov = malloc(sizeof(ocplx) * M * M);
        ocplx* inv = malloc(sizeof(ocplx) * M * M);
        ocplx* pr = malloc(sizeof(ocplx) * M * M);
        for (int s = 0; s < M; s++)
            for (int l = 0; l < M; l++)
                ov[s * M + l] = sprod(G, dx, orb + s * G, orb + l * G, w);
        info = orc_herm_inverse(M, ov, inv);
        for (int s = 0; s < M; s++)
            for (int k = 0; k < M; k++)
            {
                ocplx z = 0;
                for (int l = 0; l < M; l++) z += inv[s * M + l] * po[l * M + k];
                pr[s * M + k] = z;
            }
        memcpy(po, pr, sizeof(ocplx) * M * M);
        free(ov);
        free(inv);
        free(pr);
    }
    if (info == 0)
        for (int k = 0; k < M; k++)
            for (int i = 0; i < G; i++)
            {
                ocplx proj = 0;
                for (int s = 0; s < M; s++)
                    proj += orb[s * G + i] * po[s * M + k];
                dodt[k * G + i] = -I * time_fac * (ha[k * G + i] - proj);
            }
    free(lin);
    free(ha);
    free(po);
    free(w);
    return info;
}

/* Thomas algorithm: lo[i] A[i][i-1], md[i] A[i][i], up[i] A[i][i+1] */
static void
tridiag_solve(int n, const ocplx* lo, const ocplx* md, const ocplx* up,
              const ocplx* rhs, ocplx* x)
{
    ocplx* c = malloc(sizeof(ocplx) * n);
    ocplx* d = malloc(sizeof(ocplx) * n);
    c[0] = up[0] / md[0];
    d[0] = rhs[0] / md[0];
    for (int i = 1; i < n; i++)
    {
        const ocplx den = md[i] - lo[i] * c[i - 1];
        c[i] = up[i] / den;
        d[i] = (rhs[i] - lo[i] * d[i - 1]) / den;
    }
    x[n - 1] = d[n - 1];
    for (int i = n - 2; i >= 0; i--) x[i] = d[i] - c[i] * x[i + 1];
    free(c);
    free(d);
}

/* Crank-Nicolson half step of the linear part (split_linear_orbitals.c:
 * 23-56, 289-373): (i - dth A) f' = (i + dth A) f in the reference's
 * coefficients, dth = prop_dt / 2; periodic grids solve the cyclic system
 * on the G - 1 distinct points (Sherman-Morrison) and copy the last point */
static void
cn_half_step(int G, double dx, double a2, ocplx a1, int periodic, ocplx dth,
             ocplx* f)
{
    const ocplx mid = I + a2 * dth / dx / dx;
    const ocplx up = -a2 * dth / dx / dx / 2 - a1 * dth / dx / 4;
    const ocplx lo = -a2 * dth / dx / dx / 2 + a1 * dth / dx / 4;
    const ocplx rmid = I - a2 * dth / dx / dx;
    const ocplx rup = a2 * dth / dx / dx / 2 + a1 * dth / dx / 4;
    const ocplx rlo = a2 * dth / dx / dx / 2 - a1 * dth / dx / 4;
    const int   n = periodic ? G - 1 : G;
    ocplx*      rhs = calloc(n, sizeof(ocplx));
    ocplx*      L = calloc(n, sizeof(ocplx));
    ocplx*      D = calloc(n, sizeof(ocplx));
    ocplx*      U = calloc(n, sizeof(ocplx));
    ocplx*      x = calloc(n, sizeof(ocplx));
    for (int i = 0; i < n; i++)
    {
        ocplx r = rmid * f[i];
        if (i + 1 < n) r += rup * f[i + 1];
        else if (periodic) r += rup * f[0];
        if (i > 0) r += rlo * f[i - 1];
        else if (periodic) r += rlo * f[n - 1];
        rhs[i] = r;
        L[i] = lo;
        D[i] = mid;
        U[i] = up;
    }
    if (!periodic)
        tridiag_solve(n, L, D, U, rhs, x);
    else
    {
        /* corners A[0][n-1] = lo, A[n-1][0] = up: A = T + u v^T with
         * u = (gam, 0 .., up), v = (1, 0 .., lo / gam) */
        const ocplx gam = -mid;
        ocplx*      u = calloc(n, sizeof(ocplx));
        ocplx*      z = malloc(sizeof(ocplx) * n);
        D[0] = mid - gam;
        D[n - 1] = mid - up * lo / gam;
        u[0] = gam;
        u[n - 1] = up;
        tridiag_solve(n, L, D, U, rhs, x);
        tridiag_solve(n, L, D, U, u, z);
        const ocplx fac = (x[0] + lo / gam * x[n - 1]) / (1.0 + z[0] + lo / gam * z[n - 1]);
        for (int i = 0; i < n; i++) x[i] -= fac * z[i];
        free(u);
        free(z);
    }
    for (int i = 0; i < n; i++) f[i] = x[i];
    if (periodic) f[G - 1] = f[0];
    free(rhs);
    free(L);
    free(D);
    free(U);
    free(x);
}

/* FFT-exponential half step (split_linear_orbitals.c:57-82, 375-402):
 * f <- IDFT(exp(-i dth (i freq a1 - freq^2 a2)) DFT(f)) on the n = G - 1
 * distinct points, 1/sqrt(n) both ways, restated as direct sums */
static void
fftexp_half_step(int G, double dx, double a2, ocplx a1, ocplx dth, ocplx* f)
{
    const int    n = G - 1;
    const double pi = 3.14159265358979323846, sc = 1.0 / sqrt((double) n);
    ocplx*       F = malloc(sizeof(ocplx) * n);
    for (int k = 0; k < n; k++)
    {
        ocplx z = 0;
        for (int x = 0; x < n; x++)
            z += f[x] * cexp(-2 * I * pi * (double) (((long) k * x) % n) / n);
        const double freq = k <= (n - 1) / 2 ? 2 * pi * k / (n * dx)
                                             : 2 * pi * (k - n) / (n * dx);
        F[k] = z * sc * cexp(-I * dth * (I * a1 * freq - a2 * freq * freq));
    }
    for (int x = 0; x < n; x++)
    {
        ocplx z = 0;
        for (int k = 0; k < n; k++)
            z += F[k] * cexp(2 * I * pi * (double) (((long) k * x) % n) / n);
        f[x] = z * sc;
    }
    f[n] = f[0];
    free(F);
}

void
orc_linear_half_step(int der, int G, double dx, double a2, ocplx a1, int periodic,
                     ocplx dth, ocplx* f)
{
    if (der == 302) cn_half_step(G, dx, a2, a1, periodic, dth, f);
    else fftexp_half_step(G, dx, a2, a1, dth, f);
}

typedef struct
{
    int           M, G, periodic, robust, der, split;
    double        dx, a2, g;
    ocplx         a1, tf;
    const double* pot;
    const ocplx * rinv, *rho2, *hob, *hint;
} rhs_args;

/* split_nonlinear_orbitals.c:63-160 (orb_full_nonlinear) at point x of
 * orbital k: the interacting part with its projection through h and g,
 * over the same index ranges (s >= a, l >= q with the exchange factors) */
static ocplx
full_nonlinear(int k, int x, int M, int G, double g, const ocplx* orb,
               const ocplx* hob, const ocplx* hint, const ocplx* rho,
               const ocplx* rinv)
{
    const int mm = M * M, mmm = mm * M;
#define O(i) orb[(i) * G + x]
    ocplx red = 0;
    for (int a = 0; a < M; a++)
    {
        red -= hob[a * M + k] * O(a);
        for (int q = 0; q < M; q++)
        {
            ocplx rm = rinv[k * M + a] * rho[a + M * a + mm * q + mmm * q];
            red += g * rm * conj(O(a)) * O(q) * O(q);
            for (int j = 0; j < M; j++) red -= rm * O(j) * hint[j + a * M + q * mm + q * mmm];
            for (int l = q + 1; l < M; l++)
            {
                rm = 2 * rinv[k * M + a] * rho[a + M * a + mm * q + mmm * l];
                red += g * rm * conj(O(a)) * O(l) * O(q);
                for (int j = 0; j < M; j++)
                    red -= rm * O(j) * hint[j + a * M + l * mm + q * mmm];
            }
        }
        for (int s = a + 1; s < M; s++)
        {
            for (int q = 0; q < M; q++)
            {
                ocplx rm = rinv[k * M + a] * rho[a + M * s + mm * q + mmm * q];
                ocplx sw = rinv[k * M + s] * rho[a + M * s + mm * q + mmm * q];
                red += g * (rm * conj(O(s)) + sw * conj(O(a))) * O(q) * O(q);
                for (int j = 0; j < M; j++)
                {
                    red -= rm * O(j) * hint[j + s * M + q * mm + q * mmm];
                    red -= sw * O(j) * hint[j + a * M + q * mm + q * mmm];
                }
                for (int l = q + 1; l < M; l++)
                {
                    rm = 2 * rinv[k * M + a] * rho[a + M * s + mm * q + mmm * l];
                    sw = 2 * rinv[k * M + s] * rho[a + M * s + mm * q + mmm * l];
                    red += g * (rm * conj(O(s)) + sw * conj(O(a))) * O(l) * O(q);
                    for (int j = 0; j < M; j++)
                    {
                        red -= rm * O(j) * hint[j + s * M + l * mm + q * mmm];
                        red -= sw * O(j) * hint[j + a * M + l * mm + q * mmm];
                    }
                }
            }
        }
    }
#undef O
    return red;
}

static void
rhs_eval(const rhs_args* a, const ocplx* y, ocplx* out)
{
    if (a->split)
    {
        /* orbital_integration.c:243-281: -i tf (nonlinear + V f) */
        for (int k = 0; k < a->M; k++)
            for (int x = 0; x < a->G; x++)
                out[k * a->G + x] =
                    -I * a->tf *
                    (full_nonlinear(k, x, a->M, a->G, a->g, y, a->hob, a->hint, a->rho2,
                                    a->rinv) +
                     a->pot[x] * y[k * a->G + x]);
        return;
    }
    orc_orbital_rhs(a->M, a->G, a->dx, a->a2, a->a1, a->g, a->periodic, a->tf,
                    a->pot, a->rinv, a->rho2, y, out, a->robust, a->der);
}

/* the named tableaux of shim/odesys.h (Heun, classical RK4, Butcher RK5) */
static void
rk_step(int order, const rhs_args* a, int n, double dt, const ocplx* y,
        ocplx* yn)
{
    ocplx* k[6];
    for (int i = 0; i < 6; i++) k[i] = malloc(sizeof(ocplx) * n);
    ocplx* w = malloc(sizeof(ocplx) * n);
    if (order == 2)
    {
        rhs_eval(a, y, k[0]);
        for (int i = 0; i < n; i++) w[i] = y[i] + dt * k[0][i];
        rhs_eval(a, w, k[1]);
        for (int i = 0; i < n; i++) yn[i] = y[i] + 0.5 * dt * (k[0][i] + k[1][i]);
    }
    else if (order == 4)
    {
        rhs_eval(a, y, k[0]);
        for (int i = 0; i < n; i++) w[i] = y[i] + 0.5 * dt * k[0][i];
        rhs_eval(a, w, k[1]);
        for (int i = 0; i < n; i++) w[i] = y[i] + 0.5 * dt * k[1][i];
        rhs_eval(a, w, k[2]);
        for (int i = 0; i < n; i++) w[i] = y[i] + dt * k[2][i];
        rhs_eval(a, w, k[3]);
        for (int i = 0; i < n; i++)
            yn[i] = y[i] + dt / 6.0 * (k[0][i] + 2.0 * k[1][i] + 2.0 * k[2][i] + k[3][i]);
    }
    else
    {
        rhs_eval(a, y, k[0]);
        for (int i = 0; i < n; i++) w[i] = y[i] + dt * (0.25 * k[0][i]);
        rhs_eval(a, w, k[1]);
        for (int i = 0; i < n; i++) w[i] = y[i] + dt * (0.125 * k[0][i] + 0.125 * k[1][i]);
        rhs_eval(a, w, k[2]);
        for (int i = 0; i < n; i++) w[i] = y[i] + dt * (-0.5 * k[1][i] + k[2][i]);
        rhs_eval(a, w, k[3]);
        for (int i = 0; i < n; i++)
            w[i] = y[i] + dt * ((3.0 / 16.0) * k[0][i] + (9.0 / 16.0) * k[3][i]);
        rhs_eval(a, w, k[4]);
        for (int i = 0; i < n; i++)
            w[i] = y[i] + dt * ((-3.0 / 7.0) * k[0][i] + (2.0 / 7.0) * k[1][i] +
                                (12.0 / 7.0) * k[2][i] - (12.0 / 7.0) * k[3][i] +
                                (8.0 / 7.0) * k[4][i]);
        rhs_eval(a, w, k[5]);
        for (int i = 0; i < n; i++)
            yn[i] = y[i] + dt * ((7.0 / 90.0) * k[0][i] + (32.0 / 90.0) * k[2][i] +
                                 (12.0 / 90.0) * k[3][i] + (32.0 / 90.0) * k[4][i] +
                                 (7.0 / 90.0) * k[5][i]);
    }
    for (int i = 0; i < 6; i++) free(k[i]);
    free(w);
}

/* coefficients_integration.c:15-57: dC/dt = -i tf H C by the named tableaux
 * (classical RK4; Butcher's RK5, which order 2 also takes there, :44-47),
 * then the imaginary-time renormalisation */
static void
coef_rk(int npar, int M, const ocplx* hob, const ocplx* hint, int order,
        double dt, int imagtime, ocplx* coef)
{
    const uint64_t nc = orc_space_dimension(npar, M);
    const ocplx    tf = imagtime ? -I : 1.0;
    ocplx*         k[6];
    for (int i = 0; i < 6; i++) k[i] = malloc(sizeof(ocplx) * nc);
    ocplx* w = malloc(sizeof(ocplx) * nc);
#define DCDT(in, out)                                           \
    do                                                          \
    {                                                           \
        orc_apply_hamiltonian(npar, M, in, hob, hint, out);     \
        for (uint64_t i = 0; i < nc; i++) out[i] *= -I * tf;    \
    } while (0)
    if (order == 4)
    {
        DCDT(coef, k[0]);
        for (uint64_t i = 0; i < nc; i++) w[i] = coef[i] + 0.5 * dt * k[0][i];
        DCDT(w, k[1]);
        for (uint64_t i = 0; i < nc; i++) w[i] = coef[i] + 0.5 * dt * k[1][i];
        DCDT(w, k[2]);
        for (uint64_t i = 0; i < nc; i++) w[i] = coef[i] + dt * k[2][i];
        DCDT(w, k[3]);
        for (uint64_t i = 0; i < nc; i++)
            coef[i] += dt / 6.0 * (k[0][i] + 2.0 * k[1][i] + 2.0 * k[2][i] + k[3][i]);
    }
    else
    {
        DCDT(coef, k[0]);
        for (uint64_t i = 0; i < nc; i++) w[i] = coef[i] + dt * (0.25 * k[0][i]);
        DCDT(w, k[1]);
        for (uint64_t i = 0; i < nc; i++)
            w[i] = coef[i] + dt * (0.125 * k[0][i] + 0.125 * k[1][i]);
        DCDT(w, k[2]);
        for (uint64_t i = 0; i < nc; i++) w[i] = coef[i] + dt * (-0.5 * k[1][i] + k[2][i]);
        DCDT(w, k[3]);
        for (uint64_t i = 0; i < nc; i++)
            w[i] = coef[i] + dt * ((3.0 / 16.0) * k[0][i] + (9.0 / 16.0) * k[3][i]);
        DCDT(w, k[4]);
        for (uint64_t i = 0; i < nc; i++)
            w[i] = coef[i] + dt * ((-3.0 / 7.0) * k[0][i] + (2.0 / 7.0) * k[1][i] +
                                   (12.0 / 7.0) * k[2][i] - (12.0 / 7.0) * k[3][i] +
                                   (8.0 / 7.0) * k[4][i]);
        DCDT(w, k[5]);
        for (uint64_t i = 0; i < nc; i++)
            coef[i] += dt * ((7.0 / 90.0) * k[0][i] + (32.0 / 90.0) * k[2][i] +
                             (12.0 / 90.0) * k[3][i] + (32.0 / 90.0) * k[4][i] +
                             (7.0 / 90.0) * k[5][i]);
    }
#undef DCDT
    if (imagtime)
    {
        double n2 = 0;
        for (uint64_t i = 0; i < nc; i++) n2 += creal(coef[i] * conj(coef[i]));
        const double r = 1.0 / sqrt(n2);
        for (uint64_t i = 0; i < nc; i++) coef[i] *= r;
    }
    for (int i = 0; i < 6; i++) free(k[i]);
    free(w);
}

/* driver.c:159-201 with orbital_integration.c:284-349 */
void
orc_propagate_step(int npar, int M, int G, double dx, double dt, double a2,
                   ocplx a1, double g, int periodic, int imagtime, int rk_order,
                   int lanczos_m, double reg_fac, const double* pot, ocplx* orb,
                   ocplx* coef, ocplx* hob, ocplx* hint, ocplx* rho1,
                   ocplx* rho2, ocplx* rinv, int robust, int der, int coef_method,
                   int orb_method)
{
    int      n = M * G;
    ocplx    tf = imagtime ? -I : 1.0;
    ocplx    prop_dt = imagtime ? -I * dt : dt;
    rhs_args a = {M,  G,  periodic, robust, der, orb_method == 31, dx, a2, g,
                  a1, tf, pot,      rinv,   rho2, hob, hint};
    if (periodic)
        for (int k = 0; k < M; k++) orb[k * G + G - 1] = orb[k * G];
    ocplx* next = malloc(sizeof(ocplx) * n);
    if (orb_method == 31)
    {
        /* orbital_integration.c:352-434: linear half step, h and g of the
         * new orbitals, RK of the nonlinear part, linear half step */
        const ocplx dth = 0.5 * prop_dt;
        for (int k = 0; k < M; k++)
        {
            if (der == 302) cn_half_step(G, dx, a2, a1, periodic, dth, orb + k * G);
            else fftexp_half_step(G, dx, a2, a1, dth, orb + k * G);
        }
        orc_orbital_hob(M, G, dx, a2, a1, pot, orb, hob);
        orc_orbital_hint(M, G, dx, g, orb, hint);
        rk_step(rk_order, &a, n, dt, orb, next);
        memcpy(orb, next, sizeof(ocplx) * n);
        for (int k = 0; k < M; k++)
        {
            if (der == 302) cn_half_step(G, dx, a2, a1, periodic, dth, orb + k * G);
            else fftexp_half_step(G, dx, a2, a1, dth, orb + k * G);
        }
    }
    else
    {
        rk_step(rk_order, &a, n, dt, orb, next);
        memcpy(orb, next, sizeof(ocplx) * n);
    }
    free(next);
    if (imagtime) orc_orthonormalize(G, dx, M, orb);
    if (periodic)
        for (int k = 0; k < M; k++) orb[k * G + G - 1] = orb[k * G];
    orc_orbital_hob(M, G, dx, a2, a1, pot, orb, hob);
    orc_orbital_hint(M, G, dx, g, orb, hint);
    if (M == 1) return;
    if (coef_method == 21)
        coef_rk(npar, M, hob, hint, rk_order, dt, imagtime, coef);
    else
    {
        uint64_t nc = orc_space_dimension(npar, M);
        ocplx*   lw = malloc(sizeof(ocplx) * nc * lanczos_m);
        orc_sil_step(npar, M, hob, hint, lanczos_m, prop_dt, imagtime, coef, lw);
        free(lw);
    }
    orc_sync_density_matrices(npar, M, coef, reg_fac, rho1, rho2, rinv);
}
