/* ref_setup.c -- set-up of the compiled reference's structs for timing the
 * reference's own step on many jobs.
 *
 * TEST AND BENCH INFRASTRUCTURE: linked only into oracle/_ref/libmctdhb_ref.so
 * (with oracle.c, whose map builders it calls); nothing in the GPU product
 * path loads it.
 *
 * The reference's get_mctdhb_struct (src/assistant/types_definition.c:247-300)
 * spends its time in two places that the step never needs again:
 *   - get_multiconf_struct (:111-142) builds the jump maps serially
 *     (43.6 s at N=40 M=6);
 *   - get_orbital_workspace (:204-245) builds the DVR exponential matrix
 *     unconditionally (set_expdvr_mat, O(grid^3): 33 s at 1024 points),
 *     which only the DVR linear part reads.
 * refset_mctdhb_struct builds the same struct, member for member, from the
 * reference's own sub-constructors (get_orbital_equation,
 * get_coef_workspace, get_manybody_state, set_cn_tridiagonal, set_fft_freq,
 * set_hder_fftexp, set_expdvr_mat for DVR jobs), except that the jump maps
 * come from the oracle's OpenMP restatement of space.c:181-451
 * (orc_hash_table, orc_single_jump_map, orc_double_*_map: bit-exact with the
 * reference's tables) and dvr_mat is filled only for DVR jobs.  The trap is
 * a given grid array and the interaction a constant, both through the
 * reference's callback types (the `custom` route of its API).
 * destroy_mctdhb_struct frees the struct as it frees its own;
 * refset_destroy also frees the callback arguments.
 *
 * refset_multiconf times nothing itself; the bench times it (set-up) apart
 * from the step, and times the reference's own serial get_multiconf_struct
 * on one job for comparison. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "assistant/arrays_definition.h"
#include "assistant/types_definition.h"
#include "configurational/space.h"
#include "function_tools/calculus.h"
#include "integrator/split_linear_orbitals.h"
#include "odesys.h"

#include "oracle.h"

/* defined in types_definition.c:187 and used by get_mctdhb_struct, but not
 * declared in the reference's types_definition.h */
CoefWorkspace get_coef_workspace(CoefIntegrator coef_integ_method, uint32_t space_dim,
                                 uint16_t lan_it);

typedef struct
{
    uint16_t npts;
    double   v[];
} PotArgs;

static void
refset_pot(double t, uint16_t npts, double* pts, void* params, double* grid_pot)
{
    (void) t;
    (void) pts;
    const PotArgs* p = (const PotArgs*) params;
    memcpy(grid_pot, p->v, sizeof(double) * (npts < p->npts ? npts : p->npts));
}

static double
refset_const(double t, void* params)
{
    (void) t;
    return *(const double*) params;
}

/* maps of (npar, norb) in the reference's layout; NULL where the
 * reference's 32-bit guard (space.c:285-289, 384) would exit */
MultiConfiguration
refset_multiconf(uint16_t npar, uint16_t norb)
{
    const uint64_t dim = orc_space_dimension(npar, norb);
    const uint64_t tt = orc_double_diffjump_chunks(npar, norb);
    const uint64_t ot = orc_double_equaljump_chunks(npar, norb);
    const uint64_t M2 = (uint64_t) norb * norb;
    if (dim >= UINT32_MAX || tt * M2 >= UINT32_MAX || ot * M2 >= UINT32_MAX) return NULL;
    MultiConfiguration mc = malloc(sizeof(_MultiConfiguration));
    OperatorMappings   om = malloc(sizeof(_OperatorMappings));
    mc->npar = npar;
    mc->norb = norb;
    mc->dim = (uint32_t) dim;
    mc->subspaces_dim = get_subspaces_dim(npar, norb);
    mc->hash_table = malloc(sizeof(uint16_t) * dim * norb);
    orc_hash_table(npar, norb, mc->hash_table);
    om->map = malloc(sizeof(uint32_t) * dim * M2);
    orc_single_jump_map(npar, norb, om->map);
    uint64_t* st = malloc(sizeof(uint64_t) * dim);
    om->maptt = malloc(sizeof(uint32_t) * (tt > 0 ? tt * M2 : 1));
    orc_double_diffjump_map(npar, norb, st, om->maptt);
    om->stridett = malloc(sizeof(uint32_t) * dim);
    for (uint64_t i = 0; i < dim; i++) om->stridett[i] = (uint32_t) st[i];
    om->mapot = malloc(sizeof(uint32_t) * (ot > 0 ? ot * M2 : 1));
    orc_double_equaljump_map(npar, norb, st, om->mapot);
    om->strideot = malloc(sizeof(uint32_t) * dim);
    for (uint64_t i = 0; i < dim; i++) om->strideot[i] = (uint32_t) st[i];
    free(st);
    mc->op_maps = om;
    return mc;
}

/* get_orbital_workspace (types_definition.c:204-245) with set_expdvr_mat
 * only for DVR jobs */
static OrbitalWorkspace
refset_orbital_workspace(OrbitalEquation eq, OrbDerivative der)
{
    const uint16_t   G = eq->grid_size, M = eq->norb;
    OrbitalWorkspace w = malloc(sizeof(_OrbitalWorkspace));
    w->norb = M;
    w->grid_size = G;
    w->impr_ortho = FALSE;
    w->orb_der_method = der;
    w->dvr_mat = get_dcomplex_array((uint32_t) G * G);
    w->cn_upper = get_dcomplex_array(G);
    w->cn_lower = get_dcomplex_array(G);
    w->cn_mid = get_dcomplex_array(G);
    w->orb_work1 = get_dcomplex_matrix(M, G);
    w->orb_work2 = get_dcomplex_matrix(M, G);
    const double scale = 1.0 / sqrt((double) G - 1);
    DftiCreateDescriptor(&w->fft_desc, DFTI_DOUBLE, DFTI_COMPLEX, 1, G - 1);
    DftiSetValue(w->fft_desc, DFTI_FORWARD_SCALE, scale);
    DftiSetValue(w->fft_desc, DFTI_BACKWARD_SCALE, scale);
    DftiCommitDescriptor(w->fft_desc);
    w->extern_work = (void*) get_cplx_rungekutta_ws((uint32_t) G * M);
    w->fft_freq = get_double_array(G - 1);
    w->fft_hder_exp = get_dcomplex_array(G - 1);
    set_cn_tridiagonal(eq, w->cn_upper, w->cn_lower, w->cn_mid);
    set_fft_freq(G - 1, eq->dx, w->fft_freq);
    set_hder_fftexp(eq, w->fft_hder_exp);
    if (der == DVR) set_expdvr_mat(eq, w->dvr_mat);
    return w;
}

MCTDHBDataStruct
refset_mctdhb_struct(
    int imagtime, int coef_method, int orb_method, int der_method, int rk_order,
    int lanczos_iter, uint16_t npar, uint16_t norb, int periodic, double xi, double xf,
    uint16_t grid_size, double tstep, double d2coef, double d1re, double d1im,
    const double* pot, double g)
{
    MultiConfiguration mc = refset_multiconf(npar, norb);
    if (!mc) return NULL;
    PotArgs* pa = malloc(sizeof(PotArgs) + sizeof(double) * grid_size);
    pa->npts = grid_size;
    memcpy(pa->v, pot, sizeof(double) * grid_size);
    double* ga = malloc(sizeof(double));
    *ga = g;
    const IntegratorType it = imagtime ? IMAGTIME : REALTIME;
    MCTDHBDataStruct     m = malloc(sizeof(_MCTDHBDataStruct));
    m->integ_type = it;
    m->coef_integ_method = (CoefIntegrator) coef_method;
    m->orb_integ_method = (OrbIntegrator) orb_method;
    m->orb_der_method = (OrbDerivative) der_method;
    m->rk_order = (RungeKuttaOrder) rk_order;
    char name[] = "custom";
    m->orb_eq = get_orbital_equation(
        name, norb, grid_size, periodic ? PERIODIC_BOUNDS : ZERO_BOUNDS, it, xi, xf, tstep,
        1.0, d2coef, d1re + I * d1im, pa, ga, refset_pot, refset_const);
    m->coef_workspace =
        get_coef_workspace((CoefIntegrator) coef_method, mc->dim, (uint16_t) lanczos_iter);
    m->multiconfig_space = mc;
    m->state = get_manybody_state(npar, norb, grid_size);
    m->orb_workspace = refset_orbital_workspace(m->orb_eq, (OrbDerivative) der_method);
    return m;
}

void
refset_destroy(MCTDHBDataStruct m)
{
    if (!m) return;
    void* pa = m->orb_eq->pot_extra_args;
    void* ga = m->orb_eq->inter_extra_args;
    destroy_mctdhb_struct(m);
    free(pa);
    free(ga);
}
