/* mctdhb_types.h -- public C types of the MCTDHB configurational path.
 *
 * Binary-compatible re-declaration (for interoperability) of the structs of
 * the reference library's include/mctdhb_types.h (andriati-alex/1d-mctdhb,
 * include/mctdhb_types.h:21-240): same members, same order, same types, so
 * code compiled against either header can pass these structs to
 * libmctdhb_b200.so.  Unlike the reference header it needs no MKL headers:
 * the two MKL types it names are declared here with the same layout.
 */
#ifndef MCTDHB_B200_TYPES_H
#define MCTDHB_B200_TYPES_H

#include <inttypes.h>
#include <stdint.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> dcomplex;
extern "C" {
#else
#include <complex.h>
typedef double complex dcomplex;
#endif

/* compile-time limits of the reference (mctdhb_types.h:21-35) */
#define PI 3.141592653589793
#define STR_BUFF_SIZE 128
#define MAX_GRID_SIZE 2049
#define MIN_GRID_SIZE 50
#define MAX_ORBITALS 30
#define MAX_PARTICLES 10000
#define MAX_LANCZOS_ITER 15
#define MIN_LANCZOS_ITER 2

#ifndef MKL_Complex16
typedef struct
{
    double real, imag;
} mctdhb_mkl_complex16;
#define MKL_Complex16 mctdhb_mkl_complex16
#endif
typedef void* mctdhb_dfti_handle; /* stands for MKL's DFTI_DESCRIPTOR_HANDLE */

typedef int*           Iarray;
typedef int**          Imatrix;
typedef double*        Rarray;
typedef double**       Rmatrix;
typedef dcomplex*      Carray;
typedef dcomplex**     Cmatrix; /* row-pointer matrix: rows are separate blocks */
typedef MKL_Complex16* MKLCarray;

typedef enum { FALSE = 0, TRUE = 1 } Bool;
typedef enum { IMAGTIME = 10, REALTIME = 11 } IntegratorType;
typedef enum { LANCZOS = 20, RUNGEKUTTA = 21 } CoefIntegrator;
typedef enum { FULLSTEP_RUNGEKUTTA = 30, SPLITSTEP = 31 } OrbIntegrator;
typedef enum { DVR = 300, SPECTRAL = 301, FINITEDIFF = 302 } OrbDerivative;
typedef enum { RK2 = 2, RK4 = 4, RK5 = 5 } RungeKuttaOrder;
typedef enum { ZERO_BOUNDS = 1000, PERIODIC_BOUNDS = 1001 } BoundaryCondition;

#define DEFAULT_INTEGRATION_TYPE IMAGTIME
#define DEFAULT_COEF_INTEGRATOR LANCZOS
#define DEFAULT_ORB_INTEGRATOR FULLSTEP_RUNGEKUTTA
#define DEFAULT_ORB_DERIVATIVE DVR
#define DEFAULT_RUNGEKUTTA_ORDER RK5
#define DEFAULT_BOUNDARY_CONDITION PERIODIC_BOUNDS
#define DEFAULT_LANCZOS_ITER 5

/* trap potential V(t, x) on the grid, and a time-dependent scalar g(t) */
typedef void (*single_particle_pot)(double t, uint16_t npts, double* pts,
                                    void* params, double* grid_pot);
typedef double (*time_dependent_parameter)(double t, void* params);

/* orbital equation: grid, trap, interaction, time step */
typedef struct
{
    char                     eq_name[STR_BUFF_SIZE];
    uint16_t                 norb, grid_size;
    BoundaryCondition        bounds;
    double                   t, xi, xf, dx, tstep, tend, g, d2coef;
    dcomplex                 d1coef, prop_dt, time_fac;
    Rarray                   grid_pts;
    Rarray                   pot_grid;
    void*                    pot_extra_args;
    void*                    inter_extra_args;
    single_particle_pot      pot_func;
    time_dependent_parameter inter_param;
} _OrbitalEquation;
typedef _OrbitalEquation* OrbitalEquation;

/* jump maps of the creation/annihilation operators.  In this library maptt
 * and mapot may be NULL: the GPU path ranks configurations on the fly and
 * the tables are only built where the reference's 32-bit layout holds. */
typedef struct
{
    uint32_t *map, *mapot, *maptt, *strideot, *stridett;
} _OperatorMappings;
typedef _OperatorMappings* OperatorMappings;

/* Fock space of npar bosons in norb orbitals, dim = C(npar+norb-1, norb-1) */
typedef struct
{
    uint16_t         npar, norb;
    uint32_t         dim;
    uint16_t*        hash_table;    /* dim x norb occupations, row-major */
    uint32_t*        subspaces_dim; /* (npar+1) x (norb+1) */
    OperatorMappings op_maps;
} _MultiConfiguration;
typedef _MultiConfiguration* MultiConfiguration;

/* many-body state: coefficients, orbitals and their matrices */
typedef struct
{
    uint16_t npar, norb, grid_size;
    uint32_t space_dim;
    Carray   coef, hint, tb_denmat;
    Cmatrix  hob, orbitals, ob_denmat, inv_ob_denmat;
} _ManyBodyState;
typedef _ManyBodyState* ManyBodyState;

typedef struct
{
    uint16_t iter;
    uint32_t space_dim;
    Cmatrix  lanczos_vectors;
    Carray   decomp_diag, decomp_offd, coef_lspace, transform, hc, reortho;
    Rarray   lapack_diag, lapack_offd, lapack_eigvec;
} _WorkspaceLanczos;
typedef _WorkspaceLanczos* WorkspaceLanczos;

typedef struct
{
    uint16_t           norb, grid_size;
    OrbDerivative      orb_der_method;
    Bool               impr_ortho;
    Carray             dvr_mat;
    Carray             cn_upper, cn_lower, cn_mid, cn_rhs;
    Cmatrix            orb_work1, orb_work2;
    void*              extern_work;
    mctdhb_dfti_handle fft_desc;
    Rarray             fft_freq;
    Carray             fft_hder_exp;
} _OrbitalWorkspace;
typedef _OrbitalWorkspace* OrbitalWorkspace;

typedef struct
{
    WorkspaceLanczos lan_work;
    void*            extern_work;
} _CoefWorkspace;
typedef _CoefWorkspace* CoefWorkspace;

typedef struct
{
    IntegratorType     integ_type;
    CoefIntegrator     coef_integ_method;
    OrbIntegrator      orb_integ_method;
    OrbDerivative      orb_der_method;
    RungeKuttaOrder    rk_order;
    MultiConfiguration multiconfig_space;
    OrbitalEquation    orb_eq;
    CoefWorkspace      coef_workspace;
    OrbitalWorkspace   orb_workspace;
    ManyBodyState      state;
} _MCTDHBDataStruct;
typedef _MCTDHBDataStruct* MCTDHBDataStruct;

#ifdef __cplusplus
}
#endif
#endif
