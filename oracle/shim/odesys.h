/* Test-infrastructure replacement for odelib (github.com/andriati-alex/odelib,
 * not vendored with the reference and pinned at no version).  It declares the
 * names the reference calls (types_definition.c:194,233,402,417,
 * coefficients_integration.c:14-57, orbital_integration.c:179,308-336) and
 * implements them with NAMED explicit Runge-Kutta schemes written from their
 * published tableaux (odesys_rk.c):
 *   cplx_rungekutta2 : Heun's method (explicit trapezoid), order 2
 *   cplx_rungekutta4 : classical Runge-Kutta, order 4
 *   cplx_rungekutta5 : Butcher's six-stage method (1964), order 5
 * The GPU orbital integrator implements the same three tableaux, so orbital
 * parity is exact in scheme; parity with odelib itself is unpinned. */
#ifndef ORACLE_SHIM_ODESYS_H
#define ORACLE_SHIM_ODESYS_H
#include <complex.h>
#include <stdint.h>

typedef struct
{
    uint32_t        system_size;
    double          t;
    double complex* y;
    void*           extra_args;
} _ComplexODEInputParameters;
typedef _ComplexODEInputParameters* ComplexODEInputParameters;

typedef void (*cplx_odesys_der)(ComplexODEInputParameters, double complex*);

typedef struct
{
    uint32_t        system_size;
    double complex *k1, *k2, *k3, *k4, *k5, *k6, *work;
} _ComplexWorkspaceRK;
typedef _ComplexWorkspaceRK* ComplexWorkspaceRK;

ComplexWorkspaceRK get_cplx_rungekutta_ws(uint32_t system_size);
void               destroy_cplx_rungekutta_ws(ComplexWorkspaceRK ws);

void cplx_rungekutta2(double dt, double t, cplx_odesys_der f, void* args,
                      ComplexWorkspaceRK ws, double complex* yinp,
                      double complex* ynext);
void cplx_rungekutta4(double dt, double t, cplx_odesys_der f, void* args,
                      ComplexWorkspaceRK ws, double complex* yinp,
                      double complex* ynext);
void cplx_rungekutta5(double dt, double t, cplx_odesys_der f, void* args,
                      ComplexWorkspaceRK ws, double complex* yinp,
                      double complex* ynext);
#endif
