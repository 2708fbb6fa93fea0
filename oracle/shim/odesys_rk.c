/* Named explicit Runge-Kutta schemes standing in for odelib (see odesys.h).
 * Test infrastructure for the reference oracle only. */
#include "odesys.h"
#include <stdio.h>
#include <stdlib.h>

ComplexWorkspaceRK
get_cplx_rungekutta_ws(uint32_t n)
{
    ComplexWorkspaceRK ws = malloc(sizeof(_ComplexWorkspaceRK));
    if (ws == NULL) abort();
    ws->system_size = n;
    ws->k1 = malloc(n * sizeof(double complex));
    ws->k2 = malloc(n * sizeof(double complex));
    ws->k3 = malloc(n * sizeof(double complex));
    ws->k4 = malloc(n * sizeof(double complex));
    ws->k5 = malloc(n * sizeof(double complex));
    ws->k6 = malloc(n * sizeof(double complex));
    ws->work = malloc(n * sizeof(double complex));
    return ws;
}

void
destroy_cplx_rungekutta_ws(ComplexWorkspaceRK ws)
{
    if (ws == NULL) return;
    free(ws->k1);
    free(ws->k2);
    free(ws->k3);
    free(ws->k4);
    free(ws->k5);
    free(ws->k6);
    free(ws->work);
    free(ws);
}

static void
eval(cplx_odesys_der f, void* args, uint32_t n, double t, double complex* y,
     double complex* out)
{
    _ComplexODEInputParameters p;
    p.system_size = n;
    p.t = t;
    p.y = y;
    p.extra_args = args;
    f(&p, out);
}

/* Heun: k1 = f(y); k2 = f(y + dt k1); y' = y + dt/2 (k1 + k2) */
void
cplx_rungekutta2(double dt, double t, cplx_odesys_der f, void* args,
                 ComplexWorkspaceRK ws, double complex* y, double complex* yn)
{
    uint32_t n = ws->system_size;
    eval(f, args, n, t, y, ws->k1);
    for (uint32_t i = 0; i < n; i++) ws->work[i] = y[i] + dt * ws->k1[i];
    eval(f, args, n, t + dt, ws->work, ws->k2);
    for (uint32_t i = 0; i < n; i++)
        yn[i] = y[i] + 0.5 * dt * (ws->k1[i] + ws->k2[i]);
}

/* Classical RK4 */
void
cplx_rungekutta4(double dt, double t, cplx_odesys_der f, void* args,
                 ComplexWorkspaceRK ws, double complex* y, double complex* yn)
{
    uint32_t n = ws->system_size;
    eval(f, args, n, t, y, ws->k1);
    for (uint32_t i = 0; i < n; i++) ws->work[i] = y[i] + 0.5 * dt * ws->k1[i];
    eval(f, args, n, t + 0.5 * dt, ws->work, ws->k2);
    for (uint32_t i = 0; i < n; i++) ws->work[i] = y[i] + 0.5 * dt * ws->k2[i];
    eval(f, args, n, t + 0.5 * dt, ws->work, ws->k3);
    for (uint32_t i = 0; i < n; i++) ws->work[i] = y[i] + dt * ws->k3[i];
    eval(f, args, n, t + dt, ws->work, ws->k4);
    for (uint32_t i = 0; i < n; i++)
        yn[i] = y[i] + dt / 6.0 *
                           (ws->k1[i] + 2.0 * ws->k2[i] + 2.0 * ws->k3[i] +
                            ws->k4[i]);
}

/* Butcher's six-stage fifth-order method:
 *   c = 0, 1/4, 1/4, 1/2, 3/4, 1
 *   a21 = 1/4
 *   a31 = 1/8,  a32 = 1/8
 *   a41 = 0,    a42 = -1/2, a43 = 1
 *   a51 = 3/16, a52 = 0,    a53 = 0,     a54 = 9/16
 *   a61 = -3/7, a62 = 2/7,  a63 = 12/7,  a64 = -12/7, a65 = 8/7
 *   b   = 7/90, 0, 32/90, 12/90, 32/90, 7/90 */
void
cplx_rungekutta5(double dt, double t, cplx_odesys_der f, void* args,
                 ComplexWorkspaceRK ws, double complex* y, double complex* yn)
{
    uint32_t        n = ws->system_size;
    double complex *k1 = ws->k1, *k2 = ws->k2, *k3 = ws->k3, *k4 = ws->k4,
                   *k5 = ws->k5, *k6 = ws->k6, *w = ws->work;
    eval(f, args, n, t, y, k1);
    for (uint32_t i = 0; i < n; i++) w[i] = y[i] + dt * (0.25 * k1[i]);
    eval(f, args, n, t + 0.25 * dt, w, k2);
    for (uint32_t i = 0; i < n; i++)
        w[i] = y[i] + dt * (0.125 * k1[i] + 0.125 * k2[i]);
    eval(f, args, n, t + 0.25 * dt, w, k3);
    for (uint32_t i = 0; i < n; i++) w[i] = y[i] + dt * (-0.5 * k2[i] + k3[i]);
    eval(f, args, n, t + 0.5 * dt, w, k4);
    for (uint32_t i = 0; i < n; i++)
        w[i] = y[i] + dt * ((3.0 / 16.0) * k1[i] + (9.0 / 16.0) * k4[i]);
    eval(f, args, n, t + 0.75 * dt, w, k5);
    for (uint32_t i = 0; i < n; i++)
        w[i] = y[i] + dt * ((-3.0 / 7.0) * k1[i] + (2.0 / 7.0) * k2[i] +
                            (12.0 / 7.0) * k3[i] - (12.0 / 7.0) * k4[i] +
                            (8.0 / 7.0) * k5[i]);
    eval(f, args, n, t + dt, w, k6);
    for (uint32_t i = 0; i < n; i++)
        yn[i] = y[i] + dt * ((7.0 / 90.0) * k1[i] + (32.0 / 90.0) * k3[i] +
                             (12.0 / 90.0) * k4[i] + (32.0 / 90.0) * k5[i] +
                             (7.0 / 90.0) * k6[i]);
}
