/* oracle.h -- CPU restatement of the reference's configurational path.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline legs may load this library, and only as the checker or the
 * timed CPU baseline -- never as part of the GPU product path.
 *
 * Parity is pinned against the reference itself: the same entry points of
 * the reference, compiled from its own sources into _ref/libmctdhb_ref.so,
 * are compared with these at every size the reference can build its maps
 * for (tests/test_oracle_vs_reference.py), and golden vectors generated from
 * the compiled reference are committed under tests/golden/.
 *
 * Differences from the reference, by design:
 *   - jump-map lookups are replaced by on-the-fly combinatorial ranking, so
 *     sizes whose maps overflow the reference's 32-bit guards (space.c:285,
 *     space.c:384) still run;
 *   - matrices are row-major contiguous instead of row-pointer `Cmatrix`;
 *   - LAPACK dstev/zheev/zhesv are replaced by implicit-QL (tridiagonal),
 *     cyclic Jacobi (Hermitian) and Gauss-Jordan with partial pivoting.
 */
#ifndef MCTDHB_ORACLE_H
#define MCTDHB_ORACLE_H
#include <complex.h>
#include <stdint.h>

typedef double complex ocplx;

/* space.c:85-117 (64-bit, no overflow exit) */
uint64_t orc_space_dimension(int npar, int norb);
/* space.c:159-178 and space.c:138-156 */
uint64_t orc_rank(int npar, int norb, const uint16_t* occ);
void     orc_unrank(int npar, int norb, uint64_t idx, uint16_t* occ);
/* space.c:120-135 */
void orc_subspaces_dim(int npar, int norb, uint32_t* out);
/* space.c:181-199 */
void orc_hash_table(int npar, int norb, uint16_t* ht);
/* space.c:202-251 */
void orc_single_jump_map(int npar, int norb, uint32_t* map);
/* space.c:255-294 / 362-396: number of M^2 chunks of each double map */
uint64_t orc_double_diffjump_chunks(int npar, int norb);
uint64_t orc_double_equaljump_chunks(int npar, int norb);
/* space.c:297-358 / 399-451, with 64-bit strides */
void orc_double_diffjump_map(int npar, int norb, uint64_t* strides,
                             uint32_t* map);
void orc_double_equaljump_map(int npar, int norb, uint64_t* strides,
                              uint32_t* map);

/* hamiltonian.c:7-406; hob row-major M*M, hint M^4 */
void orc_apply_hamiltonian(int npar, int norb, const ocplx* coef,
                           const ocplx* hob, const ocplx* hint, ocplx* hc);
/* same, restricted to rows [row0, row1): the bounded CPU-baseline sample */
void orc_apply_hamiltonian_rows(int npar, int norb, const ocplx* coef,
                                const ocplx* hob, const ocplx* hint, ocplx* hc,
                                uint64_t row0, uint64_t row1);
/* density_matrices.c:9-52 (row-major M*M) */
void orc_onebody_dm(int npar, int norb, const ocplx* coef, ocplx* rho1);
/* density_matrices.c:55-443 */
void orc_twobody_dm(int npar, int norb, const ocplx* coef, ocplx* rho2);
void orc_twobody_dm_rows(int npar, int norb, const ocplx* coef, ocplx* rho2,
                         uint64_t row0, uint64_t row1);

/* implicit-QL eigen-decomposition of a real symmetric tridiagonal matrix
 * (replaces LAPACKE_dstev 'V', row-major eigenvectors in columns).
 * d[n] diagonal, e[n] off-diagonal (e[n-1] ignored), z[n*n] out.
 * Returns 0 on success, >0 when an eigenvalue failed to converge. */
int orc_tridiag_eig(int n, double* d, double* e, double* z);

/* multiconfig_lanczos.c:12-90.  lvec: m rows of nc (row-major); lvec[0]
 * holds the start vector.  Returns the iterations done. */
int orc_lanczos(int npar, int norb, const ocplx* hob, const ocplx* hint,
                int m, ocplx* diag, ocplx* offd, ocplx* lvec);
/* coefficients_integration.c:59-160; coef in/out; prop_dt = dt (real time)
 * or -i dt (imaginary time); imagtime renormalizes.  Returns iterations. */
int orc_sil_step(int npar, int norb, const ocplx* hob, const ocplx* hint,
                 int m, ocplx prop_dt, int imagtime, ocplx* coef,
                 ocplx* lvec_work);
/* multiconfig_lanczos.c:93-172; returns the lowest Ritz value */
double orc_lowest_state_lanczos(int npar, int norb, const ocplx* hob,
                                const ocplx* hint, int m, ocplx* coef,
                                ocplx* lvec_work);

/* integrator_monitor.c:56-88 */
ocplx orc_total_energy(int norb, const ocplx* rho1, const ocplx* rho2,
                       const ocplx* hob, const ocplx* hint);
/* integrator_monitor.c:10-28 */
double orc_eig_residual(int npar, int norb, const ocplx* coef, const ocplx* hob,
                        const ocplx* hint, double e);

/* ---- orbital side (function_tools, integrator) ---- */
/* calculus.c:9-40 */
ocplx orc_simpson(int n, double h, const ocplx* f);
/* calculus.c:288-305 (periodic 4th-order FD) */
void orc_dxfd(int n, double dx, const ocplx* f, ocplx* dfdx);
/* orbital_matrices.c:22-70; orb row-major M x G */
void orc_orbital_hob(int norb, int npts, double dx, double d2coef,
                     ocplx d1coef, const double* pot, const ocplx* orb,
                     ocplx* hob);
/* orbital_matrices.c:73-287 */
void orc_orbital_hint(int norb, int npts, double dx, double g,
                      const ocplx* orb, ocplx* hint);
/* calculus.c:171-191 */
void orc_orthonormalize(int npts, double dx, int nfun, ocplx* orb);
/* M x M Hermitian eigenvalues ascending (replaces zheev 'N'),
 * eigenvectors in columns of vec (may be NULL) */
int orc_herm_eig(int n, const ocplx* a, double* w, ocplx* vec);
/* Hermitian inverse (replaces zhesv with identity right-hand side) */
int orc_herm_inverse(int n, const ocplx* a, ocplx* inv);
/* synchronize.c:42-57 (rho1, rho2, regularization, inverse) */
void orc_sync_density_matrices(int npar, int norb, const ocplx* coef,
                               double reg_fac, ocplx* rho1, ocplx* rho2,
                               ocplx* rho1_inv);
/* orbital_integration.c:179-240 with the linear part of der = 302
 * FINITEDIFF (split_linear_orbitals.c:210-255), 300 DVR (the matrix of
 * split_linear_orbitals.c:83-166) or 301 SPECTRAL (:257-287),
 * orb_interacting_part (split_nonlinear_orbitals.c:4-61) and the simple
 * projector (:95-131), or with robust != 0 the robust projector (:22-92).
 * Returns 0, or the overlap inversion's error code. */
int orc_orbital_rhs(int norb, int npts, double dx, double d2coef,
                    ocplx d1coef, double g, int periodic, ocplx time_fac,
                    const double* pot, const ocplx* rho1_inv,
                    const ocplx* rho2, const ocplx* orb, ocplx* dodt,
                    int robust, int der);
/* one linear half step of the split-step integrator on one orbital (in
 * place): der 302 Crank-Nicolson (split_linear_orbitals.c:23-56, 289-373),
 * otherwise the FFT exponential (:57-82, 375-402); dth = prop_dt / 2 */
void orc_linear_half_step(int der, int npts, double dx, double d2coef, ocplx d1coef,
                          int periodic, ocplx dth, ocplx* f);
/* one full step of driver.c:159-201 (FULLSTEP_RUNGEKUTTA + LANCZOS, FD,
 * time-independent trap and interaction).  rk_order in {2,4,5} with the
 * named tableaux of shim/odesys.h; robust and der select the projector
 * and the linear part as in orc_orbital_rhs; coef_method 20 (SIL) or 21
 * (Runge-Kutta, coefficients_integration.c:15-57); orb_method 30 full
 * step or 31 split step (orbital_integration.c:352-434: Crank-Nicolson for
 * finite differences, the FFT exponential otherwise).  State arrays are
 * updated in place. */
void orc_propagate_step(int npar, int norb, int npts, double dx, double dt,
                        double d2coef, ocplx d1coef, double g, int periodic,
                        int imagtime, int rk_order, int lanczos_m,
                        double reg_fac, const double* pot, ocplx* orb,
                        ocplx* coef, ocplx* hob, ocplx* hint, ocplx* rho1,
                        ocplx* rho2, ocplx* rho1_inv, int robust, int der,
                        int coef_method, int orb_method);
#endif
