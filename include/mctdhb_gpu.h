/* mctdhb_gpu.h -- C ABI of libmctdhb_b200.so.
 *
 * Part 1 re-exports the reference's own entry points for the configurational
 * path under the same names and signatures (host pointers, reference struct
 * layout from mctdhb_types.h), so a program linked against the reference's
 * libmctdhb can link against this library instead.  Each declaration cites
 * the reference declaration it replaces (paths relative to the reference
 * project root, andriati-alex/1d-mctdhb).
 *
 * Differences of behaviour, all deliberate:
 *   - no exit(): failures are recorded and readable with
 *     mctdhb_gpu_last_error(); functions returning pointers return NULL,
 *     `lanczos` returns -1, void functions leave outputs untouched;
 *   - the index tables of a MultiConfiguration are optional: the GPU path
 *     ranks configurations on the fly, and get_multiconf_struct only builds
 *     the double-jump tables when they fit the reference's 32-bit layout
 *     (it leaves maptt / mapot and their strides NULL otherwise, where the
 *     reference would exit);
 *   - propagate_coef_sil leaves the Lanczos vectors on the device: the
 *     WorkspaceLanczos vectors are not written back (decomposition
 *     coefficients are).
 *
 * Part 2 is a device-resident API: Fock-space handles and operations on
 * device pointers with an explicit CUDA stream (passed as void*), used for
 * throughput work where coefficients, orbitals and matrices stay in HBM.
 *
 * Part 3 is the batched engine: many independent systems of uneven size
 * resident in one HBM arena, admitted by footprint and advanced together.
 */
#ifndef MCTDHB_B200_GPU_H
#define MCTDHB_B200_GPU_H

#include "mctdhb_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* errors                                                                  */
/* ---------------------------------------------------------------------- */
/* Message of the last failure on the calling thread ("" if none). */
const char* mctdhb_gpu_last_error(void);
void        mctdhb_gpu_clear_error(void);

/* ---------------------------------------------------------------------- */
/* Part 1: drop-in replacements (host memory)                              */
/* ---------------------------------------------------------------------- */
/* include/configurational/space.h:23 (space.c:85) */
uint32_t space_dimension(uint16_t npar, uint16_t norb);
/* space.h:37 (space.c:120) -- malloc'd, caller frees */
uint32_t* get_subspaces_dim(uint16_t npar, uint16_t norb);
/* space.h:54 (space.c:138) */
void set_config(uint32_t hash_i, uint16_t npar, uint16_t norb, uint16_t* conf);
/* space.h:71 (space.c:159) */
uint32_t hash_index(uint16_t npar, uint16_t norb, uint32_t* subsdim, uint16_t* conf);
/* space.h:41 (space.c:181) -- built on the GPU, malloc'd */
uint16_t* get_hash_table(uint16_t npar, uint16_t norb);
/* space.h:88 (space.c:202) -- built on the GPU, malloc'd */
uint32_t* get_single_jump_map(uint16_t npar, uint16_t norb, uint32_t* subsdim,
                              uint16_t* hash_table);
/* space.h:149 (space.c:297) -- strides: dim entries; NULL when the table
 * exceeds 32-bit indexing (the reference exits there) */
uint32_t* get_double_diffjump_map(uint16_t npar, uint16_t norb, uint32_t* subsdim,
                                  uint16_t* hash_table, uint32_t* strides);
/* space.h:186 (space.c:399) */
uint32_t* get_double_equaljump_map(uint16_t npar, uint16_t norb, uint32_t* subsdim,
                                   uint16_t* hash_table, uint32_t* strides);
/* include/assistant/types_definition.h:43 (types_definition.c:111) */
MultiConfiguration get_multiconf_struct(uint16_t npar, uint16_t norb);
/* types_definition.h:98 (types_definition.c:348) */
void destroy_multiconf_struct(MultiConfiguration multiconf);

/* include/configurational/hamiltonian.h:8 (hamiltonian.c:7) */
void apply_hamiltonian(MultiConfiguration multiconf, Carray coef, Cmatrix hob, Carray hint,
                       Carray hcoef);
/* include/configurational/density_matrices.h:8 (density_matrices.c:9) */
void set_onebody_dm(MultiConfiguration multiconf, Carray coef, Cmatrix rho);
/* density_matrices.h:12 (density_matrices.c:55) */
void set_twobody_dm(MultiConfiguration multiconf, Carray coef, Carray rho);

/* include/linalg/multiconfig_lanczos.h:32 (multiconfig_lanczos.c:12) */
int lanczos(MultiConfiguration multiconf, Cmatrix Ho, Carray Hint, int lm, Carray diag,
            Carray offdiag, Cmatrix lvec);
/* multiconfig_lanczos.h:58 (multiconfig_lanczos.c:93) */
double lowest_state_lanczos(uint16_t niter, MultiConfiguration multiconf, Cmatrix Ho,
                            Carray Hint, Carray C);
/* include/integrator/coefficients_integration.h:26 (coefficients_integration.c:59) */
void propagate_coef_sil(MCTDHBDataStruct mctdhb, Carray cnext);

/* include/integrator/synchronize.h:49 (synchronize.c:42): rho1, rho2 on the
 * GPU in one pass; regularisation and rho1^{-1} (M x M) on the host */
void sync_density_matrices(MultiConfiguration mc_space, ManyBodyState psi);
/* synchronize.h:37 (synchronize.c:12), name as spelled by the reference */
void set_regulatization_factor(double reg_fac);
/* synchronize.h:41 (synchronize.c:28) */
double get_current_regularization_factor(void);

/* include/function_tools/orbital_matrices.h:25 (orbital_matrices.c:22):
 * h_kl on the GPU (finite-difference derivative, Simpson weights) */
void set_orbital_hob(OrbitalEquation eq_desc, uint16_t norb, Cmatrix orb, Cmatrix hob);
/* orbital_matrices.h:30 (orbital_matrices.c:73): g_ksql on the GPU, one
 * complex (M^2 x G)(G x M^2) contraction on the FP64 tensor cores */
void set_orbital_hint(OrbitalEquation eq_desc, uint16_t norb, Cmatrix orb, Carray hint);
/* include/integrator/synchronize.h:45 (synchronize.c:35) */
void sync_orbital_matrices(OrbitalEquation eq_desc, ManyBodyState psi);
/* include/integrator/driver.h:67 (driver.c:159): one full step on the GPU.
 * Supported integrator settings (every method of the reference):
 *   orbitals      FULLSTEP_RUNGEKUTTA (RK2 / RK4 / RK5 as the named tableaux
 *                 Heun, classical RK4 and Butcher RK5) or SPLITSTEP
 *                 (orbital_integration.c:352-434: Crank-Nicolson or FFT
 *                 exponential half steps around a Runge-Kutta step of the
 *                 nonlinear part);
 *   derivatives   DVR (the reference's default), SPECTRAL or FINITEDIFF;
 *   coefficients  LANCZOS (needs coef_workspace->lan_work) or RUNGEKUTTA
 *                 (coefficients_integration.c:29-57; order 2 runs the RK5
 *                 tableau, as the reference's switch does);
 *   projector     the simple one, or the robust one when
 *                 orb_workspace->impr_ortho is set.
 * Any other orbital or coefficient method is reported as an error.
 * orb_works receives the orbitals after the orbital step, coef_works the
 * coefficient combination before the imaginary-time renormalisation. */
void mctdhb_propagate_step(MCTDHBDataStruct mctdhb, Carray orb_works, Carray coef_works,
                           uint32_t curr_step);

/* include/assistant/integrator_monitor.h:53 (integrator_monitor.c:56) */
dcomplex total_energy(ManyBodyState psi);
/* integrator_monitor.h:26 (integrator_monitor.c:10) */
double eig_residual(MultiConfiguration multiconf, Carray c, Cmatrix hob, Carray hint, double e);

/* ---------------------------------------------------------------------- */
/* Part 2: device-resident API                                             */
/* ---------------------------------------------------------------------- */
/* Layouts: coefficients are complex128 (interleaved re, im) of length dim;
 * hob is M x M row-major; hint and rho2 are M^4 with element (a,b,c,d) at
 * a + b M + c M^2 + d M^3 (the reference's layout); rho1 is M x M
 * row-major.  `stream` is a cudaStream_t (NULL = legacy default stream).
 * All functions return 0 on success and -1 on failure. */
typedef struct mctdhb_space_s* mctdhb_space;

int      mctdhb_space_create(uint16_t npar, uint16_t norb, mctdhb_space* out);
void     mctdhb_space_destroy(mctdhb_space sp);
uint32_t mctdhb_space_dim(mctdhb_space sp);

/* Pack h_kl and g_ksql into the coefficient table used by H.C (call after
 * each change of the orbital matrices). */
int mctdhb_dev_set_matrices(mctdhb_space sp, const void* d_hob, const void* d_hint,
                            void* stream);
/* HC = H C with the matrices of the last mctdhb_dev_set_matrices. */
int mctdhb_dev_apply_hamiltonian(mctdhb_space sp, const void* d_coef, void* d_hc,
                                 void* stream);
/* rho1 and rho2 of C in one pass. */
int mctdhb_dev_density_matrices(mctdhb_space sp, const void* d_coef, void* d_rho1,
                                void* d_rho2, void* stream);
/* One short-iterative-Lanczos step of C in place with `lanczos_iter`
 * vectors (2..15 as in the reference, up to 64 accepted); real time when
 * imagtime == 0, imaginary time (and renormalisation) otherwise. */
int mctdhb_dev_sil_step(mctdhb_space sp, void* d_coef, int lanczos_iter, double dt,
                        int imagtime, void* stream);
/* One configurational step -- the SIL step of C followed by rho1 and rho2
 * of the new C -- captured once into a CUDA graph on fixed device buffers
 * and replayed with one launch.  The matrices are read at replay time, so
 * mctdhb_dev_set_matrices between replays takes effect. */
typedef struct mctdhb_step_s* mctdhb_step;
int  mctdhb_step_create(mctdhb_space sp, void* d_coef, void* d_rho1, void* d_rho2,
                        int lanczos_iter, double dt, int imagtime, mctdhb_step* out);
int  mctdhb_step_launch(mctdhb_step st, void* stream);
int  mctdhb_step_kernel_count(mctdhb_step st); /* kernels launched per replay */
void mctdhb_step_destroy(mctdhb_step st);

/* A whole MCTDHB system resident on the device: orbitals (norb x grid),
 * coefficients, h, g, rho1, rho2, rho1^{-1}.  One step (driver.c:159-201:
 * orbital Runge-Kutta step, Gram-Schmidt in imaginary time, h and g of the
 * new orbitals, SIL step of the coefficients, density matrices, regularised
 * rho1^{-1}) is two captured CUDA graphs replayed per step.  Trap and
 * interaction are read from device memory at replay time: set them between
 * steps to follow time-dependent parameters.  Host buffers below are
 * complex128 row-major (orbitals norb x grid). */
typedef struct mctdhb_solver_s* mctdhb_solver;
int  mctdhb_solver_create(uint16_t npar, uint16_t norb, uint16_t grid_size, double xi, double xf,
                          double d2coef, double d1coef_re, double d1coef_im, int periodic,
                          int imagtime, int rk_order, int lanczos_iter, double dt,
                          mctdhb_solver* out);
void mctdhb_solver_destroy(mctdhb_solver s);
int  mctdhb_solver_set_potential(mctdhb_solver s, const double* pot); /* grid values */
int  mctdhb_solver_set_interaction(mctdhb_solver s, double g);
int  mctdhb_solver_set_regularization(mctdhb_solver s, double reg_fac);
/* initial orbitals + coefficients, then rho1, rho2, rho1^{-1}, h, g */
int  mctdhb_solver_set_state(mctdhb_solver s, const void* orb, const void* coef);
int  mctdhb_solver_step(mctdhb_solver s, int nsteps, void* stream);
/* one half of a step (mctdhb_propagate_step, driver.c:159-201): phase 0
 * advances the orbitals with the current trap and interaction, phase 1
 * forms h and g of the new orbitals and runs the SIL step and the
 * densities; a caller that follows time-dependent parameters sets the trap
 * and interaction of the new time in between (sync_equation_params,
 * synchronize.c:59-68) */
int  mctdhb_solver_step_phase(mctdhb_solver s, int phase, void* stream);
int  mctdhb_solver_kernel_count(mctdhb_solver s); /* kernels per step */
int  mctdhb_solver_get(mctdhb_solver s, void* orb, void* coef, void* hob, void* hint, void* rho1,
                       void* rho2, void* rinv);
int  mctdhb_solver_put(mctdhb_solver s, const void* orb, const void* coef, const void* rho2,
                       const void* rinv);
int  mctdhb_solver_energy(mctdhb_solver s, double* e_re_im); /* Tr(rho1 h) + rho2 g / 2 */
/* Monitor of the reference's integration_driver (src/integrator/driver.c:46-96,
 * 296-306), on the device-resident state:
 *   set_orthogonality  0: simple projector, 1: robust projector with the
 *                      inverse overlap matrix (impr_ortho,
 *                      src/integrator/orbital_integration.c:22-131)
 *   overlap_residual   sum_{k<l} |<f_k|f_l>| / M (overlap_residual,
 *                      src/assistant/integrator_monitor.c:31-42)
 *   eig_residual       max_i |e c_i - (H c)_i| / N (eig_residual,
 *                      src/assistant/integrator_monitor.c:9-28)
 *   lowest_state       coefficients <- lowest Lanczos eigenvector in the
 *                      current orbitals (lowest_state_lanczos,
 *                      include/linalg/multiconfig_lanczos.h); densities kept */
int  mctdhb_solver_set_orthogonality(mctdhb_solver s, int robust);
/* Derivative method of the orbital equation's linear part, as the
 * reference's orb_der_method (src/integrator/orbital_integration.c:137-176):
 * 302 FINITEDIFF (default), 300 DVR (the matrix of
 * src/integrator/split_linear_orbitals.c:83-166), 301 SPECTRAL (:257-287).
 * DVR and SPECTRAL need periodic boundaries and at most 8192 grid points. */
int  mctdhb_solver_set_derivative(mctdhb_solver s, int der_method);
/* Coefficient integrator, as the reference's coef_integ_method
 * (src/integrator/driver.c:190-198): 20 LANCZOS (default), 21 RUNGEKUTTA
 * (src/integrator/coefficients_integration.c:29-57, the solver's order;
 * order 2 takes the RK5 tableau as the reference does). */
int  mctdhb_solver_set_coef_method(mctdhb_solver s, int coef_method);
/* Orbital integrator, as the reference's orb_integ_method
 * (src/integrator/driver.c:165-173): 30 FULLSTEP_RUNGEKUTTA (default),
 * 31 SPLITSTEP (src/integrator/orbital_integration.c:352-434). */
int  mctdhb_solver_set_orb_method(mctdhb_solver s, int orb_method);
int  mctdhb_solver_overlap_residual(mctdhb_solver s, double* res);
int  mctdhb_solver_eig_residual(mctdhb_solver s, double e, double* res);
int  mctdhb_solver_lowest_state(mctdhb_solver s, int niter, double* e);
/* Steps on the device until the imaginary-time energy rule of the
 * reference's driver (driver.c:47-67: |E/N - E_prev/N| < energy_tol *
 * E_prev/N, checked every check_every steps; check_every 0 or real time: no
 * rule) or max_steps steps: one launch of a CUDA graph whose conditional
 * WHILE node repeats the step and a kernel evaluates the rule, so no step
 * waits for the host (the reference's loop, driver.c:248-285, checks on the
 * host).  Asynchronous on `stream`; needs norb >= 2.  No counterpart in
 * the reference as one call. */
int  mctdhb_solver_relax(mctdhb_solver s, uint32_t max_steps, double energy_tol,
                         int check_every, void* stream);
/* steps done by the last mctdhb_solver_relax and whether the energy rule
 * stopped it (synchronises with it) */
int  mctdhb_solver_relax_result(mctdhb_solver s, uint32_t* steps, int* converged);
/* 1 when the solver's last step, phase or relaxation launch has finished
 * on the device, 0 while it runs, -1 on error (does not block) */
int  mctdhb_solver_query(mctdhb_solver s);
void*  mctdhb_solver_device_coef(mctdhb_solver s);
void*  mctdhb_solver_device_orbitals(mctdhb_solver s);
double mctdhb_solver_time(mctdhb_solver s);

/* Index tables on the device, bit-exact with the reference's: hash table
 * (dim x M uint16), single-jump map (M^2 dim uint32). */
int mctdhb_dev_hash_table(mctdhb_space sp, void* d_ht, void* stream);
int mctdhb_dev_single_jump_map(mctdhb_space sp, void* d_map, void* stream);
/* Double-jump tables: chunk counts first (total chunks to *n_chunks, host),
 * then the table (n_chunks M^2 uint32) with 64-bit strides (dim uint64,
 * in units of table entries).  diff = 1: two different orbitals
 * (maptt/stridett), diff = 0: one orbital twice (mapot/strideot). */
int mctdhb_dev_double_jump_chunks(mctdhb_space sp, int diff, uint64_t* n_chunks);
int mctdhb_dev_double_jump_map(mctdhb_space sp, int diff, void* d_strides, void* d_map,
                               void* stream);

/* ---------------------------------------------------------------------- */
/* Part 3: batched engine -- many independent systems on one GPU          */
/* ---------------------------------------------------------------------- */
/* The reference integrates one system per process (driver.c:205-330; its
 * globals driver.c:15-19 make it single-instance).  These calls have no
 * counterpart there: each admitted job is one such integration (the step of
 * mctdhb_propagate_step, driver.c:159-201, with FULLSTEP_RUNGEKUTTA or
 * SPLITSTEP orbitals, FINITEDIFF, DVR or SPECTRAL derivatives and LANCZOS
 * coefficients), and all running jobs advance together, one CUDA graph launch
 * per step of the whole batch.  A job stops on the device after max_steps
 * steps or, in imaginary time, by the reference's energy rule checked every
 * check_every steps (driver.c:47-67 without the eigen-residual test):
 * |E/N - E_prev/N| < energy_tol * E_prev/N.  A job's results do not depend
 * on the other jobs of the batch (bit for bit). */
typedef struct {
    uint16_t npar, norb;        /* 2 <= norb <= 8 */
    int      grid_size;         /* 5 .. 4096 points on [xi, xf] */
    double   xi, xf;
    double   d2coef;            /* coefficient of d2/dx2 (-1/2 for the standard equation) */
    double   d1coef_re, d1coef_im;
    int      periodic;
    int      imagtime;
    int      rk_order;          /* 2, 4 or 5 */
    double   dt;
    double   g;                 /* contact interaction */
    uint32_t max_steps;
    double   energy_tol;        /* imaginary-time stop rule; 0 never stops early */
    int      check_every;       /* stop-rule period in steps (monitor rate); 0: never */
    double   reg_fac;           /* rho1 regularisation factor; 0: 1e-9 */
    const double* pot;          /* grid_size trap values (host) */
    const void*   orbitals;     /* norb x grid_size complex128, row-major (host) */
    const void*   coef;         /* space_dimension(npar, norb) complex128 (host) */
    int      der_method;        /* linear part: 0 or 302 finite differences, 300 DVR,
                                 * 301 spectral (periodic grids only) */
    /* the reference driver's monitor (driver.c:47-96), every check_every
     * steps: */
    double   eig_tol;           /* imaginary time: the energy rule also needs the
                                 * eigen residual max_i |E C_i - (H C)_i| / N
                                 * below eig_tol (driver.c:47-67; the reference's
                                 * default 1e-6); 0: the energy rule alone */
    double   ortho_tol;         /* real time: overlap residual (integrator_monitor.c:31)
                                 * above which the robust projector is switched on
                                 * (driver.c:69-96); 0: the reference's 1e-8.  Above
                                 * 1e-3 (REALTIME_OVERLAP_RESIDUE_TOL) the job stops
                                 * with state 3 (the reference exits) */
    int      impr_ortho;        /* 1: the robust projector from the first step
                                 * (orbital_integration.c:22-92) */
    int      orb_method;        /* 0 or 30 FULLSTEP_RUNGEKUTTA, 31 SPLITSTEP
                                 * (orbital_integration.c:352-434: exact linear half
                                 * steps -- Crank-Nicolson for finite differences, the
                                 * FFT exponential for DVR / spectral on periodic
                                 * grids -- around RK of the nonlinear part) */
} mctdhb_job;

typedef struct mctdhb_batch_s* mctdhb_batch;
/* arena_bytes of HBM reserved once for the jobs' state; every job uses
 * lanczos_iter (2..16) Krylov vectors per step */
int    mctdhb_batch_create(int max_slots, size_t arena_bytes, int lanczos_iter,
                           mctdhb_batch* out);
void   mctdhb_batch_destroy(mctdhb_batch b);
/* exact arena bytes one job occupies (0 and an error for an invalid job) */
size_t mctdhb_batch_job_bytes(const mctdhb_job* job, int lanczos_iter);
/* largest free arena range: a job fits when its bytes are at most this */
size_t mctdhb_batch_free_bytes(mctdhb_batch b);
/* 0: admitted into *slot (state uploaded, densities, h, g and energy set up);
 * 1: no free slot or arena range now (nothing changed); -1: error */
int    mctdhb_batch_admit(mctdhb_batch b, const mctdhb_job* job, int* slot);
/* enqueue nsteps steps of every running job (asynchronous) */
int    mctdhb_batch_step(mctdhb_batch b, int nsteps);
int    mctdhb_batch_sync(mctdhb_batch b);
/* per slot (arrays of max_slots, each may be NULL): state 0 empty,
 * 1 running, 2 stopped, 3 aborted (real time: overlap residual above 1e-3);
 * steps done; current energy.  Returns the number of running jobs
 * (synchronises). */
int    mctdhb_batch_poll(mctdhb_batch b, int* state, uint32_t* steps, double* energy);
/* a job's orbitals, coefficients, rho1, rho2 (host, each may be NULL),
 * energy, steps and whether the energy rule stopped it */
int    mctdhb_batch_fetch(mctdhb_batch b, int slot, void* orbitals, void* coef, void* rho1,
                          void* rho2, double* energy, uint32_t* steps, int* converged);
/* frees the slot and its arena range */
int    mctdhb_batch_release(mctdhb_batch b, int slot);
/* the monitor of a job (driver.c:47-96): the orbitals' overlap residual at
 * its last step (real time), the eigen residual at its last evaluation
 * (imaginary time with eig_tol set; -1 before the first), and in *robust
 * bit 0 the robust projector on, bit 1 a singular overlap matrix met by it */
int    mctdhb_batch_monitor(mctdhb_batch b, int slot, double* overlap_res, double* eig_res,
                            int* robust);
/* the final diagonalisation of driver.c:295-316 for a stopped job: its
 * coefficients become the lowest eigenvector of H in its orbitals after
 * niter Lanczos iterations (0: min(nc / 2, 50), none below 4
 * configurations, as the reference's get_appropriate_lanczos_iterations);
 * *energy is the Lanczos energy.  The densities are kept, as there.  The
 * reference runs it when an imaginary-time run ends at its final time
 * without converging. */
int    mctdhb_batch_lowest_state(mctdhb_batch b, int slot, int niter, double* energy);
int    mctdhb_batch_kernel_count(mctdhb_batch b); /* kernels per step graph */
/* The launch variant of the batched pair contraction for the jobs with
 * norb orbitals: picked by the autotuner on the running jobs when the step
 * graph is captured (0 the default tile, 2 the other output-tile grouping,
 * 3 the default tile handed over through mbarriers instead of a block
 * barrier per tile);
 * set_variant forces one (-1: tune again) and re-captures.  A variant
 * changes speed, never results.  No counterpart in the reference. */
int    mctdhb_batch_variant(mctdhb_batch b, int norb);
int    mctdhb_batch_set_variant(mctdhb_batch b, int norb, int variant);
/* one launch of the batched H.C of the running jobs with norb orbitals
 * (out = H C of each job, on the engine's stream): parts = 1 the pair
 * contraction, 2 the gather-back, 3 both; a measurement hook for timing the
 * dominant kernels of a step */
int    mctdhb_batch_launch_hc(mctdhb_batch b, int norb, int parts);
void*  mctdhb_batch_stream(mctdhb_batch b);       /* the engine's cudaStream_t */

/* The autotuner (no counterpart in the reference; the reference's only
 * tuning is OpenMP scheduling, hamiltonian.c:33-37): the launch variant in
 * use for a kernel and a Fock space -- "hcp_y" the pair contraction of the
 * single-system H.C, keyed by (npar, norb); "bhcp_y" the batched one, keyed
 * by (ceil(log2 rows of the group), norb); "hc" / "dens" the per-row
 * kernels -- or -1 when not tuned yet; set records a caller's choice (it
 * changes speed, never results).  MCTDHB_TUNE_CACHE names a file that keeps
 * the choices across processes. */
int    mctdhb_tune_get(const char* kernel, int npar, int norb);
int    mctdhb_tune_set(const char* kernel, int npar, int norb, int variant);

/* Throughput probe of the FP64 tensor cores (no counterpart in the
 * reference): `blocks` blocks of 256 threads, every warp running `iters`
 * rounds of four independent mma.sync m16n8k8 f64 chains, i.e.
 * blocks * 8 * iters * 4 * 2048 FLOPs; d_out receives blocks * 256 doubles.
 * The roofline denominator of the pair contraction. */
int    mctdhb_fp64_mma_probe(int blocks, int iters, void* d_out, void* stream);

/* rho1 and rho2 of C, as mctdhb_dev_density_matrices computes them (the
 * same kernels; for norb <= 8 the same bits), with no device allocation at
 * all.  This entry point has no counterpart in the
 * reference.  It is for callers that cannot let a library call cudaMalloc
 * or cudaFree: a process whose device memory is owned by its own pool
 * allocator (PyTorch's caching allocator, an arena reserved at start-up),
 * or a loop that cannot pay for the device-wide synchronisation that
 * cudaMalloc and cudaFree imply.  No mctdhb_space is needed (creating one
 * allocates): the space is named by (npar, norb), and its tables and the
 * partial sums live in one static device array of
 * MCTDHB_NOALLOC_SCRATCH_BYTES (8 MiB), held by every GPU that loads the
 * library until the process exits.  Spaces that do not fit are rejected
 * with an error: every space with norb <= 8 fits, and norb up to 25 on a
 * smaller grid.  The first call on each device looks up the array's device
 * address and sets kernel launch attributes; make it before any stream
 * capture.  All calls on one device share the array: calls that overlap on
 * the GPU (streams with no ordering between them) race and give undefined
 * results.  Each call rewrites every part of the array it reads. */
#define MCTDHB_NOALLOC_SCRATCH_BYTES 8388608u
int mctdhb_dev_density_matrices_noalloc(uint16_t npar, uint16_t norb, const void* d_coef,
                                        void* d_rho1, void* d_rho2, void* stream);

#ifdef __cplusplus
}
#endif
#endif
