"""The reference driver's monitor in the batched engine (driver.c:47-96,
295-316), per job:

* real time: the orbitals' overlap residual (integrator_monitor.c:31-42)
  every check; above ortho_tol the robust projector (inverse overlap
  matrix, orbital_integration.c:22-92) is switched on for the following
  steps, above 1e-3 the job is stopped as aborted (the reference exits);
* a job may start with the robust projector (impr_ortho);
* imaginary time: with eig_tol set, the energy rule also needs the eigen
  residual max_i |E C_i - (H C)_i| / N below eig_tol;
* the final lowest-state diagonalisation of a stopped relaxation.

Each is checked against the oracle (pinned to the reference's own step) and
the single-system solver, and a job's monitor gives the same bits alone and
in a mix.
"""
import numpy as np
import pytest

from helpers import rand_coef, rel_err
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

XI, XF = -8.0, 8.0


def harmonic(G):
    return 0.5 * np.linspace(XI, XF, G) ** 2


def skewed(M, G, seed, amp):
    """Hermite functions plus a periodic perturbation: not orthonormal"""
    orb, dx = hermite_orbitals(M, G, XI, XF)
    rng = np.random.default_rng(seed)
    orb = orb + amp * (rng.normal(size=orb.shape) + 1j * rng.normal(size=orb.shape))
    orb[:, -1] = orb[:, 0]
    return np.ascontiguousarray(orb), dx


def job(dim, N, M, G, imag, dt, g, steps, seed, orb=None, **kw):
    if orb is None:
        orb, _ = hermite_orbitals(M, G, XI, XF)
    j = {"npar": N, "norb": M, "grid_size": G, "xi": XI, "xf": XF, "periodic": 1,
         "imagtime": int(imag), "rk_order": 5, "dt": dt, "g": g, "max_steps": steps,
         "energy_tol": 0.0, "check_every": 0, "pot": harmonic(G), "orbitals": orb,
         "coef": rand_coef(np.random.default_rng(seed), dim(N, M)), "der_method": 302}
    j.update(kw)
    return j


def oracle_init(oracle, j):
    N, M, G = j["npar"], j["norb"], j["grid_size"]
    dx = (XF - XI) / (G - 1)
    orb, coef, pot = j["orbitals"], j["coef"], j["pot"]
    r1, r2, ri = oracle.sync_density_matrices(N, M, coef)
    return {"orb": np.ascontiguousarray(orb.copy()), "coef": np.ascontiguousarray(coef.copy()),
            "hob": np.ascontiguousarray(oracle.orbital_hob(orb, dx, -0.5, 0.0, pot)),
            "hint": np.ascontiguousarray(oracle.orbital_hint(orb, dx, j["g"])),
            "rho1": np.ascontiguousarray(r1), "rho2": np.ascontiguousarray(r2),
            "rinv": np.ascontiguousarray(ri)}, dx


def overlap_residual(oracle, orb, dx):
    M = orb.shape[0]
    return sum(abs(oracle.simpson(dx, np.conj(orb[k]) * orb[l]))
               for k in range(M) for l in range(k + 1, M)) / M


def run_batch(gpu, jobs, steps, lz=5):
    b = gpu.Batch(max(4, len(jobs)), sum(gpu.Batch.job_bytes(j, lz) for j in jobs) + (64 << 20),
                  lz)
    slots = [b.admit(j) for j in jobs]
    assert None not in slots
    b.step(steps)
    return b, slots


def test_robust_from_start_vs_oracle_and_solver(gpu, oracle):
    """impr_ortho: the robust projector from the first step, real time, on
    non-orthonormal orbitals"""
    N, M, G, dt, g, steps = 6, 4, 96, 0.005, 0.6, 4
    orb, dx = skewed(M, G, 3, 0.02)
    j = job(oracle.dim, N, M, G, False, dt, g, steps, 41, orb=orb, impr_ortho=1)
    b, (s,) = run_batch(gpu, [j], steps + 1)
    d = b.fetch(s)
    mon = b.monitor(s)
    b.close()
    st, _ = oracle_init(oracle, j)
    for _ in range(steps):
        oracle.propagate_step(st, N, dx, dt, -0.5, 0.0, g, True, False, 5, 5, j["pot"],
                              robust=True)
    assert mon["robust"] and not mon["robust_failed"]
    for k in ("orb", "coef", "rho1"):
        assert rel_err(d[k], st[k]) < 1e-10, k
    # the single-system solver with its robust projector
    sv = gpu.Solver(N, M, G, XI, XF, dt, False, 5, 5)
    sv.set_orthogonality(True)
    sv.set_potential(j["pot"])
    sv.set_interaction(g)
    sv.set_state(orb, j["coef"])
    sv.step(steps)
    e = sv.get()
    sv.close()
    for k in ("orb", "coef", "rho1"):
        assert rel_err(d[k], e[k]) < 1e-10, k


def test_overlap_check_switches_robust_projector(gpu, oracle):
    """check every step with a switch threshold below the orbitals' drift:
    step 1 runs the simple projector, the check after it switches the
    robust one on for steps 2.. (driver.c:69-96)"""
    N, M, G, dt, g, steps = 6, 3, 96, 0.005, 0.6, 4
    orb, dx = skewed(M, G, 5, 1e-4)
    j = job(oracle.dim, N, M, G, False, dt, g, steps, 42, orb=orb, check_every=1,
            ortho_tol=1e-12)
    b, (s,) = run_batch(gpu, [j], steps + 1)
    d, mon = b.fetch(s), b.monitor(s)
    b.close()
    st, _ = oracle_init(oracle, j)
    for k in range(steps):
        oracle.propagate_step(st, N, dx, dt, -0.5, 0.0, g, True, False, 5, 5, j["pot"],
                              robust=k > 0)
    assert mon["robust"]
    assert abs(mon["overlap_residual"] - overlap_residual(oracle, st["orb"], dx)) < \
        1e-10 * mon["overlap_residual"]
    for k in ("orb", "coef", "rho1"):
        assert rel_err(d[k], st[k]) < 1e-10, k


def test_overlap_check_keeps_simple_projector_below_threshold(gpu, oracle):
    """orthonormal orbitals stay below the reference's 1e-8 over a few
    steps: the simple projector throughout, the same bits as with no check"""
    N, M, G, dt, g, steps = 6, 3, 96, 0.005, 0.6, 3
    j = job(oracle.dim, N, M, G, False, dt, g, steps, 43, check_every=1)
    j0 = dict(j, check_every=0)
    b, (s, s0) = run_batch(gpu, [j, j0], steps)
    d, d0, mon = b.fetch(s), b.fetch(s0), b.monitor(s)
    b.close()
    assert not mon["robust"] and 0 <= mon["overlap_residual"] < 1e-8
    for k in ("orb", "coef", "rho1"):
        assert np.array_equal(d[k], d0[k]), k


def test_overlap_above_critical_aborts_the_job_alone(gpu, oracle):
    """overlap residual above 1e-3: the job stops as aborted (state 3) after
    its first check, the other job of the batch runs on"""
    N, M, G, dt, g = 6, 3, 96, 0.005, 0.6
    orb, _ = skewed(M, G, 9, 0.05)
    bad = job(oracle.dim, N, M, G, False, dt, g, 10, 44, orb=orb, check_every=2)
    good = job(oracle.dim, N, M, G, False, dt, g, 6, 45, check_every=2)
    b, (sb, sg) = run_batch(gpu, [bad, good], 8)
    n, state, steps, _ = b.poll()
    mon = b.monitor(sb)
    b.close()
    assert state[sb] == 3 and steps[sb] == 2
    assert mon["overlap_residual"] > 1e-3
    assert state[sg] == 2 and steps[sg] == 6


def test_eigen_residual_rule(gpu, oracle):
    """imaginary time with the energy rule always met (tolerance 1): an
    unreachable eig_tol keeps the job running to its step limit with the
    residual of the state it reports; a loose one stops it at the first
    check, converged"""
    N, M, G, dt, g, steps = 8, 4, 96, 0.01, 0.5, 5
    tight = job(oracle.dim, N, M, G, True, dt, g, steps, 46, energy_tol=1.0, check_every=1,
                eig_tol=1e-300)
    loose = job(oracle.dim, N, M, G, True, dt, g, steps, 46, energy_tol=1.0, check_every=1,
                eig_tol=1e300)
    b, (st_, sl) = run_batch(gpu, [tight, loose], steps + 2)
    n, state, steps_done, energy = b.poll()
    dt_, dl = b.fetch(st_), b.fetch(sl)
    mt = b.monitor(st_)
    b.close()
    assert state[st_] == 2 and steps_done[st_] == steps and not dt_["converged"]
    assert steps_done[sl] == 1 and dl["converged"]
    # the residual of the final state, as the reference's eig_residual
    # (integrator_monitor.c:9-28) with the state's h and g and its energy
    dx = (XF - XI) / (G - 1)
    hob = oracle.orbital_hob(dt_["orb"], dx, -0.5, 0.0, tight["pot"])
    hint = oracle.orbital_hint(dt_["orb"], dx, g)
    e = dt_["energy"]
    want = oracle.eig_residual(N, M, dt_["coef"], hob, hint, e)
    assert want > 1e-8 and abs(mt["eig_residual"] - want) < 1e-9 * want


def test_lowest_state_of_a_stopped_job(gpu, oracle):
    """final diagonalisation (driver.c:295-316) of a stopped relaxation,
    against the oracle's lowest_state_lanczos on the same coefficients and
    matrices, and against the single-system solver's"""
    N, M, G, dt, g, steps, it = 8, 4, 96, 0.01, 0.5, 3, 20
    j = job(oracle.dim, N, M, G, True, dt, g, steps, 47)
    b, (s,) = run_batch(gpu, [j], steps + 1)
    d = b.fetch(s)
    e_l = b.lowest_state(s, it)
    d2 = b.fetch(s)
    b.close()
    dx = (XF - XI) / (G - 1)
    hob = oracle.orbital_hob(d["orb"], dx, -0.5, 0.0, j["pot"])
    hint = oracle.orbital_hint(d["orb"], dx, g)
    e_o, c_o = oracle.lowest_state_lanczos(N, M, hob, hint, it, d["coef"])
    assert abs(e_l - e_o) < 1e-10 * abs(e_o)
    ph = np.vdot(d2["coef"], c_o)
    ph /= abs(ph)
    assert rel_err(d2["coef"] * ph, c_o) < 1e-8
    assert np.array_equal(d2["rho1"], d["rho1"])  # densities kept, as in the reference
    sv = gpu.Solver(N, M, G, XI, XF, dt, True, 5, 5)
    sv.set_potential(j["pot"])
    sv.set_interaction(g)
    sv.set_state(j["orbitals"], j["coef"])
    sv.step(steps)
    e_s = sv.lowest_state(it)
    sv.close()
    assert abs(e_l - e_s) < 1e-10 * abs(e_s)


def test_monitor_same_bits_alone_and_in_a_mix(gpu, oracle):
    """a real-time job whose check switches the robust projector on, and an
    imaginary-time job with the eigen-residual rule: the same bits and the
    same monitor values alone and among other jobs"""
    orb, _ = skewed(3, 96, 5, 1e-4)
    rt = job(oracle.dim, 6, 3, 96, False, 0.005, 0.6, 5, 50, orb=orb, check_every=1,
             ortho_tol=1e-12)
    it = job(oracle.dim, 8, 4, 96, True, 0.01, 0.5, 5, 51, energy_tol=1.0, check_every=1,
             eig_tol=1e-300)
    others = [job(oracle.dim, 10, 5, 128, True, 0.01, 0.3, 7, 52),
              job(oracle.dim, 7, 3, 64, False, 0.005, 0.4, 7, 53, check_every=2)]
    res = []
    for mix in ([rt, it], others[:1] + [rt] + others[1:] + [it]):
        b, slots = run_batch(gpu, mix, 8)
        pos = [mix.index(rt), mix.index(it)]
        res.append([(b.fetch(slots[p]), b.monitor(slots[p])) for p in pos])
        b.close()
    for (a, ma), (c, mc) in zip(res[0], res[1]):
        for k in ("orb", "coef", "rho1", "rho2"):
            assert np.array_equal(a[k], c[k]), k
        assert ma == mc
