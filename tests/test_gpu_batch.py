"""The batched engine (mctdhb_batch_*): many systems of uneven size advanced
by one graph launch per step.

* every job of a mixed batch against the oracle's full step (the oracle is
  pinned to the reference's own mctdhb_propagate_step);
* a job gives the same bits alone and in a mix that changes while it runs
  (other jobs admitted, stopped and released between its steps);
* stop rules: the imaginary-time energy rule of the reference's driver and
  the step limit;
* admission by footprint: a full arena refuses, a release makes room.
"""
import numpy as np
import pytest

from helpers import rand_coef, rel_err
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

XI, XF = -8.0, 8.0


def harmonic(G, xi, xf, omega=1.0):
    x = np.linspace(xi, xf, G)
    return 0.5 * omega ** 2 * x ** 2


def make_job(oracle_dim, N, M, G, imag, rk, dt, g, steps, seed, etol=0.0, check=0, der=302):
    orb, _ = hermite_orbitals(M, G, XI, XF)
    rng = np.random.default_rng(seed)
    return {"npar": N, "norb": M, "grid_size": G, "xi": XI, "xf": XF, "periodic": 1,
            "imagtime": int(imag), "rk_order": rk, "dt": dt, "g": g, "max_steps": steps,
            "energy_tol": etol, "check_every": check, "pot": harmonic(G, XI, XF),
            "orbitals": orb, "coef": rand_coef(rng, oracle_dim(N, M)), "der_method": der}


def oracle_init(oracle, N, orb, coef, dx, pot, g):
    M = orb.shape[0]
    r1, r2, ri = oracle.sync_density_matrices(N, M, coef)
    return {"orb": np.ascontiguousarray(orb.copy()), "coef": np.ascontiguousarray(coef.copy()),
            "hob": np.ascontiguousarray(oracle.orbital_hob(orb, dx, -0.5, 0.0, pot)),
            "hint": np.ascontiguousarray(oracle.orbital_hint(orb, dx, g)),
            "rho1": np.ascontiguousarray(r1), "rho2": np.ascontiguousarray(r2),
            "rinv": np.ascontiguousarray(ri)}


MIX = [  # N, M, G, imag, rk, dt, g, steps
    (4, 3, 64, True, 5, 0.01, 0.5, 5),
    (4, 3, 64, False, 5, 0.005, 0.5, 5),
    (6, 4, 96, True, 4, 0.01, 1.0, 4),
    (5, 2, 64, False, 2, 0.005, 0.3, 4),
    (8, 6, 128, False, 5, 0.005, 0.1, 3),
    (7, 5, 80, True, 5, 0.01, 0.2, 5),
    (6, 7, 96, True, 5, 0.01, 0.3, 3),
    (5, 8, 64, False, 5, 0.005, 0.2, 3),
    (6, 4, 96, True, 5, 0.005, 0.4, 4),
    (5, 3, 128, False, 4, 0.005, 0.6, 4),
]
# derivative method of the jobs (the rest: finite differences): DVR and
# spectral linear parts as the device Toeplitz sum of the orbital step
DER = {8: 300, 9: 301}


def test_batch_mix_vs_oracle(gpu, oracle):
    """each job of one mixed batch stepped to its own step limit, against the
    oracle stepped alone (Lanczos dimension 5 for all)"""
    m = 5
    b = gpu.Batch(16, 256 << 20, m)
    jobs, slots = [], []
    for i, (N, M, G, imag, rk, dt, g, steps) in enumerate(MIX):
        job = make_job(oracle.dim, N, M, G, imag, rk, dt, g, steps, 900 + i, der=DER.get(i, 302))
        jobs.append(job)
        slots.append(b.admit(job))
    assert None not in slots
    b.step(max(c[-1] for c in MIX) + 2)  # stopped jobs are skipped
    n, state, steps, _ = b.poll()
    assert n == 0
    for (N, M, G, imag, rk, dt, g, nst), job, s in zip(MIX, jobs, slots):
        assert state[s] == 2 and steps[s] == nst
        dx = (XF - XI) / (G - 1)
        st = oracle_init(oracle, N, job["orbitals"], job["coef"], dx, job["pot"], g)
        for _ in range(nst):
            oracle.propagate_step(st, N, dx, dt, -0.5, 0.0, g, True, imag, rk, m, job["pot"],
                                  der=job["der_method"])
        d = b.fetch(s)
        assert rel_err(d["orb"], st["orb"]) < 1e-10, (N, M)
        assert rel_err(d["coef"], st["coef"]) < 1e-10, (N, M)
        assert rel_err(d["rho1"], st["rho1"]) < 1e-10, (N, M)
        e_ref = oracle.total_energy(M, st["rho1"], st["rho2"], st["hob"], st["hint"])
        assert abs(d["energy"] - e_ref.real) < 1e-10 * abs(e_ref), (N, M)
        assert abs(np.linalg.norm(d["coef"]) - 1.0) < 1e-12
    assert b.kernels > 20
    b.close()


def run_alone(gpu, job, steps):
    b = gpu.Batch(4, 128 << 20, 5)
    s = b.admit(job)
    b.step(steps)
    d = b.fetch(s)
    b.close()
    return d


def test_batch_same_bits_alone_and_in_a_changing_mix(gpu, oracle):
    target = make_job(oracle.dim, 10, 4, 128, True, 5, 0.01, 0.5, 12, 31)
    alone = run_alone(gpu, target, 12)
    b = gpu.Batch(12, 512 << 20, 5)
    others = [make_job(oracle.dim, N, M, G, imag, rk, dt, g, n, 50 + i, der=DER.get(i, 302))
              for i, (N, M, G, imag, rk, dt, g, n) in enumerate(MIX)]
    # two jobs ahead of the target, so it lands in a different slot
    early = [b.admit(others[0]), b.admit(others[4])]
    s = b.admit(target)
    assert s == 2
    b.step(3)
    late = [b.admit(o) for o in others[1:4]]  # join while the target runs
    b.step(2)
    b.poll()
    b.release(early[0])  # a stopped job leaves
    b.step(4)
    late.append(b.admit(others[5]))
    late.append(b.admit(others[8]))  # a DVR job joins
    b.step(10)
    d = b.fetch(s)
    assert d["steps"] == 12
    for k in ("orb", "coef", "rho1", "rho2"):
        assert np.array_equal(d[k], alone[k]), k
    assert d["energy"] == alone["energy"]
    b.close()


def test_batch_stop_rules(gpu, oracle):
    b = gpu.Batch(4, 128 << 20, 5)
    relax = make_job(oracle.dim, 6, 3, 128, True, 5, 0.02, 0.5, 3000, 7, etol=1e-9, check=1)
    quench = make_job(oracle.dim, 6, 3, 128, False, 5, 0.005, 0.5, 17, 8)
    sr, sq = b.admit(relax), b.admit(quench)
    for _ in range(400):
        b.step(10)
        n, state, steps, energy = b.poll()
        if n == 0:
            break
    assert n == 0
    r, q = b.fetch(sr), b.fetch(sq)
    assert r["converged"] and 1 < r["steps"] < 3000
    assert not q["converged"] and q["steps"] == 17
    assert energy[sr] == r["energy"]
    b.close()


def test_batch_admission_by_footprint(gpu, oracle):
    job = make_job(oracle.dim, 20, 4, 128, True, 5, 0.01, 0.5, 5, 3)
    need = gpu.Batch.job_bytes(job, 5)
    b = gpu.Batch(8, 2 * need + need // 2, 5)
    a0, a1 = b.admit(job), b.admit(job)
    assert a0 is not None and a1 is not None
    assert b.free_bytes() < need
    assert b.admit(job) is None  # no room: refused, nothing changed
    b.release(a0)
    assert b.free_bytes() >= need
    assert b.admit(job) == a0
    b.step(5)
    n, state, steps, _ = b.poll()
    assert n == 0 and steps[a0] == 5 and steps[a1] == 5
    b.close()


SPLIT = [  # N, M, G, imag, rk, dt, g, steps, der, periodic
    (5, 3, 64, True, 5, 0.01, 0.5, 4, 302, 1),
    (6, 4, 96, False, 4, 0.005, 0.4, 3, 302, 1),
    (5, 3, 64, False, 5, 0.005, 0.3, 3, 302, 0),
    (6, 3, 64, True, 4, 0.01, 0.6, 4, 300, 1),
    (5, 5, 96, False, 5, 0.005, 0.2, 3, 301, 1),
]


def test_batch_split_step_vs_oracle(gpu, oracle):
    """split-step orbitals in the batched engine (orbital_integration.c:
    352-434): Crank-Nicolson half steps (periodic and zero bounds), the FFT
    exponential for DVR and spectral derivatives, against the oracle's split
    step, all in one batch; and the same bits alone"""
    m = 5
    b = gpu.Batch(8, 256 << 20, m)
    jobs, slots = [], []
    for i, (N, M, G, imag, rk, dt, g, steps, der, per) in enumerate(SPLIT):
        job = make_job(oracle.dim, N, M, G, imag, rk, dt, g, steps, 700 + i, der=der)
        job["periodic"], job["orb_method"] = per, 31
        jobs.append(job)
        slots.append(b.admit(job))
    assert None not in slots
    b.step(max(c[7] for c in SPLIT) + 1)
    for (N, M, G, imag, rk, dt, g, nst, der, per), job, s in zip(SPLIT, jobs, slots):
        dx = (XF - XI) / (G - 1)
        st = oracle_init(oracle, N, job["orbitals"], job["coef"], dx, job["pot"], g)
        for _ in range(nst):
            oracle.propagate_step(st, N, dx, dt, -0.5, 0.0, g, bool(per), imag, rk, m, job["pot"],
                                  der=der, orb_method=31)
        d = b.fetch(s)
        assert d["steps"] == nst
        for k in ("orb", "coef", "rho1"):
            assert rel_err(d[k], st[k]) < 1e-10, (N, M, der, per, k)
        e_ref = oracle.total_energy(M, st["rho1"], st["rho2"], st["hob"], st["hint"])
        assert abs(d["energy"] - e_ref.real) < 1e-10 * abs(e_ref)
    mixed = b.fetch(slots[3])
    b.close()
    alone = run_alone(gpu, jobs[3], SPLIT[3][7])
    for k in ("orb", "coef", "rho1", "rho2"):
        assert np.array_equal(alone[k], mixed[k]), k
