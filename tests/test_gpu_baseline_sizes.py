"""GPU parity at the workload sizes themselves (not only at small sizes).

* N=30, M=8 (nc = 10,295,472): the whole H.C vector against the oracle's
  rule-by-rule restatement of hamiltonian.c:7-406, and rho1 / rho2 element by
  element against density_matrices.c:9-443's restatement;
* the N=30, M=8 real-time quench as configured -- grid 1024 on [-15, 15],
  V = x^2/2 + 4 exp(-x^2/0.5), g = 0.1, Lanczos 6, dt = 0.005 -- three full
  steps of the device solver against the oracle's full step (driver.c:159-201).
  Orbitals by the split step with DVR derivatives (the reference's default
  derivative): at this grid and dt every explicit full-step Runge-Kutta
  scheme is outside its stability region (dt * lambda_max ~ 15 for finite
  differences, ~ 29 for DVR; the reference's own RK5 trajectory overflows
  within five steps), while the split step treats the kinetic part exactly;
* the largest job of the batched mix (N=60, M=6, grid 1024) and three jobs
  drawn from the mix's own seeded stream, advanced by the batched engine
  against the oracle stepped alone;
* the N=10, M=4 relaxation as configured (grid 256, 1000 steps of dt = 0.01)
  against the compiled reference itself: finite differences with RK5 (the
  configured method) and the Crank-Nicolson split step; with DVR
  derivatives (the reference's default; FFT half steps, which the compiled
  reference cannot run without MKL) against the oracle;
* N=100, M=6 (nc = 96,560,646): one full real-time step against the oracle
  (about 2 minutes of host CPU on 16 cores for the oracle's five
  rule-by-rule H.C products over 96.6 M configurations; MCTDHB_PARITY_QUICK=1
  skips the two largest cases for quick iterations).

Tolerances are those of the other parity tests: H.C, rho1, rho2 1e-12
(max-norm relative); orbitals, coefficients and energies after full steps
1e-10; the norm 1e-12.
"""
import os

import numpy as np
import pytest

from helpers import rand_coef, rand_hint, rand_hob, rel_err
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

QUICK = os.environ.get("MCTDHB_PARITY_QUICK") == "1"


def double_well(G, xi, xf):
    x = np.linspace(xi, xf, G)
    return 0.5 * x ** 2 + 4.0 * np.exp(-x ** 2 / 0.5)


def harmonic(G, xi, xf):
    x = np.linspace(xi, xf, G)
    return 0.5 * x ** 2


def oracle_init(oracle, N, orb, coef, dx, pot, g):
    M = orb.shape[0]
    r1, r2, ri = oracle.sync_density_matrices(N, M, coef)
    return {"orb": np.ascontiguousarray(orb.copy()), "coef": np.ascontiguousarray(coef.copy()),
            "hob": np.ascontiguousarray(oracle.orbital_hob(orb, dx, -0.5, 0.0, pot)),
            "hint": np.ascontiguousarray(oracle.orbital_hint(orb, dx, g)),
            "rho1": np.ascontiguousarray(r1), "rho2": np.ascontiguousarray(r2),
            "rinv": np.ascontiguousarray(ri)}


def test_n30_m8_hc_and_densities_full_vectors(gpu, oracle):
    """every row of H.C and every element of rho1 / rho2 at N=30, M=8, with
    an arbitrary (non-symmetric) complex g"""
    import torch

    N, M = 30, 8
    rng = np.random.default_rng(3008)
    sp = gpu.Space(N, M)
    c = rand_coef(rng, sp.dim)
    h, g = rand_hob(rng, M), rand_hint(rng, M)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    sp.set_matrices(dev(h.reshape(-1)), dev(g))
    cd = dev(c)
    hc = torch.empty_like(cd)
    sp.apply_hamiltonian(cd, hc)
    r1 = torch.empty(M * M, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(M ** 4, dtype=torch.complex128, device="cuda")
    sp.density_matrices(cd, r1, r2)
    torch.cuda.synchronize()
    got_hc = hc.cpu().numpy()
    del hc, cd
    sp.close()
    want_hc = oracle.apply_hamiltonian(N, M, c, h, g)
    assert rel_err(got_hc, want_hc) < 1e-12
    del got_hc, want_hc
    assert rel_err(r1.cpu().numpy().reshape(M, M), oracle.onebody_dm(N, M, c)) < 1e-12
    assert rel_err(r2.cpu().numpy(), oracle.twobody_dm(N, M, c)) < 1e-12


def solver_vs_oracle(gpu, oracle, N, M, G, xi, xf, pot, g, dt, lz, imag, steps, seed,
                     der=300, orb_method=31):
    orb, dx = hermite_orbitals(M, G, xi, xf)
    coef = rand_coef(np.random.default_rng(seed), oracle.dim(N, M))
    s = gpu.Solver(N, M, G, xi, xf, dt, imag, 5, lz)
    try:
        s.set_derivative(der)
        s.set_orb_method(orb_method)
        s.set_potential(pot)
        s.set_interaction(g)
        s.set_state(orb, coef)
        st = oracle_init(oracle, N, orb, coef, dx, pot, g)
        e0 = oracle.total_energy(M, st["rho1"], st["rho2"], st["hob"], st["hint"]).real
        for _ in range(steps):
            oracle.propagate_step(st, N, dx, dt, -0.5, 0.0, g, True, imag, 5, lz, pot, der=der,
                                  orb_method=orb_method)
        s.step(steps)
        d = s.get()
        e = s.energy()
    finally:
        s.close()
    e_ref = oracle.total_energy(M, st["rho1"], st["rho2"], st["hob"], st["hint"])
    assert rel_err(d["orb"], st["orb"]) < 1e-10
    assert rel_err(d["coef"], st["coef"]) < 1e-10
    assert rel_err(d["rho1"], st["rho1"]) < 1e-10
    assert abs(e - e_ref) < 1e-10 * abs(e_ref), (e, e_ref)
    assert abs(np.linalg.norm(d["coef"]) - 1.0) < 1e-12
    return e0, e_ref.real


@pytest.mark.skipif(QUICK, reason="MCTDHB_PARITY_QUICK=1")
def test_n30_m8_quench_three_steps(gpu, oracle):
    """the N=30, M=8 quench as configured, three full steps"""
    G, xi, xf = 1024, -15.0, 15.0
    e0, e3 = solver_vs_oracle(gpu, oracle, 30, 8, G, xi, xf, double_well(G, xi, xf), 0.1,
                              0.005, 6, False, 3, 1234)
    # real time: the energy is conserved up to the step's own error
    assert abs(e3 - e0) < 1e-4 * abs(e0)


@pytest.mark.skipif(QUICK, reason="MCTDHB_PARITY_QUICK=1")
def test_n100_m6_one_step(gpu, oracle):
    """N=100, M=6, grid 2048 on [-20, 20], V = x^2/2, g = 0.02, real time,
    Lanczos 5, dt = 0.001: one full step"""
    G, xi, xf = 2048, -20.0, 20.0
    solver_vs_oracle(gpu, oracle, 100, 6, G, xi, xf, harmonic(G, xi, xf), 0.02, 0.001, 5,
                     False, 1, 4321)


def mix_sample(picks):
    """jobs of the batched workload (bench.mix_jobs: seed 2024, 256 jobs) at
    the given positions, built alone (each job's coefficients have their own
    seeded stream)"""
    import bench

    return bench.mix_jobs(n=max(picks) + 1, keep=set(picks))


def test_batch_mix_largest_jobs_vs_oracle(gpu, oracle):
    """the largest size of the batched mix, N=60, M=6 on 1024 points (the
    mix's own recipe, seeded), and three jobs of the mix itself, two steps
    each in one batch, against the oracle stepped alone"""
    import bench

    jobs = [bench.make_job(np.random.default_rng(6061), 60, 6, 1024, True, 2)]
    jobs += mix_sample([0, 1, 2])
    m = bench.LZ
    b = gpu.Batch(8, sum(gpu.Batch.job_bytes(j, m) for j in jobs) + (64 << 20), m)
    try:
        slots = []
        for j in jobs:
            j["max_steps"], j["energy_tol"], j["check_every"] = 2, 0.0, 0
            slots.append(b.admit(j))
        assert None not in slots
        b.step(3)
        for j, s in zip(jobs, slots):
            N, M, G = j["npar"], j["norb"], j["grid_size"]
            dx = (j["xf"] - j["xi"]) / (G - 1)
            st = oracle_init(oracle, N, j["orbitals"], j["coef"], dx, j["pot"], j["g"])
            for _ in range(2):
                oracle.propagate_step(st, N, dx, j["dt"], -0.5, 0.0, j["g"], True, True, 5, m,
                                      j["pot"])
            d = b.fetch(s)
            assert d["steps"] == 2
            assert rel_err(d["orb"], st["orb"]) < 1e-10, (N, M, G)
            assert rel_err(d["coef"], st["coef"]) < 1e-10, (N, M, G)
            assert rel_err(d["rho1"], st["rho1"]) < 1e-10, (N, M, G)
            e_ref = oracle.total_energy(M, st["rho1"], st["rho2"], st["hob"], st["hint"])
            assert abs(d["energy"] - e_ref.real) < 1e-10 * abs(e_ref), (N, M, G)
            assert abs(np.linalg.norm(d["coef"]) - 1.0) < 1e-12
    finally:
        b.close()


def relax_vs_reference(gpu, reference, der, orb_method, steps=1000):
    """the N=10, M=4 relaxation as configured (grid 256 on [-10, 10],
    V = x^2/2, g = 0.5, dt = 0.01, Lanczos 5, RK5), one struct stepped by
    the compiled reference and one by the GPU drop-in"""
    import mctdhb_types as T

    N, M, G, xi, xf, dt, g, m = 10, 4, 256, -10.0, 10.0, 0.01, 0.5, 5
    orb, _ = hermite_orbitals(M, G, xi, xf)
    coef = rand_coef(np.random.default_rng(2024), reference.lib.space_dimension(N, M))
    kw = dict(der=der, orb=orb_method)
    A, ka = reference.make_mctdhb(N, M, G, xi, xf, True, 5, m, dt, 1.0, g, **kw)
    B, kb = reference.make_mctdhb(N, M, G, xi, xf, True, 5, m, dt, 1.0, g, **kw)
    try:
        reference.set_state(A, orb, coef)
        reference.set_state(B, orb, coef)
        L = gpu.load()
        ow = np.zeros(M * G, np.complex128)
        cw = np.zeros(len(coef), np.complex128)
        for k in range(steps):
            reference.step(A, k)
            L.mctdhb_propagate_step(B, T.carray(ow), T.carray(cw), k)
        assert gpu.last_error() == "", gpu.last_error()
        # the reference's own energy of each struct (integrator_monitor.c:56)
        ea = reference.lib.total_energy(A.contents.state).re
        eb = reference.lib.total_energy(B.contents.state).re
        a, b = reference.get_state(A), reference.get_state(B)
    finally:
        reference.destroy_mctdhb(A)
        reference.destroy_mctdhb(B)
    assert abs(np.linalg.norm(b["coef"]) - 1.0) < 1e-12
    return ea, eb, a, b


def test_relaxation_n10_m4_as_configured_vs_reference(gpu, reference):
    """finite differences + RK5 on 256 points: dt * lambda_max ~ 3.3 sits at
    the edge of RK5's stability region and the reference's own trajectory
    amplifies rounding (the oracle and the compiled reference, 1e-15 apart
    after one step, end 3.6e-9 apart in energy).  Envelope: 5e-8 in energy,
    1e-5 in orbitals."""
    import mctdhb_types as T

    ea, eb, a, b = relax_vs_reference(gpu, reference, T.FINITEDIFF, T.FULLSTEP_RUNGEKUTTA)
    assert abs(eb - ea) < 5e-8 * abs(ea), (ea, eb)
    assert rel_err(b["orb"], a["orb"]) < 1e-5
    assert 1.0 < ea / 10 < 1.4


def test_relaxation_n10_m4_split_step_vs_reference(gpu, reference):
    """the same relaxation with split-step orbitals (finite differences:
    Crank-Nicolson half steps, the one split step the compiled reference can
    run -- its FFT half steps need MKL's DFTI, which is absent).  The linear
    part is exact, the trajectory contracts: held to 1e-10 against the
    compiled reference after 1000 steps (the oracle and the reference are
    1e-15 apart there)."""
    import mctdhb_types as T

    ea, eb, a, b = relax_vs_reference(gpu, reference, T.FINITEDIFF, T.SPLITSTEP)
    assert abs(eb - ea) < 1e-10 * abs(ea), (ea, eb)
    assert rel_err(b["orb"], a["orb"]) < 1e-9
    assert rel_err(b["rho1"], a["rho1"]) < 1e-9


def test_relaxation_n10_m4_dvr_vs_oracle(gpu, oracle):
    """the relaxation with DVR derivatives, the reference's default.  A
    full-step RK5 with DVR is unstable on this grid (dt * lambda_max ~ 8),
    so the orbitals take the split step, whose DVR half steps are the FFT
    exponential (orbital_integration.c:374-379); the compiled reference
    cannot run it (MKL DFTI absent), so the check is the oracle, whose direct
    DFT is pinned to numpy's FFT.  1000 steps, 1e-10."""
    N, M, G, xi, xf, dt, g, m = 10, 4, 256, -10.0, 10.0, 0.01, 0.5, 5
    e0, e = solver_vs_oracle(gpu, oracle, N, M, G, xi, xf, harmonic(G, xi, xf), g, dt, m, True,
                             1000, 2024, der=300, orb_method=31)
    assert e < e0 and 1.0 < e / N < 1.4
