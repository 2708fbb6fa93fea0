"""The job driver (dataio.run_jobs) on the GPU solver against the
reference, through the reference's text formats.

* real time with a swept harmonic trap and a ramped interaction: every
  recorded frame (rho1, orbitals, trap) and the final energy against the
  reference's own mctdhb_propagate_step on a struct from its constructor;
* imaginary time with the final lowest-state diagonalisation: final
  orbitals and coefficients against the reference stepped and diagonalised
  the same way (lowest_state_lanczos with the driver's iteration count);
* the auto convergence rule and the LAST_JOB_OUT input chaining.
"""
import os

import numpy as np
import pytest

import dataio as D
from helpers import rand_coef, rel_err
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

RT = {"integ_type": D.REALTIME, "der_method": D.FINITEDIFF, "rk_order": 5, "lanczos_iter": 5,
      "bounds": D.PERIODIC_BOUNDS}
IT = dict(RT, integ_type=D.IMAGTIME)


def write_inputs(d, prefix, lines, orb, coef, job=1):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, prefix + D.PARAMS_SUFFIX), "w") as f:
        f.write("# npar norb grid xi xf tstep tend d2 d1 gfunc g1..g5 potfunc p1..p5\n")
        f.write("\n".join(lines) + "\n")
    D.record_raw_state(os.path.join(d, f"{prefix}_job{job}"), orb, coef)


def steps_for(tend, dt):
    n = 0
    while n * dt < tend:
        n += 1
    return n


def frames(path):
    return [np.loadtxt([ln], dtype=np.complex128) for ln in open(path).read().splitlines()]


def test_realtime_sweep_and_ramp_vs_reference(gpu, reference, tmp_path):
    N, M, G, dt, tend = 5, 3, 64, 0.005, 0.06
    xi, xf = -8.0, 8.0
    line = (f"{N} {M} {G} {xi} {xf} {dt} {tend} -0.5 0.0 linear_ramp 0.3 0.9 0.03 0 0 "
            f"harmonic 1.0 1.6 0.04 0 0")
    orb, _ = hermite_orbitals(M, G, xi, xf)
    coef = rand_coef(np.random.default_rng(9), reference.lib.space_dimension(N, M))
    inp, out = str(tmp_path / "in"), str(tmp_path / "out")
    write_inputs(inp, "rt", [line], orb, coef)
    info = D.run_jobs("rt", inp, out, integrator=RT,
                      monitor={"rec_nsteps": 3, "monitor_nsteps": 1000})
    nsteps = steps_for(tend, dt)
    assert info[0]["steps"] == nsteps
    ms, keep = reference.make_mctdhb(N, M, G, xi, xf, False, 5, 5, dt, 1.0, 0.3, omega_f=1.6,
                                     pot_period=0.04, g_f=0.9, g_period=0.03)
    try:
        reference.set_state(ms, orb, coef)
        want = [reference.get_state(ms)]
        for k in range(nsteps):
            reference.step(ms, k)
            if (k + 1) % 3 == 0:
                want.append(reference.get_state(ms))
        jp = os.path.join(out, "rt_job1")
        ob, orbs, pots = frames(jp + "_obmat.dat"), frames(jp + "_orb.dat"), \
            np.loadtxt(jp + "_obpotential.dat")
        assert len(ob) == len(want) == nsteps // 3 + 1
        for i, w in enumerate(want):
            assert rel_err(ob[i].reshape(M, M), w["rho1"]) < 1e-10, i
            assert rel_err(orbs[i].reshape(M, G), w["orb"]) < 1e-10, i
            assert rel_err(pots[i], w["pot"]) < 1e-14, i
        fin = want[-1]
        e_ref = reference.lib.total_energy(ms.contents.state).re
        row = np.loadtxt(os.path.join(out, "rt" + D.PARAMS_SUFFIX), ndmin=2)[0]
        assert abs(row[10] - e_ref / N) < 1e-9 * abs(e_ref / N)
        assert abs(row[9] - 0.9) < 1e-12  # g at the end of the ramp
        assert rel_err(frames(jp + "_tbmat.dat")[-1], fin["rho2"]) < 1e-10
        t = np.loadtxt(jp + "_timesteps.dat")
        assert np.allclose(t, 3 * dt * np.arange(len(want)))
        assert np.loadtxt(jp + "_interaction.dat")[0] == 0.3
    finally:
        reference.destroy_mctdhb(ms)


@pytest.mark.parametrize("der,orb_m,coef_m", [(D.FINITEDIFF, D.FULLSTEP_RUNGEKUTTA, D.LANCZOS),
                                              (D.DVR, D.FULLSTEP_RUNGEKUTTA, D.LANCZOS),
                                              (D.FINITEDIFF, D.SPLITSTEP, D.RUNGEKUTTA)])
def test_imagtime_final_diagonalisation_vs_reference(gpu, reference, tmp_path, der, orb_m,
                                                     coef_m):
    N, M, G, dt, tend = 6, 3, 64, 0.01, 0.1
    xi, xf = -8.0, 8.0
    line = f"{N} {M} {G} {xi} {xf} {dt} {tend} -0.5 0.0 linear_ramp 0.5 0.5 0 0 0 " \
           f"harmonic 1.0 1.0 0 0 0"
    orb, _ = hermite_orbitals(M, G, xi, xf)
    dim = reference.lib.space_dimension(N, M)
    coef = rand_coef(np.random.default_rng(10), dim)
    inp, out = str(tmp_path / "in"), str(tmp_path / "out")
    write_inputs(inp, "it", [line], orb, coef)
    info = D.run_jobs("it", inp, out,
                      integrator=dict(IT, der_method=der, orb_method=orb_m, coef_method=coef_m))
    nsteps = steps_for(tend, dt)
    assert info[0]["steps"] == nsteps and not info[0]["converged"]
    ms, keep = reference.make_mctdhb(N, M, G, xi, xf, True, 5, 5, dt, 1.0, 0.5, der=der,
                                     orb=orb_m, coef=coef_m)
    try:
        reference.set_state(ms, orb, coef)
        for k in range(nsteps):
            reference.step(ms, k)
        r = reference.get_state(ms)
        e_ref = reference.lib.total_energy(ms.contents.state).re
        lan = D.lanczos_iterations_for(dim)
        assert lan == dim // 2
        e_l, c_ref = reference.lowest_state_lanczos(ms.contents.multiconfig_space, r["hob"],
                                                    r["hint"], lan, r["coef"])
        jp = os.path.join(out, "it_job1")
        got_orb = D.read_orbitals(jp + "_orb.dat", M, G)
        got_coef = D.read_coefficients(jp + "_coef.dat", dim)
        assert rel_err(got_orb, r["orb"]) < 1e-10
        ph = np.vdot(got_coef, c_ref)
        ph /= abs(ph)
        assert rel_err(got_coef * ph, c_ref) < 1e-8
        # the initial state is recorded as read, bit for bit
        assert np.array_equal(D.read_coefficients(jp + "_init_coef.dat", dim), coef)
        assert np.array_equal(D.read_orbitals(jp + "_init_orb.dat", M, G), orb)
        row = np.loadtxt(os.path.join(out, "it" + D.PARAMS_SUFFIX), ndmin=2)[0]
        assert abs(row[10] - e_ref / N) < 1e-9 * abs(e_ref / N)  # the last step's energy
        assert rel_err(np.loadtxt(jp + "_obpotential.dat"), r["pot"]) < 1e-13
    finally:
        reference.destroy_mctdhb(ms)


def test_auto_convergence_and_job_chaining(gpu, oracle, tmp_path):
    """auto_check stops the relaxation once E/N is stable to 6 digits and the
    eigen-residual is below 1e-4; LAST_JOB_OUT starts job 2 from job 1's
    output"""
    N, M, G, dt, tend = 4, 2, 64, 0.05, 30.0
    xi, xf = -8.0, 8.0
    line = f"{N} {M} {G} {xi} {xf} {dt} {tend} -0.5 0.0 linear_ramp 0.5 0.5 0 0 0 " \
           f"harmonic 1.0 1.0 0 0 0"
    orb, dx = hermite_orbitals(M, G, xi, xf)
    coef = rand_coef(np.random.default_rng(11), oracle.dim(N, M))
    inp, out = str(tmp_path / "in"), str(tmp_path / "out")
    write_inputs(inp, "ac", [line, line], orb, coef)
    mon = {"auto_check": True, "energy_digits": 6, "eig_residue": 1e-4, "monitor_nsteps": 10,
           "job_input": D.LAST_JOB_OUT}
    info = D.run_jobs("ac", inp, out, integrator=IT, monitor=mon)
    assert info[0]["converged"] and info[0]["steps"] < steps_for(tend, dt)
    assert info[0]["steps"] % 10 == 0
    j1 = os.path.join(out, "ac_job1")
    c1 = D.read_coefficients(j1 + "_coef.dat", oracle.dim(N, M))
    o1 = D.read_orbitals(j1 + "_orb.dat", M, G)
    pot = D.builtin_potential("harmonic", 0.0, D.read_parameter_line(
        os.path.join(inp, "ac" + D.PARAMS_SUFFIX)).grid, [1.0, 1.0, 0.0])
    hob = oracle.orbital_hob(o1, dx, -0.5, 0.0, pot)
    hint = oracle.orbital_hint(o1, dx, 0.5)
    r1, r2, _ = oracle.sync_density_matrices(N, M, c1)
    e = oracle.total_energy(M, r1, r2, hob, hint).real
    assert oracle.eig_residual(N, M, c1, hob, hint, e) < 1e-4
    # job 2 read job 1's output
    j2 = os.path.join(out, "ac_job2")
    assert np.array_equal(D.read_coefficients(j2 + "_init_coef.dat", len(c1)), c1)
    assert np.array_equal(D.read_orbitals(j2 + "_init_orb.dat", M, G), o1)
    assert info[1]["converged"] and info[1]["steps"] <= info[0]["steps"]
    assert np.loadtxt(os.path.join(out, "ac" + D.PARAMS_SUFFIX), ndmin=2).shape == (2, 11)
