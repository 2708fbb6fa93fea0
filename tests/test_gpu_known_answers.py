"""Known answers of the reference (its benchmark.dat, fixture
tests/golden/benchmark_known_answers.json): converged ground states of the
harmonic trap and of the harmonic trap with a Gaussian barrier, reached by
imaginary-time relaxation on the device solver with the reference's default
derivative method (DVR) and its split-step integrator (the FFT-exponential
half steps are unconditionally stable, so a fine grid keeps dt = 0.01).  The
grid must be fine: h_kl, and so the energy, takes fourth-order finite
differences whatever the method (orbital_matrices.c:22-70), which
underestimate the kinetic energy on coarse grids.  The file quotes the
energy per particle to at least 4 digits and the condensate fraction to 2;
the grid those came from is not stated, so the energy is held to 1e-3
relative, sqrt<x^2> to 1e-2 and, in the harmonic trap, the condensate
fraction to 0.02.

The start is real (Hermite functions, equal coefficients), so the pair
contraction runs its two-product path for real W all the way.
"""
import json
import os

import numpy as np
import pytest

from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
KNOWN = json.load(open(os.path.join(HERE, "golden", "benchmark_known_answers.json")))
CASES = [("harmonic", r) for r in KNOWN["harmonic"]] + [("barrier", r) for r in KNOWN["barrier"]]


def simpson(f, h):
    n = len(f)
    w = np.ones(n)
    w[1:-1:2], w[2:-1:2] = 4, 2
    if n % 2 == 0:  # odd number of intervals: the last one by the trapezoid rule
        return simpson(f[:-1], h) + 0.5 * h * (f[-2] + f[-1])
    return h / 3 * np.dot(w, f)


@pytest.mark.parametrize("trap,known", CASES,
                         ids=[f"{t}-N{r['npar']}-M{r['norb']}-g{r['g']}" for t, r in CASES])
def test_relaxed_ground_state_matches_known_answers(gpu, trap, known):
    N, M, g = known["npar"], known["norb"], known["g"]
    # the barrier's tunnelling splitting is small: its relaxation is slow
    G, xi, xf, dt = 513, -9.0, 9.0, 0.01
    steps = 15000 if trap == "barrier" else 4000
    x = np.linspace(xi, xf, G)
    pot = 0.5 * x ** 2
    if trap == "barrier":
        pot = pot + 9.0 * np.exp(-x ** 2 / (2 * 0.5 ** 2))
    orb, dx = hermite_orbitals(M, G, xi, xf)
    dim = gpu.load().space_dimension(N, M)
    coef = np.full(dim, 1.0 / np.sqrt(dim), np.complex128)
    s = gpu.Solver(N, M, G, xi, xf, dt, True, 5, 5)
    s.set_derivative(300)  # DVR
    s.set_orb_method(31)  # split step
    s.set_potential(pot)
    s.set_interaction(g)
    s.set_state(orb, coef)
    s.step(steps)
    e = s.energy().real / N
    d = s.get()
    s.close()
    occ = np.linalg.eigvalsh(d["rho1"])[-1] / N
    phi = d["orb"]
    r2 = sum(d["rho1"][k, l] * simpson(np.conj(phi[k]) * x ** 2 * phi[l], dx)
             for k in range(M) for l in range(M)).real / N
    print(f"{trap} N={N} M={M} g={g}: E/N {e:.7f} ({known['e_per_n']}), "
          f"condensate {occ:.3f} ({known['condensate']}), "
          f"sqrt<x2> {np.sqrt(r2):.4f} ({known['sqrt_r2']})")
    # the file's 4 digits of energy were reached on a grid it does not give
    assert abs(e - known["e_per_n"]) < 1e-3 * abs(known["e_per_n"])
    assert abs(np.sqrt(r2) - known["sqrt_r2"]) < 1e-2 * known["sqrt_r2"]
    # In the double well the natural orbitals keep rotating long after the
    # energy has settled (N=5, M=4: fraction 0.64 at t = 20, 0.77 at t = 150,
    # energy within 3e-5 at both), so its condensate fraction is not held.
    if trap == "harmonic":
        assert abs(occ - known["condensate"]) < 0.02
