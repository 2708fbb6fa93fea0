"""mctdhb_solver_relax: the single-system solver stepping on the device until
the reference driver's imaginary-time energy rule (driver.c:47-67) or a step
limit, in one launch of a graph with a conditional WHILE node -- against
the same solver stepped one step at a time with the rule evaluated on the
host: the same number of steps, the same stop reason, the same bits."""
import numpy as np
import pytest

from helpers import rand_coef
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

XI, XF = -8.0, 8.0


def solver(gpu, N, M, G, imag, dt, g, seed):
    orb, _ = hermite_orbitals(M, G, XI, XF)
    s = gpu.Solver(N, M, G, XI, XF, dt, imag, 5, 5)
    s.set_potential(0.5 * np.linspace(XI, XF, G) ** 2)
    s.set_interaction(g)
    s.set_state(orb, rand_coef(np.random.default_rng(seed), s.dim))
    return s


def host_loop(s, N, max_steps, tol, check):
    """the reference's loop: step, then every `check` steps the energy rule
    on the host"""
    prev = s.energy().real / N
    k = 0
    while k < max_steps:
        s.step(1)
        k += 1
        if check and k % check == 0:
            e = s.energy().real / N
            if abs(e - prev) < tol * prev:
                return k, True
            prev = e
    return k, False


@pytest.mark.parametrize("N,M,G,tol,check", [(6, 3, 64, 1e-9, 1), (8, 4, 96, 1e-8, 3)])
def test_relax_stops_like_the_host_loop(gpu, N, M, G, tol, check):
    a = solver(gpu, N, M, G, True, 0.01, 0.5, 7)
    b = solver(gpu, N, M, G, True, 0.01, 0.5, 7)
    try:
        a.relax(4000, tol, check)
        n, conv = a.relax_result()
        m, conv_b = host_loop(b, N, 4000, tol, check)
        assert conv and conv_b and n == m and 1 < n < 4000
        da, db = a.get(), b.get()
        for k in ("orb", "coef", "rho1", "rho2"):
            assert np.array_equal(da[k], db[k]), k
        assert a.energy() == b.energy()
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("imag", [True, False])
def test_relax_step_limit(gpu, imag):
    """no rule (check 0, or real time): exactly max_steps steps, the same
    bits as step(max_steps); a second run continues from the first"""
    a = solver(gpu, 5, 3, 64, imag, 0.005, 0.4, 9)
    b = solver(gpu, 5, 3, 64, imag, 0.005, 0.4, 9)
    try:
        a.relax(7, 1e-3, 0 if imag else 1)
        assert a.relax_result() == (7, False)
        a.relax(4)
        assert a.relax_result() == (4, False)
        b.step(11)
        da, db = a.get(), b.get()
        for k in ("orb", "coef", "rho1", "rho2"):
            assert np.array_equal(da[k], db[k]), k
    finally:
        a.close()
        b.close()
