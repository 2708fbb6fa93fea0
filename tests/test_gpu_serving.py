"""The request loop (1d-mctdhb_b200/serving.py) on the batched engine:
every job's result is the same, bit for bit, served alone and served in a
stream of other jobs arriving while it runs; a full arena back-pressures
(jobs wait, none fails) and releases make room."""
import numpy as np
import pytest

from helpers import rand_coef
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

XI, XF = -8.0, 8.0


def job(dim, N, M, G, imag, dt, g, steps, seed, **kw):
    orb, _ = hermite_orbitals(M, G, XI, XF)
    j = {"npar": N, "norb": M, "grid_size": G, "xi": XI, "xf": XF, "periodic": 1,
         "imagtime": int(imag), "rk_order": 5, "dt": dt, "g": g, "max_steps": steps,
         "energy_tol": 1e-10 if imag else 0.0, "check_every": 1 if imag else 0,
         "pot": 0.5 * np.linspace(XI, XF, G) ** 2, "orbitals": orb,
         "coef": rand_coef(np.random.default_rng(seed), dim(N, M)), "der_method": 302}
    j.update(kw)
    return j


def serve(gpu, jobs, arrivals, arena, steps_per_tick=2):
    from serving import Server

    srv = Server(arena, max_slots=16, steps_per_tick=steps_per_tick)
    try:
        ids = [srv.submit(j, at=a) for j, a in zip(jobs, arrivals)]
        srv.run()
        return [srv.result(i) for i in ids], srv.stats()
    finally:
        srv.close()


def test_results_alone_equal_results_in_the_stream(gpu, oracle):
    import mctdhb_b200 as mb

    stream = [job(oracle.dim, 10, 4, 128, True, 0.01, 0.5, 60, 1),
              job(oracle.dim, 12, 3, 96, False, 0.005, 0.3, 40, 2),
              job(oracle.dim, 8, 5, 128, True, 0.01, 0.8, 80, 3),
              job(oracle.dim, 20, 4, 64, True, 0.01, 0.2, 50, 4),
              job(oracle.dim, 6, 6, 96, False, 0.005, 0.6, 30, 5)]
    arrivals = [0.0, 0.01, 0.02, 0.05, 0.08]
    arena = sum(mb.Batch.job_bytes(j, 5) for j in stream) + (64 << 20)
    mixed, stats = serve(gpu, stream, arrivals, arena)
    assert stats["jobs"] == len(stream)
    for j, m in zip(stream, mixed):
        (alone,), _ = serve(gpu, [j], [0.0], mb.Batch.job_bytes(j, 5) + (16 << 20))
        for k in ("orb", "coef", "rho1", "rho2"):
            assert np.array_equal(alone[k], m[k]), k
        assert alone["energy"] == m["energy"] and alone["steps"] == m["steps"]
        assert alone["state"] == m["state"] == 2


def test_full_arena_back_pressures(gpu, oracle):
    """an arena for two jobs and five submitted at once: at most two run,
    every job completes with its own result"""
    import mctdhb_b200 as mb

    jobs = [job(oracle.dim, 10, 4, 96, True, 0.01, 0.5, 20 + 5 * i, 10 + i) for i in range(5)]
    need = max(mb.Batch.job_bytes(j, 5) for j in jobs)
    res, stats = serve(gpu, jobs, [0.0] * 5, 2 * need + need // 2)
    assert stats["jobs"] == 5 and stats["peak_running"] == 2
    for i, r in enumerate(res):
        assert r["state"] == 2 and r["steps"] <= 20 + 5 * i
        assert np.isfinite(r["energy"])


def test_heavy_lane_beside_the_batch(gpu, oracle):
    """with heavy_nc, the large job runs in the solver lane beside the batch:
    its result is the plain solver's relaxation alone, bit for bit, and the
    light jobs' results are their batched results alone"""
    import mctdhb_b200 as mb
    from serving import Server

    heavy = job(oracle.dim, 14, 5, 128, True, 0.01, 0.4, 40, 21)  # 3060 configurations
    light = [job(oracle.dim, 8, 3, 96, True, 0.01, 0.5, 30, 22),
             job(oracle.dim, 6, 4, 64, False, 0.005, 0.3, 25, 23)]
    arena = sum(mb.Batch.job_bytes(j, 5) for j in light) + (32 << 20)
    srv = Server(arena, max_slots=8, heavy_nc=3000)
    try:
        ids = [srv.submit(j, at=0.0) for j in [heavy] + light]
        srv.run()
        res = [srv.result(i) for i in ids]
    finally:
        srv.close()
    assert res[0]["lane"] == "solver"
    s = mb.Solver(14, 5, 128, XI, XF, 0.01, True, 5, 5)
    s.set_potential(heavy["pot"])
    s.set_interaction(heavy["g"])
    s.set_state(heavy["orbitals"], heavy["coef"])
    s.relax(40, heavy["energy_tol"], heavy["check_every"])
    steps, conv = s.relax_result()
    d = s.get()
    s.close()
    assert res[0]["steps"] == steps and res[0]["converged"] == conv
    for k in ("orb", "coef", "rho1", "rho2"):
        assert np.array_equal(res[0][k], d[k]), k
    for j, r in zip(light, res[1:]):
        (alone,), _ = serve(gpu, [j], [0.0], mb.Batch.job_bytes(j, 5) + (16 << 20))
        for k in ("orb", "coef", "rho1", "rho2"):
            assert np.array_equal(alone[k], r[k]), k
