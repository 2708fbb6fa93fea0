"""The autotuner on the hot path: launch variants of the pair contraction
(rows per tile, output tiles per pass) in the single-system H.C and the
batched engine.  Every variant computes each value with the same
instructions in the same order, so a choice changes speed, never bits; the
tuner picks an existing variant on the caller's own data."""
import numpy as np
import pytest

from helpers import rand_coef, rand_hint, rand_hob, rel_err
from oracle import hermite_orbitals

pytestmark = pytest.mark.gpu

# variants of the pair contraction per orbital count (kernels.h,
# pair_variant_ok): 0 and 3 (mbarrier handover) always, 1 up to 6 orbitals,
# 2 from 6 orbitals
VARIANTS = {4: [0, 1, 3], 5: [0, 1, 3], 6: [0, 1, 2, 3], 8: [0, 2, 3]}


@pytest.mark.parametrize("N,M", [(14, 4), (12, 5), (20, 6), (12, 8)])
def test_single_system_variants_same_bits(gpu, oracle, N, M):
    import torch

    rng = np.random.default_rng(900 + N * M)
    sp = gpu.Space(N, M)
    try:
        c = rand_coef(rng, sp.dim)
        h, g = rand_hob(rng, M), rand_hint(rng, M)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        sp.set_matrices(dev(h.reshape(-1)), dev(g))
        cd = dev(c)
        out = {}
        for v in VARIANTS[M]:
            gpu.tune_set("hcp_y", N, M, v)
            assert gpu.tune_get("hcp_y", N, M) == v
            hc = torch.empty_like(cd)
            sp.apply_hamiltonian(cd, hc)
            torch.cuda.synchronize()
            out[v] = hc.cpu().numpy()
        for v in VARIANTS[M][1:]:
            assert np.array_equal(out[v], out[0]), v
        assert rel_err(out[0], oracle.apply_hamiltonian(N, M, c, h, g)) < 1e-12
    finally:
        sp.close()


def test_single_system_tuner_picks_a_variant(gpu):
    """a fresh (N, M): the first H.C outside a capture times the variants
    and keeps one that exists"""
    import torch

    N, M = 17, 6
    sp = gpu.Space(N, M)
    try:
        rng = np.random.default_rng(5)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        sp.set_matrices(dev(rand_hob(rng, M).reshape(-1)), dev(rand_hint(rng, M)))
        cd = dev(rand_coef(rng, sp.dim))
        hc = torch.empty_like(cd)
        sp.apply_hamiltonian(cd, hc)
        torch.cuda.synchronize()
        assert gpu.tune_get("hcp_y", N, M) in VARIANTS[M]
    finally:
        sp.close()


def job(dim, N, M, G, seed):
    orb, _ = hermite_orbitals(M, G, -8.0, 8.0)
    return {"npar": N, "norb": M, "grid_size": G, "xi": -8.0, "xf": 8.0, "periodic": 1,
            "imagtime": 1, "rk_order": 5, "dt": 0.01, "g": 0.4, "max_steps": 3,
            "energy_tol": 0.0, "check_every": 0, "pot": 0.5 * np.linspace(-8, 8, G) ** 2,
            "orbitals": orb, "coef": rand_coef(np.random.default_rng(seed), dim(N, M)),
            "der_method": 302}


def test_batched_variants_same_bits(gpu, oracle):
    """the same jobs stepped with the batched contraction's variants 0, 2
    (other output-tile grouping, from six orbitals) and 3 (mbarrier
    handover of the tiles) give the same bits; the tuner's own choice is an
    existing variant"""
    jobs = [job(oracle.dim, 12, 5, 96, 1), job(oracle.dim, 10, 6, 64, 2),
            job(oracle.dim, 8, 8, 64, 3)]
    res = {}
    for v in (None, 0, 2, 3):
        b = gpu.Batch(4, sum(gpu.Batch.job_bytes(j, 5) for j in jobs) + (32 << 20), 5)
        try:
            slots = [b.admit(j) for j in jobs]
            orbs = (6, 8) if v == 2 else (5, 6, 8)
            if v is not None:
                for M in orbs:
                    b.set_variant(M, v)
            b.step(3)
            res[v] = [b.fetch(s) for s in slots]
            for M in orbs:
                got = b.variant(M)
                assert got == (v if v is not None else got) and got in (0, 2, 3)
        finally:
            b.close()
    for v in (0, 3, None):
        for a, c in zip(res[2], res[v]):
            for k in ("orb", "coef", "rho1", "rho2"):
                assert np.array_equal(a[k], c[k]), (v, k)
