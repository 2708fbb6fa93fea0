"""The oracle (oracle/oracle.c) pinned against the reference.

* against the committed golden vectors (generated from the reference's own
  compiled sources by tests/golden/make_golden.py) -- runs anywhere;
* against the compiled reference itself at random sizes -- runs where
  oracle/_ref was built.
"""
import glob
import os

import numpy as np
import pytest

from helpers import phys_hint, rand_coef, rand_hint, rand_hob, rel_err

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[4:-4] for p in GOLDEN])
def gold(request):
    return dict(np.load(request.param))


def test_golden_maps_bit_exact(oracle, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    assert np.array_equal(oracle.hash_table(N, M), gold["hash_table"])
    assert np.array_equal(oracle.single_jump_map(N, M), gold["map"])
    st, mp = oracle.double_diffjump_map(N, M)
    assert np.array_equal(st.astype(np.uint32), gold["stridett"])
    assert np.array_equal(mp, gold["maptt"])
    st, mp = oracle.double_equaljump_map(N, M)
    assert np.array_equal(st.astype(np.uint32), gold["strideot"])
    assert np.array_equal(mp, gold["mapot"])


def test_golden_hamiltonian(oracle, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    hc = oracle.apply_hamiltonian(N, M, gold["coef"], gold["hob"], gold["hint"])
    # same rule order and summation as the reference: bit for bit
    assert np.array_equal(hc, gold["hc"])
    hc = oracle.apply_hamiltonian(N, M, gold["coef"], gold["hob"], gold["hint_phys"])
    assert np.array_equal(hc, gold["hc_phys"])


def test_golden_density(oracle, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    assert rel_err(oracle.onebody_dm(N, M, gold["coef"]), gold["rho1"]) < 1e-13
    assert rel_err(oracle.twobody_dm(N, M, gold["coef"]), gold["rho2"]) < 1e-13


def test_golden_lanczos(oracle, gold):
    N, M, m = int(gold["npar"]), int(gold["norb"]), int(gold["m"])
    it, diag, offd, lv = oracle.lanczos(N, M, gold["hob"], gold["hint_phys"], m, gold["coef"])
    assert it == int(gold["lanczos_iters"])
    assert rel_err(diag[:it], gold["lanczos_diag"]) < 1e-12
    assert rel_err(offd[: it - 1], gold["lanczos_offd"]) < 1e-12
    assert rel_err(lv[:it], gold["lanczos_vecs"]) < 1e-10


def test_golden_lowest_state(oracle, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    e, c = oracle.lowest_state_lanczos(N, M, gold["hob"], gold["hint_phys"],
                                       int(gold["lowest_m"]), gold["coef"])
    assert abs(e - float(gold["lowest_e"])) < 1e-10 * abs(float(gold["lowest_e"]))
    # eigenvectors are defined up to a phase (sign of the tridiagonal one)
    ph = np.vdot(c, gold["lowest_c"])
    ph /= abs(ph)
    assert rel_err(c * ph, gold["lowest_c"]) < 1e-8


def test_rank_unrank_roundtrip(oracle):
    for N, M in [(10, 4), (30, 8), (100, 6), (7, 12)]:
        nc = oracle.dim(N, M)
        rng = np.random.default_rng(N * 100 + M)
        for idx in list(rng.integers(0, nc, size=200)) + [0, nc - 1]:
            o = oracle.unrank(N, M, int(idx))
            assert o.sum() == N
            assert oracle.rank(N, M, o) == idx


def test_dimensions(oracle):
    assert oracle.dim(10, 4) == 286
    assert oracle.dim(30, 8) == 10295472
    assert oracle.dim(100, 6) == 96560646


def test_tridiag_eig_vs_numpy(oracle):
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 15, 50):
        d = rng.normal(size=n)
        e = rng.normal(size=n)
        info, w, z = oracle.tridiag_eig(d, e)
        assert info == 0
        A = np.diag(d) + np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1)
        assert np.allclose(np.sort(w), np.linalg.eigvalsh(A), atol=1e-12)
        assert np.allclose(A @ z, z * w, atol=1e-11)


def test_herm_eig_and_inverse_vs_numpy(oracle):
    rng = np.random.default_rng(4)
    for n in (1, 3, 8):
        a = rand_hob(rng, n) + n * np.eye(n)
        w, v = oracle.herm_eig(a)
        assert np.allclose(w, np.linalg.eigvalsh(a), atol=1e-12)
        assert np.allclose(a @ v, v * w, atol=1e-11)
        info, inv = oracle.herm_inverse(a)
        assert info == 0
        assert np.allclose(inv @ a, np.eye(n), atol=1e-12)


# ---------------------------------------------------------------------------
# against the compiled reference
# ---------------------------------------------------------------------------
REF_SIZES = [(10, 4), (7, 7), (20, 3), (16, 5), (9, 6), (4, 8), (1, 5), (6, 1)]


@pytest.mark.parametrize("N,M", REF_SIZES)
def test_vs_reference_kernels(oracle, reference, N, M):
    rng = np.random.default_rng(N * 31 + M)
    mc = reference.multiconf(N, M)
    try:
        nc = mc.contents.dim
        ht, mp, _, _ = reference.maps(mc)
        assert np.array_equal(oracle.hash_table(N, M), ht)
        assert np.array_equal(oracle.single_jump_map(N, M), mp)
        c, h, g = rand_coef(rng, nc), rand_hob(rng, M), rand_hint(rng, M)
        assert np.array_equal(oracle.apply_hamiltonian(N, M, c, h, g),
                              reference.apply_hamiltonian(mc, c, h, g))
        assert rel_err(oracle.onebody_dm(N, M, c), reference.onebody_dm(mc, c)) < 1e-13
        r2 = reference.twobody_dm(mc, c)
        assert not np.isnan(r2).any(), "reference leaves a rho2 element unset"
        assert rel_err(oracle.twobody_dm(N, M, c), r2) < 1e-13
        if N >= 2:  # rho1 as the partial trace of rho2, on the reference's own outputs
            trace = np.einsum("lssk->kl", r2.reshape(M, M, M, M)) / (N - 1)
            assert rel_err(trace, reference.onebody_dm(mc, c)) < 1e-13
    finally:
        reference.lib.destroy_multiconf_struct(mc)


def test_energy_identity(oracle):
    """<C|HC> = Tr(rho1 h) + 1/2 sum rho2 g for an index-symmetric g"""
    rng = np.random.default_rng(11)
    for N, M in [(10, 4), (8, 6), (5, 8)]:
        nc = oracle.dim(N, M)
        c, h, g = rand_coef(rng, nc), rand_hob(rng, M), phys_hint(rng, M)
        e1 = np.vdot(c, oracle.apply_hamiltonian(N, M, c, h, g))
        e2 = oracle.total_energy(M, oracle.onebody_dm(N, M, c), oracle.twobody_dm(N, M, c), h, g)
        assert abs(e1 - e2) < 1e-12 * abs(e1)


def test_rho1_is_partial_trace_of_rho2(oracle):
    """sum_s rho2[k,s,s,l] = (N-1) rho1[k][l]: the identity the device uses to
    form rho1 from rho2 (two or more bosons), checked on the oracle's own
    restatement of set_onebody_dm and set_twobody_dm (density_matrices.c:9,55)"""
    rng = np.random.default_rng(12)
    for N, M in [(2, 3), (10, 4), (8, 6), (5, 8), (12, 2)]:
        c = rand_coef(rng, oracle.dim(N, M))
        r1 = oracle.onebody_dm(N, M, c)
        r2 = oracle.twobody_dm(N, M, c).reshape(M, M, M, M)  # [l, q, s, k]
        trace = np.einsum("lssk->kl", r2) / (N - 1)
        assert rel_err(trace, r1) < 1e-13, (N, M)
