"""GPU parity: the CUDA path through the C ABI against the oracle (itself
pinned to the reference) and the reference's golden vectors.

Tolerances (from the stated accuracy targets): index tables bit-exact;
H.C, rho1, rho2 within 1e-12 relative (max-norm over the max-norm of the
oracle); Lanczos / SIL outputs within 1e-10.
"""
import glob
import os

import numpy as np
import pytest

from helpers import phys_hint, rand_coef, rand_hint, rand_hob, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))
TOL = 1e-12


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[4:-4] for p in GOLDEN])
def gold(request):
    return dict(np.load(request.param))


# ---------------------------------------------------------------------------
# index tables
# ---------------------------------------------------------------------------
def test_tables_vs_golden(gpu, gold):
    import torch

    N, M = int(gold["npar"]), int(gold["norb"])
    sp = gpu.Space(N, M)
    ht = torch.empty(sp.dim * M, dtype=torch.int16, device="cuda")
    sp.hash_table(ht)
    assert np.array_equal(host(ht).view(np.uint16), gold["hash_table"])
    mp = torch.empty(sp.dim * M * M, dtype=torch.int32, device="cuda")
    sp.single_jump_map(mp)
    assert np.array_equal(host(mp).view(np.uint32), gold["map"])
    for diff, key, skey in ((1, "maptt", "stridett"), (0, "mapot", "strideot")):
        n = sp.double_jump_chunks(diff)
        st = torch.empty(sp.dim + 1, dtype=torch.int64, device="cuda")
        m = torch.empty(max(n * M * M, 1), dtype=torch.int32, device="cuda")
        sp.double_jump_map(diff, st, m)
        assert np.array_equal(host(m).view(np.uint32)[: n * M * M], gold[key])
        assert np.array_equal(host(st)[: sp.dim].astype(np.uint32), gold[skey])


@pytest.mark.parametrize("N,M", [(30, 6), (40, 4), (12, 8), (5, 11)])
def test_tables_vs_oracle(gpu, oracle, N, M):
    import torch

    sp = gpu.Space(N, M)
    ht = torch.empty(sp.dim * M, dtype=torch.int16, device="cuda")
    sp.hash_table(ht)
    assert np.array_equal(host(ht).view(np.uint16), oracle.hash_table(N, M))
    mp = torch.empty(sp.dim * M * M, dtype=torch.int32, device="cuda")
    sp.single_jump_map(mp)
    assert np.array_equal(host(mp).view(np.uint32), oracle.single_jump_map(N, M))
    st_o, m_o = oracle.double_diffjump_map(N, M)
    n = sp.double_jump_chunks(1)
    st = torch.empty(sp.dim + 1, dtype=torch.int64, device="cuda")
    m = torch.empty(max(n * M * M, 1), dtype=torch.int32, device="cuda")
    sp.double_jump_map(1, st, m)
    assert np.array_equal(host(m).view(np.uint32)[: n * M * M], m_o)
    assert np.array_equal(host(st)[: sp.dim].view(np.uint64), st_o)


def test_dropin_multiconf_struct(gpu, gold):
    import mctdhb_types as T

    N, M = int(gold["npar"]), int(gold["norb"])
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        s = mc.contents
        assert s.dim == len(gold["coef"])
        assert np.array_equal(T.uint_array_to_numpy(s.hash_table, s.dim * M, np.uint16),
                              gold["hash_table"])
        om = s.op_maps.contents
        assert np.array_equal(T.uint_array_to_numpy(om.map, s.dim * M * M, np.uint32), gold["map"])
        assert np.array_equal(T.uint_array_to_numpy(om.stridett, s.dim, np.uint32),
                              gold["stridett"])
        n = len(gold["maptt"])
        if n:
            assert np.array_equal(T.uint_array_to_numpy(om.maptt, n, np.uint32), gold["maptt"])
    finally:
        D.destroy(mc)


# ---------------------------------------------------------------------------
# H.C
# ---------------------------------------------------------------------------
HC_SIZES = [(10, 4), (2, 2), (6, 1), (1, 5), (25, 3), (16, 5), (14, 6), (9, 7), (8, 8),
            (30, 6), (4, 9), (3, 12)]


@pytest.mark.parametrize("N,M", HC_SIZES)
def test_hc_vs_oracle(gpu, oracle, N, M):
    import torch

    rng = np.random.default_rng(1000 + 37 * N + M)
    sp = gpu.Space(N, M)
    nc = sp.dim
    c, h, g = rand_coef(rng, nc), rand_hob(rng, M), rand_hint(rng, M)
    sp.set_matrices(dev(h), dev(g))
    out = torch.empty(nc, dtype=torch.complex128, device="cuda")
    sp.apply_hamiltonian(dev(c), out)
    ref = oracle.apply_hamiltonian(N, M, c, h, g)
    assert rel_err(host(out), ref) < TOL


@pytest.mark.parametrize("N,M", [(10, 4), (2, 2), (16, 5), (14, 6), (9, 7), (8, 8), (30, 6)])
def test_hc_real_matrices_vs_oracle(gpu, oracle, N, M):
    """real h and g (real orbitals): the contraction's two-product path,
    complex coefficients"""
    import torch

    rng = np.random.default_rng(2000 + 37 * N + M)
    sp = gpu.Space(N, M)
    nc = sp.dim
    h = rand_hob(rng, M).real.astype(np.complex128)
    f = rng.normal(size=(M, 40))
    t = np.einsum("x,ax,bx,cx,dx->abcd", rng.uniform(0.5, 1.5, 40), f, f, f, f)
    g = np.ascontiguousarray(t.transpose(3, 2, 1, 0)).reshape(-1).astype(np.complex128)
    c = rand_coef(rng, nc)
    sp.set_matrices(dev(h), dev(g))
    out = torch.empty(nc, dtype=torch.complex128, device="cuda")
    sp.apply_hamiltonian(dev(c), out)
    assert rel_err(host(out), oracle.apply_hamiltonian(N, M, c, h, g)) < TOL
    # a complex g on the same space goes back to three products
    g2 = g + 1e-3j * rng.normal(size=g.shape)
    sp.set_matrices(dev(h), dev(g2))
    sp.apply_hamiltonian(dev(c), out)
    assert rel_err(host(out), oracle.apply_hamiltonian(N, M, c, h, g2)) < TOL


def test_hc_dropin_vs_golden(gpu, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        for gk, hk in (("hint", "hc"), ("hint_phys", "hc_phys")):
            got = D.apply_hamiltonian(mc, gold["coef"], gold["hob"], gold[gk])
            assert rel_err(got, gold[hk]) < TOL
    finally:
        D.destroy(mc)


# ---------------------------------------------------------------------------
# density matrices
# ---------------------------------------------------------------------------
DENS_SIZES = [(10, 4), (2, 2), (6, 1), (25, 3), (16, 5), (14, 6), (9, 7), (8, 8), (30, 6),
              (4, 9), (2, 7), (3, 8)]


@pytest.mark.parametrize("N,M", DENS_SIZES)
def test_density_vs_oracle(gpu, oracle, N, M):
    import torch

    rng = np.random.default_rng(2000 + 37 * N + M)
    sp = gpu.Space(N, M)
    c = rand_coef(rng, sp.dim)
    r1 = torch.empty(M * M, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(M ** 4, dtype=torch.complex128, device="cuda")
    sp.density_matrices(dev(c), r1, r2)
    assert rel_err(host(r1).reshape(M, M), oracle.onebody_dm(N, M, c)) < TOL
    assert rel_err(host(r2), oracle.twobody_dm(N, M, c)) < TOL


@pytest.mark.parametrize("M", [3, 5, 8])
def test_density_one_boson(gpu, oracle, M):
    """one boson: rho1 from its own Gram pass (with two or more bosons it is
    the partial trace of rho2), rho2 identically zero"""
    import torch

    rng = np.random.default_rng(2100 + M)
    sp = gpu.Space(1, M)
    c = rand_coef(rng, sp.dim)
    r1 = torch.empty(M * M, dtype=torch.complex128, device="cuda")
    r2 = torch.full((M ** 4,), 1.0 + 1.0j, dtype=torch.complex128, device="cuda")
    sp.density_matrices(dev(c), r1, r2)
    assert rel_err(host(r1).reshape(M, M), oracle.onebody_dm(1, M, c)) < TOL
    assert not np.any(host(r2))


def test_density_dropin_vs_golden(gpu, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        assert rel_err(D.onebody_dm(mc, gold["coef"]), gold["rho1"]) < TOL
        assert rel_err(D.twobody_dm(mc, gold["coef"]), gold["rho2"]) < TOL
    finally:
        D.destroy(mc)


def test_density_deterministic(gpu):
    """same input, same bits (fixed-order reductions)"""
    import torch

    rng = np.random.default_rng(7)
    sp = gpu.Space(20, 6)
    c = dev(rand_coef(rng, sp.dim))
    outs = []
    for _ in range(3):
        r1 = torch.empty(36, dtype=torch.complex128, device="cuda")
        r2 = torch.empty(6 ** 4, dtype=torch.complex128, device="cuda")
        sp.density_matrices(c, r1, r2)
        outs.append((host(r1), host(r2)))
    for a, b in outs[1:]:
        assert np.array_equal(a, outs[0][0]) and np.array_equal(b, outs[0][1])


# ---------------------------------------------------------------------------
# Lanczos / SIL
# ---------------------------------------------------------------------------
def test_lanczos_dropin_vs_golden(gpu, gold):
    N, M, m = int(gold["npar"]), int(gold["norb"]), int(gold["m"])
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        it, diag, offd, lv = D.lanczos(mc, gold["hob"], gold["hint_phys"], m, gold["coef"])
        assert it == int(gold["lanczos_iters"])
        assert rel_err(diag[:it], gold["lanczos_diag"]) < 1e-10
        assert rel_err(offd[: it - 1], gold["lanczos_offd"]) < 1e-10
        assert rel_err(lv[:it], gold["lanczos_vecs"]) < 1e-9
    finally:
        D.destroy(mc)


def test_lowest_state_dropin_vs_golden(gpu, gold):
    N, M = int(gold["npar"]), int(gold["norb"])
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        e, c = D.lowest_state_lanczos(mc, gold["hob"], gold["hint_phys"], int(gold["lowest_m"]),
                                      gold["coef"])
        e0 = float(gold["lowest_e"])
        assert abs(e - e0) < 1e-10 * abs(e0)
        ph = np.vdot(c, gold["lowest_c"])
        ph /= abs(ph)
        assert rel_err(c * ph, gold["lowest_c"]) < 1e-8
    finally:
        D.destroy(mc)


@pytest.mark.parametrize("N,M,m,imag", [(10, 4, 5, True), (10, 4, 5, False), (14, 6, 6, False),
                                        (8, 8, 6, True), (30, 6, 6, False), (4, 9, 4, True)])
def test_sil_step_vs_oracle(gpu, oracle, N, M, m, imag):
    rng = np.random.default_rng(3000 + N * 7 + M)
    sp = gpu.Space(N, M)
    c, h, g = rand_coef(rng, sp.dim), rand_hob(rng, M), phys_hint(rng, M)
    h = h * 0.1
    g = g * (0.05 / np.abs(g).max())
    dt = 0.01
    sp.set_matrices(dev(h), dev(g))
    cd = dev(c)
    sp.sil_step(cd, m, dt, imag)
    it, ref = oracle.sil_step(N, M, h, g, m, dt, imag, c)
    assert rel_err(host(cd), ref) < 1e-10
    assert abs(np.linalg.norm(host(cd)) - 1) < 1e-12


def test_propagate_coef_sil_dropin(gpu, oracle):
    rng = np.random.default_rng(77)
    N, M, m = 10, 4, 5
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        c, h, g = rand_coef(rng, mc.contents.dim), rand_hob(rng, M), phys_hint(rng, M)
        g = g * (0.1 / np.abs(g).max())
        for imag in (True, False):
            cnext, coef, dd, od = D.propagate_coef_sil(mc, h, g, c, m, 0.01, imag)
            it, ref = oracle.sil_step(N, M, h, g, m, 0.01, imag, c)
            assert rel_err(coef, ref) < 1e-10
            if imag:  # cnext is the combination before renormalisation
                assert rel_err(cnext / np.linalg.norm(cnext), ref) < 1e-10
            oit, odiag, ooffd, _ = oracle.lanczos(N, M, h, g, m, c)
            assert rel_err(dd[:oit], odiag[:oit]) < 1e-10
    finally:
        D.destroy(mc)


def test_step_graph_matches_calls(gpu, oracle):
    """the captured step (SIL + rho1/rho2) equals the same calls made one by one"""
    import torch

    rng = np.random.default_rng(55)
    N, M, m = 14, 6, 6
    sp = gpu.Space(N, M)
    c, h, g = rand_coef(rng, sp.dim), rand_hob(rng, M), phys_hint(rng, M)
    g = g * (0.05 / np.abs(g).max())
    sp.set_matrices(dev(h), dev(g))
    cg = dev(c)
    r1 = torch.empty(M * M, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(M ** 4, dtype=torch.complex128, device="cuda")
    step = gpu.Step(sp, cg, r1, r2, m, 0.01, False)
    assert step.kernels > 10
    step.launch()
    step.launch()
    cc = dev(c)
    s1 = torch.empty_like(r1)
    s2 = torch.empty_like(r2)
    for _ in range(2):
        sp.sil_step(cc, m, 0.01, False)
    sp.density_matrices(cc, s1, s2)
    assert np.array_equal(host(cg), host(cc))
    assert np.array_equal(host(r1), host(s1)) and np.array_equal(host(r2), host(s2))
    _, ref = oracle.sil_step(N, M, h, g, m, 0.01, False, c)
    _, ref = oracle.sil_step(N, M, h, g, m, 0.01, False, ref)
    assert rel_err(host(cg), ref) < 1e-10
    step.close()


def test_sync_density_matrices_dropin(gpu, oracle):
    import ctypes as C

    import mctdhb_types as T

    rng = np.random.default_rng(56)
    N, M = 12, 5
    D = gpu.DropIn()
    mc = D.multiconf(N, M)
    try:
        nc = mc.contents.dim
        c = rand_coef(rng, nc)
        st = T.ManyBodyStateS()
        st.npar, st.norb, st.space_dim = N, M, nc
        coef = np.ascontiguousarray(c)
        r2 = np.zeros(M ** 4, np.complex128)
        R1 = T.RowMatrix(np.zeros((M, M), np.complex128))
        RI = T.RowMatrix(np.zeros((M, M), np.complex128))
        st.coef, st.tb_denmat, st.ob_denmat, st.inv_ob_denmat = (T.carray(coef), T.carray(r2),
                                                                 R1.ptr, RI.ptr)
        D.lib.mctdhb_gpu_clear_error()
        D.lib.sync_density_matrices(mc, C.pointer(st))
        assert gpu.last_error() == ""
        o1, o2, oi = oracle.sync_density_matrices(N, M, c)
        assert rel_err(R1.a, o1) < TOL and rel_err(r2, o2) < TOL
        assert rel_err(RI.a, oi) < 1e-10
        assert np.allclose(RI.a @ R1.a, np.eye(M), atol=1e-10)
    finally:
        D.destroy(mc)


# ---------------------------------------------------------------------------
# full sizes (N=30 M=8, nc = 10,295,472; N=100 M=6, nc = 96,560,646 -- 1.5 GB
# per vector, beyond the reference's 32-bit map guards): size-independent
# properties + sampled rows
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("N,M,nc_expected", [(30, 8, 10295472), (100, 6, 96560646)])
def test_hc_large_properties(gpu, oracle, N, M, nc_expected):
    import torch

    rng = np.random.default_rng(99)
    sp = gpu.Space(N, M)
    nc = sp.dim
    assert nc == nc_expected
    h, g = rand_hob(rng, M), phys_hint(rng, M)
    sp.set_matrices(dev(h), dev(g))
    u = torch.randn(nc, dtype=torch.complex128, device="cuda", generator=None)
    u /= torch.linalg.vector_norm(u)
    v = torch.randn(nc, dtype=torch.complex128, device="cuda")
    v /= torch.linalg.vector_norm(v)
    hu = torch.empty_like(u)
    hv = torch.empty_like(v)
    sp.apply_hamiltonian(u, hu)
    sp.apply_hamiltonian(v, hv)
    # hermiticity: <u|Hv> = conj <v|Hu>
    a = torch.vdot(u, hv).item()
    b = torch.vdot(v, hu).item()
    assert abs(a - np.conj(b)) < 1e-11 * max(abs(a), 1.0)
    # energy identity <u|Hu> = Tr(rho1 h) + 1/2 sum rho2 g
    r1 = torch.empty(M * M, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(M ** 4, dtype=torch.complex128, device="cuda")
    sp.density_matrices(u, r1, r2)
    e1 = torch.vdot(u, hu).item()
    e2 = oracle.total_energy(M, host(r1).reshape(M, M), host(r2), h, g)
    assert abs(e1 - e2) < 1e-11 * abs(e1)
    # rows sampled across the space against the oracle's rows
    un = host(u)
    hun = host(hu)
    for r0 in (0, nc // 3, nc // 2 + 12345, nc - 2000):
        ref = oracle.apply_hamiltonian(N, M, un, h, g, rows=(r0, r0 + 2000))
        assert rel_err(hun[r0:r0 + 2000], ref[r0:r0 + 2000]) < TOL
    del u, v, hu, hv
    sp.close()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("N,M,m", [(30, 8, 6), (100, 6, 5)])
def test_sil_large_norm_and_energy(gpu, N, M, m):
    """real-time SIL steps conserve the norm to 1e-12 and the energy
    <C|H|C> to 1e-10 (H is time independent within the step); an
    imaginary-time step lowers the energy and renormalises"""
    import torch

    rng = np.random.default_rng(7 * N + M)
    sp = gpu.Space(N, M)
    nc = sp.dim
    h, g = rand_hob(rng, M), phys_hint(rng, M)
    sp.set_matrices(dev(h), dev(g))
    c = torch.randn(nc, dtype=torch.complex128, device="cuda")
    c /= torch.linalg.vector_norm(c)
    hc = torch.empty_like(c)

    def energy():
        sp.apply_hamiltonian(c, hc)
        return torch.vdot(c, hc).item()

    e0 = energy()
    for _ in range(3):
        sp.sil_step(c, m, 0.005, False)
    torch.cuda.synchronize()
    assert abs(torch.linalg.vector_norm(c).item() - 1.0) < 1e-12
    e1 = energy()
    assert abs(e1 - e0) < 1e-10 * abs(e0)
    sp.sil_step(c, m, 0.005, True)
    assert abs(torch.linalg.vector_norm(c).item() - 1.0) < 1e-12
    assert energy().real < e1.real
    del c, hc
    sp.close()
    torch.cuda.empty_cache()
