"""The C-ABI library on a machine without a GPU: it loads, exports every
function include/*.h declares, its host-only helpers agree with the oracle,
and device calls fail with an error status instead of exiting."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import mctdhb_b200
import mctdhb_types as T

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(REPO, "include", "mctdhb_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"if", "for", "while", "return", "sizeof"}
    return sorted({n for n in names if n not in skip})


def test_library_exports_header():
    L = mctdhb_b200.load()
    declared = header_functions()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/mctdhb_gpu.h but not exported"
    assert set(declared) == set(mctdhb_b200.EXPORTED)


def test_space_dimension_and_subspaces(oracle):
    L = mctdhb_b200.load()
    for N, M in [(10, 4), (30, 8), (100, 6), (1, 1), (5, 11)]:
        assert L.space_dimension(N, M) == oracle.dim(N, M)
        p = L.get_subspaces_dim(N, M)
        got = np.ctypeslib.as_array(p, shape=((N + 1) * (M + 1),)).copy()
        assert np.array_equal(got, oracle.subspaces_dim(N, M))
    # 32-bit overflow is reported, not fatal
    assert L.space_dimension(200, 12) == 0
    assert "overflow" in mctdhb_b200.last_error()


def test_set_config_hash_index(oracle):
    L = mctdhb_b200.load()
    rng = np.random.default_rng(5)
    for N, M in [(10, 4), (30, 8), (100, 6)]:
        nc = oracle.dim(N, M)
        sub = L.get_subspaces_dim(N, M)
        for idx in list(rng.integers(0, nc, size=100)) + [0, nc - 1]:
            conf = (C.c_uint16 * M)()
            L.set_config(int(idx), N, M, conf)
            o = np.array(conf[:], np.uint16)
            assert np.array_equal(o, oracle.unrank(N, M, int(idx)))
            assert L.hash_index(N, M, sub, conf) == idx


def test_total_energy_host(oracle):
    """total_energy (integrator_monitor.c:56) on host buffers"""
    L = mctdhb_b200.load()
    rng = np.random.default_rng(6)
    M = 4
    r1 = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    r2 = rng.normal(size=M ** 4) + 1j * rng.normal(size=M ** 4)
    h = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    g = rng.normal(size=M ** 4) + 1j * rng.normal(size=M ** 4)
    st = T.ManyBodyStateS()
    st.norb = M
    R1, H = T.RowMatrix(r1), T.RowMatrix(h)
    st.ob_denmat, st.hob = R1.ptr, H.ptr
    r2c, gc = np.ascontiguousarray(r2), np.ascontiguousarray(g)
    st.tb_denmat, st.hint = T.carray(r2c), T.carray(gc)
    e = L.total_energy(C.pointer(st)).value()
    assert abs(e - oracle.total_energy(M, r1, r2, h, g)) < 1e-12 * abs(e)


def test_device_calls_fail_cleanly_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = mctdhb_b200.load()
    h = C.c_void_p()
    assert L.mctdhb_space_create(10, 4, C.byref(h)) == -1
    assert mctdhb_b200.last_error() != ""
    with pytest.raises(mctdhb_b200.MctdhbError):
        mctdhb_b200.Space(10, 4)


def test_invalid_space_rejected():
    L = mctdhb_b200.load()
    h = C.c_void_p()
    assert L.mctdhb_space_create(0, 4, C.byref(h)) == -1
    assert "invalid" in mctdhb_b200.last_error()
    assert L.mctdhb_space_create(10, 31, C.byref(h)) == -1
    assert L.mctdhb_space_create(300, 12, C.byref(h)) == -1  # > 2^32 configurations
    assert "32-bit" in mctdhb_b200.last_error()


def test_batch_job_bytes_host():
    """the batched engine's footprint formula is host arithmetic: it needs no
    GPU, grows with the Fock space and rejects what the engine cannot run"""
    import mctdhb_b200 as B

    def job(N, M, G):
        return {"npar": N, "norb": M, "grid_size": G, "xi": -8.0, "xf": 8.0, "periodic": 1,
                "imagtime": 1, "rk_order": 5, "dt": 0.01, "g": 0.5, "max_steps": 10,
                "pot": np.zeros(G), "orbitals": np.zeros((M, G), np.complex128),
                "coef": np.zeros(1, np.complex128)}

    small = B.Batch.job_bytes(job(10, 3, 128), 5)
    big = B.Batch.job_bytes(job(40, 6, 128), 5)
    nc, d2 = 1221759, 962598  # C(45, 5), C(43, 5): the N and N-2 boson spaces
    # 5 Krylov vectors + work vector, and the pair-space H.C scratch
    # (21 pairs x the N-2 space) dominate
    core = 16 * (6 * nc + 21 * d2)
    assert core < big < 1.05 * core
    assert small > 0 and small % 256 == 0 and big % 256 == 0
    assert B.Batch.job_bytes(job(40, 6, 1024), 5) > big  # orbital buffers grow with the grid
    with pytest.raises(B.MctdhbError):
        B.Batch.job_bytes(job(10, 9, 128), 5)  # the engine runs 2..8 orbitals
    with pytest.raises(B.MctdhbError):
        B.Batch.job_bytes(job(1, 4, 128), 5)  # and at least two bosons


def test_batch_job_derivative_method_host():
    """DVR / spectral jobs hold a Toeplitz kernel of 2(G-1)-1 complex values
    in the arena; zero bounds and unknown methods are rejected"""
    import mctdhb_b200 as B

    def job(der, periodic=1, G=256):
        return {"npar": 10, "norb": 3, "grid_size": G, "xi": -8.0, "xf": 8.0,
                "periodic": periodic, "imagtime": 1, "rk_order": 5, "dt": 0.01, "g": 0.5,
                "max_steps": 10, "pot": np.zeros(G), "orbitals": np.zeros((3, G), np.complex128),
                "coef": np.zeros(1, np.complex128), "der_method": der}

    fd = B.Batch.job_bytes(job(302), 5)
    assert B.Batch.job_bytes(job(0), 5) == fd  # 0: finite differences
    for der in (300, 301):
        extra = B.Batch.job_bytes(job(der), 5) - fd
        assert 16 * (2 * 255 - 1) <= extra < 16 * (2 * 255 - 1) + 256
    with pytest.raises(B.MctdhbError):
        B.Batch.job_bytes(job(300, periodic=0), 5)
    with pytest.raises(B.MctdhbError):
        B.Batch.job_bytes(job(303), 5)
