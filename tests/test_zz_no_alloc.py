"""mctdhb_dev_density_matrices_noalloc: rho1 and rho2 for callers that cannot
let a library allocate device memory (a process whose device memory belongs
to its own pool allocator, or a loop that cannot pay for the synchronisation
of cudaMalloc/cudaFree).  All its scratch is one static device array of the
library, shared by every call.

The entry point is called through the C ABI and checked against
mctdhb_dev_density_matrices (which owns its scratch through an mctdhb_space)
and against the oracle, on two calls in a row, with a different coefficient
vector each time, so the second call sees the array as the first one left
it.  This file is named
to be collected last: the array then holds whatever earlier tests' calls
left in it, and the test also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from helpers import rand_coef, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the density tolerance of the other GPU parity tests

# register-resident kernels (norb <= 8, including the largest space, whose
# grid is capped below the other entry point's) and the generic kernel
SIZES = [(10, 4), (30, 8), (12, 6), (2, 2), (4, 9), (6, 1)]


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _densities(L, fn_args, M, noalloc):
    import torch

    r1 = torch.full((M * M,), float("nan"), dtype=torch.complex128, device="cuda")
    r2 = torch.full((M ** 4,), float("nan"), dtype=torch.complex128, device="cuda")
    if noalloc:
        N, coef = fn_args
        rc = L.mctdhb_dev_density_matrices_noalloc(N, M, _ptr(coef), _ptr(r1), _ptr(r2),
                                                   _stream())
    else:
        h, coef = fn_args
        rc = L.mctdhb_dev_density_matrices(h, _ptr(coef), _ptr(r1), _ptr(r2), _stream())
    assert rc == 0, L.mctdhb_gpu_last_error().decode()
    torch.cuda.synchronize()
    return r1.cpu().numpy(), r2.cpu().numpy()


@pytest.mark.parametrize("N,M", SIZES)
def test_noalloc_matches_density_matrices(gpu, N, M):
    import torch

    L = gpu.load()
    h = C.c_void_p()
    assert L.mctdhb_space_create(N, M, C.byref(h)) == 0, L.mctdhb_gpu_last_error().decode()
    try:
        dim = L.mctdhb_space_dim(h)
        rng = np.random.default_rng(4100 + 31 * N + M)
        for call in range(2):  # two calls in a row on the shared array
            c = torch.from_numpy(rand_coef(rng, dim)).cuda()
            want1, want2 = _densities(L, (h, c), M, noalloc=False)
            got1, got2 = _densities(L, (N, c), M, noalloc=True)
            assert np.all(np.isfinite(got1)) and np.all(np.isfinite(got2)), f"call {call}"
            assert rel_err(got1, want1) < TOL, f"rho1, call {call}"
            assert rel_err(got2, want2) < TOL, f"rho2, call {call}"
            if 2 <= M <= 8:  # the same Gram kernels and block count: the same bits
                assert np.array_equal(got1, want1) and np.array_equal(got2, want2), call
    finally:
        L.mctdhb_space_destroy(h)


# against the oracle directly: the capped grid of the register-resident
# kernel (30, 6), and the generic kernel whose grid is set by what fits in
# the array (3 particles in 20 orbitals; 2 in 25, the largest norb that fits)
ORACLE_SIZES = [(10, 4), (30, 6), (3, 20), (2, 25)]


@pytest.mark.parametrize("N,M", ORACLE_SIZES)
def test_noalloc_matches_oracle(gpu, oracle, N, M):
    import torch

    L = gpu.load()
    dim = oracle.dim(N, M)
    rng = np.random.default_rng(4300 + 31 * N + M)
    for call in range(2):
        c = rand_coef(rng, dim)
        got1, got2 = _densities(L, (N, torch.from_numpy(c).cuda()), M, noalloc=True)
        want1 = oracle.onebody_dm(N, M, c).reshape(-1)
        want2 = oracle.twobody_dm(N, M, c)
        assert rel_err(got1, want1) < TOL, f"rho1, call {call}"
        assert rel_err(got2, want2) < TOL, f"rho2, call {call}"


def test_noalloc_rejects_oversize_and_null(gpu):
    """checked on the host before any launch"""
    import torch

    L = gpu.load()
    c = torch.zeros(16, dtype=torch.complex128, device="cuda")
    r = torch.zeros(16, dtype=torch.complex128, device="cuda")
    # 5 particles in 30 orbitals: 278,256 configurations, but 191,025
    # density elements whose partial sums exceed the fixed array
    rc = L.mctdhb_dev_density_matrices_noalloc(5, 30, _ptr(c), _ptr(r), _ptr(r), _stream())
    assert rc == -1
    assert "MCTDHB_NOALLOC_SCRATCH_BYTES" in L.mctdhb_gpu_last_error().decode()
    rc = L.mctdhb_dev_density_matrices_noalloc(5, 3, None, _ptr(r), _ptr(r), _stream())
    assert rc == -1 and "null" in L.mctdhb_gpu_last_error().decode()
    L.mctdhb_gpu_clear_error()
