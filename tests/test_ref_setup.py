"""The set-up harness of the compiled reference (oracle/ref_setup.c), which
the bench uses to time the reference's own step on many jobs: a struct
built from the reference's sub-constructors with maps from the oracle's
OpenMP builders must step exactly like one from the reference's own
get_mctdhb_struct (types_definition.c:247-300), bit for bit.  CPU only."""
import ctypes as C

import numpy as np
import pytest

from helpers import rand_coef
from oracle import hermite_orbitals


def job(N, M, G, imag, dt, g, seed, dw=False):
    x = np.linspace(-8.0, 8.0, G)
    pot = 0.5 * x ** 2 + (4.0 * np.exp(-x ** 2 / 0.5) if dw else 0.0)
    return {"npar": N, "norb": M, "grid_size": G, "xi": -8.0, "xf": 8.0, "periodic": 1,
            "imagtime": int(imag), "rk_order": 5, "dt": dt, "g": g, "pot": pot, "seed": seed}


def maps_of(reference, mc, nc, M):
    import mctdhb_types as T

    s = mc.contents
    om = s.op_maps.contents
    tt = int(om.stridett[nc - 1]) + M * M * M * M  # bound: last row's chunks
    ot = int(om.strideot[nc - 1]) + M * M * M * M
    return [T.uint_array_to_numpy(s.hash_table, nc * M, np.uint16),
            T.uint_array_to_numpy(om.map, nc * M * M, np.uint32),
            T.uint_array_to_numpy(om.stridett, nc, np.uint32),
            T.uint_array_to_numpy(om.strideot, nc, np.uint32),
            T.uint_array_to_numpy(s.subspaces_dim, (s.npar + 1) * (s.norb + 1), np.uint32)]


@pytest.mark.parametrize("N,M", [(5, 3), (8, 4), (6, 6)])
def test_harness_maps_equal_reference_maps(reference, N, M):
    a = reference.multiconf(N, M)
    b = reference.lib.refset_multiconf(N, M)
    try:
        nc = a.contents.dim
        assert b.contents.dim == nc
        for x, y in zip(maps_of(reference, a, nc, M), maps_of(reference, b, nc, M)):
            assert np.array_equal(x, y)
    finally:
        reference.lib.destroy_multiconf_struct(a)
        reference.lib.destroy_multiconf_struct(b)


# real time re-evaluates the trap every step through the struct's own
# callback (driver.c:175-177), so the real-time case keeps the reference
# constructor's harmonic trap on both sides
@pytest.mark.parametrize("N,M,G,imag,dw", [(5, 3, 64, True, False), (6, 4, 96, False, False),
                                           (6, 4, 96, True, True)])
def test_harness_struct_steps_like_reference_struct(reference, N, M, G, imag, dw):
    """same inputs through both set-ups, three reference steps each: every
    array of the state is identical.  On one OpenMP thread: the reference's
    OpenMP reductions combine partial sums in no fixed order, so two runs of
    one struct on several threads already differ at the rounding level."""
    omp_threads = reference.lib.omp_get_max_threads()
    reference.lib.omp_set_num_threads(1)
    try:
        _steps_equal(reference, N, M, G, imag, dw)
    finally:
        reference.lib.omp_set_num_threads(omp_threads)


def _steps_equal(reference, N, M, G, imag, dw):
    j = job(N, M, G, imag, 0.005, 0.4, 7, dw)
    orb, _ = hermite_orbitals(M, G, j["xi"], j["xf"])
    coef = rand_coef(np.random.default_rng(11), reference.lib.space_dimension(N, M))
    A, keep = reference.make_mctdhb(N, M, G, j["xi"], j["xf"], imag, 5, 5, j["dt"], 1.0, j["g"])
    pot = np.ctypeslib.as_array(A.contents.orb_eq.contents.pot_grid, shape=(G,))
    if dw:  # the reference constructor's trap is harmonic: give it the job's
        pot[:] = j["pot"]
    else:  # the harmonic trap exactly as the reference's builtin evaluates it
        j["pot"] = pot.copy()
    B = reference.make_job_struct(j, 5)
    try:
        reference.set_state(A, orb, coef)
        reference.set_state(B, orb, coef)
        for k in range(3):
            reference.step(A, k)
            reference.step(B, k)
        a, b = reference.get_state(A), reference.get_state(B)
        for key in ("orb", "coef", "hob", "hint", "rho1", "rho2", "rinv", "pot"):
            assert np.array_equal(a[key], b[key]), key
    finally:
        reference.destroy_mctdhb(A)
        reference.destroy_job_struct(B)


def test_harness_refuses_what_the_reference_cannot_map(reference):
    """N=30, M=8: the reference's double-jump map overflows its 32-bit
    strides (space.c:285-289), the harness returns None"""
    assert reference.lib.refset_multiconf(30, 8) is None or \
        not reference.lib.refset_multiconf(30, 8)
