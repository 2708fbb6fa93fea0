"""Seeded inputs and tolerance helpers shared by the tests."""
import numpy as np


def rand_coef(rng, nc):
    c = rng.normal(size=nc) + 1j * rng.normal(size=nc)
    return c / np.linalg.norm(c)


def rand_hob(rng, M):
    h = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    return (h + h.conj().T) / 2


def rand_hint(rng, M):
    """arbitrary complex g (no symmetry): exercises exactly which g elements
    each rule reads"""
    return rng.normal(size=M ** 4) + 1j * rng.normal(size=M ** 4)


def phys_hint(rng, M, G=48):
    """index-symmetric g[a + bM + cM^2 + dM^3] = sum_x w conj(f_a f_b) f_c f_d"""
    f = rng.normal(size=(M, G)) + 1j * rng.normal(size=(M, G))
    w = rng.uniform(0.5, 1.5, size=G)
    t = np.einsum("x,ax,bx,cx,dx->abcd", w, f.conj(), f.conj(), f, f)
    return np.ascontiguousarray(t.transpose(3, 2, 1, 0)).reshape(-1)


def rel_err(a, b):
    """max-norm error relative to the max-norm of the reference"""
    a, b = np.asarray(a), np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))
