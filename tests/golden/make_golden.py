"""Generates the golden vectors in tests/golden/*.npz from the reference
itself: its own C sources compiled into oracle/_ref/libmctdhb_ref.so
(`make -C oracle ref`, reads the reference tree, so run it where the
reference source is present).  Inputs are seeded and stored with the
outputs, so the fixtures are self-contained.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
from oracle import Reference  # noqa: E402

CASES = [  # (npar, norb, seed, lanczos m)
    (10, 4, 1, 5),   # the N=10, M=4 relaxation size
    (6, 5, 2, 6),
    (12, 6, 3, 6),
    (3, 8, 4, 5),
    (5, 3, 5, 4),
    (2, 2, 6, 3),
]


def rand_inputs(rng, N, M, nc):
    c = rng.normal(size=nc) + 1j * rng.normal(size=nc)
    c /= np.linalg.norm(c)
    h = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    h = (h + h.conj().T) / 2
    g = rng.normal(size=M ** 4) + 1j * rng.normal(size=M ** 4)  # no symmetry assumed
    return c, h, g


def physical_g(rng, M, G=64):
    """index-symmetric g_{abcd} = sum_x w_x conj(f_a f_b) f_c f_d"""
    f = rng.normal(size=(M, G)) + 1j * rng.normal(size=(M, G))
    w = rng.uniform(0.5, 1.5, size=G)
    return _g_ref_layout(f, w, M)


def _g_ref_layout(f, w, M):
    # hint[a + b M + c M^2 + d M^3] = sum_x w conj(f_a f_b) f_c f_d
    t = np.einsum("x,ax,bx,cx,dx->abcd", w, f.conj(), f.conj(), f, f)
    out = np.zeros(M ** 4, np.complex128)
    for a in range(M):
        for b in range(M):
            for c in range(M):
                for d in range(M):
                    out[a + b * M + c * M * M + d * M ** 3] = t[a, b, c, d]
    return out


def main():
    R = Reference()
    for N, M, seed, m in CASES:
        rng = np.random.default_rng(seed)
        mc = R.multiconf(N, M)
        nc = mc.contents.dim
        ht, mp, st_tt, st_ot = R.maps(mc)
        om = mc.contents.op_maps.contents
        # double-map lengths: last stride + chunks of the last configuration
        n_tt = int(st_tt[-1]) + M * M * int(np.count_nonzero(ht[-M:]) * (np.count_nonzero(ht[-M:]) - 1) // 2)
        n_ot = int(st_ot[-1]) + M * M * int(np.count_nonzero(ht[-M:] > 1))
        maptt = np.ctypeslib.as_array(om.maptt, shape=(max(n_tt, 1),)).copy()[:n_tt]
        mapot = np.ctypeslib.as_array(om.mapot, shape=(max(n_ot, 1),)).copy()[:n_ot]
        c, h, g = rand_inputs(rng, N, M, nc)
        hc = R.apply_hamiltonian(mc, c, h, g)
        rho1 = R.onebody_dm(mc, c)
        rho2 = R.twobody_dm(mc, c)
        gp = physical_g(rng, M)
        hcp = R.apply_hamiltonian(mc, c, h, gp)
        it, diag, offd, lvec = R.lanczos(mc, h, gp, m, c)
        e0, c0 = R.lowest_state_lanczos(mc, h, gp, min(2 * m, nc), c)
        np.savez_compressed(
            os.path.join(HERE, f"ref_N{N}_M{M}.npz"),
            npar=N, norb=M, seed=seed, m=m,
            hash_table=ht, map=mp, stridett=st_tt, strideot=st_ot, maptt=maptt, mapot=mapot,
            coef=c, hob=h, hint=g, hc=hc, rho1=rho1, rho2=rho2,
            hint_phys=gp, hc_phys=hcp,
            lanczos_iters=it, lanczos_diag=diag[:it], lanczos_offd=offd[: max(it - 1, 0)],
            lanczos_vecs=lvec[:it], lowest_e=e0, lowest_c=c0, lowest_m=min(2 * m, nc),
        )
        R.lib.destroy_multiconf_struct(mc)
        print(f"N={N} M={M} nc={nc} lanczos it={it} E0={e0:.12f}")


if __name__ == "__main__":
    main()
