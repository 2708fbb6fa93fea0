"""Python access to the two CPU checkers of the GPU library.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / `--impl reference` legs.  Nothing in the GPU
product path imports this module.

* `Oracle`     -- liboracle.so, the C restatement in oracle.c (OpenMP).
* `Reference`  -- _ref/libmctdhb_ref.so, the reference's own C sources
                  compiled unmodified against the shim headers in shim/.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "1d-mctdhb_b200"))
import mctdhb_types as T  # noqa: E402

ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmctdhb_ref.so")

_c128p = np.ctypeslib.ndpointer(np.complex128, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


class _C128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _c(z):
    z = complex(z)
    return _C128(z.real, z.imag)


def cvec(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


class Oracle:
    """ctypes binding of oracle.h (row-major matrices, complex128)."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        i, u64 = C.c_int, C.c_uint64
        L.orc_space_dimension.restype = u64
        L.orc_space_dimension.argtypes = [i, i]
        L.orc_rank.restype = u64
        L.orc_rank.argtypes = [i, i, _u16p]
        L.orc_unrank.argtypes = [i, i, u64, _u16p]
        L.orc_subspaces_dim.argtypes = [i, i, _u32p]
        L.orc_hash_table.argtypes = [i, i, _u16p]
        L.orc_single_jump_map.argtypes = [i, i, _u32p]
        L.orc_double_diffjump_chunks.restype = u64
        L.orc_double_diffjump_chunks.argtypes = [i, i]
        L.orc_double_equaljump_chunks.restype = u64
        L.orc_double_equaljump_chunks.argtypes = [i, i]
        L.orc_double_diffjump_map.argtypes = [i, i, _u64p, _u32p]
        L.orc_double_equaljump_map.argtypes = [i, i, _u64p, _u32p]
        L.orc_apply_hamiltonian.argtypes = [i, i, _c128p, _c128p, _c128p, _c128p]
        L.orc_apply_hamiltonian_rows.argtypes = [i, i, _c128p, _c128p, _c128p, _c128p, u64, u64]
        L.orc_onebody_dm.argtypes = [i, i, _c128p, _c128p]
        L.orc_twobody_dm.argtypes = [i, i, _c128p, _c128p]
        L.orc_twobody_dm_rows.argtypes = [i, i, _c128p, _c128p, u64, u64]
        L.orc_tridiag_eig.restype = i
        L.orc_tridiag_eig.argtypes = [i, _f64p, _f64p, _f64p]
        L.orc_lanczos.restype = i
        L.orc_lanczos.argtypes = [i, i, _c128p, _c128p, i, _c128p, _c128p, _c128p]
        L.orc_sil_step.restype = i
        L.orc_sil_step.argtypes = [i, i, _c128p, _c128p, i, _C128, i, _c128p, _c128p]
        L.orc_lowest_state_lanczos.restype = C.c_double
        L.orc_lowest_state_lanczos.argtypes = [i, i, _c128p, _c128p, i, _c128p, _c128p]
        L.orc_total_energy.restype = _C128
        L.orc_total_energy.argtypes = [i, _c128p, _c128p, _c128p, _c128p]
        L.orc_eig_residual.restype = C.c_double
        L.orc_eig_residual.argtypes = [i, i, _c128p, _c128p, _c128p, C.c_double]
        L.orc_simpson.restype = _C128
        L.orc_simpson.argtypes = [i, C.c_double, _c128p]
        L.orc_dxfd.argtypes = [i, C.c_double, _c128p, _c128p]
        L.orc_orbital_hob.argtypes = [i, i, C.c_double, C.c_double, _C128, _f64p, _c128p, _c128p]
        L.orc_orbital_hint.argtypes = [i, i, C.c_double, C.c_double, _c128p, _c128p]
        L.orc_orthonormalize.argtypes = [i, C.c_double, i, _c128p]
        L.orc_herm_eig.restype = i
        L.orc_herm_eig.argtypes = [i, _c128p, _f64p, C.c_void_p]
        L.orc_herm_inverse.restype = i
        L.orc_herm_inverse.argtypes = [i, _c128p, _c128p]
        L.orc_sync_density_matrices.argtypes = [i, i, _c128p, C.c_double, _c128p, _c128p, _c128p]
        L.orc_linear_half_step.argtypes = [i, i, C.c_double, C.c_double, _C128, i, _C128,
                                           _c128p]
        L.orc_orbital_rhs.restype = i
        L.orc_orbital_rhs.argtypes = [i, i, C.c_double, C.c_double, _C128, C.c_double, i, _C128,
                                      _f64p, _c128p, _c128p, _c128p, _c128p, i, i]
        L.orc_propagate_step.argtypes = [i, i, i, C.c_double, C.c_double, C.c_double, _C128,
                                         C.c_double, i, i, i, i, C.c_double, _f64p,
                                         _c128p, _c128p, _c128p, _c128p, _c128p, _c128p, _c128p, i,
                                         i, i, i]

    # ---- space -------------------------------------------------------
    def dim(self, N, M):
        return int(self.lib.orc_space_dimension(N, M))

    def rank(self, N, M, occ):
        return int(self.lib.orc_rank(N, M, np.ascontiguousarray(occ, dtype=np.uint16)))

    def unrank(self, N, M, idx):
        o = np.zeros(M, np.uint16)
        self.lib.orc_unrank(N, M, idx, o)
        return o

    def subspaces_dim(self, N, M):
        o = np.zeros((N + 1) * (M + 1), np.uint32)
        self.lib.orc_subspaces_dim(N, M, o)
        return o

    def hash_table(self, N, M):
        ht = np.zeros(self.dim(N, M) * M, np.uint16)
        self.lib.orc_hash_table(N, M, ht)
        return ht

    def single_jump_map(self, N, M):
        m = np.zeros(self.dim(N, M) * M * M, np.uint32)
        self.lib.orc_single_jump_map(N, M, m)
        return m

    def double_diffjump_map(self, N, M):
        nc = self.dim(N, M)
        ch = int(self.lib.orc_double_diffjump_chunks(N, M))
        st = np.zeros(nc, np.uint64)
        m = np.zeros(max(ch, 1) * M * M, np.uint32)
        self.lib.orc_double_diffjump_map(N, M, st, m)
        return st, m[: ch * M * M]

    def double_equaljump_map(self, N, M):
        nc = self.dim(N, M)
        ch = int(self.lib.orc_double_equaljump_chunks(N, M))
        st = np.zeros(nc, np.uint64)
        m = np.zeros(max(ch, 1) * M * M, np.uint32)
        self.lib.orc_double_equaljump_map(N, M, st, m)
        return st, m[: ch * M * M]

    # ---- configurational kernels -------------------------------------
    def apply_hamiltonian(self, N, M, c, hob, hint, rows=None):
        c, hob, hint = cvec(c), cvec(hob).reshape(-1), cvec(hint).reshape(-1)
        out = np.zeros_like(c)
        if rows is None:
            self.lib.orc_apply_hamiltonian(N, M, c, hob, hint, out)
        else:
            self.lib.orc_apply_hamiltonian_rows(N, M, c, hob, hint, out, rows[0], rows[1])
        return out

    def onebody_dm(self, N, M, c):
        r = np.zeros(M * M, np.complex128)
        self.lib.orc_onebody_dm(N, M, cvec(c), r)
        return r.reshape(M, M)

    def twobody_dm(self, N, M, c, rows=None):
        r = np.zeros(M ** 4, np.complex128)
        if rows is None:
            self.lib.orc_twobody_dm(N, M, cvec(c), r)
        else:
            self.lib.orc_twobody_dm_rows(N, M, cvec(c), r, rows[0], rows[1])
        return r

    def tridiag_eig(self, d, e):
        n = len(d)
        d = np.array(d, np.float64)
        e2 = np.zeros(n, np.float64)
        e2[: n - 1] = e[: n - 1]
        z = np.zeros(n * n, np.float64)
        info = self.lib.orc_tridiag_eig(n, d, e2, z)
        return info, d, z.reshape(n, n)

    def lanczos(self, N, M, hob, hint, m, c0):
        nc = self.dim(N, M)
        lvec = np.zeros(m * nc, np.complex128)
        lvec[:nc] = c0
        diag = np.zeros(m, np.complex128)
        offd = np.zeros(m, np.complex128)
        it = self.lib.orc_lanczos(N, M, cvec(hob).reshape(-1), cvec(hint).reshape(-1), m,
                                  diag, offd, lvec)
        return it, diag, offd, lvec.reshape(m, nc)

    def sil_step(self, N, M, hob, hint, m, dt, imagtime, c):
        c = cvec(c).copy()
        nc = self.dim(N, M)
        work = np.zeros(m * nc, np.complex128)
        pdt = -1j * dt if imagtime else dt
        it = self.lib.orc_sil_step(N, M, cvec(hob).reshape(-1), cvec(hint).reshape(-1), m,
                                   _c(pdt), int(imagtime), c, work)
        return it, c

    def lowest_state_lanczos(self, N, M, hob, hint, m, c):
        c = cvec(c).copy()
        work = np.zeros(m * self.dim(N, M), np.complex128)
        e = self.lib.orc_lowest_state_lanczos(N, M, cvec(hob).reshape(-1),
                                              cvec(hint).reshape(-1), m, c, work)
        return e, c

    def total_energy(self, M, rho1, rho2, hob, hint):
        r = self.lib.orc_total_energy(M, cvec(rho1).reshape(-1), cvec(rho2).reshape(-1),
                                      cvec(hob).reshape(-1), cvec(hint).reshape(-1))
        return complex(r.re, r.im)

    def eig_residual(self, N, M, c, hob, hint, e):
        return self.lib.orc_eig_residual(N, M, cvec(c), cvec(hob).reshape(-1),
                                         cvec(hint).reshape(-1), e)

    # ---- orbital side ------------------------------------------------
    def simpson(self, h, f):
        r = self.lib.orc_simpson(len(f), h, cvec(f))
        return complex(r.re, r.im)

    def dxfd(self, dx, f):
        out = np.zeros(len(f), np.complex128)
        self.lib.orc_dxfd(len(f), dx, cvec(f), out)
        return out

    def orbital_hob(self, orb, dx, d2coef, d1coef, pot):
        M, G = orb.shape
        h = np.zeros(M * M, np.complex128)
        self.lib.orc_orbital_hob(M, G, dx, d2coef, _c(d1coef),
                                 np.ascontiguousarray(pot, np.float64), cvec(orb).reshape(-1), h)
        return h.reshape(M, M)

    def orbital_hint(self, orb, dx, g):
        M, G = orb.shape
        h = np.zeros(M ** 4, np.complex128)
        self.lib.orc_orbital_hint(M, G, dx, g, cvec(orb).reshape(-1), h)
        return h

    def orthonormalize(self, orb, dx):
        o = cvec(orb).copy()
        M, G = o.shape
        self.lib.orc_orthonormalize(G, dx, M, o.reshape(-1))
        return o

    def herm_eig(self, a):
        n = a.shape[0]
        w = np.zeros(n)
        v = np.zeros(n * n, np.complex128)
        self.lib.orc_herm_eig(n, cvec(a).reshape(-1), w, v.ctypes.data_as(C.c_void_p))
        return w, v.reshape(n, n)

    def herm_inverse(self, a):
        n = a.shape[0]
        inv = np.zeros(n * n, np.complex128)
        info = self.lib.orc_herm_inverse(n, cvec(a).reshape(-1), inv)
        return info, inv.reshape(n, n)

    def sync_density_matrices(self, N, M, c, reg_fac=1e-9):
        r1 = np.zeros(M * M, np.complex128)
        r2 = np.zeros(M ** 4, np.complex128)
        ri = np.zeros(M * M, np.complex128)
        self.lib.orc_sync_density_matrices(N, M, cvec(c), reg_fac, r1, r2, ri)
        return r1.reshape(M, M), r2, ri.reshape(M, M)

    def orbital_rhs(self, orb, dx, d2coef, d1coef, g, periodic, time_fac, pot, rinv, rho2,
                    robust=False, der=302):
        """der: 302 finite differences, 300 DVR, 301 spectral"""
        M, G = orb.shape
        out = np.zeros(M * G, np.complex128)
        info = self.lib.orc_orbital_rhs(M, G, dx, d2coef, _c(d1coef), g, int(periodic),
                                        _c(time_fac), np.ascontiguousarray(pot, np.float64),
                                        cvec(rinv).reshape(-1), cvec(rho2).reshape(-1),
                                        cvec(orb).reshape(-1), out, int(robust), int(der))
        if info:
            raise ValueError(f"singular overlap matrix (column {info - 1})")
        return out.reshape(M, G)

    def linear_half_step(self, der, f, dx, d2coef, d1coef, periodic, dth):
        f = cvec(f).copy()
        self.lib.orc_linear_half_step(int(der), len(f), dx, d2coef, _c(d1coef), int(periodic),
                                      _c(dth), f)
        return f

    def propagate_step(self, st, N, dx, dt, d2coef, d1coef, g, periodic, imagtime, rk_order,
                       lanczos_m, pot, reg_fac=1e-9, robust=False, der=302, coef_method=20,
                       orb_method=30):
        """One full step; `st` is a dict of numpy arrays updated in place:
        orb (M,G), coef, hob (M,M), hint, rho1 (M,M), rho2, rinv (M,M)."""
        M, G = st["orb"].shape
        args = [st[k] for k in ("orb", "coef", "hob", "hint", "rho1", "rho2", "rinv")]
        for a in args:
            assert a.dtype == np.complex128 and a.flags.c_contiguous
        self.lib.orc_propagate_step(N, M, G, dx, dt, d2coef, _c(d1coef), g, int(periodic),
                                    int(imagtime), rk_order, lanczos_m, reg_fac,
                                    np.ascontiguousarray(pot, np.float64),
                                    *[a.reshape(-1) for a in args], int(robust), int(der),
                                    int(coef_method), int(orb_method))


class Reference:
    """ctypes binding of the compiled reference (its own C API)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        L = self.lib = C.CDLL(path)
        L.space_dimension.restype = C.c_uint32
        L.space_dimension.argtypes = [C.c_uint16, C.c_uint16]
        L.get_multiconf_struct.restype = T.MultiConfiguration
        L.get_multiconf_struct.argtypes = [C.c_uint16, C.c_uint16]
        L.destroy_multiconf_struct.argtypes = [T.MultiConfiguration]
        L.apply_hamiltonian.argtypes = [T.MultiConfiguration, T.Carray, T.Cmatrix, T.Carray,
                                        T.Carray]
        L.set_onebody_dm.argtypes = [T.MultiConfiguration, T.Carray, T.Cmatrix]
        L.set_twobody_dm.argtypes = [T.MultiConfiguration, T.Carray, T.Carray]
        L.lanczos.restype = C.c_int
        L.lanczos.argtypes = [T.MultiConfiguration, T.Cmatrix, T.Carray, C.c_int, T.Carray,
                              T.Carray, T.Cmatrix]
        L.lowest_state_lanczos.restype = C.c_double
        L.lowest_state_lanczos.argtypes = [C.c_uint16, T.MultiConfiguration, T.Cmatrix,
                                           T.Carray, T.Carray]
        L.get_mctdhb_struct.restype = T.MCTDHBDataStruct
        L.get_mctdhb_struct.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint16,
                                        C.c_uint16, C.c_uint16, C.c_char_p, C.c_int, C.c_double,
                                        C.c_double, C.c_uint16, C.c_double, C.c_double,
                                        C.c_double, T.dcomplex, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
        L.destroy_mctdhb_struct.argtypes = [T.MCTDHBDataStruct]
        L.propagate_coef_sil.argtypes = [T.MCTDHBDataStruct, T.Carray]
        L.sync_density_matrices.argtypes = [T.MultiConfiguration, T.ManyBodyState]
        L.sync_orbital_matrices.argtypes = [T.OrbitalEquation, T.ManyBodyState]
        L.mctdhb_propagate_step.argtypes = [T.MCTDHBDataStruct, T.Carray, T.Carray, C.c_uint32]
        L.total_energy.restype = T.dcomplex
        L.total_energy.argtypes = [T.ManyBodyState]
        L.eig_residual.restype = C.c_double
        L.eig_residual.argtypes = [T.MultiConfiguration, T.Carray, T.Cmatrix, T.Carray,
                                   C.c_double]
        L.orthonormalize.argtypes = [C.c_uint32, C.c_double, C.c_uint32, T.Cmatrix]
        L.Csimps.restype = T.dcomplex
        L.Csimps.argtypes = [C.c_uint32, C.c_double, T.Carray]
        L.dxFD.argtypes = [C.c_uint32, C.c_double, T.Carray, T.Carray]
        # ref_setup.c: reference structs with maps from the oracle's builders
        L.refset_multiconf.restype = T.MultiConfiguration
        L.refset_multiconf.argtypes = [C.c_uint16, C.c_uint16]
        L.refset_mctdhb_struct.restype = T.MCTDHBDataStruct
        L.refset_mctdhb_struct.argtypes = [C.c_int] * 6 + [
            C.c_uint16, C.c_uint16, C.c_int, C.c_double, C.c_double, C.c_uint16, C.c_double,
            C.c_double, C.c_double, C.c_double, _f64p, C.c_double]
        L.refset_destroy.argtypes = [T.MCTDHBDataStruct]

    def multiconf(self, N, M):
        return self.lib.get_multiconf_struct(N, M)

    def maps(self, mc):
        s = mc.contents
        nc, M = s.dim, s.norb
        om = s.op_maps.contents
        ht = T.uint_array_to_numpy(s.hash_table, nc * M, np.uint16)
        mp = T.uint_array_to_numpy(om.map, nc * M * M, np.uint32)
        st_tt = T.uint_array_to_numpy(om.stridett, nc, np.uint32)
        st_ot = T.uint_array_to_numpy(om.strideot, nc, np.uint32)
        return ht, mp, st_tt, st_ot

    def apply_hamiltonian(self, mc, c, hob, hint):
        c, hint = cvec(c), cvec(hint).reshape(-1)
        out = np.zeros_like(c)
        H = T.RowMatrix(hob)
        self.lib.apply_hamiltonian(mc, T.carray(c), H.ptr, T.carray(hint), T.carray(out))
        return out

    def onebody_dm(self, mc, c):
        M = mc.contents.norb
        R = T.RowMatrix(np.zeros((M, M), np.complex128))
        self.lib.set_onebody_dm(mc, T.carray(cvec(c)), R.ptr)
        return R.a

    def twobody_dm(self, mc, c, fill=np.nan):
        M = mc.contents.norb
        r = np.full(M ** 4, fill, np.complex128)
        self.lib.set_twobody_dm(mc, T.carray(cvec(c)), T.carray(r))
        return r

    def lanczos(self, mc, hob, hint, m, c0):
        nc = mc.contents.dim
        lv = np.zeros((m, nc), np.complex128)
        lv[0] = c0
        L = T.RowMatrix(lv)
        diag = np.zeros(m, np.complex128)
        offd = np.zeros(m, np.complex128)
        H = T.RowMatrix(hob)
        hint = cvec(hint).reshape(-1)
        it = self.lib.lanczos(mc, H.ptr, T.carray(hint), m, T.carray(diag), T.carray(offd), L.ptr)
        return it, diag, offd, L.a

    def lowest_state_lanczos(self, mc, hob, hint, m, c):
        c = cvec(c).copy()
        H = T.RowMatrix(hob)
        hint = cvec(hint).reshape(-1)
        e = self.lib.lowest_state_lanczos(m, mc, H.ptr, T.carray(hint), T.carray(c))
        return e, c

    def fn(self, name):
        return C.cast(getattr(self.lib, name), C.c_void_p).value

    def make_mctdhb(self, N, M, G, xi, xf, imagtime, rk_order, lanczos_m, dt, omega, g,
                    periodic=True, omega_f=None, pot_period=0.0, g_f=None, g_period=0.0,
                    der=T.FINITEDIFF, coef=T.LANCZOS, orb=T.FULLSTEP_RUNGEKUTTA):
        """A reference MCTDHBDataStruct from its own constructor
        (types_definition.c:247): FULLSTEP_RUNGEKUTTA orbitals, `der`
        derivatives (FINITEDIFF by default), LANCZOS coefficients, harmonic trap
        (builtin_potential.c:37) swept omega -> omega_f over pot_period and
        g ramped g -> g_f over g_period (builtin_time_parameter.c:7); constant
        by default.  Returns (struct pointer, keep-alive list)."""
        L = self.lib
        pot_args = (C.c_double * 5)(omega, omega if omega_f is None else omega_f, pot_period,
                                    0.0, 0.0)
        g_args = (C.c_double * 5)(g, g if g_f is None else g_f, g_period, 0.0, 0.0)
        ms = L.get_mctdhb_struct(
            T.IMAGTIME if imagtime else T.REALTIME, coef, orb,
            der, rk_order, lanczos_m, N, M, b"harmonic",
            T.PERIODIC_BOUNDS if periodic else T.ZERO_BOUNDS, xi, xf, G, dt, 1.0, -0.5,
            T.dcomplex(0.0, 0.0), C.cast(pot_args, C.c_void_p), C.cast(g_args, C.c_void_p),
            self.fn("potfunc_harmonic"), self.fn("timeparam_linear_ramp"))
        return ms, [pot_args, g_args]

    def set_state(self, ms, orb, coef):
        """orbitals and coefficients into the struct, then the reference's
        own initial synchronisation (dataio.c full_setup)"""
        st = ms.contents.state.contents
        M, G = orb.shape
        for k in range(M):
            row = C.cast(st.orbitals[k], C.POINTER(C.c_double * (2 * G))).contents
            np.frombuffer(row, np.complex128)[:] = orb[k]
        cbuf = C.cast(st.coef, C.POINTER(C.c_double * (2 * len(coef)))).contents
        np.frombuffer(cbuf, np.complex128)[:] = coef
        self.lib.sync_orbital_matrices(ms.contents.orb_eq, ms.contents.state)
        self.lib.sync_density_matrices(ms.contents.multiconfig_space, ms.contents.state)

    def get_state(self, ms):
        st = ms.contents.state.contents
        M, G, nc = st.norb, st.grid_size, st.space_dim
        return {
            "orb": T.cmatrix_to_numpy(st.orbitals, M, G),
            "coef": T.carray_to_numpy(st.coef, nc),
            "hob": T.cmatrix_to_numpy(st.hob, M, M),
            "hint": T.carray_to_numpy(st.hint, M ** 4),
            "rho1": T.cmatrix_to_numpy(st.ob_denmat, M, M),
            "rho2": T.carray_to_numpy(st.tb_denmat, M ** 4),
            "rinv": T.cmatrix_to_numpy(st.inv_ob_denmat, M, M),
            "pot": np.ctypeslib.as_array(ms.contents.orb_eq.contents.pot_grid, shape=(G,)).copy(),
        }

    def step(self, ms, k):
        st = ms.contents.state.contents
        ow = np.zeros(st.norb * st.grid_size, np.complex128)
        cw = np.zeros(st.space_dim, np.complex128)
        self.lib.mctdhb_propagate_step(ms, T.carray(ow), T.carray(cw), k)
        return ow, cw

    def destroy_mctdhb(self, ms):
        self.lib.destroy_mctdhb_struct(ms)

    def make_job_struct(self, job, lanczos_m, der=T.FINITEDIFF, coef=T.LANCZOS,
                        orb=T.FULLSTEP_RUNGEKUTTA):
        """A reference MCTDHBDataStruct for a job dict (the batched engine's
        fields: npar, norb, grid_size, xi, xf, periodic, imagtime, rk_order,
        dt, g, pot), built by ref_setup.c: the reference's own
        sub-constructors with maps from the oracle's OpenMP builders, no DVR
        matrix unless der is DVR.  None where the reference's 32-bit map
        layout would overflow.  Free with destroy_job_struct."""
        d1 = complex(job.get("d1coef", 0j))
        ms = self.lib.refset_mctdhb_struct(
            int(job["imagtime"]), coef, orb, der, int(job["rk_order"]), lanczos_m,
            int(job["npar"]), int(job["norb"]), int(job.get("periodic", 1)), job["xi"], job["xf"],
            int(job["grid_size"]), job["dt"], job.get("d2coef", -0.5), d1.real, d1.imag,
            np.ascontiguousarray(job["pot"], np.float64), job["g"])
        return ms if ms else None

    def destroy_job_struct(self, ms):
        self.lib.refset_destroy(ms)


def hermite_orbitals(M, G, xi, xf):
    """Hermite-Gaussian orbitals n = 0..M-1 on the grid, Gram-Schmidt in
    the Simpson metric (the synthetic initial orbitals of the workloads)"""
    x = np.linspace(xi, xf, G)
    dx = x[1] - x[0]
    w = np.zeros(G)
    if G % 2 == 0:
        for i in range(0, G - 4, 2):
            w[i:i + 3] += [1, 4, 1]
        w[: G - 3] *= dx / 3
        w[G - 4:] += np.array([1, 3, 3, 1]) * 3 * dx / 8
    else:
        for i in range(0, G - 2, 2):
            w[i:i + 3] += [1, 4, 1]
        w *= dx / 3
    phi = np.zeros((M, G), np.complex128)
    hm, hc = np.zeros(G), np.exp(-x ** 2 / 2)
    for n in range(M):
        phi[n] = hc
        hm, hc = hc, (np.sqrt(2.0) * x * hc - np.sqrt(n) * hm) / np.sqrt(n + 1)
    for i in range(M):
        for j in range(i):
            phi[i] -= np.sum(w * phi[j].conj() * phi[i]) * phi[j]
        phi[i] /= np.sqrt(np.sum(w * np.abs(phi[i]) ** 2))
    return phi, dx
