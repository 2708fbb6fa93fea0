"""ctypes mirror of include/mctdhb_types.h (the reference's public C types,
include/mctdhb_types.h:136-240 of andriati-alex/1d-mctdhb).

The same layout is shared by the reference library and libmctdhb_b200.so,
so Python callers (tests, bench) can build the structs once and hand them
to either library.  Helpers convert between numpy arrays and the
reference's `Carray` / row-pointer `Cmatrix` conventions.
"""
import ctypes as C

import numpy as np

STR_BUFF_SIZE = 128

IMAGTIME, REALTIME = 10, 11
LANCZOS, RUNGEKUTTA = 20, 21
FULLSTEP_RUNGEKUTTA, SPLITSTEP = 30, 31
DVR, SPECTRAL, FINITEDIFF = 300, 301, 302
RK2, RK4, RK5 = 2, 4, 5
ZERO_BOUNDS, PERIODIC_BOUNDS = 1000, 1001


class dcomplex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]

    @classmethod
    def of(cls, z):
        z = complex(z)
        return cls(z.real, z.imag)

    def value(self):
        return complex(self.re, self.im)


Carray = C.POINTER(dcomplex)
Cmatrix = C.POINTER(Carray)
Rarray = C.POINTER(C.c_double)

single_particle_pot = C.CFUNCTYPE(None, C.c_double, C.c_uint16, Rarray, C.c_void_p, Rarray)
time_dependent_parameter = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)


class OrbitalEquationS(C.Structure):
    _fields_ = [
        ("eq_name", C.c_char * STR_BUFF_SIZE),
        ("norb", C.c_uint16), ("grid_size", C.c_uint16),
        ("bounds", C.c_int),
        ("t", C.c_double), ("xi", C.c_double), ("xf", C.c_double), ("dx", C.c_double),
        ("tstep", C.c_double), ("tend", C.c_double), ("g", C.c_double), ("d2coef", C.c_double),
        ("d1coef", dcomplex), ("prop_dt", dcomplex), ("time_fac", dcomplex),
        ("grid_pts", Rarray), ("pot_grid", Rarray),
        ("pot_extra_args", C.c_void_p), ("inter_extra_args", C.c_void_p),
        ("pot_func", C.c_void_p), ("inter_param", C.c_void_p),
    ]


class OperatorMappingsS(C.Structure):
    _fields_ = [("map", C.POINTER(C.c_uint32)), ("mapot", C.POINTER(C.c_uint32)),
                ("maptt", C.POINTER(C.c_uint32)), ("strideot", C.POINTER(C.c_uint32)),
                ("stridett", C.POINTER(C.c_uint32))]


class MultiConfigurationS(C.Structure):
    _fields_ = [("npar", C.c_uint16), ("norb", C.c_uint16), ("dim", C.c_uint32),
                ("hash_table", C.POINTER(C.c_uint16)),
                ("subspaces_dim", C.POINTER(C.c_uint32)),
                ("op_maps", C.POINTER(OperatorMappingsS))]


class ManyBodyStateS(C.Structure):
    _fields_ = [("npar", C.c_uint16), ("norb", C.c_uint16), ("grid_size", C.c_uint16),
                ("space_dim", C.c_uint32),
                ("coef", Carray), ("hint", Carray), ("tb_denmat", Carray),
                ("hob", Cmatrix), ("orbitals", Cmatrix), ("ob_denmat", Cmatrix),
                ("inv_ob_denmat", Cmatrix)]


class WorkspaceLanczosS(C.Structure):
    _fields_ = [("iter", C.c_uint16), ("space_dim", C.c_uint32),
                ("lanczos_vectors", Cmatrix),
                ("decomp_diag", Carray), ("decomp_offd", Carray), ("coef_lspace", Carray),
                ("transform", Carray), ("hc", Carray), ("reortho", Carray),
                ("lapack_diag", Rarray), ("lapack_offd", Rarray), ("lapack_eigvec", Rarray)]


class OrbitalWorkspaceS(C.Structure):
    _fields_ = [("norb", C.c_uint16), ("grid_size", C.c_uint16),
                ("orb_der_method", C.c_int), ("impr_ortho", C.c_int),
                ("dvr_mat", Carray), ("cn_upper", Carray), ("cn_lower", Carray),
                ("cn_mid", Carray), ("cn_rhs", Carray),
                ("orb_work1", Cmatrix), ("orb_work2", Cmatrix),
                ("extern_work", C.c_void_p), ("fft_desc", C.c_void_p),
                ("fft_freq", Rarray), ("fft_hder_exp", Carray)]


class CoefWorkspaceS(C.Structure):
    _fields_ = [("lan_work", C.POINTER(WorkspaceLanczosS)), ("extern_work", C.c_void_p)]


class MCTDHBDataStructS(C.Structure):
    _fields_ = [("integ_type", C.c_int), ("coef_integ_method", C.c_int),
                ("orb_integ_method", C.c_int), ("orb_der_method", C.c_int),
                ("rk_order", C.c_int),
                ("multiconfig_space", C.POINTER(MultiConfigurationS)),
                ("orb_eq", C.POINTER(OrbitalEquationS)),
                ("coef_workspace", C.POINTER(CoefWorkspaceS)),
                ("orb_workspace", C.POINTER(OrbitalWorkspaceS)),
                ("state", C.POINTER(ManyBodyStateS))]


MultiConfiguration = C.POINTER(MultiConfigurationS)
ManyBodyState = C.POINTER(ManyBodyStateS)
MCTDHBDataStruct = C.POINTER(MCTDHBDataStructS)
OrbitalEquation = C.POINTER(OrbitalEquationS)


def carray(a):
    """Pointer to a contiguous complex128 numpy array, as a `Carray`."""
    assert a.dtype == np.complex128 and a.flags.c_contiguous
    return a.ctypes.data_as(Carray)


class RowMatrix:
    """A `Cmatrix` (array of row pointers) over the rows of a 2-D complex
    numpy array; keeps the array alive while the pointer is in use."""

    def __init__(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        self.a = a
        self.rows = (Carray * a.shape[0])(*[carray(a[i]) for i in range(a.shape[0])])
        self.ptr = C.cast(self.rows, Cmatrix)


def cmatrix_to_numpy(m, nrows, ncols):
    out = np.empty((nrows, ncols), dtype=np.complex128)
    for i in range(nrows):
        buf = C.cast(m[i], C.POINTER(C.c_double * (2 * ncols))).contents
        out[i] = np.frombuffer(buf, dtype=np.complex128, count=ncols)
    return out


def carray_to_numpy(p, n):
    buf = C.cast(p, C.POINTER(C.c_double * (2 * n))).contents
    return np.frombuffer(buf, dtype=np.complex128, count=n).copy()


def uint_array_to_numpy(p, n, dtype):
    ct = {np.uint16: C.c_uint16, np.uint32: C.c_uint32}[dtype]
    buf = C.cast(p, C.POINTER(ct * n)).contents
    return np.frombuffer(buf, dtype=dtype, count=n).copy()
