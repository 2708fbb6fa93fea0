"""Python binding of libmctdhb_b200.so (include/mctdhb_gpu.h) via ctypes.

Two layers, mirroring the C ABI:

* `DropIn` -- the reference's own entry points (apply_hamiltonian,
  set_onebody_dm, set_twobody_dm, lanczos, lowest_state_lanczos,
  propagate_coef_sil, get_multiconf_struct, ...) called with host numpy
  buffers laid out as the reference's structs (mctdhb_types.py).
* `Space` -- the device-resident API on torch CUDA tensors (complex128),
  used for throughput work.

The product path has no CPU fallback: importing this module on a machine
without the built library raises, and every call checks the C status and
raises with the library's own error message.
"""
import ctypes as C
import os

import numpy as np

import mctdhb_types as T

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmctdhb_b200.so")

# every symbol include/mctdhb_gpu.h declares
EXPORTED = [
    "mctdhb_gpu_last_error", "mctdhb_gpu_clear_error",
    "space_dimension", "get_subspaces_dim", "set_config", "hash_index", "get_hash_table",
    "get_single_jump_map", "get_double_diffjump_map", "get_double_equaljump_map",
    "get_multiconf_struct", "destroy_multiconf_struct",
    "apply_hamiltonian", "set_onebody_dm", "set_twobody_dm",
    "lanczos", "lowest_state_lanczos", "propagate_coef_sil",
    "total_energy", "eig_residual",
    "mctdhb_space_create", "mctdhb_space_destroy", "mctdhb_space_dim",
    "mctdhb_dev_set_matrices", "mctdhb_dev_apply_hamiltonian", "mctdhb_dev_density_matrices",
    "mctdhb_dev_sil_step", "mctdhb_dev_hash_table", "mctdhb_dev_single_jump_map",
    "mctdhb_dev_double_jump_chunks", "mctdhb_dev_double_jump_map",
    "mctdhb_dev_density_matrices_noalloc",
    "mctdhb_batch_create", "mctdhb_batch_destroy", "mctdhb_batch_job_bytes",
    "mctdhb_batch_free_bytes", "mctdhb_batch_admit", "mctdhb_batch_step", "mctdhb_batch_sync",
    "mctdhb_batch_poll", "mctdhb_batch_fetch", "mctdhb_batch_release",
    "mctdhb_batch_monitor", "mctdhb_batch_lowest_state",
    "mctdhb_batch_kernel_count", "mctdhb_batch_stream", "mctdhb_batch_launch_hc",
    "mctdhb_batch_variant", "mctdhb_batch_set_variant", "mctdhb_tune_get", "mctdhb_tune_set",
    "mctdhb_fp64_mma_probe",
    "sync_density_matrices", "set_regulatization_factor", "get_current_regularization_factor",
    "mctdhb_step_create", "mctdhb_step_launch", "mctdhb_step_kernel_count",
    "mctdhb_solver_step_phase",
    "mctdhb_step_destroy",
    "set_orbital_hob", "set_orbital_hint", "sync_orbital_matrices", "mctdhb_propagate_step",
    "mctdhb_solver_create", "mctdhb_solver_destroy", "mctdhb_solver_set_potential",
    "mctdhb_solver_set_interaction", "mctdhb_solver_set_regularization",
    "mctdhb_solver_set_state", "mctdhb_solver_step", "mctdhb_solver_kernel_count",
    "mctdhb_solver_get", "mctdhb_solver_put", "mctdhb_solver_energy",
    "mctdhb_solver_device_coef", "mctdhb_solver_device_orbitals", "mctdhb_solver_time",
    "mctdhb_solver_set_orthogonality", "mctdhb_solver_overlap_residual",
    "mctdhb_solver_eig_residual", "mctdhb_solver_lowest_state", "mctdhb_solver_set_derivative",
    "mctdhb_solver_set_coef_method", "mctdhb_solver_set_orb_method",
    "mctdhb_solver_relax", "mctdhb_solver_relax_result", "mctdhb_solver_query",
]

_lib = None


class MctdhbError(RuntimeError):
    pass


class Job(C.Structure):
    """mctdhb_job of include/mctdhb_gpu.h (one system of the batched engine)"""
    _fields_ = [("npar", C.c_uint16), ("norb", C.c_uint16), ("grid_size", C.c_int),
                ("xi", C.c_double), ("xf", C.c_double), ("d2coef", C.c_double),
                ("d1coef_re", C.c_double), ("d1coef_im", C.c_double), ("periodic", C.c_int),
                ("imagtime", C.c_int), ("rk_order", C.c_int), ("dt", C.c_double),
                ("g", C.c_double), ("max_steps", C.c_uint32), ("energy_tol", C.c_double),
                ("check_every", C.c_int), ("reg_fac", C.c_double),
                ("pot", C.POINTER(C.c_double)), ("orbitals", C.c_void_p), ("coef", C.c_void_p),
                ("der_method", C.c_int), ("eig_tol", C.c_double), ("ortho_tol", C.c_double),
                ("impr_ortho", C.c_int), ("orb_method", C.c_int)]


def load(path=LIB_PATH):
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise MctdhbError(f"{path} is missing: build it with `python {HERE}/build.py`")
    L = C.CDLL(path, mode=C.RTLD_LOCAL)
    vp, u16, u32, i = C.c_void_p, C.c_uint16, C.c_uint32, C.c_int
    L.mctdhb_gpu_last_error.restype = C.c_char_p
    L.space_dimension.restype = u32
    L.space_dimension.argtypes = [u16, u16]
    L.get_subspaces_dim.restype = C.POINTER(u32)
    L.get_subspaces_dim.argtypes = [u16, u16]
    L.set_config.argtypes = [u32, u16, u16, C.POINTER(u16)]
    L.hash_index.restype = u32
    L.hash_index.argtypes = [u16, u16, C.POINTER(u32), C.POINTER(u16)]
    L.get_hash_table.restype = C.POINTER(u16)
    L.get_hash_table.argtypes = [u16, u16]
    L.get_single_jump_map.restype = C.POINTER(u32)
    L.get_single_jump_map.argtypes = [u16, u16, C.POINTER(u32), C.POINTER(u16)]
    for f in (L.get_double_diffjump_map, L.get_double_equaljump_map):
        f.restype = C.POINTER(u32)
        f.argtypes = [u16, u16, C.POINTER(u32), C.POINTER(u16), C.POINTER(u32)]
    L.get_multiconf_struct.restype = T.MultiConfiguration
    L.get_multiconf_struct.argtypes = [u16, u16]
    L.destroy_multiconf_struct.argtypes = [T.MultiConfiguration]
    L.apply_hamiltonian.argtypes = [T.MultiConfiguration, T.Carray, T.Cmatrix, T.Carray, T.Carray]
    L.set_onebody_dm.argtypes = [T.MultiConfiguration, T.Carray, T.Cmatrix]
    L.set_twobody_dm.argtypes = [T.MultiConfiguration, T.Carray, T.Carray]
    L.lanczos.restype = i
    L.lanczos.argtypes = [T.MultiConfiguration, T.Cmatrix, T.Carray, i, T.Carray, T.Carray,
                          T.Cmatrix]
    L.lowest_state_lanczos.restype = C.c_double
    L.lowest_state_lanczos.argtypes = [u16, T.MultiConfiguration, T.Cmatrix, T.Carray, T.Carray]
    L.propagate_coef_sil.argtypes = [T.MCTDHBDataStruct, T.Carray]
    L.total_energy.restype = T.dcomplex
    L.total_energy.argtypes = [T.ManyBodyState]
    L.eig_residual.restype = C.c_double
    L.eig_residual.argtypes = [T.MultiConfiguration, T.Carray, T.Cmatrix, T.Carray, C.c_double]
    L.mctdhb_space_create.restype = i
    L.mctdhb_space_create.argtypes = [u16, u16, C.POINTER(vp)]
    L.mctdhb_space_destroy.argtypes = [vp]
    L.mctdhb_space_dim.restype = u32
    L.mctdhb_space_dim.argtypes = [vp]
    L.mctdhb_dev_set_matrices.restype = i
    L.mctdhb_dev_set_matrices.argtypes = [vp, vp, vp, vp]
    L.mctdhb_dev_apply_hamiltonian.restype = i
    L.mctdhb_dev_apply_hamiltonian.argtypes = [vp, vp, vp, vp]
    L.mctdhb_dev_density_matrices.restype = i
    L.mctdhb_dev_density_matrices.argtypes = [vp, vp, vp, vp, vp]
    L.mctdhb_dev_sil_step.restype = i
    L.mctdhb_dev_sil_step.argtypes = [vp, vp, i, C.c_double, i, vp]
    L.mctdhb_dev_hash_table.restype = i
    L.mctdhb_dev_hash_table.argtypes = [vp, vp, vp]
    L.mctdhb_dev_single_jump_map.restype = i
    L.mctdhb_dev_single_jump_map.argtypes = [vp, vp, vp]
    L.mctdhb_dev_double_jump_chunks.restype = i
    L.mctdhb_dev_double_jump_chunks.argtypes = [vp, i, C.POINTER(C.c_uint64)]
    L.mctdhb_dev_double_jump_map.restype = i
    L.mctdhb_dev_double_jump_map.argtypes = [vp, i, vp, vp, vp]
    L.mctdhb_dev_density_matrices_noalloc.restype = i
    L.mctdhb_dev_density_matrices_noalloc.argtypes = [u16, u16, vp, vp, vp, vp]
    L.sync_density_matrices.argtypes = [T.MultiConfiguration, T.ManyBodyState]
    L.set_regulatization_factor.argtypes = [C.c_double]
    L.get_current_regularization_factor.restype = C.c_double
    L.mctdhb_step_create.restype = i
    L.mctdhb_step_create.argtypes = [vp, vp, vp, vp, i, C.c_double, i, C.POINTER(vp)]
    L.mctdhb_step_launch.restype = i
    L.mctdhb_step_launch.argtypes = [vp, vp]
    L.mctdhb_step_kernel_count.restype = i
    L.mctdhb_step_kernel_count.argtypes = [vp]
    L.mctdhb_step_destroy.argtypes = [vp]
    L.set_orbital_hob.argtypes = [T.OrbitalEquation, u16, T.Cmatrix, T.Cmatrix]
    L.set_orbital_hint.argtypes = [T.OrbitalEquation, u16, T.Cmatrix, T.Carray]
    L.sync_orbital_matrices.argtypes = [T.OrbitalEquation, T.ManyBodyState]
    L.mctdhb_propagate_step.argtypes = [T.MCTDHBDataStruct, T.Carray, T.Carray, u32]
    d = C.c_double
    L.mctdhb_solver_create.restype = i
    L.mctdhb_solver_create.argtypes = [u16, u16, u16, d, d, d, d, d, i, i, i, i, d,
                                       C.POINTER(vp)]
    L.mctdhb_solver_destroy.argtypes = [vp]
    for f in ("set_potential", "set_interaction", "set_regularization"):
        getattr(L, "mctdhb_solver_" + f).restype = i
    L.mctdhb_solver_set_potential.argtypes = [vp, C.POINTER(d)]
    L.mctdhb_solver_set_interaction.argtypes = [vp, d]
    L.mctdhb_solver_set_regularization.argtypes = [vp, d]
    L.mctdhb_solver_set_state.restype = i
    L.mctdhb_solver_set_state.argtypes = [vp, vp, vp]
    L.mctdhb_solver_step.restype = i
    L.mctdhb_solver_step.argtypes = [vp, i, vp]
    L.mctdhb_solver_kernel_count.restype = i
    L.mctdhb_solver_kernel_count.argtypes = [vp]
    L.mctdhb_solver_get.restype = i
    L.mctdhb_solver_get.argtypes = [vp] + [vp] * 7
    L.mctdhb_solver_put.restype = i
    L.mctdhb_solver_put.argtypes = [vp] + [vp] * 4
    L.mctdhb_solver_energy.restype = i
    L.mctdhb_solver_energy.argtypes = [vp, C.POINTER(d)]
    L.mctdhb_solver_set_orthogonality.restype = i
    L.mctdhb_solver_set_orthogonality.argtypes = [vp, i]
    L.mctdhb_solver_set_derivative.restype = i
    L.mctdhb_solver_set_derivative.argtypes = [vp, i]
    L.mctdhb_solver_set_coef_method.restype = i
    L.mctdhb_solver_set_coef_method.argtypes = [vp, i]
    L.mctdhb_solver_set_orb_method.restype = i
    L.mctdhb_solver_set_orb_method.argtypes = [vp, i]
    L.mctdhb_solver_overlap_residual.restype = i
    L.mctdhb_solver_overlap_residual.argtypes = [vp, C.POINTER(d)]
    L.mctdhb_solver_eig_residual.restype = i
    L.mctdhb_solver_eig_residual.argtypes = [vp, d, C.POINTER(d)]
    L.mctdhb_solver_lowest_state.restype = i
    L.mctdhb_solver_lowest_state.argtypes = [vp, i, C.POINTER(d)]
    L.mctdhb_solver_device_coef.restype = vp
    L.mctdhb_solver_device_coef.argtypes = [vp]
    L.mctdhb_solver_device_orbitals.restype = vp
    L.mctdhb_solver_device_orbitals.argtypes = [vp]
    L.mctdhb_solver_time.restype = d
    L.mctdhb_solver_time.argtypes = [vp]
    L.mctdhb_batch_create.restype = i
    L.mctdhb_batch_create.argtypes = [i, C.c_size_t, i, C.POINTER(vp)]
    L.mctdhb_batch_destroy.argtypes = [vp]
    L.mctdhb_batch_job_bytes.restype = C.c_size_t
    L.mctdhb_batch_job_bytes.argtypes = [C.POINTER(Job), i]
    L.mctdhb_batch_free_bytes.restype = C.c_size_t
    L.mctdhb_batch_free_bytes.argtypes = [vp]
    L.mctdhb_batch_admit.restype = i
    L.mctdhb_batch_admit.argtypes = [vp, C.POINTER(Job), C.POINTER(i)]
    L.mctdhb_batch_step.restype = i
    L.mctdhb_batch_step.argtypes = [vp, i]
    L.mctdhb_batch_sync.restype = i
    L.mctdhb_batch_sync.argtypes = [vp]
    L.mctdhb_batch_poll.restype = i
    L.mctdhb_batch_poll.argtypes = [vp, vp, vp, vp]
    L.mctdhb_batch_fetch.restype = i
    L.mctdhb_batch_fetch.argtypes = [vp, i, vp, vp, vp, vp, C.POINTER(d), C.POINTER(u32),
                                     C.POINTER(i)]
    L.mctdhb_batch_release.restype = i
    L.mctdhb_batch_release.argtypes = [vp, i]
    L.mctdhb_batch_monitor.restype = i
    L.mctdhb_batch_monitor.argtypes = [vp, i, C.POINTER(d), C.POINTER(d), C.POINTER(i)]
    L.mctdhb_batch_lowest_state.restype = i
    L.mctdhb_batch_lowest_state.argtypes = [vp, i, i, C.POINTER(d)]
    L.mctdhb_batch_kernel_count.restype = i
    L.mctdhb_batch_kernel_count.argtypes = [vp]
    L.mctdhb_batch_stream.restype = vp
    L.mctdhb_batch_stream.argtypes = [vp]
    L.mctdhb_batch_launch_hc.restype = i
    L.mctdhb_batch_launch_hc.argtypes = [vp, i, i]
    L.mctdhb_batch_variant.restype = i
    L.mctdhb_batch_variant.argtypes = [vp, i]
    L.mctdhb_batch_set_variant.restype = i
    L.mctdhb_batch_set_variant.argtypes = [vp, i, i]
    L.mctdhb_tune_get.restype = i
    L.mctdhb_tune_get.argtypes = [C.c_char_p, i, i]
    L.mctdhb_tune_set.restype = i
    L.mctdhb_tune_set.argtypes = [C.c_char_p, i, i, i]
    L.mctdhb_solver_step_phase.restype = i
    L.mctdhb_solver_step_phase.argtypes = [vp, i, vp]
    L.mctdhb_solver_relax.restype = i
    L.mctdhb_solver_relax.argtypes = [vp, u32, d, i, vp]
    L.mctdhb_solver_query.restype = i
    L.mctdhb_solver_query.argtypes = [vp]
    L.mctdhb_solver_relax_result.restype = i
    L.mctdhb_solver_relax_result.argtypes = [vp, C.POINTER(u32), C.POINTER(i)]
    L.mctdhb_fp64_mma_probe.restype = i
    L.mctdhb_fp64_mma_probe.argtypes = [i, i, vp, vp]
    _lib = L
    return L


def last_error():
    return load().mctdhb_gpu_last_error().decode()


def _check(rc, what):
    if rc != 0:
        raise MctdhbError(f"{what}: {last_error()}")


def _stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Space:
    """A Fock space (npar bosons, norb orbitals) on the current CUDA device."""

    def __init__(self, npar, norb):
        L = load()
        h = C.c_void_p()
        _check(L.mctdhb_space_create(npar, norb, C.byref(h)), "mctdhb_space_create")
        self.h, self.npar, self.norb = h, npar, norb
        self.dim = int(L.mctdhb_space_dim(h))

    def close(self):
        if self.h:
            load().mctdhb_space_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_matrices(self, hob, hint, stream=None):
        _check(load().mctdhb_dev_set_matrices(self.h, _ptr(hob), _ptr(hint), _stream_ptr(stream)),
               "mctdhb_dev_set_matrices")

    def apply_hamiltonian(self, coef, out, stream=None):
        _check(load().mctdhb_dev_apply_hamiltonian(self.h, _ptr(coef), _ptr(out),
                                                   _stream_ptr(stream)),
               "mctdhb_dev_apply_hamiltonian")

    def density_matrices(self, coef, rho1, rho2, stream=None):
        _check(load().mctdhb_dev_density_matrices(self.h, _ptr(coef), _ptr(rho1), _ptr(rho2),
                                                  _stream_ptr(stream)),
               "mctdhb_dev_density_matrices")

    def sil_step(self, coef, lanczos_iter, dt, imagtime, stream=None):
        _check(load().mctdhb_dev_sil_step(self.h, _ptr(coef), lanczos_iter, dt, int(imagtime),
                                          _stream_ptr(stream)),
               "mctdhb_dev_sil_step")

    def hash_table(self, out, stream=None):
        _check(load().mctdhb_dev_hash_table(self.h, _ptr(out), _stream_ptr(stream)),
               "mctdhb_dev_hash_table")

    def single_jump_map(self, out, stream=None):
        _check(load().mctdhb_dev_single_jump_map(self.h, _ptr(out), _stream_ptr(stream)),
               "mctdhb_dev_single_jump_map")

    def double_jump_chunks(self, diff):
        n = C.c_uint64()
        _check(load().mctdhb_dev_double_jump_chunks(self.h, int(diff), C.byref(n)),
               "mctdhb_dev_double_jump_chunks")
        return int(n.value)

    def double_jump_map(self, diff, strides, out, stream=None):
        _check(load().mctdhb_dev_double_jump_map(self.h, int(diff), _ptr(strides), _ptr(out),
                                                 _stream_ptr(stream)),
               "mctdhb_dev_double_jump_map")


class Step:
    """One configurational step (SIL + rho1/rho2) as a replayable CUDA graph
    over fixed device tensors."""

    def __init__(self, space, coef, rho1, rho2, lanczos_iter, dt, imagtime):
        L = load()
        h = C.c_void_p()
        _check(L.mctdhb_step_create(space.h, _ptr(coef), _ptr(rho1), _ptr(rho2), lanczos_iter,
                                    dt, int(imagtime), C.byref(h)), "mctdhb_step_create")
        self.h = h
        self.kernels = int(L.mctdhb_step_kernel_count(h))
        self._keep = (space, coef, rho1, rho2)

    def launch(self, stream=None):
        _check(load().mctdhb_step_launch(self.h, _stream_ptr(stream)), "mctdhb_step_launch")

    def close(self):
        if self.h:
            load().mctdhb_step_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """A whole MCTDHB system resident on the device (include/mctdhb_gpu.h,
    mctdhb_solver_*): orbitals, coefficients and their matrices; one step is
    the reference's mctdhb_propagate_step as two replayed CUDA graphs."""

    def __init__(self, npar, norb, grid, xi, xf, dt, imagtime, rk_order=5, lanczos_iter=5,
                 d2coef=-0.5, d1coef=0j, periodic=True):
        L = load()
        h = C.c_void_p()
        _check(L.mctdhb_solver_create(npar, norb, grid, xi, xf, d2coef, complex(d1coef).real,
                                      complex(d1coef).imag, int(periodic), int(imagtime),
                                      rk_order, lanczos_iter, dt, C.byref(h)),
               "mctdhb_solver_create")
        self.h = h
        self.npar, self.norb, self.grid = npar, norb, grid
        self.dim = int(L.space_dimension(npar, norb))

    def close(self):
        if self.h:
            load().mctdhb_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_potential(self, pot):
        pot = np.ascontiguousarray(pot, np.float64)
        _check(load().mctdhb_solver_set_potential(self.h, pot.ctypes.data_as(C.POINTER(C.c_double))),
               "mctdhb_solver_set_potential")

    def set_interaction(self, g):
        _check(load().mctdhb_solver_set_interaction(self.h, g), "mctdhb_solver_set_interaction")

    def set_state(self, orb, coef):
        orb = np.ascontiguousarray(orb, np.complex128)
        coef = np.ascontiguousarray(coef, np.complex128)
        _check(load().mctdhb_solver_set_state(self.h, orb.ctypes.data, coef.ctypes.data),
               "mctdhb_solver_set_state")

    def step(self, n=1, stream=None):
        _check(load().mctdhb_solver_step(self.h, n, _stream_ptr(stream)), "mctdhb_solver_step")

    def step_phase(self, phase, stream=None):
        """one half of a step: 0 the orbitals, 1 matrices + SIL + densities"""
        _check(load().mctdhb_solver_step_phase(self.h, phase, _stream_ptr(stream)),
               "mctdhb_solver_step_phase")

    @property
    def kernels(self):
        return int(load().mctdhb_solver_kernel_count(self.h))

    def get(self):
        M, G = self.norb, self.grid
        out = {"orb": np.zeros((M, G), np.complex128), "coef": np.zeros(self.dim, np.complex128),
               "hob": np.zeros((M, M), np.complex128), "hint": np.zeros(M ** 4, np.complex128),
               "rho1": np.zeros((M, M), np.complex128), "rho2": np.zeros(M ** 4, np.complex128),
               "rinv": np.zeros((M, M), np.complex128)}
        k = ("orb", "coef", "hob", "hint", "rho1", "rho2", "rinv")
        _check(load().mctdhb_solver_get(self.h, *[out[x].ctypes.data for x in k]),
               "mctdhb_solver_get")
        return out

    def energy(self):
        e = (C.c_double * 2)()
        _check(load().mctdhb_solver_energy(self.h, e), "mctdhb_solver_energy")
        return complex(e[0], e[1])

    def set_regularization(self, reg_fac):
        _check(load().mctdhb_solver_set_regularization(self.h, reg_fac),
               "mctdhb_solver_set_regularization")

    def set_derivative(self, der_method):
        """linear part of the orbital equation: 302 finite differences,
        300 DVR, 301 spectral"""
        _check(load().mctdhb_solver_set_derivative(self.h, int(der_method)),
               "mctdhb_solver_set_derivative")

    def set_coef_method(self, coef_method):
        """coefficient integrator: 20 short iterative Lanczos, 21 Runge-Kutta"""
        _check(load().mctdhb_solver_set_coef_method(self.h, int(coef_method)),
               "mctdhb_solver_set_coef_method")

    def set_orb_method(self, orb_method):
        """orbital integrator: 30 full-step Runge-Kutta, 31 split step"""
        _check(load().mctdhb_solver_set_orb_method(self.h, int(orb_method)),
               "mctdhb_solver_set_orb_method")

    def set_orthogonality(self, robust):
        """projector of the orbital equation: False simple, True robust"""
        _check(load().mctdhb_solver_set_orthogonality(self.h, int(bool(robust))),
               "mctdhb_solver_set_orthogonality")

    def overlap_residual(self):
        r = C.c_double()
        _check(load().mctdhb_solver_overlap_residual(self.h, C.byref(r)),
               "mctdhb_solver_overlap_residual")
        return r.value

    def eig_residual(self, e):
        r = C.c_double()
        _check(load().mctdhb_solver_eig_residual(self.h, e, C.byref(r)),
               "mctdhb_solver_eig_residual")
        return r.value

    def lowest_state(self, niter):
        e = C.c_double()
        _check(load().mctdhb_solver_lowest_state(self.h, niter, C.byref(e)),
               "mctdhb_solver_lowest_state")
        return e.value

    def relax(self, max_steps, energy_tol=0.0, check_every=0, stream=None):
        """steps on the device until the energy rule or max_steps (one graph
        launch, asynchronous); relax_result() gives (steps, converged)"""
        _check(load().mctdhb_solver_relax(self.h, int(max_steps), float(energy_tol),
                                          int(check_every), _stream_ptr(stream)),
               "mctdhb_solver_relax")

    def done(self):
        """True once the last launch has finished on the device (no wait)"""
        r = load().mctdhb_solver_query(self.h)
        if r < 0:
            raise MctdhbError(f"mctdhb_solver_query: {last_error()}")
        return r == 1

    def relax_result(self):
        n, c = C.c_uint32(), C.c_int()
        _check(load().mctdhb_solver_relax_result(self.h, C.byref(n), C.byref(c)),
               "mctdhb_solver_relax_result")
        return n.value, bool(c.value)


class DropIn:
    """The reference's C entry points, on host numpy buffers."""

    def __init__(self):
        self.lib = load()

    def space_dimension(self, N, M):
        return int(self.lib.space_dimension(N, M))

    def multiconf(self, N, M):
        mc = self.lib.get_multiconf_struct(N, M)
        if not mc:
            raise MctdhbError(f"get_multiconf_struct: {last_error()}")
        return mc

    def destroy(self, mc):
        self.lib.destroy_multiconf_struct(mc)

    def apply_hamiltonian(self, mc, c, hob, hint):
        c = np.ascontiguousarray(c, np.complex128)
        hint = np.ascontiguousarray(hint, np.complex128).reshape(-1)
        out = np.zeros_like(c)
        H = T.RowMatrix(hob)
        self.lib.mctdhb_gpu_clear_error()
        self.lib.apply_hamiltonian(mc, T.carray(c), H.ptr, T.carray(hint), T.carray(out))
        if last_error():
            raise MctdhbError(last_error())
        return out

    def onebody_dm(self, mc, c):
        M = mc.contents.norb
        R = T.RowMatrix(np.zeros((M, M), np.complex128))
        self.lib.mctdhb_gpu_clear_error()
        self.lib.set_onebody_dm(mc, T.carray(np.ascontiguousarray(c, np.complex128)), R.ptr)
        if last_error():
            raise MctdhbError(last_error())
        return R.a

    def twobody_dm(self, mc, c):
        M = mc.contents.norb
        r = np.zeros(M ** 4, np.complex128)
        self.lib.mctdhb_gpu_clear_error()
        self.lib.set_twobody_dm(mc, T.carray(np.ascontiguousarray(c, np.complex128)), T.carray(r))
        if last_error():
            raise MctdhbError(last_error())
        return r

    def lanczos(self, mc, hob, hint, m, c0):
        nc = mc.contents.dim
        lv = np.zeros((m, nc), np.complex128)
        lv[0] = c0
        L = T.RowMatrix(lv)
        diag = np.zeros(m, np.complex128)
        offd = np.zeros(m, np.complex128)
        H = T.RowMatrix(hob)
        hint = np.ascontiguousarray(hint, np.complex128).reshape(-1)
        it = self.lib.lanczos(mc, H.ptr, T.carray(hint), m, T.carray(diag), T.carray(offd), L.ptr)
        if it < 0:
            raise MctdhbError(last_error())
        return it, diag, offd, L.a

    def lowest_state_lanczos(self, mc, hob, hint, m, c):
        c = np.ascontiguousarray(c, np.complex128).copy()
        H = T.RowMatrix(hob)
        hint = np.ascontiguousarray(hint, np.complex128).reshape(-1)
        e = self.lib.lowest_state_lanczos(m, mc, H.ptr, T.carray(hint), T.carray(c))
        if np.isnan(e):
            raise MctdhbError(last_error())
        return e, c

    def propagate_coef_sil(self, mc, hob, hint, c, m, dt, imagtime):
        """Builds the parts of an MCTDHBDataStruct propagate_coef_sil reads
        (coefficients_integration.c:59-160) and runs one SIL step.
        Returns (cnext, state_coef, decomp_diag, decomp_offd)."""
        M = mc.contents.norb
        nc = mc.contents.dim
        keep = []
        coef = np.ascontiguousarray(c, np.complex128).copy()
        hintv = np.ascontiguousarray(hint, np.complex128).reshape(-1).copy()
        H = T.RowMatrix(hob)
        st = T.ManyBodyStateS()
        st.npar, st.norb, st.space_dim = mc.contents.npar, M, nc
        st.coef, st.hint, st.hob = T.carray(coef), T.carray(hintv), H.ptr
        eq = T.OrbitalEquationS()
        eq.tstep = dt
        eq.prop_dt = T.dcomplex.of(-1j * dt if imagtime else dt)
        eq.time_fac = T.dcomplex.of(-1j if imagtime else 1.0)
        lw = T.WorkspaceLanczosS()
        lw.iter, lw.space_dim = m, nc
        ddiag = np.zeros(m, np.complex128)
        doffd = np.zeros(m, np.complex128)
        lw.decomp_diag, lw.decomp_offd = T.carray(ddiag), T.carray(doffd)
        cw = T.CoefWorkspaceS()
        cw.lan_work = C.pointer(lw)
        ms = T.MCTDHBDataStructS()
        ms.integ_type = T.IMAGTIME if imagtime else T.REALTIME
        ms.coef_integ_method = T.LANCZOS
        ms.multiconfig_space = mc
        ms.orb_eq = C.pointer(eq)
        ms.coef_workspace = C.pointer(cw)
        ms.state = C.pointer(st)
        keep += [H, st, eq, lw, cw]
        cnext = np.zeros(nc, np.complex128)
        self.lib.mctdhb_gpu_clear_error()
        self.lib.propagate_coef_sil(C.pointer(ms), T.carray(cnext))
        if last_error():
            raise MctdhbError(last_error())
        return cnext, coef, ddiag, doffd


class Batch:
    """The batched engine (include/mctdhb_gpu.h, mctdhb_batch_*): independent
    systems of uneven size resident in one HBM arena, advanced together by
    one CUDA graph launch per step.  Jobs are dicts with the mctdhb_job
    fields; `pot`, `orbitals` and `coef` are numpy arrays."""

    def __init__(self, max_slots, arena_bytes, lanczos_iter=5):
        L = load()
        h = C.c_void_p()
        _check(L.mctdhb_batch_create(max_slots, int(arena_bytes), lanczos_iter, C.byref(h)),
               "mctdhb_batch_create")
        self.h, self.max_slots, self.lanczos_iter = h, max_slots, lanczos_iter
        self.jobs = {}

    def close(self):
        if self.h:
            load().mctdhb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def make_job(job):
        """(ctypes Job, arrays kept alive) from a dict"""
        keep = {k: np.ascontiguousarray(job[k], dt) for k, dt in
                (("pot", np.float64), ("orbitals", np.complex128), ("coef", np.complex128))}
        j = Job()
        for name, _ in Job._fields_:
            if name in keep:
                continue
            if name in job:
                setattr(j, name, job[name])
        d1 = complex(job.get("d1coef", 0j))
        j.d1coef_re, j.d1coef_im = d1.real, d1.imag
        if "d2coef" not in job:
            j.d2coef = -0.5
        j.pot = keep["pot"].ctypes.data_as(C.POINTER(C.c_double))
        j.orbitals = keep["orbitals"].ctypes.data
        j.coef = keep["coef"].ctypes.data
        return j, keep

    @staticmethod
    def job_bytes(job, lanczos_iter=5):
        j, _ = Batch.make_job(job)
        n = int(load().mctdhb_batch_job_bytes(C.byref(j), lanczos_iter))
        if n == 0:
            raise MctdhbError(f"mctdhb_batch_job_bytes: {last_error()}")
        return n

    def free_bytes(self):
        return int(load().mctdhb_batch_free_bytes(self.h))

    def admit(self, job):
        """slot index, or None when the batch has no room now"""
        j, keep = self.make_job(job)
        slot = C.c_int(-1)
        rc = load().mctdhb_batch_admit(self.h, C.byref(j), C.byref(slot))
        if rc == 1:
            return None
        _check(rc, "mctdhb_batch_admit")
        self.jobs[slot.value] = (int(job["npar"]), int(job["norb"]), int(job["grid_size"]))
        return slot.value

    def step(self, n=1):
        _check(load().mctdhb_batch_step(self.h, n), "mctdhb_batch_step")

    def sync(self):
        _check(load().mctdhb_batch_sync(self.h), "mctdhb_batch_sync")

    def poll(self):
        """(running count, state[], steps[], energy[]) over the slots"""
        S = self.max_slots
        st = np.zeros(S, np.int32)
        steps = np.zeros(S, np.uint32)
        en = np.zeros(S, np.float64)
        n = load().mctdhb_batch_poll(self.h, st.ctypes.data, steps.ctypes.data, en.ctypes.data)
        if n < 0:
            raise MctdhbError(f"mctdhb_batch_poll: {last_error()}")
        return n, st, steps, en

    def fetch(self, slot, out=None):
        """the slot's state; `out`: optional dict of destination arrays
        (orb, coef, rho1, rho2; e.g. views of pinned host memory)"""
        N, M, G = self.jobs[slot]
        dim = int(load().space_dimension(N, M))
        if out is None:
            out = {"orb": np.zeros((M, G), np.complex128),
                   "coef": np.zeros(dim, np.complex128),
                   "rho1": np.zeros((M, M), np.complex128),
                   "rho2": np.zeros(M ** 4, np.complex128)}
        for k, n in (("orb", M * G), ("coef", dim), ("rho1", M * M), ("rho2", M ** 4)):
            a = out[k]
            if a.dtype != np.complex128 or a.size != n or not a.flags.c_contiguous:
                raise ValueError(f"fetch: out[{k!r}] must be {n} contiguous complex128")
        e = C.c_double()
        steps = C.c_uint32()
        conv = C.c_int()
        _check(load().mctdhb_batch_fetch(self.h, slot, out["orb"].ctypes.data,
                                         out["coef"].ctypes.data, out["rho1"].ctypes.data,
                                         out["rho2"].ctypes.data, C.byref(e), C.byref(steps),
                                         C.byref(conv)), "mctdhb_batch_fetch")
        out.update(energy=e.value, steps=steps.value, converged=bool(conv.value))
        return out

    def release(self, slot):
        _check(load().mctdhb_batch_release(self.h, slot), "mctdhb_batch_release")
        self.jobs.pop(slot, None)

    def monitor(self, slot):
        """{'overlap_residual', 'eig_residual', 'robust', 'robust_failed'} of a job"""
        o, e, r = C.c_double(), C.c_double(), C.c_int()
        _check(load().mctdhb_batch_monitor(self.h, slot, C.byref(o), C.byref(e), C.byref(r)),
               "mctdhb_batch_monitor")
        return {"overlap_residual": o.value, "eig_residual": e.value,
                "robust": bool(r.value & 1), "robust_failed": bool(r.value & 2)}

    def lowest_state(self, slot, niter=0):
        """final diagonalisation of a stopped job (0: the reference's
        iteration count); returns the Lanczos energy"""
        e = C.c_double()
        _check(load().mctdhb_batch_lowest_state(self.h, slot, niter, C.byref(e)),
               "mctdhb_batch_lowest_state")
        return e.value

    @property
    def kernels(self):
        return int(load().mctdhb_batch_kernel_count(self.h))

    @property
    def stream(self):
        """the engine's CUDA stream as a torch stream"""
        import torch

        return torch.cuda.ExternalStream(int(load().mctdhb_batch_stream(self.h)))

    def variant(self, norb):
        """the batched contraction's launch variant for norb (autotuned)"""
        return int(load().mctdhb_batch_variant(self.h, norb))

    def set_variant(self, norb, variant):
        """force a variant (-1: tune again); changes speed, never results"""
        _check(load().mctdhb_batch_set_variant(self.h, norb, variant),
               "mctdhb_batch_set_variant")

    def launch_hc(self, norb, parts=3):
        """one batched H.C launch of the jobs with norb orbitals: parts = 1
        the pair contraction, 2 the gather-back, 3 both"""
        _check(load().mctdhb_batch_launch_hc(self.h, norb, parts), "mctdhb_batch_launch_hc")


def tune_get(kernel, npar, norb):
    """the autotuner's variant for a kernel and Fock space, -1 if untuned"""
    return int(load().mctdhb_tune_get(kernel.encode(), npar, norb))


def tune_set(kernel, npar, norb, variant):
    _check(load().mctdhb_tune_set(kernel.encode(), npar, norb, variant), "mctdhb_tune_set")


def fp64_mma_probe(blocks, iters, out, stream=None):
    """launch the FP64 tensor-core throughput probe (mctdhb_fp64_mma_probe):
    out is a float64 device tensor of at least blocks * 256 elements; the
    launch does blocks * 8 * iters * 8 * 512 FLOPs"""
    _check(load().mctdhb_fp64_mma_probe(blocks, iters, _ptr(out), _stream_ptr(stream)),
           "mctdhb_fp64_mma_probe")
