"""The reference's text formats and built-in functions (dataio.py), on CPU.

* the built-in traps and the interaction ramp against the reference's own
  compiled functions (builtin_potential.c, builtin_time_parameter.c);
* orbitals, coefficients and records written here, read back the way the
  reference's loaders read them (numpy.loadtxt with complex dtype, one frame
  per line; the C reader's "(re+imj)" token syntax);
* parameter lines and the integrator descriptor.
"""
import ctypes as C
import re

import numpy as np
import pytest

import dataio as D

POTS = [
    ("harmonic", [1.3, 0.7, 2.0, 0, 0]),
    ("doublewell", [0.8, 2.0, 1.5, 3.0, 0]),
    ("harmonicgauss", [1.0, 0.7, 4.0, 2.0, 5.0]),
    ("barrier", [3.0, 2.0, 1.0, 4.0, 0.25]),
    ("trapezoid_barrier", [3.0, 2.0, 1.0, 2.0, 0]),
    ("opticallattice", [4.0, 1.0, 3.0, 2.0, 0]),
    ("trapezoid_opticallattice", [4.0, 1.0, 0.5, 1.0, 0]),
    ("potfunc_step", [0.5, 1.0, 2.0, 3.0, 0]),
    ("potfunc_square_well", [2.0, -2.0, 5.0, 1.0, 4.0]),
]
REF_NAMES = {"trapezoid_barrier": "potfunc_time_trapezoid_barrier",
             "trapezoid_opticallattice": "potfunc_time_trapezoid_opticallattice"}


@pytest.mark.parametrize("name,params", POTS)
def test_builtin_potentials_match_the_reference(reference, name, params):
    x = np.linspace(-8.0, 8.0, 257)
    fn = getattr(reference.lib, REF_NAMES.get(name, name if name.startswith("potfunc_")
                                              else "potfunc_" + name))
    fn.restype = None
    fn.argtypes = [C.c_double, C.c_uint16, C.c_void_p, C.c_void_p, C.c_void_p]
    p = (C.c_double * 5)(*params)
    for t in (0.0, 0.3, 1.1, 2.5, 7.0):
        out = np.zeros_like(x)
        fn(t, x.size, x.ctypes.data, C.cast(p, C.c_void_p), out.ctypes.data)
        got = D.builtin_potential(name, t, x, params)
        assert np.allclose(got, out, rtol=1e-15, atol=1e-15), (name, t)


def test_linear_ramp_matches_the_reference(reference):
    fn = reference.lib.timeparam_linear_ramp
    fn.restype = C.c_double
    fn.argtypes = [C.c_double, C.c_void_p]
    for p in ([0.5, 1.5, 2.0], [0.2, 0.2, 0.0], [1.0, -1.0, 0.5]):
        a = (C.c_double * 3)(*p)
        for t in (0.0, 0.1, 0.5, 1.9, 2.0, 3.0):
            assert D.builtin_time_parameter("linear_ramp", t, p) == fn(t, C.cast(a, C.c_void_p))
    assert D.builtin_time_parameter("custom", 0.0, [0, 0, 0]) is None
    with pytest.raises(ValueError):
        D.builtin_potential("no_such_trap", 0.0, np.zeros(4), [])


def test_parameter_line_and_descriptor(tmp_path):
    params = tmp_path / ("p" + D.PARAMS_SUFFIX)
    params.write_text("# comment\n"
                      "10 4 256 -10.0 10.0 0.01 10.0 -0.5 0.0 linear_ramp 0.5 0.5 0 0 0 "
                      "harmonic 1.0 1.0 0 0 0\n"
                      "30 8 1024 -15 15 0.005 1.0 -0.5 0.25 linear_ramp 0.1 0.2 0.5 0 0 "
                      "harmonicgauss 1.0 0.7 4.0 4.0 0\n")
    assert D.number_of_jobs(params) == 2
    j = D.read_parameter_line(params, 2)
    assert (j.npar, j.norb, j.grid_size) == (30, 8, 1024)
    assert (j.xi, j.xf, j.tstep, j.tend, j.d2coef, j.d1coef) == (-15, 15, 0.005, 1.0, -0.5, 0.25j)
    assert j.g_func == "linear_ramp" and j.g_params == [0.1, 0.2, 0.5, 0, 0]
    assert j.pot_func == "harmonicgauss" and j.pot_params[:3] == [1.0, 0.7, 4.0]
    assert D.time_dependent(j) and not D.time_dependent(D.read_parameter_line(params, 1))
    with pytest.raises(ValueError):
        D.read_parameter_line(params, 3)
    desc = tmp_path / "integ.txt"
    desc.write_text("# type\n11\n# coef\n20\n30\n302\n4\n1000\n6\n")
    d = D.read_integrator_descriptor(desc)
    assert d == {"integ_type": 11, "coef_method": 20, "orb_method": 30, "der_method": 302,
                 "rk_order": 4, "bounds": 1000, "lanczos_iter": 6}
    assert D.read_integrator_descriptor(tmp_path / "missing") == D.DEFAULT_INTEGRATOR


def test_state_files_round_trip_and_loader_layouts(tmp_path):
    rng = np.random.default_rng(4)
    M, G, nc = 3, 17, 10
    orb = rng.normal(size=(M, G)) + 1j * rng.normal(size=(M, G))
    coef = rng.normal(size=nc) + 1j * rng.normal(size=nc)
    pre = str(tmp_path / "x_job1")
    D.record_raw_state(pre, orb, coef)
    # the reference's stationary loader: loadtxt(orb).T and loadtxt(coef)
    assert np.array_equal(np.loadtxt(pre + "_orb.dat", dtype=np.complex128).T, orb)
    assert np.array_equal(np.loadtxt(pre + "_coef.dat", dtype=np.complex128), coef)
    assert np.array_equal(D.read_orbitals(pre + "_orb.dat", M, G), orb)
    assert np.array_equal(D.read_coefficients(pre + "_coef.dat", nc), coef)
    # the C reader's token syntax " (%lf%lfj) ": two reals inside parentheses
    tok = re.compile(r"\(([-+]?[0-9.]+E[-+][0-9]+)([-+][0-9.]+E[-+][0-9]+)j\)")
    line = open(pre + "_orb.dat").readline()
    vals = [complex(float(a), float(b)) for a, b in tok.findall(line)]
    assert np.array_equal(np.array(vals), orb[:, 0])
    # real-time records, one frame per line, read as the dynamics loader does
    rho1 = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    rho2 = rng.normal(size=M ** 4) + 1j * rng.normal(size=M ** 4)
    for frame in range(3):
        D.append_processed_state(pre, rho1 * (frame + 1), rho2, orb, new=frame == 0)
        D.append_timestep_potential(pre, np.arange(G) * 0.5, new=frame == 0)
    lines = open(pre + "_obmat.dat").read().splitlines()
    assert len(lines) == 3
    got = np.loadtxt([lines[2]], dtype=np.complex128).reshape(M, M)
    assert np.array_equal(got, 3 * rho1)
    got = np.loadtxt([open(pre + "_orb.dat").read().splitlines()[1]],
                     dtype=np.complex128).reshape(M, G)
    assert np.array_equal(got, orb)
    assert np.loadtxt(pre + "_obpotential.dat").shape == (3, G)


def test_parameter_records_and_time_arrays(tmp_path):
    job = D.JobParams(npar=10, norb=4, grid_size=256, xi=-10.0, xf=10.0, tstep=0.01, tend=0.1,
                      d2coef=-0.5, d1coef=0j, g_func="linear_ramp", g_params=[0.5, 1.0, 0.05],
                      pot_func="harmonic", pot_params=[1.0, 1.0, 0.0])
    base = str(tmp_path / "run")
    D.append_mctdhb_parameters(base, job, 0.5, 12.5, new=True)
    D.append_mctdhb_parameters(base, job, 0.5, 13.0)
    rows = np.loadtxt(base + D.PARAMS_SUFFIX)
    assert rows.shape == (2, 11)
    assert rows[1, 10] == pytest.approx(1.3) and rows[0, 2] == 256
    D.record_time_array(base, job.tend, job.tstep, 2)
    t = np.loadtxt(base + "_timesteps.dat")
    assert np.allclose(t, [0.0, 0.02, 0.04, 0.06, 0.08, 0.10])
    D.record_time_interaction(base, job, 2)
    g = np.loadtxt(base + "_interaction.dat")
    assert g[0] == 0.5 and g.max() == 1.0
