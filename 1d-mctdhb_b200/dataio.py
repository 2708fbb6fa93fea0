"""Input and output in the reference's text formats, and its job driver on
the GPU solver.

Files (the layouts of the reference's `src/assistant/dataio.c`, read by its
`multiconfpy` loaders with ``numpy.loadtxt(..., dtype=complex128)``):

  <prefix>_mctdhb_parameters.dat  input: one job per line, 21 fields
      npar norb grid xi xf tstep tend d2coef imag(d1coef)
      g_func g1..g5 pot_func p1..p5                       (dataio.c:127-152)
      output: one line per job, 11 fields, the last one E/N (dataio.c:837-860)
  <prefix>_job<j>_orb.dat     grid rows x norb columns of "(re+imj)" numbers
  <prefix>_job<j>_coef.dat    one "(re+imj)" coefficient per line
  real-time records, one frame per line (dataio.c:706-746, 766-780):
  <prefix>_job<j>_obmat.dat   rho1, row-major M x M
  <prefix>_job<j>_tbmat.dat   rho2, M^4 (element k + sM + qM^2 + lM^3)
  <prefix>_job<j>_orb.dat     orbitals, row-major M x grid
  <prefix>_job<j>_obpotential.dat   trap on the grid
  <prefix>_job<j>_timesteps.dat / _interaction.dat   one value per line

The exact number formatting of the reference's writers lives in its
third-party text-I/O dependency (not in the reference tree); these writers
use 17 significant digits (an exact round trip of a double) in the same
token syntax, which both the reference's readers (" (%lf%lfj) ") and numpy
parse.
"""
import os
from dataclasses import dataclass, field

import numpy as np

PARAMS_SUFFIX = "_mctdhb_parameters.dat"

# enumerations of the reference's mctdhb_types.h
IMAGTIME, REALTIME = 10, 11
LANCZOS, RUNGEKUTTA = 20, 21
FULLSTEP_RUNGEKUTTA, SPLITSTEP = 30, 31
DVR, SPECTRAL, FINITEDIFF = 300, 301, 302
ZERO_BOUNDS, PERIODIC_BOUNDS = 1000, 1001
# and its defaults (mctdhb_types.h:98-110)
DEFAULT_INTEGRATOR = {"integ_type": IMAGTIME, "coef_method": LANCZOS,
                      "orb_method": FULLSTEP_RUNGEKUTTA, "der_method": DVR, "rk_order": 5,
                      "bounds": PERIODIC_BOUNDS, "lanczos_iter": 5}


def cplx(z):
    """one complex token: (re+imj)"""
    return f"({z.real:.16E}{z.imag:+.16E}j)"


def _data_lines(path):
    with open(path) as f:
        return [ln for ln in f if ln.strip() and not ln.lstrip().startswith("#")]


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
@dataclass
class JobParams:
    """one line of the parameters file (dataio.c:127-152)"""
    npar: int
    norb: int
    grid_size: int
    xi: float
    xf: float
    tstep: float
    tend: float
    d2coef: float
    d1coef: complex  # i * the file's value
    g_func: str
    g_params: list = field(default_factory=list)
    pot_func: str = "harmonic"
    pot_params: list = field(default_factory=list)

    @property
    def grid(self):
        """x_i = xi + i dx, dx = (xf - xi) / (grid - 1) (types_definition.c:13-16, 84)"""
        return self.xi + np.arange(self.grid_size) * ((self.xf - self.xi) / (self.grid_size - 1))


def number_of_jobs(params_path):
    """jobs in a parameters file: its non-comment lines"""
    return len(_data_lines(params_path))


def read_parameter_line(params_path, line=1):
    """job `line` (from 1) of a parameters file; comment lines starting with
    '#' are skipped like the reference's jump_comment_lines"""
    lines = _data_lines(params_path)
    if line < 1 or line > len(lines):
        raise ValueError(f"{params_path} has {len(lines)} job lines, line {line} requested")
    tok = lines[line - 1].split()
    if len(tok) < 21:
        raise ValueError(f"{params_path} line {line}: expected 21 fields, found {len(tok)}")
    return JobParams(npar=int(tok[0]), norb=int(tok[1]), grid_size=int(tok[2]),
                     xi=float(tok[3]), xf=float(tok[4]), tstep=float(tok[5]),
                     tend=float(tok[6]), d2coef=float(tok[7]), d1coef=1j * float(tok[8]),
                     g_func=tok[9], g_params=[float(v) for v in tok[10:15]],
                     pot_func=tok[15], pot_params=[float(v) for v in tok[16:21]])


def read_integrator_descriptor(path):
    """the seven integers of the integrator descriptor (dataio.c:179-245),
    comment lines skipped; missing file or values take the defaults"""
    out = dict(DEFAULT_INTEGRATOR)
    if not os.path.exists(path):
        return out
    keys = ["integ_type", "coef_method", "orb_method", "der_method", "rk_order", "bounds",
            "lanczos_iter"]
    vals = []
    for ln in _data_lines(path):
        try:
            vals.append(int(ln.split()[0]))
        except ValueError:
            break
    for k, v in zip(keys, vals):
        out[k] = v
    return out


# apps/mctdhb_main.c:11-16 and src/integrator/driver.c:15-19
COMMON_INP, MULTIPLE_INP, LAST_JOB_OUT = 0, 1, 2
REALTIME_OVERLAP_RESIDUE_TOL = 0.001  # include/integrator/driver.h:7
DEFAULT_MONITOR = {"job_input": COMMON_INP, "monitor_nsteps": 10, "auto_check": False,
                   "energy_digits": 11, "eig_residue": 1e-6, "final_diag": True,
                   "rec_nsteps": 10, "overlap_threshold": 1e-8, "reg_factor": None}


def read_monitor_config(path):
    """mctdhb_extra.conf (apps/mctdhb_main.c:28-144): job input handling,
    monitor rate, auto convergence, energy digits, eigen-residual tolerance,
    final diagonalisation, record rate, overlap threshold, regularisation
    factor, in this order, comment lines skipped.  Reading stops at the first
    value that does not parse; the values read so far are kept, the rest keep
    their defaults, as there.  Values the reference rejects raise."""
    out = dict(DEFAULT_MONITOR)
    if not os.path.exists(path):
        return out
    keys = [("job_input", int), ("monitor_nsteps", int), ("auto_check", lambda v: bool(int(v))),
            ("energy_digits", int), ("eig_residue", float), ("final_diag", lambda v: bool(int(v))),
            ("rec_nsteps", int), ("overlap_threshold", float), ("reg_factor", float)]
    for (k, conv), ln in zip(keys, _data_lines(path)):
        try:
            out[k] = conv(ln.split()[0])
        except ValueError:
            break
    if out["energy_digits"] > 13:  # driver.c:110-129
        raise ValueError(f"{out['energy_digits']} digits for convergence is too much")
    if out["overlap_threshold"] > REALTIME_OVERLAP_RESIDUE_TOL:  # driver.c:144-157
        raise ValueError(f"overlap residue threshold {out['overlap_threshold']} exceeds "
                         f"{REALTIME_OVERLAP_RESIDUE_TOL}")
    if out["reg_factor"] is not None and not 1e-13 <= out["reg_factor"] <= 1e-6:
        raise ValueError(f"regularization factor {out['reg_factor']} outside [1E-13, 1E-6]")
    return out


def lanczos_iterations_for(dim):
    """iterations of the final diagonalisation (driver.c:38-44)"""
    if dim // 2 > 50:
        return 50
    if dim < 4:
        return 0
    return dim // 2


def read_orbitals(path, norb, grid_size):
    """orbitals file: grid rows x norb columns -> (norb, grid) array"""
    a = np.loadtxt(path, dtype=np.complex128, ndmin=2)
    if a.shape != (grid_size, norb):
        raise ValueError(f"{path}: expected {grid_size} x {norb} values, found {a.shape}")
    return np.ascontiguousarray(a.T)


def read_coefficients(path, dim):
    c = np.loadtxt(path, dtype=np.complex128, ndmin=1)
    if c.size != dim:
        raise ValueError(f"{path}: expected {dim} coefficients, found {c.size}")
    return c


# ---------------------------------------------------------------------------
# the reference's built-in traps and interaction ramps
# (function_tools/builtin_potential.c, builtin_time_parameter.c)
# ---------------------------------------------------------------------------
def _linear_sweep(t, init, final, period):
    return final if period <= 0 else init + (final - init) * t / period


def _trapezoid_sweep(t, top, ramp, static):
    v = 0.0
    if t <= ramp:
        v = _linear_sweep(t, 0.0, top, ramp)
    if ramp < t < ramp + static:
        v = top
    if ramp + static <= t < 2 * ramp + static:
        v = top - (t - ramp - static) / ramp * top
    return v


def builtin_potential(name, t, x, p):
    """trap on the grid x at time t, or None for 'custom'"""
    x = np.asarray(x, dtype=np.float64)
    p = list(p) + [0.0] * (5 - len(p))
    if name == "harmonic":
        w = _linear_sweep(t, p[0], p[1], p[2])
        return 0.5 * w * w * x * x
    if name == "doublewell":
        a = _linear_sweep(t, p[1], p[2], p[3])
        b2 = p[0] * p[0]
        return b2 * (x * x - a * a / b2) * (x * x - a * a / b2)
    if name == "harmonicgauss":
        h = _linear_sweep(t, p[2], p[3], p[4])
        if p[1] < x[1] - x[0]:
            raise ValueError("harmonicgauss: barrier width below the grid step")
        return p[0] * p[0] * x * x / 2 + h * np.exp(-x * x / (p[1] * p[1]))
    if name == "barrier":
        h = _linear_sweep(t, p[1], p[2], p[3])
        if p[0] < x[1] - x[0]:
            raise ValueError("barrier: width below the grid step")
        c = np.cos(x * np.pi / p[0])
        return p[4] + np.where(np.abs(x) <= p[0] / 2, h * c * c, 0.0)
    if name == "trapezoid_barrier":
        h = _trapezoid_sweep(t, p[1], p[2], p[3])
        c = np.cos(x * np.pi / p[0])
        return np.where(np.abs(x) <= p[0] / 2, h * c * c, 0.0)
    if name in ("opticallattice", "trapezoid_opticallattice"):
        length = x[-1] - x[0]
        h = (_linear_sweep(t, p[1], p[2], p[3]) if name == "opticallattice"
             else _trapezoid_sweep(t, p[1], p[2], p[3]))
        s = np.sin(np.pi * p[0] * x / length)
        return h * s * s
    if name == "potfunc_step":
        v = _linear_sweep(t, p[1], p[2], p[3])
        return np.where(x >= p[0], v, 0.0)
    if name == "potfunc_square_well":
        v = _linear_sweep(t, p[2], p[3], p[4])
        # the reference's condition, as written there
        return np.where((x > p[0]) | (x < p[1]), 0.0, v)
    if name == "custom":
        return None
    raise ValueError(f"built-in potential '{name}' not found")


def builtin_time_parameter(name, t, p):
    """interaction strength at time t ('linear_ramp'), or None for 'custom'"""
    if name == "linear_ramp":
        g0, gf, period = p[0], p[1], p[2]
        return gf if t >= period else g0 + (gf - g0) * t / period
    if name == "custom":
        return None
    raise ValueError(f"built-in time function '{name}' not found")


def time_dependent(job):
    """whether the trap or the interaction changes with time"""
    p = list(job.pot_params) + [0.0] * 5
    sweep = {"harmonic": p[2], "doublewell": p[3], "harmonicgauss": p[4], "barrier": p[3],
             "opticallattice": p[3], "potfunc_step": p[3], "potfunc_square_well": p[4]}
    pot_td = job.pot_func in ("trapezoid_barrier", "trapezoid_opticallattice") or \
        sweep.get(job.pot_func, 0.0) > 0
    g_td = job.g_func == "linear_ramp" and job.g_params[2] > 0
    return pot_td or g_td


# ---------------------------------------------------------------------------
# outputs
# ---------------------------------------------------------------------------
def write_coefficients(path, coef):
    with open(path, "w") as f:
        f.write("\n".join(cplx(z) for z in np.asarray(coef).ravel()) + "\n")


def write_orbitals(path, orb):
    """(norb, grid) orbitals as grid rows x norb columns"""
    orb = np.asarray(orb)
    with open(path, "w") as f:
        for x in range(orb.shape[1]):
            f.write(" ".join(cplx(z) for z in orb[:, x]) + "\n")


def record_raw_state(prefix, orb, coef):
    """<prefix>_coef.dat and <prefix>_orb.dat (dataio.c:747-763)"""
    write_coefficients(prefix + "_coef.dat", coef)
    write_orbitals(prefix + "_orb.dat", orb)


def _append_line(path, values, new, fmt=cplx):
    with open(path, "w" if new else "a") as f:
        f.write(" ".join(fmt(v) for v in np.asarray(values).ravel()) + "\n")


def append_processed_state(prefix, rho1, rho2, orb, new=False):
    """one frame of _tbmat, _obmat and _orb (dataio.c:705-745)"""
    _append_line(prefix + "_tbmat.dat", rho2, new)
    _append_line(prefix + "_obmat.dat", rho1, new)
    _append_line(prefix + "_orb.dat", orb, new)


def append_timestep_potential(prefix, pot, new=False):
    _append_line(prefix + "_obpotential.dat", pot, new, fmt=lambda v: f"{v:.15E}")


def record_potential(prefix, pot):
    """the trap as one column (the imaginary-time record, driver.c:310-312)"""
    with open(prefix + "_obpotential.dat", "w") as f:
        f.write("\n".join(f"{v:.14E}" for v in pot) + "\n")


def append_mctdhb_parameters(prefix, job, g, energy, new=False):
    """one line of <prefix>_mctdhb_parameters.dat: npar norb grid xi xf tstep
    tend d2coef imag(d1coef) g E/N (dataio.c:837-860)"""
    with open(prefix + PARAMS_SUFFIX, "w" if new else "a") as f:
        f.write(f"{job.npar} {job.norb} {job.grid_size} {job.xi:.10f} {job.xf:.10f} "
                f"{job.tstep:.10f} {job.tend:.2f} {job.d2coef:.1f} {job.d1coef.imag:.10f} "
                f"{g:.10E} {energy / job.npar:.10E}\n")


def record_time_array(prefix, tend, tstep, recn):
    """recorded times (dataio.c:815-834)"""
    out, n = [0.0], 0
    while n * tstep < tend:
        n += 1
        if n % recn == 0:
            out.append(n * tstep)
    with open(prefix + "_timesteps.dat", "w") as f:
        f.write("".join(f"{t:.6f}\n" for t in out))


def record_time_interaction(prefix, job, recn):
    """interaction strength along the run (dataio.c:782-812, with its
    selection of the steps as written there)"""
    out = [builtin_time_parameter(job.g_func, 0.0, job.g_params)]
    n, t = 0, 0.0
    while t < job.tend:
        n += 1
        if n % recn:
            t = n * job.tstep
            out.append(builtin_time_parameter(job.g_func, t, job.g_params))
    with open(prefix + "_interaction.dat", "w") as f:
        f.write("".join(f"{g:.10E}\n" for g in out))


# ---------------------------------------------------------------------------
# the job driver (apps/mctdhb_main.c + integrator/driver.c:205-330)
# ---------------------------------------------------------------------------
def _job_input_paths(prefix, in_dir, out_dir, j, job_input):
    """orbital and coefficient files of job j (dataio.c:296-380)"""
    if job_input == MULTIPLE_INP:
        base = os.path.join(in_dir, f"{prefix}_job{j}")
    elif job_input == LAST_JOB_OUT and j > 1:
        base = os.path.join(out_dir, f"{prefix}_job{j - 1}")
    elif job_input in (COMMON_INP, LAST_JOB_OUT):
        base = os.path.join(in_dir, f"{prefix}_job1")
    else:
        raise ValueError(f"job input handling {job_input} not in 0..2")
    return base + "_orb.dat", base + "_coef.dat"


def run_jobs(prefix, in_dir, out_dir, integrator=None, monitor=None, stream=None):
    """Run every job of <in_dir>/<prefix>_mctdhb_parameters.dat on the GPU
    solver as the reference's application does (apps/mctdhb_main.c:146-205,
    integration_driver in src/integrator/driver.c:203-330), and write its
    output files under out_dir: per job the real-time records or the initial
    and final raw states, and one line per job of
    <out_dir>/<prefix>_mctdhb_parameters.dat.

    `integrator`: the descriptor dict (read_integrator_descriptor); the GPU
    solver runs FULLSTEP_RUNGEKUTTA or SPLITSTEP orbitals with DVR (the reference's
    default), SPECTRAL or FINITEDIFF derivatives and LANCZOS or RUNGEKUTTA
    coefficients.
    `monitor`: the dict of read_monitor_config.  Every
    monitor_nsteps steps, in imaginary time with auto_check the run stops
    once E/N changed by less than 10^-digits relative and the eigen-residual
    is below eig_residue; in real time the robust projector is switched on
    once the overlap residual exceeds overlap_threshold, and the run aborts
    (RuntimeError) above 1e-3.  An imaginary-time run that reached tend ends,
    with final_diag, with the coefficients replaced by the lowest Lanczos
    state in the final orbitals (the recorded energy is that of the last
    step, as there).  In real time the trap and the interaction follow their
    time dependence between the two phases of every step, as the reference's
    mctdhb_propagate_step does.  Returns one dict per job: the recorded
    energy E (not E/N), the steps taken and whether the auto convergence rule
    stopped the run.  Screen output of the reference's monitor is not
    reproduced."""
    import mctdhb_b200 as mb

    desc = dict(DEFAULT_INTEGRATOR, **(integrator or {}))
    mon = dict(DEFAULT_MONITOR, **(monitor or {}))
    if desc["orb_method"] not in (FULLSTEP_RUNGEKUTTA, SPLITSTEP) or \
            desc["coef_method"] not in (LANCZOS, RUNGEKUTTA) or \
            desc["der_method"] not in (DVR, SPECTRAL, FINITEDIFF):
        raise ValueError("the GPU solver runs FULLSTEP_RUNGEKUTTA or SPLITSTEP orbitals (DVR, "
                         "SPECTRAL or FINITEDIFF derivatives) and LANCZOS or RUNGEKUTTA "
                         "coefficients")
    imag = desc["integ_type"] == IMAGTIME
    rec_n, mon_n = mon["rec_nsteps"], mon["monitor_nsteps"]
    os.makedirs(out_dir, exist_ok=True)
    params = os.path.join(in_dir, prefix + PARAMS_SUFFIX)
    out_base = os.path.join(out_dir, prefix)
    energies = []
    for j in range(1, number_of_jobs(params) + 1):
        job = read_parameter_line(params, j)
        dim = int(mb.load().space_dimension(job.npar, job.norb))
        orb_path, coef_path = _job_input_paths(prefix, in_dir, out_dir, j, mon["job_input"])
        orb = read_orbitals(orb_path, job.norb, job.grid_size)
        coef = read_coefficients(coef_path, dim)
        x = job.grid
        s = mb.Solver(job.npar, job.norb, job.grid_size, job.xi, job.xf, job.tstep, imag,
                      desc["rk_order"], desc["lanczos_iter"], d2coef=job.d2coef,
                      d1coef=job.d1coef, periodic=desc["bounds"] == PERIODIC_BOUNDS)
        try:
            s.set_derivative(desc["der_method"])
            s.set_coef_method(desc["coef_method"])
            s.set_orb_method(desc["orb_method"])
            if mon["reg_factor"] is not None:
                s.set_regularization(mon["reg_factor"])
            pot = builtin_potential(job.pot_func, 0.0, x, job.pot_params)
            g = builtin_time_parameter(job.g_func, 0.0, job.g_params)
            if pot is None or g is None:
                raise ValueError("custom traps and interactions need a caller-side driver")
            s.set_potential(pot)
            s.set_interaction(g)
            s.set_state(orb, coef)
            jp = f"{out_base}_job{j}"
            if imag:
                record_raw_state(jp + "_init", orb, coef)
            else:
                d = s.get()
                append_processed_state(jp, d["rho1"], d["rho2"], d["orb"], new=True)
                append_timestep_potential(jp, pot, new=True)
            td = (not imag) and time_dependent(job)
            prev_e = s.energy().real / job.npar
            robust = converged = False
            nsteps, t = 0, 0.0
            while t < job.tend:
                if td:
                    s.step_phase(0, stream)
                    tn = (nsteps + 1) * job.tstep
                    pot = builtin_potential(job.pot_func, tn, x, job.pot_params)
                    g = builtin_time_parameter(job.g_func, tn, job.g_params)
                    s.set_potential(pot)
                    s.set_interaction(g)
                    s.step_phase(1, stream)
                else:
                    s.step(1, stream)
                nsteps += 1
                t = nsteps * job.tstep
                if not imag and nsteps % rec_n == 0:
                    d = s.get()
                    append_processed_state(jp, d["rho1"], d["rho2"], d["orb"])
                    append_timestep_potential(jp, pot)
                if nsteps % mon_n == 0:
                    if imag and mon["auto_check"]:  # driver.c:46-67
                        e_tot = s.energy().real
                        cur = e_tot / job.npar
                        etol = 0.1 ** mon["energy_digits"] * prev_e
                        if abs(cur - prev_e) < etol and \
                                s.eig_residual(e_tot) < mon["eig_residue"]:
                            converged = True
                            break
                        prev_e = cur
                    if not imag:  # driver.c:69-96
                        o = s.overlap_residual()
                        if o > mon["overlap_threshold"] and not robust:
                            s.set_orthogonality(True)
                            robust = True
                        if o > REALTIME_OVERLAP_RESIDUE_TOL:
                            raise RuntimeError(f"job {j}: overlap residue {o:.3E} above "
                                               f"{REALTIME_OVERLAP_RESIDUE_TOL} at step {nsteps}")
            e = s.energy().real
            if imag:
                lan_it = lanczos_iterations_for(dim)
                if mon["final_diag"] and t >= job.tend and lan_it > 0:
                    s.lowest_state(lan_it)
                d = s.get()
                record_potential(jp, pot)
                record_raw_state(jp, d["orb"], d["coef"])
            else:
                record_time_interaction(jp, job, rec_n)
                record_time_array(jp, job.tend, job.tstep, rec_n)
            append_mctdhb_parameters(out_base, job, g, e, new=(j == 1))
            energies.append({"energy": e, "steps": nsteps, "converged": converged})
        finally:
            s.close()
    return energies
