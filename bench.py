"""Benchmark of batched MCTDHB on B200.

Headline (the batched workload): 256 independent imaginary-time relaxations
of uneven size -- N ~ U{10..60}, M in {3,4,5,6}, grid in {256, 512, 1024}
points on [-10, 10], g ~ U(0.01, 1), harmonic or double-well trap by a
seeded coin, RK5 orbitals, Lanczos dimension 5, energy rule 1e-10 checked
every step, 5000-step limit -- resident together in the batched engine and
advanced by one CUDA graph launch per step of the whole batch.  The unit of
work is one full step (orbitals, h and g, SIL, rho1 and rho2) of one system,
an "instance-step"; value = instance-steps/s.  Beside it:

  plain       the same jobs advanced one at a time by the plain single-system
              solver (two CUDA graphs per step), instance-steps/s;
  roofline    the dominant kernel of a batch step, the batched H.C of one
              orbital count, against the measured HBM copy bandwidth;
  quench      the N=30 M=8 real-time quench (nc = 10,295,472, grid 1024 on
              [-15, 15], double well, g = 0.1, Lanczos 6, dt = 0.005):
              configurational step (SIL + rho1 + rho2, one CUDA graph) and the
              H.C kernel's HBM GB/s;
  serving     a Poisson stream of 70% relaxations and 30% real-time quenches
              admitted by HBM footprint into the running batch (continuous
              batching), p50/p99 latency and jobs/s at a sweep of arrival
              rates, against the same arrivals served one at a time by the
              plain solver (first come first served, each job's service time
              measured alone on the GPU);
  e2e         the batched workload through the public API from host memory:
              admission (state upload), steps, fetch of every result.

dt: the configured dt (0.01 imaginary, 0.005 real time) capped at
1.5 / lambda_max, lambda_max = 4 |d2coef| / dx^2 + max V the largest
eigenvalue of the finite-difference one-body operator, which keeps the
explicit RK5 orbital step inside its stability region on the finer grids.
Inputs are seeded synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  Multi-GPU: one process per GPU (torchrun),
each rank runs its own 256-job mix (independent systems shard with no
collective; weak scaling); value = instance-steps/s summed over ranks, timed
as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "1d-mctdhb_b200"))

METRIC = "batched_mctdhb_instance_steps_per_s"
HBM_FALLBACK = 6650.0

# batched workload
MIX_N, MIX_SEED = 256, 2024
BXI, BXF = -10.0, 10.0
LZ = 5  # DEFAULT_LANCZOS_ITER of the reference
GRIDS = (256, 512, 1024)

# the N=30 M=8 quench
N_PAR, N_ORB, Q_LZ, Q_DT = 30, 8, 6, 0.005
Q_GRID, Q_XI, Q_XF, Q_G = 1024, -15.0, 15.0, 0.1


# ---------------------------------------------------------------------------
# synthetic inputs
# ---------------------------------------------------------------------------
def simpson_weights(n, h):
    """composite Simpson weights, 3/8 rule on the last four points when n is
    even (calculus.c:9-40 of the reference)"""
    w = np.zeros(n)
    if n % 2 == 0:
        for i in range(0, n - 4, 2):
            w[i:i + 3] += [1.0, 4.0, 1.0]
        w[: n - 3] *= h / 3
        w[n - 4:] += np.array([1.0, 3.0, 3.0, 1.0]) * 3 * h / 8
    else:
        for i in range(0, n - 2, 2):
            w[i:i + 3] += [1.0, 4.0, 1.0]
        w *= h / 3
    return w


_ORB = {}


def hermite_orbitals(M, G, xi, xf):
    """Hermite-Gaussian orbitals n = 0..M-1 orthonormalised by Gram-Schmidt
    in the Simpson metric"""
    key = (M, G, xi, xf)
    if key not in _ORB:
        x = np.linspace(xi, xf, G)
        w = simpson_weights(G, x[1] - x[0])
        phi = np.zeros((M, G), np.complex128)
        hm, hc = np.zeros(G), np.exp(-x ** 2 / 2)
        for n in range(M):
            phi[n] = hc
            hm, hc = hc, (np.sqrt(2.0) * x * hc - np.sqrt(n) * hm) / np.sqrt(n + 1)
        for i in range(M):
            for j in range(i):
                phi[i] -= np.sum(w * phi[j].conj() * phi[i]) * phi[j]
            phi[i] /= np.sqrt(np.sum(w * np.abs(phi[i]) ** 2))
        _ORB[key] = phi
    return _ORB[key]


def trap(double_well, G, xi, xf):
    x = np.linspace(xi, xf, G)
    v = 0.5 * x ** 2
    return v + 4.0 * np.exp(-x ** 2 / 0.5) if double_well else v


def stable_dt(dt, G, pot, xi, xf, d2coef=-0.5):
    dx = (xf - xi) / (G - 1)
    lam = 4.0 * abs(d2coef) / dx ** 2 + float(np.max(pot))
    return min(dt, 1.5 / lam)


def dim(N, M):
    from math import comb

    return comb(N + M - 1, M - 1)


def distinct_couplings(N, M):
    """G = sum over configurations of the distinct neighbours reached by one
    or two boson moves (closed form over (occupied, doubly occupied) counts)."""
    from math import comb

    tot = 0
    for o in range(1, M + 1):
        for d2 in range(0, o + 1):
            R = N - o - d2
            if R < 0:
                continue
            ways = (1 if R == 0 else 0) if d2 == 0 else comb(R + d2 - 1, d2 - 1)
            cnt = comb(M, o) * comb(o, d2) * ways
            tot += cnt * (o * (M - 1) + comb(o, 2) * (M - 2) * (M - 1) // 2 +
                          d2 * (M - 1) * M // 2)
    return tot


def coefficients(nc, rng):
    c = rng.normal(size=nc) + 1j * rng.normal(size=nc)
    return c / np.linalg.norm(c)


def make_job(rng, N, M, G, imag, steps, xi=BXI, xf=BXF, big=False, coef_rng=None):
    """one job: trap (harmonic or double well by a coin), g ~ U(0.01, 1),
    Hermite-Gaussian orbitals, seeded normalised random coefficients (from
    coef_rng when given, else from rng after the job's other draws)"""
    dw = bool(rng.random() < 0.5)
    pot = trap(dw, G, xi, xf)
    g = float(rng.uniform(0.01, 1.0))
    return {"npar": int(N), "norb": int(M), "grid_size": int(G), "xi": xi, "xf": xf,
            "periodic": 1, "imagtime": int(imag), "rk_order": 5,
            "dt": stable_dt(0.01 if imag else 0.005, G, pot, xi, xf), "g": g,
            "max_steps": int(steps), "energy_tol": 1e-10 if imag else 0.0,
            "check_every": 1 if imag else 0, "pot": pot,
            "orbitals": hermite_orbitals(M, G, xi, xf),
            "coef": coefficients(dim(N, M), rng if coef_rng is None else coef_rng),
            "big": big}


def mix_sizes(n=MIX_N, seed=MIX_SEED):
    """(N, M, grid) of the batched workload's jobs: one seeded stream of
    sizes, traps and interactions; job i's coefficients come from its own
    stream (seed, i), so any subset of jobs can be built alone"""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(rng.integers(10, 61))
        M = int(rng.choice([3, 4, 5, 6]))
        G = int(rng.choice(GRIDS))
        rng.random()      # trap coin
        rng.uniform()     # interaction
        out.append((N, M, G))
    return out


def mix_jobs(n=MIX_N, seed=MIX_SEED, max_steps=5000, keep=None):
    """the batched workload: n imaginary-time relaxations of uneven size
    (only the indices in `keep`, when given, in index order)"""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        N = int(rng.integers(10, 61))
        M = int(rng.choice([3, 4, 5, 6]))
        G = int(rng.choice(GRIDS))
        if keep is not None and i not in keep:
            rng.random()
            rng.uniform()
            continue
        jobs.append(make_job(rng, N, M, G, True, max_steps,
                             coef_rng=np.random.default_rng([seed, i])))
    return jobs


def footprint(N, M, G):
    """arena bytes of a mix job (mctdhb_batch_job_bytes; finite differences,
    periodic, Lanczos LZ)"""
    import mctdhb_b200 as mb

    one = np.zeros(1)
    return mb.Batch.job_bytes({"npar": N, "norb": M, "grid_size": G, "xi": BXI, "xf": BXF,
                               "periodic": 1, "imagtime": 1, "rk_order": 5, "dt": 0.01,
                               "g": 0.5, "max_steps": 1, "pot": one, "orbitals": one,
                               "coef": one, "der_method": 302}, LZ)


def rank_jobs(rank, world):
    """this rank's jobs: the whole job is MIX_N jobs per rank drawn from one
    seeded stream (its first MIX_N are the one-GPU mix), assigned to ranks by
    HBM footprint (partition.by_footprint); every rank computes the same
    assignment and builds only its own jobs -- no collective"""
    if world == 1:
        return mix_jobs(), None
    import partition

    sizes = mix_sizes(MIX_N * world)
    fp = [footprint(*x) for x in sizes]
    share = partition.by_footprint(fp, world)
    loads = partition.loads(fp, share)
    info = {"jobs": len(sizes), "rule": "longest-processing-time by mctdhb_batch_job_bytes",
            "bytes_per_rank_max_over_mean": max(loads) / (sum(loads) / world)}
    return mix_jobs(n=MIX_N * world, keep=set(share[rank])), info


def served_jobs(njobs, seed=77, imag_steps=5000, real_steps=500, big_frac=0.05, nmax=60):
    """the served job sequence: [(unit-rate arrival time, job)].  Arrival
    times are cumulative Exp(1) gaps, divided by the rate for a given rate,
    so every rate of a sweep serves the same jobs in the same order; 70%
    imaginary-time relaxations, 30% real-time quenches, big_frac of
    N=30 M=8 grid 1024 jobs"""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for _ in range(njobs):
        t += float(rng.exponential(1.0))
        imag = bool(rng.random() < 0.7)
        if rng.random() < big_frac:
            job = make_job(rng, 30, 8, 1024, imag, imag_steps if imag else real_steps,
                           Q_XI, Q_XF, big=True)
        else:
            job = make_job(rng, int(rng.integers(10, nmax + 1)), int(rng.choice([3, 4, 5, 6])),
                           int(rng.choice(GRIDS)), imag, imag_steps if imag else real_steps)
        out.append((t, job))
    return out


def mix_summary(jobs):
    ncs = [dim(j["npar"], j["norb"]) for j in jobs]
    return {"jobs": len(jobs), "sum_nc": int(sum(ncs)), "max_nc": int(max(ncs)),
            "by_norb": {str(m): sum(1 for j in jobs if j["norb"] == m) for m in (3, 4, 5, 6)},
            "by_grid": {str(g): sum(1 for j in jobs if j["grid_size"] == g) for g in GRIDS}}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [s.strip() for s in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK, "fallback"


def ncu_traffic():
    """per-launch DRAM bytes of the H.C kernels from the committed ncu summary"""
    try:
        with open(os.path.join(REPO, "profiles", "hc_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def workload_config(args, jobs):
    return {"workload": f"batched: {len(jobs)} imaginary-time relaxations, N~U{{10..60}}, "
                        "M in {3,4,5,6}, grid in {256,512,1024} on [-10,10], g~U(0.01,1), "
                        "harmonic or double-well trap, RK5 orbitals, Lanczos 5, energy rule "
                        "1e-10 every step, 5000-step limit, dt=min(0.01, 1.5/lambda_max)",
            "mix": mix_summary(jobs), "seed": MIX_SEED, "lanczos_iter": LZ,
            "step": "one full MCTDHB step of every running system: one CUDA graph launch",
            "parallelism": (f"dp{args.gpus}: {args.gpus} x {MIX_N} jobs of one seeded stream "
                            "assigned to GPUs by HBM footprint, no collective"
                            if args.gpus > 1 else "one GPU"),
            "l2": "inputs larger than L2 (the mix holds ~12 GB of coefficient and Krylov "
                  "vectors)"}


# ---------------------------------------------------------------------------
# CPU baseline: the compiled reference's own step on a sample of the jobs
# ---------------------------------------------------------------------------
REF_SAMPLE = 24     # jobs of the mix stepped by the reference arm
CPU_SAMPLE = 12     # jobs of the mix stepped for the GPU arm's cpu_baseline


def step_bytes(j, m=LZ):
    """algorithmic bytes of one full step of a job: m H.C launches
    (32 nc + 16 G each) and the densities (16 nc + 16 G)"""
    nc, G = dim(j["npar"], j["norb"]), distinct_couplings(j["npar"], j["norb"])
    return m * (32.0 * nc + 16.0 * G) + 16.0 * nc + 16.0 * G


def systematic_sample(jobs, n):
    """n jobs at evenly spaced ranks of the mix sorted by step cost
    (algorithmic bytes), largest first: the heavy-tailed mix (its 25 largest
    jobs carry ~85% of the bytes) is represented in proportion, from the
    largest jobs to the smallest"""
    order = sorted(range(len(jobs)), key=lambda i: -step_bytes(jobs[i]))
    return [order[int((k + 0.5) * len(jobs) / n)] for k in range(n)]


def sample_cost_ratio(jobs, idx):
    """mean step bytes of the sampled jobs over the mean of the whole mix:
    the sample's throughput estimates the mix's within about this factor"""
    return (sum(step_bytes(jobs[i]) for i in idx) / len(idx)) / \
        (sum(step_bytes(j) for j in jobs) / len(jobs))


class RefTimer:
    """The compiled reference (oracle/_ref: the reference's own C sources,
    OpenMP) stepping jobs of the mix one at a time, each by the reference's
    own mctdhb_propagate_step (driver.c:159-201).  A job's struct comes from
    oracle/ref_setup.c (the reference's sub-constructors, maps from the
    oracle's OpenMP builders) and its initial synchronisation from the
    reference (sync_orbital_matrices, sync_density_matrices); set-up is
    timed apart, only the step is the measured work."""

    def __init__(self):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from oracle import Reference

        self.R = Reference()
        self.setup_s = 0.0

    def threads(self, n=None):
        if n is not None:
            self.R.lib.omp_set_num_threads(int(n))
        return int(self.R.lib.omp_get_max_threads())

    def step_job(self, j):
        import ctypes

        import mctdhb_types as T

        R = self.R
        t0 = time.perf_counter()
        ms = R.make_job_struct(j, LZ)
        if ms is None:
            raise RuntimeError(f"reference cannot map N={j['npar']} M={j['norb']}")
        try:
            R.set_state(ms, j["orbitals"], j["coef"])
            ow = np.zeros(j["norb"] * j["grid_size"], np.complex128)
            cw = np.zeros(dim(j["npar"], j["norb"]), np.complex128)
            self.setup_s += time.perf_counter() - t0
            t1 = time.perf_counter()
            R.lib.mctdhb_propagate_step(ms, T.carray(ow), T.carray(cw), ctypes.c_uint32(0))
            return time.perf_counter() - t1
        finally:
            R.destroy_job_struct(ms)

    def map_build(self, j):
        """seconds of the reference's own serial map build
        (get_multiconf_struct, types_definition.c:111-142) and of the
        oracle's parallel one used for set-up, on one job"""
        R = self.R
        out = {}
        for name, fn in (("reference_serial_s", R.lib.get_multiconf_struct),
                         ("setup_parallel_s", R.lib.refset_multiconf)):
            t0 = time.perf_counter()
            mc = fn(j["npar"], j["norb"])
            out[name] = time.perf_counter() - t0
            R.lib.destroy_multiconf_struct(mc)
        out["job"] = f"N={j['npar']} M={j['norb']} (nc={dim(j['npar'], j['norb'])})"
        return out


def port_step(O, j):
    """seconds of one full step of the oracle's C restatement on a job"""
    st, dx = oracle_state(O, j)
    t0 = time.perf_counter()
    O.propagate_step(st, j["npar"], dx, j["dt"], -0.5, 0.0, j["g"], True, bool(j["imagtime"]),
                     j["rk_order"], LZ, j["pot"])
    return time.perf_counter() - t0


def oracle_state(O, j):
    orb = np.ascontiguousarray(j["orbitals"].copy())
    G = j["grid_size"]
    dx = (j["xf"] - j["xi"]) / (G - 1)
    r1, r2, ri = O.sync_density_matrices(j["npar"], j["norb"], j["coef"])
    return {"orb": orb, "coef": np.ascontiguousarray(j["coef"].copy()),
            "hob": np.ascontiguousarray(O.orbital_hob(orb, dx, -0.5, 0.0, j["pot"])),
            "hint": np.ascontiguousarray(O.orbital_hint(orb, dx, j["g"])),
            "rho1": np.ascontiguousarray(r1), "rho2": np.ascontiguousarray(r2),
            "rinv": np.ascontiguousarray(ri)}, dx


def ref_sample_desc(jobs, idx, threads, what):
    return (f"{what}: one full step (RK5 orbitals, h, g, SIL({LZ}), rho1, rho2) of each of "
            f"{len(idx)} jobs of the {len(jobs)}-job mix at evenly spaced ranks of step cost, "
            f"by the compiled reference's own mctdhb_propagate_step (OpenMP, {threads} host "
            f"threads); set-up (maps, initial densities) not timed; sample mean step bytes "
            f"{sample_cost_ratio(jobs, idx):.3f} x the mix mean")


def cpu_sample(jobs):
    """the GPU arm's cpu_baseline: the compiled reference on a bounded
    systematic sample of the mix, all host threads"""
    rt = RefTimer()
    idx = systematic_sample(jobs, CPU_SAMPLE)
    t = sum(rt.step_job(jobs[i]) for i in idx)
    threads = rt.threads()
    return {"value": len(idx) / t, "unit": "instance-steps/s", "cores": threads,
            "kind": "reference", "seconds": t, "setup_seconds": rt.setup_s,
            "sample": ref_sample_desc(jobs, idx, threads, "measured")}


def run_reference(args):
    """the reference arm: the compiled reference's own step on the host
    cores, same metric (instance-steps/s of the batched mix).  The K timed
    steps share a systematic sample of REF_SAMPLE jobs (step s takes the
    sample's jobs s, s+K, ...); value = job-steps done / seconds of the
    reference's steps.  Rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    jobs = mix_jobs()
    rt = RefTimer()
    cores = rt.threads()
    idx = systematic_sample(jobs, max(REF_SAMPLE, args.steps))
    small = min(idx, key=lambda i: step_bytes(jobs[i]))
    for _ in range(args.warmup):
        rt.step_job(jobs[small])
    per_step = [0.0] * args.steps
    done = 0
    for s in range(args.steps):
        for i in idx[s::args.steps]:
            per_step[s] += rt.step_job(jobs[i])
            done += 1
    total = sum(per_step)
    v = done / total
    base = {"value": v, "unit": "instance-steps/s", "cores": cores, "kind": "reference",
            "seconds": total, "setup_seconds": rt.setup_s,
            "sample": ref_sample_desc(jobs, idx, cores, f"per timed step, 1/{args.steps} of")}
    # the reference application's default of half the host threads
    # (apps/mctdhb_main.c:138), on every fourth job of the sample
    half = max(1, cores // 2)
    rt.threads(half)
    sub = idx[::4]
    th = sum(rt.step_job(jobs[i]) for i in sub)
    rt.threads(cores)
    th_all = sum(rt.step_job(jobs[i]) for i in sub)
    maps = rt.map_build(jobs[idx[len(idx) // 2]])
    # the oracle's C restatement against the reference, same jobs
    from oracle import Oracle

    O = Oracle()
    calib = []
    for i in (idx[2], idx[len(idx) // 2], idx[-2]):
        j = jobs[i]
        tr, tp = rt.step_job(j), port_step(O, j)
        calib.append({"job": f"N={j['npar']} M={j['norb']} G={j['grid_size']}",
                      "reference_s": tr, "port_s": tp, "reference_over_port": tr / tp})
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "instance-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": workload_config(args, jobs), "cpu_baseline": base,
        "half_threads": {"threads": half, "value": len(sub) / th, "jobs": len(sub),
                         "unit": "instance-steps/s",
                         "what": "the reference application's default thread count "
                                 "(apps/mctdhb_main.c:138), every fourth sampled job",
                         "all_threads_value_same_jobs": len(sub) / th_all},
        "map_build": maps, "port_vs_reference": calib,
        "e2e": {"value": v, "unit": "instance-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_reference_full_mix(args):
    """one complete step of all 256 jobs of the mix by the compiled
    reference (long: minutes), with the systematic samples' estimates
    beside it"""
    jobs = mix_jobs()
    rt = RefTimer()
    t = [rt.step_job(j) for j in jobs]
    full = len(jobs) / sum(t)
    out = {"impl": "reference", "what": "one complete step of the whole mix, compiled reference",
           "value": full, "unit": "instance-steps/s", "seconds": sum(t),
           "setup_seconds": rt.setup_s, "cores": rt.threads()}
    for n in (CPU_SAMPLE, REF_SAMPLE):
        ix = systematic_sample(jobs, n)
        est = n / sum(t[i] for i in ix)
        out[f"sample_{n}"] = {"value": est, "rel_error": est / full - 1.0,
                              "cost_ratio": sample_cost_ratio(jobs, ix)}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# batched engine and the plain path
# ---------------------------------------------------------------------------
def arena_bytes(mb, jobs, slack=1.02):
    return int(sum(mb.Batch.job_bytes(j, LZ) for j in jobs) * slack) + (64 << 20)


def fp64_mma_peak(mb, torch, reps=5):
    """measured FP64 tensor-core throughput (TFLOP/s) of this GPU: the
    library's mma.sync m16n8k8 f64 probe, 4 blocks of 256 threads per SM,
    timed with CUDA events; the best of `reps` launches"""
    blocks, iters = 4 * torch.cuda.get_device_properties(0).multi_processor_count, 2048
    out = torch.empty(blocks * 256, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    mb.fp64_mma_probe(blocks, iters, out, st)
    best = float("inf")
    for _ in range(reps):
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        mb.fp64_mma_probe(blocks, iters, out, st)
        c.record(st)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(c))
    return blocks * 8 * iters * 4 * 2048 / (best / 1000.0) / 1e12


def pair_work(jobs, M):
    """per launch of the batched H.C of the jobs with M orbitals:
    contraction FLOPs (8 per complex multiply-add of Y = A W^T over the
    N-2 boson space) and gather-back bytes (every Y value read once, H.C
    written once)"""
    from math import comb

    P = M * (M + 1) // 2
    d2 = sum(comb(j["npar"] - 2 + M - 1, M - 1) for j in jobs if j["norb"] == M)
    nc = sum(dim(j["npar"], M) for j in jobs if j["norb"] == M)
    return 8.0 * d2 * P * P, 16.0 * d2 * P + 16.0 * nc, d2


def batch_hc_roofline(mb, torch, b, jobs, reps=5):
    """time each orbital count's batched H.C on the engine's stream, the pair
    contraction and the gather-back separately"""
    st = b.stream

    def timed(M, parts):
        b.launch_hc(M, parts)
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(reps):
            b.launch_hc(M, parts)
        c.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(c) / reps

    out = {}
    for M in sorted({j["norb"] for j in jobs}):
        flops, byts, d2 = pair_work(jobs, M)
        ty, tg = timed(M, 1), timed(M, 2)
        out[M] = {"contraction_ms": ty, "contraction_flops": flops,
                  "contraction_tflops": flops / (ty / 1000.0) / 1e12,
                  "gather_back_ms": tg, "gather_back_bytes": byts,
                  "gather_back_gbs": byts / (tg / 1000.0) / 1e9, "rows_n_minus_2": d2}
    return out


def plain_timed(mb, torch, jobs, warmup, steps, compare=None):
    """the same jobs one at a time through the plain solver: per job, set-up
    and `warmup` untimed steps, then `steps` steps timed with CUDA events.
    compare: {job index: total steps} -- those jobs are run on to that many
    steps in all and their energies returned."""
    compare = compare or {}
    stream = torch.cuda.current_stream()
    total, energies, per_job = 0.0, {}, []
    for i, j in enumerate(jobs):
        s = mb.Solver(j["npar"], j["norb"], j["grid_size"], j["xi"], j["xf"], j["dt"],
                      bool(j["imagtime"]), j["rk_order"], LZ, periodic=bool(j["periodic"]))
        s.set_potential(j["pot"])
        s.set_interaction(j["g"])
        s.set_state(j["orbitals"], j["coef"])
        s.step(warmup, stream)
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.step(steps, stream)
        c.record(stream)
        torch.cuda.synchronize()
        total += a.elapsed_time(c) / 1000.0
        per_job.append(a.elapsed_time(c) / 1000.0 / steps)
        if i in compare:
            extra = compare[i] - warmup - steps
            if extra > 0:
                s.step(extra, stream)
            energies[i] = s.energy().real
        s.close()
    n = len(jobs) * steps
    return {"value": n / total, "unit": "instance-steps/s", "seconds": total,
            "instance_steps": n, "seconds_per_step_by_job": per_job,
            "what": f"the same jobs one at a time through mctdhb_solver (two CUDA graphs per "
                    f"step), {steps} timed steps per job after set-up and {warmup} untimed"}, \
        energies


def e2e_batch(mb, torch, jobs, steps):
    """end to end through the public API from pinned host memory: admit
    every job (its trap, orbitals and coefficients uploaded), `steps` steps,
    fetch every job's orbitals, coefficients and densities into pinned
    buffers; wall clock around all of it.  The engine (its arena) is created
    before, as a server creates it once."""

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(a).dtype, pin_memory=True)
        v = t.numpy()
        v[...] = a
        return t, v

    keep, pjobs, outs = [], [], []
    for j in jobs:
        pj = dict(j)
        for k in ("pot", "orbitals", "coef"):
            t, v = pinned(np.ascontiguousarray(j[k]))
            keep.append(t)
            pj[k] = v
        pjobs.append(pj)
        M, G, nc = j["norb"], j["grid_size"], dim(j["npar"], j["norb"])
        o = {}
        for k, shape in (("orb", (M, G)), ("coef", (nc,)), ("rho1", (M, M)), ("rho2", (M ** 4,))):
            t, v = pinned(np.zeros(shape, np.complex128))
            keep.append(t)
            o[k] = v
        outs.append(o)
    b = mb.Batch(len(jobs), arena_bytes(mb, jobs), LZ)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    slots = [b.admit(j) for j in pjobs]
    b.step(steps)
    outs = [b.fetch(s, out=o) for s, o in zip(slots, outs)]
    t1 = time.perf_counter()
    b.close()
    h2d = sum(16 * (dim(j["npar"], j["norb"]) + j["norb"] * j["grid_size"]) + 8 * j["grid_size"]
              for j in jobs)
    d2h = sum(o["coef"].nbytes + o["orb"].nbytes + o["rho1"].nbytes + o["rho2"].nbytes
              for o in outs)
    return {"value": len(jobs) * steps / (t1 - t0), "unit": "instance-steps/s",
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "seconds": t1 - t0, "steps": steps,
            "path": "mctdhb_batch_admit (pinned host state) + mctdhb_batch_step + "
                    "mctdhb_batch_fetch (into pinned host buffers), wall clock"}


# ---------------------------------------------------------------------------
# serving: continuous batching against one-at-a-time
# ---------------------------------------------------------------------------
# jobs with at least this many configurations fill the GPU alone (N=30 M=8:
# 10.3 M); the server runs them in its solver lane beside the batch
HEAVY_NC = 9_000_000


def serve_batched(mb, arrivals, arena, max_slots=512, steps_per_tick=2):
    """continuous batching in real time through the package's request loop
    (serving.Server): jobs admitted first come first served once arrived and
    once they fit in the arena, advanced together, retired when they stop;
    jobs of HEAVY_NC configurations or more in the server's solver lane.
    Returns latencies, the makespan and the jobs' final energies."""
    from serving import Server

    srv = Server(arena, max_slots=max_slots, lanczos_iter=LZ, steps_per_tick=steps_per_tick,
                 heavy_nc=HEAVY_NC)
    try:
        ids = [srv.submit(j, at=t) for t, j in arrivals]
        srv.run()
        st = srv.stats()
        return ([srv.latency(i) for i in ids], st["makespan_s"],
                [srv.result(i)["energy"] for i in ids], st)
    finally:
        srv.close()


def plain_job(mb, torch, j):
    """one job alone through the plain solver to its own stop: the
    imaginary-time energy rule or the step limit, evaluated on the device
    (mctdhb_solver_relax: one graph launch, no host round trip per step)"""
    s = mb.Solver(j["npar"], j["norb"], j["grid_size"], j["xi"], j["xf"], j["dt"],
                  bool(j["imagtime"]), j["rk_order"], LZ, periodic=bool(j["periodic"]))
    try:
        s.set_potential(j["pot"])
        s.set_interaction(j["g"])
        s.set_state(j["orbitals"], j["coef"])
        check = j["check_every"] if j["imagtime"] else 0
        s.relax(j["max_steps"], j["energy_tol"], check, torch.cuda.current_stream())
        steps, _ = s.relax_result()
        return s.energy().real, steps
    finally:
        s.close()


def serve_plain(mb, torch, arrivals):
    """one-at-a-time serving in real time: the jobs in arrival order, each
    started when it has arrived and the previous one has finished, run alone
    by plain_job; latency = finish - arrival"""
    t0 = time.perf_counter()
    lat, energy = [], []
    for ta, j in arrivals:
        now = time.perf_counter() - t0
        if now < ta:
            time.sleep(ta - now)
        e, _ = plain_job(mb, torch, j)
        energy.append(e)
        lat.append(time.perf_counter() - t0 - ta)
    return lat, time.perf_counter() - t0 - arrivals[0][0], energy


def run_mix_convergence(mb, torch, chunk=20):
    """the batched workload as configured, to the end: every job of the mix
    relaxed until its energy changes by less than 1e-10 between steps or
    5000 steps, batched (all admitted at once, `chunk` batch steps between
    polls) against the plain path (each job alone to its own stop through
    mctdhb_solver_relax, one after the other).  Wall clock; the jobs' step
    counts and energies of the two paths are compared."""
    jobs = mix_jobs()
    b = mb.Batch(len(jobs), arena_bytes(mb, jobs), LZ)
    slots = [b.admit(j) for j in jobs]
    assert None not in slots, "the arena is sized for every job"
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done_at = {}
    while True:
        b.step(chunk)
        n, st, _, _ = b.poll()
        now = time.perf_counter() - t0
        for i, s in enumerate(slots):
            if st[s] != 1 and i not in done_at:
                done_at[i] = now
        if n == 0:
            break
    t_b = time.perf_counter() - t0
    res_b = []
    for s in slots:
        r = b.fetch(s)
        res_b.append({k: r[k] for k in ("energy", "steps", "converged")})
    b.close()
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    plain_e, plain_steps, plain_done = [], [], []
    for j in jobs:
        e, n = plain_job(mb, torch, j)
        plain_e.append(e)
        plain_steps.append(n)
        plain_done.append(time.perf_counter() - t0)
    t_p = time.perf_counter() - t0
    steps_b = [int(r["steps"]) for r in res_b]
    e_b = [float(r["energy"]) for r in res_b]
    return {
        "jobs": len(jobs), "energy_tol": 1e-10, "max_steps": 5000,
        "batched": {"makespan_s": t_b, "p50_done_s": float(np.median(list(done_at.values()))),
                    "converged": sum(1 for r in res_b if r["converged"]),
                    "steps_mean": float(np.mean(steps_b)), "steps_max": max(steps_b),
                    "poll_every_steps": chunk},
        "plain": {"makespan_s": t_p, "p50_done_s": float(np.median(plain_done))},
        "makespan_speedup": t_p / t_b,
        "steps_equal": steps_b == plain_steps,
        "energy_max_rel_diff": max(abs(a - c) / abs(c) for a, c in zip(e_b, plain_e)),
        "what": "the whole mix relaxed to its stop rule, batched against one job at a time "
                "(wall clock, both on the device with the same stop rule)"}


def percentiles(lat):
    a = np.asarray(lat)
    return {"p50_s": float(np.percentile(a, 50)), "p99_s": float(np.percentile(a, 99)),
            "mean_s": float(a.mean()), "max_s": float(a.max())}


def run_serving(mb, torch, rates, njobs, imag_steps, real_steps, big_frac, nmax):
    """the served workload: a Poisson stream of 70% imaginary-time
    ground-state jobs (energy rule 1e-10 or imag_steps steps) and 30%
    real-time quenches (real_steps steps, dt 0.005 capped for RK5
    stability), sizes as the batched mix plus big_frac N=30 M=8 jobs; at each
    arrival rate both servers run the same stream in real time"""
    seq = served_jobs(njobs, imag_steps=imag_steps, real_steps=real_steps, big_frac=big_frac,
                      nmax=nmax)
    jobs = [j for _, j in seq]
    unit = [t for t, _ in seq]
    arena = min(arena_bytes(mb, [j for j in jobs if dim(j["npar"], j["norb"]) < HEAVY_NC] or
                            jobs[:1]), 96 << 30)
    out = {"jobs": len(jobs), "imag_steps": imag_steps, "real_steps": real_steps,
           "big_frac": big_frac, "big_jobs": sum(1 for j in jobs if j["big"]), "nmax": nmax,
           "arena_bytes": arena,
           "batched_method": "serving.Server: FCFS admission by footprint into the running "
                             "batch, 2 batch steps per tick, retirement as jobs stop; jobs of "
                             f"{HEAVY_NC} configurations or more one at a time in the server's "
                             "solver lane beside the batch",
           "plain_method": "one at a time in arrival order, each alone through mctdhb_solver "
                           "with the same stop rules on the device (mctdhb_solver_relax), "
                           "run in real time at every rate",
           "rates": []}
    worst = 0.0
    for r in rates:
        arr = [u / r for u in unit]
        lat_b, t_b, e_b, st_b = serve_batched(mb, list(zip(arr, jobs)), arena)
        lat_p, t_p, e_p = serve_plain(mb, torch, list(zip(arr, jobs)))
        worst = max(worst, max(abs(x - y) / abs(y) for x, y in zip(e_b, e_p)))
        out["rates"].append({
            "rate_jobs_per_s": r,
            "batched": dict(percentiles(lat_b), jobs_per_s=len(jobs) / t_b, makespan_s=t_b,
                            peak_running=st_b["peak_running"]),
            "plain": dict(percentiles(lat_p), jobs_per_s=len(jobs) / t_p, makespan_s=t_p),
            "p99_speedup": float(np.percentile(lat_p, 99) / np.percentile(lat_b, 99)),
            "throughput_speedup": t_p / t_b})
    out["energy_max_rel_diff_batched_vs_plain"] = worst
    return out


# ---------------------------------------------------------------------------
# the N=30 M=8 quench: configurational step and the H.C roofline
# ---------------------------------------------------------------------------
SINGLE = {
    "quench_n30_m8": dict(
        N=N_PAR, M=N_ORB, G=Q_GRID, xi=Q_XI, xf=Q_XF, double_well=True, g=Q_G, m=Q_LZ,
        dt=Q_DT, seed=1234,
        workload="real-time quench N=30 M=8 (nc=10295472), grid 1024 on [-15,15], "
                 "V=x^2/2+4exp(-x^2/0.5), g=0.1, Lanczos 6, dt=0.005"),
    "memory_edge_n100_m6": dict(
        N=100, M=6, G=2048, xi=-20.0, xf=20.0, double_well=False, g=0.02, m=LZ, dt=0.001,
        seed=4321,
        workload="single system at the memory edge N=100 M=6 (nc=96560646, 1.5 GB per "
                 "vector), grid 2048 on [-20,20], V=x^2/2, g=0.02, Lanczos 5, dt=0.001, "
                 "real time"),
}


def single_inputs(mb, c):
    """h and g of the Hermite-Gaussian orbitals of a configuration (4th-order
    periodic finite differences, Simpson weights) and seeded normalised
    random coefficients"""
    N, M, G, xi, xf = c["N"], c["M"], c["G"], c["xi"], c["xf"]
    x = np.linspace(xi, xf, G)
    phi = hermite_orbitals(M, G, xi, xf)
    dx = x[1] - x[0]
    w = simpson_weights(G, dx)
    d = (np.roll(phi, 2, 1) - np.roll(phi, -2, 1) +
         8 * (np.roll(phi, -1, 1) - np.roll(phi, 1, 1))) / (12 * dx)
    hob = 0.5 * np.einsum("x,ax,bx->ab", w, d.conj(), d) + \
        np.einsum("x,ax,bx->ab", w * trap(c["double_well"], G, xi, xf), phi.conj(), phi)
    t = c["g"] * np.einsum("x,ax,bx,cx,dx->abcd", w, phi.conj(), phi.conj(), phi, phi)
    hint = np.ascontiguousarray(t.transpose(3, 2, 1, 0)).reshape(-1)
    c0 = coefficients(int(mb.load().space_dimension(N, M)), np.random.default_rng(c["seed"]))
    return np.ascontiguousarray(hob), hint, c0


def run_single(mb, torch, name, steps, warmup):
    """one system of a full-size configuration: the configurational step
    (SIL + rho1 + rho2, one CUDA graph) and its H.C and density kernels"""
    c = SINGLE[name]
    N, M = c["N"], c["M"]
    stream = torch.cuda.current_stream()
    hob, hint, c0 = single_inputs(mb, c)
    sp = mb.Space(N, M)
    nc = sp.dim
    d_c = torch.from_numpy(c0).cuda()
    del c0
    sp.set_matrices(torch.from_numpy(hob.reshape(-1)).cuda(), torch.from_numpy(hint).cuda())
    r1 = torch.empty(M * M, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(M ** 4, dtype=torch.complex128, device="cuda")
    step = mb.Step(sp, d_c, r1, r2, c["m"], c["dt"], False)
    for _ in range(warmup):
        step.launch(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step.launch(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_step = e0.elapsed_time(e1) / steps
    norm = float(torch.linalg.vector_norm(d_c).item())
    assert abs(norm - 1.0) < 1e-10, f"real-time SIL must conserve the norm, got {norm}"
    step.close()
    hc_out = torch.empty_like(d_c)
    for _ in range(2):
        sp.apply_hamiltonian(d_c, hc_out, stream)
        sp.density_matrices(d_c, r1, r2, stream)
    reps = 5
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        sp.apply_hamiltonian(d_c, hc_out, stream)
    b.record(stream)
    torch.cuda.synchronize()
    t_hc = a.elapsed_time(b) / reps / 1000.0
    a.record(stream)
    for _ in range(reps):
        sp.density_matrices(d_c, r1, r2, stream)
    b.record(stream)
    torch.cuda.synchronize()
    t_dn = a.elapsed_time(b) / reps / 1000.0
    G = distinct_couplings(N, M)
    b_hc = 32.0 * nc + 16.0 * G
    from math import comb

    P = M * (M + 1) // 2
    d2 = comb(N - 2 + M - 1, M - 1)
    f_hc = 8.0 * d2 * P * P
    f_dn = 8.0 * d2 * P * (P + 1) / 2  # upper triangle of the rho2 Gram matrix
    variant = mb.tune_get("hcp_y", N, M)
    sp.close()
    del sp, d_c, hc_out
    torch.cuda.empty_cache()
    return {"workload": c["workload"], "tuned_variant_hcp_y": variant,
            "step": f"SIL({c['m']} H.C) + rho1 + rho2, one CUDA graph",
            "steps_per_s": 1000.0 / t_step, "ms_per_step": t_step, "norm_after": norm,
            "hc": {"kernels": f"hcp_y_kernel<{M}> (pair contraction, FP64 mma.sync) + "
                              f"hcp_g_kernel<{M}> (gather-back)",
                   "ms_per_launch": t_hc * 1e3, "contraction_flops": f_hc,
                   "contraction_tflops_over_hc_time": f_hc / t_hc / 1e12,
                   "contraction_tflops_note": "the contraction's FLOPs over the whole H.C time "
                                              "(contraction + gather-back); the contraction "
                                              "alone is timed by ncu under profiles/",
                   "pair_scratch_bytes": 16.0 * d2 * P,
                   "gather_model_gbs": b_hc / t_hc / 1e9,
                   "gather_model_note": "32 nc + 16 G bytes (one 16-byte gather per distinct "
                                        "coupling) / time: the rate a gather-per-coupling H.C "
                                        "would need to match this launch"},
            "density": {"kernels": f"gram_kernel<{M},2> + finalize + rho1 from rho2",
                        "ms_per_launch": t_dn * 1e3, "gram_flops": f_dn,
                        "gram_tflops": f_dn / t_dn / 1e12}}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def combine_ranks(dist, t_ms, inst, device):
    """whole-job figures of a multi-rank run: the timed region is the max
    over ranks, instance-steps are summed (each rank runs its own mix with no
    collective in the data path)"""
    if dist is None:
        return t_ms, inst
    import torch

    t = torch.tensor([t_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([inst], dtype=torch.float64, device=device)
    dist.all_reduce(n)
    return float(t.item()), int(n.item())


def run_gpu(args):
    import torch

    import mctdhb_b200 as mb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    jobs, part = rank_jobs(rank, world)
    b = mb.Batch(len(jobs), arena_bytes(mb, jobs), LZ)
    slots = [b.admit(j) for j in jobs]
    assert None not in slots, "the arena is sized for every job"
    b.step(args.warmup)
    b.sync()
    _, _, s0, _ = b.poll()
    st = b.stream
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.profiler.start()  # ncu --profile-from-start off sees the timed steps only
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    b.step(args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_ms = e0.elapsed_time(e1)
    _, state, s1, energy = b.poll()
    inst = int(np.sum(s1.astype(np.int64) - s0.astype(np.int64)))
    t_ms, inst_all = combine_ranks(dist, t_ms, inst, "cuda")
    value = inst_all / (t_ms / 1000.0)
    kernels = b.kernels
    line = {
        "metric": METRIC, "value": value, "unit": "instance-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": workload_config(args, jobs),
        "instance_steps": inst_all, "clocks": clk, "gpu_launches": kernels * args.steps,
        "kernels_per_step": kernels,
    }
    if part is not None:
        line["partition"] = part
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        b.close()
        return

    # roofline: the dominant kernel of the step, the batched H.C per M
    peak, kind = peaks()
    groups = batch_hc_roofline(mb, torch, b, jobs)
    mma_peak = fp64_mma_peak(mb, torch)
    Mtop = max(groups, key=lambda m: groups[m]["contraction_ms"] + groups[m]["gather_back_ms"])
    gt = groups[Mtop]
    tr = ncu_traffic()
    traffic = None
    if tr.get("bhcp_y_m6_bytes_per_launch") and Mtop == 6:  # scaled by the rows processed
        traffic = tr["bhcp_y_m6_bytes_per_launch"] * gt["rows_n_minus_2"] / tr["bhcp_y_m6_rows"]
    line["tuned_variants"] = {
        "bhcp_y": {str(m): b.variant(m) for m in groups},
        "what": "launch variant of the batched pair contraction per orbital count, picked by "
                "the autotuner on the running jobs (0 the default tile, 2 the other output-tile "
                "grouping, 3 the default tile handed over through mbarriers); variants change "
                "speed, never results"}
    line["roofline"] = {
        "bound": "tensor", "kernel": f"bhcp_y_kernel<{Mtop}> (pair contraction, FP64 mma.sync)",
        "achieved": gt["contraction_tflops"], "peak": mma_peak, "unit": "TFLOP/s",
        "frac": gt["contraction_tflops"] / mma_peak,
        "peak_source": "measured in this run: FP64 mma.sync probe (mctdhb_fp64_mma_probe)",
        "traffic": traffic, "algorithmic_flops_per_launch": gt["contraction_flops"],
        "ms_per_launch": gt["contraction_ms"],
        "gather_back": {"kernel": f"bhcp_g_kernel<{Mtop}>", "bound": "hbm",
                        "achieved": gt["gather_back_gbs"], "peak": peak, "unit": "GB/s",
                        "frac": gt["gather_back_gbs"] / peak, "peak_source": kind,
                        "ms_per_launch": gt["gather_back_ms"],
                        "algorithmic_bytes_per_launch": gt["gather_back_bytes"]},
        "groups": {str(m): g for m, g in groups.items()},
        "note": "H.C = pair contraction Y = A W^T over the (N-2)-boson space (8 FLOPs per "
                "complex multiply-add counted) + gather-back (each Y value read once, H.C "
                "written once); traffic: ncu DRAM bytes of the contraction on a 24-job case "
                "scaled by the rows processed"}
    # energies of a few jobs after warmup + steps, for the agreement check
    cmp_idx = {i: int(s1[slots[i]]) for i in range(0, len(jobs), 37)}
    e_batch = {i: float(energy[slots[i]]) for i in cmp_idx}
    b.close()

    plain, e_plain = plain_timed(mb, torch, jobs, 1, args.plain_steps, compare=cmp_idx)
    per_job = plain.pop("seconds_per_step_by_job")
    line["plain"] = plain
    line["vs_plain"] = (value / world) / plain["value"]
    # how close the batched step comes to the work of the largest jobs: those
    # fill the GPU alone, so one step of each, one at a time, bounds what
    # batching can save on them
    top = sorted(range(len(jobs)), key=lambda i: -step_bytes(jobs[i]))[:25]
    big_ms = 1000.0 * sum(per_job[i] for i in top)
    line["vs_plain_bound"] = {
        "largest_jobs": len(top),
        "share_of_mix_bytes": sum(step_bytes(jobs[i]) for i in top) /
        sum(step_bytes(j) for j in jobs),
        "largest_jobs_plain_ms": big_ms, "all_jobs_plain_ms": 1000.0 * sum(per_job),
        "batched_ms_per_step": t_ms / args.steps,
        "what": "one step of each of the largest jobs one at a time (plain solver) against "
                "one batched step of the whole mix: the batched step cannot drop below the "
                "large jobs' own GPU time by more than launch overhead"}
    line["energy_agreement"] = {
        "max_rel_diff": max(abs(e_batch[i] - e_plain[i]) / abs(e_plain[i]) for i in cmp_idx),
        "jobs": len(cmp_idx), "what": "energy after the same number of steps, batched vs plain"}

    for name in SINGLE:
        line[name] = run_single(mb, torch, name, max(3, args.steps // 2), args.warmup)
    line["e2e"] = e2e_batch(mb, torch, jobs, args.steps)
    if not args.no_serving:
        line["serving"] = run_serving(mb, torch, [float(r) for r in args.serve_rates.split(",")],
                                      args.serve_jobs, args.serve_imag_steps,
                                      args.serve_real_steps, args.serve_big_frac,
                                      args.serve_nmax)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(jobs)
    print(json.dumps(line), flush=True)


def run_profile():
    """a small single-GPU case for ncu: 24 jobs of the mix admitted, two
    batch steps outside the profiled range, then one step inside it
    (cudaProfilerStart/Stop; use --profile-from-start off)"""
    import torch

    import mctdhb_b200 as mb

    jobs = mix_jobs(n=24)
    b = mb.Batch(len(jobs), arena_bytes(mb, jobs), LZ)
    for j in jobs:
        b.admit(j)
    b.step(2)
    b.sync()
    torch.cuda.profiler.start()
    b.step(1)
    b.sync()
    torch.cuda.profiler.stop()
    b.close()
    print("profile run done")


def run_profile_kernels(size):
    """single-system kernels for ncu at size "N,M" (30,8: the quench; other
    sizes: grid 512 on [-10, 10], double well, g = 0.1): set-up and one
    untimed H.C, density and configurational step outside the profiled
    range, then one H.C, one density and one step (SIL + rho1 + rho2, one
    CUDA graph) inside it (cudaProfilerStart/Stop; use
    --profile-from-start off)"""
    import torch

    import mctdhb_b200 as mb

    N, M = (int(x) for x in size.split(","))
    c = dict(SINGLE["quench_n30_m8"])
    if (N, M) != (c["N"], c["M"]):
        c.update(N=N, M=M, G=512, xi=BXI, xf=BXF)
    hob, hint, c0 = single_inputs(mb, c)
    sp = mb.Space(c["N"], c["M"])
    d_c = torch.from_numpy(c0).cuda()
    sp.set_matrices(torch.from_numpy(hob.reshape(-1)).cuda(), torch.from_numpy(hint).cuda())
    r1 = torch.empty(c["M"] ** 2, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(c["M"] ** 4, dtype=torch.complex128, device="cuda")
    out = torch.empty_like(d_c)
    stream = torch.cuda.current_stream()
    step = mb.Step(sp, d_c, r1, r2, c["m"], c["dt"], False)
    sp.apply_hamiltonian(d_c, out)
    sp.density_matrices(d_c, r1, r2)
    step.launch(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    sp.apply_hamiltonian(d_c, out)
    sp.density_matrices(d_c, r1, r2)
    step.launch(stream)  # one configurational step (SIL + rho1 + rho2, one CUDA graph)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    step.close()
    sp.close()
    print("profile run done")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--ref-full-mix", action="store_true",
                    help="with --impl reference: one complete step of the whole mix by the "
                         "compiled reference, against its sampled estimates")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="timed steps per job on the plain one-at-a-time path")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-only", action="store_true",
                    help="only the serving block (its own JSON line)")
    # the served workload as configured (sizes as the batched mix plus 5% N=30
    # M=8 jobs, relaxations to 1e-10 or 5000 steps, 500-step quenches); the
    # job count per rate is the one cap, so the block ends in minutes
    ap.add_argument("--serve-rates", default="500", help="arrival rates swept, jobs/s")
    ap.add_argument("--serve-jobs", type=int, default=16, help="jobs served per rate")
    ap.add_argument("--serve-imag-steps", type=int, default=5000)
    ap.add_argument("--serve-real-steps", type=int, default=500)
    ap.add_argument("--serve-big-frac", type=float, default=0.05)
    ap.add_argument("--serve-nmax", type=int, default=60)
    ap.add_argument("--mix-convergence", action="store_true",
                    help="the whole mix relaxed to its stop rule, batched and one at a time "
                         "(its own JSON line; tens of minutes)")
    ap.add_argument("--profile", action="store_true",
                    help="one profiled batch step of a small mix (for ncu captures)")
    ap.add_argument("--profile-kernels", metavar="N,M", nargs="?", const="30,8",
                    help="one profiled H.C and density launch of one system (for ncu captures)")
    args = ap.parse_args()
    if args.serving_only:
        import torch

        import mctdhb_b200 as mb

        torch.cuda.set_device(0)
        print(json.dumps({"serving": run_serving(
            mb, torch, [float(r) for r in args.serve_rates.split(",")], args.serve_jobs,
            args.serve_imag_steps, args.serve_real_steps, args.serve_big_frac,
            args.serve_nmax)}), flush=True)
    elif args.mix_convergence:
        import torch

        import mctdhb_b200 as mb

        torch.cuda.set_device(0)
        print(json.dumps({"mix_convergence": run_mix_convergence(mb, torch)}), flush=True)
    elif args.profile:
        run_profile()
    elif args.profile_kernels:
        run_profile_kernels(args.profile_kernels)
    elif args.impl == "reference" and args.ref_full_mix:
        run_reference_full_mix(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
