"""Benchmark of one MCTDHB time step on B200.

Workload (default): the N=30 bosons, M=8 orbitals real-time quench
(nc = 10,295,472 complex128 coefficients, 165 MB per vector), grid of 1024
points on [-15, 15], trap V = x^2/2 + 4 exp(-x^2/0.5), g = 0.1, Lanczos
dimension 6, dt = 0.005.  One step = the configurational part of the
reference's mctdhb_propagate_step (driver.c:186-200): short-iterative-Lanczos
propagation of the coefficients (6 H.C actions, full reorthogonalisation,
tridiagonal exponential, recombination) followed by rho1 and rho2 of the new
coefficients, with h_kl and g_ksql of Hermite-Gaussian orbitals.  The full
step including the Runge-Kutta orbital update is timed too ("full_step"):
at this grid and dt the explicit RK5 orbital step is unstable in the
reference's own method (it diverges within ~5 steps), so only its cost, over
its first steps, is reported.  Inputs are seeded synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  Multi-GPU: one process per GPU (torchrun),
each rank advances its own independent system (replicas: a single system
does not shard; no collective in the data path); value = steps/s summed over
ranks, timed as the max over ranks.
"""
import argparse
import ctypes as C
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

N_PAR, N_ORB, LANCZOS_M, DT = 30, 8, 6, 0.005
GRID, XI, XF, G_INT = 1024, -15.0, 15.0, 0.1
HBM_FALLBACK = 6650.0
METRIC = "mctdhb_steps_per_s"


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


def grid():
    return np.linspace(XI, XF, GRID)


def double_well(x):
    return 0.5 * x ** 2 + 4.0 * np.exp(-x ** 2 / 0.5)


def hermite_orbitals(M=N_ORB):
    """Hermite-Gaussian orbitals n = 0..M-1, Gram-Schmidt in the Simpson
    metric, periodic end point equal to the first"""
    x = grid()
    w = simpson_weights(GRID, x[1] - x[0])
    phi = np.zeros((M, GRID), np.complex128)
    hm, hc = np.zeros(GRID), np.exp(-x ** 2 / 2)
    for n in range(M):
        phi[n] = hc
        hm, hc = hc, (np.sqrt(2.0) * x * hc - np.sqrt(n) * hm) / np.sqrt(n + 1)
    for i in range(M):
        for j in range(i):
            phi[i] -= np.sum(w * phi[j].conj() * phi[i]) * phi[j]
        phi[i] /= np.sqrt(np.sum(w * np.abs(phi[i]) ** 2))
    return phi


def orbital_matrices(phi, g=G_INT):
    """h_kl (4th-order periodic derivative, Simpson) and g_ksql of `phi`
    (inputs of the stand-alone kernel timings; the solver computes its own)"""
    x = grid()
    dx = x[1] - x[0]
    w = simpson_weights(GRID, dx)
    d = (np.roll(phi, 2, 1) - np.roll(phi, -2, 1) +
         8 * (np.roll(phi, -1, 1) - np.roll(phi, 1, 1))) / (12 * dx)
    hob = 0.5 * np.einsum("x,ax,bx->ab", w, d.conj(), d) + \
        np.einsum("x,ax,bx->ab", w * double_well(x), phi.conj(), phi)
    t = g * np.einsum("x,ax,bx,cx,dx->abcd", w, phi.conj(), phi.conj(), phi, phi)
    return np.ascontiguousarray(hob), np.ascontiguousarray(t.transpose(3, 2, 1, 0)).reshape(-1)


def coefficients(nc, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=nc) + 1j * rng.normal(size=nc)
    return c / np.linalg.norm(c)


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
    """per-launch DRAM bytes of the H.C kernel from the committed ncu summary"""
    try:
        with open(os.path.join(REPO, "profiles", "hc_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def workload_config(args):
    return {"workload": "real-time quench N=30 M=8 (nc=10295472), grid 1024 on [-15,15], "
                        "V=x^2/2+4exp(-x^2/0.5), g=0.1, Lanczos 6, dt=0.005, RK5 orbitals",
            "npar": N_PAR, "norb": N_ORB, "grid": GRID, "lanczos_iter": LANCZOS_M, "dt": DT,
            "step": "SIL(6 H.C) + rho1 + rho2 (one CUDA graph)",
            "parallelism": f"replicas{args.gpus}",
            "l2": "inputs larger than L2 (165 MB coefficient vector, 1 GB of Krylov vectors)"}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle's C restatement on a bounded row sample
# ---------------------------------------------------------------------------
def cpu_step_estimate(hob, hint, rows_per_sample=200000, samples=8, m=LANCZOS_M):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle import Oracle

    O = Oracle()
    nc = O.dim(N_PAR, N_ORB)
    c = coefficients(nc, 7)
    offs = [int(nc * f) for f in np.linspace(0.0, 0.9, samples)]
    t_hc = t_dn = 0.0
    for r0 in offs:
        t0 = time.perf_counter()
        O.apply_hamiltonian(N_PAR, N_ORB, c, hob, hint, rows=(r0, r0 + rows_per_sample))
        t1 = time.perf_counter()
        O.twobody_dm(N_PAR, N_ORB, c, rows=(r0, r0 + rows_per_sample))
        t2 = time.perf_counter()
        t_hc += t1 - t0
        t_dn += t2 - t1
    rows = rows_per_sample * samples
    step_s = (m * t_hc / rows + t_dn / rows) * nc
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{samples}x{rows_per_sample} rows of H.C and rho2 (oracle C restatement, "
                      f"OpenMP, {os.cpu_count()} threads) scaled to {m} H.C + rho2 over "
                      f"{nc} rows (the orbital part, <1% of a step, is not counted); the "
                      f"reference itself cannot build its maps at this size",
            "seconds_per_step": step_s, "sample_seconds": t_hc + t_dn}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    hob, hint = orbital_matrices(hermite_orbitals())
    for _ in range(args.warmup):
        cpu_step_estimate(hob, hint, rows_per_sample=5000, samples=2)
    vals = [cpu_step_estimate(hob, hint, rows_per_sample=50000, samples=8)
            for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    base = dict(vals[0], value=v)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": workload_config(args), "cpu_baseline": base,
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
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

    phi = hermite_orbitals()
    pot = double_well(grid())
    hob, hint = orbital_matrices(phi)
    c0 = coefficients(int(mb.load().space_dimension(N_PAR, N_ORB)), 1234 + rank)

    def barrier():
        if dist is not None:
            dist.barrier()

    stream = torch.cuda.current_stream()
    # informational: the full mctdhb_propagate_step (orbital RK5 + h, g + SIL +
    # densities) over its first steps.  At this grid and dt the explicit RK5
    # orbital step is outside its stability region (dt * max eigenvalue of the
    # finite-difference kinetic operator ~ 11) and diverges after ~5 steps in
    # the reference's own method as well; its cost is timed, not its values.
    s = mb.Solver(N_PAR, N_ORB, GRID, XI, XF, DT, False, 5, LANCZOS_M)
    s.set_potential(pot)
    s.set_interaction(G_INT)
    s.set_state(phi, c0)
    s.step(1, stream)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    s.step(2, stream)
    f1.record(stream)
    torch.cuda.synchronize()
    full_step_ms = f0.elapsed_time(f1) / 2
    full_step_kernels = s.kernels
    s.close()

    # the measured step: SIL(6) + rho1, rho2 of the coefficients, one CUDA graph
    sp = mb.Space(N_PAR, N_ORB)
    nc = sp.dim
    d_c = torch.from_numpy(c0).cuda()
    sp.set_matrices(torch.from_numpy(hob.reshape(-1)).cuda(), torch.from_numpy(hint).cuda())
    r1 = torch.empty(N_ORB * N_ORB, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(N_ORB ** 4, dtype=torch.complex128, device="cuda")
    step = mb.Step(sp, d_c, r1, r2, LANCZOS_M, DT, False)
    for _ in range(args.warmup):
        step.launch(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.profiler.start()  # ncu --profile-from-start off sees the timed steps only
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step.launch(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([t_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    value = world * args.steps / (t_ms / 1000.0)
    norm = float(torch.linalg.vector_norm(d_c).item())
    assert abs(norm - 1.0) < 1e-10, f"real-time SIL must conserve the norm, got {norm}"
    kernels_per_step = step.kernels
    step.close()

    # H.C and density kernels alone on the same data (CUDA events on the
    # launching stream) for the roofline
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
    G = distinct_couplings(N_PAR, N_ORB)
    b_hc = 32.0 * nc + 16.0 * G
    b_dn = 16.0 * nc + 16.0 * G
    peak, peak_kind = peaks()
    traffic = ncu_traffic()
    del sp, d_c, hc_out

    e2e = run_e2e(args, mb, hob, hint, c0, stream)
    if dist is not None:
        t = torch.tensor([args.steps / e2e["value"]], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e["value"] = world * args.steps / float(t.item())

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": workload_config(args),
        "roofline": {
            "bound": "hbm", "kernel": "hc_kernel<8>",
            "achieved": b_hc / t_hc / 1e9, "peak": peak, "unit": "GB/s",
            "frac": b_hc / t_hc / 1e9 / peak, "peak_source": peak_kind,
            "traffic": (traffic or {}).get("hc_bytes_per_launch"),
            "algorithmic_bytes_per_launch": b_hc, "ms_per_launch": t_hc * 1e3,
            "density_ms_per_launch": t_dn * 1e3, "density_achieved_gbs": b_dn / t_dn / 1e9,
        },
        "clocks": clk,
        "gpu_launches": kernels_per_step * args.steps,
        "e2e": e2e,
        "full_step": {"ms_per_step": full_step_ms, "kernels_per_step": full_step_kernels,
                      "what": "mctdhb_propagate_step incl. RK5 orbitals, first steps only"},
    }
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_step_estimate(hob, hint)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_e2e(args, mb, hob, hint, c0, stream):
    """K steps through the reference's own calls, propagate_coef_sil
    (coefficients_integration.c:59) then sync_density_matrices
    (synchronize.c:42), on a reference-layout MCTDHBDataStruct whose buffers
    are pinned host memory: every step uploads its inputs and copies its
    results back (host<->device copies inside the timed region)."""
    import torch

    import mctdhb_types as T

    L = mb.load()
    M = N_ORB
    nc = len(c0)
    pin = lambda n: torch.empty(n, dtype=torch.complex128, pin_memory=True).numpy()
    keep = []

    def rows(a2):
        a = pin(a2.size).reshape(a2.shape)
        a[:] = a2
        ptrs = (T.Carray * a.shape[0])(*[T.carray(a[i]) for i in range(a.shape[0])])
        keep.append((a, ptrs))
        return C.cast(ptrs, T.Cmatrix)

    coef, cnext, hintv, rho2 = pin(nc), pin(nc), pin(M ** 4), pin(M ** 4)
    coef[:] = c0
    hintv[:] = hint
    mc = T.MultiConfigurationS()
    mc.npar, mc.norb, mc.dim = N_PAR, M, nc  # the GPU path ranks on the fly: no tables
    stt = T.ManyBodyStateS()
    stt.npar, stt.norb, stt.space_dim = N_PAR, M, nc
    stt.coef, stt.hint, stt.tb_denmat = T.carray(coef), T.carray(hintv), T.carray(rho2)
    stt.hob = rows(hob)
    stt.ob_denmat = rows(np.zeros((M, M), np.complex128))
    stt.inv_ob_denmat = rows(np.zeros((M, M), np.complex128))
    eq = T.OrbitalEquationS()
    eq.tstep, eq.prop_dt, eq.time_fac = DT, T.dcomplex.of(DT), T.dcomplex.of(1.0)
    lw = T.WorkspaceLanczosS()
    lw.iter, lw.space_dim = LANCZOS_M, nc
    dd, od = np.zeros(LANCZOS_M, np.complex128), np.zeros(LANCZOS_M, np.complex128)
    lw.decomp_diag, lw.decomp_offd = T.carray(dd), T.carray(od)
    cw = T.CoefWorkspaceS()
    cw.lan_work = C.pointer(lw)
    ms = T.MCTDHBDataStructS()
    ms.integ_type, ms.coef_integ_method = T.REALTIME, T.LANCZOS
    ms.multiconfig_space, ms.orb_eq = C.pointer(mc), C.pointer(eq)
    ms.coef_workspace, ms.state = C.pointer(cw), C.pointer(stt)
    pms, pmc, pst = C.pointer(ms), C.pointer(mc), C.pointer(stt)

    def one():
        L.propagate_coef_sil(pms, T.carray(cnext))
        L.sync_density_matrices(pmc, pst)

    L.mctdhb_gpu_clear_error()
    for _ in range(max(1, args.warmup)):
        one()
    if mb.last_error():
        raise mb.MctdhbError(mb.last_error())
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        one()
    b.record(stream)
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1000.0
    return {"value": args.steps / t, "unit": "steps/s",
            "h2d_bytes_per_step": 2 * nc * 16 + (M * M + M ** 4) * 16,
            "d2h_bytes_per_step": nc * 16 + (2 * M * M + M ** 4) * 16,
            "path": "propagate_coef_sil + sync_density_matrices on pinned host buffers"}


def run_profile():
    """H.C three times then the density kernel once at N=30, M=8: a small,
    single-GPU case for `ncu -k regex:<kernel> -s <n> -c 1`."""
    import torch

    import mctdhb_b200 as mb

    hob, hint = orbital_matrices(hermite_orbitals())
    sp = mb.Space(N_PAR, N_ORB)
    d_c = torch.from_numpy(coefficients(sp.dim, 1234)).cuda()
    out = torch.empty_like(d_c)
    r1 = torch.empty(N_ORB * N_ORB, dtype=torch.complex128, device="cuda")
    r2 = torch.empty(N_ORB ** 4, dtype=torch.complex128, device="cuda")
    sp.set_matrices(torch.from_numpy(hob.reshape(-1)).cuda(), torch.from_numpy(hint).cuda())
    for _ in range(2):  # autotuning happens here, outside the profiled range
        sp.apply_hamiltonian(d_c, out)
        sp.density_matrices(d_c, r1, r2)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()  # ncu --profile-from-start off: one launch of each
    sp.apply_hamiltonian(d_c, out)
    sp.density_matrices(d_c, r1, r2)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print("profile run done", float(torch.linalg.vector_norm(out).item()))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="only launch the H.C and density kernels (for ncu captures)")
    args = ap.parse_args()
    if args.profile:
        run_profile()
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
