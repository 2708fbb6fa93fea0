"""Continuous batching of MCTDHB jobs on one GPU: the request loop over the
batched engine (`mctdhb_b200.Batch`, include/mctdhb_gpu.h part 3).

The reference integrates the jobs of its parameter file one after another,
each to its end (apps/mctdhb_main.c:172-200, one `integration_driver` call
per job line).  `Server` keeps the same per-job semantics -- each job is one
such integration, stopped by its step limit, the imaginary-time energy rule
(with the eigen residual when the job sets eig_tol), or the real-time
overlap abort -- and serves a stream of them:

* arrival: `submit` queues a job with its arrival time on the server clock;
  a job whose footprint exceeds the whole arena is refused at once;
* admission: first come, first served, as soon as a slot and an arena range
  of the job's exact footprint (`Batch.job_bytes`) are free; a job that does
  not fit waits at the head of the queue (back-pressure) while the running
  jobs advance, and no later job overtakes it;
* progress: every running job advances together, `steps_per_tick` batch
  steps (one CUDA graph launch each) per tick;
* retirement: a stopped job's results are fetched (orbitals, coefficients,
  rho1, rho2, energy, steps, stop reason, monitor), the final lowest-state
  diagonalisation of driver.c:295-316 runs for relaxations that ended at
  their step limit when `final_diag` is set, and its slot and arena range
  are released for the jobs waiting.

Latency = retirement time - arrival time; `stats` gives p50 / p99 and
jobs/s over the retired jobs.

Heavy lane (`heavy_nc`): a job whose Fock space has at least heavy_nc
configurations fills the GPU on its own (N=30, M=8: one H.C is 148 blocks
of tensor-core work); batching it with small jobs only makes every small
job wait for its steps.  Such jobs go, first come first served, to a lane
of their own: one at a time through the plain solver (`SolverLane`,
mctdhb_solver_relax: the same step limit and energy rule, evaluated on the
device) on a stream of its own.  The lane advances in chunks of
`heavy_chunk` steps, and only while the batch has no job running (light
jobs first: a small job is never queued behind a heavy job's long kernels,
whose persistent blocks fill every SM), unless the heavy job has waited
`heavy_max_wait` seconds since its last chunk.

The engine and the lane are injectable (`engine=`, `lane=`): anything with
the `Batch` methods used here (admit, step, poll, fetch, monitor,
lowest_state, release, free_bytes, close, and the static job_bytes), or
with the `SolverLane` methods (busy, start, poll, close), serves, which is
how the scheduling policy is tested without a GPU.
"""
import time
from dataclasses import dataclass, field

import numpy as np

# poll states of the engine
EMPTY, RUNNING, DONE, ABORTED = 0, 1, 2, 3


def fock_dim(N, M):
    from math import comb

    return comb(N + M - 1, M - 1)


class SolverLane:
    """one job at a time through the plain single-system solver on its own
    CUDA stream, in chunks: each `advance(k)` launches mctdhb_solver_relax
    for up to k more steps (the step limit and, in imaginary time, the
    energy rule on the device; a chunk boundary changes nothing when k is a
    multiple of check_every, since the rule's reference energy is the
    current state's either way); `poll` hands a finished chunk back without
    blocking before"""

    def __init__(self, lanczos_iter=5):
        import torch

        self.lz = lanczos_iter
        # the lowest priority: the batch's stream has the highest
        self.stream = torch.cuda.Stream(priority=0)
        self.s = None
        self.job = None
        self.steps = 0
        self.launched = False

    def busy(self):
        return self.s is not None

    def start(self, job):
        import mctdhb_b200 as mb

        j = job
        s = mb.Solver(j["npar"], j["norb"], j["grid_size"], j["xi"], j["xf"], j["dt"],
                      bool(j["imagtime"]), j["rk_order"], self.lz, d2coef=j.get("d2coef", -0.5),
                      d1coef=complex(j.get("d1coef", 0j)), periodic=bool(j.get("periodic", 1)))
        try:
            der = j.get("der_method", 302)
            if der not in (0, 302):
                s.set_derivative(der)
            if j.get("impr_ortho"):
                s.set_orthogonality(True)
            if j.get("orb_method", 0) == 31:
                s.set_orb_method(31)
            s.set_potential(j["pot"])
            s.set_interaction(j["g"])
            s.set_state(j["orbitals"], j["coef"])
        except Exception:
            s.close()
            raise
        self.s, self.job, self.steps, self.launched = s, job, 0, False

    def idle(self):
        """running a job, with no chunk in flight"""
        return self.s is not None and not self.launched

    def advance(self, k):
        j = self.job
        check = j.get("check_every", 0) if j["imagtime"] else 0
        if check > 1:
            k = max(check, k // check * check)
        k = min(k, j["max_steps"] - self.steps)
        self.s.relax(k, j.get("energy_tol", 0.0), check, self.stream)
        self.launched = True

    def poll(self):
        """the job's results (the Batch.fetch fields) once it has stopped,
        else None (a finished chunk of an unfinished job leaves it idle)"""
        if self.s is None or not self.launched or not self.s.done():
            return None
        s = self.s
        n, conv = s.relax_result()
        self.steps += n
        self.launched = False
        if not conv and self.steps < self.job["max_steps"]:
            return None
        try:
            d = s.get()
            out = {k: d[k] for k in ("orb", "coef", "rho1", "rho2")}
            out.update(energy=s.energy().real, steps=self.steps, converged=conv, state=DONE,
                       monitor={}, lane="solver")
        finally:
            s.close()
            self.s = self.job = None
        return out

    def close(self):
        if self.s is not None:
            self.s.close()
            self.s = None


@dataclass
class Request:
    jid: int
    job: dict
    arrival: float
    nbytes: int
    admitted: float = None
    finished: float = None
    slot: int = None
    result: dict = field(default=None)


class Server:
    def __init__(self, arena_bytes, max_slots=256, lanczos_iter=5, steps_per_tick=2,
                 final_diag=False, heavy_nc=None, heavy_chunk=20, heavy_max_wait=None,
                 engine=None, lane=None, clock=time.perf_counter):
        if engine is None:
            import mctdhb_b200 as mb

            engine = mb.Batch(max_slots, arena_bytes, lanczos_iter)
        self.b = engine
        self.heavy_nc = heavy_nc
        self.lane = lane if lane is not None or heavy_nc is None else SolverLane(lanczos_iter)
        self.heavy = []      # arrived heavy jobs waiting for the lane (FCFS)
        self.in_lane = None
        self.heavy_chunk = int(heavy_chunk)
        self.heavy_max_wait = heavy_max_wait
        self.lane_last = None  # time of the lane's last chunk launch
        self.arena_bytes = int(arena_bytes)
        self.lz = lanczos_iter
        self.steps_per_tick = int(steps_per_tick)
        self.final_diag = final_diag
        self.clock = clock
        self.t0 = clock()
        self.reqs = []       # every request, by job id
        self.arriving = []   # submitted, arrival time not reached (sorted)
        self.waiting = []    # arrived, not admitted (FCFS order)
        self.running = {}    # slot -> request
        self.peak_running = 0

    def now(self):
        return self.clock() - self.t0

    def close(self):
        if self.b is not None:
            self.b.close()
            self.b = None
        if self.lane is not None:
            self.lane.close()
            self.lane = None

    def is_heavy(self, job):
        return self.heavy_nc is not None and fock_dim(job["npar"], job["norb"]) >= self.heavy_nc

    # -- arrival ------------------------------------------------------------
    def submit(self, job, at=None):
        """queue a job (dict of mctdhb_job fields and its arrays); `at`:
        arrival time in seconds on the server clock (default: now).
        Returns the job id."""
        nbytes = 0 if self.is_heavy(job) else int(type(self.b).job_bytes(job, self.lz))
        if nbytes > self.arena_bytes:
            raise ValueError(f"job needs {nbytes} bytes, the arena holds {self.arena_bytes}")
        r = Request(len(self.reqs), job, self.now() if at is None else float(at), nbytes)
        self.reqs.append(r)
        i = len(self.arriving)
        while i > 0 and self.arriving[i - 1].arrival > r.arrival:
            i -= 1
        self.arriving.insert(i, r)
        return r.jid

    # -- one tick of the loop ------------------------------------------------
    def _arrive(self, t):
        while self.arriving and self.arriving[0].arrival <= t:
            r = self.arriving.pop(0)
            (self.heavy if self.is_heavy(r.job) else self.waiting).append(r)

    def _lane(self, t):
        """retire the lane's finished job, start the next heavy one, launch
        its next chunk when the batch is idle (or the heavy job has waited
        heavy_max_wait seconds)"""
        done = []
        if self.in_lane is not None:
            d = self.lane.poll()
            if d is not None:
                r = self.in_lane
                r.finished, r.result = self.now(), d
                self.in_lane = None
                done.append(r.jid)
        if self.in_lane is None and self.heavy:
            r = self.heavy.pop(0)
            r.admitted = t
            self.lane.start(r.job)
            self.in_lane = r
            self.lane_last = t
        if self.in_lane is not None and self.lane.idle():
            starved = (self.heavy_max_wait is not None and
                       t - self.lane_last >= self.heavy_max_wait)
            if not self.running or starved:
                self.lane.advance(self.heavy_chunk)
                self.lane_last = t
        return done

    def _admit(self, t):
        while self.waiting:
            r = self.waiting[0]
            s = self.b.admit(r.job)
            if s is None:
                break  # back-pressure: the head waits for room, nothing overtakes it
            self.waiting.pop(0)
            r.slot, r.admitted = s, t
            self.running[s] = r
        self.peak_running = max(self.peak_running, len(self.running))

    def _retire(self, slot, state, t):
        r = self.running.pop(slot)
        d = self.b.fetch(slot)
        d["state"] = int(state)
        d["monitor"] = self.b.monitor(slot)
        if (self.final_diag and r.job.get("imagtime") and state == DONE and
                not d["converged"]):
            d["energy_lowest_state"] = self.b.lowest_state(slot, 0)
            d["coef"] = self.b.fetch(slot)["coef"]
        self.b.release(slot)
        r.finished, r.result = t, d
        return r.jid

    def tick(self):
        """admit what has arrived and fits, advance the running jobs, retire
        the stopped ones; returns the ids retired"""
        t = self.now()
        self._arrive(t)
        self._admit(t)
        done = self._lane(t) if self.lane is not None else []
        if not self.running:
            return done
        self.b.step(self.steps_per_tick)
        _, state, _, _ = self.b.poll()
        t = self.now()
        return done + [self._retire(s, state[s], t) for s in list(self.running)
                       if state[s] in (DONE, ABORTED)]

    def busy(self):
        return bool(self.arriving or self.waiting or self.running or self.heavy or
                    self.in_lane is not None)

    def run(self, sleep=0.002):
        """serve until every submitted job has retired; idle gaps before the
        next arrival, or while only the lane runs, are slept through"""
        while self.busy():
            if not self.running and not self.waiting and not self.heavy:
                nxt = self.arriving[0].arrival - self.now() if self.arriving else sleep
                time.sleep(max(0.0, min(sleep, nxt)))
            self.tick()

    # -- results --------------------------------------------------------------
    def result(self, jid):
        return self.reqs[jid].result

    def latency(self, jid):
        r = self.reqs[jid]
        return None if r.finished is None else r.finished - r.arrival

    def stats(self):
        done = [r for r in self.reqs if r.finished is not None]
        if not done:
            return {"jobs": 0}
        lat = np.array([r.finished - r.arrival for r in done])
        span = max(r.finished for r in done) - min(r.arrival for r in done)
        return {"jobs": len(done), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "max_s": float(lat.max()), "jobs_per_s": len(done) / span if span > 0 else None,
                "makespan_s": span, "peak_running": self.peak_running,
                "aborted": sum(1 for r in done if r.result["state"] == ABORTED)}
