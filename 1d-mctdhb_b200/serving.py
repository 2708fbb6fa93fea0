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

The engine is injectable (`engine=`): anything with the `Batch` methods
used here (admit, step, poll, fetch, monitor, lowest_state, release,
free_bytes, close, and the static job_bytes) serves, which is how the
scheduling policy is tested without a GPU.
"""
import time
from dataclasses import dataclass, field

import numpy as np

# poll states of the engine
EMPTY, RUNNING, DONE, ABORTED = 0, 1, 2, 3


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
                 final_diag=False, engine=None, clock=time.perf_counter):
        if engine is None:
            import mctdhb_b200 as mb

            engine = mb.Batch(max_slots, arena_bytes, lanczos_iter)
        self.b = engine
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

    # -- arrival ------------------------------------------------------------
    def submit(self, job, at=None):
        """queue a job (dict of mctdhb_job fields and its arrays); `at`:
        arrival time in seconds on the server clock (default: now).
        Returns the job id."""
        nbytes = int(type(self.b).job_bytes(job, self.lz))
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
            self.waiting.append(self.arriving.pop(0))

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
        if not self.running:
            return []
        self.b.step(self.steps_per_tick)
        _, state, _, _ = self.b.poll()
        t = self.now()
        return [self._retire(s, state[s], t) for s in list(self.running)
                if state[s] in (DONE, ABORTED)]

    def busy(self):
        return bool(self.arriving or self.waiting or self.running)

    def run(self, sleep=0.002):
        """serve until every submitted job has retired; idle gaps before the
        next arrival are slept through"""
        while self.busy():
            if not self.running and not self.waiting and self.arriving:
                time.sleep(max(0.0, min(sleep, self.arriving[0].arrival - self.now())))
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
