"""The request loop of 1d-mctdhb_b200/serving.py on a fake engine (CPU):
first-come-first-served admission by footprint, back-pressure without
overtaking, arrival times, retirement and the final diagonalisation hook."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "1d-mctdhb_b200"))

from serving import ABORTED, DONE, RUNNING, Server  # noqa: E402


class FakeBatch:
    """the Batch methods the server uses; a job runs job['max_steps'] steps
    (or stops early at job['stop_at']), occupies job['bytes'] of a
    contiguous-free-bytes arena and reports energy = its id"""

    def __init__(self, slots, arena):
        self.slots = [None] * slots
        self.free = arena
        self.log = []
        self.diag = []

    @staticmethod
    def job_bytes(job, lz):
        return job["bytes"]

    def admit(self, job):
        if job["bytes"] > self.free or None not in self.slots:
            return None
        s = self.slots.index(None)
        self.slots[s] = {"job": job, "steps": 0, "state": RUNNING}
        self.free -= job["bytes"]
        self.log.append(("admit", job["name"]))
        return s

    def step(self, n):
        for x in self.slots:
            if x is None or x["state"] != RUNNING:
                continue
            for _ in range(n):
                x["steps"] += 1
                j = x["job"]
                if x["steps"] == j.get("stop_at"):
                    x["state"] = j.get("stop_state", DONE)
                    break
                if x["steps"] >= j["max_steps"]:
                    x["state"] = DONE
                    break

    def poll(self):
        st = [0 if x is None else x["state"] for x in self.slots]
        return sum(1 for s in st if s == RUNNING), st, None, None

    def fetch(self, s):
        x = self.slots[s]
        return {"energy": x["job"]["name"], "steps": x["steps"],
                "converged": x["steps"] == x["job"].get("stop_at"), "coef": [x["steps"]]}

    def monitor(self, s):
        return {}

    def lowest_state(self, s, niter):
        self.diag.append(self.slots[s]["job"]["name"])
        return -1.0

    def release(self, s):
        self.free += self.slots[s]["job"]["bytes"]
        self.log.append(("release", self.slots[s]["job"]["name"]))
        self.slots[s] = None

    def close(self):
        pass


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def server(slots=8, arena=100, **kw):
    clock = Clock()
    fb = FakeBatch(slots, arena)
    return Server(arena, engine=fb, clock=clock, steps_per_tick=1, **kw), fb, clock


def job(name, nbytes, steps, **kw):
    return dict(name=name, bytes=nbytes, max_steps=steps, imagtime=1, **kw)


def test_full_arena_back_pressures_and_release_makes_room():
    srv, fb, clock = server(arena=100)
    for i in range(4):
        srv.submit(job(i, 40, 3 + i), at=0.0)
    srv.tick()
    assert len(srv.running) == 2 and len(srv.waiting) == 2  # 80 of 100 bytes
    while srv.busy():
        clock.t += 0.1
        srv.tick()
        assert len(srv.running) <= 2
    admits = [n for a, n in fb.log if a == "admit"]
    assert admits == [0, 1, 2, 3]  # first come, first served
    # job 2 is admitted only after a release
    assert fb.log.index(("admit", 2)) > fb.log.index(("release", 0))
    for i in range(4):
        r = srv.result(i)
        assert r["steps"] == 3 + i and r["energy"] == i and r["state"] == DONE
    assert srv.stats()["jobs"] == 4 and srv.peak_running == 2


def test_head_of_queue_is_not_overtaken():
    srv, fb, clock = server(arena=100)
    srv.submit(job("a", 60, 5), at=0.0)
    srv.submit(job("big", 70, 2), at=0.0)   # does not fit beside a
    srv.submit(job("small", 10, 2), at=0.0)  # would fit, must wait behind big
    srv.tick()
    assert [r.job["name"] for r in srv.running.values()] == ["a"]
    while srv.busy():
        clock.t += 0.1
        srv.tick()
    admits = [n for a, n in fb.log if a == "admit"]
    assert admits == ["a", "big", "small"]


def test_arrival_times_are_honoured():
    srv, fb, clock = server()
    srv.submit(job("late", 10, 2), at=5.0)
    srv.submit(job("early", 10, 2), at=1.0)
    clock.t = 0.5
    assert srv.tick() == [] and not srv.running
    clock.t = 1.0
    srv.tick()
    assert [r.job["name"] for r in srv.running.values()] == ["early"]
    while srv.busy():
        clock.t += 0.5
        srv.tick()
    assert srv.reqs[0].admitted >= 5.0
    lat = srv.latency(1)
    assert lat is not None and lat > 0


def test_oversized_job_is_refused_at_submission():
    srv, _, _ = server(arena=100)
    with pytest.raises(ValueError):
        srv.submit(job("huge", 101, 1))


def test_final_diagonalisation_only_for_unconverged_relaxations():
    srv, fb, clock = server(final_diag=True)
    srv.submit(job("limit", 10, 3))                    # step limit, not converged
    srv.submit(job("conv", 10, 9, stop_at=2))          # energy rule
    srv.submit(dict(job("quench", 10, 3), imagtime=0))  # real time
    srv.submit(job("abort", 10, 9, stop_at=1, stop_state=ABORTED))
    while srv.busy():
        clock.t += 0.1
        srv.tick()
    assert fb.diag == ["limit"]
    assert srv.result(0)["energy_lowest_state"] == -1.0
    assert srv.result(3)["state"] == ABORTED and srv.stats()["aborted"] == 1


class FakeLane:
    """the SolverLane methods: a job needs job['lane_steps'] steps, a chunk
    of k steps is done at the next poll"""

    def __init__(self):
        self.cur = None
        self.started = []
        self.chunks = []

    def busy(self):
        return self.cur is not None

    def idle(self):
        return self.cur is not None and not self.cur["launched"]

    def start(self, job):
        self.cur = {"job": job, "steps": 0, "launched": 0}
        self.started.append(job["name"])

    def advance(self, k):
        self.cur["launched"] = min(k, self.cur["job"]["lane_steps"] - self.cur["steps"])
        self.chunks.append(self.cur["job"]["name"])

    def poll(self):
        if self.cur is None or not self.cur["launched"]:
            return None
        self.cur["steps"] += self.cur["launched"]
        self.cur["launched"] = 0
        if self.cur["steps"] < self.cur["job"]["lane_steps"]:
            return None
        job = self.cur["job"]
        self.cur = None
        return {"energy": job["name"], "steps": job["lane_steps"], "converged": False,
                "state": DONE, "monitor": {}, "lane": "solver"}

    def close(self):
        pass


def test_heavy_jobs_take_their_own_lane_light_jobs_first():
    """jobs of at least heavy_nc configurations run one at a time in the
    solver lane, FCFS among themselves; the lane advances only while the
    batch has no job running (light jobs first); a heavy job needs no arena
    room"""
    clock = Clock()
    fb = FakeBatch(8, 30)
    lane = FakeLane()
    srv = Server(30, engine=fb, lane=lane, heavy_nc=1000, heavy_chunk=4, clock=clock,
                 steps_per_tick=1)
    heavy = lambda name, n: dict(job(name, 10 ** 9, n), npar=30, norb=8, lane_steps=n)
    srv.submit(heavy("H1", 10), at=0.0)
    srv.submit(job("a", 20, 3, npar=4, norb=3), at=0.0)
    srv.submit(heavy("H2", 4), at=0.0)
    srv.submit(job("b", 20, 2, npar=4, norb=3), at=0.0)  # waits for a's arena room
    srv.tick()
    assert lane.started == ["H1"] and lane.chunks == []  # light jobs running: lane waits
    assert [r.job["name"] for r in srv.running.values()] == ["a"]
    order = []
    while srv.busy():
        clock.t += 0.1
        order += [srv.reqs[i].job["name"] for i in srv.tick()]
    assert order == ["a", "b", "H1", "H2"]
    assert lane.started == ["H1", "H2"] and lane.chunks == ["H1"] * 3 + ["H2"]
    assert srv.result(0)["lane"] == "solver" and srv.result(0)["steps"] == 10
    assert srv.stats()["jobs"] == 4


def test_starved_heavy_job_gets_chunks_beside_the_batch():
    clock = Clock()
    fb = FakeBatch(8, 30)
    lane = FakeLane()
    srv = Server(30, engine=fb, lane=lane, heavy_nc=1000, heavy_chunk=1, heavy_max_wait=0.25,
                 clock=clock, steps_per_tick=1)
    srv.submit(dict(job("H", 10 ** 9, 3), npar=30, norb=8, lane_steps=3), at=0.0)
    srv.submit(job("long", 20, 40, npar=4, norb=3), at=0.0)
    order = []
    while srv.busy():
        clock.t += 0.1
        order += [srv.reqs[i].job["name"] for i in srv.tick()]
    assert order == ["H", "long"]  # every 0.3 s a chunk despite the running batch
