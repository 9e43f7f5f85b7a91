"""Continuous-batching server for "run N steps of this system" jobs.

Every admitted job is one system in the engine's arena, and all admitted
systems advance together in the same kernels.  The loop:

  1. admit queued jobs (in arrival order) while the resident particles stay
     under a cap and their estimated device footprint fits the HBM budget;
     newly admitted systems and the removal of finished ones take effect at
     one ``commit`` (which keeps the state of the systems that stay);
  2. advance every running job by ``min(chunk, fewest steps any running job
     still needs)`` steps (fewer if that would take longer than
     ``chunk_seconds``), so each job ends exactly on its step count;
  3. read back the jobs that finished, freeze them (they stop advancing and
     cost no force evaluation) and retire them at the next commit.

Jobs arriving while others run wait in the queue and join at the next
admission; their work then overlaps with every other running job.  In the
mixed form a job's result is bit-for-bit the same alone and in any mix
(tests/test_gpu_serve.py).
"""
from __future__ import annotations

import collections
import dataclasses
import statistics
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, Optional

import numpy as np

from .engine import Engine
from .systems import SystemDesc


@dataclasses.dataclass
class Job:
    job_id: int
    nsteps: int
    arrival: float                                  # seconds since server start
    desc: Optional[SystemDesc] = None
    build: Optional[Callable[[], SystemDesc]] = None  # builds desc lazily
    n: int = 0
    sid: Optional[int] = None
    done: int = 0
    admitted: Optional[float] = None
    finished: Optional[float] = None
    pos: Optional[np.ndarray] = None
    vel: Optional[np.ndarray] = None

    @property
    def latency(self) -> Optional[float]:
        """Completion latency: arrival to completion (queueing included)."""
        return None if self.finished is None else self.finished - self.arrival

    @property
    def service(self) -> Optional[float]:
        """Service latency: admission to completion (on the GPU)."""
        return None if self.finished is None or self.admitted is None else self.finished - self.admitted


class Server:
    """Admission control: a queued job is admitted (in arrival order) when the
    resident particles stay within ``max_particles`` and the device footprint
    within ``hbm_fraction`` of device memory, the footprint counted at the
    arena's measured bytes per particle (mjg_device_bytes after the last
    commit).  ``max_particles`` is
    the concurrency at which the arena's throughput has saturated: admitting
    more raises no throughput, only every running job's latency.  Chunks are
    sized so one lasts about ``chunk_seconds`` (at most ``chunk`` steps), which
    bounds how long an arrival waits for the next admission."""

    def __init__(self, precision: str = "mixed", chunk: int = 500, hbm_fraction: float = 0.8,
                 device: int = 0, bytes_per_particle: float = 2048.0, min_commit_interval: float = 0.0,
                 keep_results: bool = True, builders: int = 4, max_particles: int = 2_000_000,
                 chunk_seconds: Optional[float] = None, lookahead: int = 64,
                 tuned: Optional[dict] = None):
        self.eng = Engine(precision, device=device)
        self.eng.reserve(max_particles)          # page-lock once, at start-up
        # per global term: {"margin", "schedule", "threads_per_particle", "unroll"}
        # as :func:`mjolnir_b200.autotune.tune` returns them; the margin
        # replaces each admitted job's, the launch shape is set after every
        # commit (it changes no result in the mixed form)
        self.tuned = tuned or {}
        self.chunk = int(chunk)
        self.chunk_seconds = chunk_seconds
        self.keep_results = keep_results
        self.min_commit_interval = min_commit_interval
        self.max_particles = int(max_particles)
        self.lookahead = int(lookahead)
        total = self._device_total(device)
        self.budget = hbm_fraction * total
        # device bytes per resident particle: this estimate until the first
        # commit, then the arena's measured footprint (mjg_device_bytes)
        self.bpp = bytes_per_particle
        self.queue = collections.deque()        # arrived, not admitted
        self.running = {}                       # sid -> Job
        self.retiring = []                      # finished sids awaiting the next commit
        self.finished = []
        self.t0 = time.perf_counter()
        self.lock = threading.Lock()
        self.pool = ThreadPoolExecutor(max_workers=builders)
        self.futures = {}
        self.last_commit = -1e9
        self.particle_steps = 0
        self.commits = 0
        self.commit_s = 0.0
        self.step_s = 0.0
        self.steps_run = 0
        self.sec_per_step = None                # of the current arena, measured
        self.max_queue = 0

    @staticmethod
    def _device_total(device: int) -> float:
        try:
            import torch
            return float(torch.cuda.mem_get_info(device)[1])
        except Exception:
            return 180e9

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # ---------------------------------------------------------------- input
    def submit(self, job: Job):
        """Queues a job (thread safe); its system is built in the background
        once it is near the head of the queue."""
        with self.lock:
            self.queue.append(job)
            self.max_queue = max(self.max_queue, len(self.queue))
            self._prefetch()

    def _prefetch(self):
        for k, job in enumerate(self.queue):
            if k >= self.lookahead:
                break
            if job.desc is None and job.build is not None and job.job_id not in self.futures:
                self.futures[job.job_id] = self.pool.submit(job.build)

    # ---------------------------------------------------------------- loop
    def _resident_particles(self) -> int:
        return sum(j.n for j in self.running.values())

    def _admit(self) -> bool:
        """Adds every queued job that fits; returns True if the arena changed."""
        changed = False
        resident = self._resident_particles()
        with self.lock:
            while self.queue:
                job = self.queue[0]
                if job.desc is None:
                    fut = self.futures.get(job.job_id)
                    if fut is None or not fut.done():
                        break                   # keep arrival order
                    job.desc = fut.result()
                    del self.futures[job.job_id]
                n = job.desc.n
                if self.running and ((resident + n) * self.bpp > self.budget
                                     or resident + n > self.max_particles):
                    break
                self.queue.popleft()
                job.n = n
                for key, cfg in self.tuned.items():
                    term = getattr(job.desc, key, None)
                    if term is not None and "margin" in cfg:
                        term.margin = cfg["margin"]
                job.sid = self.eng.add_system(job.desc)
                job.admitted = self.now()
                if not self.keep_results:
                    job.desc = None
                self.running[job.sid] = job
                resident += n
                changed = True
            self._prefetch()
        return changed

    def _commit(self):
        t = time.perf_counter()
        for sid in self.retiring:
            self.eng.remove_system(sid)
        self.retiring = []
        self.eng.commit()
        for key, cfg in self.tuned.items():
            try:
                self.eng.get_threads_per_particle(key)
            except Exception:
                continue                         # term not in the arena now
            if self.eng.precision == "mixed" and self.eng.get_half_lists(key) != cfg.get("half_lists", False):
                self.eng.set_half_lists(key, cfg.get("half_lists", False))
            if self.eng.get_pair_schedule(key) != cfg.get("schedule", 0):
                self.eng.set_pair_schedule(key, cfg.get("schedule", 0))
            if self.eng.get_threads_per_particle(key) != cfg.get("threads_per_particle", 1):
                self.eng.set_threads_per_particle(key, cfg.get("threads_per_particle", 1))
            if self.eng.get_pair_unroll(key) != cfg.get("unroll", 1):
                self.eng.set_pair_unroll(key, cfg.get("unroll", 1))
            if "build_lanes" in cfg and self.eng.get_build_lanes(key) != cfg["build_lanes"]:
                self.eng.set_build_lanes(key, cfg["build_lanes"])
        self.commits += 1
        self.commit_s += time.perf_counter() - t
        self.last_commit = self.now()
        self.sec_per_step = None
        n = self._resident_particles()
        if n > 0:
            self.bpp = self.eng.device_bytes() / n      # measured after this commit

    def _chunk_steps(self, live) -> int:
        k = min(self.chunk, min(j.nsteps - j.done for j in live))
        if self.chunk_seconds is not None and self.sec_per_step:
            k = min(k, max(10, int(self.chunk_seconds / self.sec_per_step)))
        return max(1, k)

    def step_once(self) -> bool:
        """One admission/advance/retire round; False when nothing is running."""
        pending_retire = bool(self.retiring)
        if (self.now() - self.last_commit >= self.min_commit_interval) or not self.running:
            if self._admit() or (pending_retire and not self.running):
                self._commit()
        live = [j for j in self.running.values()]
        if not live:
            if self.retiring:
                self._commit()
            return False
        k = self._chunk_steps(live)
        t = time.perf_counter()
        self.eng.step(k)
        dt = time.perf_counter() - t
        self.step_s += dt
        self.steps_run += k
        if k >= 10:
            self.sec_per_step = dt / k
        t = self.now()
        for j in live:
            j.done += k
            self.particle_steps += j.n * k
        for j in live:
            if j.done >= j.nsteps:
                if self.keep_results:
                    p, v, _ = self.eng.state(j.sid)
                    j.pos, j.vel = p, v
                j.finished = t
                self.eng.freeze(j.sid)
                del self.running[j.sid]
                self.retiring.append(j.sid)
                self.finished.append(j)
        return True

    def run_until_idle(self, timeout: float = 3600.0):
        end = self.now() + timeout
        while self.now() < end:
            if not self.step_once():
                with self.lock:
                    if not self.queue:
                        return
                time.sleep(0.001)

    def stats(self, wall: float) -> dict:
        lat = sorted(j.latency for j in self.finished)
        svc = sorted(j.service for j in self.finished)
        q = lambda v, p: v[min(len(v) - 1, int(p * len(v)))] if v else None  # noqa: E731
        return {"completed": len(lat), "queued": len(self.queue), "running": len(self.running),
                "resident_particles": self._resident_particles(), "max_queue": self.max_queue,
                "latency_p50_s": q(lat, 0.50), "latency_p90_s": q(lat, 0.90), "latency_p99_s": q(lat, 0.99),
                "latency_mean_s": statistics.mean(lat) if lat else None,
                "service_p50_s": q(svc, 0.50), "service_p90_s": q(svc, 0.90), "service_p99_s": q(svc, 0.99),
                "device_bytes_per_particle": self.bpp,
                "particle_steps_per_s": self.particle_steps / wall if wall > 0 else None,
                "commits": self.commits, "commit_s": self.commit_s, "step_s": self.step_s,
                "md_steps": self.steps_run}

    def close(self):
        self.pool.shutdown(wait=False, cancel_futures=True)
        self.eng.close()


def poisson_workload(rate: float, duration: float, seed: int = 7, nmin: int = 200, nmax: int = 50000,
                     smin: int = 1000, smax: int = 100000, periodic_fraction: float = 0.5):
    """Jobs of the serving configuration: Poisson arrivals at `rate` per second;
    size log-uniform in [nmin, nmax] beads of the config-2 composition, steps
    log-uniform in [smin, smax], T ~ U[280, 360] K; a `periodic_fraction` of
    them in a periodic cube of side 2R around the chains' sphere of radius R
    (10,000 beads per 300 A sphere density), the rest in unbounded space."""
    from . import systems as S
    rng = np.random.default_rng(seed)
    t, jobs, k = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        steps = int(np.exp(rng.uniform(np.log(smin), np.log(smax))))
        temp = float(rng.uniform(280.0, 360.0))
        periodic = bool(rng.uniform() < periodic_fraction)
        jseed = int(rng.integers(1, 2 ** 31))

        def build(n=n, temp=temp, periodic=periodic, jseed=jseed):
            nchains = max(1, round(n / 200))
            nbeads = max(4, round(n / nchains))
            radius = 300.0 * (nchains * nbeads / 10000.0) ** (1.0 / 3.0)
            d = S.polymer_melt(nchains=nchains, nbeads=nbeads, radius=radius, temperature=temp,
                               seed=jseed)
            if periodic:
                d.boundary = "PeriodicCuboid"
                d.lower = (0.0, 0.0, 0.0)
                d.upper = (2 * radius,) * 3
                d.pos = d.pos + radius
            return d

        jobs.append(Job(job_id=k, nsteps=steps, arrival=t, build=build))
        k += 1
    return jobs


def serve_poisson(duration: float = 60.0, rate: float = 200.0, chunk: int = 2000, seed: int = 7,
                  precision: str = "mixed", max_particles: int = 2_000_000,
                  chunk_seconds: float = 1.0, min_commit_interval: float = 1.0,
                  tuned: Optional[dict] = None) -> dict:
    """Replays a Poisson stream in real time for `duration` seconds and
    reports completion latency, queue depth and aggregate throughput.
    `tuned`: margins and launch shapes to serve with (autotuner output)."""
    jobs = poisson_workload(rate, duration, seed=seed)
    srv = Server(precision=precision, chunk=chunk, keep_results=False,
                 min_commit_interval=min_commit_interval, max_particles=max_particles,
                 chunk_seconds=chunk_seconds, tuned=tuned)
    srv.t0 = time.perf_counter()
    i = 0
    while srv.now() < duration:
        while i < len(jobs) and jobs[i].arrival <= srv.now():
            srv.submit(jobs[i])
            i += 1
        if not srv.step_once():
            time.sleep(0.002)
    wall = srv.now()
    out = srv.stats(wall)
    out.update({"arrived": i, "duration_s": wall, "rate_jobs_per_s": rate, "max_chunk_steps": chunk,
                "chunk_seconds": chunk_seconds, "max_particles": max_particles})
    srv.close()
    return out
