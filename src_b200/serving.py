"""Serving loop: space-charge tracking jobs admitted as they arrive and
advanced together in batched steps (continuous batching over scgpu_batch_*).

The reference's optimizer runs one complete OPAL simulation per design point
(optimizer/Pilot/Worker.h:31-190 -> OpalSimulation::run,
src/Optimize/OpalSimulation.cpp:232), one bunch per process.  Here one host
thread drives one GPU:

* jobs arrive with an arrival time (a Poisson process in the benchmark);
* a job is admitted when it has arrived and its device footprint fits the
  HBM budget (first come, first served; a job that does not fit holds the
  queue until memory frees);
* every admitted job becomes a slot of one Batch and all slots advance
  together, a few steps per round, so jobs that arrive while others run share
  the device with them;
* a job that has taken its steps is (optionally downloaded and) removed,
  which frees its memory for waiting jobs.

Because the batched kernels never mix bunches and all sums are exact, a job's
result does not depend on which other jobs shared its steps.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import scgpu
from .workloads import DT, MASS_EV, Job

MAX_ROUND_STEPS = 16


@dataclass
class Result:
    job: Job
    admitted_s: float
    done_s: float
    R: np.ndarray = field(default=None, repr=False)   # kept only with keep_results
    P: np.ndarray = field(default=None, repr=False)

    @property
    def latency_s(self):
        return self.done_s - self.job.arrival_s


class MasterBunches:
    """A few large seeded unit bunches; a job's bunch is the first N
    particles of one of them, scaled to the job's sigma and beta*gamma, so
    job data costs a host-side scaling instead of a fresh draw."""

    def __init__(self, count=4, size=2_000_000):
        from .bunch import gaussian_bunch

        self.masters = [gaussian_bunch(size, sigma=(1.0, 1.0, 1.0), bg_z=1.0, bunch_id=900 + k) for k in range(count)]

    def bunch(self, job: Job):
        R0, P0 = self.masters[job.job_id % len(self.masters)]
        n = job.particles
        R = R0[:n] * np.asarray(job.sigma)
        P = P0[:n].copy()
        P[:, 2] *= job.bg_z
        return R, P


class Preparer:
    """Prepares the bunches of arriving jobs on a worker thread, ahead of
    admission: each job's scaled copy of its master bunch is written into one
    of a few page-locked host buffers (sized for the largest job), so the
    serving thread only uploads (from pinned memory, at full link speed) while
    the device runs a round.  Jobs are prepared in arrival order, at most
    `depth` ahead; a buffer returns to the pool once its job is uploaded."""

    def __init__(self, masters, max_particles, depth=4, realtime=True):
        import queue
        import threading

        import torch

        self.masters = masters
        self.realtime = realtime
        self.free = queue.Queue()
        pin = torch.cuda.is_available()
        for _ in range(depth):
            self.free.put(tuple(torch.empty((max_particles, 3), dtype=torch.float64, pin_memory=pin).numpy()
                                for _ in range(2)))
        self.ready = collections.deque()
        self.cv = threading.Condition()
        self.jobs = None
        self.t0 = None
        self.prep_s = 0.0
        self.stop = False
        self.thread = None

    def start(self, jobs, t0):
        import threading

        self.jobs = list(jobs)
        self.t0 = t0
        self.thread = threading.Thread(target=self._work, daemon=True)
        self.thread.start()

    def _work(self):
        for job in self.jobs:
            # a job is prepared once it has arrived, never before
            while self.realtime and not self.stop and time.perf_counter() - self.t0 < job.arrival_s:
                time.sleep(min(0.002, max(0.0, job.arrival_s - (time.perf_counter() - self.t0))))
            if self.stop:
                return
            bufs = self.free.get()
            if self.stop or bufs is None:
                return
            ta = time.perf_counter()
            n = job.particles
            R, P = bufs[0][:n], bufs[1][:n]
            if hasattr(self.masters, "masters"):
                R0, P0 = self.masters.masters[job.job_id % len(self.masters.masters)]
                np.multiply(R0[:n], np.asarray(job.sigma), out=R)
                P[:] = P0[:n]
                P[:, 2] *= job.bg_z
            else:
                R[:], P[:] = self.masters.bunch(job)
            self.prep_s += time.perf_counter() - ta
            with self.cv:
                self.ready.append((job, R, P, bufs))
                self.cv.notify_all()

    def take(self, job, timeout=60.0):
        """The prepared (R, P, buffers) of `job` (the next one in arrival order)."""
        with self.cv:
            ok = self.cv.wait_for(lambda: self.ready and self.ready[0][0] is job, timeout=timeout)
            if not ok:
                raise RuntimeError(f"job {job.job_id} was not prepared in time")
            _, R, P, bufs = self.ready.popleft()
        return R, P, bufs

    def give_back(self, bufs):
        self.free.put(bufs)

    def close(self):
        self.stop = True
        for _ in range(2):
            self.free.put(None)
        if self.thread is not None:
            self.thread.join(timeout=10)


class Server:
    def __init__(self, precision=scgpu.PLAIN_FP64, hbm_budget_bytes=None, device=0, masters=None, batch=None,
                 keep_results=False):
        self.precision = precision
        self.device = device
        self.batch = batch if batch is not None else scgpu.Batch(precision=precision, device=device)
        self.keep_results = keep_results
        if hbm_budget_bytes is None:
            import torch

            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget_bytes = int(0.8 * free)
        self.budget = hbm_budget_bytes
        self.used = 0
        self.masters = masters or MasterBunches()
        self.rounds = 0
        self.steps = 0
        self.particle_steps = 0
        self.makespan_s = 0.0
        self.tuning = {}
        # host wall time by activity, and device time of the batched steps
        self.time = {"admit_s": 0.0, "track_wall_s": 0.0, "track_gpu_s": 0.0, "release_s": 0.0}

    def calibrate(self, jobs, trial_steps=3):
        """Runs the autotuner on a separate batch of `jobs` (one per mesh size
        is enough) and applies its choices to the serving batch, so that the
        served jobs take exactly their requested steps."""
        with scgpu.Batch(precision=self.precision, device=self.device) as cal:
            for job in jobs:
                R, P = self.masters.bunch(job)
                cal.add((job.mesh,) * 3, R, P, DT, job.q_macro, MASS_EV, ref_P=job.ref_P)
            cal.autotune(trial_steps)
            lengths = sorted({2 * job.mesh for job in jobs})
            self.tuning = {L: cal.tuning(L) for L in lengths}
        for L, t in self.tuning.items():
            self.batch.set_tuning(t["deposit_threads"], L, t["fft_variant"])
        return self.tuning

    def close(self):
        self.batch.close()

    def run(self, jobs, realtime=True, prepare_ahead=4):
        """Serves `jobs`.  With realtime the arrivals are honoured on the wall
        clock; otherwise every job is available at once.  Returns the list of
        Results in completion order.

        Each round launches k steps for the current slots and, while the
        device works, admits the jobs that have arrived (their bunches were
        prepared in pinned memory by the Preparer thread and are uploaded
        meanwhile; they join at the next round) until the round has
        finished on the device; jobs not yet admitted wait for the next
        round.  prepare_ahead = 0 prepares
        each bunch on the serving thread at admission instead."""
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival_s))
        active = {}   # slot -> [job, remaining steps, admitted_s, footprint]
        joining = {}  # admitted during the current round
        results = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        prep = None
        if prepare_ahead > 0 and pending:
            prep = Preparer(self.masters, max(j.particles for j in pending), depth=prepare_ahead, realtime=realtime)
            prep.start(pending, t0)

        def admit(in_round):
            # While a round runs, admit until it has finished on the device:
            # an admission waits for its upload, and a round left finished
            # behind a long admission would idle the device.
            t = now()
            while pending and (not realtime or pending[0].arrival_s <= t):
                if in_round and self.batch.done():
                    break
                job = pending[0]
                fp = job.footprint_bytes(self.precision)
                if (active or joining) and self.used + fp > self.budget:
                    break
                pending.popleft()
                ta = time.perf_counter()
                if prep is not None:
                    R, P, bufs = prep.take(job)
                else:
                    R, P = self.masters.bunch(job)
                slot = self.batch.add((job.mesh,) * 3, R, P, DT, job.q_macro, MASS_EV, ref_P=job.ref_P)
                if prep is not None:
                    prep.give_back(bufs)
                self.time["admit_s"] += time.perf_counter() - ta
                joining[slot] = [job, job.steps, now(), fp]
                self.used += fp

        while pending or active or joining:
            k = 0
            if active:
                # every active job takes k steps this round (k <= its remaining steps)
                k = min(MAX_ROUND_STEPS, min(a[1] for a in active.values()))
                tt = time.perf_counter()
                self.batch.launch(k)
                self.time["track_wall_s"] += time.perf_counter() - tt
            admit(k > 0)
            if k:
                tt = time.perf_counter()
                gpu_ms = self.batch.wait()
                self.time["track_wall_s"] += time.perf_counter() - tt
                self.time["track_gpu_s"] += gpu_ms * 1e-3
                self.rounds += 1
                self.steps += k
                for slot, a in list(active.items()):
                    self.particle_steps += a[0].particles * k
                    a[1] -= k
                    if a[1] <= 0:
                        tr = time.perf_counter()
                        R = P = None
                        if self.keep_results:
                            R, P = self.batch.member(slot).download()
                        self.batch.remove(slot)
                        self.time["release_s"] += time.perf_counter() - tr
                        self.used -= a[3]
                        results.append(Result(a[0], a[2], now(), R, P))
                        del active[slot]
            active.update(joining)
            joining.clear()
            if not active and pending and realtime:
                time.sleep(max(0.0, min(pending[0].arrival_s - now(), 0.01)))
        self.makespan_s = now()
        if prep is not None:
            self.time["prepare_s"] = prep.prep_s
            prep.close()
        return results


def latency_summary(results):
    lat = np.array([r.latency_s for r in results])
    return {"jobs": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}


def run_alone(job: Job, precision, masters: MasterBunches, steps=None, device=0):
    """The job tracked by itself in a single-bunch context."""
    R, P = masters.bunch(job)
    with scgpu.Context((job.mesh,) * 3, precision=precision, device=device) as c:
        c.upload(R, P, DT, job.q_macro, MASS_EV, ref_P=job.ref_P)
        c.track(job.steps if steps is None else steps)
        return c.download()
