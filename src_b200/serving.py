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

    def run(self, jobs, realtime=True):
        """Serves `jobs`.  With realtime the arrivals are honoured on the wall
        clock; otherwise every job is available at once.  Returns the list of
        Results in completion order.

        Each round launches k steps for the current slots and, while the
        device works, admits the jobs that have arrived (their bunches are
        prepared and uploaded meanwhile; they join at the next round)."""
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival_s))
        active = {}   # slot -> [job, remaining steps, admitted_s, footprint]
        joining = {}  # admitted during the current round
        results = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731

        def admit():
            t = now()
            while pending and (not realtime or pending[0].arrival_s <= t):
                job = pending[0]
                fp = job.footprint_bytes(self.precision)
                if (active or joining) and self.used + fp > self.budget:
                    break
                pending.popleft()
                ta = time.perf_counter()
                R, P = self.masters.bunch(job)
                slot = self.batch.add((job.mesh,) * 3, R, P, DT, job.q_macro, MASS_EV, ref_P=job.ref_P)
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
            admit()
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
