"""Seeded synthetic workloads of the batched and serving forms.

Batched (64 bunches): particle counts log-uniform in [1e4, 5e5], meshes from
{16^3, 32^3, 48^3, 64^3}, sigma_x, sigma_y, sigma_z each uniform in
[0.5, 3] mm, charge uniform in [0.1, 2] nC, mean beta*gamma uniform in
[2, 20], 200 steps at dt = 1 ps.

Serving: Poisson arrivals at 50 jobs/s for 60 s; each job one Gaussian bunch
with particle count log-uniform in [1e4, 2e6], mesh n^3 with n from
{16, 24, 32, 48, 64, 96, 128} (transform lengths with fast kernels),
50..500 steps, the batched workload's distributions otherwise.

Every draw comes from numpy's PCG64 seeded with the workload seed, so a
workload is the same list of jobs on every run.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

MASS_EV = 0.51099892e6
DT = 1e-12


@dataclass
class Job:
    job_id: int
    arrival_s: float
    particles: int
    mesh: int
    sigma: tuple
    bg_z: float
    charge_nc: float
    steps: int

    @property
    def q_macro(self):
        return -self.charge_nc * 1e-9 / self.particles

    @property
    def ref_P(self):
        return (0.0, 0.0, self.bg_z)

    def footprint_bytes(self, precision):
        """Device memory of the job's context (particles and grids), as
        allocated by scgpu_create + scgpu_bunch_upload."""
        n = self.mesh
        M = n ** 3
        S = (n + 1) * (2 * n) ** 2
        G3 = (n + 1) ** 3
        T3 = (n + 2) ** 3
        r = 8 if precision == 0 else 4
        particles = self.particles * (6 * 8 + 5 * 4 + 6 * 8)
        grids = M * (16 + 8 + r + 4 * r + 8) + S * 16 + (S * 8 if precision else 0) + T3 * 8 + G3 * (8 + r)
        return particles + grids + (1 << 20)


def batched_jobs(count=64, seed=20261203, steps=200):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(count):
        n_part = int(round(np.exp(rng.uniform(np.log(1e4), np.log(5e5)))))
        mesh = int(rng.choice([16, 32, 48, 64]))
        sigma = tuple(float(v) for v in rng.uniform(0.5e-3, 3e-3, size=3))
        charge = float(rng.uniform(0.1, 2.0))
        bg = float(rng.uniform(2.0, 20.0))
        jobs.append(Job(i, 0.0, n_part, mesh, sigma, bg, charge, steps))
    return jobs


def serving_jobs(rate_hz=50.0, duration_s=60.0, seed=20261204):
    rng = np.random.default_rng(seed)
    jobs = []
    t = 0.0
    i = 0
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t >= duration_s:
            break
        n_part = int(round(np.exp(rng.uniform(np.log(1e4), np.log(2e6)))))
        mesh = int(rng.choice([16, 24, 32, 48, 64, 96, 128]))
        sigma = tuple(float(v) for v in rng.uniform(0.5e-3, 3e-3, size=3))
        charge = float(rng.uniform(0.1, 2.0))
        bg = float(rng.uniform(2.0, 20.0))
        steps = int(rng.integers(50, 501))
        jobs.append(Job(i, t, n_part, mesh, sigma, bg, charge, steps))
        i += 1
    return jobs
