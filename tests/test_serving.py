"""Host logic of the serving loop (admission by HBM footprint, rounds of
batched steps, completion) against a fake batch: no GPU needed."""
import numpy as np

from src_b200.serving import Server, latency_summary
from src_b200.workloads import Job, batched_jobs, serving_jobs


class FakeBatch:
    """done_after: the round in flight reports itself finished on the device
    once that many bunches were admitted during it (None: never)."""

    def __init__(self, done_after=None):
        self.slots = {}
        self.steps = {}
        self.tracked = []
        self.peak = 0
        self.done_after = done_after
        self.in_round = 0
        self.admits_per_round = []

    def add(self, nr, R, P, dT, q, mass, **kw):
        self.in_round += 1
        slot = min(set(range(len(self.slots) + 1)) - set(self.slots))
        self.slots[slot] = R.shape[0]
        self.steps[slot] = 0
        self.peak = max(self.peak, len(self.slots))
        return slot

    def remove(self, slot):
        del self.slots[slot]

    def done(self):
        return self.done_after is not None and self.in_round >= self.done_after

    def launch(self, k):
        self.admits_per_round.append(self.in_round)
        self.in_round = 0
        self.tracked.append((k, len(self.slots)))
        for s in self.slots:
            self.steps[s] += k

    def wait(self):
        return 0.0

    def set_tuning(self, *a):
        pass

    def close(self):
        pass


class FakeMasters:
    def bunch(self, job):
        return np.zeros((job.particles, 3)), np.zeros((job.particles, 3))


def job(i, n=1000, mesh=16, steps=40, t=0.0):
    return Job(i, t, n, mesh, (1e-3, 1e-3, 1e-3), 10.0, 1.0, steps)


def test_every_job_takes_exactly_its_steps():
    jobs = [job(i, steps=s) for i, s in enumerate([5, 17, 40, 33, 16, 1])]
    fb = FakeBatch()
    srv = Server(hbm_budget_bytes=1 << 40, batch=fb, masters=FakeMasters())
    res = srv.run(jobs, realtime=False)
    assert sorted(r.job.job_id for r in res) == list(range(6))
    # a slot never steps past its job's request
    assert all(fb.steps[s] <= 40 for s in fb.steps)
    assert srv.particle_steps == sum(j.particles * j.steps for j in jobs)
    assert all(k <= 16 for k, _ in fb.tracked)
    # completion order follows the requested step counts
    assert [r.job.steps for r in res] == sorted(j.steps for j in jobs)


def test_admission_respects_the_hbm_budget():
    jobs = [job(i, n=200_000, mesh=64, steps=20) for i in range(6)]
    one = jobs[0].footprint_bytes(0)
    fb = FakeBatch()
    srv = Server(hbm_budget_bytes=int(2.5 * one), batch=fb, masters=FakeMasters())
    res = srv.run(jobs, realtime=False)
    assert len(res) == 6
    assert fb.peak == 2          # never more than two jobs' footprint resident
    assert srv.used == 0         # everything released


def test_a_job_larger_than_the_budget_still_runs_alone():
    jobs = [job(0, n=2_000_000, mesh=128, steps=3)]
    fb = FakeBatch()
    srv = Server(hbm_budget_bytes=1, batch=fb, masters=FakeMasters())
    assert len(srv.run(jobs, realtime=False)) == 1


def test_arrivals_are_honoured_in_realtime():
    jobs = [job(i, steps=3, t=0.05 * i) for i in range(4)]
    srv = Server(hbm_budget_bytes=1 << 40, batch=FakeBatch(), masters=FakeMasters())
    res = srv.run(jobs, realtime=True)
    assert all(r.admitted_s >= r.job.arrival_s for r in res)
    assert all(r.latency_s >= 0 for r in res)


def test_workloads_are_seeded_and_in_range():
    a, b = serving_jobs(), serving_jobs()
    assert [(j.arrival_s, j.particles, j.mesh, j.steps) for j in a] == [(j.arrival_s, j.particles, j.mesh, j.steps)
                                                                        for j in b]
    assert 2700 < len(a) < 3300                      # ~50 jobs/s for 60 s
    assert all(1e4 <= j.particles <= 2e6 and 50 <= j.steps <= 500 and j.arrival_s < 60 for j in a)
    c4 = batched_jobs()
    assert len(c4) == 64 and {j.mesh for j in c4} <= {16, 32, 48, 64}
    assert all(1e4 <= j.particles <= 5e5 and 2 <= j.bg_z <= 20 and 0.1 <= j.charge_nc <= 2 for j in c4)


def test_latency_summary():
    class R:
        def __init__(self, lat):
            self.latency_s = lat
    s = latency_summary([R(v) for v in range(1, 101)])
    assert s["jobs"] == 100 and abs(s["p50_s"] - 50.5) < 1e-9 and s["p99_s"] > 98


def test_preparer_thread_matches_inline_preparation():
    """Bunches prepared ahead on the worker thread (into reusable host
    buffers) give the same admissions and rounds as bunches prepared on the
    serving thread at admission."""
    jobs = [job(i, n=500 + 37 * i, steps=10 + 3 * i) for i in range(12)]
    out = []
    for ahead in (0, 3):
        fb = FakeBatch()
        srv = Server(hbm_budget_bytes=1 << 40, batch=fb, masters=FakeMasters())
        res = srv.run(jobs, realtime=False, prepare_ahead=ahead)
        out.append(([r.job.job_id for r in res], fb.tracked))
    assert out[0] == out[1]


def test_admission_stops_when_the_round_has_finished():
    """While a round runs, jobs are admitted until the device reports the
    round finished; the rest wait for the next round, and every job still
    takes exactly its steps.  The HBM budget holds three jobs, so all but
    the first three are admitted during rounds."""
    jobs = [job(i, steps=2 + (i % 4)) for i in range(12)]
    fp = jobs[0].footprint_bytes(0)
    for done_after, bound in ((1, 1), (2, 2), (None, 3)):
        fb = FakeBatch(done_after=done_after)
        srv = Server(hbm_budget_bytes=3 * fp, batch=fb, masters=FakeMasters())
        res = srv.run(jobs, realtime=False)
        assert sorted(r.job.job_id for r in res) == list(range(12))
        assert srv.particle_steps == sum(j.particles * j.steps for j in jobs)
        assert fb.admits_per_round[0] == 3  # no round in flight yet: as many as fit
        assert sum(fb.admits_per_round) + fb.in_round == 12
        assert max(fb.admits_per_round[1:]) <= bound
        if done_after is not None:
            assert max(fb.admits_per_round[1:]) == bound
