"""Batched stepping (scgpu_batch_*): many bunches of different sizes and
meshes in one set of launches.  Every bunch's result must be the one it gets
when it is tracked alone: the kernels never mix bunches and every sum is
exact, so the comparison is bitwise."""
import numpy as np
import pytest

from src_b200.bunch import gaussian_bunch

pytestmark = pytest.mark.gpu

MASS = 0.51099892e6
DT = 1e-12

# (particles, mesh, sigma, beta*gamma, charge [nC], B_z)
BUNCHES = [
    (20_000, (16, 16, 16), (1e-3, 1e-3, 2e-3), 10.0, 1.0, 0.0),
    (75_000, (32, 32, 32), (0.7e-3, 1.5e-3, 1e-3), 4.0, 0.3, 0.2),
    (150_000, (48, 48, 48), (2e-3, 2e-3, 3e-3), 15.0, 2.0, 0.0),
    (40_000, (24, 32, 16), (1e-3, 0.6e-3, 2.5e-3), 6.0, 0.5, 0.0),
    (110_000, (64, 64, 64), (1.2e-3, 1e-3, 1.8e-3), 20.0, 1.5, 0.2),
]


def make(i, spec):
    n, nr, sig, bg, qnc, bz = spec
    R, P = gaussian_bunch(n, sigma=sig, bg_z=bg, bunch_id=100 + i)
    return dict(R=R, P=P, nr=nr, Q=-qnc * 1e-9 / n, bz=bz, ref_P=(0.0, 0.0, bg))


def alone(gpu, b, steps, precision):
    with gpu.Context(b["nr"], precision=precision) as c:
        c.upload(b["R"], b["P"], DT, b["Q"], MASS, bz_ext=b["bz"], ref_P=b["ref_P"])
        c.track(steps)
        R, P = c.download()
        return R, P, c.tracker_state(), c.field(gpu.FIELD_E)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_alone(gpu, precision):
    steps = 20
    bunches = [make(i, s) for i, s in enumerate(BUNCHES)]
    with gpu.Batch(precision=precision) as bt:
        slots = [bt.add(b["nr"], b["R"], b["P"], DT, b["Q"], MASS, bz_ext=b["bz"], ref_P=b["ref_P"]) for b in bunches]
        assert bt.size() == len(bunches)
        bt.track(steps)
        got = []
        for s in slots:
            m = bt.member(s)
            R, P = m.download()
            got.append((R, P, m.tracker_state(), m.field(gpu.FIELD_E)))
    for b, (R, P, st, E) in zip(bunches, got):
        Ra, Pa, sta, Ea = alone(gpu, b, steps, precision)
        np.testing.assert_array_equal(R, Ra)
        np.testing.assert_array_equal(P, Pa)
        np.testing.assert_array_equal(E, Ea)
        assert st["step"] == sta["step"] == steps
        assert st["path_length"] == sta["path_length"] and st["t"] == sta["t"]


def test_batch_done_reports_the_round(gpu):
    """scgpu_batch_done never blocks: true with nothing in flight, and true
    once launched steps have finished (polled with a bounded wait); the
    steps' results are those of a plain track."""
    import time

    b = make(0, BUNCHES[2])
    with gpu.Batch(precision=0) as bt:
        assert bt.done()
        s = bt.add(b["nr"], b["R"], b["P"], DT, b["Q"], MASS, bz_ext=b["bz"], ref_P=b["ref_P"])
        bt.launch(6)
        t0 = time.perf_counter()
        while not bt.done() and time.perf_counter() - t0 < 30.0:
            time.sleep(1e-3)
        assert bt.done()
        bt.wait()
        assert bt.done()
        R, P = bt.member(s).download()
    Ra, Pa, _, _ = alone(gpu, b, 6, 0)
    np.testing.assert_array_equal(R, Ra)
    np.testing.assert_array_equal(P, Pa)


def test_batch_membership_changes_and_autotune(gpu):
    """Bunches join and leave between steps (continuous batching) and the
    autotuner switches launch shapes; each bunch still matches its alone run
    for the number of steps it took."""
    bunches = [make(i, s) for i, s in enumerate(BUNCHES)]
    with gpu.Batch(precision=1) as bt:
        s0 = bt.add(bunches[0]["nr"], bunches[0]["R"], bunches[0]["P"], DT, bunches[0]["Q"], MASS,
                    bz_ext=bunches[0]["bz"], ref_P=bunches[0]["ref_P"])
        s1 = bt.add(bunches[1]["nr"], bunches[1]["R"], bunches[1]["P"], DT, bunches[1]["Q"], MASS,
                    bz_ext=bunches[1]["bz"], ref_P=bunches[1]["ref_P"])
        bt.track(7)
        R0, P0 = bt.member(s0).download()
        bt.remove(s0)
        s2 = bt.add(bunches[2]["nr"], bunches[2]["R"], bunches[2]["P"], DT, bunches[2]["Q"], MASS,
                    bz_ext=bunches[2]["bz"], ref_P=bunches[2]["ref_P"])
        s4 = bt.add(bunches[4]["nr"], bunches[4]["R"], bunches[4]["P"], DT, bunches[4]["Q"], MASS,
                    bz_ext=bunches[4]["bz"], ref_P=bunches[4]["ref_P"])
        taken = bt.autotune(2)
        assert taken > 0
        for L in (32, 64, 96, 128):
            t = bt.tuning(L)
            assert t["deposit_threads"] in (128, 256, 512) and t["fft_variant"] in (0, 1, 2, 3, 4)
        bt.track(5)
        R1, P1 = bt.member(s1).download()
        R2, P2 = bt.member(s2).download()
        R4, P4 = bt.member(s4).download()
    for b, (R, P), steps in ((bunches[0], (R0, P0), 7), (bunches[1], (R1, P1), 7 + taken + 5),
                             (bunches[2], (R2, P2), taken + 5), (bunches[4], (R4, P4), taken + 5)):
        Ra, Pa, _, _ = alone(gpu, b, steps, 1)
        np.testing.assert_array_equal(R, Ra)
        np.testing.assert_array_equal(P, Pa)


def test_serving_results_equal_alone(gpu):
    """Continuous batching: jobs of different sizes admitted as they arrive
    (and as memory frees) give, job by job, the result of running alone."""
    from src_b200.serving import MasterBunches, Server, run_alone
    from src_b200.workloads import Job

    rng = np.random.default_rng(7)
    jobs = [Job(i, 0.002 * i, int(rng.integers(10_000, 60_000)), int(rng.choice([16, 24, 32])),
                tuple(rng.uniform(0.5e-3, 3e-3, 3)), float(rng.uniform(2, 20)), float(rng.uniform(0.1, 2)),
                int(rng.integers(5, 40))) for i in range(10)]
    masters = MasterBunches(count=2, size=60_000)
    for prec in (gpu.PLAIN_FP64, gpu.MIXED):
        # a budget of about three jobs forces queueing and slot reuse
        budget = 3 * max(j.footprint_bytes(prec) for j in jobs)
        srv = Server(precision=prec, hbm_budget_bytes=budget, masters=masters, keep_results=True)
        try:
            res = srv.run(jobs, realtime=True)
        finally:
            srv.close()
        assert len(res) == len(jobs)
        for r in res:
            Ra, Pa = run_alone(r.job, prec, masters)
            np.testing.assert_array_equal(r.R, Ra)
            np.testing.assert_array_equal(r.P, Pa)


def test_batch_errors(gpu):
    with gpu.Batch() as bt:
        with pytest.raises(gpu.ScgpuError):
            bt.remove(3)
        with pytest.raises(gpu.ScgpuError):
            bt.member(0)
        assert bt.track(2) == 0.0  # an empty batch does nothing
