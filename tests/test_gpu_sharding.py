"""A bunch sharded over ranks (scgpu_set_exchange) evolves bitwise as the
whole bunch in one context: bounds combine by min, and the deposit's node
sums and the momentum / moment sums are exact integers, so no result depends
on which rank holds which particle.

Only one GPU is available to these tests: the ranks are host threads with one
context each (HostExchange), two processes on the same GPU that exchange
through gloo (TorchExchange), or one rank of an NCCL group (TorchExchange's
device all-reduces).  No kernel waits on another rank; the ranks
meet on the host between kernels.
"""
import os
import threading

import numpy as np
import pytest

from src_b200.bunch import gaussian_bunch

pytestmark = pytest.mark.gpu

MASS = 0.51099892e6


def _single(gpu, R, P, nr, steps, Q):
    with gpu.Context(nr) as c:
        c.set_reorder_interval(7)
        c.upload(R, P, 1e-12, Q, MASS)
        stats = np.zeros((steps, gpu.NSTATS))
        c.track(steps, stats)
        Rg, Pg = c.download()
        return Rg, Pg, c.tracker_state(), c.beam_parameters(), stats, c.stat_row()


def _sharded(gpu, R, P, nr, steps, Q, bounds):
    from src_b200.sharding import HostExchange, attach

    nranks = len(bounds) - 1
    ex = HostExchange(nranks)
    out = [None] * nranks
    errors = []

    def rank(r):
        try:
            lo, hi = bounds[r], bounds[r + 1]
            with gpu.Context(nr) as c:
                attach(c, ex.callback(r), R.shape[0])
                c.set_reorder_interval(5)  # the shards reorder at other steps than the whole bunch
                c.upload(R[lo:hi], P[lo:hi], 1e-12, Q, MASS)
                stats = np.zeros((steps, gpu.NSTATS))
                c.track(steps, stats)
                Rg, Pg = c.download()
                out[r] = (Rg, Pg, c.tracker_state(), c.beam_parameters(), stats, c.stat_row())
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    threads = [threading.Thread(target=rank, args=(r,)) for r in range(nranks)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not errors, errors
    return out


@pytest.mark.parametrize("N,nr,steps,cuts", [(40_000, (32, 32, 32), 20, (0, 20_000, 40_000)),
                                              (30_001, (16, 24, 32), 5, (0, 7_000, 19_999, 30_001))])
def test_shards_equal_whole_bunch(gpu, N, nr, steps, cuts):
    R, P = gaussian_bunch(N, bunch_id=8)
    Q = -1e-9 / N
    Rs, Ps, st, bp, stats, row = _single(gpu, R, P, nr, steps, Q)
    parts = _sharded(gpu, R, P, nr, steps, Q, cuts)
    np.testing.assert_array_equal(np.concatenate([p[0] for p in parts]), Rs)
    np.testing.assert_array_equal(np.concatenate([p[1] for p in parts]), Ps)
    for Rg, Pg, st_r, bp_r, stats_r, row_r in parts:
        assert st_r["path_length"] == st["path_length"] and st_r["q_macro"] == st["q_macro"]
        np.testing.assert_array_equal(stats_r, stats)  # per-step moment sums of the whole bunch
        for k in ("rmean", "rrms", "prms", "eps_norm", "moments"):
            np.testing.assert_array_equal(bp_r[k], bp[k])
        # the statistics row (all but the particle-0 columns) is the whole bunch's
        np.testing.assert_array_equal(row_r[:42], row[:42])


def _gloo_rank(rank, world, port, path, backend="gloo"):
    import datetime

    import torch
    import torch.distributed as dist
    from src_b200 import scgpu
    from src_b200.sharding import TorchExchange, attach

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(0)
        kw["device_id"] = torch.device("cuda", 0)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120), **kw)
    try:
        d = np.load(path)
        R, P, cuts = d["R"], d["P"], d["cuts"]
        ex = TorchExchange()
        with scgpu.Context((16, 16, 16)) as c:
            attach(c, ex.callback(), R.shape[0])
            lo, hi = int(cuts[rank]), int(cuts[rank + 1])
            c.upload(R[lo:hi], P[lo:hi], 1e-12, -1e-9 / R.shape[0], MASS)
            c.track(6)
            Rg, Pg = c.download()
        np.savez(path.replace(".npz", f"_r{rank}.npz"), R=Rg, P=Pg)
    finally:
        dist.destroy_process_group()


def test_two_processes_over_gloo(gpu, tmp_path):
    import socket

    import torch.multiprocessing as mp

    N = 20_000
    R, P = gaussian_bunch(N, bunch_id=9)
    Rs, Ps, *_ = _single(gpu, R, P, (16, 16, 16), 6, -1e-9 / N)
    path = str(tmp_path / "bunch.npz")
    np.savez(path, R=R, P=P, cuts=np.array([0, 11_000, N]))
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_gloo_rank, args=(2, port, path), nprocs=2, start_method="spawn", join=True)
    parts = [np.load(path.replace(".npz", f"_r{r}.npz")) for r in range(2)]
    np.testing.assert_array_equal(np.concatenate([p["R"] for p in parts]), Rs)
    np.testing.assert_array_equal(np.concatenate([p["P"] for p in parts]), Ps)


def test_one_rank_over_nccl(gpu, tmp_path):
    """TorchExchange's NCCL branch on the hardware: one rank of an NCCL
    process group (the only GPU these tests have) runs the exchanges -- the
    bounds' min and the exact integer sums as device all-reduces on the
    context's stream -- and must give the single context's bits."""
    import socket

    import torch.multiprocessing as mp

    N = 20_000
    R, P = gaussian_bunch(N, bunch_id=10)
    Rs, Ps, *_ = _single(gpu, R, P, (16, 16, 16), 6, -1e-9 / N)
    path = str(tmp_path / "bunch.npz")
    np.savez(path, R=R, P=P, cuts=np.array([0, N]))
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_gloo_rank, args=(1, port, path, "nccl"), nprocs=1, start_method="spawn", join=True)
    d = np.load(path.replace(".npz", "_r0.npz"))
    np.testing.assert_array_equal(d["R"], Rs)
    np.testing.assert_array_equal(d["P"], Ps)


def test_shard_limits(gpu):
    from src_b200.sharding import HostExchange, attach

    R, P = gaussian_bunch(2000)
    with gpu.Context((16, 16, 16)) as c:
        attach(c, HostExchange(1).callback(0), 2000)
        c.upload(R, P, 1e-12, -1e-12, MASS)
        with pytest.raises(gpu.ScgpuError) as e:
            c.profile(1)
        assert e.value.code == -8
        with pytest.raises(gpu.ScgpuError) as e:
            c.set_energy_bins(np.zeros(2000, np.int32), 2)
        assert e.value.code == -8
        c.track(2)  # one rank: the plain step through the exchange
