"""Host side of the sharded bunch, on CPU: the exchange arithmetic and its
torch.distributed (gloo, world size 2) path, and the 128-bit limb encoding
the library uses for exact sums (sc_particles.cu put_limbs / get_limbs)."""
import os
import socket

import numpy as np
import pytest


def _limbs(v):
    u = v % (1 << 128)
    return np.array([(u >> (32 * j)) & 0xFFFFFFFF for j in range(4)], dtype=np.uint64)


def _unlimbs(a):
    u = sum(int(a[j]) << (32 * j) for j in range(4)) % (1 << 128)
    return u - (1 << 128) if u >= (1 << 127) else u


def test_limb_sums_are_exact():
    from src_b200.sharding import SUM_U64, combine
    rng = np.random.default_rng(4)
    for _ in range(200):
        vals = [int(rng.integers(-(1 << 62), 1 << 62)) * int(rng.integers(1, 1 << 40)) for _ in range(5)]
        total = combine([_limbs(v) for v in vals], SUM_U64)
        assert _unlimbs(total) == sum(vals)


def test_min_combine():
    from src_b200.sharding import MIN_F64, combine
    a = np.array([1.0, -2.0, np.inf, -0.0])
    b = np.array([0.5, 3.0, 7.0, 0.0])
    np.testing.assert_array_equal(combine([a, b], MIN_F64), [0.5, -2.0, 7.0, -0.0])


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from src_b200.sharding import MIN_F64, SUM_U64, TorchExchange

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ex = TorchExchange()
        s = ex.combine_host(np.array([2**63 + rank, 5 + rank, 2**64 - 1], dtype=np.uint64), SUM_U64)
        m = ex.combine_host(np.array([float(rank), -float(rank), 3.0]), MIN_F64)
        np.savez(os.path.join(out, f"r{rank}.npz"), s=s, m=m)
    finally:
        dist.destroy_process_group()


def test_torch_exchange_gloo_world_size_2(tmp_path):
    import torch.multiprocessing as mp
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        d = np.load(tmp_path / f"r{r}.npz")
        np.testing.assert_array_equal(d["s"], np.array([1, 11, 2**64 - 2], dtype=np.uint64))
        np.testing.assert_array_equal(d["m"], [0.0, -1.0, 3.0])
