"""Host logic of the ensemble's multi-GPU sharding (no GPU): the partition of
instances over ranks and the end-of-run gather of per-instance results, run
as two gloo ranks on 127.0.0.1."""
import os
import socket

import numpy as np
import pytest


def ens_mod():
    import importlib
    return importlib.import_module("2d4_b200.ensemble")


def test_partition_covers_and_balances():
    e = ens_mod()
    rng = np.random.default_rng(2000)
    ns = (rng.integers(32, 1025, size=512) * 2).tolist()  # even N in [64, 2048]
    for world in (1, 2, 4, 8):
        parts = e.partition(ns, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(ns)))
        loads = [sum(float(ns[k]) ** 3 for k in p) for p in parts]
        # LPT greedy: within one largest job of the mean
        assert max(loads) - min(loads) <= max(float(n) ** 3 for n in ns) + 1e-6
        assert all(p == sorted(p) for p in parts)
    assert e.partition([64, 64], 4)[2:] == [[], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, ns, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    e = ens_mod()
    mine = e.partition(ns, world)[rank]
    # stand-in results: a row per owned instance derived from its index
    rows = np.array([[k + 0.5, 1e-3 * k, 0.0, k, 2 * k, 3 * k, 0, rank] for k in mine],
                    dtype=np.float64).reshape(len(mine), len(e.RESULT_FIELDS))
    full = e.gather_results(mine, rows, len(ns))
    np.save(os.path.join(out_dir, "rank%d.npy" % rank), full)
    dist.barrier()
    dist.destroy_process_group()


def test_gather_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    e = ens_mod()
    ns = [64, 2048, 1000, 500, 1500, 64, 128, 256, 96]
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, ns, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    a0 = np.load(tmp_path / "rank0.npy")
    a1 = np.load(tmp_path / "rank1.npy")
    assert np.array_equal(a0, a1)
    owner = {k: r for r, p in enumerate(e.partition(ns, 2)) for k in p}
    for k in range(len(ns)):
        assert a0[k, 0] == k + 0.5 and a0[k, 3] == k and a0[k, 7] == owner[k]
