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


class StubEnsemble:
    """Stands in for Ensemble on CPU: deterministic per-instance results from
    the instance's own positions, so the gathered rows show which instances
    each rank ran."""

    def __init__(self, sd, configs, device=0):
        self.configs = configs

    def run(self, max_rounds=0):
        import types
        out = []
        for x, y in self.configs:
            out.append(types.SimpleNamespace(
                sim_time=float(np.sum(x)), step_size=1e-6, strain=float(np.sum(y)),
                successful_steps=len(x), failed_steps=max_rounds, attempts=len(x) + max_rounds,
                singular_factorizations=0, device_seconds=0.25))
        return out

    def positions(self, j):
        return self.configs[j]

    def close(self):
        pass


def _sharded_main(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    e = ens_mod()
    rng = np.random.default_rng(2000)
    ns = (rng.integers(2, 40, size=11) * 2).tolist()
    configs = [(np.random.default_rng(3000 + k).uniform(-0.5, 0.5, n),
                np.random.default_rng(4000 + k).uniform(-0.5, 0.5, n)) for k, n in enumerate(ns)]
    full, pos = e.run_sharded(None, configs, max_rounds=3, ensemble_cls=StubEnsemble)
    np.save(os.path.join(out_dir, "full%d.npy" % rank), full)
    np.save(os.path.join(out_dir, "mine%d.npy" % rank), np.array(sorted(pos)))
    dist.barrier()
    dist.destroy_process_group()


def test_run_sharded_two_gloo_ranks(tmp_path):
    """partition -> one ensemble per rank -> gather_results, composed by
    run_sharded: every rank ends with every instance's row, each computed by
    exactly the rank that owns the instance."""
    import torch.multiprocessing as mp
    e = ens_mod()
    port = _free_port()
    mp.start_processes(_sharded_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    f0, f1 = np.load(tmp_path / "full0.npy"), np.load(tmp_path / "full1.npy")
    assert np.array_equal(f0, f1)
    rng = np.random.default_rng(2000)
    ns = (rng.integers(2, 40, size=11) * 2).tolist()
    parts = e.partition(ns, 2)
    assert sorted(np.load(tmp_path / "mine0.npy").tolist()) == parts[0]
    assert sorted(np.load(tmp_path / "mine1.npy").tolist()) == parts[1]
    for k, n in enumerate(ns):
        x = np.random.default_rng(3000 + k).uniform(-0.5, 0.5, n)
        assert f0[k, 0] == np.sum(x) and f0[k, 3] == n and f0[k, 4] == 3
