"""Batched ensembles of independent systems (d4_ensemble_* of include/d4core.h).

The reference studies statistics over many realisations by running one
Simulation per process (src/simulation.cpp:30-281).  ``Ensemble`` advances
all realisations on one GPU together, every phase of the implicit step one
launch over all of them; each instance reproduces the single-system engine's
arithmetic.  Across GPUs the instances shard with no data-path exchange:
``partition`` splits them over ranks (one process per GPU) balancing the
dense-LU work, and ``gather_results`` collects the per-instance results on
every rank through ``torch.distributed`` (NCCL on GPUs, gloo on CPU).
"""
import ctypes as C

import numpy as np

from . import _lib


class Ensemble:
    """Instances share ``sd``'s parameters (protocol, precisions, limits,
    cutoff); ``configs`` is a list of (x, y) in internal order (b = +1 first),
    each of even length."""

    def __init__(self, sd, configs, device=0):
        self.lib = _lib.load()
        p = sd.to_params()
        p.device = device
        self.ns = [len(x) for x, _ in configs]
        n = (C.c_int * len(self.ns))(*self.ns)
        ens = C.c_void_p()
        st = self.lib.d4_ensemble_create(C.byref(ens), len(self.ns), n, C.byref(p))
        if st < 0:
            raise _lib.D4Error("d4_ensemble_create failed: %s" % _lib.D4_ERR.get(st, st))
        self.ens = ens
        for k, (x, y) in enumerate(configs):
            x = np.ascontiguousarray(x, dtype=np.float64)
            y = np.ascontiguousarray(y, dtype=np.float64)
            self._call("d4_ensemble_set_positions", C.c_int(k), _lib.ptr(x), _lib.ptr(y))

    def _call(self, name, *args):
        st = getattr(self.lib, name)(self.ens, *args)
        if st < 0:
            msg = self.lib.d4_ensemble_last_error(self.ens) or b""
            raise _lib.D4Error("%s failed: %s (%s)" % (name, _lib.D4_ERR.get(st, st),
                                                       msg.decode()))
        return st

    def run(self, max_rounds=0):
        """Attempt rounds until every instance is interrupted (or max_rounds
        rounds); returns the per-instance d4_run_result list."""
        res = (_lib.RunResult * len(self.ns))()
        self._call("d4_ensemble_run", C.c_longlong(max_rounds), res)
        return list(res)

    def positions(self, k):
        x, y = np.empty(self.ns[k]), np.empty(self.ns[k])
        self._call("d4_ensemble_get_positions", C.c_int(k), _lib.ptr(x), _lib.ptr(y))
        return x, y

    def close(self):
        if getattr(self, "ens", None):
            self.lib.d4_ensemble_destroy(self.ens)
            self.ens = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def partition(ns, world_size):
    """Instance indices per rank: longest-processing-time greedy on n^3 (the
    dense LU dominates an instance's step), ties to the lower rank; each
    rank's list is in ascending instance order."""
    load = [0.0] * world_size
    parts = [[] for _ in range(world_size)]
    for k in sorted(range(len(ns)), key=lambda k: (-ns[k], k)):
        r = min(range(world_size), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += float(ns[k]) ** 3
    return [sorted(p) for p in parts]


RESULT_FIELDS = ("sim_time", "step_size", "strain", "successful_steps", "failed_steps",
                 "attempts", "singular_factorizations", "device_seconds")


def results_array(results):
    """d4_run_result list -> float64 array (instances x RESULT_FIELDS)."""
    return np.array([[float(getattr(r, f)) for f in RESULT_FIELDS] for r in results],
                    dtype=np.float64).reshape(len(results), len(RESULT_FIELDS))


def gather_results(local_idx, local_rows, count, group=None):
    """All ranks' per-instance rows (results_array) assembled in instance
    order on every rank, with one all_reduce of a count x fields tensor (rows
    a rank does not own are zero, so the sum assembles disjoint parts)."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if (
        dist.get_backend(group) == "nccl") else torch.device("cpu")
    full = torch.zeros(count, len(RESULT_FIELDS), dtype=torch.float64, device=dev)
    if len(local_idx):
        full[torch.as_tensor(local_idx, dtype=torch.long, device=dev)] = torch.as_tensor(
            local_rows, dtype=torch.float64, device=dev)
    dist.all_reduce(full, group=group)
    return full.cpu().numpy()


def run_sharded(sd, configs, max_rounds=0, group=None, device=None, ensemble_cls=None):
    """The ensemble sharded over the ranks of a torch.distributed process group
    (one process per GPU): rank r runs the instances ``partition(ns, world)[r]``
    as one ``Ensemble`` on its own device, with no data-path exchange; at the
    end one all_reduce (``gather_results``) gives every rank every instance's
    results.  Returns (results rows in instance order, {instance: (x, y)} for
    this rank's instances).  Every rank makes the same collective call, also a
    rank that owns no instance.  ``ensemble_cls`` stands in for ``Ensemble``
    (same constructor, run, positions and close)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    ns = [len(x) for x, _ in configs]
    mine = partition(ns, world)[rank]
    if device is None:
        device = torch.cuda.current_device() if torch.cuda.is_available() else 0
    cls = ensemble_cls or Ensemble
    rows = np.zeros((0, len(RESULT_FIELDS)))
    positions = {}
    if mine:
        ens = cls(sd, [configs[k] for k in mine], device=device)
        try:
            rows = results_array(ens.run(max_rounds))
            positions = {k: ens.positions(j) for j, k in enumerate(mine)}
        finally:
            ens.close()
    return gather_results(mine, rows, len(ns), group), positions
