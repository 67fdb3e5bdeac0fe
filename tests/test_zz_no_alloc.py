"""The allocation-free stress sweep, d4_speeds_noalloc (marked gpu).

It exists for callers that cannot allocate device memory (code running under
CUDA-graph stream capture, real-time loops that must not wait on an allocator,
hosts whose device memory belongs to another framework).  Its scratch is a
fixed 8 MiB device array inside the library, so it takes n <= 1024.  This test
calls it through the C ABI with device buffers owned by the caller and checks
two calls in a row against the regular entry point d4_speeds, with the
tolerance of the other GPU tests.  The second call uses a smaller n, so it runs
on scratch that still holds the first call's values.  This file is named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def regular_speeds(pkg, x, y, precision):
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.precision = precision
    eng = pkg.Engine(sd)
    v, tol = eng.speeds(x, y, 0.0)
    eng.close()
    return v, tol


def test_speeds_noalloc_matches_speeds(pkg):
    import torch

    lib = pkg._lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    precision = 1e-5
    min_prec_sq = precision * precision / (0.05 * 0.05)  # -P 1e-5 -p 0.05
    cases = [(1024, 1001), (512, 77)]
    expected = [regular_speeds(pkg, *pkg.dconf.generate_internal(n, s)[:2], precision)
                for n, s in cases]
    bufs = []
    for n, s in cases:
        x, y, _ = pkg.dconf.generate_internal(n, s)
        bufs.append((torch.from_numpy(x).to(dev), torch.from_numpy(y).to(dev),
                     torch.empty(n, dtype=torch.float64, device=dev),
                     torch.full((n,), min_prec_sq, dtype=torch.float64, device=dev)))
    torch.cuda.synchronize()
    allocs_before = lib.d4_device_allocations()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for (n, _), (xd, yd, vd, td), (v_ref, tol_ref) in zip(cases, bufs, expected):
        st = lib.d4_speeds_noalloc(n, xd.data_ptr(), yd.data_ptr(), C.c_double(0.0),
                                   vd.data_ptr(), td.data_ptr(), C.c_double(min_prec_sq), None)
        assert st == 0
        torch.cuda.synchronize()
        v = vd.cpu().numpy()
        assert rel_err(v, v_ref) < 1e-11
        assert np.array_equal(td.cpu().numpy(), tol_ref)
    # nothing allocated: the library's own allocation counter is unchanged;
    # the device's free memory, which other processes and lazily loaded
    # modules can also change, is a secondary check within 2 MiB
    assert lib.d4_device_allocations() == allocs_before
    assert abs(torch.cuda.mem_get_info(dev)[0] - free_before) <= 2 * 1024 * 1024


def test_speeds_noalloc_rejects_sizes(pkg):
    lib = pkg._lib.load()
    import torch
    x = torch.zeros(1026, dtype=torch.float64, device="cuda")
    for n in (1026, 63, 0):
        assert lib.d4_speeds_noalloc(n, x.data_ptr(), x.data_ptr(), C.c_double(0.0),
                                     x.data_ptr(), None, C.c_double(0.0), None) == -1
