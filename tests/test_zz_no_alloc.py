"""tpicb200_sort_static: the context-free sort on the library's fixed
scratch array, called through the C ABI twice in a row and compared with
tpicb200_sort (the context's sort) on the same records; both are exact
integer reorderings, so the comparison is bit for bit. Also the capacity
checks, which reject oversized inputs before any device work."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tpic_b200 import _lib
from tpic_b200.plasma import GridSpec

pytestmark = pytest.mark.gpu


def records(g, n, seed, precision):
    rng = np.random.default_rng(seed)
    vdt = np.float64 if precision == 0 else np.float32
    keys = g.encode(rng.integers(0, g.nx, n), rng.integers(0, g.ny, n), rng.integers(0, g.nz, n)).astype(np.int32)
    idx = np.arange(n)
    return {"rx": rng.random(n), "ry": rng.random(n), "rz": rng.random(n), "u": (idx * 0.5).astype(vdt),
            "v": (idx * -0.25).astype(vdt), "w": rng.normal(size=n).astype(vdt), "q": idx * 2.0, "cell": keys,
            "id": (idx + 7).astype(np.uint64)}


@pytest.mark.parametrize("precision", [0, 1])
def test_static_sort_matches_the_context_sort_twice(torch_cuda, precision):
    from gpu_helpers import StageContext
    g = GridSpec(12, 10, 9, 1.0, 1.0, 1.0)
    ctx = StageContext(g, precision, max_particles=200000)
    lib = ctx.lib
    grid = _lib.Grid(g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)
    invalid = torch_cuda.zeros(1, dtype=torch_cuda.int32, device="cuda")
    for call, (n, seed) in enumerate([(150000, 1), (90001, 2)]):
        d = records(g, n, seed, precision)
        src = ctx.upload_particles(d)
        want, wc, wo = ctx.sort(src, n, with_id=True)
        dst = ctx.empty_particles(n, True)
        counts = torch_cuda.full((ctx.layout.bin_count,), 7, dtype=torch_cuda.int32, device="cuda")
        offsets = torch_cuda.full((ctx.layout.bin_count + 1,), 7, dtype=torch_cuda.int32, device="cuda")
        pin, pout = ctx.struct(src, n), ctx.struct(dst, n)
        _lib.check(lib.tpicb200_sort_static(C.byref(grid), precision, C.byref(pin), C.byref(pout), counts.data_ptr(),
                                            offsets.data_ptr(), invalid.data_ptr(), ctx.stream))
        torch_cuda.cuda.synchronize()
        got, ref = ctx.download(dst, n), ctx.download(want, n)
        assert np.array_equal(counts.cpu().numpy(), wc.cpu().numpy()), call
        assert np.array_equal(offsets.cpu().numpy(), wo.cpu().numpy()), call
        for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell", "id"):
            assert np.array_equal(got[k], ref[k]), (call, k)
    assert int(invalid.item()) == 0 and ctx.invalid_count() == 0


def test_static_sort_rejects_oversized_inputs(torch_cuda):
    lib = _lib.load()
    big = GridSpec(100, 100, 100, 1.0, 1.0, 1.0)  # 104^3 halo-2 bins > 1048576
    grid = _lib.Grid(big.nx, big.ny, big.nz, 1.0, 1.0, 1.0)
    p = _lib.Particles()
    p.count = 10
    out = _lib.Particles()
    dummy = torch_cuda.zeros(8, dtype=torch_cuda.int32, device="cuda")
    status = lib.tpicb200_sort_static(C.byref(grid), 1, C.byref(p), C.byref(out), dummy.data_ptr(),
                                      dummy.data_ptr(), None, None)
    assert status == _lib.CAPACITY_EXCEEDED
    assert "TPICB200_SORT_STATIC_MAX_BINS" in lib.tpicb200_last_error().decode()
    small = _lib.Grid(4, 4, 4, 1.0, 1.0, 1.0)
    p.count = 1048577
    status = lib.tpicb200_sort_static(C.byref(small), 1, C.byref(p), C.byref(out), dummy.data_ptr(),
                                      dummy.data_ptr(), None, None)
    assert status == _lib.CAPACITY_EXCEEDED
    assert "TPICB200_SORT_STATIC_MAX_RECORDS" in lib.tpicb200_last_error().decode()
