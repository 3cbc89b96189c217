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


RESET_SCRIPT = r'''
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from tpic_b200 import _lib
from tpic_b200.plasma import GridSpec

lib = _lib.load()
rt = C.CDLL("libcudart.so.12")
H2D, D2H = 1, 2
g = GridSpec(10, 9, 8, 1.0, 1.0, 1.0)
grid = _lib.Grid(g.nx, g.ny, g.nz, 1.0, 1.0, 1.0)
bins = (g.nx + 4) * (g.ny + 4) * (g.nz + 4)


def dalloc(nbytes):
    ptr = C.c_void_p()
    assert rt.cudaMalloc(C.byref(ptr), C.c_size_t(max(nbytes, 8))) == 0
    return ptr


def run(n, seed):
    rng = np.random.default_rng(seed)
    keys = g.encode(rng.integers(0, g.nx, n), rng.integers(0, g.ny, n), rng.integers(0, g.nz, n)).astype(np.int32)
    host = {"rx": rng.random(n), "ry": rng.random(n), "rz": rng.random(n), "u": rng.random(n).astype(np.float32),
            "v": rng.random(n).astype(np.float32), "w": rng.random(n).astype(np.float32), "q": rng.random(n),
            "cell": keys}
    src, dst = _lib.Particles(), _lib.Particles()
    outs = {}
    for k, a in host.items():
        d = dalloc(a.nbytes)
        assert rt.cudaMemcpy(d, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes), H2D) == 0
        setattr(src, k, d.value)
        o = dalloc(a.nbytes)
        setattr(dst, k, o.value)
        outs[k] = o
    src.count = n
    counts, offsets = dalloc(4 * bins), dalloc(4 * (bins + 1))
    status = lib.tpicb200_sort_static(C.byref(grid), 1, C.byref(src), C.byref(dst), counts, offsets, None, None)
    assert status == 0, lib.tpicb200_last_error()
    assert rt.cudaDeviceSynchronize() == 0
    order = np.argsort(keys, kind="stable")
    for k, o in outs.items():
        got = np.empty_like(host[k])
        assert rt.cudaMemcpy(got.ctypes.data_as(C.c_void_p), o, C.c_size_t(got.nbytes), D2H) == 0
        assert np.array_equal(got, host[k][order]), k
    got = np.empty(bins + 1, dtype=np.uint32)
    assert rt.cudaMemcpy(got.ctypes.data_as(C.c_void_p), offsets, C.c_size_t(got.nbytes), D2H) == 0
    assert np.array_equal(got, np.concatenate([[0], np.cumsum(np.bincount(keys, minlength=bins))]))


run(70000, 5)
assert rt.cudaDeviceReset() == 0  # ends this process's context; the next call runs in a new one
run(50001, 6)
print("ok")
'''


def test_static_sort_after_a_device_reset(torch_cuda, tmp_path):
    """The scratch array's address is per CUDA context. After cudaDeviceReset
    the next call runs in a new primary context and must resolve the address
    there again rather than reuse the old one (fresh process; the buffers are
    allocated by the test, the sort itself allocates nothing)."""
    import subprocess
    import sys
    from pathlib import Path
    script = tmp_path / "reset.py"
    script.write_text(RESET_SCRIPT)
    root = str(Path(__file__).resolve().parents[1])
    done = subprocess.run([sys.executable, str(script), root], capture_output=True, text=True, timeout=300)
    assert done.returncode == 0 and done.stdout.strip().endswith("ok"), done.stdout + done.stderr
