"""tpicb200_sort_binned: the post-mover sort of records grouped by the bins of
an earlier sort. Its output, counts and offsets must be bit-identical to the
stable host sort (lpfx/algorithm/particle/host/sort.hpp:205-290, restated in
the oracle) on every input: neighbour moves (transfer-count path), far moves,
bins that do not describe the input, invalid keys and small grids (general
path)."""
from __future__ import annotations

import numpy as np
import pytest

from tpic_b200.plasma import GridSpec
from reference_fixtures import oracle_sort
from test_gpu_stages import make_ctx

pytestmark = pytest.mark.gpu


def grouped_records(g, rng, mean_ppc, precision):
    """Records sorted by cell (random counts per interior cell) with
    distinguishable attributes."""
    counts = rng.poisson(mean_ppc, g.cells)
    cell = np.repeat(np.arange(g.cells), counts)
    i, j, k = cell % g.nx, (cell // g.nx) % g.ny, cell // (g.nx * g.ny)
    keys = g.encode(i, j, k).astype(np.int32)
    n = len(keys)
    vdt = np.float64 if precision == 0 else np.float32
    idx = np.arange(n)
    d = {"rx": idx * 0.125, "ry": idx * -0.25, "rz": idx * 0.5, "u": (idx * -0.5).astype(vdt),
         "v": (idx * 0.25).astype(vdt), "w": (idx * -0.125).astype(vdt), "q": idx * 2.0, "cell": keys,
         "id": (idx + 100).astype(np.uint64)}
    return d, (i, j, k)


def move(g, rng, ijk, fraction, reach=1):
    i, j, k = ijk
    n = len(i)
    moved = rng.random(n) < fraction
    step = lambda: np.where(moved, rng.integers(-reach, reach + 1, n), 0)
    return g.encode((i + step()) % g.nx, (j + step()) % g.ny, (k + step()) % g.nz).astype(np.int32)


def check(g, ctx, d, n, in_counts, in_offsets, alias=False):
    src = ctx.upload_particles(d)
    dst, counts, offsets = ctx.sort_binned(src, n, in_counts, in_offsets, with_id=True, alias=alias)
    got = ctx.download(dst, n)
    perm, wc, wo = oracle_sort(g, d["cell"])
    assert np.array_equal(counts.cpu().numpy().view(np.uint32), wc)
    assert np.array_equal(offsets.cpu().numpy().view(np.uint32), wo)
    for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell", "id"):
        assert np.array_equal(got[k], d[k][perm]), k
    return got


def old_bins(ctx, g, d):
    """Bins of the unmoved records from the general sort."""
    src = ctx.upload_particles(d)
    _, counts, offsets = ctx.sort(src, len(d["cell"]), with_id=True)
    return counts, offsets


@pytest.mark.parametrize("precision,alias", [(0, False), (1, False), (1, True)])
def test_binned_sort_neighbour_moves(torch_cuda, precision, alias):
    g = GridSpec(8, 7, 6, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(11 + precision)
    d, ijk = grouped_records(g, rng, 40, precision)
    n = len(d["cell"])
    ctx = make_ctx(g, precision, max_particles=n)
    counts, offsets = old_bins(ctx, g, d)
    d["cell"] = move(g, rng, ijk, 0.3)
    check(g, ctx, d, n, counts, offsets, alias=alias)
    assert ctx.invalid_count() == 0


def test_binned_sort_every_record_moves_across_the_periodic_faces(torch_cuda):
    g = GridSpec(3, 4, 5, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(3)
    d, ijk = grouped_records(g, rng, 60, 1)
    n = len(d["cell"])
    ctx = make_ctx(g, 1, max_particles=n)
    counts, offsets = old_bins(ctx, g, d)
    d["cell"] = move(g, rng, ijk, 1.0)
    check(g, ctx, d, n, counts, offsets, alias=True)


def test_binned_sort_far_moves_take_the_general_path(torch_cuda):
    g = GridSpec(8, 8, 8, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(5)
    d, ijk = grouped_records(g, rng, 20, 1)
    n = len(d["cell"])
    ctx = make_ctx(g, 1, max_particles=n)
    counts, offsets = old_bins(ctx, g, d)
    keys = move(g, rng, ijk, 0.2)
    far = rng.integers(0, n, 5)
    keys[far] = g.encode(np.full(5, 4), np.full(5, 4), np.full(5, 4))  # several cells away for most
    d["cell"] = keys
    check(g, ctx, d, n, counts, offsets)


def test_binned_sort_bins_that_do_not_describe_the_input(torch_cuda):
    g = GridSpec(6, 6, 6, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(7)
    d, ijk = grouped_records(g, rng, 10, 0)
    n = len(d["cell"])
    ctx = make_ctx(g, 0, max_particles=n)
    import torch
    zeros = torch.zeros(ctx.layout.bin_count, dtype=torch.int32, device="cuda")
    zeros1 = torch.zeros(ctx.layout.bin_count + 1, dtype=torch.int32, device="cuda")
    d["cell"] = move(g, rng, ijk, 0.5)
    check(g, ctx, d, n, zeros, zeros1)
    # Shifted bins: the ranges no longer tile the records.
    counts, offsets = old_bins(ctx, g, d)
    offsets = offsets.clone()
    offsets[5] += 3
    check(g, ctx, d, n, counts, offsets)


def test_binned_sort_invalid_key_reported(torch_cuda):
    g = GridSpec(4, 4, 4, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(9)
    d, ijk = grouped_records(g, rng, 4, 0)
    n = len(d["cell"])
    ctx = make_ctx(g, 0, max_particles=n)
    counts, offsets = old_bins(ctx, g, d)
    keys = move(g, rng, ijk, 0.2)
    keys[n // 2] = -1
    d["cell"] = keys
    src = ctx.upload_particles(d)
    ctx.sort_binned(src, n, counts, offsets, with_id=True)
    assert ctx.invalid_count() == 1


@pytest.mark.parametrize("shape", [(2, 5, 5), (1, 1, 1)])
def test_binned_sort_small_grids(torch_cuda, shape):
    g = GridSpec(*shape, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(13)
    d, ijk = grouped_records(g, rng, 30, 1)
    n = len(d["cell"])
    ctx = make_ctx(g, 1, max_particles=n)
    counts, offsets = old_bins(ctx, g, d)
    d["cell"] = move(g, rng, ijk, 0.5)
    check(g, ctx, d, n, counts, offsets)


def test_binned_sort_empty(torch_cuda):
    g = GridSpec(4, 4, 4, 1.0, 1.0, 1.0)
    ctx = make_ctx(g, 0, max_particles=1)
    import torch
    counts = torch.zeros(ctx.layout.bin_count, dtype=torch.int32, device="cuda")
    offsets = torch.zeros(ctx.layout.bin_count + 1, dtype=torch.int32, device="cuda")
    src = ctx.empty_particles(0, True)
    _, c2, o2 = ctx.sort_binned(src, 0, counts, offsets, with_id=True)
    assert int(c2.sum()) == 0 and int(o2.abs().sum()) == 0
    assert ctx.invalid_count() == 0
