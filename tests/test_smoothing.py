"""Energy-conserving smoothing on the host: the oracle's pass against the
reference's own node_smoothing_value (ecsim/fields/node_smoothing.hpp:24-52,
compiled into the pin harness), its invariants, and the option checks of
tpicb200_create (config/physics.cpp:65-70), which reject before any device
work."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from fieldutil import periodic_node_field, smooth_random_unique
from reference_fixtures import ogrid
from tpic_b200 import _lib
from tpic_b200.plasma import GridSpec

GRID = GridSpec(6, 5, 4, 3.0, 2.5, 2.0)


@pytest.mark.parametrize("op,alpha", [(0, 0.5), (0, 0.0), (0, 0.875), (1, 0.5)])
def test_oracle_pass_equals_the_reference_operator(op, alpha):
    ref = O.load_reference()
    if ref is None or not hasattr(ref, "ref_smooth_node"):
        pytest.skip("reference pin harness not built")
    g = GRID
    rng = np.random.default_rng(3)
    f = periodic_node_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    lib = O.load()
    nodes = lib.oracle_node_count(C.byref(ogrid(g)))
    comp = np.ascontiguousarray(f[:nodes])
    for (i, j, k) in [(0, 0, 0), (g.nx, g.ny, g.nz), (3, 2, 1), (5, 4, 3), (0, 4, 2)]:
        want = ref.ref_smooth_node(g.nx, g.ny, op, alpha, O.ptr(comp), i, j, k)
        got = lib.oracle_smooth_node(C.byref(ogrid(g)), op, alpha, O.ptr(comp), i, j, k)
        assert got == want  # bit for bit: same operations in the same order


def smoothed(g, field, niter, alpha, op):
    out = np.zeros_like(field)
    O.load().oracle_smooth(C.byref(ogrid(g)), niter, alpha, op, O.ptr(field), O.ptr(out))
    return out


@pytest.mark.parametrize("op", [0, 1])
def test_oracle_smoothing_invariants(op):
    g = GRID
    rng = np.random.default_rng(5)
    f = periodic_node_field(g, smooth_random_unique(g, rng, 1.0))
    nodes = len(f) // 3
    const = np.full_like(f, 2.5)
    # Weights sum to one: a constant field is unchanged; Face7 with alpha 1 is the identity.
    assert np.allclose(smoothed(g, const, 3, 0.5, op), 2.5, rtol=0, atol=1e-15)
    if op == 0:
        assert np.array_equal(smoothed(g, f, 2, 1.0, 0), f)
    # Linear, and the mean over the unique nodes is conserved.
    a, b = smoothed(g, f, 2, 0.5, op), smoothed(g, 3.0 * f, 2, 0.5, op)
    assert np.allclose(b, 3.0 * a, rtol=1e-14, atol=1e-14)
    from fieldutil import interior_nodes
    u0, u1 = interior_nodes(g, f)[:, :-1, :-1, :-1], interior_nodes(g, a)[:, :-1, :-1, :-1]
    assert np.allclose(u0.sum(axis=(1, 2, 3)), u1.sum(axis=(1, 2, 3)), rtol=1e-12, atol=1e-12)
    # It damps: the variance of the unique nodes drops.
    assert u1.var() < u0.var()
    assert nodes > 0


@pytest.mark.parametrize("iters,alpha,op", [(-1, 0.5, 0), (2, 1.5, 0), (2, -0.1, 0), (2, float("nan"), 0),
                                            (2, 0.5, 7)])
def test_create_rejects_invalid_smoothing(iters, alpha, op):
    lib = _lib.load()
    grid = _lib.Grid(4, 4, 4, 1.0, 1.0, 1.0)
    opts = _lib.Options(0.1, 0.5, 1.0, 1e-8, 30, 100, 0, 1024, 1, iters, alpha, op)
    h = C.c_void_p()
    assert lib.tpicb200_create(C.byref(grid), C.byref(opts), C.byref(h)) == _lib.INVALID_ARGUMENT
    assert b"smoothing" in lib.tpicb200_last_error()
