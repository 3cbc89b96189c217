"""The tiled mass layout and the operator apply that stages mass rows by TMA.

The tiled layout (TPICB200_MASS_LAYOUT_TILED) is the stencil-major layout
with each x row of a mass plane padded to a multiple of 4 vertices, so that
every row starts on a 16-byte boundary. The Maxwell operator apply then reads
the mass through 4-D tensor-memory-access boxes (one per stencil, streamed
through shared memory) instead of per-thread loads. Both applies form every
product and sum in the same order, so a field solve, and the adjoint's
transposed solve, on the same mass agree BIT FOR BIT between

- a stencil-major context whose x extent (nx + 3) is not a multiple of 4
  (the per-thread-load apply), and
- a tiled context on the same inputs (the TMA apply).

Grids cover partial tiles on every axis (12 x 10 x 8, 38 x 9 x 5) and the
thin tile of grids one cell deep along z (256 x 296 x 1). The tiled
deposition and cycle are checked against the oracle beside the other layouts
(test_gpu_stages.py, test_gpu_cycle.py).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from fieldutil import periodic_cell_field, periodic_node_field, smooth_random_unique
from reference_fixtures import periodic_node_field_records
from tpic_b200 import _lib
from tpic_b200.plasma import GridSpec

pytestmark = pytest.mark.gpu

GRIDS = {
    "partial3d": GridSpec(12, 10, 8, 3.0, 2.5, 2.0),
    "ragged3d": GridSpec(38, 9, 5, 7.6, 1.8, 1.0),
    "thin": GridSpec(256, 296, 1, 25.6, 29.6, 0.1),
}


def contexts(g, precision, dt=0.2, tol=1e-10):
    from gpu_helpers import StageContext
    assert (g.nx + 3) % 4 != 0  # the stencil-major context takes the per-thread-load apply
    return (StageContext(g, precision=precision, dt=dt, tol=tol, mass_layout=1),
            StageContext(g, precision=precision, dt=dt, tol=tol, mass_layout=2))


def random_mass(g, rng, dt=0.2, theta=0.5):
    """Mass records small enough that A = I + d^2 C2N N2C + (k/V) M stays
    near the identity (GMRES converges in a few iterations)."""
    volume = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    kfac = 4 * math.pi * theta * dt
    unique = 0.02 * volume / kfac * rng.normal(size=(126, g.nz, g.ny, g.nx))
    return periodic_node_field_records(g, unique)


def solve_inputs(g, rng):
    e = periodic_node_field(g, smooth_random_unique(g, rng, 0.01))
    b = periodic_cell_field(g, smooth_random_unique(g, rng, 0.05))
    j = periodic_node_field(g, smooth_random_unique(g, rng, 0.02))
    return e, b, j


def solve_backward(ctx, mass, etheta_bar):
    import torch
    nodes, cells = ctx.layout.node_count, ctx.layout.cell_count
    lam = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    e_bar = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    b_bar = torch.zeros(3 * cells, dtype=torch.float64, device="cuda")
    res = _lib.GmresResult()
    _lib.check(ctx.lib.tpicb200_field_solve_backward(ctx.ctx, mass.data_ptr(), etheta_bar.data_ptr(), lam.data_ptr(),
                                                     e_bar.data_ptr(), b_bar.data_ptr(), C.byref(res), ctx.stream))
    torch.cuda.synchronize()
    return lam, e_bar, b_bar, res


def assert_same_result(a, b):
    assert a.converged == b.converged == 1
    assert a.iterations == b.iterations
    assert a.residual == b.residual and a.relative_residual == b.relative_residual


@pytest.mark.parametrize("name", sorted(GRIDS))
@pytest.mark.parametrize("precision", [0, 1])
def test_tiled_solve_equals_stencil_major(torch_cuda, name, precision):
    import torch
    g = GRIDS[name]
    rng = np.random.default_rng(17)
    sm, tl = contexts(g, precision)
    m = random_mass(g, rng)
    e, b, j = solve_inputs(g, rng)
    et_sm, res_sm = sm.field_solve(sm.field(e), sm.field(b), sm.field(j), sm.mass_from_records(m))
    et_tl, res_tl = tl.field_solve(tl.field(e), tl.field(b), tl.field(j), tl.mass_from_records(m))
    torch.cuda.synchronize()
    assert_same_result(res_sm, res_tl)
    assert torch.equal(et_sm, et_tl)
    # The adjoint's transposed solve (every mass block transposed).
    etheta_bar = torch.from_numpy(periodic_node_field(g, smooth_random_unique(g, rng, 1.0))).cuda()
    got_sm = solve_backward(sm, sm.mass_from_records(m), etheta_bar)
    got_tl = solve_backward(tl, tl.mass_from_records(m), etheta_bar)
    assert_same_result(got_sm[3], got_tl[3])
    for x, y in zip(got_sm[:3], got_tl[:3]):
        assert torch.equal(x, y)
    assert sm.invalid_count() == 0 and tl.invalid_count() == 0
    sm.close()
    tl.close()


def test_tiled_layout_size(torch_cuda):
    from gpu_helpers import StageContext
    g = GRIDS["ragged3d"]
    ctx = StageContext(g, precision=0, mass_layout=2)
    mx = (g.nx + 3 + 3) // 4 * 4
    assert ctx.layout.mass_count == 126 * mx * (g.ny + 3) * (g.nz + 3)
    ctx.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_tiled_solve_of_a_deposited_mass_matches_the_oracle(torch_cuda, precision):
    """The TMA apply inside GMRES on the oracle's deposited mass: the solve
    converges in the oracle's iteration count to the oracle's field."""
    from test_gpu_stages import prepared_oracle
    from fieldutil import interior_nodes
    g = GRIDS["partial3d"]
    oc = prepared_oracle(g, 0)
    rng = np.random.default_rng(4)
    oc.e = periodic_node_field(g, smooth_random_unique(g, rng, 0.01))
    bcell = periodic_cell_field(g, smooth_random_unique(g, rng, 0.05))
    oc.b = bcell
    _, tl = contexts(g, precision)
    et, res = tl.field_solve(tl.field(oc.e), tl.field(bcell), tl.field(oc.j), tl.mass_from_records(oc.m))
    ores = oc.solve()
    assert res.converged and res.relative_residual <= 1e-10
    got, want = interior_nodes(g, et.cpu().numpy()), interior_nodes(g, oc.theta_field)
    if precision == 0:
        assert res.iterations == ores.iterations
        assert np.abs(got - want).max() <= 3e-10 * np.abs(want).max() + 3e-12
    else:
        assert np.abs(got - want).max() <= 3e-5 * np.abs(want).max() + 3e-7
    tl.close()
