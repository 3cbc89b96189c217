"""Energy-conserving smoothing on the GPU against the oracle: the smoothing
passes (tpicb200_smooth) bit for bit in FP64, the smoothed field solve
(S^n on the right-hand side's J-hat and around every mass apply,
maxwell_device.hpp:152-172,389-432) with the oracle's iteration counts, and
whole smoothed cycles whose movers gather S^n(E_theta)
(maxwell_device.hpp:213-228)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from fieldutil import interior_nodes, periodic_cell_field, periodic_node_field, smooth_random_unique
from reference_fixtures import ogrid
from tpic_b200.plasma import GridSpec

pytestmark = pytest.mark.gpu
GRID = GridSpec(6, 5, 4, 3.0, 2.5, 2.0)


@pytest.mark.parametrize("niter,alpha,op", [(1, 0.5, 0), (2, 0.25, 0), (3, 0.5, 1), (6, 0.0, 0)])
def test_smoothing_passes_match_oracle_bit_for_bit(torch_cuda, niter, alpha, op):
    from gpu_helpers import StageContext
    g = GRID
    rng = np.random.default_rng(11)
    f = periodic_node_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    want = np.zeros_like(f)
    O.load().oracle_smooth(C.byref(ogrid(g)), niter, alpha, op, O.ptr(f), O.ptr(want))
    ctx = StageContext(g, 0, smoothing=(niter, alpha, op))
    src = ctx.field(f, np.float64)
    out = torch_cuda.zeros_like(src)
    assert ctx.lib.tpicb200_smooth(ctx.ctx, src.data_ptr(), out.data_ptr(), ctx.stream) == 0
    got = out.cpu().numpy()
    assert np.array_equal(interior_nodes(g, got), interior_nodes(g, want))
    # The mixed mode smooths in float arithmetic (FP64 storage).
    ctx1 = StageContext(g, 1, smoothing=(niter, alpha, op))
    out1 = torch_cuda.zeros_like(src)
    assert ctx1.lib.tpicb200_smooth(ctx1.ctx, src.data_ptr(), out1.data_ptr(), ctx1.stream) == 0
    got1 = interior_nodes(g, out1.cpu().numpy())
    assert np.abs(got1 - interior_nodes(g, want)).max() <= 1e-6 * np.abs(want).max()


def test_smooth_needs_a_smoothing_context(torch_cuda):
    from gpu_helpers import StageContext
    from tpic_b200 import _lib
    ctx = StageContext(GRID, 0)
    x = torch_cuda.zeros(3 * ctx.layout.node_count, dtype=torch_cuda.float64, device="cuda")
    y = torch_cuda.zeros_like(x)
    assert ctx.lib.tpicb200_smooth(ctx.ctx, x.data_ptr(), y.data_ptr(), ctx.stream) == _lib.INVALID_STATE


@pytest.mark.parametrize("precision,op,layout", [(0, 0, 1), (0, 1, 0), (1, 0, 1)])
def test_smoothed_field_solve_matches_oracle(torch_cuda, precision, op, layout):
    from gpu_helpers import StageContext
    from test_gpu_stages import prepared_oracle
    g = GRID
    oc = prepared_oracle(g, 0)
    oc.smoothing = (2, 0.5, op)
    rng = np.random.default_rng(4)
    oc.e = periodic_node_field(g, smooth_random_unique(g, rng, 0.01))
    bcell = periodic_cell_field(g, smooth_random_unique(g, rng, 0.05))
    oc.b = bcell
    ctx = StageContext(g, precision, dt=0.2, tol=1e-10, mass_layout=layout, smoothing=(2, 0.5, op))
    et, res = ctx.field_solve(ctx.field(oc.e), ctx.field(bcell), ctx.field(oc.j), ctx.mass_from_records(oc.m))
    ores = oc.solve()
    assert res.converged and res.relative_residual <= 1e-10
    got, want = interior_nodes(g, et.cpu().numpy()), interior_nodes(g, oc.theta_field).copy()
    if precision == 0:
        assert res.iterations == ores.iterations
        assert np.abs(got - want).max() <= 3e-10 * np.abs(want).max() + 3e-12
    else:
        assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()
    # Smoothing changes the solution: the unsmoothed solve differs.
    oc.smoothing = (0, 1.0, 0)
    oc.solve()
    assert np.abs(interior_nodes(g, oc.theta_field) - want).max() > 1e-6 * np.abs(want).max()


@pytest.mark.parametrize("op", [0, 1])
def test_smoothed_cycles_match_oracle_fp64(op):
    from tpic_b200.plasma import generate_species
    from tpic_b200.simulation import Simulation
    from test_gpu_cycle import c1_case
    case = c1_case(n=12)
    sm = (2, 0.5, op)
    sim = Simulation(case, precision="double", mass_kind="scalar", mass_layout="stencil-major", smoothing=sm)
    sim.prepare()
    reports = sim.run(2)
    arrays = O.case_species_arrays(case, 0, generate_species)
    oc = O.OracleCycle(case.grid, arrays, case.dt, case.theta, case.c, case.gmres_tol, 0, b0=case.fields.b0,
                       smoothing=sm)
    oc.prepare()
    energies = [oc.cycle() for _ in range(2)]
    for r, e, og in zip(reports, energies, oc.gmres):
        assert r.gmres_iterations == og.iterations
        assert abs(r.total_energy - O.total_energy(e, 2)) <= 1e-10 * abs(O.total_energy(e, 2))
    for s in range(2):
        live = {k: v.cpu().numpy() for k, v in sim.live(s).items()}
        want = oc.species[s][1]
        assert np.array_equal(live["cell"], want["cell"])
        assert np.allclose(live["rx"], want["rx"], rtol=0, atol=1e-11)
        assert np.allclose(live["u"], want["u"], rtol=1e-9, atol=1e-13)
    g = case.grid
    e_gpu, e_cpu = interior_nodes(g, sim.field("e").cpu().numpy()), interior_nodes(g, oc.e)
    assert np.abs(e_gpu - e_cpu).max() <= 3e-10 * np.abs(e_cpu).max() + 3e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_smoothing_flags_a_nonfinite_value(torch_cuda, precision):
    """A NaN reaching a smoothing pass raises the context's invalid counter,
    as the reference's pass flags a nonfinite stored value
    (node_smoothing_device.hpp:30-36); a finite field leaves it at zero."""
    from gpu_helpers import StageContext
    g = GRID
    rng = np.random.default_rng(3)
    f = periodic_node_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    ctx = StageContext(g, precision, smoothing=(2, 0.5, 0))
    count = C.c_uint32(99)
    src = ctx.field(f, np.float64)
    out = torch_cuda.zeros_like(src)
    assert ctx.lib.tpicb200_smooth(ctx.ctx, src.data_ptr(), out.data_ptr(), ctx.stream) == 0
    assert ctx.lib.tpicb200_read_invalid(ctx.ctx, C.byref(count), 1, ctx.stream) == 0
    assert count.value == 0
    bad = f.copy()
    nodes = (g.nx + 3) * (g.ny + 3) * (g.nz + 3)
    bad[nodes + 3 + (g.nx + 3) * (2 + (g.ny + 3) * 2)] = np.nan  # component y, an interior node
    src = ctx.field(bad, np.float64)
    assert ctx.lib.tpicb200_smooth(ctx.ctx, src.data_ptr(), out.data_ptr(), ctx.stream) == 0
    assert ctx.lib.tpicb200_read_invalid(ctx.ctx, C.byref(count), 1, ctx.stream) == 0
    assert count.value > 0
    assert ctx.lib.tpicb200_read_invalid(ctx.ctx, C.byref(count), 0, ctx.stream) == 0
    assert count.value == 0
