"""Stage-by-stage parity of the CUDA path (through the C ABI) with the CPU
oracle on the same seeded inputs.

Bars: mover cell keys, fractions and velocities bit-exact; sort permutation,
counts and offsets bit-exact (stable order); current and mass within TPIC's
sorted-mass tolerances (3e-12*max|coef| + 1e-15 FP64, 3e-5*max|coef| + 1e-15
FP32, docs/developer/testing.md:255-260); fields within rtol 3e-10 / atol
3e-12 (FP64 storage) and 3e-5 / 3e-7 (FP32), testing.md:262-273.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from tpic_b200 import _lib
from fieldutil import (bits, interior_nodes, interior_records, periodic_cell_field, periodic_node_field,
                       smooth_random_unique)
from reference_fixtures import (host_matrix_core_mass, mover_edge_records, ogrid, oracle_moments, oracle_mover,
                                oracle_sort, periodic_node_field_records, reference_mass_fixture, reference_sort_keys,
                                species_arrays)
from tpic_b200.plasma import GridSpec, SpeciesSpec, generate_species

pytestmark = pytest.mark.gpu

GRID = GridSpec(6, 5, 4, 3.0, 2.5, 2.0)


def make_ctx(g, precision, **kw):
    from gpu_helpers import StageContext
    return StageContext(g, precision=precision, **kw)


@pytest.mark.parametrize("precision", [0, 1])
def test_mover_bit_exact(torch_cuda, precision):
    g = GRID
    rng = np.random.default_rng(11)
    d = species_arrays(g, precision)
    n = len(d["cell"])
    ctx = make_ctx(g, precision, dt=0.3)
    etheta = periodic_node_field(g, smooth_random_unique(g, rng, 0.4))
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9)).astype(ctx.np_fdt)
    parts = ctx.upload_particles(d)
    ctx.mover(-4.0, parts, n, ctx.field(etheta, np.float64), ctx.field(bnode))
    got = ctx.download(parts, n)
    want, bad = oracle_mover(g, precision, -4.0, 0.3, d, etheta, bnode)
    assert bad == 0 and ctx.invalid_count() == 0
    assert np.array_equal(got["cell"], want["cell"])
    for k in ("rx", "ry", "rz", "u", "v", "w"):
        assert np.array_equal(bits(got[k]), bits(want[k])), k
    # The flight crossed cells and periodic boundaries.
    assert np.mean(got["cell"] != d["cell"]) > 0.3


@pytest.mark.parametrize("precision", [0, 1])
def test_mover_edge_records(torch_cuda, precision):
    """Endpoint fractions, sub-ULP negative crossings and invalid records
    (which keep every attribute), as sorted_current_mover_device.cpp:126-140,241-259."""
    g, d = mover_edge_records(precision)
    n = len(d["cell"])
    ctx = make_ctx(g, precision, dt=0.5)
    etheta = np.zeros(3 * ctx.layout.node_count)
    bnode = np.zeros(3 * ctx.layout.node_count, dtype=ctx.np_fdt)
    parts = ctx.upload_particles(d)
    ctx.mover(-1.0, parts, n, ctx.field(etheta, np.float64), ctx.field(bnode))
    got = ctx.download(parts, n)
    want, bad = oracle_mover(g, precision, -1.0, 0.5, d, etheta, bnode)
    assert bad == 4 and ctx.invalid_count() == 4  # halo key, fraction 1, NaN velocity, key out of range
    assert np.array_equal(got["cell"], want["cell"])
    for k in ("rx", "ry", "rz", "u", "v", "w"):
        assert np.array_equal(bits(got[k]), bits(want[k])), k
    for r in (6, 7, 8, 9):  # invalid records are unchanged
        assert got["cell"][r] == d["cell"][r] and bits(got["rx"])[r] == bits(d["rx"])[r]
    assert ((got["rx"][:6] >= 0) & (got["rx"][:6] < 1)).all()


def run_sort_case(g, keys, precision=0):
    n = len(keys)
    vdt = np.float64 if precision == 0 else np.float32
    idx = np.arange(n)
    d = {"rx": idx * 0.125, "ry": idx * -0.25, "rz": idx * 0.5, "u": (idx * -0.5).astype(vdt),
         "v": (idx * 0.25).astype(vdt), "w": (idx * -0.125).astype(vdt), "q": idx * 2.0,
         "cell": np.asarray(keys, dtype=np.int32), "id": (idx + 100).astype(np.uint64)}
    ctx = make_ctx(g, precision, max_particles=max(n, 1))
    src = ctx.upload_particles(d) if n else ctx.empty_particles(0, True)
    dst, counts, offsets = ctx.sort(src, n, with_id=True)
    got = ctx.download(dst, n)
    perm, wc, wo = oracle_sort(g, d["cell"])
    assert ctx.invalid_count() == 0
    assert np.array_equal(counts.cpu().numpy().view(np.uint32), wc)
    assert np.array_equal(offsets.cpu().numpy().view(np.uint32), wo)
    for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell", "id"):
        assert np.array_equal(got[k], d[k][perm]), k
    # The attribute mapping of particle_sort_device.cpp:96-131 holds.
    ident = got["id"].astype(np.int64) - 100
    assert np.array_equal(got["rx"], ident * 0.125) and np.array_equal(got["q"], ident * 2.0)
    assert (np.diff(got["cell"]) >= 0).all()


def test_sort_stable_random(torch_cuda):
    g = GridSpec(8, 7, 6, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(5)
    i, j, k = rng.integers(0, 8, 40000), rng.integers(0, 7, 40000), rng.integers(0, 6, 40000)
    run_sort_case(g, g.encode(i, j, k))


def test_sort_nearly_sorted_and_fixture_keys(torch_cuda):
    g = GridSpec(16, 8, 8, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(9)
    i = np.repeat(np.arange(16 * 8 * 8), 50)
    keys = g.encode(i % 16, (i // 16) % 8, i // 128)
    moved = rng.random(len(keys)) < 0.08
    keys = np.where(moved, g.encode(rng.integers(0, 16, len(keys)), rng.integers(0, 8, len(keys)),
                                    rng.integers(0, 8, len(keys))), keys)
    run_sort_case(g, keys, precision=1)
    # The reference fixture: key = (i*7+3) % 19 (particle_sort_device.cpp:67).
    run_sort_case(*reference_sort_keys())


@pytest.mark.parametrize("n", [0, 1, 33, 300, 9000, 20000])
def test_sort_one_bin_and_empty(torch_cuda, n):
    g = GridSpec(3, 3, 3, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(n)
    keys = np.full(n, g.encode(1, 2, 0))
    if n > 3:  # a few foreign keys interleaved so the big bin is not already in order after placement
        keys[rng.integers(0, n, n // 10)] = g.encode(0, 0, 0)
    run_sort_case(g, keys)


def test_sort_rejects_out_of_range_key(torch_cuda):
    g = GridSpec(3, 3, 3, 1.0, 1.0, 1.0)
    ctx = make_ctx(g, 0, max_particles=10)
    d = {k: np.zeros(4) for k in ("rx", "ry", "rz", "u", "v", "w", "q")}
    d["cell"] = np.array([5, 6, -1, 7], dtype=np.int32)
    src = ctx.upload_particles(d)
    ctx.sort(src, 4)
    assert ctx.invalid_count() == 1


# --------------------------------------------------------------------------
def assert_moments(g, jg, mg, jw, mw, rel):
    jw_i, jg_i = interior_nodes(g, jw), interior_nodes(g, jg)
    scale = np.abs(jw_i).max()
    assert np.abs(jg_i - jw_i).max() <= rel * scale + 1e-15
    mw_i, mg_i = interior_records(g, mw), interior_records(g, mg)
    scale = np.abs(mw_i).max()
    assert np.abs(mg_i - mw_i).max() <= rel * scale + 1e-15


@pytest.mark.parametrize("precision,kind,sorted_bins,layout", [
    (0, 0, True, 0), (0, 0, False, 0), (1, 0, True, 0), (1, 0, False, 0), (1, 1, True, 0), (0, 1, True, 0),
    (0, 0, True, 1), (1, 0, False, 1), (1, 0, True, 1), (0, 0, True, 2), (1, 0, False, 2)])
def test_deposit_matches_oracle(torch_cuda, precision, kind, sorted_bins, layout):
    g = GRID
    rng = np.random.default_rng(21)
    d = species_arrays(g, precision, vth=(0.2, 0.1, 0.3), npcel=(3, 3, 3))
    n = len(d["cell"])
    ctx = make_ctx(g, precision, dt=0.2, mass_layout=layout)
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9)).astype(ctx.np_fdt)
    parts = ctx.upload_particles(d)
    bn = ctx.field(bnode)
    j, m = ctx.moments()
    if sorted_bins:
        parts, counts, offsets = ctx.sort(parts, n)
        ctx.deposit(-4.0, parts, n, bn, j, m, counts, offsets, kind=kind)
    else:
        ctx.deposit(-4.0, parts, n, bn, j, m, kind=kind)
    ctx.fold(j, m)
    jw, mw, bad = oracle_moments(g, precision, -4.0, 0.2, d, bnode)
    assert bad == 0 and ctx.invalid_count() == 0
    rel = 3e-12 if precision == 0 else 3e-5
    assert_moments(g, j.cpu().numpy().astype(np.float64), ctx.records(m), jw, mw, rel)


@pytest.mark.parametrize("precision,kind", [(0, 0), (1, 0), (1, 1), (0, 4)])
def test_reference_mass_fixture(torch_cuda, precision, kind):
    g, d, bnode = reference_mass_fixture(precision)
    n = len(d["cell"])
    ctx = make_ctx(g, precision, dt=0.14, max_particles=n)
    parts = ctx.upload_particles(d)
    parts, counts, offsets = ctx.sort(parts, n)  # the fixture is already in key order
    j, m = ctx.moments()
    if kind != 4:  # the moment form deposits J-hat and the mass together
        j = None
    ctx.deposit(-1.0, parts, n, ctx.field(bnode), j, m, counts, offsets, kind=kind)
    ctx.fold(j, m)
    want = host_matrix_core_mass(g, d, bnode, -0.07)
    got = m.cpu().numpy().astype(np.float64)
    wi, gi = interior_records(g, want), interior_records(g, got)
    rel = 3e-12 if precision == 0 else 3e-5
    assert ctx.invalid_count() == 0
    assert np.abs(gi - wi).max() <= rel * np.abs(wi).max() + 1e-15


@pytest.mark.parametrize("layout", [0, 1, 2])
def test_mass_apply_matches_oracle(torch_cuda, layout):
    g = GRID
    rng = np.random.default_rng(2)
    nodes = (g.nz + 3) * (g.ny + 3) * (g.nx + 3)
    unique = rng.normal(size=(126, g.nz, g.ny, g.nx))
    m = periodic_node_field_records(g, unique)
    v = periodic_node_field(g, smooth_random_unique(g, rng, 1.0))
    ctx = make_ctx(g, 0, mass_layout=layout)
    out = ctx.mass_apply(ctx.mass_from_records(m), ctx.field(v, np.float64)).cpu().numpy()
    want = np.zeros(3 * nodes)
    O.load().oracle_mass_apply(0, C.byref(ogrid(g)), O.ptr(m), O.ptr(v), O.ptr(want))
    assert np.allclose(interior_nodes(g, out), interior_nodes(g, want), rtol=1e-13, atol=1e-13)
    ref = O.load_reference()
    if ref is not None:  # the reference's own apply_mass_matrix_node at a few nodes
        for (i, j, k) in [(0, 0, 0), (6, 5, 4), (3, 2, 1)]:
            o = np.zeros(3)
            ref.ref_mass_apply_node(g.nx, g.ny, g.nz, O.ptr(m), O.ptr(v), 1.0 / ((0.5 * 0.5) * 0.5), i, j, k, O.ptr(o))
            assert np.allclose(interior_nodes(g, out)[:, k, j, i], o, rtol=1e-13, atol=1e-13)


# --------------------------------------------------------------------------
def prepared_oracle(g, precision, seed=1):
    from tpic_b200.plasma import generate_species as gen
    species = [SpeciesSpec(qom=-16.0, npcel=(2, 2, 2), vth=(0.08,) * 3), SpeciesSpec(qom=1.0, npcel=(2, 2, 2),
                                                                                      vth=(0.01,) * 3)]
    arrays = []
    for s, sp in enumerate(species):
        dd = gen(g, sp, s, seed=seed, velocity_dtype=np.float64 if precision == 0 else np.float32)
        dd.pop("id")
        arrays.append((sp.qom, dd))
    oc = O.OracleCycle(g, arrays, 0.2, 0.5, 1.0, 1e-10, precision, b0=(0.1, -0.05, 0.2))
    oc.prepare()
    return oc


@pytest.mark.parametrize("layout", [0, 1, 2])
def test_field_solve_matches_oracle(torch_cuda, layout):
    g = GRID
    oc = prepared_oracle(g, 0)
    rng = np.random.default_rng(4)
    oc.e = periodic_node_field(g, smooth_random_unique(g, rng, 0.01))
    bcell = periodic_cell_field(g, smooth_random_unique(g, rng, 0.05))
    oc.b = bcell
    ctx = make_ctx(g, 0, dt=0.2, tol=1e-10, mass_layout=layout)
    et, res = ctx.field_solve(ctx.field(oc.e), ctx.field(bcell), ctx.field(oc.j), ctx.mass_from_records(oc.m))
    ores = oc.solve()
    assert res.converged and res.relative_residual <= 1e-10
    assert res.iterations == ores.iterations
    got, want = interior_nodes(g, et.cpu().numpy()), interior_nodes(g, oc.theta_field)
    assert np.abs(got - want).max() <= 3e-10 * np.abs(want).max() + 3e-12


def test_gmres_iteration_limit_commits_nothing(torch_cuda):
    """gmres_device.cpp:220-222: a solve stopped by the iteration limit reports
    it and leaves the solution field untouched."""
    g = GRID
    oc = prepared_oracle(g, 0)
    rng = np.random.default_rng(4)
    e = periodic_node_field(g, smooth_random_unique(g, rng, 0.01))
    bcell = periodic_cell_field(g, smooth_random_unique(g, rng, 0.05))
    import torch
    ctx = make_ctx(g, 0, dt=0.2, tol=1e-14, max_iterations=1)
    et = torch.full((3 * ctx.layout.node_count,), 7.0, dtype=torch.float64, device="cuda")
    res = _lib.GmresResult()
    status = ctx.lib.tpicb200_field_solve(ctx.ctx, ctx.field(e).data_ptr(), ctx.field(bcell).data_ptr(),
                                          ctx.field(oc.j).data_ptr(), ctx.mass_from_records(oc.m).data_ptr(),
                                          et.data_ptr(), C.byref(res), ctx.stream)
    assert status == _lib.NOT_CONVERGED
    assert not res.converged and res.iterations == 1
    assert bool((et == 7.0).all())


@pytest.mark.parametrize("precision", [0, 1])
def test_gmres_short_restarts_converge(torch_cuda, precision):
    """gmres_device.cpp:223-235: restart length 2, several restart cycles to
    1e-10 (the mixed mode through its refined cycles), the solution equal to
    the oracle's GMRES(2) solution; one host wait per restart cycle plus one."""
    g = GRID
    oc = prepared_oracle(g, precision)
    rng = np.random.default_rng(6)
    oc.e = periodic_node_field(g, smooth_random_unique(g, rng, 0.01))
    bcell = periodic_cell_field(g, smooth_random_unique(g, rng, 0.05))
    oc.b = bcell
    oc.restart = 2
    ctx = make_ctx(g, precision, dt=0.2, tol=1e-10, restart=2)
    mass = ctx.mass_from_records(oc.m.astype(ctx.np_fdt).astype(np.float64))
    et, res = ctx.field_solve(ctx.field(oc.e), ctx.field(bcell), ctx.field(oc.j), mass)
    assert res.converged and res.iterations > 2 and res.relative_residual <= 1e-10
    assert res.host_waits == 1 + (res.iterations + 1) // 2 or precision == 1
    if precision == 0:
        ores = oc.solve()
        assert res.iterations == ores.iterations
        got, want = interior_nodes(g, et.cpu().numpy()), interior_nodes(g, oc.theta_field)
        assert np.abs(got - want).max() <= 3e-10 * np.abs(want).max() + 3e-12


def test_gmres_zero_rhs(torch_cuda):
    """gmres_device.cpp:243-248: a zero right-hand side (no field, current or
    mass) converges at once with a zero solution."""
    g = GRID
    ctx = make_ctx(g, 0, dt=0.2, tol=1e-10)
    nodes, cells = ctx.layout.node_count, ctx.layout.cell_count
    zero_nodes = np.zeros(3 * nodes)
    et, res = ctx.field_solve(ctx.field(zero_nodes), ctx.field(np.zeros(3 * cells)), ctx.field(zero_nodes),
                              ctx.mass_from_records(np.zeros(126 * nodes)))
    assert res.converged and res.iterations == 0 and res.rhs_norm == 0.0 and res.host_waits == 1
    assert float(et.abs().max()) == 0.0


@pytest.mark.parametrize("precision", [0, 1])
def test_field_advance_matches_oracle(torch_cuda, precision):
    g = GRID
    rng = np.random.default_rng(8)
    ctx = make_ctx(g, precision, dt=0.2)
    fdt = ctx.np_fdt
    e = periodic_node_field(g, smooth_random_unique(g, rng, 0.3)).astype(fdt)
    b = periodic_cell_field(g, smooth_random_unique(g, rng, 0.3)).astype(fdt)
    th = periodic_node_field(g, smooth_random_unique(g, rng, 0.3))
    et = ctx.field(e)
    bnext, bnode = ctx.field_advance(et, ctx.field(b), ctx.field(th, np.float64))
    we, wb, wbn = e.astype(np.float64), np.zeros(b.size), np.zeros(e.size)
    O.load().oracle_field_advance(C.byref(ogrid(g)), 0.2, 0.5, 1.0, O.ptr(we), O.ptr(b.astype(np.float64)),
                                  O.ptr(th), O.ptr(wb), O.ptr(wbn))
    rtol, atol = (3e-10, 3e-12) if precision == 0 else (3e-5, 3e-7)
    assert np.allclose(interior_nodes(g, et.cpu().numpy()), interior_nodes(g, we), rtol=rtol, atol=atol)
    assert np.allclose(bnext.cpu().numpy(), wb, rtol=rtol, atol=atol)
    assert np.allclose(bnode.cpu().numpy(), wbn, rtol=rtol, atol=atol)


# --------------------------------------------------------------------------
# Tensor-core (tcgen05) mass assembly.
@pytest.mark.parametrize("nx", [5, 8])
@pytest.mark.parametrize("kind", [2, 3])
def test_tc_exact_inputs(torch_cuda, kind, nx):
    """Inputs exactly representable in TF32 (fractions in {0, 1/4, 1/2, 3/4},
    B = 0 so alpha = I, power-of-two charges): every product is exact, so the
    tensor-core mass matrix must equal the FP64 oracle to FP32 accumulation
    rounding. Checks the operand layouts, descriptors and the pair epilogue;
    nx = 8 takes the four-node assembly, nx = 5 the per-node one."""
    g = GridSpec(nx, 4, 3, float(nx), 4.0, 3.0)
    rng = np.random.default_rng(17)
    rows = []
    for cell in range(g.cells):
        i, j, k = cell % g.nx, (cell // g.nx) % g.ny, cell // (g.nx * g.ny)
        for _ in range(int(rng.integers(0, 90))):
            rows.append((g.encode(i, j, k), *(rng.integers(0, 4, 3) / 4.0), rng.choice([0.5, -0.25, 1.0])))
    rows = np.array(rows)
    n = len(rows)
    d = {"cell": rows[:, 0].astype(np.int32), "rx": rows[:, 1].copy(), "ry": rows[:, 2].copy(), "rz": rows[:, 3].copy(),
         "q": rows[:, 4].copy(), "u": np.zeros(n, np.float32), "v": np.zeros(n, np.float32), "w": np.zeros(n, np.float32)}
    ctx = make_ctx(g, 1, dt=1.0, max_particles=n)
    parts = ctx.upload_particles(d)
    parts, counts, offsets = ctx.sort(parts, n)
    bnode = np.zeros(3 * ctx.layout.node_count, np.float32)
    j, m = ctx.moments()
    ctx.deposit(1.0, parts, n, ctx.field(bnode), j, m, counts, offsets, kind=kind)
    ctx.fold(j, m)
    jw, mw, bad = oracle_moments(g, 1, 1.0, 1.0, d, bnode)
    assert bad == 0 and ctx.invalid_count() == 0
    got = interior_records(g, m.cpu().numpy().astype(np.float64))
    want = interior_records(g, mw)
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


@pytest.mark.parametrize("kind,rel,layout,nx", [(2, 3e-3, 0, 6), (3, 1e-4, 0, 6), (2, 3e-3, 1, 6), (3, 1e-4, 1, 6),
                                                 (3, 1e-4, 1, 8), (2, 3e-3, 0, 8), (3, 1e-4, 2, 6)])
def test_tc_mass_matches_oracle(torch_cuda, kind, rel, layout, nx):
    g = GRID if nx == GRID.nx else GridSpec(nx, GRID.ny, GRID.nz, GRID.lx * nx / GRID.nx, GRID.ly, GRID.lz)
    rng = np.random.default_rng(23)
    d = species_arrays(g, 1, vth=(0.2, 0.1, 0.3), npcel=(4, 4, 4))
    n = len(d["cell"])
    ctx = make_ctx(g, 1, dt=0.2, max_particles=n, mass_layout=layout)
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9)).astype(np.float32)
    parts = ctx.upload_particles(d)
    parts, counts, offsets = ctx.sort(parts, n)
    j, m = ctx.moments()
    ctx.deposit(-4.0, parts, n, ctx.field(bnode), j, m, counts, offsets, kind=kind)
    ctx.fold(j, m)
    jw, mw, bad = oracle_moments(g, 1, -4.0, 0.2, d, bnode)
    assert bad == 0 and ctx.invalid_count() == 0
    jg, mg = j.cpu().numpy().astype(np.float64), ctx.records(m)
    jw_i, jg_i = interior_nodes(g, jw), interior_nodes(g, jg)
    # J-hat rides in the same contraction (sum_b W_a W_b = W_a), so it carries
    # the form's operand rounding too.
    assert np.abs(jg_i - jw_i).max() <= rel * np.abs(jw_i).max() + 1e-15
    mw_i, mg_i = interior_records(g, mw), interior_records(g, mg)
    err = np.abs(mg_i - mw_i).max() / np.abs(mw_i).max()
    assert err <= rel, err


@pytest.mark.parametrize("layout,nx", [(0, 6), (1, 6), (1, 8), (0, 8), (2, 6), (2, 8)])
def test_fp64_moments_match_oracle(torch_cuda, layout, nx):
    """The FP64 moment form (double precision): J-hat and the mass records
    equal the oracle's scalar deposition to the rounding of the regrouped
    sums, for both mass layouts and both assembly paths (nx a multiple of
    four or not), two species adding into one set of moments."""
    g = GRID if nx == GRID.nx else GridSpec(nx, GRID.ny, GRID.nz, GRID.lx * nx / GRID.nx, GRID.ly, GRID.lz)
    rng = np.random.default_rng(31)
    d1 = species_arrays(g, 0, seed=5, vth=(0.2, 0.1, 0.3), npcel=(4, 4, 4), qom=-4.0)
    d2 = species_arrays(g, 0, seed=6, vth=(0.02, 0.01, 0.03), npcel=(3, 3, 3), qom=1.0)
    ctx = make_ctx(g, 0, dt=0.2, max_particles=len(d1["cell"]), mass_layout=layout)
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9))
    bn = ctx.field(bnode)
    j, m = ctx.moments()
    jw = np.zeros(3 * ctx.layout.node_count)
    mw = np.zeros(126 * ctx.layout.node_count)
    for qom, d in ((-4.0, d1), (1.0, d2)):
        n = len(d["cell"])
        parts, counts, offsets = ctx.sort(ctx.upload_particles(d), n)
        ctx.deposit(qom, parts, n, bn, j, m, counts, offsets, kind=4)
        js, ms, bad = oracle_moments(g, 0, qom, 0.2, d, bnode)
        assert bad == 0
        jw += js
        mw += ms
    ctx.fold(j, m)
    assert ctx.invalid_count() == 0
    assert_moments(g, j.cpu().numpy(), ctx.records(m), jw, mw, 1e-13)


@pytest.mark.parametrize("kind", [2, 3])
def test_tc_mass_sparse_batches(torch_cuda, kind):
    """Records in scattered cells only (every 13th cell), so many batches of
    four cells are empty and a warp's stream runs through one-chunk batches:
    the per-batch metadata of a chunk must survive the walk three chunks
    ahead into later batches. The moments equal the oracle's and no record
    is flagged."""
    # More batches than the launch has warps (4 x 148 CTAs x 4 warps), so each
    # warp walks several batches.
    g = GridSpec(64, 64, 16, 6.4, 6.4, 1.6)
    rng = np.random.default_rng(41)
    d = species_arrays(g, 1, vth=(0.2, 0.1, 0.3), npcel=(2, 2, 2))
    ex, ey = g.nx + 4, g.ny + 4
    key = d["cell"].astype(np.int64)
    i, j, k = key % ex - 2, (key // ex) % ey - 2, key // (ex * ey) - 2
    keep = ((i + g.nx * (j + g.ny * k)) % 13) == 0
    d = {name: np.ascontiguousarray(v[keep]) for name, v in d.items()}
    n = len(d["cell"])
    assert 0 < n < 60000
    ctx = make_ctx(g, 1, dt=0.2, max_particles=n, mass_layout=1)
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9)).astype(np.float32)
    parts = ctx.upload_particles(d)
    parts, counts, offsets = ctx.sort(parts, n)
    j_, m = ctx.moments()
    ctx.deposit(-4.0, parts, n, ctx.field(bnode), j_, m, counts, offsets, kind=kind)
    ctx.fold(j_, m)
    jw, mw, bad = oracle_moments(g, 1, -4.0, 0.2, d, bnode)
    assert bad == 0 and ctx.invalid_count() == 0
    rel = 3e-3 if kind == 2 else 1e-4
    jw_i, jg_i = interior_nodes(g, jw), interior_nodes(g, j_.cpu().numpy().astype(np.float64))
    assert np.abs(jg_i - jw_i).max() <= rel * np.abs(jw_i).max() + 1e-15
    mw_i, mg_i = interior_records(g, mw), interior_records(g, ctx.records(m))
    assert np.abs(mg_i - mw_i).max() <= rel * np.abs(mw_i).max()


@pytest.mark.parametrize("kind", [2, 3])
def test_tc_moments_accumulate_two_species(torch_cuda, kind):
    """Two species deposited with the tensor-core forms before one fold: the
    second species adds to the cell moments of the first (compare with the
    oracle's sum of both)."""
    g = GRID
    rng = np.random.default_rng(29)
    d1 = species_arrays(g, 1, seed=5, vth=(0.2, 0.1, 0.3), npcel=(3, 3, 3), qom=-4.0)
    d2 = species_arrays(g, 1, seed=6, vth=(0.02, 0.01, 0.03), npcel=(2, 2, 2), qom=1.0)
    ctx = make_ctx(g, 1, dt=0.2, max_particles=len(d1["cell"]), mass_layout=1)
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9)).astype(np.float32)
    bn = ctx.field(bnode)
    j, m = ctx.moments()
    jw = np.zeros(3 * ctx.layout.node_count)
    mw = np.zeros(126 * ctx.layout.node_count)
    for qom, d in ((-4.0, d1), (1.0, d2)):
        n = len(d["cell"])
        parts, counts, offsets = ctx.sort(ctx.upload_particles(d), n)
        ctx.deposit(qom, parts, n, bn, j, m, counts, offsets, kind=kind)
        js, ms, bad = oracle_moments(g, 1, qom, 0.2, d, bnode)
        assert bad == 0
        jw += js
        mw += ms
    ctx.fold(j, m)
    assert ctx.invalid_count() == 0
    jg, mg = j.cpu().numpy().astype(np.float64), ctx.records(m)
    rel = 3e-3 if kind == 2 else 1e-4
    assert np.abs(interior_nodes(g, jg) - interior_nodes(g, jw)).max() <= rel * np.abs(interior_nodes(g, jw)).max()
    mi = interior_records(g, mw)
    assert np.abs(interior_records(g, mg) - mi).max() <= rel * np.abs(mi).max()


@pytest.mark.parametrize("kind,nspecies", [(2, 2), (3, 2), (2, 3), (3, 3)])
def test_tc_fused_species_ragged_cells(torch_cuda, kind, nspecies):
    """Both species in one tensor-core pass over ragged cells: per cell each
    species keeps 0 %, 30 %, 70 % or all of 64 records by a cell pattern, so
    cells hold only species 0, only species 1, neither, or both with counts
    that cross 32-record chunk boundaries anywhere (a chunk may run from the
    cell's species-0 records into its species-1 records). The moments equal
    the oracle's sum of both species. With three species the call runs two
    passes (species 0 and 1, then species 2 added into the same moments)."""
    g = GridSpec(24, 20, 16, 2.4, 2.0, 1.6)
    rng = np.random.default_rng(53)
    keep_fraction = (0.0, 0.3, 0.7, 1.0)
    species = []
    params = ((-4.0, 11, (0.2, 0.1, 0.3)), (1.0, 12, (0.02, 0.01, 0.03)), (-1.0, 13, (0.1, 0.1, 0.1)))
    for s, (qom, seed, vth) in enumerate(params[:nspecies]):
        d = species_arrays(g, 1, seed=seed, vth=vth, npcel=(4, 4, 4), qom=qom)
        key = d["cell"].astype(np.int64)
        ex, ey = g.nx + 4, g.ny + 4
        i, j, k = key % ex - 2, (key // ex) % ey - 2, key // (ex * ey) - 2
        pattern = (i + 3 * j + 7 * k + s) % 4
        keep = rng.random(len(key)) < np.take(keep_fraction, pattern)
        species.append((qom, {name: np.ascontiguousarray(v[keep]) for name, v in d.items()}))
    counts_per_cell = [np.bincount(d["cell"], minlength=(g.nx + 4) * (g.ny + 4) * (g.nz + 4)) for _, d in species]
    both = (counts_per_cell[0] > 0) & (counts_per_cell[1] > 0)
    assert both.any() and ((counts_per_cell[0] > 0) & ~both).any() and ((counts_per_cell[1] > 0) & ~both).any()
    assert (counts_per_cell[0][both] % 32 != 0).any()
    nmax = max(len(d["cell"]) for _, d in species)
    ctx = make_ctx(g, 1, dt=0.2, max_particles=nmax, mass_layout=1)
    bnode = periodic_node_field(g, smooth_random_unique(g, rng, 0.9)).astype(np.float32)
    bn = ctx.field(bnode)
    j, m = ctx.moments()
    sorted_species, structs, jw, mw = [], [], 0.0, 0.0
    for qom, d in species:
        n = len(d["cell"])
        parts, counts, offsets = ctx.sort(ctx.upload_particles(d), n)
        sorted_species.append((parts, counts, offsets))
        structs.append(ctx.struct(parts, n))
        js, ms, bad = oracle_moments(g, 1, qom, 0.2, d, bnode)
        assert bad == 0
        jw, mw = jw + js, mw + ms
    qoms = (C.c_double * nspecies)(*[qom for qom, _ in species])
    parts_arr = (_lib.Particles * nspecies)(*structs)
    counts_arr = (C.c_void_p * nspecies)(*[c.data_ptr() for _, c, _ in sorted_species])
    offsets_arr = (C.c_void_p * nspecies)(*[o.data_ptr() for _, _, o in sorted_species])
    _lib.check(ctx.lib.tpicb200_deposit_species(ctx.ctx, nspecies, qoms, parts_arr, counts_arr, offsets_arr,
                                                bn.data_ptr(), j.data_ptr(), m.data_ptr(), kind,
                                                ctx.invalid.data_ptr(), ctx.stream))
    ctx.fold(j, m)
    assert ctx.invalid_count() == 0
    jg, mg = j.cpu().numpy().astype(np.float64), ctx.records(m)
    rel = 3e-3 if kind == 2 else 1e-4
    assert np.abs(interior_nodes(g, jg) - interior_nodes(g, jw)).max() <= rel * np.abs(interior_nodes(g, jw)).max()
    mi = interior_records(g, mw)
    assert np.abs(interior_records(g, mg) - mi).max() <= rel * np.abs(mi).max()
