"""Size-independent properties of the oracle's restatement of the path (CPU,
no GPU): energy conservation of the ECSIM cycle to the GMRES tolerance,
GMRES convergence, stability of the counting sort, the
periodic fold's conservation and periodicity and linearity of the mass
apply."""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle as O
from fieldutil import periodic_node_field, smooth_random_unique
from reference_fixtures import ogrid, oracle_sort, periodic_node_field_records
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec, generate_species


def small_case(n=6):
    g = GridSpec(n, n, n, 4.0, 4.0, 4.0)
    sp = [SpeciesSpec(qom=-64.0, npcel=(2, 2, 2), vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, npcel=(2, 2, 2), vth=(0.0056,) * 3)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-10, ncycles=3, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))


def test_energy_conserved_and_gmres_converges():
    case = small_case()
    arrays = O.case_species_arrays(case, 0, generate_species)
    oc = O.OracleCycle(case.grid, arrays, case.dt, case.theta, case.c, case.gmres_tol, 0, b0=case.fields.b0)
    oc.prepare()
    w0 = O.total_energy(oc.energy(), 2)
    for _ in range(3):
        w = O.total_energy(oc.cycle(), 2)
        assert abs(w - w0) <= 1e-9 * abs(w0)
    for res in oc.gmres:
        assert res.converged and res.relative_residual <= 1e-10


def test_sort_is_stable_with_consistent_bins():
    g = GridSpec(5, 4, 3, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(0)
    keys = g.encode(rng.integers(0, 5, 5000), rng.integers(0, 4, 5000), rng.integers(0, 3, 5000)).astype(np.int32)
    perm, counts, offsets = oracle_sort(g, keys)
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))
    assert offsets[-1] == len(keys) and np.array_equal(np.diff(offsets), counts)


def test_fold_conserves_and_makes_periodic():
    """The shared-node sum conserves the total over the interior vertices
    [0, n]^3 (ghost values are replaced, not added) and leaves every
    duplicate and ghost vertex equal to its periodic unique vertex."""
    g = GridSpec(4, 3, 5, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(1)
    shape = (g.nz + 3, g.ny + 3, g.nx + 3)
    nodes = shape[0] * shape[1] * shape[2]
    j, m = rng.normal(size=3 * nodes), rng.normal(size=126 * nodes)
    before = j.reshape(3, *shape)[:, 1:-1, 1:-1, 1:-1].sum(axis=(1, 2, 3))
    O.load().oracle_fold(C.byref(ogrid(g)), O.ptr(j), O.ptr(m))
    f = j.reshape(3, *shape)
    after = f[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1].sum(axis=(1, 2, 3))
    assert np.allclose(after, before, rtol=1e-13, atol=1e-12)
    k = (np.arange(-1, g.nz + 2) % g.nz) + 1
    jj = (np.arange(-1, g.ny + 2) % g.ny) + 1
    i = (np.arange(-1, g.nx + 2) % g.nx) + 1
    assert np.array_equal(f, f[:, k][:, :, jj][:, :, :, i])
    mr = m.reshape(*shape, 126)
    assert np.array_equal(mr, mr[k][:, jj][:, :, i])


def test_mass_apply_is_linear():
    g = GridSpec(4, 4, 3, 2.0, 2.0, 1.5)
    rng = np.random.default_rng(2)
    m = periodic_node_field_records(g, rng.normal(size=(126, g.nz, g.ny, g.nx)))
    x = periodic_node_field(g, smooth_random_unique(g, rng, 1.0))
    y = periodic_node_field(g, smooth_random_unique(g, rng, 1.0))
    nodes = (g.nx + 3) * (g.ny + 3) * (g.nz + 3)
    lib = O.load()

    def apply(v):
        out = np.zeros(3 * nodes)
        lib.oracle_mass_apply(0, C.byref(ogrid(g)), O.ptr(m), O.ptr(np.ascontiguousarray(v)), O.ptr(out))
        return out

    a, b = 0.75, -1.25
    assert np.allclose(apply(a * x + b * y), a * apply(x) + b * apply(y), rtol=1e-12, atol=1e-12)
