"""The oracle's discrete adjoint of the ECSIM cycle (FP64, CPU).

TPIC has no adjoint, so nothing in the reference pins it: the adjoint is
checked against the oracle's own forward cycle. First the transposes it is
built from, by dot-product identities on random periodic fields (full and
thin grids): N2C^T = C2N, cell_to_node^T, and the solve with A^T
(<A^-1 r1, r2> = <r1, A^-T r2>). Then whole cycles: the gradient of the
final field energy with respect to the initial state (E, B, positions,
velocities, charges) along a random direction, against a central finite
difference of the forward cycles (GMRES at 1e-13 in both directions)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from fieldutil import periodic_cell_field, periodic_node_field
from reference_fixtures import ogrid
from tpic_b200.plasma import GridSpec, SpeciesSpec, generate_species

GRIDS = [GridSpec(5, 4, 3, 2.5, 2.0, 1.5), GridSpec(6, 4, 1, 3.0, 2.0, 0.5), GridSpec(8, 1, 1, 4.0, 0.5, 0.5)]


def unique_dot_nodes(g, a, b):
    fa = a.reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]
    fb = b.reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]
    return float(np.sum(fa * fb))


def unique_dot_cells(g, a, b):
    fa = a.reshape(3, g.nz + 2, g.ny + 2, g.nx + 2)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]
    fb = b.reshape(3, g.nz + 2, g.ny + 2, g.nx + 2)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]
    return float(np.sum(fa * fb))


def consistent(g, node_field):
    """A node field whose duplicate endpoints and ghosts copy the unique nodes."""
    f = node_field.reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]
    return periodic_node_field(g, f)


@pytest.mark.parametrize("g", GRIDS, ids=["3d", "2d", "1d"])
def test_curl_and_average_transposes(g):
    lib = O.load()
    og = C.byref(ogrid(g))
    rng = np.random.default_rng(1)
    u = periodic_node_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    w = periodic_cell_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    n2c = np.zeros_like(w)
    lib.oracle_curl_n2c(og, O.ptr(u), O.ptr(n2c))
    c2n = np.zeros_like(u)
    lib.oracle_curl_c2n(og, O.ptr(w), O.ptr(c2n))
    lhs, rhs = unique_dot_cells(g, n2c, w), unique_dot_nodes(g, u, consistent(g, c2n))
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + np.abs(u).max() * np.abs(w).max())
    # cell_to_node^T through the field adjoint with lambda = 0.
    avg = np.zeros_like(u)
    lib.oracle_cell_to_node(og, O.ptr(w), O.ptr(avg))
    e_bar, b_bar = np.zeros_like(u), np.zeros_like(w)
    lib.oracle_adjoint_fields(og, 0.1, 0.5, 1.0, O.ptr(np.zeros_like(u)), O.ptr(u), O.ptr(e_bar), O.ptr(b_bar))
    lhs, rhs = unique_dot_nodes(g, consistent(g, avg), u), unique_dot_cells(g, w, b_bar)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def random_mass(g, rng):
    """Mass records of a real deposition (random particles), folded."""
    lib = O.load()
    og = C.byref(ogrid(g))
    sp = SpeciesSpec(qom=-4.0, npcel=(2, 2, 2), vth=(0.1,) * 3)
    d = generate_species(g, sp, 0, seed=3)
    nodes = lib.oracle_node_count(og)
    bnode = periodic_node_field(g, 0.3 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    m = np.zeros(126 * nodes)
    lib.oracle_deposit(0, og, sp.qom, 0.5, 1.0, *[O.ptr(d[k]) for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell")],
                       len(d["cell"]), O.ptr(bnode), None, O.ptr(m))
    lib.oracle_fold(og, None, O.ptr(m))
    return m


@pytest.mark.parametrize("g", GRIDS, ids=["3d", "2d", "1d"])
def test_adjoint_solve_is_the_transpose(g):
    lib = O.load()
    og = C.byref(ogrid(g))
    rng = np.random.default_rng(2)
    m = random_mass(g, rng)
    dt, th = 0.5, 0.5
    r1 = periodic_node_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    r2 = periodic_node_field(g, rng.normal(size=(3, g.nz, g.ny, g.nx)))
    zero_b = np.zeros(3 * lib.oracle_cell_count(og))
    x1 = np.zeros_like(r1)
    res = O.OGmres()
    # rhs = E + delta C2N(0) - k 0 = r1.
    assert lib.oracle_field_solve(og, dt, th, 1.0, O.ptr(r1), O.ptr(zero_b), O.ptr(np.zeros_like(r1)), O.ptr(m),
                                  O.ptr(x1), 30, 500, 1e-14, C.byref(res)) == 0
    lam = np.zeros_like(r2)
    assert lib.oracle_adjoint_solve(og, dt, th, 1.0, O.ptr(m), O.ptr(r2), O.ptr(lam), 30, 500, 1e-14,
                                    C.byref(res)) == 0
    lhs, rhs = unique_dot_nodes(g, x1, r2), unique_dot_nodes(g, r1, lam)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
    # A is not symmetric (the response matrix is not), so A^T differs from A.
    lam_plain = np.zeros_like(r2)
    assert lib.oracle_field_solve(og, dt, th, 1.0, O.ptr(r2), O.ptr(zero_b), O.ptr(np.zeros_like(r2)), O.ptr(m),
                                  O.ptr(lam_plain), 30, 500, 1e-14, C.byref(res)) == 0
    assert np.abs(lam_plain - lam).max() > 1e-8 * np.abs(lam).max()


def small_case(g, seed=0):
    species = [SpeciesSpec(qom=-16.0, npcel=(2, 2, 2), vth=(0.08,) * 3),
               SpeciesSpec(qom=1.0, npcel=(2, 2, 2), vth=(0.02,) * 3)]
    arrays = []
    for s, sp in enumerate(species):
        d = generate_species(g, sp, s, seed=seed)
        arrays.append((sp.qom, d))
    return arrays


def run_forward(g, arrays, e0, b0, cycles, dt=0.4, theta=0.5):
    oc = O.OracleCycle(g, [(qom, {k: v.copy() for k, v in d.items()}) for qom, d in arrays], dt, theta, 1.0, 1e-13,
                       0, max_iterations=500, e_node=e0, b_cell=b0)
    oc.prepare()
    energies = oc.energy()
    for _ in range(cycles):
        energies = oc.cycle()
    return oc, energies[0] + energies[1]


def perturbed(g, arrays, e0, b0, direction, s):
    de, db, dparts = direction
    e = e0 + s * de
    b = b0 + s * db
    out = []
    for (qom, d), dp in zip(arrays, dparts):
        d2 = {k: v.copy() for k, v in d.items()}
        for k in ("rx", "ry", "rz", "u", "v", "w", "q"):
            d2[k] = d[k] + s * dp[k]
        out.append((qom, d2))
    return out, e, b


@pytest.mark.parametrize("g,theta", [(GRIDS[0], 0.5), (GRIDS[1], 0.6), (GRIDS[2], 1.0)], ids=["3d", "2d", "1d"])
def test_cycle_adjoint_matches_central_differences(g, theta):
    rng = np.random.default_rng(5)
    arrays = small_case(g)
    e0 = periodic_node_field(g, 0.01 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    b0 = periodic_cell_field(g, 0.0195 + 0.005 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    cycles = 3
    oc, _ = run_forward(g, arrays, e0, b0, 0, theta=theta)
    adj = O.OracleAdjoint(oc)
    adj.forward(cycles)
    e_bar, b_bar = adj.energy_gradient(1.0, 1.0)
    e_grad, b_grad, parts = adj.backward(e_bar, b_bar)
    # A random direction over the whole initial state (records in load order,
    # the arrays' order; the adjoints are indexed by id = load index).
    de = periodic_node_field(g, 0.01 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    db = periodic_cell_field(g, 0.005 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    dparts = []
    predicted = unique_dot_nodes(g, e_grad, de) + unique_dot_cells(g, b_grad, db)
    for (qom, d), pa in zip(arrays, parts):
        n = len(d["q"])
        dp = {k: 0.05 * rng.normal(size=n) for k in ("rx", "ry", "rz")}
        dp.update({k: 0.05 * rng.normal(size=n) for k in ("u", "v", "w")})
        dp["q"] = 0.1 * np.abs(d["q"]) * rng.normal(size=n)
        dparts.append(dp)
        ids = d["id"].astype(np.int64)
        for a, k in enumerate(("rx", "ry", "rz")):
            predicted += float(np.sum(pa["x"][a * n + ids] * dp[k]))
        for a, k in enumerate(("u", "v", "w")):
            predicted += float(np.sum(pa["v"][a * n + ids] * dp[k]))
        predicted += float(np.sum(pa["q"][ids] * dp["q"]))
    s = 1e-5
    lp = run_forward(g, *perturbed(g, arrays, e0, b0, (de, db, dparts), s), cycles, theta=theta)[1]
    lm = run_forward(g, *perturbed(g, arrays, e0, b0, (de, db, dparts), -s), cycles, theta=theta)[1]
    fd = (lp - lm) / (2 * s)
    assert abs(predicted - fd) <= 1e-6 * abs(fd), (predicted, fd)
