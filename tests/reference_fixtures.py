"""Oracle helpers and the reference's test fixtures, restated for the tests.

The fixtures follow the reference's own device tests (file:line in each
docstring); the helpers call the CPU oracle (test infrastructure). Shared by
the GPU parity tests and the CPU tests of the oracle itself.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle as O
from tpic_b200.plasma import GridSpec, SpeciesSpec, generate_species


def ogrid(g):
    return O.OGrid(g.nx, g.ny, g.nz, g.lx / g.nx, g.ly / g.ny, g.lz / g.nz)


def species_arrays(g, precision, seed=3, vth=(0.6, 0.5, 0.4), npcel=(2, 2, 2), qom=-4.0):
    vdt = np.float64 if precision == 0 else np.float32
    d = generate_species(g, SpeciesSpec(qom=qom, npcel=npcel, vth=vth), 0, seed=seed, velocity_dtype=vdt)
    return d


def oracle_mover(g, precision, qom, dt, d, etheta, bnode):
    lib = O.load()
    a = {k: np.ascontiguousarray(v.copy()) for k, v in d.items()}
    bad = lib.oracle_mover(precision, C.byref(ogrid(g)), qom, dt, 1.0, *[O.ptr(a[k]) for k in
                           ("rx", "ry", "rz", "u", "v", "w", "q", "cell")], len(a["cell"]), O.ptr(etheta),
                           O.ptr(bnode))
    return a, bad


def oracle_sort(g, keys):
    lib = O.load()
    n = len(keys)
    nb = lib.oracle_bin_count(C.byref(ogrid(g)))
    perm = np.empty(max(n, 1), np.uint32)
    counts = np.empty(nb, np.uint32)
    offsets = np.empty(nb + 1, np.uint32)
    assert lib.oracle_sort(C.byref(ogrid(g)), O.ptr(np.ascontiguousarray(keys)), n, O.ptr(perm), O.ptr(counts),
                           O.ptr(offsets)) == 0
    return perm[:n], counts, offsets


def oracle_moments(g, precision, qom, dt, d, bnode):
    lib = O.load()
    og = ogrid(g)
    nodes = lib.oracle_node_count(C.byref(og))
    j = np.zeros(3 * nodes)
    m = np.zeros(126 * nodes)
    bad = lib.oracle_deposit(precision, C.byref(og), qom, dt, 1.0, *[O.ptr(np.ascontiguousarray(d[k])) for k in
                             ("rx", "ry", "rz", "u", "v", "w", "q", "cell")], len(d["cell"]),
                             O.ptr(np.ascontiguousarray(bnode)), O.ptr(j), O.ptr(m))
    lib.oracle_fold(C.byref(og), O.ptr(j), O.ptr(m))
    return j, m, bad


def reference_mass_fixture(precision):
    """sorted_mass_device.cpp:190-297 ordinary case: a thin 4x2x2 grid, 16
    cells with occupancies {0,1,3,4,5,31,32,33,65,129,257,64,127,128,130,19},
    fractions (n%17)/17, (n%13)/13, (n%11)/11, charges, beta = -0.07 and
    linear nodal B profiles."""
    g = GridSpec(4, 2, 2, 4.0, 2.0, 2.0)
    occupancy = [0, 1, 3, 4, 5, 31, 32, 33, 65, 129, 257, 64, 127, 128, 130, 19]
    rx, ry, rz, q, keys = [], [], [], [], []
    for compact, occ in enumerate(occupancy):
        i, j, k = compact % 4, (compact // 4) % 2, compact // 8
        for n in range(occ):
            rx.append((n % 17) / 17.0)
            ry.append((n % 13) / 13.0)
            rz.append((n % 11) / 11.0)
            q.append((-0.3 if n % 7 == 0 else 0.8) * (1 + 0.05 * compact))
            keys.append(g.encode(i, j, k))
    total = len(keys)
    vdt = np.float64 if precision == 0 else np.float32
    d = {"rx": np.array(rx), "ry": np.array(ry), "rz": np.array(rz), "u": np.zeros(total, vdt),
         "v": np.zeros(total, vdt), "w": np.zeros(total, vdt), "q": np.array(q), "cell": np.array(keys, np.int32)}
    nodes = (g.nz + 3) * (g.ny + 3) * (g.nx + 3)
    b = np.zeros((3, g.nz + 3, g.ny + 3, g.nx + 3))
    for k in range(3):
        for j in range(3):
            for i in range(5):
                b[0, k + 1, j + 1, i + 1] = 0.2 + 0.07 * i - 0.03 * j + 0.01 * k
                b[1, k + 1, j + 1, i + 1] = -0.4 + 0.02 * i + 0.05 * j - 0.04 * k
                b[2, k + 1, j + 1, i + 1] = 0.7 - 0.01 * i + 0.03 * j + 0.02 * k
    assert b.size == 3 * nodes
    return g, d, b.ravel()


def host_matrix_core_mass(g, d, bnode, beta):
    """Restatement of the fixture oracle host_matrix_core_mass,
    sorted_mass_device.cpp:111-182: an FP64 8x8x9 tensor per cell, flushed to
    the canonical pairs, then summed over periodic copies (this build keeps
    the reference's cell-local nodes only inside the fold)."""
    nodes = (g.nz + 3) * (g.ny + 3) * (g.nx + 3)
    b = bnode.reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)
    result = np.zeros(126 * nodes)
    stencil = [[O.load().oracle_pair_stencil(a, bb) for bb in range(8)] for a in range(8)]
    cells = {}
    for n, key in enumerate(d["cell"]):
        cells.setdefault(int(key), []).append(n)
    for key, members in cells.items():
        yz = key // (g.nx + 4)
        i, j, k = key % (g.nx + 4) - 2, yz % (g.ny + 4) - 2, yz // (g.ny + 4) - 2
        tensor = np.zeros((8, 8, 9))
        for n in members:
            x, y, z = d["rx"][n], d["ry"][n], d["rz"][n]
            w = np.array([((x if a & 1 else 1.0 - x) * (y if a & 2 else 1.0 - y)) * (z if a & 4 else 1.0 - z)
                          for a in range(8)])
            field = np.zeros(3)
            for a in range(8):
                at = (k + ((a >> 2) & 1) + 1, j + ((a >> 1) & 1) + 1, i + (a & 1) + 1)
                field += w[a] * b[:, at[0], at[1], at[2]]
            x_, y_, z_ = beta * field
            inv = 1.0 / (1.0 + (x_ * x_ + y_ * y_ + z_ * z_))
            alpha = np.array([(1 + x_ * x_) * inv, x_ * y_ * inv + z_ * inv, x_ * z_ * inv - y_ * inv,
                              x_ * y_ * inv - z_ * inv, (1 + y_ * y_) * inv, y_ * z_ * inv + x_ * inv,
                              x_ * z_ * inv + y_ * inv, y_ * z_ * inv - x_ * inv, (1 + z_ * z_) * inv])
            scale = beta * d["q"][n]
            tensor += (alpha * scale)[None, None, :] * (w[:, None] * w[None, :])[:, :, None]
        for a in range(8):
            vertex = (i + (a & 1) + 1) + (g.nx + 3) * ((j + ((a >> 1) & 1) + 1) + (g.ny + 3) * (k + ((a >> 2) & 1) + 1))
            for bb in range(8):
                s = stencil[a][bb]
                if s >= 0:
                    result[vertex * 126 + s * 9: vertex * 126 + s * 9 + 9] += tensor[a, bb]
    O.load().oracle_fold(C.byref(ogrid(g)), 0, O.ptr(result))
    return result


def periodic_node_field_records(g, unique):
    k = (np.arange(-1, g.nz + 2) % g.nz)[:, None, None]
    j = (np.arange(-1, g.ny + 2) % g.ny)[None, :, None]
    i = (np.arange(-1, g.nx + 2) % g.nx)[None, None, :]
    return np.stack([unique[e][k, j, i] for e in range(126)], axis=-1).ravel()


def reference_sort_keys(count=1000):
    """The key pattern of the reference's particle sort test,
    key = (i*7 + 3) % 19 (particle_sort_device.cpp:67), on a 2x2x2 grid."""
    return GridSpec(2, 2, 2, 1.0, 1.0, 1.0), (np.arange(count) * 7 + 3) % 19


def mover_edge_records(precision):
    """Endpoint fractions, sub-ULP negative crossings and invalid records, as
    sorted_current_mover_device.cpp:126-140,241-259: a 3x2x2 grid, ten
    records of which four are invalid (halo key, fraction 1, NaN velocity,
    key out of range) and keep every attribute."""
    g = GridSpec(3, 2, 2, 3.0, 2.0, 2.0)
    vdt = np.float64 if precision == 0 else np.float32
    n = 10
    key = lambda i, j, k: g.encode(i, j, k)
    d = {
        "rx": np.array([0.0, 1 - 2**-53, 0.0, 2**-60, 0.25, 0.5, 0.5, 1.0, 0.5, 0.5]),
        "ry": np.full(n, 0.5), "rz": np.full(n, 0.5),
        "u": np.array([0.0, 0.0, -1e-17, -2**-70, 7.3, -9.1, 0.0, 0.0, np.nan, 0.0], dtype=vdt),
        "v": np.array([0.0, 1e-3, 0.0, 0.0, -3.3, 2.2, 0.0, 0.0, 0.0, 0.0], dtype=vdt),
        "w": np.zeros(n, dtype=vdt), "q": np.full(n, -0.1),
        "cell": np.array([key(0, 0, 0), key(2, 1, 1), key(0, 0, 0), key(0, 1, 0), key(1, 1, 1), key(2, 0, 1),
                          key(-1, 0, 0), key(1, 0, 0), key(1, 1, 0), 10**6], dtype=np.int32),
    }
    d["rx"][5] = 0.0
    return g, d
