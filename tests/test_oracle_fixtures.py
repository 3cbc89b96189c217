"""The oracle against the reference's own test fixtures (CPU, no GPU):
the particle-sort key pattern (particle_sort_device.cpp:67), the mover's
endpoint, sub-ULP and long-flight cases (sorted_current_mover_device.cpp:126-140,
241-290) and the sorted-mass occupancy fixture checked against the restated
host_matrix_core_mass (sorted_mass_device.cpp:111-182,190-297)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from fieldutil import bits, interior_records
from reference_fixtures import (host_matrix_core_mass, mover_edge_records, ogrid, oracle_mover, oracle_sort,
                                reference_mass_fixture, reference_sort_keys)
from tpic_b200.plasma import GridSpec


def test_sort_reference_key_pattern():
    g, keys = reference_sort_keys()
    perm, counts, offsets = oracle_sort(g, keys.astype(np.int32))
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))
    nb = (g.nx + 4) * (g.ny + 4) * (g.nz + 4)
    assert np.array_equal(counts, np.bincount(keys, minlength=nb))
    assert np.array_equal(offsets, np.concatenate([[0], np.cumsum(counts)]))


@pytest.mark.parametrize("precision", [0, 1])
def test_mover_edge_records(precision):
    g, d = mover_edge_records(precision)
    nodes = (g.nx + 3) * (g.ny + 3) * (g.nz + 3)
    vdt = np.float64 if precision == 0 else np.float32
    got, bad = oracle_mover(g, precision, -1.0, 0.5, d, np.zeros(3 * nodes), np.zeros(3 * nodes, vdt))
    assert bad == 4  # halo key, fraction 1, NaN velocity, key out of range
    for r in (6, 7, 8, 9):  # invalid records keep every attribute
        assert got["cell"][r] == d["cell"][r]
        for k in ("rx", "u", "v"):
            assert bits(got[k])[r] == bits(d[k])[r]
    assert ((got["rx"][:6] >= 0) & (got["rx"][:6] < 1)).all()
    # A tiny negative crossing from the left face rounds up to the endpoint and
    # is carried back: same cell, fraction exactly zero.
    assert got["cell"][2] == d["cell"][2] and got["rx"][2] == 0.0


@pytest.mark.parametrize("precision", [0, 1])
def test_mover_sub_ulp_crossing_and_long_flights(precision):
    """With E = B = 0 the velocity is unchanged; a sub-ULP negative crossing
    stays canonical, and whole-domain flights fold periodically."""
    g = GridSpec(8, 3, 2, 8.0, 3.0, 2.0)
    vdt = np.float64 if precision == 0 else np.float32
    d = {"rx": np.array([0.0, 0.25]), "ry": np.array([0.5, 0.25]), "rz": np.array([0.5, 0.25]),
         "u": np.array([-1e-30, 2 * g.nx + 0.5], vdt), "v": np.array([0.0, -(2 * g.ny + 1.5)], vdt),
         "w": np.array([0.0, -(2 * g.nz + 0.5)], vdt), "q": np.array([-1.0, 0.5]),
         "cell": np.array([g.encode(3, 1, 1), g.encode(0, 0, 0)], np.int32)}
    nodes = (g.nx + 3) * (g.ny + 3) * (g.nz + 3)
    got, bad = oracle_mover(g, precision, 0.0, 1.0, d, np.zeros(3 * nodes), np.zeros(3 * nodes, vdt))
    assert bad == 0
    assert got["cell"][0] == g.encode(3, 1, 1) and got["rx"][0] == 0.0
    # 0.25 + 16.5 -> cell 16 = 0 (mod 8), 0.75; 0.25 - 7.5 -> -8 = 1 (mod 3)
    # with 0.75; 0.25 - 4.5 -> -5 = 1 (mod 2) with 0.75.
    assert got["cell"][1] == g.encode(0, 1, 1)
    assert (got["rx"][1], got["ry"][1], got["rz"][1]) == (0.75, 0.75, 0.75)
    assert np.array_equal(bits(got["u"]), bits(d["u"]))


def test_reference_mass_fixture():
    g, d, bnode = reference_mass_fixture(0)
    want = host_matrix_core_mass(g, d, bnode, -0.07)
    lib = O.load()
    og = ogrid(g)
    nodes = lib.oracle_node_count(C.byref(og))
    j = np.zeros(3 * nodes)
    m = np.zeros(126 * nodes)
    bad = lib.oracle_deposit(0, C.byref(og), -1.0, 0.14, 1.0, *[O.ptr(np.ascontiguousarray(d[k])) for k in
                             ("rx", "ry", "rz", "u", "v", "w", "q", "cell")], len(d["cell"]), O.ptr(bnode),
                             O.ptr(j), O.ptr(m))
    assert bad == 0
    lib.oracle_fold(C.byref(og), O.ptr(j), O.ptr(m))
    wi, gi = interior_records(g, want), interior_records(g, m)
    assert np.abs(gi - wi).max() <= 3e-12 * np.abs(wi).max() + 1e-15
    assert np.abs(j).max() == 0.0  # the fixture's particles are at rest
