"""The oracle pinned against the reference itself (CPU, no GPU).

oracle/Makefile compiles the reference's own header-only numerics into
oracle/_ref/libtpicref.so (oracle/refpin/refpin.cpp only calls them). Every
shared building block of the path must agree with it bit for bit: CIC
weights (ecsim/particles/cic.hpp:24-36), the particle response
(ecsim/particles/particle_response.hpp:16-42), the canonical pair stencils and
their offsets (ecsim/mass_matrix/mass_matrix_stencil.hpp:13-40,
data/mass_matrix/mass_matrix_layout.hpp:17-24), the cell keys
(data/particles/particle_cell.hpp:34-46), both curls
(ecsim/fields/node_cell_curl.hpp:116-126), the cell-to-node average
(ecsim/fields/cell_to_node.hpp:19-32) and the mass apply
(ecsim/mass_matrix/mass_matrix_stencil.hpp:119-149)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from fieldutil import bits, periodic_cell_field, periodic_node_field, smooth_random_unique
from reference_fixtures import ogrid, periodic_node_field_records
from tpic_b200.plasma import GridSpec


@pytest.fixture(scope="module")
def ref():
    lib = O.load_reference()
    if lib is None:
        pytest.skip("the reference pin library was not built (no reference tree on this host)")
    return lib


@pytest.fixture(scope="module")
def orc():
    return O.load()


def edge_fractions(rng, n, dtype):
    eps = np.finfo(dtype).eps
    special = np.array([0.0, 0.5, 1.0 - eps / 2, 1.0 - eps, eps, 0.25, 0.75], dtype=dtype)
    return np.concatenate([special, rng.random(n).astype(dtype)])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cic_weights(ref, orc, dtype):
    rng = np.random.default_rng(1)
    f = edge_fractions(rng, 300, dtype)
    name = "f64" if dtype == np.float64 else "f32"
    want, got = np.zeros(8, dtype), np.zeros(8, dtype)
    for x, y, z in zip(f, np.roll(f, 3), np.roll(f, 7)):
        getattr(ref, f"ref_cic_weights_{name}")(x, y, z, O.ptr(want))
        getattr(orc, f"oracle_cic_weights_{name}")(x, y, z, O.ptr(got))
        assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_particle_response(ref, orc, dtype):
    rng = np.random.default_rng(2)
    name = "f64" if dtype == np.float64 else "f32"
    want, got = np.zeros(9, dtype), np.zeros(9, dtype)
    cases = [(0.0, 0.0, 0.0, 0.3), (1.0, -2.0, 0.5, 0.0), (1e3, 1e-3, -7.0, 2.5)]
    cases += [tuple(rng.normal(scale=s, size=3)) + (rng.normal(),) for s in (0.01, 1.0, 30.0) for _ in range(60)]
    for bx, by, bz, boc in cases:
        getattr(ref, f"ref_response_{name}")(dtype(bx), dtype(by), dtype(bz), dtype(boc), O.ptr(want))
        getattr(orc, f"oracle_response_{name}")(dtype(bx), dtype(by), dtype(bz), dtype(boc), O.ptr(got))
        assert np.array_equal(bits(got), bits(want))


def test_pair_stencils_and_offsets(ref, orc):
    for a in range(8):
        for b in range(8):
            assert orc.oracle_pair_stencil(a, b) == ref.ref_pair_stencil(a, b)
    # 36 canonical pairs: 8 centre, 28 off-centre (each unordered pair once).
    owned = [(a, b) for a in range(8) for b in range(8) if orc.oracle_pair_stencil(a, b) >= 0]
    assert len(owned) == 36
    want, got = np.zeros(3, np.int32), np.zeros(3, np.int32)
    for s in range(14):
        ref.ref_stencil_offset(s, O.ptr(want))
        orc.oracle_stencil_offset(s, O.ptr(got))
        assert np.array_equal(got, want)


def test_cell_keys(ref):
    """The product's key encoding (tpic_b200.plasma.GridSpec.encode, the same
    expression as Geom::encode) against the reference's ParticleCellMap."""
    g = GridSpec(7, 5, 3, 1.0, 1.0, 1.0)
    out = np.zeros(3, np.int32)
    for i in range(-2, g.nx + 2):
        for j in range(-2, g.ny + 2):
            for k in range(-2, g.nz + 2):
                key = ref.ref_encode_key(g.nx, g.ny, g.nz, i, j, k)
                assert key == g.encode(i, j, k)
                ref.ref_decode_key(g.nx, g.ny, g.nz, key, O.ptr(out))
                assert tuple(out) == (i, j, k)


def test_curls_and_cell_to_node(ref, orc):
    g = GridSpec(5, 4, 3, 2.5, 2.0, 3.0)
    rng = np.random.default_rng(3)
    node = periodic_node_field(g, smooth_random_unique(g, rng, 1.0))
    cell = periodic_cell_field(g, smooth_random_unique(g, rng, 1.0))
    og = ogrid(g)
    ncell = (g.nx + 2) * (g.ny + 2) * (g.nz + 2)
    nnode = (g.nx + 3) * (g.ny + 3) * (g.nz + 3)
    curl_c = np.zeros(3 * ncell)
    curl_n = np.zeros(3 * nnode)
    c2n = np.zeros(3 * nnode)
    orc.oracle_curl_n2c(C.byref(og), O.ptr(node), O.ptr(curl_c))
    orc.oracle_curl_c2n(C.byref(og), O.ptr(cell), O.ptr(curl_n))
    orc.oracle_cell_to_node(C.byref(og), O.ptr(cell), O.ptr(c2n))
    inv = (g.nx / g.lx, g.ny / g.ly, g.nz / g.lz)
    o = np.zeros(3)
    for k in range(g.nz):
        for j in range(g.ny):
            for i in range(g.nx):
                ref.ref_curl_n2c(g.nx, g.ny, g.nz, O.ptr(node), *inv, i, j, k, O.ptr(o))
                at = (i + 1) + (g.nx + 2) * ((j + 1) + (g.ny + 2) * (k + 1))
                assert np.array_equal(bits(curl_c[at::ncell][:3]), bits(o))
    for k in range(g.nz + 1):
        for j in range(g.ny + 1):
            for i in range(g.nx + 1):
                ref.ref_curl_c2n(g.nx, g.ny, g.nz, O.ptr(cell), *inv, i, j, k, O.ptr(o))
                at = (i + 1) + (g.nx + 3) * ((j + 1) + (g.ny + 3) * (k + 1))
                assert np.array_equal(bits(curl_n[at::nnode][:3]), bits(o))
                for comp in range(3):
                    avg = ref.ref_cell_to_node(g.nx, g.ny, O.ptr(cell[comp * ncell:]), i, j, k)
                    assert bits(np.array([c2n[comp * nnode + at]]))[0] == bits(np.array([avg]))[0]


def test_mass_apply(ref, orc):
    g = GridSpec(4, 3, 5, 2.0, 1.5, 2.5)
    rng = np.random.default_rng(4)
    m = periodic_node_field_records(g, rng.normal(size=(126, g.nz, g.ny, g.nx)))
    v = periodic_node_field(g, smooth_random_unique(g, rng, 1.0))
    nnode = (g.nx + 3) * (g.ny + 3) * (g.nz + 3)
    out = np.zeros(3 * nnode)
    orc.oracle_mass_apply(0, C.byref(ogrid(g)), O.ptr(m), O.ptr(v), O.ptr(out))
    volume = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    o = np.zeros(3)
    for k in range(g.nz + 1):
        for j in range(g.ny + 1):
            for i in range(g.nx + 1):
                ref.ref_mass_apply_node(g.nx, g.ny, g.nz, O.ptr(m), O.ptr(v), 1.0 / volume, i, j, k, O.ptr(o))
                at = (i + 1) + (g.nx + 3) * ((j + 1) + (g.ny + 3) * (k + 1))
                assert np.allclose(out[at::nnode][:3], o, rtol=1e-14, atol=1e-14)


def reference_serial_sort(ref, g, keys):
    n = len(keys)
    nb = (g.nx + 4) * (g.ny + 4) * (g.nz + 4)
    perm = np.empty(max(n, 1), np.uint32)
    counts = np.empty(nb, np.uint32)
    offsets = np.empty(nb + 1, np.uint32)
    ref.ref_serial_sort.restype = C.c_int
    ref.ref_serial_sort.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
    status = ref.ref_serial_sort(O.ptr(np.ascontiguousarray(keys, dtype=np.int32)), n, nb, O.ptr(perm),
                                 O.ptr(counts), O.ptr(offsets))
    assert status == 0, status
    return perm[:n], counts, offsets


@pytest.mark.parametrize("case", ["reference_pattern", "random", "halo_keys", "one_bin", "single", "ragged"])
def test_sort_matches_the_reference_serial_sort(ref, case):
    """The oracle's stable counting sort against the reference's own
    PreparedSerialParticleSort::run (lpfx/algorithm/particle/host/sort.hpp:205-290),
    compiled from its header: permutation, counts and offsets bit for bit.
    Cases: the key pattern of the reference's sort test, random interior
    keys, keys spread over the halo-2 bins too, every record in one bin, one
    record, and a grid with very uneven bins."""
    from reference_fixtures import oracle_sort, reference_sort_keys
    rng = np.random.default_rng(7)
    if case == "reference_pattern":
        g, keys = reference_sort_keys(1000)
    elif case == "random":
        g = GridSpec(7, 5, 6, 1.0, 1.0, 1.0)
        keys = g.encode(rng.integers(0, g.nx, 20000), rng.integers(0, g.ny, 20000), rng.integers(0, g.nz, 20000))
    elif case == "halo_keys":
        g = GridSpec(4, 3, 5, 1.0, 1.0, 1.0)
        keys = rng.integers(0, (g.nx + 4) * (g.ny + 4) * (g.nz + 4), 5000)
    elif case == "one_bin":
        g = GridSpec(3, 3, 3, 1.0, 1.0, 1.0)
        keys = np.full(777, g.encode(1, 2, 0))
    elif case == "single":
        g = GridSpec(2, 2, 2, 1.0, 1.0, 1.0)
        keys = np.array([g.encode(1, 0, 1)])
    else:
        g = GridSpec(9, 4, 3, 1.0, 1.0, 1.0)
        cells = rng.integers(0, 3, 30000) ** 3 % (g.nx * g.ny * g.nz)
        keys = g.encode(cells % g.nx, (cells // g.nx) % g.ny, cells // (g.nx * g.ny))
    keys = np.asarray(keys, dtype=np.int32)
    want = reference_serial_sort(ref, g, keys)
    got = oracle_sort(g, keys)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    # Stability: equal keys keep their input order.
    perm = got[0]
    same = keys[perm][1:] == keys[perm][:-1]
    assert np.all(perm[1:][same] > perm[:-1][same])
