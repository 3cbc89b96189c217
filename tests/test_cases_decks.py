"""Input decks and analytic initial cases, on the host (no GPU).

The startup fields are pinned bit for bit against TPIC's golden table
(tests/data/golden/field_profiles.txt, rows of the cases built here copied to
tests/golden/field_profiles_cases.txt by tests/golden/make_field_profiles.py),
with the fixture parameters of tests/initialization/field_profile_tests.cpp:115-311.
The deck reader follows src/config/simulation_parameters.cpp's rules.
"""
from __future__ import annotations

import math
import struct
from pathlib import Path

import numpy as np
import pytest

from tpic_b200 import _lib, deck as D
from tpic_b200.plasma import GridSpec, SpeciesSpec, generate_species

GOLDEN = Path(__file__).resolve().parent / "golden" / "field_profiles_cases.txt"
DECKS = Path(__file__).resolve().parent.parent / "tpic_b200" / "decks"


def fixture_deck(name: str) -> _lib.Deck:
    """The field-profile fixture (field_profile_tests.cpp:118-190) for one case."""
    d = _lib.Deck()
    d.case_name = name.encode()
    d.grid = _lib.Grid(17, 13, 9, 9.5, 14.25, 5.5)
    d.dt, d.c, d.theta, d.gmres_tol, d.ncycles = .07, 1.7, 1.0, 1e-3, 1
    d.b0[:] = (.19, -.23, .37)
    d.delta, d.harris_b0x = 1.3, -.47
    d.pert_gem, d.pert_hump = 0.0, 0.0
    d.deltax_hump, d.deltay_hump, d.kx_hump, d.ky_hump = 8.0, 4.0, -1.0, -1.0
    d.weibel_mode_x, d.weibel_amplitude, d.weibel_growth_rate = 3, -.043, .71
    d.two_stream_mode_x, d.two_stream_amplitude, d.two_stream_phase = 2, -.13, .29
    d.ns = 3
    for s in range(3):
        sp = d.species[s]
        sp.qom = 1.0 if s == 2 else -64.0
        sp.rho = 1.2 if s == 2 else .6
        sp.vth[:] = (.13, .17, .19)
        sp.drift[:] = (.11 if s == 0 else -.11 if s == 1 else 0.0, 0.0, 0.0)
        sp.npcel[:] = (2, 3, 4)
    return d


def _swap_species(d, a, b):
    sa, sb = _lib.DeckSpecies(), _lib.DeckSpecies()
    C = __import__("ctypes")
    C.memmove(C.byref(sa), C.byref(d.species[a]), C.sizeof(sa))
    C.memmove(C.byref(sb), C.byref(d.species[b]), C.sizeof(sb))
    d.species[a], d.species[b] = sb, sa


def fixtures() -> dict:
    """Label -> deck, for the golden labels of the cases built here
    (field_profile_tests.cpp:207-311)."""
    out = {name: fixture_deck(name) for name in
           ("Weibel", "TwoStream", "plasmoidChain", "DoubleGEM", "DoubleGEMnoPert", "GEM", "GEMnoPert", "Uniform",
            "GEMHarris")}

    def add(name, label, modify):
        d = fixture_deck(name)
        modify(d)
        out[label] = d

    for growth in (0.0, -.31):
        add("Weibel", f"Weibel growth={growth:f}", lambda d, g=growth: setattr(d, "weibel_growth_rate", g))

    def no_weibel(d):
        d.weibel_amplitude, d.weibel_mode_x = 0.0, 0

    def no_two_stream(d):
        d.two_stream_amplitude, d.two_stream_mode_x = 0.0, 0

    def smaller(d):
        d.grid.ny, d.grid.nz = 5, 5

    def hump_only(d):
        d.pert_hump, d.deltax_hump, d.deltay_hump = .11, 2.5, 1.5

    def hump_kx_zero(d):
        d.pert_hump, d.kx_hump, d.ky_hump = .11, 0.0, .9

    def gem_keys(d):
        pi = 3.14159265358979323846
        d.pert_hump = .04 * pi
        d.deltax_hump = d.deltay_hump = 1.0
        d.kx_hump = d.ky_hump = pi / (10.0 * d.delta)

    add("Weibel", "Weibel no seed", no_weibel)
    add("TwoStream", "TwoStream no seed", no_two_stream)
    add("TwoStream", "TwoStream reordered species", lambda d: _swap_species(d, 0, 2))
    add("GEM", "Harris no sheet field", lambda d: setattr(d, "harris_b0x", 0.0))
    add("DoubleGEM", "Double Harris positive amplitude", lambda d: setattr(d, "harris_b0x", .71))
    add("Uniform", "Uniform smaller transverse axes", smaller)
    add("GEMHarris", "GEMHarris mode only", lambda d: setattr(d, "pert_gem", .09))
    add("GEMHarris", "GEMHarris hump only", hump_only)
    add("GEMHarris", "GEMHarris hump kx zero", hump_kx_zero)
    add("GEMHarris", "GEMHarris GEM keys", gem_keys)
    return out


def sample_points(d):
    """field_profile_tests.cpp:315-322 (the flux-rope centre is the fixture's 3.17, 5.91)."""
    lx, ly, lz = d.grid.lx, d.grid.ly, d.grid.lz
    return [(0.0, 0.0, 0.0), (lx * .5, ly * .5, lz * .5), (lx * .25 + .37, ly * .25 - .21, .17),
            (lx * .75 - .31, ly * .75 + .19, .71), (3.17, 5.91, .23), (lx * .5 + .13, ly * .5 - .29, -.11)]


def bits(v: float) -> int:
    return struct.unpack("<q", struct.pack("<d", v))[0]


def golden_rows():
    rows = {}
    for line in GOLDEN.read_text().splitlines():
        label, point, field, *values = line.split("\t")
        rows[(label, int(point), field)] = [float.fromhex(v) for v in values]
    return rows


def test_golden_table_covers_the_built_cases():
    labels = {k[0] for k in golden_rows()}
    assert labels == set(fixtures())
    assert len(golden_rows()) == 12 * len(labels)


@pytest.mark.parametrize("label", sorted(fixtures()))
def test_case_fields_match_the_golden_table_bit_for_bit(label):
    d = fixtures()[label]
    rows = golden_rows()
    pts = np.array(sample_points(d))
    e, b = D.fields_at(d, pts[:, 0], pts[:, 1], pts[:, 2])
    for p in range(6):
        for field, got in (("B", b[:, p]), ("E", e[:, p])):
            want = rows[(label, p, field)]
            assert [bits(float(g)) for g in got] == [bits(w) for w in want], (label, p, field, got, want)


def test_seeded_gem_is_the_x_point_expression():
    """The fixed GEM seed written out (field_profile_tests.cpp:398-446): a
    Gaussian X-point hump of amplitude 0.4 B_H around the sheet centre."""
    d = fixtures()["GEM"]
    lx, ly, delta, b_h = d.grid.lx, d.grid.ly, d.delta, d.harris_b0x
    for x, y, z in sample_points(d):
        _, b = D.fields_at(d, x, y, z)
        xp, yp = x - .5 * lx, y - .5 * ly
        env = math.exp(-(xp / delta) ** 2 - (yp / delta) ** 2)
        cx, sx = math.cos(math.pi * xp / 10.0 / delta), math.sin(math.pi * xp / 10.0 / delta)
        cy, sy = math.cos(math.pi * yp / 10.0 / delta), math.sin(math.pi * yp / 10.0 / delta)
        bx = b_h * math.tanh(yp / delta) + b_h * 0.4 * env * (-cx * cy * 2.0 * yp / delta - cx * sy * math.pi / 10.0)
        by = b_h * 0.4 * env * (cx * cy * 2.0 * xp / delta + sx * cy * math.pi / 10.0)
        assert b[0, 0] == pytest.approx(bx + d.b0[0], rel=1e-13, abs=1e-15)
        assert b[1, 0] == pytest.approx(by + d.b0[1], rel=1e-13, abs=1e-15)
        assert b[2, 0] == d.b0[2]


def test_profiles():
    """Loading profiles: the TwoStream electron density seed, the Harris
    sech^2 density averaged over the cell's two y nodes (drifting species
    only) and the double sheet's drift reversal (cases/harris_sheet.hpp:68-106,
    cases/two_stream.hpp:14-24)."""
    ts = fixtures()["TwoStream"]
    x = np.array([0.0, 1.3, 4.7])
    dens, mult, drift = D.profile_at(ts, 0, x, x, x, np.zeros(3, np.int32))
    k = 2 * math.pi * 2 / ts.grid.lx
    np.testing.assert_array_equal(mult, 1.0 + ts.two_stream_amplitude * np.cos(k * x + ts.two_stream_phase))
    np.testing.assert_array_equal(dens, np.full(3, .6 / (4 * math.pi)))
    np.testing.assert_array_equal(drift[0], np.full(3, .11))
    dens, mult, _ = D.profile_at(ts, 2, x, x, x, np.zeros(3, np.int32))
    np.testing.assert_array_equal(mult, np.ones(3))

    for name in ("GEM", "DoubleGEM"):
        h = fixtures()[name]
        ly, delta, dy = h.grid.ly, h.delta, h.grid.ly / h.grid.ny
        cj = np.arange(h.grid.ny, dtype=np.int32)
        y = (cj + 0.5) * dy
        dens, mult, drift = D.profile_at(h, 0, y, y, y, cj)

        def shape(v):
            if name == "DoubleGEM":
                return 1 / np.cosh((v - .25 * ly) / delta) ** 2 + 1 / np.cosh((v - .75 * ly) / delta) ** 2
            return 1 / np.cosh((v - .5 * ly) / delta) ** 2

        want = .6 / (4 * math.pi) * 0.5 * (shape(cj * dy) + shape(cj * dy + dy))
        np.testing.assert_allclose(dens, want, rtol=1e-14)
        assert np.all(mult == 1.0)
        dens_ion, _, _ = D.profile_at(h, 2, y, y, y, cj)
        np.testing.assert_array_equal(dens_ion, np.full(h.grid.ny, 1.2 / (4 * math.pi)))
    d2 = fixtures()["DoubleGEM"]
    d2.species[0].drift[:] = (0.0, 0.0, .3)
    y = np.array([1.0, 7.125, 13.0])
    _, _, drift = D.profile_at(d2, 0, y, y, y, np.zeros(3, np.int32))
    np.testing.assert_allclose(drift[2], .3 * -np.tanh((y - 7.125) / d2.delta), rtol=1e-15)


def test_initial_fields_cover_the_stored_extent():
    d = fixtures()["Weibel"]
    f = D.initial_fields(d)
    nx, ny, nz = d.grid.nx, d.grid.ny, d.grid.nz
    nodes, cells = (nx + 3) * (ny + 3) * (nz + 3), (nx + 2) * (ny + 2) * (nz + 2)
    assert f.e_node.shape == (3 * nodes,) and f.b_cell.shape == (3 * cells,)
    dx = d.grid.lx / nx
    e = f.e_node.reshape(3, nz + 3, ny + 3, nx + 3)
    b = f.b_cell.reshape(3, nz + 2, ny + 2, nx + 2)
    # Node i at x = i dx (the halo node -1 at x = -dx, unwrapped); cell centres at (i + 1/2) dx.
    for i in (-1, 0, 5, nx, nx + 1):
        ev, _ = D.fields_at(d, i * dx, 0.0, 0.0)
        assert e[1, 1, 1, i + 1] == ev[1, 0]
    for i in (-1, 0, nx):
        _, bv = D.fields_at(d, (i + .5) * dx, .5 * d.grid.ly / ny, .5 * d.grid.lz / nz)
        assert b[2, 1, 1, i + 1] == bv[2, 0]


DECK_TEXT = """
# a comment line
Case = Weibel
dt = 0.125     # trailing comment
ncycles = 3
ncycles = 4
ns = 2
nxc = 8
nyc = 4
nzc = 1
Lx = 6.0
Ly = 3.0
Lz = 0.75
qom = -1 1 99
rhoINIT = 1 1
npcelx = 2 2
npcely = 2 2
npcelz = 1 1
uth = .1 .1
vth = .1 .1
wth = .3 .3
u0 = 0 0
v0 = 0 0
w0 = 0 0
CenterInitialVelocity = true false
QuietStart = 1
WeibelSeedModeX = 1
WeibelSeedAmplitude = 1e-3
XLEN = 2
SaveDirName = out
"""


def test_deck_reader_rules():
    d = D.parse(DECK_TEXT)
    assert D.case_name(d) == "Weibel"
    assert (d.dt, d.ncycles, d.ns) == (0.125, 4, 2)           # last assignment wins
    assert (d.grid.nx, d.grid.ny, d.grid.nz, d.grid.lx, d.grid.ly, d.grid.lz) == (8, 4, 1, 6.0, 3.0, 0.75)
    assert [d.species[s].qom for s in range(2)] == [-1.0, 1.0]  # extra list entries are ignored
    assert d.species[0].center_velocity == 1 and d.species[1].center_velocity == 0
    assert d.quiet_start == 1
    assert (d.theta, d.c, d.gmres_tol, d.delta) == (1.0, 1.0, 1e-3, 0.5)  # defaults
    assert d.ignored_keys == 2                                   # XLEN, SaveDirName
    assert d.weibel_growth_rate == 0.0


def test_deck_reads_energy_conserving_smoothing():
    text = DECK_TEXT + ("ECSimSmoothing = energy_conserving\nSmooth = 0.5\nSmoothNiter = 2\n"
                        "ECSimSmoothingOperator = binomial27\n")
    d = D.parse(text)
    assert (d.smooth_iterations, d.smooth_alpha, d.smooth_operator) == (2, 0.5, 1)
    assert D.to_case(d).smoothing == (2, 0.5, 1)
    # Defaults: six Face7 passes; Smooth = 1 (the default) leaves smoothing off.
    d = D.parse(DECK_TEXT + "ECSimSmoothing = energy_conserving\nSmooth = 0.25\n")
    assert (d.smooth_iterations, d.smooth_alpha, d.smooth_operator) == (6, 0.25, 0)
    d = D.parse(DECK_TEXT + "ECSimSmoothing = energy_conserving\n")
    assert d.smooth_iterations == 0 and D.to_case(d).smoothing == (0, 1.0, 0)
    assert D.parse(DECK_TEXT).smooth_iterations == 0


@pytest.mark.parametrize("extra, message", [
    ("ECSimSmoothing = energy_conserving\nSmooth = 1.5\n", "Smooth"),
    ("ECSimSmoothing = energy_conserving\nSmoothNiter = -1\n", "SmoothNiter"),
    ("ECSimSmoothing = energy_conserving\nECSimSmoothingOperator = face9\n", "ECSimSmoothingOperator"),
])
def test_deck_smoothing_errors(extra, message):
    with pytest.raises(_lib.TpicError) as err:
        D.parse(DECK_TEXT + extra)
    assert err.value.status == _lib.INVALID_ARGUMENT
    assert message in str(err.value)


@pytest.mark.parametrize("edit, message", [
    (lambda t: t.replace("dt = 0.125", ""), "dt"),
    (lambda t: t.replace("Case = Weibel", "Case = Whistler"), "Whistler"),
    (lambda t: t.replace("rhoINIT = 1 1", "rhoINIT = 1"), "rhoINIT"),
    (lambda t: t.replace("nxc = 8", "nxc = 8x"), "nxc"),
    (lambda t: t.replace("QuietStart = 1", "QuietStart = yes"), "QuietStart"),
    (lambda t: t + "PERIODICY = false\n", "PERIODICY"),
    (lambda t: t + "ECSimSmoothing = binomial\n", "ECSimSmoothing"),
    (lambda t: t + "nsTestPart = 1\n", "nsTestPart"),
    (lambda t: t + "just a line\n", "key = value"),
    (lambda t: t.replace("WeibelSeedModeX = 1", "WeibelSeedModeX = 0"), "WeibelSeedModeX"),
])
def test_deck_errors(edit, message):
    with pytest.raises(_lib.TpicError) as err:
        D.parse(edit(DECK_TEXT))
    assert err.value.status == _lib.INVALID_ARGUMENT
    assert message in str(err.value)


def test_two_stream_admission():
    d = fixtures()["TwoStream"]
    d.species[1].drift[0] = .12   # not equal and opposite
    with pytest.raises(_lib.TpicError):
        D.fields_at(d, 0.0, 0.0, 0.0)


@pytest.mark.parametrize("path", sorted(DECKS.glob("*.inp")), ids=lambda p: p.name)
def test_shipped_decks_parse(path):
    d = D.load(path)
    assert d.ignored_keys == 0, path
    case = D.to_case(d, ncycles=1)
    assert case.grid.cells == d.grid.nx * d.grid.ny * d.grid.nz


def test_velocity_centring():
    """CenterInitialVelocity (particle_centering_device.hpp:36-100): the
    charge-weighted mean of v - drift vanishes, the drift stays."""
    g = GridSpec(6, 4, 2, 3.0, 2.0, 1.0)
    sp = SpeciesSpec(qom=-1.0, npcel=(2, 2, 1), vth=(.3, .2, .1), drift=(.05, 0.0, -.02), center=True)
    raw = generate_species(g, SpeciesSpec(qom=-1.0, npcel=(2, 2, 1), vth=(.3, .2, .1), drift=(.05, 0.0, -.02)),
                           0, seed=5)
    d = generate_species(g, sp, 0, seed=5)
    for k, drift in zip("uvw", (.05, 0.0, -.02)):
        mean = np.sum(d["q"] * (d[k] - drift)) / np.sum(d["q"])
        assert abs(mean) < 1e-15
        assert abs(np.mean(raw[k] - drift)) > 1e-4   # the sample had a mean to remove
    np.testing.assert_array_equal(d["rx"], raw["rx"])
