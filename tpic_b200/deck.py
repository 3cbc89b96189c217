"""TPIC input decks and analytic initial cases over the C ABI.

`parse`/`load` read a TPIC `.inp` deck with TPIC's rules
(src/config/simulation_parameters.cpp:55-200) into a `tpicb200_deck`;
`to_case` turns it into a `plasma.Case` as TPIC's startup does
(src/initialization/initial_case.cpp, include/tpic/initialization/fields/field_image.hpp:30-90):
E sampled at the nodes and B at the cell centres of the whole stored extent,
halos included, at unwrapped coordinates, and each species loaded with its
case profile (charge and drift per particle), QuietStart and
CenterInitialVelocity. The case arithmetic runs in the library
(`tpicb200_case_fields`, `tpicb200_case_profile`).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from .plasma import Case, FieldInit, GridSpec, SpeciesSpec


def parse(text: str) -> _lib.Deck:
    """The deck a TPIC input text describes; raises TpicError (with the line
    and key) on a malformed deck or a case or option not built here."""
    deck = _lib.Deck()
    _lib.check(_lib.load().tpicb200_deck_parse(text.encode(), C.byref(deck)))
    return deck


def load(path) -> _lib.Deck:
    return parse(Path(path).read_text())


def case_name(deck: _lib.Deck) -> str:
    return deck.case_name.decode()


def _f64(a, n):
    return np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (n,)))


def fields_at(deck: _lib.Deck, x, y, z):
    """(E, B) of the case at the points, each (3, n) float64."""
    n = int(np.broadcast(np.asarray(x), np.asarray(y), np.asarray(z)).size)
    xs, ys, zs = _f64(x, n), _f64(y, n), _f64(z, n)
    e = np.empty((3, n), np.float64)
    b = np.empty((3, n), np.float64)
    _lib.check(_lib.load().tpicb200_case_fields(C.byref(deck), n, xs.ctypes.data, ys.ctypes.data, zs.ctypes.data,
                                                e.ctypes.data, b.ctypes.data))
    return e, b


def profile_at(deck: _lib.Deck, species: int, x, y, z, cell_j):
    """(density, multiplier, drift[3, n]) of one species' loading profile at
    the particles' physical positions; cell_j is each particle's y cell."""
    n = int(np.asarray(x).size)
    xs, ys, zs = _f64(x, n), _f64(y, n), _f64(z, n)
    cj = np.ascontiguousarray(np.broadcast_to(np.asarray(cell_j, dtype=np.int32), (n,)))
    density = np.empty(n, np.float64)
    multiplier = np.empty(n, np.float64)
    drift = np.empty((3, n), np.float64)
    _lib.check(_lib.load().tpicb200_case_profile(C.byref(deck), species, n, xs.ctypes.data, ys.ctypes.data,
                                                 zs.ctypes.data, cj.ctypes.data, density.ctypes.data,
                                                 multiplier.ctypes.data, drift.ctypes.data))
    return density, multiplier, drift


def grid_of(deck: _lib.Deck) -> GridSpec:
    g = deck.grid
    return GridSpec(g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)


def _sample(deck: _lib.Deck, grid: GridSpec, nodal: bool):
    """One field over the stored extent (nodes -1..n+1, or cells -1..n per
    axis), x fastest, at unwrapped coordinates (i + offset) * spacing."""
    offset, extra = (0.0, 1) if nodal else (0.5, 0)
    axes = []
    for cells, h in zip((grid.nx, grid.ny, grid.nz), grid.spacing):
        idx = np.arange(-1, cells + extra + 1, dtype=np.float64)
        axes.append((idx + offset) * h)
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    e, b = fields_at(deck, x.reshape(-1), y.reshape(-1), z.reshape(-1))
    return e if nodal else b


def initial_fields(deck: _lib.Deck) -> FieldInit:
    """E at the node-field layout and B at the cell-field layout of
    include/tpicb200.h, halos included, as TPIC's host field image samples them."""
    grid = grid_of(deck)
    return FieldInit(e_node=_sample(deck, grid, True).reshape(-1), b_cell=_sample(deck, grid, False).reshape(-1))


def species_of(deck: _lib.Deck):
    """The deck's species, each loading through its case profile."""
    out = []
    for s in range(deck.ns):
        sp = deck.species[s]

        def profile(x, y, z, cell_j, s=s):
            return profile_at(deck, s, x, y, z, cell_j)

        out.append(SpeciesSpec(qom=sp.qom, rho=sp.rho, npcel=tuple(sp.npcel), vth=tuple(sp.vth),
                               drift=tuple(sp.drift), quiet=bool(deck.quiet_start),
                               center=bool(sp.center_velocity), profile=profile))
    return out


def to_case(deck: _lib.Deck, seed: int = 0, ncycles: int | None = None) -> Case:
    """The run the deck describes, ready for Simulation (and the oracle)."""
    return Case(grid=grid_of(deck), species=species_of(deck), dt=deck.dt, theta=deck.theta, c=deck.c,
                gmres_tol=deck.gmres_tol, ncycles=deck.ncycles if ncycles is None else ncycles,
                fields=initial_fields(deck), seed=seed, deck=deck,
                smoothing=(deck.smooth_iterations, deck.smooth_alpha, deck.smooth_operator))


def deck_of(case: Case) -> _lib.Deck:
    """The deck a case was made from, or, for a case of uniform species
    built in code, the Uniform deck that loads the same records."""
    if case.deck is not None:
        return case.deck
    if any(sp.profile is not None for sp in case.species):
        raise ValueError("a species with a loading profile needs the deck it came from")
    quiet = {bool(sp.quiet) for sp in case.species}
    if len(quiet) > 1:
        raise ValueError("QuietStart applies to every species of a deck")
    if len(case.species) > _lib.MAX_SPECIES:
        raise ValueError("too many species")
    d = _lib.Deck()
    d.case_name = b"Uniform"
    g = case.grid
    d.grid = _lib.Grid(g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)
    d.dt, d.theta, d.c, d.gmres_tol, d.ncycles = case.dt, case.theta, case.c, case.gmres_tol, case.ncycles
    d.ns = len(case.species)
    d.b0[:] = tuple(case.fields.b0)
    d.delta, d.deltax_hump, d.deltay_hump, d.kx_hump, d.ky_hump = 0.5, 8.0, 4.0, -1.0, -1.0
    d.quiet_start = int(quiet.pop()) if quiet else 0
    for s, sp in enumerate(case.species):
        ds = d.species[s]
        ds.rho, ds.qom = sp.rho, sp.qom
        ds.vth[:] = tuple(sp.vth)
        ds.drift[:] = tuple(sp.drift)
        ds.npcel[:] = tuple(sp.npcel)
        ds.center_velocity = int(bool(sp.center))
    return d
