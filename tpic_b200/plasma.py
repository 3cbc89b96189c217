"""Seeded synthetic plasmas for the ECSIM cycle.

TPIC loads particles with cuRAND's XORWOW stream
(initialization/particles/particle_loading_device.hpp:32-53); that generator
is not reproduced. This module defines its own counter-based stream,
Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
as 1, 2, 3", SC'11). `generate_species` is its host (numpy) form, which
feeds the CPU oracle and the tests; the library's loader
(tpicb200_load_species) is the device form of the same stream.

Per particle with global load index `n` of species `s`:
  block A = philox((n_lo, n_hi, s, 0), seed) -> subcell offsets x, y, z and u1
  block B = philox((n_lo, n_hi, s, 1), seed) -> u2, u3, u4
  uniforms are (r + 0.5) * 2**-32, normals come from Box-Muller:
  (n0, n1) from (u1, u2), n2 from (u3, u4).
The load order follows TPIC's dense path (particle_loading_device.hpp:85-120):
cell = n // ppc (x fastest), subcell = n % ppc (x fastest), fraction =
(subcell + offset) / npcel on each axis, a stored fraction of exactly one
carries into the next cell; velocity = drift + thermal * normal; macro-charge
q = sign(qom) * V/ppc * rho/(4 pi) (src/initialization/prepared_initialization.cpp:36-70),
shaped by a case profile where the species has one.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32(c0, c1, c2, c3, k0: int, k1: int, xp=np):
    """Philox-4x32-10 on int64 arrays holding 32-bit words (numpy or torch).

    The 32x32-bit products may wrap in int64; their low 64 bits are exact, and
    the arithmetic shift followed by the 32-bit mask recovers the high word."""
    for _ in range(10):
        p0 = c0 * M0
        p1 = c2 * M1
        hi0, lo0 = (p0 >> 32) & MASK, p0 & MASK
        hi1, lo1 = (p1 >> 32) & MASK, p1 & MASK
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + W0) & MASK
        k1 = (k1 + W1) & MASK
    return c0, c1, c2, c3


def _uniform(r):
    return r.astype(np.float64) * 2.0**-32 + 2.0**-33


@dataclass
class SpeciesSpec:
    """One species' loading: q/m, rhoINIT, particles per cell per axis,
    thermal speeds and drift. quiet: particles at their subcell centres
    (TPIC's QuietStart). center: the charge-weighted mean of the sampled
    velocities is removed around the loaded drift (CenterInitialVelocity).
    profile: a case's loading profile, profile(x, y, z, cell_j) ->
    (density, multiplier, drift[3, n]) at the particles' physical positions
    (None: uniform, density rho/(4 pi))."""
    qom: float
    rho: float = 1.0
    npcel: tuple = (2, 2, 2)
    vth: tuple = (0.0, 0.0, 0.0)
    drift: tuple = (0.0, 0.0, 0.0)
    quiet: bool = False
    center: bool = False
    profile: object = None

    @property
    def ppc(self) -> int:
        return int(self.npcel[0] * self.npcel[1] * self.npcel[2])


@dataclass
class GridSpec:
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float

    @property
    def spacing(self):
        return (self.lx / self.nx, self.ly / self.ny, self.lz / self.nz)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def encode(self, i, j, k):
        return (i + 2) + (self.nx + 4) * ((j + 2) + (self.ny + 4) * (k + 2))


def generate_species(grid: GridSpec, sp: SpeciesSpec, species_index: int, seed: int = 0,
                     velocity_dtype=np.float64, first: int = 0, count: int | None = None) -> dict:
    """Records [first, first+count) of one species, in load order, on the
    host (numpy). The library's loader (tpicb200_load_species) produces the
    same records on the device: positions, keys and ids bit for bit,
    velocities and charges to the last bits of log/cos/sin/cosh.
    """
    ppc = sp.ppc
    total = grid.cells * ppc
    if count is None:
        count = total - first
    k0, k1 = seed & MASK, (seed >> 32) & MASK
    n = np.arange(first, first + count, dtype=np.int64)
    zeros = np.zeros_like(n)
    ones = np.ones_like(n)
    sidx = np.full_like(n, species_index)
    lo, hi = n & MASK, (n >> 32) & MASK
    a = philox4x32(lo, hi, sidx, zeros, k0, k1)
    b = philox4x32(lo, hi, sidx, ones, k0, k1)
    cell = n // ppc
    sub = n % ppc
    npx, npy, npz = sp.npcel
    sub_x, sub_y, sub_z = sub % npx, (sub // npx) % npy, sub // (npx * npy)
    ci, cj, ck = cell % grid.nx, (cell // grid.nx) % grid.ny, cell // (grid.nx * grid.ny)
    out = {}
    cells = [ci, cj, ck]
    fr = []
    for axis, (s, r, npc) in enumerate(zip((sub_x, sub_y, sub_z), a[:3], (npx, npy, npz))):
        off = np.full_like(_uniform(r), 0.5) if sp.quiet else _uniform(r)
        f = (s.astype(np.float64) + off) * (1.0 / npc)
        carry = f >= 1.0
        f = np.where(carry, np.zeros_like(f), f)
        cells[axis] = cells[axis] + carry.astype(np.int64)
        fr.append(f)
    extents = (grid.nx, grid.ny, grid.nz)
    for axis in range(3):
        cells[axis] = cells[axis] % extents[axis]
    u1, u2, u3, u4 = _uniform(a[3]), _uniform(b[0]), _uniform(b[1]), _uniform(b[2])
    r12 = np.sqrt(-2.0 * np.log(u1))
    r34 = np.sqrt(-2.0 * np.log(u3))
    normals = (r12 * np.cos(2.0 * math.pi * u2), r12 * np.sin(2.0 * math.pi * u2),
               r34 * np.cos(2.0 * math.pi * u4))
    dx, dy, dz = grid.spacing
    volume = (dx * dy) * dz
    q_factor = (1.0 if sp.qom > 0 else -1.0) * volume / ppc
    drift = [np.full(count, sp.drift[axis]) for axis in range(3)]
    if sp.profile is not None:
        # The case profile at the stored position and cell (after the
        # endpoint carry), as TPIC's loader evaluates it
        # (particle_loading_device.hpp:120-143): q = (q_factor*density)*multiplier.
        x = (cells[0] + fr[0]) * dx
        y = (cells[1] + fr[1]) * dy
        z = (cells[2] + fr[2]) * dz
        density, multiplier, drift3 = sp.profile(x, y, z, cells[1].astype(np.int32))
        q = (q_factor * density) * multiplier
        drift = [drift3[axis] for axis in range(3)]
    else:
        q = q_factor * (sp.rho / (4 * math.pi))
    vel = [(drift[axis] + sp.vth[axis] * normals[axis]).astype(velocity_dtype) for axis in range(3)]
    if sp.center:
        if first != 0 or count != total:
            raise ValueError("velocity centring needs the whole species")
        vel = center_velocities(vel, drift, np.broadcast_to(q, (count,)), velocity_dtype)
    key = grid.encode(cells[0], cells[1], cells[2])
    out.update(rx=fr[0], ry=fr[1], rz=fr[2], u=vel[0], v=vel[1], w=vel[2],
               q=np.broadcast_to(np.asarray(q, dtype=np.float64), (count,)).copy(),
               cell=key.astype(np.int32), id=n.astype(np.uint64))
    return out


def center_velocities(vel, drift, q, velocity_dtype):
    """TPIC's velocity centring (initialization/particles/particle_centering_device.hpp:36-100):
    the loaded drift is removed (stored in the velocity type), the
    charge-weighted mean of what remains is subtracted and the drift put back
    (each stored velocity formed in double and narrowed once)."""
    rest = [(vel[a].astype(np.float64) - 0.0 + -1.0 * drift[a]).astype(velocity_dtype) for a in range(3)]
    qsum = float(np.sum(q))
    mean = [float(np.sum(q * rest[a].astype(np.float64))) / qsum if qsum != 0.0 else 0.0 for a in range(3)]
    return [((rest[a].astype(np.float64) - mean[a]) + 1.0 * drift[a]).astype(velocity_dtype) for a in range(3)]


@dataclass
class FieldInit:
    """Initial fields: uniform E and B, or full node (E) and cell (B) arrays
    in the layouts of include/tpicb200.h, halos included (e_node: 3 x
    (nx+3)(ny+3)(nz+3), b_cell: 3 x (nx+2)(ny+2)(nz+2), component-major)."""
    e0: tuple = (0.0, 0.0, 0.0)
    b0: tuple = (0.0, 0.0, 0.0)
    e_node: object = None
    b_cell: object = None


@dataclass
class Case:
    """A periodic ECSIM run: grid, species, time integration and fields."""
    grid: GridSpec
    species: list
    dt: float
    theta: float = 0.5
    c: float = 1.0
    gmres_tol: float = 1e-8
    ncycles: int = 1
    fields: FieldInit = field(default_factory=FieldInit)
    seed: int = 0
    deck: object = None   # the tpicb200_deck it came from (tpic_b200.deck), if any
    # Energy-conserving smoothing (passes, Face7 centre weight, operator 0
    # Face7 / 1 Binomial27); off with 0 passes.
    smoothing: tuple = (0, 1.0, 0)
