"""Numpy helpers for the field and particle layouts of include/tpicb200.h."""
from __future__ import annotations

import numpy as np


def node_shape(g):
    return (g.nz + 3, g.ny + 3, g.nx + 3)


def cell_shape(g):
    return (g.nz + 2, g.ny + 2, g.nx + 2)


def periodic_node_field(g, unique: np.ndarray) -> np.ndarray:
    """unique: (3, nz, ny, nx) -> flat 3*(nx+3)(ny+3)(nz+3) node field whose
    duplicate endpoint nodes and ghosts repeat the periodic unique values."""
    k = (np.arange(-1, g.nz + 2) % g.nz)[:, None, None]
    j = (np.arange(-1, g.ny + 2) % g.ny)[None, :, None]
    i = (np.arange(-1, g.nx + 2) % g.nx)[None, None, :]
    return np.concatenate([unique[c][k, j, i].ravel() for c in range(3)])


def periodic_cell_field(g, unique: np.ndarray) -> np.ndarray:
    k = (np.arange(-1, g.nz + 1) % g.nz)[:, None, None]
    j = (np.arange(-1, g.ny + 1) % g.ny)[None, :, None]
    i = (np.arange(-1, g.nx + 1) % g.nx)[None, None, :]
    return np.concatenate([unique[c][k, j, i].ravel() for c in range(3)])


def interior_nodes(g, field: np.ndarray, components: int = 3) -> np.ndarray:
    """(components, nz+1, ny+1, nx+1) view of the interior nodes 0..n."""
    f = field.reshape(components, g.nz + 3, g.ny + 3, g.nx + 3)
    return f[:, 1:g.nz + 2, 1:g.ny + 2, 1:g.nx + 2]


def unique_nodes(g, field: np.ndarray, components: int = 3) -> np.ndarray:
    f = field.reshape(components, g.nz + 3, g.ny + 3, g.nx + 3)
    return f[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]


def interior_records(g, mass: np.ndarray) -> np.ndarray:
    """(nz+1, ny+1, nx+1, 126) records of the interior nodes 0..n."""
    m = mass.reshape(g.nz + 3, g.ny + 3, g.nx + 3, 126)
    return m[1:g.nz + 2, 1:g.ny + 2, 1:g.nx + 2]


def smooth_random_unique(g, rng, amplitude=1.0, components=3, modes=3):
    """A smooth periodic random vector field on the unique nodes/cells."""
    z, y, x = np.meshgrid(np.arange(g.nz) / g.nz, np.arange(g.ny) / g.ny, np.arange(g.nx) / g.nx, indexing="ij")
    out = np.zeros((components, g.nz, g.ny, g.nx))
    for c in range(components):
        for _ in range(modes):
            kx, ky, kz = rng.integers(0, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi)
            out[c] += amplitude * rng.uniform(0.5, 1.0) * np.cos(2 * np.pi * (kx * x + ky * y + kz * z) + ph)
    return out


def bits(a: np.ndarray) -> np.ndarray:
    """Integer view for bitwise comparison of floating-point arrays."""
    a = np.ascontiguousarray(a)
    return a.view(np.int64 if a.dtype.itemsize == 8 else np.int32)
