"""A slab-distributed ECSIM cycle on the host: the oracle's per-stage
operators on each rank's slab grid, composed with the partition and the
exchanges of tpic_b200.slab (fold, halos, dot sums, migration). Test
infrastructure: it checks the decomposition logic against the single-rank
oracle cycle (test_slab_gloo.py).

Each rank holds the library's node and cell layouts of its slab (nz cells
along z). The oracle's stage functions fill ghosts periodically on the grid
they are given; on a slab that is right along x and y and wrong along z, so
every such call is followed by the z halo exchange. The mover runs on the
global grid (its periodic wrap of the cell index is the global one) with the
slab's fields placed at their global planes; the records it moves out of the
slab then migrate.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

import oracle as O
from tpic_b200.plasma import GridSpec
from tpic_b200.slab import SlabExchange, gmres

ATTRS = ("rx", "ry", "rz", "u", "v", "w", "q", "cell", "id")


def _og(g):
    return O.OGrid(g.nx, g.ny, g.nz, g.lx / g.nx, g.ly / g.ny, g.lz / g.nz)


def fold_xy(f: np.ndarray, nx: int, ny: int) -> None:
    """Shared-node sums along x and y of a node field (..., NY, NX) with
    one-node halos, then the x and y ghosts (periodic in-plane)."""
    f[..., :, 1] += f[..., :, nx + 1]
    f[..., :, nx + 1] = f[..., :, 1]
    f[..., 1, :] += f[..., ny + 1, :]
    f[..., ny + 1, :] = f[..., 1, :]
    ghosts_xy(f, nx, ny)


def ghosts_xy(f: np.ndarray, nx: int, ny: int) -> None:
    f[..., :, 0] = f[..., :, nx]
    f[..., :, nx + 2] = f[..., :, 2]
    f[..., 0, :] = f[..., ny, :]
    f[..., ny + 2, :] = f[..., 2, :]


class SlabCycle:
    def __init__(self, grid, species, dt, theta, c, tol, e_node, b_cell, exchange: SlabExchange, precision=0,
                 restart=30, max_iterations=100):
        self.lib = O.load()
        self.x = exchange
        p = exchange.plan
        self.plan = p
        self.grid = grid
        self.local = GridSpec(grid.nx, grid.ny, p.nz, grid.lx, grid.ly, grid.lz * p.nz / grid.nz)
        self.og, self.og_global = _og(self.local), _og(grid)
        self.dt, self.theta, self.c, self.tol = dt, theta, c, tol
        self.restart, self.max_iterations = restart, max_iterations
        self.precision = precision
        self.fdt = np.float64 if precision == 0 else np.float32
        nx, ny, nz = grid.nx, grid.ny, p.nz
        self.NX, self.NY, self.NZ = nx + 3, ny + 3, nz + 3
        self.CX, self.CY, self.CZ = nx + 2, ny + 2, nz + 2
        self.ex, self.ey = nx + 4, ny + 4
        self.key_shift = self.ex * self.ey * p.z0
        # Local fields: global planes z0 - 1 .. z0 + nz + 1 (periodic).
        gE = np.asarray(e_node, dtype=np.float64).reshape(3, grid.nz + 3, self.NY, self.NX)
        gB = np.asarray(b_cell, dtype=np.float64).reshape(3, grid.nz + 2, self.CY, self.CX)
        node_planes = [(p.z0 + k) % grid.nz + 1 for k in range(-1, nz + 2)]
        cell_planes = [(p.z0 + k) % grid.nz + 1 for k in range(-1, nz + 1)]
        self.e = np.ascontiguousarray(gE[:, node_planes]).astype(self.fdt).astype(np.float64)
        self.b = np.ascontiguousarray(gB[:, cell_planes]).astype(self.fdt).astype(np.float64)
        self.bnode = np.zeros_like(self.e)
        self.j = np.zeros_like(self.e)
        self.m = np.zeros((self.NZ, self.NY, self.NX, 126))
        self.theta_field = np.zeros_like(self.e)
        self.species = []
        for qom, d in species:
            kg = d["cell"].astype(np.int64) // (self.ex * self.ey) - 2
            keep = p.owns_cell(kg)
            loc = {k: np.ascontiguousarray(v[keep]) for k, v in d.items() if not k.startswith("_")}
            loc["cell"] = (loc["cell"].astype(np.int64) - self.key_shift).astype(np.int32)
            self.species.append((qom, loc))
        self.iterations = []

    # -- exchanges on numpy arrays (torch views share the memory) -----------
    def node_halo(self, f):
        self.x.node_halo(torch.from_numpy(f))

    def cell_halo(self, f):
        self.x.cell_halo(torch.from_numpy(f))

    def node_ghosts(self, f):
        """Periodic x/y ghosts and the z halo of a 3-component node field."""
        self.lib.oracle_node_ghosts(C.byref(self.og), O.ptr(f))
        self.node_halo(f)

    def _ptrs(self, d):
        return [O.ptr(d[k]) for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell")]

    # -- stages ------------------------------------------------------------
    def sort(self):
        nbins = self.lib.oracle_bin_count(C.byref(self.og))
        for qom, d in self.species:
            n = len(d["cell"])
            perm = np.empty(max(n, 1), dtype=np.uint32)
            counts = np.empty(nbins, dtype=np.uint32)
            offsets = np.empty(nbins + 1, dtype=np.uint32)
            assert self.lib.oracle_sort(C.byref(self.og), O.ptr(d["cell"]), n, O.ptr(perm), O.ptr(counts),
                                        O.ptr(offsets)) == 0
            for k in list(d):
                d[k] = np.ascontiguousarray(d[k][perm[:n]])

    def deposit(self, bnode):
        self.j[:] = 0
        self.m[:] = 0
        bn = np.ascontiguousarray(bnode.astype(self.fdt))
        for qom, d in self.species:
            bad = self.lib.oracle_deposit(self.precision, C.byref(self.og), qom, self.dt, self.c, *self._ptrs(d),
                                          len(d["cell"]), O.ptr(bn), O.ptr(self.j), O.ptr(self.m))
            assert bad == 0
        nx, ny = self.grid.nx, self.grid.ny
        fold_xy(self.j, nx, ny)
        mt = np.moveaxis(self.m, 3, 0)  # (126, NZ, NY, NX) view
        fold_xy(mt, nx, ny)
        self.x.fold_nodes(torch.from_numpy(self.j))
        self.x.fold_nodes(torch.from_numpy(self.m).permute(3, 0, 1, 2))
        self.j = self.j.astype(self.fdt).astype(np.float64)
        self.m = self.m.astype(self.fdt).astype(np.float64)

    def prepare(self):
        self.lib.oracle_cell_ghosts(C.byref(self.og), O.ptr(self.b))
        self.cell_halo(self.b)
        self.bnode = self.cell_to_node(self.b)
        self.sort()
        self.deposit(self.bnode)

    def cell_to_node(self, cellf):
        out = np.zeros_like(self.e)
        self.lib.oracle_cell_to_node(C.byref(self.og), O.ptr(cellf), O.ptr(out))
        self.node_halo(out)
        return out.astype(self.fdt).astype(np.float64)

    # Solver vectors: the owned node planes' interior rows, components outer.
    def pack(self, f):
        rows = self.plan.owned_node_planes
        nx, ny = self.grid.nx, self.grid.ny
        return torch.from_numpy(np.ascontiguousarray(f[:, 1:rows + 1, 1:ny + 2, 1:nx + 2]).reshape(-1))

    def unpack(self, vec, f):
        rows = self.plan.owned_node_planes
        nx, ny = self.grid.nx, self.grid.ny
        f[:, 1:rows + 1, 1:ny + 2, 1:nx + 2] = vec.numpy().reshape(3, rows, ny + 1, nx + 1)
        ghosts_xy(f, nx, ny)
        self.node_halo(f)

    def solve(self):
        g = self.local
        dx, dy, dz = g.lx / g.nx, g.ly / g.ny, g.lz / g.nz
        delta = self.c * self.theta * self.dt
        kfac = 4 * math.pi * (self.theta * self.dt)
        curl_node = np.zeros_like(self.e)
        self.lib.oracle_curl_c2n(C.byref(self.og), O.ptr(self.b), O.ptr(curl_node))
        rhs = (1.0 * self.e + delta * curl_node) + (-kfac) * self.j
        inp = np.zeros_like(self.e)
        curl_cell = np.zeros_like(self.b)
        mimage = np.zeros_like(self.e)
        d2 = delta * delta

        def apply(v, out):
            self.unpack(v, inp)
            self.lib.oracle_curl_n2c(C.byref(self.og), O.ptr(inp), O.ptr(curl_cell))
            self.cell_halo(curl_cell)
            self.lib.oracle_curl_c2n(C.byref(self.og), O.ptr(curl_cell), O.ptr(curl_node))
            self.lib.oracle_mass_apply(0, C.byref(self.og), O.ptr(self.m), O.ptr(inp), O.ptr(mimage))
            image = (1.0 * inp + d2 * curl_node) + kfac * mimage
            out.copy_(self.pack(image))

        def dot(u, v):
            return self.x.allreduce_sum(torch.dot(u, v).reshape(1))[0]

        x = self.pack(self.e).clone()
        res = gmres(apply, self.pack(rhs).clone(), x, dot, self.restart, self.max_iterations, self.tol)
        assert res.converged
        self.iterations.append(res.iterations)
        self.theta_field = np.zeros_like(self.e)
        self.unpack(x, self.theta_field)
        return res

    def move(self):
        """The mover on the global grid (global keys), then the migration."""
        p = self.plan
        gz = self.grid.nz + 3
        theta_g = np.zeros((3, gz, self.NY, self.NX))
        bnode_g = np.zeros((3, gz, self.NY, self.NX))
        planes = slice(p.z0 + 1, p.z0 + p.nz + 2)  # global node planes z0 .. z0 + nz
        theta_g[:, planes] = self.theta_field[:, 1:p.nz + 2]
        bnode_g[:, planes] = self.bnode[:, 1:p.nz + 2]
        bn = np.ascontiguousarray(bnode_g.astype(self.fdt))
        moved = []
        for qom, d in self.species:
            d["cell"] = (d["cell"].astype(np.int64) + self.key_shift).astype(np.int32)
            bad = self.lib.oracle_mover(self.precision, C.byref(self.og_global), qom, self.dt, self.c,
                                        *self._ptrs(d), len(d["cell"]), O.ptr(theta_g), O.ptr(bn))
            assert bad == 0
            kg = torch.from_numpy(d["cell"].astype(np.int64) // (self.ex * self.ey) - 2)
            # Record ids travel as int64 bytes.
            out = self.x.migrate({k: torch.from_numpy(d[k].view(np.int64) if k == "id" else d[k]) for k in ATTRS},
                                 kg)
            loc = {k: np.ascontiguousarray(out[k].numpy()) for k in ATTRS}
            loc["id"] = loc["id"].view(np.uint64)
            loc["cell"] = (loc["cell"].astype(np.int64) - self.key_shift).astype(np.int32)
            moved.append((qom, loc))
        self.species = moved

    def advance(self):
        bnext = np.zeros_like(self.b)
        bnode_next = np.zeros_like(self.bnode)
        self.lib.oracle_field_advance(C.byref(self.og), self.dt, self.theta, self.c, O.ptr(self.e), O.ptr(self.b),
                                      O.ptr(self.theta_field), O.ptr(bnext), O.ptr(bnode_next))
        self.node_halo(self.e)
        self.e = self.e.astype(self.fdt).astype(np.float64)
        self.cell_halo(bnext)
        self.bnext = bnext.astype(self.fdt).astype(np.float64)
        self.bnode_next = self.cell_to_node(self.bnext)

    def energy(self):
        out = np.zeros(2)
        self.lib.oracle_field_energy(C.byref(self.og), O.ptr(self.e), O.ptr(self.b), O.ptr(out))
        res = [out[0], out[1]]
        for qom, d in self.species:
            s = np.zeros(5)
            self.lib.oracle_species_scalars(self.precision, qom, O.ptr(d["u"]), O.ptr(d["v"]), O.ptr(d["w"]),
                                            O.ptr(d["q"]), len(d["q"]), O.ptr(s))
            res.extend(s)
        return self.x.allreduce_sum(torch.tensor(res, dtype=torch.float64)).numpy()

    def cycle(self):
        self.solve()
        self.move()
        self.advance()
        self.sort()
        self.deposit(self.bnode_next)
        self.b, self.bnode = self.bnext, self.bnode_next
        return self.energy()
