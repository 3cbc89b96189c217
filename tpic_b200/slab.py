"""Slab decomposition of the periodic grid along z: the partition and the
exchange steps of a multi-rank ECSIM cycle, one process per GPU.

The hot path of this library runs one cycle per GPU on the whole grid; a
multi-rank run (TPIC's MPI/NCCL decomposition, ecsim/maxwell/maxwell_device.hpp,
communication/mass_halo/mass_halo_device.hpp:91-160,
communication/particles/particle_boundaries.hpp:112-160) splits the grid
into z-slabs and adds these exchanges to every cycle:

- the fold of the deposited moments (J and the 126 mass entries of a node):
  a rank's particles add into the node plane it shares with the rank above,
  which owns that plane and adds the contribution into its own sums;
- the node halos (E, the solver's trial vectors, E_theta, the mass records,
  the particle-facing B) and cell halos (B, the cell curl of each operator
  apply): one-plane ghosts from the neighbours, and the shared plane from
  the rank above;
- the sums of the GMRES dot products and of the energy diagnostics;
- the migration of the records that the mover took across a slab face
  (one slab per cycle at most, as TPIC's PARTICLE_MIGRATION_HOPS = 1).

Rank r owns the cells [z0, z0 + nz) of its slab and the node planes
z0 .. z0 + nz - 1; its arrays are the library's node and cell layouts of a
grid of nz cells along z (nz + 3 node planes: local plane k at index k + 1
for k = -1 .. nz + 1; nz + 2 cell planes), so local node plane nz is the
rank above's plane 0. The exchanges run over torch.distributed point-to-point
operations, with gloo on the host and NCCL between GPUs (device tensors over
NVLink, copied into this rank's buffers: no kernel reads a peer's memory).
With one rank the exchanges wrap onto the rank itself and reproduce the
periodic ghost fill and fold.

This module holds the partition and the exchanges; the tests compose them
with per-slab stage operators into a distributed cycle and compare it with
the single-rank cycle. The device path itself stays one GPU per process
(replicas) until the library's stages take slab grids.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


@dataclass(frozen=True)
class SlabPlan:
    """z-slab of one rank: cells [z0, z0 + nz) of a periodic grid of nz_global
    cells along z, with the neighbouring ranks below and above (periodic)."""
    nz_global: int
    world: int
    rank: int
    z0: int
    nz: int
    lower: int
    upper: int

    @classmethod
    def make(cls, nz_global: int, world: int, rank: int) -> "SlabPlan":
        if world < 1 or not 0 <= rank < world:
            raise ValueError("rank outside the world")
        base, extra = divmod(nz_global, world)
        if base < 1:
            raise ValueError(f"{nz_global} cell planes cannot give each of {world} ranks a slab")
        z0 = rank * base + min(rank, extra)
        nz = base + (1 if rank < extra else 0)
        return cls(nz_global, world, rank, z0, nz, (rank - 1) % world, (rank + 1) % world)

    def owns_cell(self, k_global):
        """Whether global cell plane k lies in this slab (numpy or torch arrays)."""
        return (k_global >= self.z0) & (k_global < self.z0 + self.nz)

    @property
    def owned_node_planes(self) -> int:
        """Node planes of this rank in the solver vector: its nz planes, and the
        last rank also the global plane nz (the duplicate of plane 0 that
        TPIC's interior-node vectors carry)."""
        return self.nz + (1 if self.rank == self.world - 1 else 0)


class SlabExchange:
    """The exchanges of one rank's slab. Node fields are tensors shaped
    (components, nz + 3, NY, NX), cell fields (components, nz + 2, CY, CX),
    with their x and y ghosts already filled (periodic in-plane); the
    exchanges fill the z ghosts and the shared plane."""

    def __init__(self, plan: SlabPlan, group=None):
        self.plan = plan
        self.group = group

    # -- point-to-point ----------------------------------------------------
    def _swap(self, down: torch.Tensor | None, up: torch.Tensor | None, from_upper_like, from_lower_like):
        """Sends `down` to the rank below and `up` to the rank above; returns
        what the rank above sent down and what the rank below sent up."""
        p = self.plan
        if p.world == 1:
            return (down.clone() if down is not None else None), (up.clone() if up is not None else None)
        def fresh(like):
            return None if like is None else torch.empty(like.shape, dtype=like.dtype, device=like.device)

        from_upper, from_lower = fresh(from_upper_like), fresh(from_lower_like)
        ops = []
        # Tags keep the two directions apart when the same rank is both
        # neighbours (two ranks); NCCL matches the operations in this order.
        if down is not None:
            ops.append(dist.P2POp(dist.isend, down.contiguous(), p.lower, self.group, tag=1))
        if up is not None:
            ops.append(dist.P2POp(dist.isend, up.contiguous(), p.upper, self.group, tag=2))
        if from_upper is not None:
            ops.append(dist.P2POp(dist.irecv, from_upper, p.upper, self.group, tag=1))
        if from_lower is not None:
            ops.append(dist.P2POp(dist.irecv, from_lower, p.lower, self.group, tag=2))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        return from_upper, from_lower

    # -- fields ------------------------------------------------------------
    def node_halo(self, f: torch.Tensor) -> None:
        """Local node planes -1 (the rank below's plane nz - 1), nz and nz + 1
        (the rank above's planes 0 and 1)."""
        nz = self.plan.nz
        down = f[:, 1:3]          # planes 0, 1: the rank below's planes nz, nz + 1
        up = f[:, nz:nz + 1]      # plane nz - 1: the rank above's plane -1
        from_upper, from_lower = self._swap(down, up, down, up)
        f[:, nz + 1:nz + 3] = from_upper
        f[:, 0:1] = from_lower

    def cell_halo(self, f: torch.Tensor) -> None:
        """Local cell planes -1 (the rank below's cell nz - 1) and nz (the rank
        above's cell 0)."""
        nz = self.plan.nz
        down = f[:, 1:2]
        up = f[:, nz:nz + 1]
        from_upper, from_lower = self._swap(down, up, down, up)
        f[:, nz + 1:nz + 2] = from_upper
        f[:, 0:1] = from_lower

    def fold_nodes(self, f: torch.Tensor) -> None:
        """Moments deposited into the shared plane nz belong to the rank above's
        plane 0: they are added there, then every rank's halo is refreshed."""
        nz = self.plan.nz
        up = f[:, nz + 1:nz + 2]
        _, from_lower = self._swap(None, up, None, up)
        f[:, 1:2] += from_lower
        self.node_halo(f)

    def allreduce_sum(self, t: torch.Tensor) -> torch.Tensor:
        if self.plan.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    # -- particles ---------------------------------------------------------
    def migrate(self, records: dict, k_global: torch.Tensor) -> dict:
        """Records whose (moved) global cell plane k_global lies outside this
        slab go to the neighbouring slab that holds it; the records of the
        neighbours that entered this slab are appended, in the order
        (kept, from below, from above). A record more than one slab away is an
        error (one hop per cycle). `records` maps names to 1-D tensors of one
        length; every tensor is sent as its bytes."""
        p = self.plan
        nzg = p.nz_global
        inside = p.owns_cell(k_global)
        if p.world == 1:
            if not bool(inside.all()):
                raise ValueError("a record left the single slab")
            return records
        below = (k_global == (p.z0 - 1) % nzg) & ~inside
        above = (k_global == (p.z0 + p.nz) % nzg) & ~inside
        if p.world == 2:
            # The other rank is both neighbours: one direction carries all.
            above = ~inside
            below = torch.zeros_like(inside)
        if not bool((inside | below | above).all()):
            raise ValueError("a record moved more than one slab in one cycle")
        names = sorted(records)

        def pack(mask):
            parts = [records[n][mask].contiguous().view(torch.uint8) for n in names]
            return torch.cat(parts) if parts else torch.empty(0, dtype=torch.uint8)

        sizes = {n: records[n].element_size() for n in names}
        per_record = sum(sizes.values())
        device = records[names[0]].device
        send_down, send_up = pack(below), pack(above)
        counts = torch.tensor([send_down.numel(), send_up.numel()], dtype=torch.int64, device=device)
        got_from_upper, got_from_lower = self._swap(counts[0:1], counts[1:2], counts[0:1], counts[1:2])
        n_upper, n_lower = int(got_from_upper.item()), int(got_from_lower.item())
        buf_upper = torch.empty(n_upper, dtype=torch.uint8, device=device)
        buf_lower = torch.empty(n_lower, dtype=torch.uint8, device=device)
        from_upper, from_lower = self._swap(send_down if send_down.numel() else None,
                                            send_up if send_up.numel() else None,
                                            buf_upper if n_upper else None, buf_lower if n_lower else None)

        def unpack(buf):
            if buf is None or buf.numel() == 0:
                return {n: records[n][:0] for n in names}
            count = buf.numel() // per_record
            out, offset = {}, 0
            for n in names:
                width = sizes[n] * count
                # A fresh copy starts the bytes at offset 0 (aligned for any type).
                out[n] = buf[offset:offset + width].clone().view(records[n].dtype)
                offset += width
            return out

        lower_in, upper_in = unpack(from_lower), unpack(from_upper)
        return {n: torch.cat([records[n][inside], lower_in[n], upper_in[n]]) for n in names}


@dataclass
class GmresResult:
    converged: bool = False
    iterations: int = 0
    initial_residual: float = 0.0
    residual: float = 0.0
    rhs_norm: float = 0.0
    relative_residual: float = 0.0


def gmres(apply, b: torch.Tensor, x: torch.Tensor, dot, restart: int = 30, max_iterations: int = 100,
          tol: float = 1e-8) -> GmresResult:
    """Restarted GMRES over a slab-distributed vector, the steps of
    Gmres::host_blocking_solve (ecsim/gmres/gmres_device.hpp:355-454, with the
    device tails of :52-98): classical Gram-Schmidt, Givens rotations on the
    least-squares right-hand side, back substitution, true-residual
    acceptance. `b` and `x` hold this rank's rows (FP64); `apply(v, out)`
    writes this rank's rows of A v (exchanging halos itself); `dot(u, v)`
    returns the sum over every rank's rows (one allreduce). x is updated in
    place."""
    n = b.numel()
    r = b - _applied(apply, x)
    res = GmresResult()
    res.residual = res.initial_residual = float(dot(r, r)) ** 0.5
    res.rhs_norm = float(dot(b, b)) ** 0.5
    scale = res.rhs_norm if res.rhs_norm != 0 else 1.0
    atol = scale * tol
    res.relative_residual = res.residual / scale
    res.converged = res.residual <= atol
    V = torch.zeros(restart + 1, n, dtype=torch.float64, device=b.device)
    while not res.converged and res.iterations < max_iterations:
        H = [[0.0] * (restart + 1) for _ in range(restart)]
        cs, sn, s = [0.0] * restart, [0.0] * restart, [0.0] * (restart + 1)
        y = [0.0] * restart
        rn2 = float(dot(r, r))
        V[0] = r * (1.0 / rn2 ** 0.5 if rn2 > 0 else 0.0)
        s[0] = rn2 ** 0.5
        columns = min(restart, max_iterations - res.iterations)
        completed, breakdown = 0, False
        for col in range(columns):
            w = _applied(apply, V[col])
            dots = [float(dot(V[jj], w)) for jj in range(col + 1)]
            for jj in range(col + 1):
                w = w - dots[jj] * V[jj]
            n2 = float(dot(w, w))
            h = H[col]
            h[:col + 1] = dots
            sub = n2 ** 0.5
            h[col + 1] = sub
            for row in range(col):
                up, lo = h[row], h[row + 1]
                h[row] = cs[row] * up + sn[row] * lo
                h[row + 1] = -sn[row] * up + cs[row] * lo
            diag = h[col]
            den = (diag * diag + sub * sub) ** 0.5
            cc = diag / den if den != 0 else 1.0
            ss = sub / den if den != 0 else 0.0
            cs[col], sn[col] = cc, ss
            h[col] = cc * diag + ss * sub
            h[col + 1] = 0.0
            up, lo = s[col], s[col + 1]
            s[col] = cc * up + ss * lo
            s[col + 1] = -ss * up + cc * lo
            estimate = abs(s[col + 1])
            V[col + 1] = w * (1.0 / n2 ** 0.5 if n2 > 0 else 0.0)
            completed = col + 1
            breakdown = sub == 0
            if estimate != estimate or estimate == float("inf"):
                raise FloatingPointError("GMRES estimate is not finite")
            if estimate <= atol or breakdown:
                break
        for row in range(completed - 1, -1, -1):
            acc = 0.0
            for col in range(row + 1, completed):
                acc += H[col][row] * y[col]
            d = H[row][row]
            y[row] = (s[row] - acc) / d if d != 0 else 0.0
        for col in range(completed):
            x += y[col] * V[col]
        res.iterations += completed
        r = b - _applied(apply, x)
        res.residual = float(dot(r, r)) ** 0.5
        res.relative_residual = res.residual / scale
        res.converged = res.residual <= atol
        if breakdown and not res.converged:
            break
    return res


def _applied(apply, v: torch.Tensor) -> torch.Tensor:
    out = torch.empty_like(v)
    apply(v, out)
    return out
