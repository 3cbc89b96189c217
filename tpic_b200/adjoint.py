"""Reverse-mode gradients of an ECSIM run through the library's adjoint C ABI.

The forward run keeps a checkpoint (the state at a cycle's start: sorted
records with ids, E and B) every `every` cycles in device memory. The
backward run carries the gradient of an objective of the final fields back
segment by segment: the segment's cycles are recomputed from its checkpoint
with tpicb200_cycle_forward, which saves one tape per cycle, and
tpicb200_cycle_backward then walks the tapes in reverse. Device memory is
therefore (ncycles / every) checkpoints plus `every` tapes, instead of one
tape per cycle.

The gradient comes back with respect to the state the run started from:
E at the unique nodes, B at the cells, and per species the positions,
velocities and charges of every record, indexed by record id (the load
index). Parameter gradients contract it with the derivative of that
starting state with respect to a parameter (a tangent): the helpers below
give the tangents of the two-stream deck's beam drift and density-seed
amplitude and of a species' thermal anisotropy.

TPIC has no adjoint: this is built on the library's own forward cycle.
PyTorch only owns the device buffers and the stream.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib


def _ptr(t) -> int:
    return t.data_ptr() if t is not None else 0


class TapeBuffers:
    """Device buffers of one tape entry (tpicb200_tape) for a Simulation."""

    def __init__(self, sim):
        dev, st = sim.device, sim.state
        nodes, cells, bins = sim.layout.node_count, sim.layout.cell_count, sim.layout.bin_count
        self.struct = _lib.Tape()
        self.struct.ns = st.ns
        self.species = []
        self.bins = []
        for s in range(st.ns):
            n = st.slot[s][st.current[s]].count
            t = {k: torch.empty(max(n, 1), dtype=dt, device=dev) for k, dt in
                 (("rx", torch.float64), ("ry", torch.float64), ("rz", torch.float64), ("u", sim.vdt),
                  ("v", sim.vdt), ("w", sim.vdt), ("q", torch.float64), ("cell", torch.int32),
                  ("id", torch.int64))}
            self.species.append(t)
            p = self.struct.species[s]
            for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell", "id"):
                setattr(p, k, t[k].data_ptr())
            p.count = n
            cnt = torch.empty(bins, dtype=torch.int32, device=dev)
            off = torch.empty(bins + 1, dtype=torch.int32, device=dev)
            self.bins.append((cnt, off))
            self.struct.counts[s] = cnt.data_ptr()
            self.struct.offsets[s] = off.data_ptr()
            self.struct.qom[s] = st.qom[s]
        self.e = torch.empty(3 * nodes, dtype=sim.fdt, device=dev)
        self.b_cell = torch.empty(3 * cells, dtype=sim.fdt, device=dev)
        self.e_theta = torch.empty(3 * nodes, dtype=torch.float64, device=dev)
        self.struct.e, self.struct.b_cell, self.struct.e_theta = _ptr(self.e), _ptr(self.b_cell), _ptr(self.e_theta)
        self.struct.mass_kind = st.mass_kind

    def nbytes(self) -> int:
        tensors = [t for d in self.species for t in d.values()] + [t for b in self.bins for t in b]
        tensors += [self.e, self.b_cell, self.e_theta]
        return sum(t.numel() * t.element_size() for t in tensors)


class AdjointBuffers:
    """Gradients (tpicb200_adjoint) of a Simulation's state, with the backward's scratch."""

    def __init__(self, sim):
        dev, st = sim.device, sim.state
        nodes, cells = sim.layout.node_count, sim.layout.cell_count
        f64 = torch.float64
        self.e_bar = torch.zeros(3 * nodes, dtype=f64, device=dev)
        self.b_bar = torch.zeros(3 * cells, dtype=f64, device=dev)
        self.x_bar, self.v_bar, self.q_bar, self.count = [], [], [], []
        self.struct = _lib.Adjoint()
        self.struct.ns = st.ns
        for s in range(st.ns):
            n = st.slot[s][st.current[s]].count
            self.count.append(n)
            self.x_bar.append(torch.zeros(3 * max(n, 1), dtype=f64, device=dev))
            self.v_bar.append(torch.zeros(3 * max(n, 1), dtype=f64, device=dev))
            self.q_bar.append(torch.zeros(max(n, 1), dtype=f64, device=dev))
            self.struct.x_bar[s] = self.x_bar[s].data_ptr()
            self.struct.v_bar[s] = self.v_bar[s].data_ptr()
            self.struct.q_bar[s] = self.q_bar[s].data_ptr()
            self.struct.count[s] = n
        self.e_theta_bar = torch.zeros(3 * nodes, dtype=f64, device=dev)
        self.lam = torch.zeros(3 * nodes, dtype=f64, device=dev)
        self.b_node_bar = torch.zeros(3 * nodes, dtype=f64, device=dev)
        self.b_node = torch.zeros(3 * nodes, dtype=sim.fdt, device=dev)
        self.j = torch.zeros(3 * nodes, dtype=sim.fdt, device=dev)
        self.mass = torch.zeros(sim.layout.mass_count, dtype=sim.fdt, device=dev)
        a = self.struct
        a.e_bar, a.b_bar = _ptr(self.e_bar), _ptr(self.b_bar)
        a.e_theta_bar, a.lambda_, a.b_node_bar = _ptr(self.e_theta_bar), _ptr(self.lam), _ptr(self.b_node_bar)
        a.b_node, a.j, a.mass = _ptr(self.b_node), _ptr(self.j), _ptr(self.mass)

    def species_gradients(self, s: int) -> dict:
        """x (3, n), v (3, n) and q (n) of species s, indexed by record id (host numpy)."""
        n = self.count[s]
        return {"x": self.x_bar[s][:3 * n].view(3, n).cpu().numpy(),
                "v": self.v_bar[s][:3 * n].view(3, n).cpu().numpy(),
                "q": self.q_bar[s][:n].cpu().numpy()}


@dataclass
class Tangent:
    """The derivative of a run's starting state with respect to one
    parameter: E (node field, consistent) and B (cell field) tangents, and per
    species {"x": (3, n), "v": (3, n), "q": (n,)} arrays indexed by record id
    (any may be absent)."""
    e: np.ndarray | None = None
    b: np.ndarray | None = None
    species: dict = field(default_factory=dict)


@dataclass
class BackwardStats:
    forward_s: float = 0.0
    recompute_s: float = 0.0
    backward_s: float = 0.0
    adjoint_iterations: list = field(default_factory=list)
    checkpoints: int = 0
    tapes: int = 0
    device_bytes: int = 0


class AdjointRun:
    """A Simulation run forward with checkpoints every `every` cycles, then
    the adjoint of an energy objective carried back to the run's start."""

    def __init__(self, sim, every: int = 20):
        if every < 1:
            raise ValueError("checkpoint interval must be positive")
        for s in range(sim.state.ns):
            if "id" not in sim.slots[s][0]:
                raise ValueError("the adjoint needs record ids: Simulation(..., keep_ids=True)")
        self.sim = sim
        self.every = every
        self.checkpoints: list[TapeBuffers] = []
        self.ncycles = 0
        self.reports = []
        self.stats = BackwardStats()

    def _stream(self):
        return C.c_void_p(self.sim.stream.cuda_stream)

    def _cycle_forward(self, tape: TapeBuffers, report=None):
        sim = self.sim
        _lib.check(sim.lib.tpicb200_cycle_forward(sim.ctx, C.byref(sim.state), C.byref(tape.struct),
                                                  C.byref(report) if report is not None else None, self._stream()))

    def forward(self, ncycles: int):
        """ncycles cycles from the simulation's current (prepared) state; the
        state at every `every`-th cycle start is kept as a checkpoint."""
        sim = self.sim
        if not sim.prepared:
            sim.prepare()
        t0 = time.perf_counter()
        for n in range(ncycles):
            if n % self.every == 0:
                tape = TapeBuffers(sim)
                self.checkpoints.append(tape)
                report = _lib.CycleReport()
                self._cycle_forward(tape, report)
                self.reports.append(report.total_energy)
            else:
                self.reports.append(sim.run(1)[0].total_energy)
        torch.cuda.synchronize()
        self.stats.forward_s = time.perf_counter() - t0
        self.ncycles = ncycles
        self.stats.checkpoints = len(self.checkpoints)
        return self.reports

    def restore(self, tape: TapeBuffers) -> None:
        """The simulation's state from a checkpoint, with the startup redone
        (B at the nodes, the sort, the deposition)."""
        sim, st = self.sim, self.sim.state
        sim.materialize()
        for s in range(st.ns):
            live = sim.slots[s][st.current[s]]
            for k, t in tape.species[s].items():
                live[k].copy_(t)
            st.ranked[s] = 0
        sim.field("e").copy_(tape.e)
        sim.field("b_cell").copy_(tape.b_cell)
        _lib.check(sim.lib.tpicb200_prepare(sim.ctx, C.byref(st), self._stream()))

    def backward(self, we: float = 1.0, wb: float = 1.0) -> AdjointBuffers:
        """Gradient of we * W_E + wb * W_B of the final fields with respect to
        the run's starting state."""
        sim, st = self.sim, self.sim.state
        lib = sim.lib
        adj = AdjointBuffers(sim)
        _lib.check(lib.tpicb200_adjoint_energy(sim.ctx, st.e, st.b_cell, we, wb, C.byref(adj.struct),
                                               self._stream()))
        pool = [TapeBuffers(sim) for _ in range(min(self.every, self.ncycles) - 1)]
        self.stats.tapes = len(pool) + len(self.checkpoints)
        self.stats.device_bytes = sum(t.nbytes() for t in pool + self.checkpoints)
        result = _lib.GmresResult()
        for seg in reversed(range(len(self.checkpoints))):
            start = seg * self.every
            stop = min(start + self.every, self.ncycles)
            t0 = time.perf_counter()
            self.restore(self.checkpoints[seg])
            tapes = [self.checkpoints[seg]] + pool[:stop - start - 1]
            for tape in tapes:
                self._cycle_forward(tape)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            for tape in reversed(tapes):
                _lib.check(lib.tpicb200_cycle_backward(sim.ctx, C.byref(tape.struct), C.byref(adj.struct),
                                                       C.byref(result), self._stream()))
                self.stats.adjoint_iterations.append(result.iterations)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            self.stats.recompute_s += t1 - t0
            self.stats.backward_s += t2 - t1
        # The state the gradient refers to: the run's start (checkpoint 0).
        self.start = self.checkpoints[0]
        return adj


def unique_nodes(sim, field: torch.Tensor) -> torch.Tensor:
    g = sim.case.grid
    f = field.view(3, g.nz + 3, g.ny + 3, g.nx + 3)
    return f[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]


def unique_cells(sim, field: torch.Tensor) -> torch.Tensor:
    g = sim.case.grid
    f = field.view(3, g.nz + 2, g.ny + 2, g.nx + 2)
    return f[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]


def contract(sim, adj: AdjointBuffers, tangent: Tangent) -> float:
    """<gradient, tangent> over the starting state."""
    total = 0.0
    if tangent.e is not None:
        e = torch.as_tensor(np.asarray(tangent.e, dtype=np.float64), device=sim.device)
        total += float((unique_nodes(sim, adj.e_bar) * unique_nodes(sim, e)).sum())
    if tangent.b is not None:
        b = torch.as_tensor(np.asarray(tangent.b, dtype=np.float64), device=sim.device)
        total += float((unique_cells(sim, adj.b_bar) * unique_cells(sim, b)).sum())
    for s, parts in tangent.species.items():
        n = adj.count[s]
        grads = {"x": adj.x_bar[s][:3 * n].view(3, n), "v": adj.v_bar[s][:3 * n].view(3, n), "q": adj.q_bar[s][:n]}
        for k, t in parts.items():
            tt = torch.as_tensor(np.asarray(t, dtype=np.float64), device=sim.device)
            total += float((grads[k] * tt).sum())
    return total


def start_records(run: AdjointRun, s: int) -> dict:
    """Species s of the run's starting state, ordered by record id (host numpy)."""
    t = run.start.species[s]
    n = run.start.struct.species[s].count
    ids = t["id"][:n].cpu().numpy().astype(np.int64)
    order = np.argsort(ids)
    return {k: v[:n].cpu().numpy()[order] for k, v in t.items()}


def record_positions(sim, rec: dict) -> tuple:
    """Physical positions (x, y, z) of records from their keys and fractions."""
    g = sim.case.grid
    key = rec["cell"].astype(np.int64)
    ex, ey = g.nx + 4, g.ny + 4
    i, j, k = key % ex - 2, (key // ex) % ey - 2, key // (ex * ey) - 2
    dx, dy, dz = g.spacing
    return (i + rec["rx"]) * dx, (j + rec["ry"]) * dy, (k + rec["rz"]) * dz


def two_stream_tangents(run: AdjointRun, deck) -> dict:
    """Tangents of the two-stream deck's parameters: `drift` (u0 of the first
    electron beam, the second beam at -u0) and `amplitude` (the density seed
    a: electron charges times 1 + a cos(k x + phase) and E_x = -(n_e a / k)
    sin(k x + phase), both linear in a; the cases are restated in
    tpicb200_case_profile / tpicb200_case_fields)."""
    sim = run.sim
    a = deck.two_stream_amplitude
    k = 2 * math.pi * deck.two_stream_mode_x / deck.grid.lx
    phase = deck.two_stream_phase
    drift = Tangent()
    amplitude = Tangent()
    beams = [s for s in range(deck.ns) if deck.species[s].qom < 0]
    for s in beams:
        n = run.start.struct.species[s].count
        v = np.zeros((3, n))
        v[0] = 1.0 if deck.species[s].drift[0] > 0 else -1.0
        drift.species[s] = {"v": v}
        rec = start_records(run, s)
        x, _, _ = record_positions(sim, rec)
        c = np.cos(k * x + phase)
        amplitude.species[s] = {"q": rec["q"] * c / (1.0 + a * c)}
    if a == 0.0:
        raise ValueError("the amplitude tangent needs a nonzero seed amplitude")
    amplitude.e = run.start.e.double().cpu().numpy() / a
    return {"drift": drift, "amplitude": amplitude}


def anisotropy_tangent(run: AdjointRun, species: int, parallel_axis: int, ratio: float) -> Tangent:
    """Tangent of the species' T_perp/T_par at fixed parallel temperature: the
    perpendicular thermal speed is vth_par sqrt(ratio), so each perpendicular
    velocity (less its drift, zero here) scales as sqrt(ratio); velocity
    centring, linear in the thermal part, keeps that."""
    rec = start_records(run, species)
    v = np.zeros((3, len(rec["q"])))
    for axis, key in enumerate(("u", "v", "w")):
        if axis != parallel_axis:
            v[axis] = rec[key].astype(np.float64) / (2.0 * ratio)
    return Tangent(species={species: {"v": v}})
