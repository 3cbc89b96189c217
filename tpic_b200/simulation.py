"""Host driver of the ECSIM cycle over the C ABI (include/tpicb200.h).

Mirrors TPIC's run path for the one-rank device case: a prepared case
(grid, species, time integration, fields) becomes a context, persistent
device owners and a `tpicb200_state`; `prepare()` performs the startup
(B nodes from cells, first sort, bootstrap deposition,
docs/developer/architecture.md:161-171) and `run(n)` the cycles
(solve, move, advance, sort, deposit, commit; Pipeline::run_cycles,
include/tpic/simulation/driver/pipeline.hpp:437-540).

PyTorch is used only to own device memory and the stream; every stage runs
in the sm_100a library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .deck import deck_of
from .plasma import Case, generate_species


@dataclass
class Report:
    gmres_iterations: int
    gmres_relative_residual: float
    field_energy: tuple
    kinetic: tuple
    total_energy: float
    stage_ms: tuple
    gmres_host_waits: int = 0
    species_scalars: tuple = ()  # per species: kinetic energy, charge, momentum x, y, z


def _ptr(t) -> int:
    return t.data_ptr() if t is not None else 0


class Simulation:
    def __init__(self, case: Case, precision: str = "double", mass_kind: str = "scalar",
                 device: int = 0, gmres_restart: int = 30, gmres_max_iterations: int = 100,
                 keep_ids: bool = False, generate_on_device: bool = False, mass_layout: str = "stencil-major",
                 smoothing: tuple | None = None,
                 generate: bool = True):
        self.case = case
        self.lib = _lib.load()
        self.precision = _lib.PRECISIONS[precision]
        self.mass_kind = _lib.MASS_KINDS[mass_kind]
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.fdt = torch.float64 if self.precision == _lib.PRECISION_DOUBLE else torch.float32
        self.vdt = self.fdt
        g = case.grid
        counts = [g.cells * sp.ppc for sp in case.species]
        if len(counts) > _lib.MAX_SPECIES:
            raise ValueError("too many species")
        grid = _lib.Grid(g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)
        self.mass_layout = {"records": _lib.MASS_LAYOUT_RECORDS,
                            "stencil-major": _lib.MASS_LAYOUT_STENCIL_MAJOR,
                            "tiled": _lib.MASS_LAYOUT_TILED}[mass_layout]
        # Energy-conserving smoothing: (passes, Face7 centre weight, operator
        # 0 Face7 / 1 Binomial27); on when passes > 0 and the weight < 1.
        smoothing = tuple(case.smoothing if smoothing is None else smoothing)
        self.smoothing = smoothing
        opts = _lib.Options(case.dt, case.theta, case.c, case.gmres_tol, gmres_restart,
                            gmres_max_iterations, self.precision, max(counts), self.mass_layout,
                            int(smoothing[0]), float(smoothing[1]), int(smoothing[2]))
        handle = C.c_void_p()
        _lib.check(self.lib.tpicb200_create(C.byref(grid), C.byref(opts), C.byref(handle)))
        self.ctx = handle
        layout = _lib.Layout()
        _lib.check(self.lib.tpicb200_get_layout(self.ctx, C.byref(layout)))
        self.layout = layout
        nodes, cells, bins = layout.node_count, layout.cell_count, layout.bin_count
        dev = self.device
        self.e = torch.zeros(3 * nodes, dtype=self.fdt, device=dev)
        self.b_cell = torch.zeros(3 * cells, dtype=self.fdt, device=dev)
        self.b_cell_next = torch.zeros(3 * cells, dtype=self.fdt, device=dev)
        self.b_node = torch.zeros(3 * nodes, dtype=self.fdt, device=dev)
        self.b_node_next = torch.zeros(3 * nodes, dtype=self.fdt, device=dev)
        self.j = torch.zeros(3 * nodes, dtype=self.fdt, device=dev)
        self.mass = torch.zeros(layout.mass_count, dtype=self.fdt, device=dev)
        self.e_theta = torch.zeros(3 * nodes, dtype=torch.float64, device=dev)
        for k in range(3):
            self.e[k * nodes:(k + 1) * nodes] = case.fields.e0[k]
            self.b_cell[k * cells:(k + 1) * cells] = case.fields.b0[k]
        if case.fields.e_node is not None:
            self.e.copy_(torch.as_tensor(np.asarray(case.fields.e_node, dtype=np.float64).reshape(-1)))
        if case.fields.b_cell is not None:
            self.b_cell.copy_(torch.as_tensor(np.asarray(case.fields.b_cell, dtype=np.float64).reshape(-1)))
        self.stream = torch.cuda.current_stream(dev)
        self.slots = []
        self.bins = []
        self.ranks = []
        st = _lib.State()
        st.ns = len(case.species)
        for s, sp in enumerate(case.species):
            n = counts[s]
            slot = []
            for _ in range(2):
                slot.append({k: torch.empty(n, dtype=t, device=dev) for k, t in
                             (("rx", torch.float64), ("ry", torch.float64), ("rz", torch.float64),
                              ("u", self.vdt), ("v", self.vdt), ("w", self.vdt), ("q", torch.float64),
                              ("cell", torch.int32))})
                if keep_ids:
                    slot[-1]["id"] = torch.empty(n, dtype=torch.int64, device=dev)
            if not generate:
                pass  # the records come from a checkpoint (Simulation.restart)
            elif generate_on_device:
                self._load_on_device(deck_of(case), s, sp, slot[0], n)
            else:
                vdt_np = np.float64 if self.precision == _lib.PRECISION_DOUBLE else np.float32
                data = generate_species(g, sp, s, seed=case.seed, velocity_dtype=vdt_np)
                for k, t in slot[0].items():
                    src = data[k]
                    t.copy_(torch.from_numpy(src.view(np.int64) if k == "id" else src))
            self.slots.append(slot)
            cnt = torch.zeros(bins, dtype=torch.int32, device=dev)
            off = torch.zeros(bins + 1, dtype=torch.int32, device=dev)
            self.bins.append((cnt, off))
            # Rank buffer: the cycle keeps the species ranked (the live slot
            # plus its ranks is the sorted view; materialize() writes it out).
            rk = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
            self.ranks.append(rk)
            st.ranks[s] = rk.data_ptr()
            st.ranked[s] = 0
            st.qom[s] = sp.qom
            for k in range(2):
                st.slot[s][k] = self._particles(slot[k], n)
            st.current[s] = 0
            st.counts[s] = cnt.data_ptr()
            st.offsets[s] = off.data_ptr()
        st.e, st.b_cell, st.b_node = _ptr(self.e), _ptr(self.b_cell), _ptr(self.b_node)
        st.b_cell_next, st.b_node_next = _ptr(self.b_cell_next), _ptr(self.b_node_next)
        st.j, st.mass, st.e_theta = _ptr(self.j), _ptr(self.mass), _ptr(self.e_theta)
        st.mass_kind = self.mass_kind
        self.state = st
        self.reports: list[Report] = []
        self.prepared = False
        self.cycle = 0  # cycles completed (restored from a checkpoint by restart)

    def _load_on_device(self, deck, s: int, sp, slot: dict, n: int) -> None:
        """Species s loaded (and centred) by the library's device loader."""
        p = self._particles(slot, n)
        invalid = torch.zeros(1, dtype=torch.int32, device=self.device)
        stream = self._stream()
        _lib.check(self.lib.tpicb200_load_species(self.ctx, C.byref(deck), s, self.case.seed, 0, C.byref(p),
                                                  invalid.data_ptr(), stream))
        if sp.center:
            _lib.check(self.lib.tpicb200_center_velocities(self.ctx, C.byref(deck), s, C.byref(p),
                                                           invalid.data_ptr(), stream))
        if int(invalid.item()) != 0:
            raise _lib.TpicError(_lib.OVERFLOW, f"species {s}: nonfinite velocity or charge at loading")

    @staticmethod
    def _particles(slot: dict, n: int) -> _lib.Particles:
        p = _lib.Particles()
        for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell"):
            setattr(p, k, slot[k].data_ptr())
        p.id = slot["id"].data_ptr() if "id" in slot else 0
        p.count = n
        return p

    def _stream(self) -> C.c_void_p:
        return C.c_void_p(self.stream.cuda_stream)

    def materialize(self) -> None:
        """Writes the sorted records of every ranked species into its live slot."""
        _lib.check(self.lib.tpicb200_materialize(self.ctx, C.byref(self.state), self._stream()))

    def live(self, s: int) -> dict:
        """Live records of species s, sorted by cell (materialized first)."""
        self.materialize()
        return self.slots[s][self.state.current[s]]

    def prepare(self) -> None:
        _lib.check(self.lib.tpicb200_prepare(self.ctx, C.byref(self.state), self._stream()))
        self.prepared = True

    def run(self, ncycles: int) -> list[Report]:
        if not self.prepared:
            self.prepare()
        reports = (_lib.CycleReport * max(ncycles, 1))()
        _lib.check(self.lib.tpicb200_cycle(self.ctx, C.byref(self.state), ncycles, reports, self._stream()))
        self.cycle += ncycles
        out = []
        ns = self.state.ns
        for r in reports[:ncycles]:
            out.append(Report(r.gmres.iterations, r.gmres.relative_residual, tuple(r.field_energy),
                              tuple(r.species[s][0] for s in range(ns)), r.total_energy, tuple(r.stage_ms),
                              r.gmres.host_waits, tuple(tuple(r.species[s][:5]) for s in range(ns))))
        self.reports.extend(out)
        return out

    def checkpoint(self, directory) -> str:
        """Writes the checkpoint of the current cycle under `directory`
        (E, B and every record; older checkpoints there are removed) and
        returns the piece's path."""
        if not self.prepared:
            self.prepare()
        _lib.check(self.lib.tpicb200_checkpoint_write(self.ctx, C.byref(self.state), str(directory).encode(),
                                                      self.cycle, self._stream()))
        return find_checkpoint(directory)

    @classmethod
    def restart(cls, case: Case, directory, **kwargs) -> "Simulation":
        """The run continued from the newest complete checkpoint under
        `directory`: the case's grid, dt, c, species and storage precision
        must be the checkpoint's; E, B and the records come from it and
        everything else is rebuilt (tpicb200_prepare)."""
        path = find_checkpoint(directory)
        info = checkpoint_info(path)
        sim = cls(case, generate=False, **kwargs)
        for s in range(info.ns):
            if info.count[s] != sim.state.slot[s][0].count:
                raise ValueError(f"species {s}: the checkpoint holds {info.count[s]} records, the case "
                                 f"{sim.state.slot[s][0].count}")
        _lib.check(sim.lib.tpicb200_checkpoint_read(sim.ctx, C.byref(sim.state), path.encode(), C.byref(info),
                                                    sim._stream()))
        sim.cycle = info.cycle
        sim.prepare()
        return sim

    def energy(self) -> np.ndarray:
        ns = self.state.ns
        parts = (_lib.Particles * ns)(*[self.state.slot[s][self.state.current[s]] for s in range(ns)])
        qom = (C.c_double * ns)(*[self.case.species[s].qom for s in range(ns)])
        out = (C.c_double * (2 + 5 * ns))()
        b_cell = self.state.b_cell
        _lib.check(self.lib.tpicb200_energy(self.ctx, self.state.e, b_cell, parts, qom, ns, out, self._stream()))
        return np.array(out[:])

    def field(self, name: str) -> torch.Tensor:
        """Device tensor of a committed field (the pointer swap of the commit included)."""
        st = self.state
        ptrs = {"e": st.e, "b_cell": st.b_cell, "b_node": st.b_node, "j": st.j, "mass": st.mass,
                "e_theta": st.e_theta}
        target = ptrs[name]
        for t in (self.e, self.b_cell, self.b_cell_next, self.b_node, self.b_node_next, self.j, self.mass,
                  self.e_theta):
            if t.data_ptr() == target:
                return t
        raise KeyError(name)

    def close(self) -> None:
        if self.ctx:
            self.lib.tpicb200_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def find_checkpoint(directory) -> str:
    """The newest complete checkpoint piece under `directory`."""
    buf = C.create_string_buffer(4096)
    _lib.check(_lib.load().tpicb200_checkpoint_find(str(directory).encode(), buf, len(buf)))
    return buf.value.decode()


def checkpoint_info(path) -> _lib.CheckpointInfo:
    info = _lib.CheckpointInfo()
    _lib.check(_lib.load().tpicb200_checkpoint_info_read(str(path).encode(), C.byref(info)))
    return info
