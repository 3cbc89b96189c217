"""Field and particle snapshots of a Simulation in TPIC's default (VTK) layout.

TPIC's output channels (docs/user/output.md): every `FieldOutputCycle` cycles
a field snapshot, one `<array>_tNNNNNN.vti` per array, and every
`ParticlesOutputCycle` cycles a particle snapshot, `particles_tNNNNNN.pvtp`
with its `.vtp` piece; both channels also write the final state. A snapshot
at cycle n holds the state before that cycle's solve (E and B at the nodes),
at time n*dt. `FieldOutputTag` and `MomentsOutputTag` select the arrays
(src/config/output selection rules restated in `select_arrays`): E, B and the
output moments rho = 4 pi sum(qW)/V, J = sum(qvW)/V and P_ij =
sum((q/qom) v_i v_j W)/V, per species (`<name>_<s>`) or summed (`<name>`).

The moments and the particles' output coordinates are computed by the
library (`tpicb200_output_moments`, `tpicb200_output_particles`); the files
are written by its host functions (`tpicb200_vtk_write_field`,
`tpicb200_vtk_write_particles`). Only the VTK engine is built: the ADIOS2 and
HDF5 engines of TPIC are optional there too and are refused here.
"""
from __future__ import annotations

import ctypes as C
import math
import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from . import _lib

MOMENTS = ("rho", "J", "PXX", "PXY", "PXZ", "PYY", "PYZ", "PZZ")
PRESSURE = MOMENTS[2:]
VTK_METHODS = ("vtk", "pvtk", "default", "")
OTHER_METHODS = ("adios2", "bp", "bp5", "hdf5", "h5")


def deck_keys(text: str) -> dict:
    """key -> value of a TPIC deck text (the last assignment of a key wins;
    `#` starts a comment)."""
    keys = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0]
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        keys[k.strip()] = v.strip()
    return keys


@dataclass
class OutputPlan:
    """The snapshot channels of a run (deck keys and their TPIC defaults)."""
    save_dir: Path
    field_cycle: int = 100
    particles_cycle: int = 0
    field_tag: str = ""
    moments_tag: str = ""
    field_method: str = ""
    particles_method: str = ""
    overwrite: bool = True
    gauss_cycle: int = 0
    written: list = field(default_factory=list)

    @classmethod
    def from_deck(cls, text: str, root: Path, **override) -> "OutputPlan":
        k = deck_keys(text)
        method = k.get("WriteMethod", "")
        plan = cls(save_dir=Path(root) / k.get("SaveDirName", "data"),
                   field_cycle=int(k.get("FieldOutputCycle", 100)),
                   particles_cycle=int(k.get("ParticlesOutputCycle", 0)),
                   field_tag=k.get("FieldOutputTag", ""), moments_tag=k.get("MomentsOutputTag", ""),
                   field_method=k.get("FieldWriteMethod", "") or method,
                   particles_method=k.get("ParticlesWriteMethod", "") or method,
                   gauss_cycle=int(k.get("DiagnosticGaussCycle", 0)))
        for name, value in override.items():
            if value is not None:
                setattr(plan, name, value)
        plan.check()
        return plan

    def check(self) -> None:
        for key, method, cadence in (("FieldWriteMethod", self.field_method, self.field_cycle),
                                     ("ParticlesWriteMethod", self.particles_method, self.particles_cycle)):
            if method in VTK_METHODS:
                continue
            if method in OTHER_METHODS:
                if cadence > 0:
                    raise ValueError(f"{key}={method}: only the VTK engine is built")
                continue
            raise ValueError(f"{key}: unknown write method {method!r}")

    def due(self, cycle: int, final: bool) -> tuple[bool, bool]:
        f = self.field_cycle > 0 and (final or cycle % self.field_cycle == 0)
        p = self.particles_cycle > 0 and (final or cycle % self.particles_cycle == 0)
        return f, p

    @property
    def output_gauss(self) -> bool:
        """The FieldOutputTag token Gauss, effective with a field channel."""
        return self.field_cycle > 0 and "Gauss" in _tokens(self.field_tag, "FieldOutputTag")

    def gauss_enabled(self) -> bool:
        return self.gauss_cycle > 0 or self.output_gauss

    def next_gauss_begin(self, cycle: int, last: int) -> int | None:
        """The first cycle after `cycle` at which a sample begins, if any."""
        for m in range(cycle + 1, last):
            if self.gauss_begins(m, last):
                return m
        return None

    def gauss_begins(self, cycle: int, last: int) -> bool:
        """A Gauss-law sample begins at cycle n < last when n is a multiple of
        DiagnosticGaussCycle, or, with the Gauss array selected, when n + 1 is
        a field snapshot cycle or the final state (PreparedOutput::
        should_sample_gauss, src/config/output.cpp)."""
        if cycle >= last:
            return False
        if self.gauss_cycle > 0 and cycle % self.gauss_cycle == 0:
            return True
        return self.output_gauss and ((cycle + 1) % self.field_cycle == 0 or cycle + 1 == last)


def _tokens(tag: str, key: str) -> list[str]:
    if tag == "":
        return []
    out = tag.split("+")
    for t in out:
        if t == "" or any(c.isspace() for c in t):
            raise ValueError(f"{key}: empty or spaced token in {tag!r}")
    return out


def select_arrays(field_tag: str, moments_tag: str, ns: int):
    """(field arrays, moment arrays): the field names ('E', 'B') and the moment
    arrays as (array name, quantity, species index or None for the total)."""
    ftok = _tokens(field_tag, "FieldOutputTag")
    mtok = _tokens(moments_tag, "MomentsOutputTag")
    if not ftok and not mtok:
        moments = [(q, q, None) for q in ("rho", "J")]
        moments += [(f"{q}_{s}", q, s) for q in ("rho", "J") for s in range(ns)]
        return ["E", "B"], moments
    fields = []
    for t in ftok:
        if t not in ("B", "E", "Gauss"):
            raise ValueError(f"FieldOutputTag: unknown token {t!r}")
        if t not in fields:
            fields.append(t)
    totals, indexed, bare = [], {}, []
    for t in mtok:
        m = re.fullmatch(r"(rho|J|PXX|PXY|PXZ|PYY|PYZ|PZZ)(_tot|\d+)?", t)
        if not m:
            raise ValueError(f"MomentsOutputTag: unknown token {t!r}")
        q, suffix = m.group(1), m.group(2)
        if suffix == "_tot":
            totals.append(q)
        elif suffix is None:
            bare.append(q)
        else:
            index = int(suffix)
            if index >= 2 ** 31:
                raise ValueError(f"MomentsOutputTag: index out of range in {t!r}")
            if index < ns:
                indexed.setdefault(q, []).append(index)
    moments = []
    for q in MOMENTS:
        if q in totals:
            moments.append((q, q, None))
        species = sorted(set(indexed.get(q, [])))
        if q in bare and not species:
            species = list(range(ns))
        moments += [(f"{q}_{s}", q, s) for s in species]
    return fields, moments


def precision_strings(sim) -> tuple[str, str]:
    """The precision profile name and roles written into every snapshot."""
    if sim.precision == _lib.PRECISION_DOUBLE:
        return "double/double", ("storage: position=float64 velocity=float64 weight=float64 E=float64 B=float64 "
                                 "J=float64 mass=float64 cell=int32 ID=uint64; compute: position=float64 "
                                 "velocity=float64 E=float64 B=float64 J=float64 mass=float64 "
                                 "solver-reduction=float64 reduction=float64 output-moment-accumulation=float64")
    return "mixed/mixed", ("storage: position=float64 velocity=float32 weight=float64 E=float32 B=float32 "
                           "J=float32 mass=float32 cell=int32 ID=uint64; compute: position=float64 "
                           "velocity=float32 E=float32 B=float32 J=float32 mass=float32 solver-reduction=float64 "
                           "reduction=float64 output-moment-accumulation=float64")


def _nodes(sim, name: str) -> np.ndarray:
    """A node field as the snapshot's (nz+1, ny+1, nx+1, 3) FP64 array."""
    g = sim.case.grid
    f = sim.field(name).double().view(3, g.nz + 3, g.ny + 3, g.nx + 3)
    return f[:, 1:g.nz + 2, 1:g.ny + 2, 1:g.nx + 2].permute(1, 2, 3, 0).contiguous().cpu().numpy()


def _wrap_unique(sim, u: torch.Tensor, components: int) -> np.ndarray:
    """Unique-node arrays (components, nz, ny, nx) onto the snapshot's node grid
    with the periodic end nodes: (nz+1, ny+1, nx+1, components)."""
    g = sim.case.grid
    u = u.view(components, g.nz, g.ny, g.nx)
    dev = u.device
    k = torch.arange(g.nz + 1, device=dev) % g.nz
    j = torch.arange(g.ny + 1, device=dev) % g.ny
    i = torch.arange(g.nx + 1, device=dev) % g.nx
    full = u[:, k][:, :, j][:, :, :, i]
    return full.permute(1, 2, 3, 0).contiguous().cpu().numpy()


def _grid(sim) -> _lib.Grid:
    g = sim.case.grid
    return _lib.Grid(g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)


def write_fields(sim, plan: OutputPlan, cycle: int, final: bool, gauss: "GaussSampler | None" = None) -> list[Path]:
    """The field snapshot of the simulation's current state at `cycle`; with
    the Gauss array selected, the residual of the sample that finished at
    `cycle` as cell data (absent when none did)."""
    lib = sim.lib
    g = sim.case.grid
    ns = len(sim.case.species)
    fields, moments = select_arrays(plan.field_tag, plan.moments_tag, ns)
    plan.save_dir.mkdir(parents=True, exist_ok=True)
    profile, roles = precision_strings(sim)
    time = cycle * sim.case.dt
    unique = g.nx * g.ny * g.nz
    stream = C.c_void_p(sim.stream.cuda_stream)
    written = []

    def put(name: str, values: np.ndarray, components: int) -> None:
        path = plan.save_dir / f"{name}_t{cycle:06d}.vti"
        values = np.ascontiguousarray(values, dtype=np.float64)
        _lib.check(lib.tpicb200_vtk_write_field(str(path).encode(), name.encode(), components, C.byref(_grid(sim)),
                                                values.ctypes.data, cycle, time, int(final), profile.encode(),
                                                roles.encode(), int(plan.overwrite)))
        written.append(path)

    sim.materialize()
    if "Gauss" in fields and gauss is not None and gauss.finished is not None and gauss.finished + 1 == cycle:
        path = plan.save_dir / f"Gauss_t{cycle:06d}.vti"
        values = np.ascontiguousarray(gauss.residual_cells(), dtype=np.float64)
        _lib.check(lib.tpicb200_vtk_write_cells(str(path).encode(), b"Gauss", C.byref(_grid(sim)), values.ctypes.data,
                                                cycle, time, int(final), profile.encode(), roles.encode(),
                                                int(plan.overwrite)))
        written.append(path)
    if "E" in fields:
        put("E", _nodes(sim, "e"), 3)
    if "B" in fields:
        put("B", _nodes(sim, "b_node"), 3)
    if moments:
        needed = {}
        for _, q, s in moments:
            kind = "P" if q in PRESSURE else q
            needed.setdefault(kind, set()).add(s)
        per = {}
        st = sim.state
        for kind, species in needed.items():
            comps = {"rho": 1, "J": 3, "P": 6}[kind]
            for s in range(ns):
                buf = torch.zeros(comps * unique, dtype=torch.float64, device=sim.device)
                part = st.slot[s][st.current[s]]
                args = [None, None, None]
                args[("rho", "J", "P").index(kind)] = buf.data_ptr()
                _lib.check(lib.tpicb200_output_moments(sim.ctx, sim.case.species[s].qom, C.byref(part), *args,
                                                       stream))
                per[(kind, s)] = buf
            per[(kind, None)] = sum(per[(kind, s)] for s in range(ns)) if ns else None
        sim.stream.synchronize()
        count = C.c_uint32(0)
        _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 0, stream))
        if count.value:
            raise ValueError("output moments: invalid records in the snapshot state")
        for name, q, s in moments:
            if q in PRESSURE:
                c = PRESSURE.index(q)
                comp = per[("P", s)].view(6, unique)[c]
                put(name, _wrap_unique(sim, comp.contiguous(), 1), 1)
            else:
                comps = 1 if q == "rho" else 3
                put(name, _wrap_unique(sim, per[(q, s)], comps), comps)
    plan.written += written
    return written


def write_particles(sim, plan: OutputPlan, cycle: int, final: bool) -> Path:
    """The particle snapshot of the simulation's current state at `cycle`
    (the simulation must keep record ids)."""
    lib = sim.lib
    ns = len(sim.case.species)
    plan.save_dir.mkdir(parents=True, exist_ok=True)
    profile, roles = precision_strings(sim)
    stream = C.c_void_p(sim.stream.cuda_stream)
    sim.materialize()
    st = sim.state
    keep, species = [], (_lib.VtkSpecies * max(ns, 1))()
    for s in range(ns):
        part = st.slot[s][st.current[s]]
        n = part.count
        if n and not part.id:
            raise ValueError("particle output needs record ids (Simulation(keep_ids=True))")
        pos = torch.empty(3 * max(n, 1), dtype=torch.float64, device=sim.device)
        vel = torch.empty_like(pos)
        chg = torch.empty(max(n, 1), dtype=torch.float64, device=sim.device)
        _lib.check(lib.tpicb200_output_particles(sim.ctx, C.byref(part), pos.data_ptr(), vel.data_ptr(),
                                                 chg.data_ptr(), stream))
        ids = sim.live(s)["id"] if n else torch.zeros(1, dtype=torch.int64, device=sim.device)
        host = [pos.cpu().numpy(), vel.cpu().numpy(), chg.cpu().numpy(),
                np.ascontiguousarray(ids.cpu().numpy()).view(np.uint64)]
        keep.append(host)
        species[s] = _lib.VtkSpecies(n, host[0].ctypes.data, host[1].ctypes.data, host[2].ctypes.data,
                                     host[3].ctypes.data, s)
    sim.stream.synchronize()
    count = C.c_uint32(0)
    _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 0, stream))
    if count.value:
        raise ValueError("particle output: invalid records in the snapshot state")
    _lib.check(lib.tpicb200_vtk_write_particles(str(plan.save_dir).encode(), cycle, cycle * sim.case.dt, int(final),
                                                profile.encode(), roles.encode(), ns, species,
                                                int(plan.overwrite)))
    path = plan.save_dir / f"particles_t{cycle:06d}.pvtp"
    plan.written.append(path)
    return path


GAUSS_HEADER = (
    "# TPIC Gauss-law residual v1\n"
    "# A sample begins at cycle n and finishes at n + 1: per cell r = (divC(E^n) + divC(E^{n+1}))/2 - c, where divC is\n"
    "# the solver's node-to-cell divergence and c = 4*pi times the eight-node mean of the charge density of the particles\n"
    "# at x^{n+1/2} (dual-volume scaled, zero on PEC wall nodes, smoothed like the solver's current). time = (n + 1/2)*dt.\n"
    "# Root mean squares over the global cells: residual_rms of r; drift_rms of r minus the first finished sample of the\n"
    "# run (a restart starts a new baseline); wall_residual_rms of r over the cells touching a physical wall (0 without\n"
    "# walls); charge_rms of c.\n"
    "cycle,time,residual_rms,drift_rms,wall_residual_rms,charge_rms\n")


def csv_number(value: float) -> str:
    """A double as TPIC's CSV rows print it: general format, 17 significant
    digits (io::detail::CsvBuffer::append, src/io/diagnostics_writer.cpp:31-34)."""
    return format(value, ".17g")


@dataclass
class GaussSample:
    cycle: int             # the begin cycle n
    time: float            # (n + 1/2) dt
    rms: tuple             # residual, drift, wall, charge

    def row(self) -> str:
        return ",".join([str(self.cycle), csv_number(self.time)] + [csv_number(v) for v in self.rms])


class GaussSampler:
    """The Gauss-law residual samples of a Simulation
    (diagnostics/gauss_residual_device.hpp, docs/developer/gauss_diagnostic.md):
    begin(n) at state n stores divC(E^n)/2 - c per cell, finish() at state
    n + 1 adds divC(E^{n+1})/2 and returns the sample's root mean squares;
    `residual` holds r of the last finished sample. The cell buffers are FP64
    device tensors of the nx*ny*nz cells; the kernels are the library's
    (tpicb200_gauss_field, tpicb200_gauss_charge)."""

    def __init__(self, sim):
        g = sim.case.grid
        self.sim = sim
        self.cells = g.nx * g.ny * g.nz
        mk = lambda: torch.zeros(self.cells, dtype=torch.float64, device=sim.device)
        self.stash, self.first, self.residual = mk(), mk(), mk()
        self.sums = torch.zeros(4, dtype=torch.float64, device=sim.device)
        self.begun = None        # the begin cycle of the open sample
        self.first_set = False
        self.finished = None     # the begin cycle of the last finished sample

    def _species(self):
        sim = self.sim
        st = sim.state
        ns = st.ns
        sim.materialize()
        return ns, (_lib.Particles * max(ns, 1))(*[st.slot[s][st.current[s]] for s in range(ns)])

    def step(self, cycle: int, begin: bool) -> GaussSample | None:
        """At state `cycle`: finish the open sample (begun at cycle - 1), then
        begin a new one when `begin`; returns the finished sample, if any."""
        sim = self.sim
        lib = sim.lib
        stream = C.c_void_p(sim.stream.cuda_stream)
        finish = self.begun is not None
        if finish and self.begun != cycle - 1:
            raise RuntimeError("a Gauss sample finishes at the cycle after its begin")
        if not finish and not begin:
            return None
        e = sim.state.e
        _lib.check(lib.tpicb200_gauss_field(sim.ctx, e, self.stash.data_ptr(), self.first.data_ptr(),
                                            self.residual.data_ptr(), int(begin), int(finish),
                                            int(finish and not self.first_set), self.sums.data_ptr(), stream))
        sample = None
        if finish:
            sim.stream.synchronize()
            s = self.sums.cpu().numpy()
            rms = (math.sqrt(s[0] / self.cells), math.sqrt(s[1] / self.cells), 0.0)
            # The charge sum was taken at the begin.
            rms = rms + (math.sqrt(self.charge_sum / self.cells),)
            if not all(math.isfinite(v) for v in rms):
                raise ValueError("Gauss residual: nonfinite sample")
            sample = GaussSample(self.begun, (self.begun + 0.5) * sim.case.dt, rms)
            self.first_set = True
            self.finished = self.begun
            self.begun = None
        if begin:
            ns, species = self._species()
            _lib.check(lib.tpicb200_gauss_charge(sim.ctx, ns, species, self.stash.data_ptr(), self.sums.data_ptr(),
                                                 stream))
            sim.stream.synchronize()
            count = C.c_uint32(0)
            _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 0, stream))
            if count.value:
                raise ValueError("Gauss residual: invalid records in the sampled state")
            self.charge_sum = float(self.sums[3].item())
            self.begun = cycle
        return sample

    def residual_cells(self) -> np.ndarray:
        """r of the last finished sample as a host array of the nx*ny*nz cells."""
        return self.residual.cpu().numpy()


class GaussWriter:
    """gauss.csv under SaveDirName (io::GaussWriter, src/io/diagnostics_writer.cpp:215-232):
    the precision header, the column definitions and one row per finished sample;
    a restart keeps the rows below its cycle and adds a restart line."""

    def __init__(self, path: Path, profile: str, roles: str, restart_cycle: int | None = None):
        self.path = Path(path)
        self.path.parent.mkdir(parents=True, exist_ok=True)
        head = f"# precision_profile = {profile}\n# precision_roles = {roles}\n" + GAUSS_HEADER
        if restart_cycle is None or not self.path.exists():
            self.path.write_text(head if restart_cycle is None else
                                 head + f"# restart at cycle {restart_cycle}: precision_profile = {profile}, "
                                        f"precision_roles = {roles}\n")
            return
        kept = []
        for line in self.path.read_text().splitlines():
            if line and line[0].isdigit() and int(line.split(",")[0]) >= restart_cycle:
                continue
            kept.append(line)
        kept.append(f"# restart at cycle {restart_cycle}: precision_profile = {profile}, precision_roles = {roles}")
        self.path.write_text("\n".join(kept) + "\n")

    def write(self, sample: GaussSample) -> None:
        with open(self.path, "a") as f:
            f.write(sample.row() + "\n")
