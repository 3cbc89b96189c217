"""ctypes front end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA path. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it; the product
(tpic_b200/) never imports it.

`OracleCycle` runs TPIC's one-rank cycle on the host in the layouts of
include/tpicb200.h: solve, move (old B), advance, stable sort, deposit
(next B), fold, commit (include/tpic/simulation/driver/pipeline.hpp:437-540).
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liboracle.so"
REF_LIBRARY = HERE / "_ref" / "libtpicref.so"

_lib = None
_ref = None

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class OGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class OGmres(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual", C.c_double),
                ("residual", C.c_double), ("rhs_norm", C.c_double), ("relative_residual", C.c_double)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            build()
        lib = C.CDLL(str(LIBRARY))
        vp = C.c_void_p
        lib.oracle_mover.restype = C.c_long
        lib.oracle_mover.argtypes = [C.c_int, C.POINTER(OGrid), C.c_double, C.c_double, C.c_double,
                                     vp, vp, vp, vp, vp, vp, vp, vp, C.c_long, vp, vp]
        lib.oracle_sort.restype = C.c_long
        lib.oracle_sort.argtypes = [C.POINTER(OGrid), vp, C.c_long, vp, vp, vp]
        lib.oracle_deposit.restype = C.c_long
        lib.oracle_deposit.argtypes = [C.c_int, C.POINTER(OGrid), C.c_double, C.c_double, C.c_double,
                                       vp, vp, vp, vp, vp, vp, vp, vp, C.c_long, vp, vp, vp]
        lib.oracle_fold.argtypes = [C.POINTER(OGrid), vp, vp]
        lib.oracle_mass_apply.argtypes = [C.c_int, C.POINTER(OGrid), vp, vp, vp]
        for name in ("oracle_curl_n2c", "oracle_curl_c2n", "oracle_cell_to_node"):
            getattr(lib, name).argtypes = [C.POINTER(OGrid), vp, vp]
        lib.oracle_node_ghosts.argtypes = [C.POINTER(OGrid), vp]
        lib.oracle_cell_ghosts.argtypes = [C.POINTER(OGrid), vp]
        lib.oracle_field_solve.restype = C.c_int
        lib.oracle_field_solve.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, C.c_double, vp, vp, vp, vp,
                                           vp, C.c_int, C.c_int, C.c_double, C.POINTER(OGmres)]
        lib.oracle_field_solve_smoothed.restype = C.c_int
        lib.oracle_field_solve_smoothed.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, C.c_double, vp, vp,
                                                    vp, vp, vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double,
                                                    C.c_int, C.POINTER(OGmres)]
        lib.oracle_smooth.argtypes = [C.POINTER(OGrid), C.c_int, C.c_double, C.c_int, vp, vp]
        lib.oracle_smooth_node.restype = C.c_double
        lib.oracle_smooth_node.argtypes = [C.POINTER(OGrid), C.c_int, C.c_double, vp, C.c_int, C.c_int, C.c_int]
        lib.oracle_field_advance.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, C.c_double, vp, vp, vp,
                                             vp, vp]
        lib.oracle_field_energy.argtypes = [C.POINTER(OGrid), vp, vp, vp]
        lib.oracle_species_scalars.argtypes = [C.c_int, C.c_double, vp, vp, vp, vp, C.c_long, vp]
        lib.oracle_stencil_offset.argtypes = [C.c_int, vp]
        lib.oracle_pair_stencil.restype = C.c_int
        lib.oracle_pair_stencil.argtypes = [C.c_int, C.c_int]
        lib.oracle_cic_weights_f64.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        lib.oracle_cic_weights_f32.argtypes = [C.c_float, C.c_float, C.c_float, vp]
        lib.oracle_response_f64.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, vp]
        lib.oracle_response_f32.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, vp]
        lib.oracle_adjoint_advance.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, C.c_double, vp, vp, vp, vp,
                                               vp]
        lib.oracle_adjoint_mover_scatter.restype = C.c_long
        lib.oracle_adjoint_mover_scatter.argtypes = [C.c_int, C.POINTER(OGrid), C.c_double, C.c_double, C.c_double,
                                                     vp, vp, vp, vp, vp, vp, vp, vp, C.c_long, C.c_long, vp, vp, vp,
                                                     vp, vp]
        lib.oracle_adjoint_particles.restype = C.c_long
        lib.oracle_adjoint_particles.argtypes = [C.c_int, C.POINTER(OGrid), C.c_double, C.c_double, C.c_double,
                                                 C.c_double, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_long, C.c_long,
                                                 vp, vp, vp, vp, vp, vp, vp]
        lib.oracle_adjoint_solve.restype = C.c_int
        lib.oracle_adjoint_solve.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, C.c_double, vp, vp, vp,
                                             C.c_int, C.c_int, C.c_double, C.POINTER(OGmres)]
        lib.oracle_adjoint_fields.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, C.c_double, vp, vp, vp, vp]
        lib.oracle_energy_gradient.argtypes = [C.POINTER(OGrid), C.c_double, C.c_double, vp, vp, vp, vp]
        for name in ("oracle_node_count", "oracle_cell_count", "oracle_bin_count"):
            getattr(lib, name).restype = C.c_long
            getattr(lib, name).argtypes = [C.POINTER(OGrid)]
        _lib = lib
    return _lib


def load_reference():
    """The reference's own header numerics compiled by oracle/Makefile, or None."""
    global _ref
    if _ref is None and REF_LIBRARY.exists():
        lib = C.CDLL(str(REF_LIBRARY))
        vp = C.c_void_p
        lib.ref_cic_weights_f64.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        lib.ref_cic_weights_f32.argtypes = [C.c_float, C.c_float, C.c_float, vp]
        lib.ref_response_f64.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, vp]
        lib.ref_response_f32.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, vp]
        if hasattr(lib, "ref_smooth_node"):
            lib.ref_smooth_node.restype = C.c_double
            lib.ref_smooth_node.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, C.c_int, C.c_int]
        lib.ref_pair_stencil.restype = C.c_int
        lib.ref_pair_stencil.argtypes = [C.c_int, C.c_int]
        lib.ref_stencil_offset.argtypes = [C.c_int, vp]
        lib.ref_encode_key.restype = C.c_int
        lib.ref_encode_key.argtypes = [C.c_int] * 6
        lib.ref_decode_key.argtypes = [C.c_int] * 4 + [vp]
        for name in ("ref_curl_n2c", "ref_curl_c2n"):
            getattr(lib, name).argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_double, C.c_double, C.c_double,
                                           C.c_int, C.c_int, C.c_int, vp]
        lib.ref_cell_to_node.restype = C.c_double
        lib.ref_cell_to_node.argtypes = [C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int]
        lib.ref_mass_apply_node.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, C.c_double, C.c_int, C.c_int,
                                            C.c_int, vp]
        _ref = lib
    return _ref


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class OracleCycle:
    """The ECSIM cycle on the host (FP64 fields and moments; the mover in the
    storage/compute types of the selected precision, bit-identical to the GPU
    mover)."""

    def __init__(self, grid, species, dt, theta=0.5, c=1.0, gmres_tol=1e-8, precision=0,
                 restart=30, max_iterations=100, e0=(0.0, 0.0, 0.0), b0=(0.0, 0.0, 0.0), e_node=None,
                 b_cell=None, smoothing=(0, 1.0, 0)):
        self.lib = load()
        self.og = OGrid(grid.nx, grid.ny, grid.nz, grid.lx / grid.nx, grid.ly / grid.ny, grid.lz / grid.nz)
        self.grid = grid
        self.dt, self.theta, self.c, self.tol = dt, theta, c, gmres_tol
        self.restart, self.max_iterations = restart, max_iterations
        # Energy-conserving smoothing (passes, Face7 centre weight, operator
        # 0 Face7 / 1 Binomial27); on when passes > 0 and the weight < 1.
        self.smoothing = tuple(smoothing) if smoothing[0] > 0 and smoothing[1] < 1 else (0, 1.0, 0)
        self.precision = precision
        self.vdt = np.float64 if precision == 0 else np.float32
        self.fdt = np.float64 if precision == 0 else np.float32
        og = C.byref(self.og)
        self.nodes = self.lib.oracle_node_count(og)
        self.cells = self.lib.oracle_cell_count(og)
        self.nbins = self.lib.oracle_bin_count(og)
        n, cl = self.nodes, self.cells
        self.e = np.zeros(3 * n)
        self.b = np.zeros(3 * cl)
        for k in range(3):
            self.e[k * n:(k + 1) * n] = e0[k]
            self.b[k * cl:(k + 1) * cl] = b0[k]
        # Sampled initial fields (node and cell layouts, halos included).
        if e_node is not None:
            self.e[:] = np.asarray(e_node, dtype=np.float64).reshape(-1)
        if b_cell is not None:
            self.b[:] = np.asarray(b_cell, dtype=np.float64).reshape(-1)
        # Fields are stored in the precision's storage type between stages.
        self.e = self.e.astype(self.fdt).astype(np.float64)
        self.b = self.b.astype(self.fdt).astype(np.float64)
        self.bnode = np.zeros(3 * n)
        self.j = np.zeros(3 * n)
        self.m = np.zeros(126 * n)
        self.theta_field = np.zeros(3 * n)
        self.species = species  # list of (qom, dict of arrays)
        self.gmres = []

    def _ptrs(self, d):
        return [ptr(d[k]) for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell")]

    def sort(self):
        for qom, d in self.species:
            n = len(d["cell"])
            perm = np.empty(n, dtype=np.uint32)
            counts = np.empty(self.nbins, dtype=np.uint32)
            offsets = np.empty(self.nbins + 1, dtype=np.uint32)
            status = self.lib.oracle_sort(C.byref(self.og), ptr(d["cell"]), n, ptr(perm), ptr(counts),
                                          ptr(offsets))
            if status != 0:
                raise ValueError("out-of-range cell key")
            for k in [k for k in d if not k.startswith("_")]:
                d[k] = np.ascontiguousarray(d[k][perm])
            d["_counts"], d["_offsets"] = counts, offsets

    def deposit(self, bnode):
        self.j[:] = 0
        self.m[:] = 0
        bn = bnode.astype(self.fdt)
        for qom, d in self.species:
            bad = self.lib.oracle_deposit(self.precision, C.byref(self.og), qom, self.dt, self.c, *self._ptrs(d),
                                          len(d["cell"]), ptr(bn), ptr(self.j), ptr(self.m))
            if bad:
                raise ValueError(f"{bad} invalid records in deposition")
        self.lib.oracle_fold(C.byref(self.og), ptr(self.j), ptr(self.m))
        # Moments are stored in the precision's storage type.
        self.j = self.j.astype(self.fdt).astype(np.float64)
        self.m = self.m.astype(self.fdt).astype(np.float64)

    def prepare(self):
        self.lib.oracle_cell_ghosts(C.byref(self.og), ptr(self.b))
        self.lib.oracle_cell_to_node(C.byref(self.og), ptr(self.b), ptr(self.bnode))
        self.bnode = self.bnode.astype(self.fdt).astype(np.float64)
        self.sort()
        self.deposit(self.bnode)

    def solve(self):
        res = OGmres()
        niter, alpha, op = self.smoothing
        status = self.lib.oracle_field_solve_smoothed(C.byref(self.og), self.dt, self.theta, self.c, ptr(self.e),
                                                      ptr(self.b), ptr(self.j), ptr(self.m), ptr(self.theta_field),
                                                      self.restart, self.max_iterations, self.tol, niter, alpha, op,
                                                      C.byref(res))
        self.gmres.append(res)
        if status != 0:
            raise RuntimeError("oracle GMRES did not converge")
        return res

    def particle_field(self):
        """The field the movers gather: E_theta, or S^n(E_theta) when smoothing."""
        niter, alpha, op = self.smoothing
        if niter == 0:
            return self.theta_field
        out = np.zeros_like(self.theta_field)
        self.lib.oracle_smooth(C.byref(self.og), niter, alpha, op, ptr(self.theta_field), ptr(out))
        return out

    def move(self):
        bn = self.bnode.astype(self.fdt)
        field = self.particle_field()
        for qom, d in self.species:
            bad = self.lib.oracle_mover(self.precision, C.byref(self.og), qom, self.dt, self.c, *self._ptrs(d),
                                        len(d["cell"]), ptr(field), ptr(bn))
            if bad:
                raise ValueError(f"{bad} invalid records in the mover")

    def advance(self):
        bnext = np.zeros_like(self.b)
        bnode_next = np.zeros_like(self.bnode)
        self.lib.oracle_field_advance(C.byref(self.og), self.dt, self.theta, self.c, ptr(self.e), ptr(self.b),
                                      ptr(self.theta_field), ptr(bnext), ptr(bnode_next))
        self.e = self.e.astype(self.fdt).astype(np.float64)
        self.bnext = bnext.astype(self.fdt).astype(np.float64)
        self.bnode_next = bnode_next.astype(self.fdt).astype(np.float64)

    def energy(self):
        out = np.zeros(2)
        self.lib.oracle_field_energy(C.byref(self.og), ptr(self.e), ptr(self.b), ptr(out))
        res = [out[0], out[1]]
        for qom, d in self.species:
            s = np.zeros(5)
            self.lib.oracle_species_scalars(self.precision, qom, ptr(d["u"]), ptr(d["v"]), ptr(d["w"]), ptr(d["q"]),
                                            len(d["q"]), ptr(s))
            res.extend(s)
        return np.array(res)

    def cycle(self):
        self.solve()
        self.move()
        self.advance()
        self.sort()
        self.deposit(self.bnode_next)
        self.b, self.bnode = self.bnext, self.bnode_next
        return self.energy()


class OracleAdjoint:
    """The discrete adjoint of OracleCycle's cycles in FP64 (test
    infrastructure: the checker of the library's adjoint kernels).

    `forward(n)` runs n cycles of `oc` (prepared, species carrying dense ids
    0..count-1) and keeps a tape entry per cycle: the sorted records, E and B
    at the cycle start and the cycle's E_theta. `backward(e_bar, b_bar)`
    carries the gradient of an objective of the final E and B back through
    the tape: per cycle the advance adjoint, the mover's E_theta scatter and
    fold, the solve with A^T, the per-record adjoint (mover, current, mass),
    the B scatter and fold, and the field adjoint. Particle adjoints are per
    species, indexed by id: x_bar [3][count] (per axis, in cells), v_bar
    [3][count], q_bar [count]."""

    def __init__(self, oc: OracleCycle, tol: float = 1e-13, max_iterations: int = 500):
        self.oc = oc
        self.lib = oc.lib
        self.tol = tol
        self.max_iterations = max_iterations
        self.tape = []
        self.solves = []

    def forward(self, ncycles: int):
        oc = self.oc
        for _ in range(ncycles):
            snap = {"e": oc.e.copy(), "b": oc.b.copy(),
                    "species": [(qom, {k: v.copy() for k, v in d.items()}) for qom, d in oc.species]}
            energies = oc.cycle()
            snap["theta"] = oc.theta_field.copy()
            self.tape.append(snap)
        return energies

    def energy_gradient(self, we: float = 1.0, wb: float = 1.0):
        oc = self.oc
        e_bar, b_bar = np.zeros(3 * oc.nodes), np.zeros(3 * oc.cells)
        self.lib.oracle_energy_gradient(C.byref(oc.og), we, wb, ptr(oc.e), ptr(oc.b), ptr(e_bar), ptr(b_bar))
        return e_bar, b_bar

    def _mass_and_bnode(self, snap):
        oc = self.oc
        og = C.byref(oc.og)
        b = snap["b"].copy()
        self.lib.oracle_cell_ghosts(og, ptr(b))
        bnode = np.zeros(3 * oc.nodes)
        self.lib.oracle_cell_to_node(og, ptr(b), ptr(bnode))
        bnode = bnode.astype(oc.fdt)
        m = np.zeros(126 * oc.nodes)
        for qom, d in snap["species"]:
            bad = self.lib.oracle_deposit(oc.precision, og, qom, oc.dt, oc.c, *[ptr(d[k]) for k in
                                          ("rx", "ry", "rz", "u", "v", "w", "q", "cell")], len(d["cell"]),
                                          ptr(bnode), None, ptr(m))
            if bad:
                raise ValueError(f"{bad} invalid records in the adjoint's deposition")
        self.lib.oracle_fold(og, None, ptr(m))
        return m.astype(oc.fdt).astype(np.float64), bnode

    def backward(self, e_bar, b_bar):
        oc = self.oc
        og = C.byref(oc.og)
        lib = self.lib
        counts = [len(d["cell"]) for _, d in oc.species]
        parts = [{"x": np.zeros(3 * n), "v": np.zeros(3 * n), "q": np.zeros(n)} for n in counts]
        e_bar, b_bar = e_bar.copy(), b_bar.copy()
        for snap in reversed(self.tape):
            m, bnode = self._mass_and_bnode(snap)
            theta = snap["theta"]
            e_theta_bar, e_new, b_new = np.zeros(3 * oc.nodes), np.zeros(3 * oc.nodes), np.zeros(3 * oc.cells)
            lib.oracle_adjoint_advance(og, oc.dt, oc.theta, oc.c, ptr(e_bar), ptr(b_bar), ptr(e_theta_bar),
                                       ptr(e_new), ptr(b_new))
            scatter = np.zeros(3 * oc.nodes)
            for (qom, d), pa, n in zip(snap["species"], parts, counts):
                bad = lib.oracle_adjoint_mover_scatter(oc.precision, og, qom, oc.dt, oc.c, *[ptr(d[k]) for k in
                                                       ("rx", "ry", "rz", "u", "v", "w", "cell", "id")], n, n,
                                                       ptr(pa["x"]), ptr(pa["v"]), ptr(theta), ptr(bnode),
                                                       ptr(scatter))
                if bad:
                    raise ValueError(f"{bad} invalid records in the mover adjoint")
            lib.oracle_fold(og, ptr(scatter), None)
            e_theta_bar += scatter
            lam = np.zeros(3 * oc.nodes)
            res = OGmres()
            status = lib.oracle_adjoint_solve(og, oc.dt, oc.theta, oc.c, ptr(m), ptr(e_theta_bar), ptr(lam),
                                              oc.restart, self.max_iterations, self.tol, C.byref(res))
            self.solves.append(res)
            if status != 0:
                raise RuntimeError("oracle adjoint GMRES did not converge")
            bscatter = np.zeros(3 * oc.nodes)
            for (qom, d), pa, n in zip(snap["species"], parts, counts):
                bad = lib.oracle_adjoint_particles(oc.precision, og, qom, oc.dt, oc.theta, oc.c,
                                                   *[ptr(d[k]) for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell",
                                                                         "id")], n, n, ptr(pa["x"]), ptr(pa["v"]),
                                                   ptr(pa["q"]), ptr(theta), ptr(bnode), ptr(lam), ptr(bscatter))
                if bad:
                    raise ValueError(f"{bad} invalid records in the particle adjoint")
            lib.oracle_fold(og, ptr(bscatter), None)
            lib.oracle_adjoint_fields(og, oc.dt, oc.theta, oc.c, ptr(lam), ptr(bscatter), ptr(e_new), ptr(b_new))
            e_bar, b_bar = e_new, b_new
        return e_bar, b_bar, parts


def total_energy(scalars: np.ndarray, ns: int) -> float:
    return float(scalars[0] + scalars[1] + sum(scalars[2 + 5 * s] for s in range(ns)))


def case_species_arrays(case, precision: int, generate) -> list:
    """(qom, arrays) per species in the storage types of `precision`."""
    vdt = np.float64 if precision == 0 else np.float32
    out = []
    for s, sp in enumerate(case.species):
        d = generate(case.grid, sp, s, seed=case.seed, velocity_dtype=vdt)
        d.pop("id", None)
        out.append((sp.qom, d))
    return out


__all__ = ["OracleCycle", "OracleAdjoint", "load", "load_reference", "build", "total_energy", "case_species_arrays", "OGrid", "ptr",
           "math"]


def output_moments(grid, d: dict, qom: float, precision: int = 0):
    """Output moments of one species at the nx*ny*nz unique nodes (FP64),
    restating deposit_output_moments_kernel
    (diagnostics/output_moment_deposition_device.hpp:30-107) with the
    shared-node sum of a periodic grid: per record the amounts q/V, q/V v and
    (q/V)(1/qom) v_i v_j times the CIC weights of its cell corners
    ((wx*wy)*wz, ecsim/particles/cic.hpp:24-36). Returns (4 pi rho, J[3],
    P[6] as xx, xy, xz, yy, yz, zz), each (components, nz, ny, nx)."""
    g = grid
    vol = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    ex, ey = g.nx + 4, g.ny + 4
    key = d["cell"].astype(np.int64)
    ci, cj, ck = key % ex - 2, (key // ex) % ey - 2, key // (ex * ey) - 2
    fx, fy, fz = (np.asarray(d[k], dtype=np.float64) for k in ("rx", "ry", "rz"))
    u, v, w = (np.asarray(d[k]).astype(np.float64) for k in ("u", "v", "w"))
    charge = np.asarray(d["q"], dtype=np.float64) * (1.0 / vol)
    mass = charge * (1.0 / qom)
    amounts = [charge * (4.0 * np.pi)] + [charge * u, charge * v, charge * w] + \
              [mass * u * u, mass * u * v, mass * u * w, mass * v * v, mass * v * w, mass * w * w]
    out = np.zeros((10, g.nz, g.ny, g.nx))
    cx, cy, cz = 1.0 - fx, 1.0 - fy, 1.0 - fz
    for a in range(8):
        wx = fx if a & 1 else cx
        wy = fy if a & 2 else cy
        wz = fz if a & 4 else cz
        wt = (wx * wy) * wz
        i = (ci + (a & 1)) % g.nx
        j = (cj + ((a >> 1) & 1)) % g.ny
        k = (ck + ((a >> 2) & 1)) % g.nz
        for c in range(10):
            np.add.at(out[c], (k, j, i), amounts[c] * wt)
    return out[0:1], out[1:4], out[4:10]


def _node_samples(grid, f: np.ndarray):
    """The eight corner samples of every cell from a halo-layout node field
    component (nz+3, ny+3, nx+3): base, x, y, z, xy, xz, yz, xyz
    (load_node_cell_samples, ecsim/fields/node_cell_curl.hpp:84-98)."""
    g = grid

    def at(a, b, d):
        return f[1 + d:1 + d + g.nz, 1 + b:1 + b + g.ny, 1 + a:1 + a + g.nx]
    return [at(0, 0, 0), at(1, 0, 0), at(0, 1, 0), at(0, 0, 1), at(1, 1, 0), at(1, 0, 1), at(0, 1, 1), at(1, 1, 1)]


def gauss_half_divergence(grid, e: np.ndarray) -> np.ndarray:
    """divC(E)/2 per cell in FP64 (nz, ny, nx), restating node_cell_divergence
    (ecsim/fields/node_cell_curl.hpp:129-141) with NodeCellSamples::derivative's
    edge differences in their order (:63-80) and the residual's 0.5 factor
    (diagnostics/gauss_residual_device.hpp:46-47). `e` is the node field in
    the library's halo layout, (3, nz+3, ny+3, nx+3) (float storage widened)."""
    g = grid
    e = np.asarray(e, dtype=np.float64).reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)
    inv = (1.0 / (g.lx / g.nx), 1.0 / (g.ly / g.ny), 1.0 / (g.lz / g.nz))
    q = _node_samples(g, e[0])
    dx = 0.25 * inv[0] * ((((q[1] - q[0]) + (q[5] - q[3])) + (q[4] - q[2])) + (q[7] - q[6]))
    q = _node_samples(g, e[1])
    dy = 0.25 * inv[1] * ((((q[2] - q[0]) + (q[6] - q[3])) + (q[4] - q[1])) + (q[7] - q[5]))
    q = _node_samples(g, e[2])
    dz = 0.25 * inv[2] * ((((q[3] - q[0]) + (q[5] - q[1])) + (q[6] - q[2])) + (q[7] - q[4]))
    return 0.5 * ((dx + dy) + dz)


def gauss_cell_charge(grid, species: list, smoothing=(0, 1.0, 0)) -> np.ndarray:
    """c per cell in FP64 (nz, ny, nx): 4 pi times the 8-node mean of the
    charge density rho = sum(q W)/V of every species' records (the rho of
    output_moments before its 4 pi), after `smoothing` = (passes, alpha,
    operator) passes of the oracle's smoothing (gauss_residual_device.hpp:82-99,
    the complete_charge steps of docs/developer/gauss_diagnostic.md)."""
    g = grid
    vol = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    ex, ey = g.nx + 4, g.ny + 4
    rho = np.zeros((g.nz, g.ny, g.nx))
    for d in species:
        key = d["cell"].astype(np.int64)
        ci, cj, ck = key % ex - 2, (key // ex) % ey - 2, key // (ex * ey) - 2
        fx, fy, fz = (np.asarray(d[k], dtype=np.float64) for k in ("rx", "ry", "rz"))
        charge = np.asarray(d["q"], dtype=np.float64) * (1.0 / vol)
        cx, cy, cz = 1.0 - fx, 1.0 - fy, 1.0 - fz
        for a in range(8):
            wt = ((fx if a & 1 else cx) * (fy if a & 2 else cy)) * (fz if a & 4 else cz)
            np.add.at(rho, ((ck + ((a >> 2) & 1)) % g.nz, (cj + ((a >> 1) & 1)) % g.ny, (ci + (a & 1)) % g.nx),
                      charge * wt)
    # The node field with its periodic ghosts and end nodes, component 0.
    k = (np.arange(g.nz + 3) - 1) % g.nz
    j = (np.arange(g.ny + 3) - 1) % g.ny
    i = (np.arange(g.nx + 3) - 1) % g.nx
    field = np.zeros((3, g.nz + 3, g.ny + 3, g.nx + 3))
    field[0] = rho[k][:, j][:, :, i]
    passes, alpha, op = smoothing
    if passes > 0:
        out = np.zeros_like(field)
        grid_struct = OGrid(g.nx, g.ny, g.nz, g.lx / g.nx, g.ly / g.ny, g.lz / g.nz)
        load().oracle_smooth(C.byref(grid_struct), int(passes), float(alpha), int(op), ptr(field), ptr(out))
        field = out
    q = _node_samples(g, field[0])
    return np.pi / 2 * (((((((q[0] + q[1]) + q[2]) + q[4]) + q[3]) + q[5]) + q[6]) + q[7])
