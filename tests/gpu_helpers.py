"""Thin test-side wrappers of the C ABI stage entry points over torch device
buffers (the tests call the library exactly as an external caller would)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from tpic_b200 import _lib

ATTRS = ("rx", "ry", "rz", "u", "v", "w", "q", "cell")


class StageContext:
    def __init__(self, grid, precision=0, dt=0.15, theta=0.5, c=1.0, tol=1e-8, max_particles=1 << 20,
                 restart=30, max_iterations=100, mass_layout=0, smoothing=(0, 1.0, 0)):
        self.lib = _lib.load()
        self.g = grid
        self.precision = precision
        self.fdt = torch.float64 if precision == 0 else torch.float32
        self.np_fdt = np.float64 if precision == 0 else np.float32
        opts = _lib.Options(dt, theta, c, tol, restart, max_iterations, precision, max_particles, mass_layout,
                            *smoothing)
        self.mass_layout = mass_layout
        gr = _lib.Grid(grid.nx, grid.ny, grid.nz, grid.lx, grid.ly, grid.lz)
        h = C.c_void_p()
        _lib.check(self.lib.tpicb200_create(C.byref(gr), C.byref(opts), C.byref(h)))
        self.ctx = h
        lay = _lib.Layout()
        _lib.check(self.lib.tpicb200_get_layout(self.ctx, C.byref(lay)))
        self.layout = lay
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        self.invalid = torch.zeros(1, dtype=torch.int32, device="cuda")

    def close(self):
        if self.ctx:
            self.lib.tpicb200_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- buffers -----------------------------------------------------------
    def upload_particles(self, arrays: dict):
        t = {}
        for k in ATTRS:
            a = np.ascontiguousarray(arrays[k])
            t[k] = torch.from_numpy(a).cuda()
        if "id" in arrays:
            t["id"] = torch.from_numpy(np.ascontiguousarray(arrays["id"]).view(np.int64)).cuda()
        return t

    def empty_particles(self, n: int, with_id=False):
        vdt = self.fdt
        t = {k: torch.empty(max(n, 1), dtype=d, device="cuda") for k, d in
             (("rx", torch.float64), ("ry", torch.float64), ("rz", torch.float64), ("u", vdt), ("v", vdt),
              ("w", vdt), ("q", torch.float64), ("cell", torch.int32))}
        if with_id:
            t["id"] = torch.empty(max(n, 1), dtype=torch.int64, device="cuda")
        return t

    @staticmethod
    def struct(t: dict, n: int) -> _lib.Particles:
        p = _lib.Particles()
        for k in ATTRS:
            setattr(p, k, t[k].data_ptr())
        p.id = t["id"].data_ptr() if "id" in t else 0
        p.count = n
        return p

    @staticmethod
    def download(t: dict, n: int) -> dict:
        out = {k: v[:n].cpu().numpy() for k, v in t.items()}
        if "id" in out:
            out["id"] = out["id"].view(np.uint64)
        return out

    def field(self, values: np.ndarray, dtype=None):
        return torch.from_numpy(np.ascontiguousarray(values.astype(dtype or self.np_fdt))).cuda()

    # -- stages --------------------------------------------------------------
    def invalid_count(self) -> int:
        torch.cuda.synchronize()
        return int(self.invalid.item())

    def mover(self, qom, parts: dict, n: int, etheta: torch.Tensor, bnode: torch.Tensor):
        p = self.struct(parts, n)
        _lib.check(self.lib.tpicb200_mover(self.ctx, qom, C.byref(p), etheta.data_ptr(), bnode.data_ptr(),
                                           self.invalid.data_ptr(), self.stream))

    def sort(self, src: dict, n: int, with_id=None):
        dst = self.empty_particles(n, ("id" in src) if with_id is None else with_id)
        counts = torch.zeros(self.layout.bin_count, dtype=torch.int32, device="cuda")
        offsets = torch.zeros(self.layout.bin_count + 1, dtype=torch.int32, device="cuda")
        pin, pout = self.struct(src, n), self.struct(dst, n)
        _lib.check(self.lib.tpicb200_sort(self.ctx, C.byref(pin), C.byref(pout), counts.data_ptr(),
                                          offsets.data_ptr(), self.invalid.data_ptr(), self.stream))
        return dst, counts, offsets

    def sort_binned(self, src: dict, n: int, in_counts, in_offsets, with_id=None, alias=False):
        """tpicb200_sort_binned; with `alias` the new bins overwrite in_counts/in_offsets."""
        dst = self.empty_particles(n, ("id" in src) if with_id is None else with_id)
        if alias:
            counts, offsets = in_counts, in_offsets
        else:
            counts = torch.zeros(self.layout.bin_count, dtype=torch.int32, device="cuda")
            offsets = torch.zeros(self.layout.bin_count + 1, dtype=torch.int32, device="cuda")
        pin, pout = self.struct(src, n), self.struct(dst, n)
        _lib.check(self.lib.tpicb200_sort_binned(self.ctx, C.byref(pin), in_counts.data_ptr(), in_offsets.data_ptr(),
                                                 C.byref(pout), counts.data_ptr(), offsets.data_ptr(),
                                                 self.invalid.data_ptr(), self.stream))
        return dst, counts, offsets

    def _tiled_shape(self):
        g = self.g
        mx = (g.nx + 3 + 3) // 4 * 4
        return (126, g.nz + 3, g.ny + 3, mx)

    def records(self, m) -> np.ndarray:
        """Mass coefficients of a device buffer in TPIC's record order (float64)."""
        a = m.cpu().numpy().astype(np.float64)
        if self.mass_layout == 1:
            a = np.ascontiguousarray(a.reshape(126, -1).T).ravel()
        elif self.mass_layout == 2:
            t = a.reshape(self._tiled_shape())[..., :self.g.nx + 3]
            a = np.ascontiguousarray(t.reshape(126, -1).T).ravel()
        return a

    def mass_from_records(self, rec: np.ndarray):
        a = rec.astype(self.np_fdt)
        if self.mass_layout == 1:
            a = np.ascontiguousarray(a.reshape(-1, 126).T).ravel()
        elif self.mass_layout == 2:
            g = self.g
            t = np.zeros(self._tiled_shape(), dtype=self.np_fdt)
            t[..., :g.nx + 3] = a.reshape(-1, 126).T.reshape(126, g.nz + 3, g.ny + 3, g.nx + 3)
            a = t.ravel()
        return torch.from_numpy(a).cuda()

    def moments(self):
        nodes = self.layout.node_count
        j = torch.zeros(3 * nodes, dtype=self.fdt, device="cuda")
        m = torch.zeros(self.layout.mass_count, dtype=self.fdt, device="cuda")
        return j, m

    def deposit(self, qom, parts: dict, n: int, bnode, j, m, counts=None, offsets=None, kind=0):
        p = self.struct(parts, n)
        _lib.check(self.lib.tpicb200_deposit(self.ctx, qom, C.byref(p), counts.data_ptr() if counts is not None else 0,
                                             offsets.data_ptr() if offsets is not None else 0, bnode.data_ptr(),
                                             j.data_ptr() if j is not None else 0,
                                             m.data_ptr() if m is not None else 0, kind,
                                             self.invalid.data_ptr(), self.stream))

    def fold(self, j, m):
        _lib.check(self.lib.tpicb200_fold_periodic(self.ctx, j.data_ptr() if j is not None else 0,
                                                   m.data_ptr() if m is not None else 0, self.stream))

    def mass_apply(self, m, vin):
        out = torch.zeros_like(vin)
        _lib.check(self.lib.tpicb200_mass_apply(self.ctx, m.data_ptr(), vin.data_ptr(), out.data_ptr(), self.stream))
        return out

    def field_solve(self, e, b, j, m):
        et = torch.zeros(3 * self.layout.node_count, dtype=torch.float64, device="cuda")
        res = _lib.GmresResult()
        _lib.check(self.lib.tpicb200_field_solve(self.ctx, e.data_ptr(), b.data_ptr(), j.data_ptr(), m.data_ptr(),
                                                 et.data_ptr(), C.byref(res), self.stream))
        return et, res

    def field_advance(self, e, b, etheta):
        bnext = torch.zeros_like(b)
        bnode = torch.zeros(3 * self.layout.node_count, dtype=self.fdt, device="cuda")
        _lib.check(self.lib.tpicb200_field_advance(self.ctx, e.data_ptr(), b.data_ptr(), etheta.data_ptr(),
                                                   bnext.data_ptr(), bnode.data_ptr(), self.stream))
        return bnext, bnode

    def magnetic_to_nodes(self, b):
        bnode = torch.zeros(3 * self.layout.node_count, dtype=self.fdt, device="cuda")
        _lib.check(self.lib.tpicb200_magnetic_to_nodes(self.ctx, b.data_ptr(), bnode.data_ptr(), self.stream))
        return bnode
