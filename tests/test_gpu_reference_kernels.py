"""The library against the reference's own device kernels on the same GPU.

oracle/_ref/librefgpu.so (built by oracle/Makefile from oracle/refgpu/refgpu.cu
and the reference's headers) launches TPIC's sorted_current_kernel,
sorted_mass_matrix_scalar_kernel, sorted_mass_matrix_mma_kernel (FP64
mma.sync) and sorted_particle_mover_kernel on the sorted records, bins and
fields of a Simulation. In FP64 the library's deposition (current and mass,
folded by the oracle's restatement of the reference's fold) and mover agree
with them; every kernel of both sides is also timed
with CUDA events on the same inputs, and with TPICB200_REFERENCE_TIMINGS set
the figures are written to that path as JSON.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle as O
from reference_fixtures import ogrid
from tpic_b200 import _lib
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "librefgpu.so"


class RefGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("dz", C.c_double)]


class RefRecords(C.Structure):
    _fields_ = [("rx", C.c_void_p), ("ry", C.c_void_p), ("rz", C.c_void_p), ("u", C.c_void_p), ("v", C.c_void_p),
                ("w", C.c_void_p), ("q", C.c_void_p), ("cell", C.c_void_p), ("id", C.c_void_p),
                ("count", C.c_uint)]


def reference():
    if not LIB.exists():
        pytest.skip("oracle/_ref/librefgpu.so not built (make -C oracle with the reference tree)")
    lib = C.CDLL(str(LIB))
    args = [C.c_int, C.c_int, C.POINTER(RefGrid), C.POINTER(RefRecords)] + [C.c_void_p] * 4 + [C.c_double] * 3 + \
        [C.c_void_p] * 3
    lib.refgpu_deposit.argtypes = args
    lib.refgpu_move.argtypes = [C.c_int, C.POINTER(RefGrid), C.POINTER(RefRecords)] + [C.c_void_p] * 4 + \
        [C.c_double] * 3 + [C.c_void_p] * 3
    return lib


def uniform_case(n, ppc_axis):
    g = GridSpec(n, n, n, 10.0 * n / 16, 10.0 * n / 16, 10.0 * n / 16)
    npcel = (ppc_axis,) * 3
    sp = [SpeciesSpec(qom=-64.0, rho=1.0, npcel=npcel, vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, rho=1.0, npcel=npcel, vth=(0.0056,) * 3)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.01, -0.013, 0.0195)), seed=5)


def ref_records(slot, count, float_level=False):
    """The records as the reference's level reads them (float copies for the
    single-precision levels; a fraction that rounds to one in float is kept
    just below one, as a float store of the loader would)."""
    keep = []

    def as_float(t):
        f = t.float()
        if t.dtype == torch.float64 and t is not slot["u"] and t is not slot["v"] and t is not slot["w"]:
            f = torch.clamp(f, max=float(np.nextafter(np.float32(1), np.float32(0))))
        keep.append(f)
        return f

    pick = (lambda k: as_float(slot[k])) if float_level else (lambda k: slot[k])
    r = RefRecords(*[pick(k).data_ptr() for k in ("rx", "ry", "rz", "u", "v", "w")], slot["q"].data_ptr(),
                   slot["cell"].data_ptr(), slot["id"].data_ptr() if "id" in slot else 0, count)
    return r, keep


def timed(fn, stream, repeats=3, setup=None):
    total = 0.0
    for r in range(repeats + 1):
        if setup:
            setup()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        if r:
            total += a.elapsed_time(b)
    return total / repeats


def test_deposition_and_mover_match_the_reference_kernels_fp64():
    from tpic_b200.simulation import Simulation
    ref = reference()
    case = uniform_case(16, 3)
    sim = Simulation(case, precision="double", mass_layout="records", keep_ids=True, generate_on_device=True)
    sim.prepare()
    sim.materialize()
    lib, st, stream = sim.lib, sim.state, sim.stream
    s_ = sim._stream()
    g = case.grid
    grid = RefGrid(g.nx, g.ny, g.nz, *g.spacing)
    nodes = sim.layout.node_count
    j = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    failure = torch.zeros(1, dtype=torch.int32, device="cuda")
    invalid = torch.zeros(1, dtype=torch.int32, device="cuda")
    for kind in (1, 2):
        j.zero_()
        mass = torch.zeros(126 * nodes, dtype=torch.float64, device="cuda")
        for s, sp in enumerate(case.species):
            slot = sim.slots[s][st.current[s]]
            r, _ = ref_records(slot, st.slot[s][st.current[s]].count)
            cnt, off = sim.bins[s]
            for k, out in ((0, j), (kind, mass)):
                assert ref.refgpu_deposit(0, k, C.byref(grid), C.byref(r), cnt.data_ptr(), off.data_ptr(),
                                          st.b_node, out.data_ptr(), sp.qom, case.dt, case.c, failure.data_ptr(),
                                          invalid.data_ptr(), s_) == 0
        torch.cuda.synchronize()
        assert int(invalid.item()) == 0
        # The reference deposits into the endpoint nodes n as well; its fold
        # (shared-node sum, then ghosts) is the oracle's.
        jh, mh = j.cpu().numpy().copy(), mass.cpu().numpy().copy()
        O.load().oracle_fold(C.byref(ogrid(g)), O.ptr(jh), O.ptr(mh))
        for got, want in ((jh, sim.field("j").cpu().numpy()), (mh, sim.field("mass").cpu().numpy())):
            scale = float(np.abs(want).max())
            assert float(np.abs(got - want).max()) <= 1e-12 * scale, kind

    # Mover: the same sorted records, E_theta and B through both movers.
    rng = np.random.default_rng(3)
    etheta = torch.from_numpy(rng.normal(0.0, 0.02, 3 * nodes)).cuda()
    for s, sp in enumerate(case.species):
        slot = sim.slots[s][st.current[s]]
        n = st.slot[s][st.current[s]].count
        mine = {k: v.clone() for k, v in slot.items()}
        theirs = {k: v.clone() for k, v in slot.items()}
        p = sim._particles(mine, n)
        _lib.check(lib.tpicb200_mover(sim.ctx, sp.qom, C.byref(p), etheta.data_ptr(), st.b_node,
                                      invalid.data_ptr(), s_))
        r, _ = ref_records(theirs, n)
        cnt, off = sim.bins[s]
        assert ref.refgpu_move(0, C.byref(grid), C.byref(r), cnt.data_ptr(), off.data_ptr(), st.b_node,
                               etheta.data_ptr(), sp.qom, case.dt, case.c, failure.data_ptr(),
                               invalid.data_ptr(), s_) == 0
        torch.cuda.synchronize()
        assert int(invalid.item()) == 0
        assert torch.equal(mine["cell"], theirs["cell"])
        for k in ("rx", "ry", "rz", "u", "v", "w"):
            assert float((mine[k] - theirs[k]).abs().max()) <= 1e-13, k
        assert float((mine["cell"] != slot["cell"]).float().mean()) > 0.0


def stage_timings(precision, mass_kind, level_deposit, level_move, n=64, ppc_axis=4):
    """Device times (ms) of the deposition (all species, J and mass) and the
    mover (all species) of the library and of the reference's kernels at the
    given level, on the same sorted records and fields."""
    from tpic_b200.simulation import Simulation
    ref = reference()
    case = uniform_case(n, ppc_axis)
    sim = Simulation(case, precision=precision, mass_kind=mass_kind, mass_layout="stencil-major",
                     generate_on_device=True)
    sim.prepare()
    sim.materialize()
    lib, st, stream = sim.lib, sim.state, sim.stream
    s_ = sim._stream()
    g = case.grid
    grid = RefGrid(g.nx, g.ny, g.nz, *g.spacing)
    nodes = sim.layout.node_count
    ns = len(case.species)
    float_level = level_deposit != 0
    fdt = torch.float32 if float_level else torch.float64
    failure = torch.zeros(1, dtype=torch.int32, device="cuda")
    invalid = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = {"particles": int(sum(st.slot[s][st.current[s]].count for s in range(ns))), "cells": n ** 3}

    # The library: all species in one deposition call, as the cycle runs it.
    parts = (_lib.Particles * ns)(*[st.slot[s][st.current[s]] for s in range(ns)])
    qom = (C.c_double * ns)(*[sp.qom for sp in case.species])
    counts = (C.c_void_p * ns)(*[st.counts[s] for s in range(ns)])
    offsets = (C.c_void_p * ns)(*[st.offsets[s] for s in range(ns)])
    clear = lambda: _lib.check(lib.tpicb200_clear_moments(sim.ctx, st.j, st.mass, s_))
    out["ours_deposit_ms"] = timed(lambda: _lib.check(lib.tpicb200_deposit_species(
        sim.ctx, ns, qom, parts, counts, offsets, st.b_node, st.j, st.mass, st.mass_kind, invalid.data_ptr(), s_)),
        stream, setup=clear)
    out["ours_fold_ms"] = timed(lambda: _lib.check(lib.tpicb200_fold_periodic(sim.ctx, st.j, st.mass, s_)), stream,
                                setup=lambda: (clear(), _lib.check(lib.tpicb200_deposit_species(
                                    sim.ctx, ns, qom, parts, counts, offsets, st.b_node, st.j, st.mass,
                                    st.mass_kind, invalid.data_ptr(), s_))))

    # The reference: current, then scalar and matrix-core mass, per species.
    b = sim.field("b_node").to(fdt)
    j = torch.zeros(3 * nodes, dtype=fdt, device="cuda")
    recs = []
    for s in range(ns):
        r, keep = ref_records(sim.slots[s][st.current[s]], st.slot[s][st.current[s]].count, float_level)
        recs.append((r, keep))
    cnts = [sim.bins[s] for s in range(ns)]

    def ref_deposit(level, kind, target):
        for s, sp in enumerate(case.species):
            assert ref.refgpu_deposit(level, kind, C.byref(grid), C.byref(recs[s][0]), cnts[s][0].data_ptr(),
                                      cnts[s][1].data_ptr(), b.data_ptr(), target.data_ptr(), sp.qom, case.dt,
                                      case.c, failure.data_ptr(), invalid.data_ptr(), s_) == 0

    out["ref_current_ms"] = timed(lambda: ref_deposit(level_deposit, 0, j), stream, setup=j.zero_)
    mass_scalar = torch.zeros(126 * nodes, dtype=fdt, device="cuda")
    out["ref_mass_scalar_ms"] = timed(lambda: ref_deposit(level_deposit, 1, mass_scalar), stream,
                                      setup=mass_scalar.zero_)
    del mass_scalar
    mma_level = 0 if level_deposit == 0 else 2
    mass_mma = torch.zeros(126 * nodes, dtype=torch.float64, device="cuda")
    b_mma = b if mma_level == 0 else sim.field("b_node").float()
    if mma_level == 2:
        b = b_mma
    out["ref_mass_mma_ms"] = timed(lambda: ref_deposit(mma_level, 2, mass_mma), stream, setup=mass_mma.zero_)
    del mass_mma

    # Movers: on copies of the records (restored before each run).
    etheta = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    etheta_ref = etheta.to(fdt)
    saved = [{k: v.clone() for k, v in sim.slots[s][st.current[s]].items()} for s in range(ns)]

    def restore():
        for s in range(ns):
            for k, v in saved[s].items():
                sim.slots[s][st.current[s]][k].copy_(v)

    def our_move():
        for s, sp in enumerate(case.species):
            _lib.check(lib.tpicb200_mover(sim.ctx, sp.qom, C.byref(st.slot[s][st.current[s]]), etheta.data_ptr(),
                                          st.b_node, invalid.data_ptr(), s_))

    out["ours_mover_ms"] = timed(our_move, stream, setup=restore)
    if level_move is not None:
        b_move = sim.field("b_node").to(fdt)

        def ref_move():
            for s, sp in enumerate(case.species):
                assert ref.refgpu_move(level_move, C.byref(grid), C.byref(recs[s][0]), cnts[s][0].data_ptr(),
                                       cnts[s][1].data_ptr(), b_move.data_ptr(), etheta_ref.data_ptr(), sp.qom,
                                       case.dt, case.c, failure.data_ptr(), invalid.data_ptr(), s_) == 0

        def restore_ref():
            for s in range(ns):
                slot = sim.slots[s][st.current[s]]
                for k in ("rx", "ry", "rz", "u", "v", "w", "cell"):
                    src = saved[s][k]
                    if float_level and k != "cell":
                        src = src.float()
                        if k in ("rx", "ry", "rz"):
                            src = torch.clamp(src, max=float(np.nextafter(np.float32(1), np.float32(0))))
                    target = recs[s][1][("rx", "ry", "rz", "u", "v", "w").index(k)] if float_level and k != "cell" \
                        else slot[k]
                    target.copy_(src)

        out["ref_mover_ms"] = timed(ref_move, stream, setup=restore_ref)
    restore()
    sim.close()
    return out


@pytest.mark.parametrize("form", ["fp64", "fp64-moments", "mixed-bf16x3"])
def test_stage_times_against_the_reference_kernels(form):
    """Both sides timed on the same records (64^3 cells, 2 species x 64 per
    cell, sorted): the figures are reported; the check is that every kernel
    ran without raising the invalid flag."""
    if form == "fp64":
        t = stage_timings("double", "scalar", 0, 0)
    elif form == "fp64-moments":
        t = stage_timings("double", "moments-f64", 0, None)
    else:
        t = stage_timings("mixed", "bf16x3", 1, 1)
    t["form"] = form
    print(json.dumps(t))
    path = os.environ.get("TPICB200_REFERENCE_TIMINGS")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(t) + "\n")
    assert all(v > 0 for k, v in t.items() if k.endswith("_ms"))
