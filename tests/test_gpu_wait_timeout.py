"""Bounded device waits, tested without a fault.

tpicb200_inject_stall points one device wait at an mbarrier that nothing
arrives on, and tpicb200_set_wait_limit makes its bound short, so the wait
runs out every time:

- TPICB200_STALL_DEPOSIT: the BF16X3 tensor-core deposition's wait for the
  MMAs of chunk 0. Every CTA whose wait gives up leaves its chunk loop, waits
  (with the default bound) for the MMAs it has in flight, frees its tensor
  memory and adds 1 << 20 to the invalid counter; tpicb200_cycle returns
  TPICB200_INVALID_DATA.
- TPICB200_STALL_APPLY: the TMA-staged operator apply's wait for a stencil's
  mass box (tiled layout). The CTA waits (with the default bound) for its
  copies in flight and returns; the apply adds 1 << 21.

With the stall off and the default bound again, the next deposition / solve
on the same context equals the one before, bit for bit (both sum in a fixed
order), so the kernels that gave up left the device usable.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec

pytestmark = pytest.mark.gpu
DEPOSIT_BIT = 1 << 20
APPLY_BIT = 1 << 21
POLLS = 64


def small_case():
    g = GridSpec(12, 10, 8, 6.0, 5.0, 4.0)
    sp = [SpeciesSpec(qom=-64.0, npcel=(3, 3, 3), vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, npcel=(3, 3, 3), vth=(0.0056,) * 3)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))


def test_deposition_wait_timeout_is_reported_and_the_device_recovers(torch_cuda):
    import torch
    from tpic_b200 import _lib
    from tpic_b200.simulation import Simulation
    sim = Simulation(small_case(), precision="mixed", mass_kind="bf16x3", mass_layout="stencil-major")
    sim.prepare()
    lib, st = sim.lib, sim.state
    stream = C.c_void_p(sim.stream.cuda_stream)
    ns = st.ns
    parts = (_lib.Particles * ns)(*[st.slot[s][st.current[s]] for s in range(ns)])
    qom = (C.c_double * ns)(*[st.qom[s] for s in range(ns)])
    counts = (C.c_void_p * ns)(*[st.counts[s] for s in range(ns)])
    offsets = (C.c_void_p * ns)(*[st.offsets[s] for s in range(ns)])
    invalid = torch.zeros(1, dtype=torch.int32, device="cuda")

    def deposit():
        invalid.zero_()
        _lib.check(lib.tpicb200_clear_moments(sim.ctx, st.j, st.mass, stream))
        _lib.check(lib.tpicb200_deposit_species(sim.ctx, ns, qom, parts, counts, offsets, st.b_node, st.j, st.mass,
                                                st.mass_kind, invalid.data_ptr(), stream))
        _lib.check(lib.tpicb200_fold_periodic(sim.ctx, st.j, st.mass, stream))
        torch.cuda.synchronize()
        return sim.field("mass").clone(), sim.field("j").clone(), int(invalid.item())

    ref_mass, ref_j, bad = deposit()
    assert bad == 0
    assert lib.tpicb200_inject_stall(sim.ctx, _lib.STALL_DEPOSIT, 0) == _lib.INVALID_ARGUMENT
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, POLLS))
    _lib.check(lib.tpicb200_inject_stall(sim.ctx, _lib.STALL_DEPOSIT, 1))
    for _ in range(3):
        _, _, bad = deposit()
        assert bad >= DEPOSIT_BIT and bad % DEPOSIT_BIT == 0, bad
    # Stall off, default bound: the same moments as before the timeouts.
    _lib.check(lib.tpicb200_inject_stall(sim.ctx, _lib.STALL_NONE, 0))
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, 0))
    mass, j, bad = deposit()
    assert bad == 0
    assert torch.equal(mass, ref_mass) and torch.equal(j, ref_j)
    # A cycle whose deposition gives up returns TPICB200_INVALID_DATA.
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, POLLS))
    _lib.check(lib.tpicb200_inject_stall(sim.ctx, _lib.STALL_DEPOSIT, 1))
    count = C.c_uint32(0)
    _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 1, stream))
    status = lib.tpicb200_cycle(sim.ctx, C.byref(st), 1, None, stream)
    assert status == _lib.INVALID_DATA, lib.tpicb200_last_error()
    assert b"invalid" in lib.tpicb200_last_error()
    _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 1, stream))
    assert count.value >= DEPOSIT_BIT
    _lib.check(lib.tpicb200_inject_stall(sim.ctx, _lib.STALL_NONE, 0))
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, 0))
    sim.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_apply_wait_timeout_is_reported_and_the_device_recovers(torch_cuda, precision):
    import torch
    from fieldutil import periodic_cell_field, periodic_node_field, smooth_random_unique
    from gpu_helpers import StageContext
    from test_gpu_tiled_apply import random_mass
    from tpic_b200 import _lib
    g = GridSpec(12, 10, 8, 3.0, 2.5, 2.0)
    rng = np.random.default_rng(3)
    ctx = StageContext(g, precision=precision, dt=0.2, tol=1e-10, mass_layout=2)
    m = ctx.mass_from_records(random_mass(g, rng))
    e = ctx.field(periodic_node_field(g, smooth_random_unique(g, rng, 0.01)))
    b = ctx.field(periodic_cell_field(g, smooth_random_unique(g, rng, 0.05)))
    j = ctx.field(periodic_node_field(g, smooth_random_unique(g, rng, 0.02)))
    lib = ctx.lib
    count = C.c_uint32(0)

    def solve():
        et = torch.zeros(3 * ctx.layout.node_count, dtype=torch.float64, device="cuda")
        res = _lib.GmresResult()
        status = lib.tpicb200_field_solve(ctx.ctx, e.data_ptr(), b.data_ptr(), j.data_ptr(), m.data_ptr(),
                                          et.data_ptr(), C.byref(res), ctx.stream)
        _lib.check(lib.tpicb200_read_invalid(ctx.ctx, C.byref(count), 1, ctx.stream))
        return status, et, res, count.value

    status, ref, ref_res, bad = solve()
    assert status == _lib.SUCCESS and bad == 0 and ref_res.converged
    assert lib.tpicb200_inject_stall(ctx.ctx, _lib.STALL_APPLY, 14) == _lib.INVALID_ARGUMENT
    _lib.check(lib.tpicb200_set_wait_limit(ctx.ctx, POLLS))
    for stencil in (0, 5, 13):
        _lib.check(lib.tpicb200_inject_stall(ctx.ctx, _lib.STALL_APPLY, stencil))
        status, _, _, bad = solve()
        # The solve runs on rows the apply did not write; whatever it reports,
        # the counter names the apply's timeouts.
        assert status in (_lib.SUCCESS, _lib.NOT_CONVERGED, _lib.INVALID_DATA), lib.tpicb200_last_error()
        assert bad >= APPLY_BIT, (stencil, bad)
    _lib.check(lib.tpicb200_inject_stall(ctx.ctx, _lib.STALL_NONE, 0))
    _lib.check(lib.tpicb200_set_wait_limit(ctx.ctx, 0))
    status, et, res, bad = solve()
    assert status == _lib.SUCCESS and bad == 0
    assert res.iterations == ref_res.iterations and torch.equal(et, ref)
    ctx.close()
