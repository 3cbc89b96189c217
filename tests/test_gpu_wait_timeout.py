"""Bounded device waits of the BF16X3 tensor-core deposition.

tpicb200_set_wait_limit(ctx, 1) leaves the stream kernel's chunk-loop waits
(the wait for a chunk's MMAs and for the issuer's published decision) one
poll each, so they give up whenever the awaited event has not happened at
the first poll. A CTA whose wait gave up leaves its chunk loop, waits (with
the default bound) for the last chunk it issued and frees its tensor memory;
the deposition adds 1 << 20 to the invalid counter and tpicb200_cycle returns
TPICB200_INVALID_DATA. With the default bound restored, the next deposition on
the same context equals the one before the timeouts bit for bit (the BF16x3
moments are summed in a fixed order), so the kernels that gave up left the
device usable. No fault is caused: every wait ends by its bound.
"""
from __future__ import annotations

import ctypes as C

import pytest

from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec

pytestmark = pytest.mark.gpu
ERROR_BIT = 1 << 20


def small_case():
    g = GridSpec(12, 10, 8, 6.0, 5.0, 4.0)
    sp = [SpeciesSpec(qom=-64.0, npcel=(3, 3, 3), vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, npcel=(3, 3, 3), vth=(0.0056,) * 3)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))


def test_wait_timeout_is_reported_and_the_device_recovers(torch_cuda):
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
        _lib.check(lib.tpicb200_clear_moments(sim.ctx, st.j, st.mass, stream))
        _lib.check(lib.tpicb200_deposit_species(sim.ctx, ns, qom, parts, counts, offsets, st.b_node, st.j, st.mass,
                                                st.mass_kind, invalid.data_ptr(), stream))
        _lib.check(lib.tpicb200_fold_periodic(sim.ctx, st.j, st.mass, stream))
        torch.cuda.synchronize()
        return sim.field("mass").clone(), sim.field("j").clone(), int(invalid.item())

    ref_mass, ref_j, bad = deposit()
    assert bad == 0
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, 1))
    timed_out = 0
    for _ in range(10):
        invalid.zero_()
        _, _, bad = deposit()
        assert bad == 0 or bad >= ERROR_BIT, bad
        timed_out += bad >= ERROR_BIT
    assert timed_out > 0
    # The default bound again: the same moments as before the timeouts.
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, 0))
    invalid.zero_()
    mass, j, bad = deposit()
    assert bad == 0
    assert torch.equal(mass, ref_mass) and torch.equal(j, ref_j)
    # A cycle whose deposition gives up returns TPICB200_INVALID_DATA.
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, 1))
    statuses = []
    for _ in range(5):
        count = C.c_uint32(0)
        _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 1, stream))
        statuses.append(lib.tpicb200_cycle(sim.ctx, C.byref(st), 1, None, stream))
        assert statuses[-1] in (_lib.SUCCESS, _lib.INVALID_DATA), lib.tpicb200_last_error()
        if statuses[-1] == _lib.INVALID_DATA:
            break
    assert _lib.INVALID_DATA in statuses
    assert b"invalid" in lib.tpicb200_last_error()
    count = C.c_uint32(0)
    _lib.check(lib.tpicb200_read_invalid(sim.ctx, C.byref(count), 1, stream))
    assert count.value >= ERROR_BIT
    _lib.check(lib.tpicb200_set_wait_limit(sim.ctx, 0))
    sim.close()
