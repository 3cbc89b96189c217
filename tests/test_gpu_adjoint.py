"""The adjoint C ABI on the GPU.

- Whole backward cycles (tpicb200_cycle_forward / tpicb200_cycle_backward)
  against the oracle's FP64 adjoint on the same seeded plasma: the gradients
  of the final field energy with respect to the starting E, B and every
  record's position, velocity and charge.
- The per-stage backward entry points composed by hand equal the fused
  cycle backward.
- Checkpoint-recompute equals keeping every tape.
- Parameter gradients on shrunk two-stream (beam drift, density-seed
  amplitude) and anisotropy (T_perp/T_par) decks against central finite
  differences of the FP64 forward run, for the FP64 adjoint and for the
  mixed-precision runs the decks use (FP32 scalar mass on the two-stream
  deck, BF16x3 tensor-core mass on the anisotropy deck): within 1e-4
  relative.

A PIC run with CIC weights is only piecewise smooth in its parameters: the
weights are continuous but their slopes jump where a particle's trajectory
meets a cell face, so the final energy has kinks at the parameter values
where that happens. The adjoint is the exact derivative of the discrete run
at the nominal parameter; a central difference equals it only when no kink
lies within +-h. The differences here therefore shrink h (from 1e-4 of the
parameter by factors of 10) until the two one-sided differences agree within
1e-3, which a kink inside the interval breaks.

TPIC has no adjoint: nothing in the reference pins these; the oracle's
adjoint is itself pinned to central differences (test_oracle_adjoint.py).
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from fieldutil import periodic_cell_field, periodic_node_field
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec, generate_species

pytestmark = pytest.mark.gpu
DECKS = Path(__file__).resolve().parents[1] / "tpic_b200" / "decks"


def small_case(seed=5, g=GridSpec(6, 5, 4, 3.0, 2.5, 2.0), tol=1e-12):
    rng = np.random.default_rng(seed)
    species = [SpeciesSpec(qom=-16.0, npcel=(2, 2, 2), vth=(0.08,) * 3),
               SpeciesSpec(qom=1.0, npcel=(2, 2, 2), vth=(0.02,) * 3)]
    e0 = periodic_node_field(g, 0.01 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    b0 = periodic_cell_field(g, 0.0195 + 0.005 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    return Case(g, species, dt=0.4, theta=0.5, gmres_tol=tol, fields=FieldInit(e_node=e0, b_cell=b0))


def simulation(case, precision="double", mass_kind="scalar", **kw):
    from tpic_b200.simulation import Simulation
    return Simulation(case, precision=precision, mass_kind=mass_kind, keep_ids=True, gmres_max_iterations=500, **kw)


def gpu_gradients(case, cycles, every, mass_kind="scalar", precision="double", we=1.0, wb=1.0):
    from tpic_b200.adjoint import AdjointRun
    sim = simulation(case, precision, mass_kind)
    sim.prepare()
    run = AdjointRun(sim, every=every)
    run.forward(cycles)
    adj = run.backward(we, wb)
    return sim, run, adj


def oracle_gradients(case, cycles):
    arrays = [(sp.qom, generate_species(case.grid, sp, s, seed=case.seed)) for s, sp in enumerate(case.species)]
    oc = O.OracleCycle(case.grid, arrays, case.dt, case.theta, case.c, case.gmres_tol, 0, max_iterations=500,
                       e_node=case.fields.e_node, b_cell=case.fields.b_cell)
    oc.prepare()
    oa = O.OracleAdjoint(oc)
    oa.forward(cycles)
    e_bar, b_bar = oa.energy_gradient(1.0, 1.0)
    return oa.backward(e_bar, b_bar)


def unique_node_values(g, f):
    return f.reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]


def unique_cell_values(g, f):
    return f.reshape(3, g.nz + 2, g.ny + 2, g.nx + 2)[:, 1:g.nz + 1, 1:g.ny + 1, 1:g.nx + 1]


def relative(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("mass_kind", ["scalar", "moments-f64"])
def test_cycle_backward_matches_the_oracle_adjoint(torch_cuda, mass_kind):
    case = small_case()
    g = case.grid
    sim, run, adj = gpu_gradients(case, 3, 3, mass_kind)
    e_want, b_want, parts = oracle_gradients(case, 3)
    assert relative(unique_node_values(g, adj.e_bar.cpu().numpy()), unique_node_values(g, e_want)) <= 1e-9
    assert relative(unique_cell_values(g, adj.b_bar.cpu().numpy()), unique_cell_values(g, b_want)) <= 1e-9
    for s in range(2):
        got = adj.species_gradients(s)
        n = adj.count[s]
        want = {"x": parts[s]["x"].reshape(3, n), "v": parts[s]["v"].reshape(3, n), "q": parts[s]["q"]}
        for k in ("x", "v", "q"):
            assert relative(got[k], want[k]) <= 1e-9, (s, k, relative(got[k], want[k]))
    sim.close()


def test_checkpoint_recompute_equals_keeping_every_tape(torch_cuda):
    case = small_case(seed=7)
    g = case.grid
    _, run_all, full = gpu_gradients(case, 6, 6, "moments-f64")
    _, run_cp, part = gpu_gradients(case, 6, 2, "moments-f64")
    assert run_cp.stats.checkpoints == 3 and run_all.stats.checkpoints == 1
    assert relative(part.e_bar.cpu().numpy(), full.e_bar.cpu().numpy()) <= 1e-12
    assert relative(part.b_bar.cpu().numpy(), full.b_bar.cpu().numpy()) <= 1e-12
    for s in range(2):
        a, b = part.species_gradients(s), full.species_gradients(s)
        for k in ("x", "v", "q"):
            assert relative(a[k], b[k]) <= 1e-12, (s, k)


@pytest.mark.parametrize("precision,mass_kind", [("double", "scalar"), ("mixed", "bf16x3")])
def test_stage_backwards_compose_to_the_cycle_backward(torch_cuda, precision, mass_kind):
    """One cycle's backward through the per-stage entry points equals
    tpicb200_cycle_backward on the same tape. Both deposit M again from the
    tape, so the forms here are ones whose deposition sums in a fixed order
    or in FP64 (the FP32 scalar form's float atomics would make the two M
    differ at 1e-7)."""
    import torch
    from tpic_b200 import _lib
    from tpic_b200.adjoint import AdjointBuffers, TapeBuffers
    case = small_case(seed=3)
    sim = simulation(case, precision, mass_kind)
    sim.prepare()
    lib, st = sim.lib, sim.state
    stream = C.c_void_p(sim.stream.cuda_stream)
    tape = TapeBuffers(sim)
    _lib.check(lib.tpicb200_cycle_forward(sim.ctx, C.byref(st), C.byref(tape.struct), None, stream))
    fused, staged = AdjointBuffers(sim), AdjointBuffers(sim)
    for a in (fused, staged):
        _lib.check(lib.tpicb200_adjoint_energy(sim.ctx, st.e, st.b_cell, 1.0, 1.0, C.byref(a.struct), stream))
        # Nonzero record gradients, as after a later cycle's backward.
        gen = torch.Generator(device="cuda").manual_seed(1)
        for s in range(2):
            a.x_bar[s].copy_(1e-3 * torch.randn(a.x_bar[s].shape, generator=gen, device="cuda", dtype=torch.float64))
            a.v_bar[s].copy_(1e-2 * torch.randn(a.v_bar[s].shape, generator=gen, device="cuda", dtype=torch.float64))
    _lib.check(lib.tpicb200_cycle_backward(sim.ctx, C.byref(tape.struct), C.byref(fused.struct), None, stream))
    # By stage.
    a = staged
    dt, th = case.dt, case.theta
    kfac = 4 * math.pi * th * dt
    g = case.grid
    volume = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    _lib.check(lib.tpicb200_magnetic_to_nodes(sim.ctx, tape.struct.b_cell, a.struct.b_node, stream))
    _lib.check(lib.tpicb200_clear_moments(sim.ctx, a.struct.j, a.struct.mass, stream))
    parts = (_lib.Particles * 2)(*tape.struct.species[:2])
    qom = (C.c_double * 2)(*tape.struct.qom[:2])
    counts = (C.c_void_p * 2)(*tape.struct.counts[:2])
    offsets = (C.c_void_p * 2)(*tape.struct.offsets[:2])
    _lib.check(lib.tpicb200_deposit_species(sim.ctx, 2, qom, parts, counts, offsets, a.struct.b_node, a.struct.j,
                                            a.struct.mass, tape.struct.mass_kind, None, stream))
    _lib.check(lib.tpicb200_fold_periodic(sim.ctx, a.struct.j, a.struct.mass, stream))
    _lib.check(lib.tpicb200_field_advance_backward(sim.ctx, a.e_bar.data_ptr(), a.b_bar.data_ptr(),
                                                   a.e_theta_bar.data_ptr(), stream))
    a.b_node_bar.zero_()
    for s in range(2):
        p = tape.struct.species[s]
        _lib.check(lib.tpicb200_mover_backward(sim.ctx, tape.struct.qom[s], C.byref(p), tape.struct.e_theta,
                                               a.struct.b_node, a.count[s], a.x_bar[s].data_ptr(),
                                               a.v_bar[s].data_ptr(), a.e_theta_bar.data_ptr(),
                                               a.b_node_bar.data_ptr(), None, stream))
    _lib.check(lib.tpicb200_field_solve_backward(sim.ctx, a.struct.mass, a.e_theta_bar.data_ptr(), a.lam.data_ptr(),
                                                 a.e_bar.data_ptr(), a.b_bar.data_ptr(), None, stream))
    for s in range(2):
        p = tape.struct.species[s]
        _lib.check(lib.tpicb200_deposit_backward(sim.ctx, tape.struct.qom[s], C.byref(p), a.struct.b_node,
                                                 a.lam.data_ptr(), -kfac, a.lam.data_ptr(), tape.struct.e_theta,
                                                 -kfac / volume, a.count[s], a.x_bar[s].data_ptr(),
                                                 a.v_bar[s].data_ptr(), a.q_bar[s].data_ptr(),
                                                 a.b_node_bar.data_ptr(), None, stream))
    _lib.check(lib.tpicb200_magnetic_to_nodes_backward(sim.ctx, a.b_node_bar.data_ptr(), a.b_bar.data_ptr(), stream))
    torch.cuda.synchronize()
    assert relative(staged.e_bar.cpu().numpy(), fused.e_bar.cpu().numpy()) <= 1e-12
    assert relative(staged.b_bar.cpu().numpy(), fused.b_bar.cpu().numpy()) <= 1e-12
    for s in range(2):
        x, y = staged.species_gradients(s), fused.species_gradients(s)
        for k in ("x", "v", "q"):
            assert relative(x[k], y[k]) <= 1e-12, (s, k)
    sim.close()


def test_backward_rejects_smoothing_and_missing_ids(torch_cuda):
    from tpic_b200 import _lib
    from tpic_b200.adjoint import AdjointBuffers, TapeBuffers
    from tpic_b200.simulation import Simulation
    case = small_case()
    sim = Simulation(case, precision="double", keep_ids=True, smoothing=(2, 0.5, 0))
    sim.prepare()
    tape = TapeBuffers(sim)
    stream = C.c_void_p(sim.stream.cuda_stream)
    assert sim.lib.tpicb200_cycle_forward(sim.ctx, C.byref(sim.state), C.byref(tape.struct), None,
                                          stream) == _lib.INVALID_STATE
    sim.close()
    plain = Simulation(case, precision="double")
    plain.prepare()
    with pytest.raises(ValueError):
        from tpic_b200.adjoint import AdjointRun
        AdjointRun(plain)
    tape = TapeBuffers(plain)
    adj = AdjointBuffers(plain)
    for s in range(2):
        tape.struct.species[s].id = None
    assert plain.lib.tpicb200_cycle_backward(plain.ctx, C.byref(tape.struct), C.byref(adj.struct), None,
                                             stream) == _lib.INVALID_ARGUMENT
    plain.close()


# ---- parameter gradients on shrunk decks --------------------------------------------

TWO_STREAM = ("twostream1d_1024.inp", "\nnxc = 64\nnpcelx = 32 32 32\nncycles = 10\nGMREStol = 1e-14\n")
ANISOTROPY = ("anisotropy2d_512.inp", "\nnxc = 24\nnyc = 24\nLx = 2.4\nLy = 2.4\nnpcelx = 4 4\nnpcely = 4 4\n"
                                      "ncycles = 20\nGMREStol = 1e-14\n")


def deck_text(spec, extra=""):
    path, overrides = spec
    return (DECKS / path).read_text() + overrides + extra


def final_energy(text, precision, mass_kind, which):
    from tpic_b200 import deck as D
    from tpic_b200.simulation import Simulation
    parsed = D.parse(text)
    case = D.to_case(parsed)
    sim = Simulation(case, precision=precision, mass_kind=mass_kind, gmres_max_iterations=500)
    sim.prepare()
    r = sim.run(parsed.ncycles)[-1]
    sim.close()
    return sum(r.field_energy[i] for i in which)


def deck_adjoint(text, precision, mass_kind, every, we, wb):
    from tpic_b200 import deck as D
    parsed = D.parse(text)
    case = D.to_case(parsed)
    sim, run, adj = gpu_gradients(case, parsed.ncycles, every, mass_kind, precision, we, wb)
    return parsed, sim, run, adj


def kink_free_difference(energy, p0, rel=1e-4, levels=6, agree=1e-3):
    """Central difference of energy(p) at p0 with the largest h = rel |p0|
    10^-k whose one-sided differences agree within `agree` (no kink inside
    +-h); returns (difference, h)."""
    l0 = energy(p0)
    h = rel * abs(p0)
    for _ in range(levels):
        lp, lm = energy(p0 + h), energy(p0 - h)
        right, left = (lp - l0) / h, (l0 - lm) / h
        if abs(right - left) <= agree * max(abs(right), abs(left)):
            return (lp - lm) / (2 * h), h
        h /= 10
    raise AssertionError(f"no kink-free step down to h = {h * 10:g}")


@pytest.mark.parametrize("precision,mass_kind", [("double", "scalar"), ("mixed", "scalar")])
def test_two_stream_gradients_match_central_differences(torch_cuda, precision, mass_kind):
    from tpic_b200.adjoint import contract, two_stream_tangents
    text = deck_text(TWO_STREAM)
    parsed, sim, run, adj = deck_adjoint(text, precision, mass_kind, 10, 1.0, 1.0)
    tangents = two_stream_tangents(run, parsed)
    grad_drift = contract(sim, adj, tangents["drift"])
    grad_amp = contract(sim, adj, tangents["amplitude"])
    sim.close()
    u0, a = parsed.species[0].drift[0], parsed.two_stream_amplitude
    fd_drift, _ = kink_free_difference(
        lambda u: final_energy(deck_text(TWO_STREAM, f"\nu0 = {u!r} {-u!r} 0.0\n"), "double", "scalar", (0, 1)), u0)
    fd_amp, _ = kink_free_difference(
        lambda x: final_energy(deck_text(TWO_STREAM, f"\nTwoStreamSeedDensityAmplitude = {x!r}\n"), "double",
                               "scalar", (0, 1)), a)
    assert abs(grad_drift - fd_drift) <= 1e-4 * abs(fd_drift), (grad_drift, fd_drift)
    assert abs(grad_amp - fd_amp) <= 1e-4 * abs(fd_amp), (grad_amp, fd_amp)


@pytest.mark.parametrize("precision,mass_kind", [("double", "moments-f64"), ("mixed", "bf16x3")])
def test_anisotropy_gradient_matches_central_differences(torch_cuda, precision, mass_kind):
    from tpic_b200.adjoint import anisotropy_tangent, contract
    text = deck_text(ANISOTROPY)
    parsed, sim, run, adj = deck_adjoint(text, precision, mass_kind, 20, 0.0, 1.0)
    vpar, vperp = parsed.species[0].vth[0], parsed.species[0].vth[1]
    ratio = (vperp / vpar) ** 2
    grad = contract(sim, adj, anisotropy_tangent(run, 0, 0, ratio))
    sim.close()

    def energy(r):
        v = vpar * math.sqrt(r)
        return final_energy(deck_text(ANISOTROPY, f"\nvth = {v!r} 0.003\nwth = {v!r} 0.003\n"), "double",
                            "moments-f64", (1,))
    fd, _ = kink_free_difference(energy, ratio)
    assert abs(grad - fd) <= 1e-4 * abs(fd), (grad, fd)
