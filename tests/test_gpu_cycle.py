"""Whole-cycle parity: the CUDA cycle driver (tpicb200_prepare / tpicb200_cycle)
against the oracle's cycle on the same seeded plasma, and energy conservation
to the GMRES tolerance as the ECSIM method guarantees."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from fieldutil import interior_nodes, interior_records
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec, generate_species

pytestmark = pytest.mark.gpu


def c1_case(n=16, ncycles=3, npcel=(3, 3, 3)):
    """Plain ECSIM FP64 uniform plasma: 16^3 cells, 10^3 d_i, electrons q/m=-64,
    ions q/m=1, 27 ppc/species, vth_e=0.045, vth_i=0.0056, B0=(0,0,0.0195),
    dt=0.15, theta=0.5, GMRES rtol 1e-8."""
    g = GridSpec(n, n, n, 10.0, 10.0, 10.0)
    sp = [SpeciesSpec(qom=-64.0, rho=1.0, npcel=npcel, vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, rho=1.0, npcel=npcel, vth=(0.0056,) * 3)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, ncycles=ncycles, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))


def run_both(case, precision, cycles, mass_kind="scalar", mass_layout="records"):
    from tpic_b200.simulation import Simulation
    sim = Simulation(case, precision={0: "double", 1: "mixed"}[precision], mass_kind=mass_kind,
                     mass_layout=mass_layout)
    sim.prepare()
    reports = sim.run(cycles)
    arrays = O.case_species_arrays(case, precision, generate_species)
    oc = O.OracleCycle(case.grid, arrays, case.dt, case.theta, case.c, case.gmres_tol, precision, b0=case.fields.b0)
    oc.prepare()
    energies = [oc.cycle() for _ in range(cycles)]
    return sim, reports, oc, energies


@pytest.mark.parametrize("mass_layout,mass_kind", [("records", "scalar"), ("stencil-major", "scalar"),
                                                   ("records", "moments-f64"), ("stencil-major", "moments-f64"),
                                                   ("tiled", "scalar"), ("tiled", "moments-f64")])
def test_c1_cycle_matches_oracle_fp64(mass_layout, mass_kind):
    case = c1_case(n=16)
    sim, reports, oc, energies = run_both(case, 0, 3, mass_kind=mass_kind, mass_layout=mass_layout)
    for r, e, og in zip(reports, energies, oc.gmres):
        assert r.gmres_iterations == og.iterations
        # The Arnoldi steps of a restart cycle run as one graph: one wait for
        # the initial residual and one per restart cycle.
        assert r.gmres_host_waits == 1 + (r.gmres_iterations + 29) // 30
        assert abs(r.total_energy - O.total_energy(e, 2)) <= 1e-10 * abs(O.total_energy(e, 2))
        assert abs(r.field_energy[0] - e[0]) <= 1e-9 * abs(e[0]) + 1e-15
    for s in range(2):
        live = {k: v.cpu().numpy() for k, v in sim.live(s).items()}
        want = oc.species[s][1]
        assert np.array_equal(live["cell"], want["cell"])
        assert np.allclose(live["rx"], want["rx"], rtol=0, atol=1e-11)
        assert np.allclose(live["u"], want["u"], rtol=1e-9, atol=1e-13)
    g = case.grid
    e_gpu = interior_nodes(g, sim.field("e").cpu().numpy())
    e_cpu = interior_nodes(g, oc.e)
    # The plain FP64 form's field bar: 1e-10 relative to the field's scale.
    assert np.abs(e_gpu - e_cpu).max() <= 1e-10 * np.abs(e_cpu).max(), np.abs(e_gpu - e_cpu).max() / np.abs(e_cpu).max()
    b_gpu, b_cpu = sim.field("b_cell").cpu().numpy(), oc.b
    assert np.abs(b_gpu - b_cpu).max() <= 1e-10 * np.abs(b_cpu).max()


def test_c1_energy_conserved_fp64():
    case = c1_case(n=16)
    from tpic_b200.simulation import Simulation
    sim = Simulation(case, precision="double")
    sim.prepare()
    w0 = sim.energy()
    total0 = w0[0] + w0[1] + w0[2] + w0[7]
    reports = sim.run(3)
    for r in reports:
        assert abs(r.total_energy - total0) <= 1e-9 * total0
        assert r.gmres_relative_residual <= 1e-8


@pytest.mark.parametrize("mass_kind", ["scalar", "scalar-f64"])
def test_c1_mixed_precision_energy(mass_kind):
    case = c1_case(n=16)
    from tpic_b200.simulation import Simulation
    sim = Simulation(case, precision="mixed", mass_kind=mass_kind)
    sim.prepare()
    w0 = sim.energy()
    total0 = w0[0] + w0[1] + w0[2] + w0[7]
    reports = sim.run(3)
    for r in reports:
        assert abs(r.total_energy - total0) <= 1e-6 * total0


@pytest.mark.parametrize("mass_kind,bound", [("tf32", 1e-4), ("bf16x3", 1e-5)])
def test_c1_tensor_core_energy(mass_kind, bound):
    case = c1_case(n=16)
    from tpic_b200.simulation import Simulation
    sim = Simulation(case, precision="mixed", mass_kind=mass_kind)
    sim.prepare()
    w0 = sim.energy()
    total0 = w0[0] + w0[1] + w0[2] + w0[7]
    reports = sim.run(3)
    for r in reports:
        assert abs(r.total_energy - total0) <= bound * total0


@pytest.mark.parametrize("mass_kind,rel", [("tf32", 3e-3), ("bf16x3", 1e-4)])
def test_c1_fused_species_deposition(mass_kind, rel):
    """The cycle driver deposits every species of a cell in one tensor-core
    pass (species 0 then species 1 in one record stream per cell): the
    bootstrap deposition of both C1 species equals the oracle's sum within
    the form's operand rounding."""
    case = c1_case(n=16)
    from tpic_b200.simulation import Simulation
    sim = Simulation(case, precision="mixed", mass_kind=mass_kind, mass_layout="stencil-major")
    sim.prepare()
    arrays = O.case_species_arrays(case, 1, generate_species)
    oc = O.OracleCycle(case.grid, arrays, case.dt, case.theta, case.c, case.gmres_tol, 1, b0=case.fields.b0)
    oc.prepare()
    g = case.grid
    jg = interior_nodes(g, sim.field("j").cpu().numpy().astype(np.float64))
    jw = interior_nodes(g, oc.j)
    assert np.abs(jg - jw).max() <= rel * np.abs(jw).max()
    mass = sim.field("mass").cpu().numpy().astype(np.float64)
    mg = interior_records(g, np.ascontiguousarray(mass.reshape(126, -1).T).ravel())
    mw = interior_records(g, oc.m)
    assert np.abs(mg - mw).max() <= rel * np.abs(mw).max()


def test_cycle_fast_particles_fall_back_to_the_general_sort():
    """Electrons fast enough that some records cross two cells in one step:
    the mover's direction codes raise the fallback flag and the general sort
    produces the records; the cycle still matches the oracle bit for bit."""
    g = GridSpec(8, 8, 8, 5.0, 5.0, 5.0)
    sp = [SpeciesSpec(qom=-64.0, rho=1.0, npcel=(2, 2, 2), vth=(2.5,) * 3),
          SpeciesSpec(qom=1.0, rho=1.0, npcel=(2, 2, 2), vth=(0.01,) * 3)]
    case = Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, ncycles=2, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))
    sim, reports, oc, energies = run_both(case, 0, 2, mass_layout="stencil-major")
    for s in range(2):
        live = {k: v.cpu().numpy() for k, v in sim.live(s).items()}
        want = oc.species[s][1]
        assert np.array_equal(live["cell"], want["cell"])
        assert np.allclose(live["rx"], want["rx"], rtol=0, atol=1e-11)
    # Electrons fast enough to cross more than one cell per step exist.
    u = np.abs(oc.species[0][1]["u"])
    assert (u * case.dt / (g.lx / g.nx)).max() > 1.5
