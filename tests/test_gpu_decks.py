"""Deck-driven runs: the shipped TPIC-format decks, shrunk by appending
overrides (the last assignment of a key wins), loaded through the case
profiles and sampled startup fields, run through the CUDA cycle and the
oracle's cycle on the same particles and fields. Thin periodic axes (one
cell along z, or along y and z) are on the path, as in TPIC."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle as O
from fieldutil import interior_nodes
from tpic_b200 import deck as D
from tpic_b200.plasma import generate_species

pytestmark = pytest.mark.gpu

DECKS = Path(__file__).resolve().parent.parent / "tpic_b200" / "decks"

SMALL = {
    # Weibel seed on the anisotropic 2D plasma (centred electron velocities).
    "weibel2d": ("anisotropy2d_512.inp", """
Case = Weibel
WeibelSeedModeX = 1
WeibelSeedAmplitude = 2e-3
WeibelSeedGrowthRate = 0.05
nxc = 24
nyc = 16
Lx = 2.4
Ly = 1.6
npcelx = 3 3
npcely = 3 3
GMREStol = 1e-12
"""),
    # Two beams with the mode-1 density seed, one cell along y and z.
    "twostream1d": ("twostream1d_1024.inp", """
nxc = 64
npcelx = 16 16 16
Ly = 0.09817477042468103
Lz = 0.09817477042468103
GMREStol = 1e-12
"""),
    # Two Harris sheets with their X-point seeds, one cell along z.
    "harris2d": ("harris2d_256x128.inp", """
nxc = 32
nyc = 24
Lx = 8.0
Ly = 6.0
npcelx = 3 3 3 3
npcely = 2 2 2 2
GMREStol = 1e-12
"""),
}


def small_case(name):
    path, overrides = SMALL[name]
    return D.to_case(D.parse((DECKS / path).read_text() + overrides), seed=11)


def run_both(case, cycles, precision="double", mass_kind="scalar", mass_layout="stencil-major"):
    from tpic_b200.simulation import Simulation
    sim = Simulation(case, precision=precision, mass_kind=mass_kind, mass_layout=mass_layout)
    sim.prepare()
    reports = sim.run(cycles)
    p = 0 if precision == "double" else 1
    arrays = O.case_species_arrays(case, p, generate_species)
    oc = O.OracleCycle(case.grid, arrays, case.dt, case.theta, case.c, case.gmres_tol, p,
                       e_node=case.fields.e_node, b_cell=case.fields.b_cell)
    oc.prepare()
    energies = [oc.cycle() for _ in range(cycles)]
    return sim, reports, oc, energies


@pytest.mark.parametrize("name", sorted(SMALL))
def test_deck_cycle_matches_oracle_fp64(name):
    case = small_case(name)
    ns = len(case.species)
    sim, reports, oc, energies = run_both(case, 2)
    for r, e, og in zip(reports, energies, oc.gmres):
        assert r.gmres_iterations == og.iterations
        total = O.total_energy(e, ns)
        assert abs(r.total_energy - total) <= 1e-10 * abs(total)
        assert abs(r.field_energy[1] - e[1]) <= 1e-9 * abs(e[1]) + 1e-18
    for s in range(ns):
        live = {k: v.cpu().numpy() for k, v in sim.live(s).items()}
        want = oc.species[s][1]
        assert np.array_equal(live["cell"], want["cell"])
        assert np.allclose(live["rx"], want["rx"], rtol=0, atol=1e-11)
        assert np.allclose(live["u"], want["u"], rtol=1e-9, atol=1e-13)
    g = case.grid
    e_gpu = interior_nodes(g, sim.field("e").cpu().numpy())
    e_cpu = interior_nodes(g, oc.e)
    assert np.abs(e_gpu - e_cpu).max() <= 3e-10 * np.abs(e_cpu).max() + 1e-15


@pytest.mark.parametrize("name", sorted(SMALL))
@pytest.mark.parametrize("mass_kind,bound", [("scalar", 1e-6), ("bf16x3", 1e-5)])
def test_deck_cycle_energy_mixed(name, mass_kind, bound):
    """FP32 storage with the scalar and the BF16x3 tensor-core mass: the
    total energy stays at its start value to the form's bound."""
    from tpic_b200.simulation import Simulation
    case = small_case(name)
    sim = Simulation(case, precision="mixed", mass_kind=mass_kind, mass_layout="stencil-major")
    sim.prepare()
    w = sim.energy()
    ns = len(case.species)
    total0 = w[0] + w[1] + sum(w[2 + 5 * s] for s in range(ns))
    for r in sim.run(3):
        assert abs(r.total_energy - total0) <= bound * total0
