"""Device particle loading (tpicb200_load_species, tpicb200_center_velocities)
against the host generator on the same seeds: positions, cell keys and ids
bit for bit; velocities and charges within the last bits of the device's
log/cos/sin/cosh (FP64), or two FP32 ulps; centred velocities within the
rounding of the charge-weighted mean (fixed-order FP64 sums on the device,
pairwise sums on the host)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from test_gpu_decks import small_case
from tpic_b200 import _lib
from tpic_b200 import deck as D
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec, generate_species

pytestmark = pytest.mark.gpu


def uniform_case(quiet=False, center=False):
    g = GridSpec(6, 5, 4, 3.0, 2.5, 2.0)
    sp = [SpeciesSpec(qom=-64.0, rho=1.0, npcel=(3, 2, 2), vth=(0.045, 0.03, 0.02), drift=(0.01, -0.02, 0.0),
                      quiet=quiet, center=center),
          SpeciesSpec(qom=1.0, rho=0.7, npcel=(2, 2, 1), vth=(0.0056,) * 3, quiet=quiet)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.0, 0.0, 0.0195)), seed=9)


CASES = {
    "uniform": lambda: uniform_case(),
    "uniform-quiet-centred": lambda: uniform_case(quiet=True, center=True),
    "weibel2d-centred": lambda: small_case("weibel2d"),
    "twostream1d": lambda: small_case("twostream1d"),
    "harris2d": lambda: small_case("harris2d"),
}


def velocity_close(dev, host, scale, precision):
    if precision == "double":
        return np.all(np.abs(dev - host) <= 1e-13 * np.abs(host) + 1e-15 * scale)
    # Two FP32 ulps: the sampled value may round to a neighbour, and centring
    # narrows once more.
    ulp = np.spacing(np.abs(host.astype(np.float32))).astype(np.float64)
    return np.all(np.abs(dev.astype(np.float64) - host.astype(np.float64)) <= 2 * ulp)


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_load_matches_host_generator(name, precision):
    from tpic_b200.simulation import Simulation
    case = CASES[name]()
    sim = Simulation(case, precision=precision, keep_ids=True, generate_on_device=True)
    vdt = np.float64 if precision == "double" else np.float32
    for s, sp in enumerate(case.species):
        dev = {k: t.cpu().numpy() for k, t in sim.slots[s][0].items()}
        host = generate_species(case.grid, sp, s, seed=case.seed, velocity_dtype=vdt)
        for k in ("rx", "ry", "rz", "cell"):
            assert np.array_equal(dev[k], host[k]), (name, s, k)
        assert np.array_equal(dev["id"].view(np.uint64), host["id"])
        np.testing.assert_allclose(dev["q"], host["q"], rtol=1e-14, atol=0)
        scale = max(sp.vth) + max(abs(v) for v in sp.drift) + 1e-300
        for k in "uvw":
            assert velocity_close(dev[k], host[k], scale, precision), (name, s, k)
        if sp.center:
            drift = np.array(sp.drift)
            if sp.profile is not None:
                g = case.grid
                j = (dev["cell"] // (g.nx + 4)) % (g.ny + 4) - 2
                y = (j + dev["ry"]) * g.spacing[1]
                drift = sp.profile(y, y, y, j)[2]
                drift = [drift[a] for a in range(3)]
            for a, k in enumerate("uvw"):
                rest = dev[k].astype(np.float64) - drift[a]
                mean = np.sum(dev["q"] * rest) / np.sum(dev["q"])
                assert abs(mean) <= (1e-14 if precision == "double" else 1e-7) * scale


def test_device_load_chunks_equal_the_whole():
    """Any chunk [first, first + count) of a species loads on its own."""
    from tpic_b200.simulation import Simulation
    case = small_case("harris2d")
    sim = Simulation(case, precision="double", keep_ids=True, generate_on_device=True)
    deck = D.deck_of(case)
    lib = _lib.load()
    s, sp = 0, case.species[0]
    whole = {k: t.cpu().numpy() for k, t in sim.slots[s][0].items()}
    total = len(whole["q"])
    for first, count in ((0, 1), (137, 1000), (total - 77, 77)):
        buf = {k: torch.empty(count, dtype=t.dtype, device=t.device) for k, t in sim.slots[s][0].items()}
        p = Simulation._particles(buf, count)
        _lib.check(lib.tpicb200_load_species(sim.ctx, C.byref(deck), s, case.seed, first, C.byref(p), None,
                                             sim._stream()))
        for k, t in buf.items():
            assert np.array_equal(t.cpu().numpy(), whole[k][first:first + count]), (first, k)
    buf = {k: torch.empty(2, dtype=t.dtype, device=t.device) for k, t in sim.slots[s][0].items()}
    p = Simulation._particles(buf, 2)
    with pytest.raises(_lib.TpicError):
        _lib.check(lib.tpicb200_load_species(sim.ctx, C.byref(deck), s, case.seed, total - 1, C.byref(p), None,
                                             sim._stream()))
    other = D.deck_of(uniform_case())
    with pytest.raises(_lib.TpicError):
        _lib.check(lib.tpicb200_load_species(sim.ctx, C.byref(other), 0, 0, 0, C.byref(p), None, sim._stream()))


def test_device_loaded_run_equals_host_loaded_run():
    """The same deck run from device-loaded and host-loaded records (FP64):
    equal GMRES iteration counts and energies to 1e-12."""
    from tpic_b200.simulation import Simulation
    case = small_case("harris2d")
    runs = []
    for on_device in (True, False):
        sim = Simulation(case, precision="double", generate_on_device=on_device)
        sim.prepare()
        runs.append(sim.run(2))
    for a, b in zip(*runs):
        assert a.gmres_iterations == b.gmres_iterations
        assert abs(a.total_energy - b.total_energy) <= 1e-12 * abs(b.total_energy)
