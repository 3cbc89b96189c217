"""Snapshot output on the GPU: the output moments and the particles' output
coordinates (tpicb200_output_moments, tpicb200_output_particles) against the
oracle's restatement (oracle.output_moments), and snapshots written by the
runner (python -m tpic_b200 --run) read back."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from vtkread import field_data, read

pytestmark = pytest.mark.gpu
DECKS = Path(__file__).resolve().parents[1] / "tpic_b200" / "decks"


@pytest.mark.parametrize("precision", [0, 1])
def test_output_moments_and_particles_match_the_oracle(torch_cuda, precision):
    import torch
    from gpu_helpers import StageContext
    from reference_fixtures import species_arrays
    from tpic_b200 import _lib
    from tpic_b200.plasma import GridSpec
    g = GridSpec(6, 5, 4, 3.0, 2.5, 2.0)
    d = species_arrays(g, precision, vth=(0.2, 0.1, 0.3), npcel=(3, 2, 2), qom=-4.0)
    ctx = StageContext(g, precision=precision)
    parts = ctx.upload_particles(d)
    n = len(d["cell"])
    p = ctx.struct(parts, n)
    unique = g.nx * g.ny * g.nz
    rho = torch.zeros(unique, dtype=torch.float64, device="cuda")
    j = torch.zeros(3 * unique, dtype=torch.float64, device="cuda")
    pr = torch.zeros(6 * unique, dtype=torch.float64, device="cuda")
    _lib.check(ctx.lib.tpicb200_output_moments(ctx.ctx, -4.0, C.byref(p), rho.data_ptr(), j.data_ptr(),
                                               pr.data_ptr(), ctx.stream))
    pos = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    vel = torch.empty_like(pos)
    chg = torch.empty(n, dtype=torch.float64, device="cuda")
    _lib.check(ctx.lib.tpicb200_output_particles(ctx.ctx, C.byref(p), pos.data_ptr(), vel.data_ptr(),
                                                 chg.data_ptr(), ctx.stream))
    assert ctx.invalid_count() == 0
    want_rho, want_j, want_p = O.output_moments(g, d, -4.0)
    for got, want in ((rho, want_rho), (j, want_j), (pr, want_p)):
        got = got.cpu().numpy().reshape(want.shape)
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    # Charge is conserved exactly up to the sums' rounding.
    vol = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    assert rho.sum().item() * vol / (4 * np.pi) == pytest.approx(d["q"].sum(), rel=1e-13)
    ex, ey = g.nx + 4, g.ny + 4
    key = d["cell"].astype(np.int64)
    cell = [key % ex - 2, (key // ex) % ey - 2, key // (ex * ey) - 2]
    spacing = (g.lx / g.nx, g.ly / g.ny, g.lz / g.nz)
    want_pos = np.stack([(cell[a] + d[k]) * spacing[a] for a, k in enumerate(("rx", "ry", "rz"))], axis=1)
    assert np.array_equal(pos.cpu().numpy().reshape(n, 3), want_pos)
    want_vel = np.stack([d[k].astype(np.float64) for k in ("u", "v", "w")], axis=1)
    assert np.array_equal(vel.cpu().numpy().reshape(n, 3), want_vel)
    assert np.array_equal(chg.cpu().numpy(), d["q"])
    ctx.close()


def test_runner_writes_snapshots(torch_cuda, tmp_path):
    """A shrunk two-stream deck for 2 cycles with fields every cycle and
    particles every 2: E, B, rho and J files at cycles 0, 1, 2 and particle
    snapshots at 0 and 2; the final E file equals the run's E, the particle
    file holds every record once."""
    import torch
    from tpic_b200 import deck as D
    from tpic_b200.runner import main
    from tpic_b200.simulation import Simulation
    text = (DECKS / "twostream1d_1024.inp").read_text() + "\nnxc = 32\nnpcelx = 4 4 4\nncycles = 2\n"
    deck_path = tmp_path / "small.inp"
    deck_path.write_text(text)
    assert main(["--run", str(deck_path), "--output", str(tmp_path), "--precision", "double",
                 "--mass-matrix", "moments-f64", "--field-output-cycle", "1", "--particles-output-cycle", "2"]) == 0
    data = tmp_path / "data"
    names = sorted(p.name for p in data.iterdir())
    ns = D.parse(text).ns
    for cycle in (0, 1, 2):
        for arr in ["E", "B", "rho", "J"] + [f"{q}_{s}" for q in ("rho", "J") for s in range(ns)]:
            assert f"{arr}_t{cycle:06d}.vti" in names, (arr, cycle)
    assert "particles_t000000.pvtp" in names and "particles_t000002.pvtp" in names
    assert "particles_t000001.pvtp" not in names
    root, arrays, _ = read(data / "E_t000002.vti")
    fd = field_data(root)
    assert fd["cycle"] == 2 and fd["final_state"] == 1 and fd["state"] == "final"
    case = D.to_case(D.parse(text))
    assert fd["TimeValue"] == pytest.approx(2 * case.dt)
    sim = Simulation(case, precision="double", mass_kind="moments-f64", generate_on_device=True)
    sim.prepare()
    sim.run(2)
    g = case.grid
    e = sim.field("e").view(3, g.nz + 3, g.ny + 3, g.nx + 3)[:, 1:g.nz + 2, 1:g.ny + 2, 1:g.nx + 2]
    want = e.permute(1, 2, 3, 0).reshape(-1, 3).cpu().numpy()
    assert np.abs(arrays["E"] - want).max() <= 1e-12 * max(np.abs(want).max(), 1e-300)
    # Total rho is the sum of the species' rho.
    _, total, _ = read(data / "rho_t000002.vti")
    parts = [read(data / f"rho_{s}_t000002.vti")[1][f"rho_{s}"] for s in range(ns)]
    assert np.allclose(total["rho"], sum(parts), rtol=1e-14, atol=1e-14 * np.abs(total["rho"]).max())
    root, parr, _ = read(data / "particles_t000002_r000000.vtp")
    count = sum(case.grid.cells * sp.ppc for sp in case.species)
    assert int(root.find("PolyData/Piece").get("NumberOfPoints")) == count
    # Ids count within a species: (species, id) names a record.
    assert len(np.unique(parr["species"].astype(np.uint64) * np.uint64(1 << 40) + parr["id"])) == count
    lo = np.zeros(3)
    hi = np.array([g.lx, g.ly, g.lz])
    assert np.all(parr["position"] >= lo) and np.all(parr["position"] < hi)
    sim.close()
