"""Gauss-law residual on the GPU (tpicb200_gauss_field, tpicb200_gauss_charge,
tpic_b200.output.GaussSampler) against the oracle's restatement
(oracle.gauss_half_divergence, oracle.gauss_cell_charge), in the form of the
reference's own check (docs/developer/gauss_diagnostic.md, section 10): two
chained samples, the second begun where the first finishes, compared cell by
cell and sum by sum. The oracle evaluates the same states (E and the records
read back from the device); the charge is deposited with FP64 atomics, in any
order, so the cells agree to 1e-12 of the largest value rather than bit for
bit. Double and mixed storage, with and without smoothing."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec

pytestmark = pytest.mark.gpu


def small_case():
    g = GridSpec(12, 10, 8, 6.0, 5.0, 4.0)
    sp = [SpeciesSpec(qom=-64.0, npcel=(3, 3, 3), vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, npcel=(3, 3, 3), vth=(0.0056,) * 3)]
    return Case(g, sp, dt=0.15, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))


def host_state(sim):
    e = sim.field("e").double().cpu().numpy()
    species = []
    for s in range(sim.state.ns):
        live = sim.live(s)
        species.append({k: live[k].cpu().numpy() for k in ("rx", "ry", "rz", "q", "cell")})
    return e, species


def close(got, want, rel=1e-12):
    scale = max(np.abs(want).max(), 1e-300)
    assert np.abs(got - want).max() <= rel * scale, np.abs(got - want).max() / scale


@pytest.mark.parametrize("precision,smoothing", [("double", (0, 1.0, 0)), ("mixed", (0, 1.0, 0)),
                                                 ("double", (2, 0.5, 0)), ("mixed", (3, 0.5, 1))])
def test_chained_samples_match_the_oracle(torch_cuda, precision, smoothing):
    from tpic_b200.output import GaussSampler
    from tpic_b200.simulation import Simulation
    case = small_case()
    g = case.grid
    sim = Simulation(case, precision=precision, mass_kind="scalar", mass_layout="stencil-major", smoothing=smoothing)
    sim.prepare()
    gs = GaussSampler(sim)
    cells = g.nx * g.ny * g.nz
    sm = smoothing if smoothing[0] > 0 else (0, 1.0, 0)

    # Begin at state 0: stash = divC(E^0)/2 - c(x^{1/2}).
    assert gs.step(0, True) is None
    e, species = host_state(sim)
    c0 = O.gauss_cell_charge(g, species, sm)
    stash0 = O.gauss_half_divergence(g, e) - c0
    close(gs.stash.cpu().numpy().reshape(g.nz, g.ny, g.nx), stash0)

    # State 1 finishes sample 0 and begins sample 1.
    sim.run(1)
    s0 = gs.step(1, True)
    e, species = host_state(sim)
    r0 = stash0 + O.gauss_half_divergence(g, e)
    close(gs.residual.cpu().numpy().reshape(g.nz, g.ny, g.nx), r0)
    assert s0.cycle == 0 and s0.time == pytest.approx(0.5 * case.dt)
    assert s0.rms[0] == pytest.approx(math.sqrt(np.sum(r0 * r0) / cells), rel=1e-12)
    assert s0.rms[1] == 0.0 and s0.rms[2] == 0.0
    assert s0.rms[3] == pytest.approx(math.sqrt(np.sum(c0 * c0) / cells), rel=1e-12)
    c1 = O.gauss_cell_charge(g, species, sm)
    stash1 = O.gauss_half_divergence(g, e) - c1

    # State 2 finishes sample 1: its drift is measured against sample 0.
    sim.run(1)
    s1 = gs.step(2, False)
    e, _ = host_state(sim)
    r1 = stash1 + O.gauss_half_divergence(g, e)
    close(gs.residual.cpu().numpy().reshape(g.nz, g.ny, g.nx), r1)
    assert s1.cycle == 1 and s1.time == pytest.approx(1.5 * case.dt)
    assert s1.rms[0] == pytest.approx(math.sqrt(np.sum(r1 * r1) / cells), rel=1e-12)
    drift = math.sqrt(np.sum((r1 - r0) ** 2) / cells)
    assert s1.rms[1] == pytest.approx(drift, rel=1e-9, abs=1e-12 * s1.rms[0])
    assert s1.rms[3] == pytest.approx(math.sqrt(np.sum(c1 * c1) / cells), rel=1e-12)
    # The residual is small against the charge (Gauss's law holds to the
    # particle noise and the solver tolerance).
    assert s1.rms[1] < s1.rms[3]
    assert gs.step(2, False) is None
    sim.close()


def test_runner_writes_gauss_rows_and_arrays(torch_cuda, tmp_path):
    """A deck run with DiagnosticGaussCycle = 2 and the Gauss array on the
    field snapshots every 2 cycles: gauss.csv rows for the samples begun at
    0, 1, 2 and 3 (the field snapshots at 2 and 4 begin samples at 1 and 3),
    and Gauss arrays at 2 and 4 but not at 0."""
    from tpic_b200.runner import main
    from vtkread import field_data, read
    deck = tmp_path / "gauss.inp"
    shipped = Path(__file__).resolve().parents[1] / "tpic_b200" / "decks" / "uniform3d_16.inp"
    # The shipped uniform deck, shrunk (the last assignment of a key wins).
    deck.write_text(shipped.read_text() + "\nncycles = 4\nLx = 6\nLy = 5\nLz = 4\nnxc = 12\nnyc = 10\nnzc = 8\n"
                    "npcelx = 2 2\nnpcely = 2 2\nnpcelz = 2 2\n"
                    "DiagnosticGaussCycle = 2\nFieldOutputCycle = 2\nFieldOutputTag = E+Gauss\n")
    assert main(["--run", str(deck), "--output", str(tmp_path), "--precision", "double",
                 "--mass-matrix", "moments-f64"]) == 0
    data = tmp_path / "data"
    rows = [line.split(",") for line in (data / "gauss.csv").read_text().splitlines() if line and line[0].isdigit()]
    assert [int(r[0]) for r in rows] == [0, 1, 2, 3]
    assert all(float(r[1]) == pytest.approx((int(r[0]) + 0.5) * 0.15) for r in rows)
    assert float(rows[0][3]) == 0.0 and all(float(r[3]) > 0.0 for r in rows[1:])
    names = sorted(p.name for p in data.iterdir())
    assert "Gauss_t000000.vti" not in names and "Gauss_t000002.vti" in names and "Gauss_t000004.vti" in names
    root, arrays, _ = read(data / "Gauss_t000004.vti")
    assert arrays["Gauss"].shape == (12 * 10 * 8,)
    assert field_data(root)["cycle"] == 4
    # rms of the array = the row of the sample that finished at cycle 4.
    assert math.sqrt(np.mean(arrays["Gauss"] ** 2)) == pytest.approx(float(rows[3][2]), rel=1e-12)
