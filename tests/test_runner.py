"""The deck runner (`python -m tpic_b200`): diagnostics.csv rows and columns
as TPIC writes them (docs/user/output.md, "diagnostics.csv"), on the host; a
deck run with checkpoints and a restart that continues the file, on the GPU."""
from __future__ import annotations

from pathlib import Path

import pytest

from tpic_b200 import runner

DECKS = Path(__file__).resolve().parent.parent / "tpic_b200" / "decks"


def test_columns_and_rows():
    cols = runner.columns(2).split(",")
    assert cols[:12] == ["cycle", "time", "state", "electric_energy", "magnetic_energy", "kinetic_energy",
                         "total_energy", "total_energy_change", "charge", "momentum_x", "momentum_y", "momentum_z"]
    assert cols[12:17] == ["kinetic_energy_0", "charge_0", "momentum_x_0", "momentum_y_0", "momentum_z_0"]
    assert len(cols) == 22
    species = ((1.0, -2.0, 0.1, 0.2, 0.3), (3.0, 2.0, -0.1, 0.0, 0.5))
    line = runner.row(4, 0.25, False, (0.5, 0.25), species, 4.0).split(",")
    assert line[:3] == ["4", "1.0", "pre_solve"]
    assert [float(x) for x in line[3:12]] == [0.5, 0.25, 4.0, 4.75, 0.75, 0.0, 0.0, 0.2, 0.8]
    assert float(line[12]) == 1.0 and float(line[17]) == 3.0
    assert runner.row(5, 0.25, True, (0.5, 0.25), species, 4.0).split(",")[2] == "final"


def test_mass_matrix_names():
    assert runner.resolve_form("matrix-core", "mixed") == "bf16x3"
    assert runner.resolve_form("matrix-core", "double") == "moments-f64"
    assert runner.resolve_form("tf32", "mixed") == "tf32"
    args = runner.parse_args(["--run", "x.inp", "--mass-matrix", "scalar", "--restart"])
    assert args.mass_matrix == "scalar" and args.restart and args.precision == "mixed" and args.input == "x.inp"
    # TPIC's command line: one of three commands and one input, scalar by default, exit code 1 otherwise.
    assert runner.parse_args(["x.inp", "--run"]).mass_matrix == "scalar"
    for argv in (["x.inp"], ["--run", "--check-input", "x.inp"], ["--check-input", "x.inp", "--restart"],
                 ["--run", "x.inp", "--order", "random"]):
        with pytest.raises(SystemExit) as e:
            runner.parse_args(argv)
        assert e.value.code == 1


def test_check_input_writes_nothing(tmp_path, capsys):
    out = tmp_path / "o"
    assert runner.main(["--check-input", str(DECKS / "uniform3d_16.inp"), "--output", str(out)]) == 0
    assert "16x16x16 cells, 2 species, 3 cycles, mass form scalar" in capsys.readouterr().out
    assert not out.exists()


@pytest.mark.gpu
def test_deck_run_with_checkpoints_and_restart(tmp_path):
    deck = tmp_path / "run.inp"
    deck.write_text((DECKS / "harris2d_256x128.inp").read_text() +
                    "\nnxc = 16\nnyc = 16\nLx = 4.0\nLy = 4.0\nnpcelx = 2 2 2 2\nnpcely = 2 2 2 2\nncycles = 4\n")
    out = tmp_path / "out"
    assert runner.main(["--run", str(deck), "--output", str(out), "--restart-cycle", "2",
                        "--diagnostics-cycle", "1"]) == 0
    rows = [l.split(",") for l in (out / "data" / "diagnostics.csv").read_text().splitlines() if l[:1].isdigit()]
    assert [r[0] for r in rows] == ["0", "1", "2", "3", "4"]
    assert [r[2] for r in rows] == ["pre_solve"] * 4 + ["final"]
    assert float(rows[0][7]) == 0.0
    assert abs(float(rows[-1][7])) <= 1e-5 * float(rows[0][6])
    names = sorted(p.name for p in (out / "data").iterdir())
    assert [n for n in names if n.startswith("checkpoint")] == ["checkpoint_t000004_n000001"]
    assert "diagnostics.csv" in names
    # Field snapshots (FieldOutputCycle defaults to 100): the first and the final state.
    assert "E_t000000.vti" in names and "E_t000004.vti" in names and "B_t000004.vti" in names
    # Continue to cycle 6 from the checkpoint of cycle 4.
    assert runner.main(["--run", str(deck), "--output", str(out), "--restart", "--cycles", "6",
                        "--diagnostics-cycle", "1"]) == 0
    text = (out / "data" / "diagnostics.csv").read_text()
    assert "# restart at cycle 4" in text
    rows = [l.split(",") for l in text.splitlines() if l[:1].isdigit()]
    assert [r[0] for r in rows] == ["0", "1", "2", "3", "4", "5", "6"]
    assert rows[4][2] == "pre_solve" and rows[-1][2] == "final"
