"""The C++ host driver on the GPU: a shrunk C1 deck run by tpicb200_run and
by `python -m tpic_b200 --run` gives the same diagnostics.csv (both load the
records on the device from the same seed and run the same cycles through the
C ABI), and a driver run restarted from its checkpoint continues the
straight run (bit for bit after the restart)."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from tpic_b200 import build as B

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
C1 = ROOT / "tpic_b200" / "decks" / "uniform3d_16.inp"
# The row at a restart's checkpoint cycle comes from tpicb200_energy over the
# restored records (its own summation order); the movers' scalars give the
# straight run's row, so that row agrees to rounding and every other row bit
# for bit. Rounding there is relative to the size of the summed terms: the
# energies and charges (sums of terms of one sign) to 1e-12 of their value;
# the energy change (total minus the first total) to 1e-12 of the total; the
# momenta (sums of terms of both signs over 2^17 records, whose net is about
# sqrt(n) times smaller than the sum of magnitudes) to 1e-12 of the
# largest momentum entry times sqrt(n).


def rows(path: Path) -> np.ndarray:
    data = [line.split(",") for line in path.read_text().splitlines() if line and line[0].isdigit()]
    return np.array([[float(v) for i, v in enumerate(r) if i != 2] for r in data])


def driver(*argv, cwd):
    done = subprocess.run([str(B.DRIVER), *argv], capture_output=True, text=True, timeout=600, cwd=cwd)
    assert done.returncode == 0, done.stdout + done.stderr
    return done


@pytest.mark.parametrize("form,precision", [("matrix-core", "mixed"), ("moments-f64", "double")])
def test_driver_matches_the_python_runner(tmp_path, form, precision):
    B.build()
    a, b = tmp_path / "cpp", tmp_path / "py"
    args = ["--run", str(C1), "--mass-matrix", form, "--precision", precision, "--cycles", "4",
            "--diagnostics-cycle", "1"]
    driver(*args, "--output", str(a), cwd=tmp_path)
    done = subprocess.run([sys.executable, "-m", "tpic_b200", *args, "--output", str(b)], capture_output=True,
                          text=True, timeout=600, cwd=ROOT)
    assert done.returncode == 0, done.stdout + done.stderr
    x, y = rows(a / "data" / "diagnostics.csv"), rows(b / "data" / "diagnostics.csv")
    assert (a / "data" / "diagnostics.csv").read_text().splitlines()[:2] == \
        (b / "data" / "diagnostics.csv").read_text().splitlines()[:2]
    assert x.shape == y.shape == (5, 11 + 2 * 5)
    assert np.array_equal(x, y)


def test_driver_restart_continues_the_run(tmp_path):
    B.build()
    straight, restarted = tmp_path / "straight", tmp_path / "restarted"
    base = ["--run", str(C1), "--mass-matrix", "matrix-core", "--diagnostics-cycle", "1"]
    driver(*base, "--cycles", "6", "--output", str(straight), cwd=tmp_path)
    driver(*base, "--cycles", "4", "--restart-cycle", "2", "--output", str(restarted), cwd=tmp_path)
    driver(*base, "--cycles", "6", "--restart", "--output", str(restarted), cwd=tmp_path)
    text = (restarted / "data" / "diagnostics.csv").read_text()
    assert "# restart at cycle 4: precision_profile = mixed/mixed" in text
    a, b = rows(straight / "data" / "diagnostics.csv"), rows(restarted / "data" / "diagnostics.csv")
    assert a.shape == b.shape == (7, 21)
    other = np.arange(7) != 4
    assert np.array_equal(a[other], b[other])
    assert_rounding(a[4], b[4], ns=2, records=2 * 16 ** 3 * 27)


def assert_rounding(x, y, ns, records):
    """Row x equals row y to rounding (columns of diagnostics.csv without
    `state`: cycle, time, E, B, kinetic, total, change, charge, momentum x/y/z,
    then kinetic, charge, momentum x/y/z per species)."""
    momentum = [8, 9, 10] + [11 + 5 * s + k for s in range(ns) for k in (2, 3, 4)]
    scale = np.abs(x).copy()
    scale[6] = abs(x[5])
    scale[momentum] = np.abs(x[momentum]).max() * np.sqrt(records)
    bad = np.abs(x - y) > 1e-12 * scale
    assert not bad.any(), (np.nonzero(bad)[0], x[bad], y[bad])


def test_driver_snapshots_match_the_python_runner(tmp_path):
    """Field snapshots every cycle and particle snapshots every 2 cycles of the
    shrunk C1 deck, written by the driver and by the runner: the same files;
    E, B and the records (matched by species and id) bit for bit, the
    moments (device atomics, any summation order) to rounding."""
    from vtkread import field_data, read
    B.build()
    a, b = tmp_path / "cpp", tmp_path / "py"
    args = ["--run", str(C1), "--mass-matrix", "matrix-core", "--cycles", "3", "--field-output-cycle", "1",
            "--particles-output-cycle", "2"]
    driver(*args, "--output", str(a), cwd=tmp_path)
    done = subprocess.run([sys.executable, "-m", "tpic_b200", *args, "--output", str(b)], capture_output=True,
                          text=True, timeout=600, cwd=ROOT)
    assert done.returncode == 0, done.stdout + done.stderr
    names = sorted(p.name for p in (a / "data").iterdir())
    assert names == sorted(p.name for p in (b / "data").iterdir())
    for cycle in (0, 1, 2, 3):
        assert f"rho_1_t{cycle:06d}.vti" in names
    assert "particles_t000002.pvtp" in names and "particles_t000003_r000000.vtp" in names
    assert "particles_t000001.pvtp" not in names
    for name in names:
        if name.endswith(".csv"):
            continue
        if name.endswith(".pvtp"):
            assert (a / "data" / name).read_bytes() == (b / "data" / name).read_bytes()
            continue
        ra, xa, _ = read(a / "data" / name)
        rb, xb, _ = read(b / "data" / name)
        assert field_data(ra) == field_data(rb), name
        if name.endswith(".vtp"):
            order = [np.lexsort((x["id"], x["species"])) for x in (xa, xb)]
            for key in ("position", "velocity", "charge", "id", "species"):
                assert np.array_equal(xa[key][order[0]], xb[key][order[1]]), (name, key)
            assert np.array_equal(xa["connectivity"], xb["connectivity"])
            continue
        (key,) = xa.keys()
        if key in ("E", "B"):
            assert np.array_equal(xa[key], xb[key]), name
        else:
            scale = max(np.abs(xb[key]).max(), 1e-300)
            assert np.abs(xa[key] - xb[key]).max() <= 1e-12 * scale, name


def test_driver_gauss_rows_match_the_python_runner(tmp_path):
    """A shrunk C1 deck with Gauss-law samples every cycle and the Gauss array
    on the field snapshots, run by the driver and by the runner: the same
    gauss.csv cycles and times, the root mean squares and the Gauss arrays
    to rounding (the charge is summed with FP64 atomics)."""
    from vtkread import read
    B.build()
    deck = tmp_path / "gauss.inp"
    deck.write_text(C1.read_text() + "\nDiagnosticGaussCycle = 1\nFieldOutputCycle = 2\nFieldOutputTag = E+Gauss\n")
    a, b = tmp_path / "cpp", tmp_path / "py"
    args = ["--run", str(deck), "--mass-matrix", "matrix-core", "--cycles", "3"]
    driver(*args, "--output", str(a), cwd=tmp_path)
    done = subprocess.run([sys.executable, "-m", "tpic_b200", *args, "--output", str(b)], capture_output=True,
                          text=True, timeout=600, cwd=ROOT)
    assert done.returncode == 0, done.stdout + done.stderr

    def gauss_rows(path):
        lines = (path / "data" / "gauss.csv").read_text().splitlines()
        return lines[:2], np.array([[float(v) for v in line.split(",")] for line in lines if line and line[0].isdigit()])

    head_a, x = gauss_rows(a)
    head_b, y = gauss_rows(b)
    assert head_a == head_b
    assert x.shape == y.shape == (3, 6)
    assert np.array_equal(x[:, :2], y[:, :2])
    assert np.allclose(x[:, 2:], y[:, 2:], rtol=1e-10, atol=0)
    for cycle in (2, 3):
        ga = read(a / "data" / f"Gauss_t{cycle:06d}.vti")[1]["Gauss"]
        gb = read(b / "data" / f"Gauss_t{cycle:06d}.vti")[1]["Gauss"]
        assert np.abs(ga - gb).max() <= 1e-12 * np.abs(gb).max()
    assert not (a / "data" / "Gauss_t000000.vti").exists()


def test_initialize_writes_nothing_and_fresh_runs_refuse_existing_files(tmp_path):
    """--initialize completes the startup and writes no output; a fresh --run
    refuses an existing diagnostics.csv unless --overwrite-output, and a
    restart replaces its outputs (TPIC's --overwrite-output rule)."""
    B.build()
    out = tmp_path / "o"
    done = driver("--initialize", str(C1), "--output", str(out), cwd=tmp_path)
    assert "initialized" in done.stdout and not out.exists()
    base = ["--run", str(C1), "--cycles", "1", "--diagnostics-cycle", "1", "--output", str(out)]
    driver(*base, cwd=tmp_path)
    again = subprocess.run([str(B.DRIVER), *base], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert again.returncode == 1 and "--overwrite-output" in again.stderr
    driver(*base, "--overwrite-output", cwd=tmp_path)
    rows = [line for line in (out / "data" / "diagnostics.csv").read_text().splitlines() if line[:1].isdigit()]
    assert [r.split(",")[0] for r in rows] == ["0", "1"]
