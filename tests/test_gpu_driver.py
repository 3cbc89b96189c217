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
# for bit.


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
    args = ["--run", str(C1), "--mass-matrix", form, "--precision", precision, "--cycles", "4"]
    driver(*args, "--output", str(a), cwd=tmp_path)
    done = subprocess.run([sys.executable, "-m", "tpic_b200", *args, "--output", str(b)], capture_output=True,
                          text=True, timeout=600, cwd=ROOT)
    assert done.returncode == 0, done.stdout + done.stderr
    x, y = rows(a / "diagnostics.csv"), rows(b / "diagnostics.csv")
    assert x.shape == y.shape == (5, 11 + 2 * 5)
    assert np.array_equal(x, y)


def test_driver_restart_continues_the_run(tmp_path):
    B.build()
    straight, restarted = tmp_path / "straight", tmp_path / "restarted"
    base = ["--run", str(C1), "--mass-matrix", "matrix-core"]
    driver(*base, "--cycles", "6", "--output", str(straight), cwd=tmp_path)
    driver(*base, "--cycles", "4", "--restart-cycle", "2", "--output", str(restarted), cwd=tmp_path)
    driver(*base, "--cycles", "6", "--restart", "--output", str(restarted), cwd=tmp_path)
    text = (restarted / "diagnostics.csv").read_text()
    assert "# restart at cycle 4" in text
    a, b = rows(straight / "diagnostics.csv"), rows(restarted / "diagnostics.csv")
    assert a.shape == b.shape == (7, 21)
    other = np.arange(7) != 4
    assert np.array_equal(a[other], b[other])
    assert np.allclose(a[4], b[4], rtol=1e-12, atol=1e-300)
