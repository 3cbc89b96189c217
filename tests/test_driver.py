"""The C++ host driver tpicb200_run (tpic_b200/host/tpicb200_run.cpp), on the
host: it builds against include/tpicb200.h and the library, parses every
shipped deck (--check-input needs no device), and rejects bad command lines."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from tpic_b200 import build as B

DECKS = sorted((Path(B.HERE) / "decks").glob("*.inp"))


@pytest.fixture(scope="module")
def driver():
    B.build()
    return str(B.DRIVER)


@pytest.mark.parametrize("deck", DECKS, ids=[d.name for d in DECKS])
def test_dry_run_of_every_shipped_deck(driver, deck):
    done = subprocess.run([driver, "--check-input", str(deck)], capture_output=True, text=True, timeout=60)
    assert done.returncode == 0, done.stderr
    assert "cells" in done.stdout and "records" in done.stdout


def test_bad_command_lines(driver, tmp_path):
    deck = str(DECKS[0])
    # TPIC's exit code of an invalid command line or input is 1.
    for argv in ([], ["--run"], ["--check-input", deck, "--mass-matrix", "nope"], ["--run", "--check-input", deck],
                 ["--run", deck, deck], ["--run", deck, "--precision", "half"], ["--check-input", deck, "--restart"],
                 ["--run", deck, "--order", "random"], ["--run", str(tmp_path / "absent.inp")], ["--bogus"]):
        done = subprocess.run([driver, *argv], capture_output=True, text=True, timeout=60)
        assert done.returncode == 1, (argv, done.stdout, done.stderr)
        assert "usage" in done.stderr
    done = subprocess.run([driver, "--help"], capture_output=True, text=True, timeout=60)
    assert done.returncode == 0 and "--check-input|--initialize|--run" in done.stdout
    # --dry-run is --check-input; --order takes TPIC's three values; the form defaults to scalar.
    for argv in (["--dry-run", deck], ["--check-input", deck, "--order", "full"], [deck, "--check-input"]):
        done = subprocess.run([driver, *argv], capture_output=True, text=True, timeout=60)
        assert done.returncode == 0 and "mass form 0" in done.stdout, (argv, done.stderr)
    bad = tmp_path / "bad.inp"
    bad.write_text("Case = Whistler\n")
    done = subprocess.run([driver, "--check-input", str(bad)], capture_output=True, text=True, timeout=60)
    assert done.returncode == 1 and "deck" in done.stderr


TAGS = [("", ""), ("B", ""), ("", "rho+rho0"), ("E", "J_tot+PXX1+PZZ+rho5"), ("E+B", "PXY+PXY_tot+J1+J0"),
        ("", "rho007"), ("Gauss+B+E", "rho")]


@pytest.mark.parametrize("field_tag,moments_tag", TAGS)
def test_snapshot_selection_matches_the_runner(driver, tmp_path, field_tag, moments_tag):
    """The driver's reading of FieldOutputTag / MomentsOutputTag (printed by
    --dry-run) selects the runner's arrays in the runner's order."""
    from tpic_b200.output import select_arrays
    deck = tmp_path / "tagged.inp"
    keys = "FieldOutputCycle = 5\nParticlesOutputCycle = 3\nSaveDirName = snaps # comment\n"
    if field_tag:
        keys += f"FieldOutputTag = {field_tag}\n"
    if moments_tag:
        keys += f"MomentsOutputTag = {moments_tag}\n"
    deck.write_text(DECKS[0].read_text() + keys)
    done = subprocess.run([driver, "--check-input", str(deck), "--output", str(tmp_path)], capture_output=True,
                          text=True, timeout=60)
    assert done.returncode == 0, done.stderr
    line = [x for x in done.stdout.splitlines() if x.startswith("snapshots under")][0]
    ns = int(done.stdout.split(" species")[0].rsplit(" ", 1)[1])
    fields, moments = select_arrays(field_tag, moments_tag, ns)
    listed = line.split("(", 1)[1].split(")", 1)[0].split()
    assert listed == fields + [m[0] for m in moments]
    assert f"under {tmp_path}/snaps:" in line and "fields every 5 cycles" in line
    assert line.endswith("particles every 3 cycles")
    over = subprocess.run([driver, "--check-input", str(deck), "--field-output-cycle", "0",
                           "--particles-output-cycle", "7", "--save-dir", "x"], capture_output=True, text=True,
                          timeout=60)
    assert over.returncode == 0, over.stderr
    assert "under ./x:" in over.stdout and "fields every 0 cycles" in over.stdout
    assert "particles every 7 cycles" in over.stdout


@pytest.mark.parametrize("keys", ["FieldOutputTag = EB\n", "FieldOutputTag = B+\n", "FieldOutputTag = Gauss+Q\n",
                                  "MomentsOutputTag = rhoJ\n", "MomentsOutputTag = rho-1\n",
                                  "MomentsOutputTag = PXX_totally\n", "MomentsOutputTag = rho++J\n",
                                  "MomentsOutputTag = rho2147483648\n", "WriteMethod = hdf5\n",
                                  "FieldWriteMethod = csv\n"])
def test_bad_snapshot_keys(driver, tmp_path, keys):
    deck = tmp_path / "bad.inp"
    deck.write_text(DECKS[0].read_text() + keys)
    done = subprocess.run([driver, "--check-input", str(deck)], capture_output=True, text=True, timeout=60)
    assert done.returncode == 1, (keys, done.stdout, done.stderr)
    assert "Tag" in done.stderr or "Method" in done.stderr
    ok = tmp_path / "off.inp"
    ok.write_text(DECKS[0].read_text() + "WriteMethod = hdf5\nFieldOutputCycle = 0\n")
    done = subprocess.run([driver, "--check-input", str(ok)], capture_output=True, text=True, timeout=60)
    assert done.returncode == 0, done.stderr


def test_gauss_cadence_of_the_driver(driver, tmp_path):
    """--dry-run prints the Gauss-law cadence: DiagnosticGaussCycle (or
    --gauss-cycle) and, with the Gauss array on a field channel, the samples
    before each field snapshot."""
    deck = tmp_path / "g.inp"
    deck.write_text(DECKS[0].read_text() + "DiagnosticGaussCycle = 4\nFieldOutputCycle = 5\nFieldOutputTag = E+Gauss\n")
    done = subprocess.run([driver, "--check-input", str(deck)], capture_output=True, text=True, timeout=60)
    assert done.returncode == 0, done.stderr
    assert "Gauss-law samples every 4 cycles and before each field snapshot" in done.stdout
    done = subprocess.run([driver, "--check-input", str(deck), "--gauss-cycle", "0", "--field-output-cycle", "0"],
                          capture_output=True, text=True, timeout=60)
    assert "Gauss-law samples every 0 cycles\n" in done.stdout


def test_diagnostics_and_checkpoint_keys(driver, tmp_path):
    """DiagnosticsOutputCycle defaults to FieldOutputCycle, RestartOutputCycle to
    0 and RestartDirName to data; the options override the keys."""
    deck = tmp_path / "k.inp"
    deck.write_text(DECKS[0].read_text() + "FieldOutputCycle = 7\n")
    done = subprocess.run([driver, "--check-input", str(deck), "--output", "o"], capture_output=True, text=True,
                          timeout=60)
    assert "diagnostics.csv rows every 7 cycles, checkpoints every 0 cycles under o/data" in done.stdout
    deck.write_text(DECKS[0].read_text() + "DiagnosticsOutputCycle = 3\nRestartOutputCycle = 5\nRestartDirName = ck\n")
    done = subprocess.run([driver, "--check-input", str(deck), "--output", "o"], capture_output=True, text=True,
                          timeout=60)
    assert "diagnostics.csv rows every 3 cycles, checkpoints every 5 cycles under o/ck" in done.stdout
    done = subprocess.run([driver, "--check-input", str(deck), "--output", "o", "--diagnostics-cycle", "1",
                           "--restart-cycle", "2", "--restart-dir", "r"], capture_output=True, text=True, timeout=60)
    assert "diagnostics.csv rows every 1 cycles, checkpoints every 2 cycles under o/r" in done.stdout
