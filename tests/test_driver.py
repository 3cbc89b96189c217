"""The C++ host driver tpicb200_run (tpic_b200/host/tpicb200_run.cpp), on the
host: it builds against include/tpicb200.h and the library, parses every
shipped deck (--dry-run needs no device), and rejects bad command lines."""
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
    done = subprocess.run([driver, "--run", str(deck), "--dry-run"], capture_output=True, text=True, timeout=60)
    assert done.returncode == 0, done.stderr
    assert "cells" in done.stdout and "records" in done.stdout


def test_bad_command_lines(driver, tmp_path):
    deck = str(DECKS[0])
    for argv in ([], ["--run"], ["--run", deck, "--mass-matrix", "nope", "--dry-run"],
                 ["--run", deck, "--precision", "half"], ["--run", str(tmp_path / "absent.inp")], ["--bogus"]):
        done = subprocess.run([driver, *argv], capture_output=True, text=True, timeout=60)
        assert done.returncode == 2, (argv, done.stdout, done.stderr)
        assert "usage" in done.stderr
    bad = tmp_path / "bad.inp"
    bad.write_text("Case = Whistler\n")
    done = subprocess.run([driver, "--run", str(bad), "--dry-run"], capture_output=True, text=True, timeout=60)
    assert done.returncode == 1 and "deck" in done.stderr
