"""The C++ adapter shown in INTEGRATION.md compiles against include/tpicb200.h.

The test takes the adapter's code block from the document as written, puts
a stand-in header of the TPIC-side types in front of it
(tests/adapter/tpic_shapes.hpp: owners, slots, bins, executor, report,
lpfx::ErrorCode, with TPIC's member names) and compiles it with g++ -std=c++20.
It checks the adapter's calls against the real ABI: argument counts, pointer
types and the status mapping. Nothing is run."""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def adapter_block() -> str:
    text = (ROOT / "INTEGRATION.md").read_text()
    section = text[text.index("## The C++ adapter a TPIC maintainer would add"):]
    match = re.search(r"```cpp\n(.*?)```", section, re.S)
    assert match, "no C++ block in the adapter section"
    return match.group(1)


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is not available")
def test_adapter_compiles_against_the_header(tmp_path):
    source = tmp_path / "b200_backend.cpp"
    source.write_text('#include "tpic_shapes.hpp"\n' + adapter_block())
    done = subprocess.run(["g++", "-std=c++20", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                           f"-I{ROOT / 'include'}", f"-I{ROOT / 'tests' / 'adapter'}", str(source)],
                          capture_output=True, text=True, timeout=120)
    assert done.returncode == 0, done.stderr
