"""Extracts the startup-field golden rows of the cases built here.

TPIC's field-profile test (tests/initialization/field_profile_tests.cpp:115-345)
samples B and E of every case fixture at six points and keeps the hex
values in tests/data/golden/field_profiles.txt. This script copies the rows
of the fixtures whose cases the library builds (Uniform, Weibel, TwoStream
and the Harris family, with their parameter variants) into
field_profiles_cases.txt beside it. It reads the reference checkout, so it
runs where that checkout is present:

    python tests/golden/make_field_profiles.py /path/to/TPIC
"""
from __future__ import annotations

import pathlib
import sys

LABELS = (
    "Weibel", "TwoStream", "plasmoidChain", "DoubleGEM", "DoubleGEMnoPert", "GEM", "GEMnoPert",
    "Uniform", "GEMHarris", "Weibel growth=0.000000", "Weibel growth=-0.310000", "Weibel no seed",
    "TwoStream no seed", "TwoStream reordered species", "Harris no sheet field",
    "Double Harris positive amplitude", "Uniform smaller transverse axes", "GEMHarris mode only",
    "GEMHarris hump only", "GEMHarris hump kx zero", "GEMHarris GEM keys",
)


def main(root: str) -> None:
    source = pathlib.Path(root) / "tests" / "data" / "golden" / "field_profiles.txt"
    rows = [line for line in source.read_text().splitlines() if line.split("\t")[0] in LABELS]
    found = {line.split("\t")[0] for line in rows}
    missing = set(LABELS) - found
    if missing:
        raise SystemExit(f"labels absent from {source}: {sorted(missing)}")
    out = pathlib.Path(__file__).with_name("field_profiles_cases.txt")
    out.write_text("\n".join(rows) + "\n")
    print(f"{len(rows)} rows -> {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_field_profiles.py <TPIC source tree>")
    main(sys.argv[1])
