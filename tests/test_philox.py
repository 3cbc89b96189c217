"""The synthetic-plasma generator's Philox-4x32-10 against the published
known-answer vectors of Salmon et al., "Parallel random numbers: as easy as
1, 2, 3" (SC'11; the Random123 distribution's kat_vectors), and the
generator's documented layout (CPU, no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from tpic_b200.plasma import GridSpec, SpeciesSpec, generate_species, philox4x32

KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("counter,key,want", KAT)
def test_philox_known_answers(counter, key, want):
    out = philox4x32(*[np.array([c], np.int64) for c in counter], *key)
    assert tuple(int(o[0]) for o in out) == want


def test_philox_torch_matches_numpy():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    c = [rng.integers(0, 2**32, 64, dtype=np.int64) for _ in range(4)]
    a = philox4x32(*c, 0x12345678, 0x9ABCDEF0)
    b = philox4x32(*[torch.from_numpy(x) for x in c], 0x12345678, 0x9ABCDEF0, xp=torch)
    for x, y in zip(a, b):
        assert np.array_equal(x, y.numpy())


def test_species_layout_and_charge():
    g = GridSpec(3, 2, 2, 3.0, 2.0, 2.0)
    sp = SpeciesSpec(qom=-4.0, rho=2.0, npcel=(2, 1, 2), vth=(0.1, 0.2, 0.3))
    d = generate_species(g, sp, 1, seed=7)
    n = g.cells * sp.ppc
    assert len(d["cell"]) == n
    # Dense load order: cell = n // ppc, x fastest; fractions stay in [0, 1).
    cell = np.arange(n) // sp.ppc
    keys = g.encode(cell % g.nx, (cell // g.nx) % g.ny, cell // (g.nx * g.ny))
    carried = d["cell"] != keys
    assert carried.sum() <= 2  # a fraction that rounds to one carries into the next cell
    for k in ("rx", "ry", "rz"):
        assert ((d[k] >= 0) & (d[k] < 1)).all()
    # q = sign(qom) V / ppc * rho / (4 pi)
    volume = (g.lx / g.nx) * (g.ly / g.ny) * (g.lz / g.nz)
    assert np.allclose(d["q"], -volume / sp.ppc * 2.0 / (4 * np.pi))
    assert np.array_equal(generate_species(g, sp, 1, seed=7)["u"], d["u"])  # deterministic
    assert not np.array_equal(generate_species(g, sp, 1, seed=8)["u"], d["u"])
