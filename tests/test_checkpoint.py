"""Checkpoints and restart: the directory layout and the piece format on the
host (no GPU), and, on the GPU, a restarted run that continues the original
bit for bit (TPIC's checkpoint semantics, docs/user/output.md "Checkpoints
and restart": E at the nodes, B at the cells and every record; everything
else rebuilt)."""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import pytest

from tpic_b200 import _lib
from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec


def fake_piece(path, grid=(4, 3, 2), ns=1, count=5, precision=0, corrupt=False, truncate=False):
    """A piece of this library's format written from the header definition:
    magic, tpicb200_checkpoint_info, the arrays, FNV-1a 64 of the arrays."""
    info = _lib.CheckpointInfo()
    info.version, info.precision, info.cycle, info.ns = 1, precision, 7, ns
    info.grid = _lib.Grid(*grid, 2.0, 1.5, 1.0)
    info.dt, info.c = 0.1, 1.0
    for s in range(ns):
        info.qom[s], info.count[s] = -1.0, count
    nx, ny, nz = grid
    fb = 8 if precision == 0 else 4
    nodes, cells = (nx + 3) * (ny + 3) * (nz + 3), (nx + 2) * (ny + 2) * (nz + 2)
    payload_len = 3 * nodes * fb + 3 * cells * fb + ns * count * (3 * 8 + 3 * fb + 8 + 4)
    payload = bytes(np.random.default_rng(1).integers(0, 256, payload_len, dtype=np.uint8))
    h = 1469598103934665603
    for b in payload:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    if corrupt:
        payload = bytes([payload[0] ^ 1]) + payload[1:]
    data = b"TPICB200" + bytes(info) + payload + struct.pack("<Q", h)
    if truncate:
        data = data[:-9]
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_bytes(data)
    return info


def test_find_newest_complete_checkpoint(tmp_path):
    lib = _lib.load()
    buf = C.create_string_buffer(4096)
    assert lib.tpicb200_checkpoint_find(str(tmp_path).encode(), buf, len(buf)) == _lib.INVALID_ARGUMENT
    fake_piece(tmp_path / "checkpoint_t000004_n000001" / "checkpoint_t000004_r000000.tpcb")
    fake_piece(tmp_path / "checkpoint_t000010_n000001" / "checkpoint_t000010_r000000.tpcb")
    # Incomplete (only the hidden partial) and foreign names are not checkpoints.
    (tmp_path / "checkpoint_t000012_n000001").mkdir()
    (tmp_path / "checkpoint_t000012_n000001" / ".checkpoint_t000012_r000000.tpcb.partial").write_bytes(b"x")
    (tmp_path / "checkpoint_t000099_n000002").mkdir()
    (tmp_path / "abandoned_checkpoint_t000050_n000001").mkdir()
    assert lib.tpicb200_checkpoint_find(str(tmp_path).encode(), buf, len(buf)) == 0
    assert buf.value.decode().endswith("checkpoint_t000010_n000001/checkpoint_t000010_r000000.tpcb")


@pytest.mark.parametrize("precision", [0, 1])
def test_piece_header_and_completeness(tmp_path, precision):
    lib = _lib.load()
    path = tmp_path / "p.tpcb"
    want = fake_piece(path, precision=precision)
    info = _lib.CheckpointInfo()
    assert lib.tpicb200_checkpoint_info_read(str(path).encode(), C.byref(info)) == 0
    assert (info.cycle, info.ns, info.count[0], info.precision) == (7, 1, 5, precision)
    assert (info.grid.nx, info.grid.ny, info.grid.nz, info.grid.lx) == (4, 3, 2, 2.0)
    fake_piece(path, truncate=True, precision=precision)
    assert lib.tpicb200_checkpoint_info_read(str(path).encode(), C.byref(info)) == _lib.INVALID_DATA
    path.write_bytes(b"NOTAPIECE" * 20)
    assert lib.tpicb200_checkpoint_info_read(str(path).encode(), C.byref(info)) == _lib.INVALID_DATA
    assert want.version == 1


# --------------------------------------------------------------------------
# GPU: restart continues the run bit for bit.

def small_case(dt=0.15):
    g = GridSpec(8, 8, 4, 5.0, 5.0, 2.5)
    sp = [SpeciesSpec(qom=-64.0, rho=1.0, npcel=(2, 2, 2), vth=(0.045,) * 3),
          SpeciesSpec(qom=1.0, rho=1.0, npcel=(2, 2, 2), vth=(0.0056,) * 3)]
    return Case(g, sp, dt=dt, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.0, 0.0, 0.0195)), seed=4)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,mass_kind", [("double", "moments-f64"), ("mixed", "bf16x3")])
def test_restart_continues_bit_for_bit(tmp_path, precision, mass_kind):
    from tpic_b200.simulation import Simulation
    case = small_case()
    kw = dict(precision=precision, mass_kind=mass_kind, keep_ids=True)
    a = Simulation(case, generate_on_device=True, **kw)
    a.run(2)
    path = a.checkpoint(tmp_path)
    assert path.endswith("checkpoint_t000002_n000001/checkpoint_t000002_r000000.tpcb")
    after = a.run(3)
    b = Simulation.restart(case, tmp_path, **kw)
    assert b.cycle == 2
    again = b.run(3)
    for x, y in zip(after, again):
        assert x.gmres_iterations == y.gmres_iterations
        assert x.total_energy == y.total_energy
        assert x.field_energy == y.field_energy
    for s in range(2):
        la, lb = a.live(s), b.live(s)
        for k in ("rx", "ry", "rz", "u", "v", "w", "q", "cell", "id"):
            assert bool((la[k] == lb[k]).all()), (s, k)
    assert bool((a.field("e") == b.field("e")).all())
    assert bool((a.field("b_cell") == b.field("b_cell")).all())
    # A second checkpoint replaces the first.
    b.checkpoint(tmp_path)
    assert sorted(p.name for p in tmp_path.iterdir()) == ["checkpoint_t000005_n000001"]


@pytest.mark.gpu
def test_restart_rejects_another_run_and_a_corrupt_piece(tmp_path):
    from tpic_b200.simulation import Simulation
    case = small_case()
    a = Simulation(case, precision="double", generate_on_device=True)
    a.run(1)
    path = a.checkpoint(tmp_path)
    with pytest.raises(_lib.TpicError) as err:
        Simulation.restart(small_case(dt=0.2), tmp_path, precision="double")
    assert err.value.status == _lib.INVALID_ARGUMENT
    with pytest.raises(_lib.TpicError) as err:
        Simulation.restart(case, tmp_path, precision="mixed")
    assert err.value.status == _lib.INVALID_ARGUMENT
    data = bytearray(open(path, "rb").read())
    data[len(data) // 2] ^= 0x10
    open(path, "wb").write(bytes(data))
    with pytest.raises(_lib.TpicError) as err:
        Simulation.restart(case, tmp_path, precision="double")
    assert err.value.status == _lib.INVALID_DATA
