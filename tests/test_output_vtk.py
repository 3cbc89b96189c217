"""Snapshot files (tpic_b200/csrc/output.cu, tpic_b200/output.py) on the host:
the VTK writers of the library, read back byte for byte, and the output
selection rules of TPIC's FieldOutputTag / MomentsOutputTag and write-method
keys (docs/user/output.md). No GPU: the writers are host functions."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tpic_b200 import _lib
from tpic_b200.output import GaussSample, GaussWriter, OutputPlan, csv_number, deck_keys, select_arrays
from vtkread import field_data, read


def test_field_file_round_trip(tmp_path):
    lib = _lib.load()
    grid = _lib.Grid(4, 3, 2, 2.0, 1.5, 0.5)
    rng = np.random.default_rng(1)
    values = rng.normal(size=(3, 4, 5, 3))  # (nz+1, ny+1, nx+1, components)
    path = tmp_path / "E_t000007.vti"
    _lib.check(lib.tpicb200_vtk_write_field(str(path).encode(), b"E", 3, C.byref(grid),
                                            np.ascontiguousarray(values).ctypes.data, 7, 7 * 0.125, 0,
                                            b"double/double", b"storage: E=float64", 1))
    root, arrays, head = read(path)
    assert root.get("type") == "ImageData" and root.get("header_type") == "UInt64"
    img = root.find("ImageData")
    assert img.get("WholeExtent") == "0 4 0 3 0 2"
    assert [float(x) for x in img.get("Spacing").split()] == [0.5, 0.5, 0.25]
    fd = field_data(root)
    assert fd == {"TimeValue": 0.875, "cycle": 7, "final_state": 0, "state": "pre_solve",
                  "precision_profile": "double/double", "precision_roles": "storage: E=float64"}
    assert np.array_equal(arrays["E"], values.reshape(-1, 3))
    # Existing files are refused unless overwriting.
    assert lib.tpicb200_vtk_write_field(str(path).encode(), b"E", 3, C.byref(grid),
                                        np.ascontiguousarray(values).ctypes.data, 7, 0.0, 1, b"", b"", 0) \
        == _lib.BACKEND_FAILURE
    assert b"E_t000007.vti" in lib.tpicb200_last_error()


def test_particle_snapshot_round_trip(tmp_path):
    lib = _lib.load()
    rng = np.random.default_rng(2)
    counts = [5, 0, 3]
    keep, species = [], (_lib.VtkSpecies * 3)()
    for s, n in enumerate(counts):
        arrs = [rng.normal(size=3 * max(n, 1)), rng.normal(size=3 * max(n, 1)), rng.normal(size=max(n, 1)),
                rng.integers(0, 2 ** 63, size=max(n, 1)).astype(np.uint64)]
        keep.append(arrs)
        species[s] = _lib.VtkSpecies(n, *(a.ctypes.data for a in arrs), s)
    _lib.check(lib.tpicb200_vtk_write_particles(str(tmp_path).encode(), 12, 1.5, 1, b"mixed/mixed", b"r", 3,
                                                species, 1))
    root, arrays, _ = read(tmp_path / "particles_t000012_r000000.vtp")
    piece = root.find("PolyData/Piece")
    assert piece.get("NumberOfPoints") == "8" and piece.get("NumberOfVerts") == "8"
    assert field_data(root)["state"] == "final" and field_data(root)["cycle"] == 12
    want = {k: np.concatenate([a[i][:(3 if k in ("position", "velocity") else 1) * n]
                               for a, n in zip(keep, counts)])
            for i, k in enumerate(("position", "velocity", "charge", "id"))}
    assert np.array_equal(arrays["position"].reshape(-1), want["position"])
    assert np.array_equal(arrays["velocity"].reshape(-1), want["velocity"])
    assert np.array_equal(arrays["charge"], want["charge"])
    assert np.array_equal(arrays["id"], want["id"])
    assert arrays["species"].tolist() == [0] * 5 + [2] * 3
    assert arrays["connectivity"].tolist() == list(range(8))
    assert arrays["offsets"].tolist() == list(range(1, 9))
    manifest = (tmp_path / "particles_t000012.pvtp").read_text()
    assert '<Piece Source="particles_t000012_r000000.vtp"/>' in manifest
    assert 'type="PPolyData"' in manifest


def test_default_and_tagged_selection():
    fields, moments = select_arrays("", "", 2)
    assert fields == ["E", "B"]
    assert [m[0] for m in moments] == ["rho", "J", "rho_0", "rho_1", "J_0", "J_1"]
    fields, moments = select_arrays("B", "", 2)
    assert fields == ["B"] and moments == []
    _, moments = select_arrays("", "rho+rho0", 2)
    assert [m[0] for m in moments] == ["rho_0"]
    _, moments = select_arrays("E", "J_tot+PXX1+PZZ+rho5", 2)
    assert [m[0] for m in moments] == ["J", "PXX_1", "PZZ_0", "PZZ_1"]
    for bad in ("EB", "none", "rhoJ", "rho-1", "PXX_totally", "B+", "rho++J"):
        with pytest.raises(ValueError):
            select_arrays(bad if bad in ("EB", "none", "B+") else "", bad if bad not in ("EB", "none", "B+") else "",
                          2)
    fields, moments = select_arrays("Gauss+E", "", 1)
    assert fields == ["Gauss", "E"] and moments == []


def test_plan_from_deck(tmp_path):
    text = "ncycles = 10\nFieldOutputCycle = 5\nParticlesOutputCycle = 0 # off\nSaveDirName = out\n"
    assert deck_keys(text)["ParticlesOutputCycle"] == "0"
    plan = OutputPlan.from_deck(text, tmp_path)
    assert plan.save_dir == tmp_path / "out" and plan.field_cycle == 5 and plan.particles_cycle == 0
    assert plan.due(5, False) == (True, False) and plan.due(7, True) == (True, False)
    plan = OutputPlan.from_deck("WriteMethod = hdf5\nFieldOutputCycle = 0\n", tmp_path)
    assert plan.field_cycle == 0
    with pytest.raises(ValueError):
        OutputPlan.from_deck("WriteMethod = hdf5\n", tmp_path)
    with pytest.raises(ValueError):
        OutputPlan.from_deck("FieldWriteMethod = csv\n", tmp_path)
    plan = OutputPlan.from_deck("", tmp_path, field_cycle=2, particles_cycle=3)
    assert (plan.field_cycle, plan.particles_cycle, plan.save_dir) == (2, 3, tmp_path / "data")


def test_cell_file_round_trip(tmp_path):
    """The Gauss array: Float64 CellData over the node extent, nx*ny*nz values."""
    lib = _lib.load()
    grid = _lib.Grid(4, 3, 2, 2.0, 1.5, 0.5)
    values = np.random.default_rng(5).normal(size=(2, 3, 4))
    path = tmp_path / "Gauss_t000004.vti"
    _lib.check(lib.tpicb200_vtk_write_cells(str(path).encode(), b"Gauss", C.byref(grid),
                                            np.ascontiguousarray(values).ctypes.data, 4, 0.5, 0, b"mixed/mixed",
                                            b"roles", 1))
    root, arrays, _ = read(path)
    piece = root.find("ImageData/Piece")
    assert piece.find("CellData/DataArray").get("Name") == "Gauss"
    assert len(piece.find("PointData")) == 0
    assert root.find("ImageData").get("WholeExtent") == "0 4 0 3 0 2"
    assert np.array_equal(arrays["Gauss"], values.ravel())
    assert field_data(root)["cycle"] == 4


def test_gauss_cadence():
    """PreparedOutput::should_sample_gauss (src/config/output.cpp): multiples of
    DiagnosticGaussCycle below the last cycle, and with the Gauss array one
    cycle before every field snapshot and before the final state."""
    plan = OutputPlan.from_deck("DiagnosticGaussCycle = 3\nFieldOutputCycle = 0\n", "/tmp")
    assert plan.gauss_enabled() and not plan.output_gauss
    assert [n for n in range(12) if plan.gauss_begins(n, 10)] == [0, 3, 6, 9]
    assert plan.next_gauss_begin(3, 10) == 6 and plan.next_gauss_begin(9, 10) is None
    plan = OutputPlan.from_deck("FieldOutputCycle = 4\nFieldOutputTag = E+Gauss\n", "/tmp")
    assert plan.output_gauss and plan.gauss_cycle == 0
    assert [n for n in range(12) if plan.gauss_begins(n, 10)] == [3, 7, 9]
    # Gauss has no effect without a field channel.
    plan = OutputPlan.from_deck("FieldOutputCycle = 0\nFieldOutputTag = Gauss\n", "/tmp")
    assert not plan.gauss_enabled()
    plan = OutputPlan.from_deck("DiagnosticGaussCycle = 1\n", "/tmp")
    assert [n for n in range(6) if plan.gauss_begins(n, 5)] == [0, 1, 2, 3, 4]


def test_gauss_csv(tmp_path):
    """gauss.csv: precision lines, TPIC's column definitions and header, rows of
    17-significant-digit numbers; a restart keeps the rows below its cycle."""
    path = tmp_path / "data" / "gauss.csv"
    w = GaussWriter(path, "mixed/mixed", "roles")
    for n in (0, 2, 4):
        w.write(GaussSample(n, (n + 0.5) * 0.15, (1e-3 * (n + 1), 0.0 if n == 0 else 1e-5 * n, 0.0, 0.1)))
    text = path.read_text()
    lines = text.splitlines()
    assert lines[0] == "# precision_profile = mixed/mixed" and lines[1] == "# precision_roles = roles"
    assert "cycle,time,residual_rms,drift_rms,wall_residual_rms,charge_rms" in lines
    rows = [line for line in lines if line and line[0].isdigit()]
    assert rows[1].split(",")[:2] == ["2", csv_number(2.5 * 0.15)]
    assert [float(v) for v in rows[2].split(",")[2:]] == [5e-3, 4e-5, 0.0, 0.1]
    assert csv_number(0.1) == "0.10000000000000001"
    GaussWriter(path, "mixed/mixed", "roles", restart_cycle=2)
    rows = [line for line in path.read_text().splitlines() if line and line[0].isdigit()]
    assert [r.split(",")[0] for r in rows] == ["0"]
    assert path.read_text().splitlines()[-1].startswith("# restart at cycle 2: precision_profile = mixed/mixed")
