"""Snapshot files (tpic_b200/csrc/output.cu, tpic_b200/output.py) on the host:
the VTK writers of the library, read back byte for byte, and the output
selection rules of TPIC's FieldOutputTag / MomentsOutputTag and write-method
keys (docs/user/output.md). No GPU: the writers are host functions."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tpic_b200 import _lib
from tpic_b200.output import OutputPlan, deck_keys, select_arrays
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
    with pytest.raises(ValueError):
        select_arrays("Gauss", "", 1)


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
