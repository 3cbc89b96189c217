"""The z-slab decomposition (tpic_b200.slab) against the single-rank cycle,
on the host: ranks run as gloo processes, each on its slab with the
oracle's stage operators (tests/slab_cycle.py), exchanging the moment fold,
the node and cell halos, the GMRES dot sums and the migrating records.

- World sizes 1, 2 and 3 (slabs of 4+4 and 3+3+2 cell planes): three cycles
  of a two-species plasma give the single-rank energies (field energies,
  kinetic energies, charge, momentum) within 1e-12 relative, the same GMRES
  iteration counts, and the same records: every id once, keys equal, and
  positions and velocities within 1e-12 (the dot sums run in another order,
  so the fields differ in the last bits).
- The exchanges alone: halos and fold of a random field equal the periodic
  single-rank ghost fill and fold; migration keeps every record once.
"""
from __future__ import annotations

import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests"))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def make_case():
    from fieldutil import periodic_cell_field, periodic_node_field
    from tpic_b200.plasma import GridSpec, SpeciesSpec, generate_species
    g = GridSpec(6, 5, 8, 3.0, 2.5, 4.0)
    rng = np.random.default_rng(12)
    e0 = periodic_node_field(g, 0.01 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    b0 = periodic_cell_field(g, 0.0195 + 0.005 * rng.normal(size=(3, g.nz, g.ny, g.nx)))
    specs = [SpeciesSpec(qom=-16.0, npcel=(2, 2, 2), vth=(0.15,) * 3),
             SpeciesSpec(qom=1.0, npcel=(2, 2, 2), vth=(0.03,) * 3)]
    species = [(sp.qom, generate_species(g, sp, s, seed=4)) for s, sp in enumerate(specs)]
    return g, species, e0, b0


DT, THETA, C, TOL, CYCLES = 0.3, 0.5, 1.0, 1e-12, 3


def run_single():
    import oracle as O
    g, species, e0, b0 = make_case()
    oc = O.OracleCycle(g, [(q, {k: v.copy() for k, v in d.items()}) for q, d in species], DT, THETA, C, TOL, 0,
                       max_iterations=300, e_node=e0, b_cell=b0)
    oc.prepare()
    energies = [oc.cycle() for _ in range(CYCLES)]
    return oc, energies


def slab_rank(rank, world, port, queue):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from slab_cycle import SlabCycle
    from tpic_b200.slab import SlabExchange, SlabPlan
    if world > 1:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g, species, e0, b0 = make_case()
        plan = SlabPlan.make(g.nz, world, rank)
        sc = SlabCycle(g, species, DT, THETA, C, TOL, e0, b0, SlabExchange(plan), max_iterations=300)
        sc.prepare()
        energies = [sc.cycle() for _ in range(CYCLES)]
        queue.put((rank, energies, sc.iterations, sc.species, plan.z0, plan.nz, sc.e, sc.b))
    except Exception:
        import traceback
        queue.put((rank, "error", traceback.format_exc()))
        raise
    finally:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()


def run_slabs(world):
    import torch.multiprocessing as mp
    if world == 1:
        import queue as q
        out = q.Queue()
        slab_rank(0, 1, 0, out)
        return [out.get()]
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=slab_rank, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((queue.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for r in results:
        assert r[1] != "error", r[2]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return results


@pytest.fixture(scope="module")
def single():
    return run_single()


@pytest.mark.parametrize("world", [1, 2, 3])
def test_slab_cycle_matches_single_rank(single, world):
    oc, want = single
    results = run_slabs(world)
    g = oc.grid
    for r in results:
        got = r[1]
        for a, b in zip(got, want):
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15 * np.abs(b).max())
        assert r[2] == [res.iterations for res in oc.gmres[1:]] or r[2] == [res.iterations for res in oc.gmres]
    # Records: every id once, in the slab of its cell, equal to the single-rank record.
    ex, ey = g.nx + 4, g.ny + 4
    for s, (qom, d) in enumerate(oc.species):
        order = np.argsort(d["id"])
        parts = []
        for r in results:
            loc = dict(r[3][s][1])
            z0 = r[4]
            k = loc["cell"].astype(np.int64) // (ex * ey) - 2
            assert np.all((k >= 0) & (k < r[5]))
            loc["cell"] = (loc["cell"].astype(np.int64) + ex * ey * z0).astype(np.int32)
            parts.append(loc)
        merged = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
        mo = np.argsort(merged["id"])
        np.testing.assert_array_equal(merged["id"][mo], d["id"][order])
        np.testing.assert_array_equal(merged["cell"][mo], d["cell"][order])
        for k in ("rx", "ry", "rz", "u", "v", "w", "q"):
            np.testing.assert_allclose(merged[k][mo], d[k][order], rtol=1e-12, atol=1e-14)
    # Fields at each slab's owned planes.
    E = oc.e.reshape(3, g.nz + 3, g.ny + 3, g.nx + 3)
    B = oc.b.reshape(3, g.nz + 2, g.ny + 2, g.nx + 2)
    for r in results:
        z0, nz = r[4], r[5]
        np.testing.assert_allclose(r[6][:, 1:nz + 1], E[:, z0 + 1:z0 + nz + 1], rtol=0, atol=1e-13 * np.abs(E).max())
        np.testing.assert_allclose(r[7][:, 1:nz + 1], B[:, z0 + 1:z0 + nz + 1], rtol=0, atol=1e-13 * np.abs(B).max())


def exchange_rank(rank, world, port, queue):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from tpic_b200.slab import SlabExchange, SlabPlan
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nzg, ny, nx = 7, 3, 4
        plan = SlabPlan.make(nzg, world, rank)
        x = SlabExchange(plan)
        rng = np.random.default_rng(5)
        glob = rng.normal(size=(2, nzg + 3, ny + 3, nx + 3))
        # Halo: owned planes from the global field, ghosts and the shared plane from the neighbours.
        f = np.zeros((2, plan.nz + 3, ny + 3, nx + 3))
        f[:, 1:plan.nz + 1] = glob[:, plan.z0 + 1:plan.z0 + plan.nz + 1]
        x.node_halo(torch.from_numpy(f))
        want = glob[:, [(plan.z0 + k) % nzg + 1 for k in range(-1, plan.nz + 2)]]
        halo_ok = np.array_equal(f, want)
        # Fold: every rank deposits ones into all of its planes 0..nz; a node
        # plane shared by two slabs then holds 2.
        m = np.zeros_like(f)
        m[:, 1:plan.nz + 2] = 1.0
        x.fold_nodes(torch.from_numpy(m))
        fold_ok = np.all(m[:, 1] == 2.0) and np.all(m[:, 2:plan.nz + 1] == 1.0) and np.all(m[:, plan.nz + 1] == 2.0)
        # Migration: records of slab z0 moved by -1, 0, +1 planes.
        n = 9
        ids = torch.arange(rank * 100, rank * 100 + n, dtype=torch.int64)
        k = torch.tensor([(plan.z0 + d) % nzg for d in (-1, 0, 1)] * 3, dtype=torch.int64)
        k[1::3] = plan.z0 + torch.arange(3) % plan.nz
        out = x.migrate({"id": ids, "k": k}, k)
        mig_ok = bool(plan.owns_cell(out["k"]).all())
        total = torch.tensor([out["id"].numel()], dtype=torch.int64)
        dist.all_reduce(total)
        queue.put((rank, halo_ok, fold_ok, mig_ok, int(total.item()), sorted(out["id"].tolist())))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_exchanges(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=exchange_rank, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((queue.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in results:
        assert r[1] and r[2] and r[3], r
        assert r[4] == 9 * world
    ids = sorted(i for r in results for i in r[5])
    assert ids == sorted(r * 100 + i for r in range(world) for i in range(9))


def test_slab_plan():
    from tpic_b200.slab import SlabPlan
    plans = [SlabPlan.make(8, 3, r) for r in range(3)]
    assert [(p.z0, p.nz) for p in plans] == [(0, 3), (3, 3), (6, 2)]
    assert [(p.lower, p.upper) for p in plans] == [(2, 1), (0, 2), (1, 0)]
    assert [p.owned_node_planes for p in plans] == [3, 3, 3]
    with pytest.raises(ValueError):
        SlabPlan.make(2, 3, 0)
