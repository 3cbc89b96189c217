#!/usr/bin/env python
"""Benchmark of the single-GPU ECSIM particle cycle (particles*cycles/s).

Workload (default): the 3-D uniform thermal plasma at scale -- 128^3 cells,
box 20^3 d_i, electrons (q/m = -64) and ions (q/m = 1), 64 particles per cell
per species (268,435,456 particles), Maxwellian vth_e = 0.045c, vth_i =
0.0056c, B0 = (0, 0, 0.0195), FP64 positions / FP32 velocities (mixed
precision), dt = 0.15/omega_pi, theta = 0.5, GMRES rtol 1e-8 -- seeded
synthetic inputs from tpic_b200.plasma (no dataset is involved).

A step is one full ECSIM cycle (solve, move, field advance, stable sort,
current + mass deposition, fold, commit, energy diagnostics) through the C
ABI's tpicb200_cycle. Inputs stay resident in HBM (13 GB of particle
records per slot, far larger than the 126 MB L2).

The headline form (--mass-matrix, default the BF16x3 tensor-core assembly)
and the comparison form (--compare, default the plain FP32 CUDA-core
assembly) are each timed on the same workload; each runs --drift-cycles
cycles (default 100) from the same initial state for its relative energy
drift. The line reports both and their ratio ("plain_fp32_form").

  python bench.py [--gpus N --steps K --warmup W] [--mass-matrix scalar|scalar-f64|tf32|bf16x3]
  python bench.py --deck tpic_b200/decks/harris2d_256x128.inp ...   (a deck's workload)
  python bench.py --impl reference ...   (the CPU implementation of the path)

N > 1 runs N independent replicas (the path is timed on one GPU; the
replicas share nothing), launched by torchrun; rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particles*cycles/s on 1 B200, tensor-core vs plain FP32 assembly at equal energy error"
UNIT = "particles*cycles/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def workload(scale: int = 128, ppc_axis: int = 4):
    from tpic_b200.plasma import Case, FieldInit, GridSpec, SpeciesSpec
    box = 20.0 * scale / 128
    g = GridSpec(scale, scale, scale, box, box, box)
    npcel = (ppc_axis,) * 3
    species = [SpeciesSpec(qom=-64.0, rho=1.0, npcel=npcel, vth=(0.045,) * 3),
               SpeciesSpec(qom=1.0, rho=1.0, npcel=npcel, vth=(0.0056,) * 3)]
    return Case(g, species, dt=0.15, theta=0.5, gmres_tol=1e-8, fields=FieldInit(b0=(0.0, 0.0, 0.0195)))


def peaks():
    try:
        data = json.loads(PEAKS.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, enabled: bool = True):
        self.index = index
        self.enabled = enabled
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        if not self.enabled:
            return self
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.flush()
        rows = [r.split(", ") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        rows = [r for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


def cpu_oracle_rate(scale: int, ppc_axis: int, cycles: int, warmup: int, precision: int = 1) -> dict:
    """The oracle cycle (the CPU restatement of the path) on a bounded sample
    of the workload: `scale`^3 cells at the workload's cell size and loading."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from tpic_b200.plasma import generate_species
    case = workload(scale, ppc_axis)
    oc = O.OracleCycle(case.grid, O.case_species_arrays(case, precision, generate_species), case.dt, case.theta,
                       case.c, case.gmres_tol, precision, b0=case.fields.b0)
    oc.prepare()
    for _ in range(warmup):
        oc.cycle()
    n = sum(len(d["cell"]) for _, d in oc.species)
    t0 = time.perf_counter()
    for _ in range(cycles):
        oc.cycle()
    dt = time.perf_counter() - t0
    return {"particles": n, "cycles": cycles, "seconds": dt}


def _cpu_worker(args):
    scale, ppc_axis, cycles, warmup = args
    return cpu_oracle_rate(scale, ppc_axis, cycles, warmup)


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = args.cpu_workers or os.cpu_count() or 1
    scale = args.cpu_scale
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        results = pool.map(_cpu_worker, [(scale, 4, args.steps, args.warmup)] * cores)
    wall = time.perf_counter() - t0
    value = sum(r["particles"] * r["cycles"] for r in results) / max(r["seconds"] for r in results)
    sample = (f"{cores} independent replicas of a {scale}^3-cell slice of the workload "
              f"({results[0]['particles']} particles each, same cell size and loading), "
              f"{args.steps} timed oracle cycles after {args.warmup} warm-up cycles")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * max(r["seconds"] for r in results) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32 (host)",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "3-D uniform thermal plasma, 128^3 cells, 2 species x 64 ppc (bounded CPU sample)",
                       "sample_cells": scale ** 3, "precision": "mixed"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def run_adjoint(args) -> None:
    """Gradient of a deck's final-state objective by the adjoint (the deck's
    precision and mass form, checkpoints every --checkpoint-every cycles)
    against central differences of the FP64 forward run, over one or more
    horizons (--horizons, default the deck's ncycles): at h = 1e-4 of the
    parameter, and at the largest h = 1e-4 |p| 10^-k (k <= 6) whose one-sided
    differences agree within 1e-3 (no cell-crossing kink inside +-h), if any.
    Two-stream decks: d(W_E + W_B)/d(beam drift) and d/d(density-seed
    amplitude); anisotropy decks (Uniform with a bi-Maxwellian species):
    d(W_B)/d(T_perp/T_par) of species 0 about x. With --adjoint-fp64 the FP64
    adjoint (FP64 moment form) runs beside the deck's precision."""
    import torch
    from tpic_b200 import deck as D
    from tpic_b200.adjoint import AdjointRun, anisotropy_tangent, contract, two_stream_tangents
    from tpic_b200.simulation import Simulation
    if not args.deck:
        raise SystemExit("--adjoint needs --deck")
    text = Path(args.deck).read_text()
    parsed = D.parse(text)
    name = D.case_name(parsed)
    horizons = [int(h) for h in args.horizons.split(",")] if args.horizons else [parsed.ncycles]
    case = D.to_case(parsed)
    nparticles = sum(case.grid.cells * sp.ppc for sp in case.species)
    torch.cuda.set_device(0)
    if name == "TwoStream":
        we, wb, objective = 1.0, 1.0, "W_E + W_B"
    else:
        we, wb, objective = 0.0, 1.0, "W_B"

    def adjoint(ncycles: int, precision: str, mass_matrix: str):
        sim = Simulation(case, precision=precision, mass_kind=mass_matrix, keep_ids=True, generate_on_device=True,
                         gmres_max_iterations=args.gmres_max_iterations, mass_layout=args.mass_layout)
        sim.prepare()
        run = AdjointRun(sim, every=args.checkpoint_every)
        t0 = time.perf_counter()
        run.forward(ncycles)
        adj = run.backward(we, wb)
        torch.cuda.synchronize()
        total_s = time.perf_counter() - t0
        grads = {}
        if name == "TwoStream":
            tangents = two_stream_tangents(run, parsed)
            grads["drift"] = contract(sim, adj, tangents["drift"])
            grads["amplitude"] = contract(sim, adj, tangents["amplitude"])
        else:
            vpar, vperp = parsed.species[0].vth[0], parsed.species[0].vth[1]
            grads["anisotropy"] = contract(sim, adj, anisotropy_tangent(run, 0, 0, (vperp / vpar) ** 2))
        stats = run.stats
        sim.close()
        del sim, run, adj
        torch.cuda.empty_cache()
        return grads, stats, total_s

    def param_value(param: str) -> float:
        if param == "drift":
            return parsed.species[0].drift[0]
        if param == "amplitude":
            return parsed.two_stream_amplitude
        return (parsed.species[0].vth[1] / parsed.species[0].vth[0]) ** 2

    def energy(param: str, value: float, ncycles: int) -> float:
        if param == "drift":
            extra = f"\nu0 = {value!r} {-value!r} 0.0\n"
        elif param == "amplitude":
            extra = f"\nTwoStreamSeedDensityAmplitude = {value!r}\n"
        else:
            v = parsed.species[0].vth[0] * math.sqrt(value)
            extra = f"\nvth = {v!r} {parsed.species[1].vth[1]!r}\nwth = {v!r} {parsed.species[1].vth[2]!r}\n"
        dk = D.parse(text + extra + "\nGMREStol = 1e-12\n")
        fd_sim = Simulation(D.to_case(dk), precision="double", mass_kind="moments-f64", generate_on_device=True,
                            gmres_max_iterations=max(args.gmres_max_iterations, 500))
        fd_sim.prepare()
        r = fd_sim.run(ncycles)[-1]
        fd_sim.close()
        return we * r.field_energy[0] + wb * r.field_energy[1]

    results = []
    for ncycles in horizons:
        grads, stats, total_s = adjoint(ncycles, args.precision, args.mass_matrix)
        entry = {"cycles": ncycles, "seconds": total_s, "forward_s": stats.forward_s,
                 "recompute_s": stats.recompute_s, "backward_s": stats.backward_s,
                 "backward_over_forward": (stats.recompute_s + stats.backward_s) / stats.forward_s,
                 "checkpoints": stats.checkpoints, "tapes": stats.tapes, "tape_bytes": stats.device_bytes,
                 "adjoint_gmres_iterations_mean": float(np.mean(stats.adjoint_iterations)), "gradients": {}}
        fp64 = adjoint(ncycles, "double", "moments-f64")[0] if args.adjoint_fp64 else None
        for param, grad in grads.items():
            p0 = param_value(param)
            l0 = energy(param, p0, ncycles)
            h = 1e-4 * abs(p0)
            lp, lm = energy(param, p0 + h, ncycles), energy(param, p0 - h, ncycles)
            fd4 = (lp - lm) / (2 * h)
            g = {"adjoint": grad, "fd_h1e-4": fd4, "rel_err_h1e-4": abs(grad - fd4) / abs(fd4),
                 "one_sided_h1e-4": [(l0 - lm) / h, (lp - l0) / h]}
            if fp64 is not None:
                g["adjoint_fp64"] = fp64[param]
                g["rel_diff_fp64_adjoint"] = abs(grad - fp64[param]) / abs(fp64[param])
            kink_free = None
            for _ in range(6):
                right, left = (lp - l0) / h, (l0 - lm) / h
                if abs(right - left) <= 1e-3 * max(abs(right), abs(left)):
                    fd = (lp - lm) / (2 * h)
                    kink_free = {"h_rel": h / abs(p0), "fd": fd, "rel_err": abs(grad - fd) / abs(fd)}
                    break
                h /= 10
                lp, lm = energy(param, p0 + h, ncycles), energy(param, p0 - h, ncycles)
            g["kink_free"] = kink_free
            entry["gradients"][param] = g
        results.append(entry)
        print(json.dumps({"horizon": entry}), flush=True)
    line = {"metric": "adjoint gradient of the final field energy: forward + recompute + backward",
            "value": results[-1]["seconds"], "unit": "s", "higher_is_better": False, "impl": "tpic_b200",
            "n_gpus": 1,
            "config": {"workload": f"deck {Path(args.deck).name}: {name}", "particles": nparticles,
                       "precision": args.precision, "mass_matrix": args.mass_matrix, "mass_layout": args.mass_layout,
                       "checkpoint_every": args.checkpoint_every, "objective": objective},
            "horizons": results}
    print(json.dumps(line), flush=True)


def max_over_ranks(seconds: float, dist, device) -> float:
    """The slowest rank's time (every rank takes part; a no-op on one rank)."""
    if dist is None:
        return seconds
    import torch
    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, particles: int, steps: int, seconds: float) -> float:
    """Whole-job particles*cycles/s of `world` replicas timed as the slowest."""
    return world * particles * steps / seconds


def run_gpu(args) -> None:
    import torch
    from tpic_b200 import _lib
    from tpic_b200.simulation import Simulation

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    if args.deck:
        from tpic_b200 import deck as D
        parsed = D.load(args.deck)
        case = D.to_case(parsed)
    else:
        case = workload(args.scale, 4)
    nparticles = sum(case.grid.cells * sp.ppc for sp in case.species)
    g = case.grid
    # Energy-conserving smoothing: passes,alpha,operator (0 Face7, 1 Binomial27).
    smoothing = tuple(case.smoothing)  # a deck's own keys, unless --smoothing is given
    if args.smoothing:
        n_, a_, o_ = args.smoothing.split(",")
        smoothing = (int(n_), float(a_), int(o_))
    if args.deck:
        ppcs = "/".join(str(sp.ppc) for sp in case.species)
        workload_name = (f"deck {Path(args.deck).name}: {D.case_name(parsed)}, {g.nx}x{g.ny}x{g.nz} cells, "
                         f"box {g.lx:g}x{g.ly:g}x{g.lz:g}, {len(case.species)} species x {ppcs} ppc")
    else:
        workload_name = (f"3-D uniform thermal plasma, {args.scale}^3 cells, box 20^3 d_i, "
                         f"2 species x 64 ppc, mass ratio 64")
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def bootstrap_errors(sim, reference):
        """Max and RMS relative error of the bootstrap deposition's mass
        entries and J-hat against the FP64 moment form's on the same state."""
        if reference is None:
            return {}
        out = {}
        for name in ("mass", "j"):
            got = sim.field(name).double()
            want = reference[name]
            diff = got - want
            out[f"{name}_rel_err_max"] = float(diff.abs().max() / want.abs().max())
            out[f"{name}_rel_err_rms"] = float(diff.square().mean().sqrt() / want.square().mean().sqrt())
            del got, diff
        torch.cuda.synchronize()
        return out

    def timed_form(mass_kind, sample_clocks, precision=None, reference=None, keep=False):
        """Warm-up, the timed cycles, then more cycles up to --drift-cycles for
        the energy drift (the simulation stays open for the caller). With
        `reference` (bootstrap mass and J of the FP64 moment form) the
        bootstrap deposition's errors against it are measured; keep=True
        returns this form's own bootstrap mass and J (double) for that."""
        precision = precision or args.precision
        t_gen = time.perf_counter()
        sim = Simulation(case, precision=precision, mass_kind=mass_kind, device=local, generate_on_device=True,
                         gmres_max_iterations=args.gmres_max_iterations, smoothing=smoothing,
                         mass_layout=args.mass_layout)
        if precision == "double" and args.precision == "mixed":
            # The same state as the mixed forms: their FP32 velocities, widened.
            for s in range(len(case.species)):
                for k in ("u", "v", "w"):
                    t = sim.slots[s][sim.state.current[s]][k]
                    t.copy_(t.float().double())
        gen_s = time.perf_counter() - t_gen
        sim.prepare()
        errors = bootstrap_errors(sim, reference)
        own = {name: sim.field(name).double().clone() for name in ("mass", "j")} if keep else None
        w0 = sim.energy()
        total0 = w0[0] + w0[1] + sum(w0[2 + 5 * s] for s in range(len(case.species)))
        history = sim.run(args.warmup)
        launches0 = sim.lib.tpicb200_launch_count()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        with ClockSampler(local, enabled=sample_clocks) as clocks:
            start.record(stream)
            reports = sim.run(args.steps)
            stop.record(stream)
            barrier()
        launches = sim.lib.tpicb200_launch_count() - launches0
        seconds = max_over_ranks(start.elapsed_time(stop) / 1e3, dist, "cuda")
        history += reports
        if len(history) < args.drift_cycles:
            history += sim.run(args.drift_cycles - len(history))
        drift = max(abs(r.total_energy - total0) / abs(total0) for r in history)
        stage_names = ["solve", "move", "advance", "sort", "deposit", "fold_diagnostics"]
        result = {"value": replica_rate(world, nparticles, args.steps, seconds),
                  "ms_per_step": 1e3 * seconds / args.steps,
                  "energy_drift": {"cycles": len(history), "max_relative": drift},
                  "stages_ms": {name: float(np.mean([r.stage_ms[k] for r in reports]))
                                for k, name in enumerate(stage_names)},
                  "gmres_iterations": float(np.mean([r.gmres_iterations for r in reports])),
                  "gmres_host_waits": float(np.mean([r.gmres_host_waits for r in reports])),
                  "launches": int(launches), "generation_s": gen_s, **errors}
        if keep:
            return sim, result, clocks, own
        return sim, result, clocks

    def sweep_entry(form, precision, result):
        keys = ("value", "ms_per_step", "energy_drift", "gmres_iterations", "mass_rel_err_max", "mass_rel_err_rms",
                "j_rel_err_max", "j_rel_err_rms")
        return {"mass_matrix": form, "precision": precision, **{k: result[k] for k in keys if k in result}}

    # ---- the precision sweep's reference: the FP64 moment form ------------------
    sweep, reference = [], None
    if args.sweep and not args.deck:
        ref_sim, ref_result, _, reference = timed_form("moments-f64", False, precision="double", keep=True)
        ref_sim.close()
        del ref_sim
        sweep.append(sweep_entry("moments-f64", "double",
                                 {**ref_result, "mass_rel_err_max": 0.0, "j_rel_err_max": 0.0}))

    sim, headline, clocks = timed_form(args.mass_matrix, True, reference=reference)
    value = headline["value"]
    seconds = headline["ms_per_step"] * args.steps / 1e3
    lib = sim.lib

    # ---- dominant-kernel roofline: per-stage kernels timed alone -----------------
    kernels = stage_kernel_times(sim, args, stream)
    hbm, peak_kind = peaks()
    dominant = max(kernels, key=lambda k: kernels[k]["ms"])
    dk = kernels[dominant]
    achieved = dk["bytes"] / (dk["ms"] / 1e3) / 1e9
    traffic = None if args.deck else load_traffic(dominant, nparticles)
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes": dk["bytes"],
                "algorithmic_basis": dk["basis"],
                "record_bytes": dk.get("record_bytes"),
                "all_kernels": {k: {"ms": v["ms"], "GB/s": v["bytes"] / (v["ms"] / 1e3) / 1e9,
                                    "frac": v["bytes"] / (v["ms"] / 1e3) / 1e9 / hbm} for k, v in kernels.items()}}

    # ---- end to end through the public API with host buffers -----------------------
    e2e = end_to_end(sim, args, stream, barrier, nparticles, world, dist)
    sim.close()
    del sim

    # ---- the plain FP32 CUDA-core form on the same workload -------------------------
    comparison = None
    if args.compare != "none":
        other, plain, _ = timed_form(args.compare, False, reference=reference)
        other.close()
        del other
        comparison = {"mass_matrix": args.compare, **plain,
                      "speedup": value / plain["value"]}
    if reference is not None:
        sweep.append(sweep_entry(args.mass_matrix, args.precision, headline))
        if comparison is not None:
            sweep.append(sweep_entry(args.compare, args.precision, plain))
        for form in ("scalar", "tf32", "bf16x3"):
            if form in (args.mass_matrix, args.compare):
                continue
            extra_sim, extra, _ = timed_form(form, False, reference=reference)
            extra_sim.close()
            del extra_sim
            sweep.append(sweep_entry(form, args.precision, extra))
        del reference
        torch.cuda.empty_cache()

    record_bytes = 24 + 3 * (4 if args.precision == "mixed" else 8) + 8 + 4
    l2_note = ("inputs larger than L2" if nparticles * record_bytes > 126e6 else
               "inputs smaller than L2 (not flushed: a cycle's records fit in L2)")
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": headline["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": workload_name, "particles": nparticles,
                           "precision": args.precision, "mass_matrix": args.mass_matrix, "mass_layout": args.mass_layout, "dt": case.dt,
                           "theta": case.theta, "gmres_tol": case.gmres_tol,
                           "gmres_max_iterations": args.gmres_max_iterations, "l2": l2_note,
                           "smoothing": ({"passes": smoothing[0], "alpha": smoothing[1],
                                          "operator": ("face7", "binomial27")[smoothing[2]]}
                                         if smoothing[0] > 0 and smoothing[1] < 1 else None),
                           "parallelism": f"replicas x{world}"},
                "energy_drift": headline["energy_drift"], "gmres_iterations": headline["gmres_iterations"],
                "gmres_host_waits": headline["gmres_host_waits"],
                "stages_ms": headline["stages_ms"], "plain_fp32_form": comparison,
                "clocks": clocks.summary(), "e2e": e2e, "gpu_launches": headline["launches"],
                "roofline": roofline, "cycle_roofline": cycle_roofline(headline, nparticles, g, args, hbm),
                "generation_s": headline["generation_s"]}
        if sweep:
            line["sweep"] = sweep
        if not args.no_cpu_baseline and not args.deck:
            cb = cpu_oracle_rate(args.cpu_scale, 4, 2, 0)
            line["cpu_baseline"] = {"value": cb["particles"] * cb["cycles"] / cb["seconds"], "unit": UNIT,
                                    "cores": 1, "kind": "port",
                                    "sample": f"oracle cycle on a {args.cpu_scale}^3-cell slice of the workload "
                                              f"({cb['particles']} particles), {cb['cycles']} cycles, 1 thread"}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def stage_kernel_times(sim, args, stream, repeats: int = 5) -> dict:
    """Average device time of each stage's kernels launched alone through the
    C ABI, with the algorithmic bytes of one launch (HBM roofline)."""
    import torch
    from tpic_b200 import _lib
    lib, st = sim.lib, sim.state
    s_ = C.c_void_p(stream.cuda_stream)
    g = sim.case.grid
    sim.materialize()  # the stage calls below take sorted live slots
    ns = st.ns
    vb = 4 if args.precision == "mixed" else 8
    fb = vb
    n_total = sum(st.slot[s][st.current[s]].count for s in range(ns))
    nodes = sim.layout.node_count
    out = {}

    def timed(fn):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(repeats):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / repeats

    scratch_inv = torch.zeros(1, dtype=torch.int32, device="cuda")

    # Deposition (current + mass) of all species from the sorted records, as
    # the cycle runs it: one multi-species call. The tensor-core forms write
    # per-cell moments (267 floats per cell, groups of four cells), which the
    # fold assembles; the scalar forms deposit J and the mass records.
    cells = g.nx * g.ny * g.nz
    tc_form = st.mass_kind in (_lib.MASS_KINDS["tf32"], _lib.MASS_KINDS["bf16x3"], _lib.MASS_KINDS["moments-f64"])
    moment_bytes = 267 * (8 if st.mass_kind == _lib.MASS_KINDS["moments-f64"] else 4) * ((cells + 3) // 4 * 4)
    parts = (_lib.Particles * ns)(*[st.slot[s][st.current[s]] for s in range(ns)])
    qom = (C.c_double * ns)(*[st.qom[s] for s in range(ns)])
    counts = (C.c_void_p * ns)(*[st.counts[s] for s in range(ns)])
    offsets = (C.c_void_p * ns)(*[st.offsets[s] for s in range(ns)])

    def deposit():
        _lib.check(lib.tpicb200_deposit_species(sim.ctx, ns, qom, parts, counts, offsets, st.b_node, st.j, st.mass,
                                                st.mass_kind, scratch_inv.data_ptr(), s_))

    def clear_and_deposit():
        _lib.check(lib.tpicb200_clear_moments(sim.ctx, st.j, st.mass, s_))
        deposit()

    def fold():
        _lib.check(lib.tpicb200_fold_periodic(sim.ctx, st.j, st.mass, s_))

    def timed_after(setup, fn):
        """Device time of fn alone, after an untimed setup before each run."""
        setup()
        fn()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(repeats):
            setup()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            fn()
            ev1.record(stream)
            torch.cuda.synchronize()
            total += ev0.elapsed_time(ev1)
        return total / repeats

    clear = lambda: _lib.check(lib.tpicb200_clear_moments(sim.ctx, st.j, st.mass, s_))
    # Algorithmic bytes per particle: positions, velocities and charge (the
    # current's inputs; the mass assembly reads a subset of them in the same
    # pass). record_bytes adds what the kernels move beyond that: the key,
    # and the per-cell moments or the node outputs.
    out["deposit"] = {"ms": timed_after(clear, deposit), "bytes": n_total * (24 + 3 * vb + 8),
                      "basis": f"positions 24 B + velocities 3 x {vb} B + charge 8 B per particle, mass assembly "
                               "fused into the same pass",
                      "record_bytes": n_total * (24 + 3 * vb + 8 + 4) + (moment_bytes if tc_form else
                                                                         nodes * (126 + 3) * fb)}
    # The fold: for the tensor-core forms the moment assembly (moments read,
    # J and the mass records written) and the periodic fold.
    out["assembly"] = {"ms": timed_after(clear_and_deposit, fold),
                       "bytes": (moment_bytes if tc_form else 0) + nodes * (126 + 3) * fb,
                       "basis": ("per-cell moments read, " if tc_form else "") +
                                f"126 mass entries + 3 current components x {fb} B per node written"}

    # Sort of all species as the cycle runs it (the binned sort of records
    # grouped by the live bins; ping-pong into the idle slot and back).
    def sort_once():
        for s in range(ns):
            cur = st.current[s]
            _lib.check(lib.tpicb200_sort_binned(sim.ctx, C.byref(st.slot[s][cur]), st.counts[s], st.offsets[s],
                                                C.byref(st.slot[s][1 - cur]), st.counts[s], st.offsets[s],
                                                scratch_inv.data_ptr(), s_))
            st.current[s] = 1 - cur
    out["sort"] = {"ms": timed(sort_once), "bytes": n_total * (4 + 2 * (24 + 3 * vb + 8 + 4)),
                   "basis": f"key 4 B read, record ({24 + 3 * vb + 12} B) read and written per particle"}
    # Make sure the live slot is the sorted one with valid bins (an even number of sorts ran).
    if (repeats + 1) % 2:
        sort_once()

    # Mover of all species (E_theta and B as left by the last cycle).
    saved = {}
    for s in range(ns):
        cur = st.current[s]
        saved[s] = {k: v.clone() for k, v in sim.slots[s][cur].items()}

    def move():
        for s in range(ns):
            p = st.slot[s][st.current[s]]
            _lib.check(lib.tpicb200_mover(sim.ctx, st.qom[s], C.byref(p), st.e_theta, st.b_node,
                                          scratch_inv.data_ptr(), s_))
    out["mover"] = {"ms": timed(move), "bytes": n_total * 2 * (4 + 24 + 3 * vb),
                    "basis": f"key 4 B, positions 24 B, velocities 3 x {vb} B read and written per particle"}
    for s in range(ns):
        for k, v in saved[s].items():
            sim.slots[s][st.current[s]][k].copy_(v)
    del saved
    torch.cuda.synchronize()
    return out


def cycle_roofline(result: dict, particles: int, g, args, hbm: float) -> dict:
    """Whole-cycle algorithmic bytes against the cycle time: per particle the
    mover (key, positions, velocities read and written), the binned sort (key
    read, record read and written) and the fused deposition (positions,
    velocities, charge); per node the mass records per GMRES apply plus six
    double vectors of three components, and the mass written and cleared once."""
    vb = 4 if args.precision == "mixed" else 8
    record = 24 + 3 * vb + 8 + 4
    per_particle = 2 * (4 + 24 + 3 * vb) + (4 + 2 * record) + (24 + 3 * vb + 8)
    nodes = (g.nx + 1) * (g.ny + 1) * (g.nz + 1)
    mass_bytes = 126 * vb
    applies = result["gmres_iterations"]
    total = particles * per_particle + nodes * (applies * (mass_bytes + 6 * 3 * 8) + 2 * mass_bytes)
    achieved = total / (result["ms_per_step"] / 1e3) / 1e9
    return {"bytes_per_cycle": total, "bytes_per_particle": per_particle, "gmres_applies": applies,
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm}


def load_traffic(stage: str, particles: int):
    """DRAM bytes of one launch of a stage at this workload, from the committed
    ncu capture summary (bytes per particle at the workload's loading of 128
    particles per cell, captured on a smaller grid of the same loading), if any."""
    path = ROOT / "profiles" / "traffic.json"
    try:
        entry = json.loads(path.read_text())[stage]
        return entry["dram_bytes_per_particle"] * particles
    except Exception:
        return None


def end_to_end(sim, args, stream, barrier, nparticles, world, dist) -> dict:
    """The metric through the public API from host buffers, as one episode of
    a fixed --e2e-cycles cycles (independent of --steps): the full state
    (particle records of the live slots and the fields) is uploaded from
    pinned host memory, the startup runs (tpicb200_prepare), then the cycles
    (tpicb200_cycle), each reading its energy report back to the host. The
    upload is charged to the episode's cycles (h2d_bytes_per_step = upload /
    cycles); a cycle's own inputs are the previous cycle's device state."""
    import torch
    sim.materialize()
    live = []
    for s in range(sim.state.ns):
        slot = sim.slots[s][sim.state.current[s]]
        live.append({k: (v, v.cpu().pin_memory()) for k, v in slot.items()})
    fields = [(t, t.cpu().pin_memory()) for t in (sim.field("e"), sim.field("b_cell"))]
    h2d = sum(h.numel() * h.element_size() for d in live for _, h in d.values()) + \
        sum(h.numel() * h.element_size() for _, h in fields)
    steps = args.e2e_cycles
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for d in live:
        for dev, host in d.values():
            dev.copy_(host, non_blocking=True)
    for dev, host in fields:
        dev.copy_(host, non_blocking=True)
    sim.prepare()
    reports = sim.run(steps)  # energy scalars read back to the host every cycle
    stop.record(stream)
    barrier()
    seconds = max_over_ranks(start.elapsed_time(stop) / 1e3, dist, "cuda")
    d2h = (2 + 5 * sim.state.ns) * 8 + 4
    return {"value": replica_rate(world, nparticles, steps, seconds), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / steps), "d2h_bytes_per_step": d2h,
            "seconds": seconds, "cycles": len(reports)}


def run_solve(args) -> None:
    """Field solves alone: the workload's bootstrap state (deposited mass and
    J, startup E and B) solved --steps times after --warmup untimed solves,
    timed with CUDA events on the context's stream. One JSON line with ms per
    solve and the GMRES iterations. With TPICB200_STEP_GRAPH=0 in the
    environment the Arnoldi steps are launched one by one (for a kernel
    profiler's launch list)."""
    import ctypes as C
    import torch
    from tpic_b200 import _lib
    from tpic_b200.simulation import Simulation
    case = workload(args.scale)
    torch.cuda.set_device(0)
    sim = Simulation(case, precision=args.precision, mass_kind=args.mass_matrix, generate_on_device=True,
                     gmres_max_iterations=args.gmres_max_iterations, mass_layout=args.mass_layout)
    sim.prepare()
    st = sim.state
    stream = C.c_void_p(sim.stream.cuda_stream)
    e_theta = torch.zeros(3 * sim.layout.node_count, dtype=torch.float64, device=sim.device)
    res = _lib.GmresResult()

    def solve():
        _lib.check(sim.lib.tpicb200_field_solve(sim.ctx, st.e, st.b_cell, st.j, st.mass, e_theta.data_ptr(),
                                                C.byref(res), stream))

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(sim.stream)
    for _ in range(args.steps):
        solve()
    stop.record(sim.stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / args.steps
    print(json.dumps({"metric": "field solve time", "value": ms, "unit": "ms", "steps": args.steps,
                      "warmup": args.warmup, "gmres_iterations": res.iterations, "host_waits": res.host_waits,
                      "relative_residual": res.relative_residual,
                      "config": {"workload": f"bootstrap state of the {args.scale}^3-cell uniform plasma",
                                 "precision": args.precision, "mass_matrix": args.mass_matrix,
                                 "mass_layout": args.mass_layout,
                                 "step_graph": os.environ.get("TPICB200_STEP_GRAPH", "1") != "0"}}))
    sim.close()


def run_peaks(args) -> None:
    """Dense FP32 peaks the roofline of the FP32 CUDA-core and TF32 forms
    divides by: cuBLAS SGEMM with TF32 off (FP32 SIMT FMA) and with TF32 on
    (tensor cores), 8192^3, timed with CUDA events after warm-up. One JSON
    line of TFLOP/s."""
    import torch
    torch.cuda.set_device(0)
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    out = {}
    for name, tf32 in (("fp32_simt_tflops", False), ("tf32_tflops", True)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        for _ in range(3):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10 if tf32 else 3
        start.record()
        for _ in range(reps):
            torch.matmul(a, b)
        stop.record()
        torch.cuda.synchronize()
        out[name] = 2.0 * n ** 3 * reps / (start.elapsed_time(stop) * 1e-3) / 1e12
    torch.backends.cuda.matmul.allow_tf32 = False
    print(json.dumps({"metric": "dense FP32 peaks", **out, "unit": "TFLOP/s", "size": n,
                      "method": "cuBLAS SGEMM via torch.matmul, TF32 off and on"}))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["tpic_b200", "reference"], default="tpic_b200")
    ap.add_argument("--mass-matrix", default="bf16x3", choices=["scalar", "scalar-f64", "tf32", "bf16x3", "moments-f64"])
    ap.add_argument("--compare", default="scalar",
                    choices=["scalar", "scalar-f64", "tf32", "bf16x3", "moments-f64", "none"],
                    help="second form timed on the same workload (default: the plain FP32 CUDA-core form)")
    ap.add_argument("--drift-cycles", type=int, default=100, help="cycles of the energy-drift run of each form")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "double"])
    ap.add_argument("--mass-layout", default="tiled", choices=["records", "stencil-major", "tiled"],
                    help="mass buffer layout (tiled: 16-byte rows, the operator apply stages them by TMA)")
    ap.add_argument("--scale", type=int, default=128, help="cells per axis of the workload")
    ap.add_argument("--smoothing", default="",
                    help="energy-conserving smoothing as PASSES,ALPHA,OPERATOR (0 face7, 1 binomial27); off by default")
    ap.add_argument("--gmres-max-iterations", type=int, default=100,
                    help="GMRES step limit per solve (TPIC fixes 100, config/physics.hpp:20)")
    ap.add_argument("--deck", default=None,
                    help="a TPIC input deck (e.g. tpic_b200/decks/*.inp) as the workload instead of the default")
    ap.add_argument("--cpu-scale", type=int, default=24, help="cells per axis of the CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the FP64 moment and TF32 forms and state every form's bootstrap mass and J "
                         "error against the FP64 moment form (default on; off for decks)")
    ap.add_argument("--adjoint", action="store_true",
                    help="with --deck (two-stream or anisotropy): gradients by the adjoint with checkpoint-recompute, "
                         "against central differences of the FP64 forward run, and the backward/forward time ratio")
    ap.add_argument("--checkpoint-every", type=int, default=20, help="adjoint checkpoint interval (cycles)")
    ap.add_argument("--horizons", default="", help="adjoint: comma-separated cycle counts (default: the deck's)")
    ap.add_argument("--adjoint-fp64", action="store_true", help="adjoint: also the FP64 adjoint at each horizon")
    ap.add_argument("--e2e-cycles", type=int, default=20,
                    help="cycles of the end-to-end episode (upload, startup, cycles, energy readback)")
    ap.add_argument("--cpu-workers", type=int, default=0, help="host processes of the reference arm (0: all cores)")
    ap.add_argument("--peaks", action="store_true", help="measure the FP32 SIMT and TF32 GEMM peaks (cuBLAS)")
    ap.add_argument("--solve", action="store_true",
                    help="time field solves alone on the workload's bootstrap state (ms per solve)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        run_reference(args)
    elif args.adjoint:
        run_adjoint(args)
    elif args.solve:
        run_solve(args)
    elif args.peaks:
        run_peaks(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
