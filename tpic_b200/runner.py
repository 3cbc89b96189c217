"""Deck runner: `python -m tpic_b200 --run deck.inp --mass-matrix ...`.

Runs a TPIC input deck through the library the way TPIC's driver runs a
one-rank periodic case (src/main.cpp `--run`, `--mass-matrix`, `--restart`):
the deck's case and species, `ncycles` cycles, the energy diagnostics rows of
TPIC's `diagnostics.csv` (docs/user/output.md, "diagnostics.csv": cycle, time,
state, electric, magnetic, kinetic and total energy, the change of the total
energy from the run's first state, charge and momentum, then per species
kinetic energy, charge and momentum) every `DiagnosticsOutputCycle` cycles and
at the final state, in `SaveDirName` after the precision lines, and checkpoints
every `RestartOutputCycle` cycles under `RestartDirName` (deck keys with TPIC's
defaults, docs/user/input_keys.md: DiagnosticsOutputCycle = FieldOutputCycle,
RestartOutputCycle = 0, both directories `data`; a nonpositive diagnostics
cadence disables the file; the command-line options override the keys).
`--restart` continues from the newest complete checkpoint, and the diagnostics
file continues after a `# restart at cycle N` line.
"""
from __future__ import annotations

import argparse
import math
import sys
from pathlib import Path

from . import deck as D

FORMS = ("scalar", "scalar-f64", "tf32", "bf16x3", "moments-f64", "matrix-core")

HEADER = (
    "# electric_energy = V/(8 pi) sum over unique nodes |E|^2; magnetic_energy = V/(8 pi) sum over cells |B|^2;\n"
    "# kinetic_energy = sum 1/2 (q/qom) |v|^2; momentum = sum (q/qom) v; charge = sum q.\n"
    "# state=pre_solve identifies the state before the cycle's solve/push; state=final identifies the completed "
    "run state.\n"
    "# time is physical simulation time at the recorded state; total_energy_change = total_energy - the total "
    "energy of the run's first state, kept across restarts (absolute units).\n")


def columns(ns: int) -> str:
    cols = ["cycle", "time", "state", "electric_energy", "magnetic_energy", "kinetic_energy", "total_energy",
            "total_energy_change", "charge", "momentum_x", "momentum_y", "momentum_z"]
    for s in range(ns):
        cols += [f"kinetic_energy_{s}", f"charge_{s}", f"momentum_x_{s}", f"momentum_y_{s}", f"momentum_z_{s}"]
    return ",".join(cols)


def row(cycle: int, dt: float, final: bool, field: tuple, species: tuple, initial_total: float) -> str:
    """One diagnostics.csv row from the field energies (E, B) and the species
    scalars (kinetic, charge, momentum x, y, z per species)."""
    kinetic = sum(sp[0] for sp in species)
    total = field[0] + field[1] + kinetic
    sums = [sum(sp[k] for sp in species) for k in range(1, 5)]
    values = [field[0], field[1], kinetic, total, total - initial_total, *sums]
    for sp in species:
        values += list(sp)
    return ",".join([str(cycle), repr(cycle * dt), "final" if final else "pre_solve"] + [repr(float(v)) for v in values])


def first_total(csv_path: Path) -> float | None:
    """The total energy of the first row of an existing diagnostics file."""
    if not csv_path.exists():
        return None
    for line in csv_path.read_text().splitlines():
        if line and line[0].isdigit():
            fields = line.split(",")
            return float(fields[6])
    return None


def resolve_form(form: str, precision: str) -> str:
    """TPIC's `--mass-matrix matrix-core` is its tensor-core form: here BF16x3
    in mixed precision and the FP64 moment form in double precision."""
    if form == "matrix-core":
        return "moments-f64" if precision == "double" else "bf16x3"
    return form


class _Parser(argparse.ArgumentParser):
    """An invalid command line exits with code 1, as TPIC's."""

    def error(self, message):
        self.print_usage(sys.stderr)
        self.exit(1, f"{self.prog}: error: {message}\n")


def parse_args(argv=None):
    ap = _Parser(prog="python -m tpic_b200", description="Run a TPIC input deck on one B200.")
    # TPIC's command line (src/app/main.cpp:60-120): exactly one of the three
    # commands and one input file.
    mode = ap.add_mutually_exclusive_group(required=True)
    mode.add_argument("--check-input", action="store_true", help="parse and check the deck, no device, no output")
    mode.add_argument("--initialize", action="store_true", help="complete the startup and exit before the cycles")
    mode.add_argument("--run", action="store_true", help="advance the deck's cycles")
    ap.add_argument("input", metavar="DECK", help="TPIC input deck (.inp)")
    ap.add_argument("--mass-matrix", default="scalar", choices=FORMS)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "double"])
    ap.add_argument("--order", default="partial", choices=["full", "partial", "unsorted"],
                    help="accepted for TPIC's command line: the records are sorted by cell every cycle")
    ap.add_argument("--overwrite-output", action="store_true",
                    help="replace output files that exist (a fresh run refuses them otherwise)")
    ap.add_argument("--restart", action="store_true", help="continue from the newest complete checkpoint")
    ap.add_argument("--output", default=".", help="directory of diagnostics.csv and RestartDirName")
    ap.add_argument("--cycles", type=int, default=None, help="last cycle of the run (default: the deck's ncycles)")
    ap.add_argument("--diagnostics-cycle", type=int, default=None,
                    help="DiagnosticsOutputCycle (default: the deck's, else FieldOutputCycle; <= 0: no file)")
    ap.add_argument("--restart-cycle", type=int, default=None,
                    help="RestartOutputCycle (default: the deck's, else 0: no checkpoints)")
    ap.add_argument("--restart-dir", default=None, help="RestartDirName, under --output (default: the deck's, else data)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--gmres-max-iterations", type=int, default=100)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--field-output-cycle", type=int, default=None,
                    help="FieldOutputCycle (default: the deck's, else 100; <= 0: no field snapshots)")
    ap.add_argument("--particles-output-cycle", type=int, default=None,
                    help="ParticlesOutputCycle (default: the deck's, else 0: no particle snapshots)")
    ap.add_argument("--save-dir", default=None, help="SaveDirName of the snapshots, under --output (default: the "
                                                     "deck's, else data)")
    ap.add_argument("--gauss-cycle", type=int, default=None,
                    help="DiagnosticGaussCycle (default: the deck's, else 0: no Gauss-law samples)")
    args = ap.parse_args(argv)
    if args.restart and args.check_input:
        ap.error("--restart is only valid with --run or --initialize")
    return args


def run(args) -> int:
    from .simulation import Simulation
    from .output import (GaussSampler, GaussWriter, OutputPlan, deck_keys, precision_strings, select_arrays,
                         write_fields, write_particles)
    text = Path(args.input).read_text()
    deck = D.parse(text)
    case = D.to_case(deck, seed=args.seed)
    last = deck.ncycles if args.cycles is None else args.cycles
    form = resolve_form(args.mass_matrix, args.precision)
    out = Path(args.output)
    plan = OutputPlan.from_deck(text, out, field_cycle=args.field_output_cycle,
                                particles_cycle=args.particles_output_cycle, gauss_cycle=args.gauss_cycle)
    if args.save_dir is not None:
        plan.save_dir = out / args.save_dir
    select_arrays(plan.field_tag, plan.moments_tag, len(case.species))  # the tags are checked before any work
    plan.overwrite = args.overwrite_output or args.restart
    keys = deck_keys(text)
    ckpt_dir = out / (args.restart_dir if args.restart_dir is not None else (keys.get("RestartDirName", "") or "data"))
    if args.check_input:
        g = case.grid
        print(f"deck {args.input}: {g.nx}x{g.ny}x{g.nz} cells, {len(case.species)} species, "
              f"{last} cycles, mass form {form}, {args.precision} precision; output under {plan.save_dir}")
        return 0
    csv_path = plan.save_dir / "diagnostics.csv"
    diagnostics_cycle = (args.diagnostics_cycle if args.diagnostics_cycle is not None else
                         int(keys.get("DiagnosticsOutputCycle", plan.field_cycle)))
    restart_cycle = (args.restart_cycle if args.restart_cycle is not None else
                     int(keys.get("RestartOutputCycle", 0)))
    kw = dict(precision=args.precision, mass_kind=form, device=args.device,
              gmres_max_iterations=args.gmres_max_iterations, keep_ids=plan.particles_cycle > 0)
    ns = len(case.species)
    diagnostics = diagnostics_cycle > 0
    if args.restart:
        sim = Simulation.restart(case, ckpt_dir, **kw)
        initial = first_total(csv_path)
    else:
        sim = Simulation(case, generate_on_device=True, **kw)
        sim.prepare()
        initial = None
    if args.initialize:
        # The startup is complete; --initialize writes no output.
        print(f"initialized: cycle {sim.cycle}, {len(case.species)} species, context ready")
        sim.close()
        return 0
    out.mkdir(parents=True, exist_ok=True)
    plan.save_dir.mkdir(parents=True, exist_ok=True)
    if not args.restart and not plan.overwrite:
        for path, used in ((csv_path, diagnostics), (plan.save_dir / "gauss.csv", plan.gauss_enabled())):
            if used and path.exists():
                raise SystemExit(f"{path} exists (--overwrite-output replaces it)")
    profile, roles = precision_strings(sim)
    head = f"# precision_profile = {profile}\n# precision_roles = {roles}\n" + HEADER + columns(ns)
    if diagnostics and args.restart:
        # The restarted run replaces the rows from its checkpoint cycle on.
        kept = []
        if csv_path.exists():
            for line in csv_path.read_text().splitlines():
                if line and line[0].isdigit() and int(line.split(",")[0]) >= sim.cycle:
                    continue
                kept.append(line)
        else:
            kept = head.splitlines()
        kept.append(f"# restart at cycle {sim.cycle}: precision_profile = {profile}, precision_roles = {roles}")
        csv_path.write_text("\n".join(kept) + "\n")
    elif diagnostics:
        csv_path.write_text(head + "\n")
    if last < sim.cycle:
        raise SystemExit(f"the run's last cycle {last} lies before the checkpoint cycle {sim.cycle}")
    w = sim.energy()
    field = (w[0], w[1])
    species = tuple(tuple(w[2 + 5 * s:7 + 5 * s]) for s in range(ns))
    if initial is None:
        initial = field[0] + field[1] + sum(sp[0] for sp in species)
    cadence = diagnostics_cycle if diagnostics else 0
    ckpt = restart_cycle if restart_cycle > 0 else 0
    gauss = gauss_writer = None
    if plan.gauss_enabled():
        gauss = GaussSampler(sim)
        gauss_writer = GaussWriter(plan.save_dir / "gauss.csv", profile, roles,
                                   restart_cycle=sim.cycle if args.restart else None)

    def record(final: bool) -> None:
        if diagnostics:
            with open(csv_path, "a") as f:
                f.write(row(sim.cycle, case.dt, final, field, species, initial) + "\n")
        total = field[0] + field[1] + sum(sp[0] for sp in species)
        print(f"cycle {sim.cycle:6d}  total energy {total:.10e}  change {total - initial:+.3e}", flush=True)

    def gauss_step() -> None:
        if gauss is None:
            return
        sample = gauss.step(sim.cycle, plan.gauss_begins(sim.cycle, last))
        if sample is not None:
            gauss_writer.write(sample)
            r, d, w, c = sample.rms
            print(f"  Gauss residual: cycle {sample.cycle} t = {sample.time:e}  rms = {r:e}  drift = {d:e}  "
                  f"wall = {w:e}  charge = {c:e}", flush=True)

    def snapshots() -> None:
        final = sim.cycle == last
        fields_due, particles_due = plan.due(sim.cycle, final)
        if fields_due:
            write_fields(sim, plan, sim.cycle, final, gauss)
        if particles_due:
            write_particles(sim, plan, sim.cycle, final)

    if (cadence and sim.cycle % cadence == 0) or sim.cycle == last:
        record(sim.cycle == last)
    gauss_step()
    snapshots()
    while sim.cycle < last:
        stops = [last]
        if cadence:
            stops.append((sim.cycle // cadence + 1) * cadence)
        if ckpt:
            stops.append((sim.cycle // ckpt + 1) * ckpt)
        for channel in (plan.field_cycle, plan.particles_cycle):
            if channel > 0:
                stops.append((sim.cycle // channel + 1) * channel)
        if gauss is not None:
            if gauss.begun is not None:
                stops.append(gauss.begun + 1)
            nxt = plan.next_gauss_begin(sim.cycle, last)
            if nxt is not None:
                stops.append(nxt)
        n = min(stops) - sim.cycle
        reports = sim.run(n)
        r = reports[-1]
        field, species = tuple(r.field_energy), r.species_scalars
        if ckpt and (sim.cycle % ckpt == 0 or sim.cycle == last):
            sim.checkpoint(ckpt_dir)
        if sim.cycle == last or (cadence and sim.cycle % cadence == 0):
            record(sim.cycle == last)
        gauss_step()
        snapshots()
        if not all(math.isfinite(x) for x in field):
            raise SystemExit("nonfinite field energy")
    sim.close()
    return 0


def main(argv=None) -> int:
    return run(parse_args(argv))


if __name__ == "__main__":
    sys.exit(main())
