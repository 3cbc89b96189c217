// tpicb200_run: runs a TPIC input deck on one GPU through the library's C ABI.
//
//   tpicb200_run --run deck.inp [--mass-matrix matrix-core|scalar|scalar-f64|tf32|bf16x3|moments-f64]
//                [--precision mixed|double] [--restart] [--output DIR] [--cycles N]
//                [--diagnostics-cycle K] [--restart-cycle R] [--restart-dir NAME] [--seed S]
//                [--gmres-max-iterations M] [--device D] [--dry-run]
//
// The command line of TPIC's one-rank run (`tpic --run deck.inp --mass-matrix
// scalar|matrix-core [--restart]`, src/app/main.cpp:60-127), as a C++ host
// program that links libtpicb200.so and owns its device memory through the
// CUDA runtime: the deck is read by tpicb200_deck_parse, the initial fields
// are sampled on the host from the case (tpicb200_case_fields), the species
// are loaded and centred on the device (tpicb200_load_species,
// tpicb200_center_velocities), and the cycles run through tpicb200_cycle.
// It writes TPIC's diagnostics.csv rows (docs/user/output.md; columns of
// src/io/diagnostics_writer.cpp:60-62) every --diagnostics-cycle cycles and
// at the final state, and checkpoints every --restart-cycle cycles under
// --output/--restart-dir; --restart continues from the newest complete
// checkpoint and the diagnostics file after a `# restart at cycle N` line.
// `matrix-core` (TPIC's tensor-core form) selects BF16x3 in mixed precision
// and the FP64 moment form in double. --dry-run parses the deck and prints
// the run's sizes without touching a device.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/tpicb200.h"

namespace {

struct Args {
  std::string deck, form = "matrix-core", precision = "mixed", output = ".", restart_dir = "data";
  bool restart = false, dry_run = false;
  long long cycles = -1;
  int diagnostics_cycle = 1, restart_cycle = 0, gmres_max_iterations = 100, device = 0;
  unsigned long long seed = 0;
};

[[noreturn]] void usage(const char* why) {
  std::fprintf(stderr, "tpicb200_run: %s\n", why);
  std::fprintf(stderr,
               "usage: tpicb200_run --run deck.inp [--mass-matrix matrix-core|scalar|scalar-f64|tf32|bf16x3|"
               "moments-f64] [--precision mixed|double] [--restart] [--output DIR] [--cycles N] "
               "[--diagnostics-cycle K] [--restart-cycle R] [--restart-dir NAME] [--seed S] "
               "[--gmres-max-iterations M] [--device D] [--dry-run]\n");
  std::exit(2);
}

Args parse_args(int argc, char** argv) {
  Args a;
  auto value = [&](int& i) -> std::string {
    if (i + 1 >= argc) usage((std::string("missing value of ") + argv[i]).c_str());
    return argv[++i];
  };
  for (int i = 1; i < argc; ++i) {
    const std::string k = argv[i];
    if (k == "--run") a.deck = value(i);
    else if (k == "--mass-matrix") a.form = value(i);
    else if (k == "--precision") a.precision = value(i);
    else if (k == "--restart") a.restart = true;
    else if (k == "--dry-run") a.dry_run = true;
    else if (k == "--output") a.output = value(i);
    else if (k == "--restart-dir") a.restart_dir = value(i);
    else if (k == "--cycles") a.cycles = std::atoll(value(i).c_str());
    else if (k == "--diagnostics-cycle") a.diagnostics_cycle = std::atoi(value(i).c_str());
    else if (k == "--restart-cycle") a.restart_cycle = std::atoi(value(i).c_str());
    else if (k == "--gmres-max-iterations") a.gmres_max_iterations = std::atoi(value(i).c_str());
    else if (k == "--device") a.device = std::atoi(value(i).c_str());
    else if (k == "--seed") a.seed = std::strtoull(value(i).c_str(), nullptr, 10);
    else if (k == "--help" || k == "-h") usage("help");
    else usage(("unknown option " + k).c_str());
  }
  if (a.deck.empty()) usage("--run DECK is required");
  if (a.precision != "mixed" && a.precision != "double") usage("--precision is mixed or double");
  return a;
}

int mass_kind(const std::string& form, bool dbl) {
  if (form == "matrix-core") return dbl ? TPICB200_MASS_MOMENTS_F64 : TPICB200_MASS_BF16X3;
  if (form == "scalar") return TPICB200_MASS_SCALAR;
  if (form == "scalar-f64" || form == "fp64") return TPICB200_MASS_SCALAR_F64;
  if (form == "tf32") return TPICB200_MASS_TF32;
  if (form == "bf16x3") return TPICB200_MASS_BF16X3;
  if (form == "moments-f64") return TPICB200_MASS_MOMENTS_F64;
  usage(("unknown --mass-matrix " + form).c_str());
}

void check(int status, const char* what) {
  if (status != TPICB200_SUCCESS) {
    std::fprintf(stderr, "tpicb200_run: %s: status %d: %s\n", what, status, tpicb200_last_error());
    std::exit(1);
  }
}

void cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "tpicb200_run: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(1);
  }
}

// Shortest round-trip decimal of a double (the form Python's repr prints).
std::string num(double v) {
  char buf[64];
  const auto r = std::to_chars(buf, buf + sizeof(buf), v);
  return std::string(buf, r.ptr);
}

// Device memory owned by the driver, freed at exit.
struct Device {
  std::vector<void*> blocks;
  void* alloc(size_t bytes) {
    void* p = nullptr;
    cuda(cudaMalloc(&p, bytes ? bytes : 8), "device allocation");
    blocks.push_back(p);
    return p;
  }
  ~Device() {
    for (void* p : blocks) cudaFree(p);
  }
};

// One field over the stored extent (nodes -1..n+1 or cells -1..n per axis,
// x fastest) at unwrapped coordinates (i + offset) * spacing, as TPIC's host
// field image samples it (initialization/fields/field_image.hpp:30-90):
// component-major values in the node or cell layout of the header.
std::vector<double> sample_field(const tpicb200_deck& deck, bool nodal) {
  const tpicb200_grid& g = deck.grid;
  const double h[3] = {g.lx / g.nx, g.ly / g.ny, g.lz / g.nz};
  const int n[3] = {g.nx, g.ny, g.nz};
  const int extra = nodal ? 1 : 0;
  const double offset = nodal ? 0.0 : 0.5;
  const long long ex = n[0] + extra + 2, ey = n[1] + extra + 2, ez = n[2] + extra + 2;
  const long long count = ex * ey * ez;
  std::vector<double> x(count), y(count), z(count), e(3 * count), b(3 * count);
  for (long long k = 0; k < ez; ++k)
    for (long long j = 0; j < ey; ++j)
      for (long long i = 0; i < ex; ++i) {
        const long long p = i + ex * (j + ey * k);
        x[p] = (double(i - 1) + offset) * h[0];
        y[p] = (double(j - 1) + offset) * h[1];
        z[p] = (double(k - 1) + offset) * h[2];
      }
  check(tpicb200_case_fields(&deck, count, x.data(), y.data(), z.data(), e.data(), b.data()), "case fields");
  return nodal ? e : b;
}

void upload(void* dst, const std::vector<double>& values, bool as_float) {
  if (as_float) {
    std::vector<float> f(values.begin(), values.end());
    cuda(cudaMemcpy(dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice), "field upload");
  } else {
    cuda(cudaMemcpy(dst, values.data(), values.size() * 8, cudaMemcpyHostToDevice), "field upload");
  }
}

std::string columns(int ns) {
  std::string s = "cycle,time,state,electric_energy,magnetic_energy,kinetic_energy,total_energy,"
                  "total_energy_change,charge,momentum_x,momentum_y,momentum_z";
  for (int sp = 0; sp < ns; ++sp) {
    const std::string i = std::to_string(sp);
    s += ",kinetic_energy_" + i + ",charge_" + i + ",momentum_x_" + i + ",momentum_y_" + i + ",momentum_z_" + i;
  }
  return s;
}

const char* kHeader =
    "# electric_energy = V/(8 pi) sum over unique nodes |E|^2; magnetic_energy = V/(8 pi) sum over cells |B|^2;\n"
    "# kinetic_energy = sum 1/2 (q/qom) |v|^2; momentum = sum (q/qom) v; charge = sum q.\n"
    "# state=pre_solve identifies the state before the cycle's solve/push; state=final identifies the completed "
    "run state.\n"
    "# time is physical simulation time at the recorded state; total_energy_change = total_energy - the total "
    "energy of the run's first state, kept across restarts (absolute units).\n";

// One diagnostics.csv row: field energies (E, B) and per species kinetic
// energy, charge and momentum x/y/z.
std::string row(long long cycle, double dt, bool final, const double field[2], const double species[][5], int ns,
                double initial) {
  double kinetic = 0, sums[4] = {0, 0, 0, 0};
  for (int sp = 0; sp < ns; ++sp) {
    kinetic += species[sp][0];
    for (int k = 0; k < 4; ++k) sums[k] += species[sp][1 + k];
  }
  const double total = field[0] + field[1] + kinetic;
  std::string s = std::to_string(cycle) + "," + num(double(cycle) * dt) + "," + (final ? "final" : "pre_solve");
  const double values[] = {field[0], field[1], kinetic, total, total - initial, sums[0], sums[1], sums[2], sums[3]};
  for (double v : values) s += "," + num(v);
  for (int sp = 0; sp < ns; ++sp)
    for (int k = 0; k < 5; ++k) s += "," + num(species[sp][k]);
  return s;
}

bool file_exists(const std::string& path) {
  struct stat st{};
  return ::stat(path.c_str(), &st) == 0;
}

}  // namespace

int main(int argc, char** argv) {
  const Args args = parse_args(argc, argv);
  std::ifstream in(args.deck);
  if (!in) usage(("cannot read " + args.deck).c_str());
  std::stringstream text;
  text << in.rdbuf();
  tpicb200_deck deck{};
  check(tpicb200_deck_parse(text.str().c_str(), &deck), "deck");
  const bool dbl = args.precision == "double";
  const int kind = mass_kind(args.form, dbl);
  const long long last = args.cycles >= 0 ? args.cycles : deck.ncycles;
  const tpicb200_grid grid = deck.grid;
  const long long cells = (long long)grid.nx * grid.ny * grid.nz;
  uint32_t count[TPICB200_MAX_SPECIES] = {};
  uint32_t largest = 0;
  for (int s = 0; s < deck.ns; ++s) {
    const long long ppc = (long long)deck.species[s].npcel[0] * deck.species[s].npcel[1] * deck.species[s].npcel[2];
    if (cells * ppc > 0xffffffffLL) usage("a species has more than 2^32 - 1 records");
    count[s] = uint32_t(cells * ppc);
    largest = std::max(largest, count[s]);
  }
  if (args.dry_run) {
    std::printf("deck %s: case %s, %dx%dx%d cells, %d species", args.deck.c_str(), deck.case_name, grid.nx, grid.ny,
                grid.nz, deck.ns);
    for (int s = 0; s < deck.ns; ++s) std::printf(" %s%u", s ? "+" : " ", count[s]);
    std::printf(" records, %lld cycles, mass form %d, %s precision\n", last, kind, args.precision.c_str());
    return 0;
  }

  cuda(cudaSetDevice(args.device), "device selection");
  tpicb200_options opt{};
  opt.dt = deck.dt;
  opt.theta = deck.theta;
  opt.c = deck.c;
  opt.gmres_tol = deck.gmres_tol;
  opt.gmres_restart = 30;
  opt.gmres_max_iterations = args.gmres_max_iterations;
  opt.precision = dbl ? TPICB200_PRECISION_DOUBLE : TPICB200_PRECISION_MIXED;
  opt.max_particles = largest;
  opt.mass_layout = TPICB200_MASS_LAYOUT_STENCIL_MAJOR;
  opt.smooth_iterations = deck.smooth_iterations;
  opt.smooth_alpha = deck.smooth_alpha;
  opt.smooth_operator = deck.smooth_operator;
  tpicb200_context* ctx = nullptr;
  check(tpicb200_create(&grid, &opt, &ctx), "context");
  tpicb200_layout lay{};
  check(tpicb200_get_layout(ctx, &lay), "layout");

  Device dev;
  const size_t fb = lay.field_scalar_bytes, vb = lay.velocity_scalar_bytes;
  tpicb200_state st{};
  st.ns = deck.ns;
  st.e = dev.alloc(3 * lay.node_count * fb);
  st.b_cell = dev.alloc(3 * lay.cell_count * fb);
  st.b_cell_next = dev.alloc(3 * lay.cell_count * fb);
  st.b_node = dev.alloc(3 * lay.node_count * fb);
  st.b_node_next = dev.alloc(3 * lay.node_count * fb);
  st.j = dev.alloc(3 * lay.node_count * fb);
  st.mass = dev.alloc(size_t(lay.mass_count) * lay.mass_scalar_bytes);
  st.e_theta = (double*)dev.alloc(3 * lay.node_count * 8);
  st.mass_kind = kind;
  for (int s = 0; s < deck.ns; ++s) {
    st.qom[s] = deck.species[s].qom;
    const size_t n = count[s];
    for (int k = 0; k < 2; ++k) {
      tpicb200_particles& p = st.slot[s][k];
      p.rx = dev.alloc(8 * n);
      p.ry = dev.alloc(8 * n);
      p.rz = dev.alloc(8 * n);
      p.u = dev.alloc(vb * n);
      p.v = dev.alloc(vb * n);
      p.w = dev.alloc(vb * n);
      p.q = (double*)dev.alloc(8 * n);
      p.cell = (int32_t*)dev.alloc(4 * n);
      p.id = (uint64_t*)dev.alloc(8 * n);
      p.count = count[s];
    }
    st.current[s] = 0;
    st.counts[s] = (uint32_t*)dev.alloc(4 * lay.bin_count);
    st.offsets[s] = (uint32_t*)dev.alloc(4 * (lay.bin_count + 1));
    st.ranks[s] = (uint32_t*)dev.alloc(4 * n);
  }
  cudaStream_t stream = nullptr;
  cuda(cudaStreamCreate(&stream), "stream");
  const tpicb200_stream s_ = (tpicb200_stream)stream;

  const std::string out = args.output;
  ::mkdir(out.c_str(), 0755);
  const std::string ckpt_dir = out + "/" + args.restart_dir;
  const std::string csv = out + "/diagnostics.csv";
  long long cycle = 0;
  double initial = NAN;
  if (args.restart) {
    char path[4096];
    check(tpicb200_checkpoint_find(ckpt_dir.c_str(), path, sizeof(path)), "checkpoint search");
    tpicb200_checkpoint_info info{};
    check(tpicb200_checkpoint_info_read(path, &info), "checkpoint header");
    for (int s = 0; s < deck.ns; ++s)
      if (info.count[s] != count[s]) usage("the checkpoint's record counts are not the deck's");
    check(tpicb200_checkpoint_read(ctx, &st, path, &info, s_), "checkpoint read");
    cycle = info.cycle;
    // The restarted run replaces the rows from its checkpoint cycle on and
    // keeps the first state's total energy as the reference of the change.
    std::vector<std::string> kept;
    if (file_exists(csv)) {
      std::ifstream old(csv);
      std::string line;
      while (std::getline(old, line)) {
        if (!line.empty() && std::isdigit((unsigned char)line[0])) {
          if (std::isnan(initial)) {
            std::stringstream fields(line);
            std::string f;
            for (int c = 0; c < 7 && std::getline(fields, f, ','); ++c) {
            }
            initial = std::strtod(f.c_str(), nullptr);
          }
          if (std::atoll(line.c_str()) >= cycle) continue;
        }
        kept.push_back(line);
      }
    } else {
      std::stringstream h(std::string(kHeader) + columns(deck.ns));
      std::string line;
      while (std::getline(h, line)) kept.push_back(line);
    }
    kept.push_back("# restart at cycle " + std::to_string(cycle));
    std::ofstream f(csv);
    for (const std::string& line : kept) f << line << "\n";
  } else {
    upload(st.e, sample_field(deck, true), !dbl);
    upload(st.b_cell, sample_field(deck, false), !dbl);
    for (int s = 0; s < deck.ns; ++s) {
      check(tpicb200_load_species(ctx, &deck, s, args.seed, 0, &st.slot[s][0], nullptr, s_), "species loading");
      if (deck.species[s].center_velocity)
        check(tpicb200_center_velocities(ctx, &deck, s, &st.slot[s][0], nullptr, s_), "velocity centring");
    }
    std::ofstream f(csv);
    f << kHeader << columns(deck.ns) << "\n";
  }
  if (last < cycle) usage("the run's last cycle lies before the checkpoint cycle");
  check(tpicb200_prepare(ctx, &st, s_), "startup");
  {
    uint32_t bad = 0;
    check(tpicb200_read_invalid(ctx, &bad, 1, s_), "invalid-counter read");
    if (bad) {
      std::fprintf(stderr, "tpicb200_run: %u nonfinite records at startup\n", bad);
      return 1;
    }
  }
  double field[2], species[TPICB200_MAX_SPECIES][5];
  {
    tpicb200_particles live[TPICB200_MAX_SPECIES];
    for (int s = 0; s < deck.ns; ++s) live[s] = st.slot[s][st.current[s]];
    std::vector<double> w(2 + 5 * deck.ns);
    check(tpicb200_energy(ctx, st.e, st.b_cell, live, st.qom, deck.ns, w.data(), s_), "energy");
    field[0] = w[0];
    field[1] = w[1];
    for (int s = 0; s < deck.ns; ++s)
      for (int k = 0; k < 5; ++k) species[s][k] = w[2 + 5 * s + k];
  }
  auto total_of = [&] {
    double t = field[0] + field[1];
    for (int s = 0; s < deck.ns; ++s) t += species[s][0];
    return t;
  };
  if (std::isnan(initial)) initial = total_of();
  const int cadence = args.diagnostics_cycle > 0 ? args.diagnostics_cycle : 0;
  const int every = args.restart_cycle > 0 ? args.restart_cycle : 0;
  auto record = [&](bool final) {
    std::ofstream f(csv, std::ios::app);
    f << row(cycle, deck.dt, final, field, species, deck.ns, initial) << "\n";
    const double t = total_of();
    std::printf("cycle %6lld  total energy %.10e  change %+.3e\n", cycle, t, t - initial);
    std::fflush(stdout);
  };
  if ((cadence && cycle % cadence == 0) || cycle == last) record(cycle == last);
  std::vector<tpicb200_cycle_report> reports;
  while (cycle < last) {
    long long stop = last;
    if (cadence) stop = std::min(stop, (cycle / cadence + 1) * cadence);
    if (every) stop = std::min(stop, (cycle / every + 1) * every);
    const int n = int(stop - cycle);
    reports.assign(n, tpicb200_cycle_report{});
    check(tpicb200_cycle(ctx, &st, n, reports.data(), s_), "cycle");
    cycle = stop;
    const tpicb200_cycle_report& r = reports.back();
    field[0] = r.field_energy[0];
    field[1] = r.field_energy[1];
    for (int s = 0; s < deck.ns; ++s)
      for (int k = 0; k < 5; ++k) species[s][k] = r.species[s][k];
    if (every && (cycle % every == 0 || cycle == last))
      check(tpicb200_checkpoint_write(ctx, &st, ckpt_dir.c_str(), int(cycle), s_), "checkpoint write");
    if (cycle == last || (cadence && cycle % cadence == 0)) record(cycle == last);
    if (!std::isfinite(field[0]) || !std::isfinite(field[1])) {
      std::fprintf(stderr, "tpicb200_run: nonfinite field energy\n");
      return 1;
    }
  }
  cudaStreamDestroy(stream);
  check(tpicb200_destroy(ctx), "context release");
  return 0;
}
