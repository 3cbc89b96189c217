// tpicb200_run: runs a TPIC input deck on one GPU through the library's C ABI.
//
//   tpicb200_run --run deck.inp [--mass-matrix matrix-core|scalar|scalar-f64|tf32|bf16x3|moments-f64]
//                [--precision mixed|double] [--restart] [--output DIR] [--cycles N]
//                [--diagnostics-cycle K] [--restart-cycle R] [--restart-dir NAME] [--seed S]
//                [--gmres-max-iterations M] [--device D] [--field-output-cycle F]
//                [--particles-output-cycle P] [--save-dir NAME] [--gauss-cycle K] [--dry-run]
//
// The command line of TPIC's one-rank run (`tpic --run deck.inp --mass-matrix
// scalar|matrix-core [--restart]`, src/app/main.cpp:60-127), as a C++ host
// program that links libtpicb200.so and owns its device memory through the
// CUDA runtime: the deck is read by tpicb200_deck_parse, the initial fields
// are sampled on the host from the case (tpicb200_case_fields), the species
// are loaded and centred on the device (tpicb200_load_species,
// tpicb200_center_velocities), and the cycles run through tpicb200_cycle.
// Output follows TPIC's channels and deck keys (docs/user/output.md,
// docs/user/input_keys.md), each key overridden by its option:
// - diagnostics.csv in SaveDirName (precision lines, then the columns of
//   src/io/diagnostics_writer.cpp:60-62): a row every DiagnosticsOutputCycle
//   cycles (default FieldOutputCycle; <= 0: no file) and at the final state;
// - checkpoints every RestartOutputCycle cycles (default 0) under
//   RestartDirName (default data); --restart continues from the newest
//   complete checkpoint and the diagnostics file after a
//   `# restart at cycle N: ...` line;
// - snapshots every FieldOutputCycle cycles (one `<array>_tNNNNNN.vti` per
//   array selected by FieldOutputTag / MomentsOutputTag) and every
//   ParticlesOutputCycle cycles (`particles_tNNNNNN.pvtp` with its piece),
//   both also at the final state, under SaveDirName (default data);
// - Gauss-law samples every DiagnosticGaussCycle cycles and, with the Gauss
//   array, before every field snapshot: gauss.csv rows and the Gauss array.
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
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/tpicb200.h"

namespace {

struct Args {
  std::string deck, form = "scalar", precision = "mixed", output = ".", restart_dir, order = "partial";
  std::string mode;  // check, initialize or run
  bool restart = false, overwrite = false;
  long long cycles = -1;
  // Unset (has_* false): the deck's DiagnosticsOutputCycle, RestartOutputCycle, RestartDirName.
  bool has_diagnostics_cycle = false, has_restart_cycle = false, has_restart_dir = false;
  int diagnostics_cycle = 0, restart_cycle = 0, gmres_max_iterations = 100, device = 0;
  unsigned long long seed = 0;
  // Snapshot overrides of the deck's keys (unset: the deck's value).
  bool has_field_cycle = false, has_particles_cycle = false, has_save_dir = false, has_gauss_cycle = false;
  int field_cycle = 0, particles_cycle = 0, gauss_cycle = 0;
  std::string save_dir;
};

const char* kUsage =
    "usage: tpicb200_run --check-input|--initialize|--run deck.inp [--mass-matrix scalar|matrix-core|scalar-f64|"
    "tf32|bf16x3|moments-f64] [--precision mixed|double] [--order full|partial|unsorted] [--overwrite-output] "
    "[--restart] [--output DIR] [--cycles N] [--diagnostics-cycle K] [--restart-cycle R] [--restart-dir NAME] "
    "[--seed S] [--gmres-max-iterations M] [--device D] [--field-output-cycle F] [--particles-output-cycle P] "
    "[--save-dir NAME] [--gauss-cycle K]\n";

// An invalid command line or input: exit code 1, as TPIC's.
[[noreturn]] void usage(const char* why) {
  std::fprintf(stderr, "tpicb200_run: %s\n", why);
  std::fputs(kUsage, stderr);
  std::exit(1);
}

// TPIC's command line (src/app/main.cpp:60-120): exactly one of --check-input,
// --initialize or --run and one input file (--dry-run is --check-input); the
// options of this driver follow.
Args parse_args(int argc, char** argv) {
  Args a;
  auto value = [&](int& i) -> std::string {
    if (i + 1 >= argc) usage((std::string("missing value of ") + argv[i]).c_str());
    return argv[++i];
  };
  int modes = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string k = argv[i];
    if (k == "--help" || k == "-h") {
      std::fputs(kUsage, stdout);
      std::exit(0);
    }
    if (k == "--check-input" || k == "--dry-run") { a.mode = "check"; ++modes; }
    else if (k == "--initialize") { a.mode = "initialize"; ++modes; }
    else if (k == "--run") { a.mode = "run"; ++modes; }
    else if (k == "--mass-matrix") a.form = value(i);
    else if (k == "--precision") a.precision = value(i);
    else if (k == "--order") a.order = value(i);
    else if (k == "--overwrite-output") a.overwrite = true;
    else if (k == "--restart") a.restart = true;
    else if (k == "--output") a.output = value(i);
    else if (k == "--restart-dir") {
      a.has_restart_dir = true;
      a.restart_dir = value(i);
    }
    else if (k == "--cycles") a.cycles = std::atoll(value(i).c_str());
    else if (k == "--diagnostics-cycle") {
      a.has_diagnostics_cycle = true;
      a.diagnostics_cycle = std::atoi(value(i).c_str());
    } else if (k == "--restart-cycle") {
      a.has_restart_cycle = true;
      a.restart_cycle = std::atoi(value(i).c_str());
    }
    else if (k == "--gmres-max-iterations") a.gmres_max_iterations = std::atoi(value(i).c_str());
    else if (k == "--device") a.device = std::atoi(value(i).c_str());
    else if (k == "--seed") a.seed = std::strtoull(value(i).c_str(), nullptr, 10);
    else if (k == "--field-output-cycle") {
      a.has_field_cycle = true;
      a.field_cycle = std::atoi(value(i).c_str());
    } else if (k == "--particles-output-cycle") {
      a.has_particles_cycle = true;
      a.particles_cycle = std::atoi(value(i).c_str());
    } else if (k == "--save-dir") {
      a.has_save_dir = true;
      a.save_dir = value(i);
    } else if (k == "--gauss-cycle") {
      a.has_gauss_cycle = true;
      a.gauss_cycle = std::atoi(value(i).c_str());
    }
    else if (!k.empty() && k[0] == '-') usage(("unknown option " + k).c_str());
    else if (!a.deck.empty()) usage("expected exactly one input file");
    else a.deck = k;
  }
  if (modes != 1 || a.deck.empty()) usage("give exactly one of --check-input, --initialize or --run and one input file");
  if (a.restart && a.mode == "check") usage("--restart is only valid with --run or --initialize");
  if (a.precision != "mixed" && a.precision != "double") usage("--precision is mixed or double");
  // Records are kept sorted by cell every cycle whatever the order: TPIC's
  // three orders differ in its kernels' access patterns, not in the results.
  if (a.order != "full" && a.order != "partial" && a.order != "unsorted")
    usage("--order must be full, partial or unsorted");
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

[[noreturn]] void fail(const std::string& why) {
  std::fprintf(stderr, "tpicb200_run: %s\n", why.c_str());
  std::exit(1);
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

// mkdir -p: every missing directory of the path.
void make_dirs(const std::string& path) {
  for (size_t at = path.find('/', 1); ; at = path.find('/', at + 1)) {
    const std::string part = path.substr(0, at);
    if (!part.empty() && ::mkdir(part.c_str(), 0755) != 0 && !file_exists(part))
      fail("cannot create " + part);
    if (at == std::string::npos) break;
  }
}

// key -> value of a deck text: the last assignment of a key wins, `#` starts
// a comment (the reading of TPIC's key = value decks).
std::map<std::string, std::string> deck_keys(const std::string& text) {
  std::map<std::string, std::string> keys;
  auto trim = [](std::string v) {
    const char* ws = " \t\r\n\f\v";
    const size_t a = v.find_first_not_of(ws);
    if (a == std::string::npos) return std::string();
    return v.substr(a, v.find_last_not_of(ws) - a + 1);
  };
  std::stringstream in(text);
  std::string line;
  while (std::getline(in, line)) {
    line = line.substr(0, line.find('#'));
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    keys[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
  }
  return keys;
}

// The output moments TPIC names: charge density, current and the six
// pressure components (quantity index 2..7).
const char* const kMoments[8] = {"rho", "J", "PXX", "PXY", "PXZ", "PYY", "PYZ", "PZZ"};

struct MomentArray {
  std::string name;
  int quantity;  // index into kMoments
  int species;   // -1: the sum over species
};

// The snapshot channels of a run: cadences, directory and selected arrays.
struct OutputPlan {
  std::string save_dir;
  int field_cycle = 100, particles_cycle = 0;
  int gauss_cycle = 0;                 // DiagnosticGaussCycle
  int diagnostics_cycle = 100;         // DiagnosticsOutputCycle (default FieldOutputCycle; <= 0: no file)
  int restart_cycle = 0;               // RestartOutputCycle
  std::string restart_dir = "data";    // RestartDirName
  bool overwrite = false;              // replace existing output files (--overwrite-output, or a restart)
  bool e = false, b = false, gauss = false;
  std::vector<std::string> fields;     // the field arrays in tag order
  std::vector<MomentArray> moments;
  bool fields_due(long long cycle, bool final) const {
    return field_cycle > 0 && (final || cycle % field_cycle == 0);
  }
  bool particles_due(long long cycle, bool final) const {
    return particles_cycle > 0 && (final || cycle % particles_cycle == 0);
  }
  // The Gauss array selected, with a field channel to write it.
  bool output_gauss() const { return gauss && field_cycle > 0; }
  bool gauss_enabled() const { return gauss_cycle > 0 || output_gauss(); }
  // A Gauss-law sample begins at cycle n < last at the multiples of
  // DiagnosticGaussCycle and, with the Gauss array, one cycle before every
  // field snapshot and before the final state (PreparedOutput::
  // should_sample_gauss, src/config/output.cpp).
  bool gauss_begins(long long n, long long last) const {
    if (n >= last) return false;
    if (gauss_cycle > 0 && n % gauss_cycle == 0) return true;
    return output_gauss() && ((n + 1) % field_cycle == 0 || n + 1 == last);
  }
  long long next_gauss_begin(long long n, long long last) const {
    for (long long m = n + 1; m < last; ++m)
      if (gauss_begins(m, last)) return m;
    return -1;
  }
};

std::vector<std::string> tag_tokens(const std::string& tag, const char* key) {
  std::vector<std::string> out;
  if (tag.empty()) return out;
  size_t start = 0;
  while (true) {
    const size_t plus = tag.find('+', start);
    const std::string t = tag.substr(start, plus == std::string::npos ? std::string::npos : plus - start);
    if (t.empty() || t.find_first_of(" \t\r\n\f\v") != std::string::npos)
      fail(std::string(key) + ": empty or spaced token in '" + tag + "'");
    out.push_back(t);
    if (plus == std::string::npos) break;
    start = plus + 1;
  }
  return out;
}

// The plan from the deck's keys and the command line: the write methods
// (only the VTK engine is built; ADIOS2 and HDF5 are refused where their
// channel is on) and TPIC's array selection of FieldOutputTag and
// MomentsOutputTag. Both tags empty select E, B, rho, J and rho_s, J_s of
// every species. A moment token is a quantity with no suffix (every
// species), `_tot` (the sum) or a species index (ignored beyond the run's
// species); totals come first, then the species in index order, per
// quantity in TPIC's order.
OutputPlan output_plan(const std::string& text, const Args& args, int ns) {
  const std::map<std::string, std::string> k = deck_keys(text);
  auto get = [&](const char* key, const std::string& fallback) {
    const auto it = k.find(key);
    return it == k.end() ? fallback : it->second;
  };
  OutputPlan plan;
  std::string save = args.has_save_dir ? args.save_dir : get("SaveDirName", "data");
  if (save.empty()) save = "data";
  plan.save_dir = args.output + "/" + save;
  plan.field_cycle = args.has_field_cycle ? args.field_cycle : std::atoi(get("FieldOutputCycle", "100").c_str());
  plan.particles_cycle =
      args.has_particles_cycle ? args.particles_cycle : std::atoi(get("ParticlesOutputCycle", "0").c_str());
  plan.gauss_cycle = args.has_gauss_cycle ? args.gauss_cycle : std::atoi(get("DiagnosticGaussCycle", "0").c_str());
  plan.diagnostics_cycle = args.has_diagnostics_cycle
                               ? args.diagnostics_cycle
                               : std::atoi(get("DiagnosticsOutputCycle", std::to_string(plan.field_cycle)).c_str());
  plan.restart_cycle =
      args.has_restart_cycle ? args.restart_cycle : std::atoi(get("RestartOutputCycle", "0").c_str());
  plan.restart_dir = args.has_restart_dir ? args.restart_dir : get("RestartDirName", "data");
  if (plan.restart_dir.empty()) plan.restart_dir = "data";
  plan.overwrite = args.overwrite || args.restart;
  const std::string method = get("WriteMethod", "");
  const std::pair<const char*, int> channels[2] = {{"FieldWriteMethod", plan.field_cycle},
                                                   {"ParticlesWriteMethod", plan.particles_cycle}};
  for (const auto& [key, cadence] : channels) {
    std::string m = get(key, "");
    if (m.empty()) m = method;
    if (m == "vtk" || m == "pvtk" || m == "default" || m.empty()) continue;
    if (m == "adios2" || m == "bp" || m == "bp5" || m == "hdf5" || m == "h5") {
      if (cadence > 0) fail(std::string(key) + "=" + m + ": only the VTK engine is built");
      continue;
    }
    fail(std::string(key) + ": unknown write method '" + m + "'");
  }
  const std::vector<std::string> ftok = tag_tokens(get("FieldOutputTag", ""), "FieldOutputTag");
  const std::vector<std::string> mtok = tag_tokens(get("MomentsOutputTag", ""), "MomentsOutputTag");
  if (ftok.empty() && mtok.empty()) {
    plan.e = plan.b = true;
    plan.fields = {"E", "B"};
    for (int q = 0; q < 2; ++q) plan.moments.push_back({kMoments[q], q, -1});
    for (int q = 0; q < 2; ++q)
      for (int s = 0; s < ns; ++s) plan.moments.push_back({std::string(kMoments[q]) + "_" + std::to_string(s), q, s});
    return plan;
  }
  for (const std::string& t : ftok) {
    if (t == "E") plan.e = true;
    else if (t == "B") plan.b = true;
    else if (t == "Gauss") plan.gauss = true;
    else fail("FieldOutputTag: unknown token '" + t + "'");
    if (std::find(plan.fields.begin(), plan.fields.end(), t) == plan.fields.end()) plan.fields.push_back(t);
  }
  bool total[8] = {}, bare[8] = {};
  std::vector<bool> indexed(8 * size_t(ns), false);
  for (const std::string& t : mtok) {
    int q = -1;
    for (int c = 0; c < 8 && q < 0; ++c)
      if (t.compare(0, std::strlen(kMoments[c]), kMoments[c]) == 0) q = c;
    if (q < 0) fail("MomentsOutputTag: unknown token '" + t + "'");
    const std::string suffix = t.substr(std::strlen(kMoments[q]));
    if (suffix.empty()) {
      bare[q] = true;
    } else if (suffix == "_tot") {
      total[q] = true;
    } else {
      if (suffix.find_first_not_of("0123456789") != std::string::npos)
        fail("MomentsOutputTag: unknown token '" + t + "'");
      const size_t digits = suffix.find_first_not_of('0');
      const std::string value = digits == std::string::npos ? "0" : suffix.substr(digits);
      if (value.size() > 10 || std::strtoull(value.c_str(), nullptr, 10) >= (1ull << 31))
        fail("MomentsOutputTag: index out of range in '" + t + "'");
      const long long index = std::atoll(value.c_str());
      if (index < ns) indexed[8 * size_t(index) + q] = true;
    }
  }
  for (int q = 0; q < 8; ++q) {
    if (total[q]) plan.moments.push_back({kMoments[q], q, -1});
    bool any = false;
    for (int s = 0; s < ns; ++s) any = any || indexed[8 * size_t(s) + q];
    for (int s = 0; s < ns; ++s)
      if (indexed[8 * size_t(s) + q] || (bare[q] && !any))
        plan.moments.push_back({std::string(kMoments[q]) + "_" + std::to_string(s), q, s});
  }
  return plan;
}

// The precision profile name and roles written into every snapshot.
std::pair<std::string, std::string> precision_strings(bool dbl) {
  if (dbl)
    return {"double/double",
            "storage: position=float64 velocity=float64 weight=float64 E=float64 B=float64 J=float64 "
            "mass=float64 cell=int32 ID=uint64; compute: position=float64 velocity=float64 E=float64 "
            "B=float64 J=float64 mass=float64 solver-reduction=float64 reduction=float64 "
            "output-moment-accumulation=float64"};
  return {"mixed/mixed",
          "storage: position=float64 velocity=float32 weight=float64 E=float32 B=float32 J=float32 "
          "mass=float32 cell=int32 ID=uint64; compute: position=float64 velocity=float32 E=float32 "
          "B=float32 J=float32 mass=float32 solver-reduction=float64 reduction=float64 "
          "output-moment-accumulation=float64"};
}

std::string tagged(const std::string& dir, const std::string& name, long long cycle, const char* ext) {
  char num[32];
  std::snprintf(num, sizeof(num), "_t%06lld", cycle);
  return dir + "/" + name + num + ext;
}

// One node field of the state (3 components over the stored extent, nodes
// -1..n+1 per axis, FP32 or FP64) as the snapshot's nodes 0..n per axis,
// x fastest, components interleaved, FP64.
std::vector<double> snapshot_nodes(const void* field, const tpicb200_grid& g, bool dbl, cudaStream_t stream) {
  const size_t ex = g.nx + 3, ey = g.ny + 3, ez = g.nz + 3, plane = ex * ey * ez;
  std::vector<double> all(3 * plane);
  if (dbl) {
    cuda(cudaMemcpyAsync(all.data(), field, all.size() * 8, cudaMemcpyDeviceToHost, stream), "field read");
    cuda(cudaStreamSynchronize(stream), "field read");
  } else {
    std::vector<float> f(3 * plane);
    cuda(cudaMemcpyAsync(f.data(), field, f.size() * 4, cudaMemcpyDeviceToHost, stream), "field read");
    cuda(cudaStreamSynchronize(stream), "field read");
    std::copy(f.begin(), f.end(), all.begin());
  }
  const size_t nx = g.nx + 1, ny = g.ny + 1, nz = g.nz + 1;
  std::vector<double> out(3 * nx * ny * nz);
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i)
        for (size_t c = 0; c < 3; ++c)
          out[3 * (i + nx * (j + ny * k)) + c] = all[c * plane + (i + 1) + ex * ((j + 1) + ey * (k + 1))];
  return out;
}

// Unique-node values (components planes of nz*ny*nx, x fastest) onto the
// snapshot's node grid with the periodic end nodes, components interleaved.
std::vector<double> wrap_unique(const double* u, int components, size_t stride, const tpicb200_grid& g) {
  const size_t nx = g.nx + 1, ny = g.ny + 1, nz = g.nz + 1;
  std::vector<double> out(size_t(components) * nx * ny * nz);
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        const size_t src = i % g.nx + size_t(g.nx) * (j % g.ny + size_t(g.ny) * (k % g.nz));
        for (int c = 0; c < components; ++c)
          out[size_t(components) * (i + nx * (j + ny * k)) + c] = u[c * stride + src];
      }
  return out;
}

// The Gauss-law samples of a run (docs/developer/gauss_diagnostic.md): the
// cell buffers on the device (tpicb200_gauss_field / _charge) and gauss.csv.
struct GaussRun {
  bool on = false;
  double *stash = nullptr, *first = nullptr, *residual = nullptr, *sums = nullptr;
  long long cells = 0;
  long long begun = -1, finished = -1;  // begin cycle of the open / last finished sample
  bool first_set = false;
  double charge_sum = 0.0;
  std::string csv;
};

const char* kGaussHeader =
    "# TPIC Gauss-law residual v1\n"
    "# A sample begins at cycle n and finishes at n + 1: per cell r = (divC(E^n) + divC(E^{n+1}))/2 - c, where divC is\n"
    "# the solver's node-to-cell divergence and c = 4*pi times the eight-node mean of the charge density of the particles\n"
    "# at x^{n+1/2} (dual-volume scaled, zero on PEC wall nodes, smoothed like the solver's current). time = (n + 1/2)*dt.\n"
    "# Root mean squares over the global cells: residual_rms of r; drift_rms of r minus the first finished sample of the\n"
    "# run (a restart starts a new baseline); wall_residual_rms of r over the cells touching a physical wall (0 without\n"
    "# walls); charge_rms of c.\n"
    "cycle,time,residual_rms,drift_rms,wall_residual_rms,charge_rms\n";

// A double as TPIC's CSV rows print it: 17 significant digits, general format.
std::string csv_number(double v) {
  char buf[40];
  std::snprintf(buf, sizeof(buf), "%.17g", v);
  return buf;
}

// gauss.csv: the precision lines and the header; a restart keeps the rows
// below its cycle and adds its restart line.
void open_gauss_csv(const std::string& path, bool dbl, long long restart_cycle) {
  const auto [profile, roles] = precision_strings(dbl);
  const std::string head = "# precision_profile = " + profile + "\n# precision_roles = " + roles + "\n" + kGaussHeader;
  std::vector<std::string> kept;
  if (restart_cycle >= 0 && file_exists(path)) {
    std::ifstream old(path);
    std::string line;
    while (std::getline(old, line)) {
      if (!line.empty() && std::isdigit((unsigned char)line[0]) && std::atoll(line.c_str()) >= restart_cycle) continue;
      kept.push_back(line);
    }
  } else {
    std::stringstream h(head);
    std::string line;
    while (std::getline(h, line)) kept.push_back(line);
  }
  if (restart_cycle >= 0)
    kept.push_back("# restart at cycle " + std::to_string(restart_cycle) + ": precision_profile = " + profile +
                   ", precision_roles = " + roles);
  std::ofstream f(path);
  for (const std::string& line : kept) f << line << "\n";
}

// The field snapshot of the state at `cycle` (the records materialized):
// E and B at the nodes and the selected output moments, one .vti per array.
void write_fields(tpicb200_context* ctx, const tpicb200_state& st, const tpicb200_grid& g, const OutputPlan& plan,
                  int ns, bool dbl, long long cycle, double time, bool final, const GaussRun& gauss,
                  cudaStream_t stream) {
  const auto [profile, roles] = precision_strings(dbl);
  // The Gauss array: r of the sample that finished at this cycle, as cell data.
  if (plan.output_gauss() && gauss.on && gauss.finished >= 0 && gauss.finished + 1 == cycle) {
    std::vector<double> r(gauss.cells);
    cuda(cudaMemcpyAsync(r.data(), gauss.residual, r.size() * 8, cudaMemcpyDeviceToHost, stream), "Gauss read");
    cuda(cudaStreamSynchronize(stream), "Gauss read");
    check(tpicb200_vtk_write_cells(tagged(plan.save_dir, "Gauss", cycle, ".vti").c_str(), "Gauss", &g, r.data(),
                                   int(cycle), time, final ? 1 : 0, profile.c_str(), roles.c_str(),
                                   plan.overwrite ? 1 : 0),
          "Gauss snapshot");
  }
  auto put = [&](const std::string& name, const std::vector<double>& values, int components) {
    check(tpicb200_vtk_write_field(tagged(plan.save_dir, name, cycle, ".vti").c_str(), name.c_str(), components, &g,
                                   values.data(), int(cycle), time, final ? 1 : 0, profile.c_str(), roles.c_str(),
                                   plan.overwrite ? 1 : 0),
          "field snapshot");
  };
  if (plan.e) put("E", snapshot_nodes(st.e, g, dbl, stream), 3);
  if (plan.b) put("B", snapshot_nodes(st.b_node, g, dbl, stream), 3);
  if (plan.moments.empty()) return;
  // kind 0 rho (1 component), 1 J (3), 2 the pressure tensor (6); per[kind]
  // holds every species' moments and, last, their sum.
  const size_t unique = size_t(g.nx) * g.ny * g.nz;
  const int comps[3] = {1, 3, 6};
  bool needed[3] = {};
  for (const MomentArray& m : plan.moments) needed[m.quantity < 2 ? m.quantity : 2] = true;
  std::vector<double> per[3];
  double* buf = nullptr;
  cuda(cudaMalloc((void**)&buf, 6 * unique * 8), "moment buffer");
  for (int kind = 0; kind < 3; ++kind) {
    if (!needed[kind]) continue;
    const size_t n = comps[kind] * unique;
    per[kind].assign((ns + 1) * n, 0.0);
    for (int s = 0; s < ns; ++s) {
      const tpicb200_particles part = st.slot[s][st.current[s]];
      double* args[3] = {nullptr, nullptr, nullptr};
      args[kind] = buf;
      cuda(cudaMemsetAsync(buf, 0, n * 8, stream), "moment buffer");
      check(tpicb200_output_moments(ctx, st.qom[s], &part, args[0], args[1], args[2], stream), "output moments");
      cuda(cudaMemcpyAsync(per[kind].data() + s * n, buf, n * 8, cudaMemcpyDeviceToHost, stream), "moment read");
    }
    cuda(cudaStreamSynchronize(stream), "moment read");
    double* sum = per[kind].data() + ns * n;
    for (int s = 0; s < ns; ++s)
      for (size_t i = 0; i < n; ++i) sum[i] += per[kind][s * n + i];
  }
  cudaFree(buf);
  uint32_t bad = 0;
  check(tpicb200_read_invalid(ctx, &bad, 0, stream), "invalid-counter read");
  if (bad) fail("output moments: invalid records in the snapshot state");
  for (const MomentArray& m : plan.moments) {
    const int kind = m.quantity < 2 ? m.quantity : 2;
    const size_t n = comps[kind] * unique;
    const double* base = per[kind].data() + (m.species < 0 ? ns : m.species) * n;
    if (kind == 2) put(m.name, wrap_unique(base + (m.quantity - 2) * unique, 1, unique, g), 1);
    else put(m.name, wrap_unique(base, comps[kind], unique, g), comps[kind]);
  }
}

// The particle snapshot of the state at `cycle` (the records materialized,
// their ids kept): positions, velocities, charges and ids of every species.
void write_particles(tpicb200_context* ctx, const tpicb200_state& st, const OutputPlan& plan, int ns, bool dbl,
                     long long cycle, double time, bool final, cudaStream_t stream) {
  const auto [profile, roles] = precision_strings(dbl);
  std::vector<std::vector<double>> pos(ns), vel(ns), chg(ns);
  std::vector<std::vector<uint64_t>> ids(ns);
  std::vector<tpicb200_vtk_species> species(std::max(ns, 1));
  for (int s = 0; s < ns; ++s) {
    const tpicb200_particles part = st.slot[s][st.current[s]];
    const size_t n = part.count;
    pos[s].resize(3 * std::max<size_t>(n, 1));
    vel[s].resize(3 * std::max<size_t>(n, 1));
    chg[s].resize(std::max<size_t>(n, 1));
    ids[s].resize(std::max<size_t>(n, 1));
    if (n) {
      double* d = nullptr;
      cuda(cudaMalloc((void**)&d, 7 * n * 8), "particle buffer");
      check(tpicb200_output_particles(ctx, &part, d, d + 3 * n, d + 6 * n, stream), "output particles");
      cuda(cudaMemcpyAsync(pos[s].data(), d, 3 * n * 8, cudaMemcpyDeviceToHost, stream), "particle read");
      cuda(cudaMemcpyAsync(vel[s].data(), d + 3 * n, 3 * n * 8, cudaMemcpyDeviceToHost, stream), "particle read");
      cuda(cudaMemcpyAsync(chg[s].data(), d + 6 * n, n * 8, cudaMemcpyDeviceToHost, stream), "particle read");
      cuda(cudaMemcpyAsync(ids[s].data(), part.id, n * 8, cudaMemcpyDeviceToHost, stream), "particle read");
      cuda(cudaStreamSynchronize(stream), "particle read");
      cudaFree(d);
    }
    species[s] = tpicb200_vtk_species{n, pos[s].data(), vel[s].data(), chg[s].data(), ids[s].data(), uint64_t(s)};
  }
  uint32_t bad = 0;
  check(tpicb200_read_invalid(ctx, &bad, 0, stream), "invalid-counter read");
  if (bad) fail("particle output: invalid records in the snapshot state");
  check(tpicb200_vtk_write_particles(plan.save_dir.c_str(), int(cycle), time, final ? 1 : 0, profile.c_str(),
                                     roles.c_str(), ns, species.data(), plan.overwrite ? 1 : 0),
        "particle snapshot");
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
  const OutputPlan plan = output_plan(text.str(), args, deck.ns);
  if (args.mode == "check") {
    std::printf("deck %s: case %s, %dx%dx%d cells, %d species", args.deck.c_str(), deck.case_name, grid.nx, grid.ny,
                grid.nz, deck.ns);
    for (int s = 0; s < deck.ns; ++s) std::printf(" %s%u", s ? "+" : " ", count[s]);
    std::printf(" records, %lld cycles, mass form %d, %s precision\n", last, kind, args.precision.c_str());
    std::printf("snapshots under %s: fields every %d cycles (", plan.save_dir.c_str(), plan.field_cycle);
    const char* sep = "";
    for (const std::string& f : plan.fields) {
      std::printf("%s%s", sep, f.c_str());
      sep = " ";
    }
    for (const MomentArray& m : plan.moments) {
      std::printf("%s%s", sep, m.name.c_str());
      sep = " ";
    }
    std::printf("), particles every %d cycles\n", plan.particles_cycle);
    std::printf("Gauss-law samples every %d cycles%s\n", plan.gauss_cycle,
                plan.output_gauss() ? " and before each field snapshot" : "");
    std::printf("diagnostics.csv rows every %d cycles, checkpoints every %d cycles under %s/%s\n",
                plan.diagnostics_cycle, plan.restart_cycle, args.output.c_str(), plan.restart_dir.c_str());
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
  if (args.mode == "run") ::mkdir(out.c_str(), 0755);
  const std::string ckpt_dir = out + "/" + plan.restart_dir;
  // --initialize completes the startup and writes no output.
  const bool advance = args.mode == "run";
  if (advance) make_dirs(plan.save_dir);
  const std::string csv = plan.save_dir + "/diagnostics.csv";
  const bool diagnostics = plan.diagnostics_cycle > 0;
  const auto [profile, roles] = precision_strings(dbl);
  const std::string head = "# precision_profile = " + profile + "\n# precision_roles = " + roles + "\n" + kHeader +
                           columns(deck.ns);
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
    if (!diagnostics) {
    } else if (file_exists(csv)) {
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
      std::stringstream h(head);
      std::string line;
      while (std::getline(h, line)) kept.push_back(line);
    }
    if (diagnostics && advance) {
      kept.push_back("# restart at cycle " + std::to_string(cycle) + ": precision_profile = " + profile +
                     ", precision_roles = " + roles);
      std::ofstream f(csv);
      for (const std::string& line : kept) f << line << "\n";
    }
  } else {
    upload(st.e, sample_field(deck, true), !dbl);
    upload(st.b_cell, sample_field(deck, false), !dbl);
    for (int s = 0; s < deck.ns; ++s) {
      check(tpicb200_load_species(ctx, &deck, s, args.seed, 0, &st.slot[s][0], nullptr, s_), "species loading");
      if (deck.species[s].center_velocity)
        check(tpicb200_center_velocities(ctx, &deck, s, &st.slot[s][0], nullptr, s_), "velocity centring");
    }
  }
  if (last < cycle) usage("the run's last cycle lies before the checkpoint cycle");
  // A fresh run refuses output files that exist unless --overwrite-output.
  if (advance && !args.restart && !plan.overwrite)
    for (const std::string& path : {csv, plan.save_dir + "/gauss.csv"})
      if (file_exists(path) && (path == csv ? diagnostics : plan.gauss_enabled()))
        fail(path + " exists (--overwrite-output replaces it)");
  if (advance && !args.restart && diagnostics) {
    std::ofstream f(csv);
    f << head << "\n";
  }
  GaussRun gauss;
  if (advance && plan.gauss_enabled()) {
    gauss.on = true;
    gauss.cells = cells;
    gauss.stash = (double*)dev.alloc(8 * cells);
    gauss.first = (double*)dev.alloc(8 * cells);
    gauss.residual = (double*)dev.alloc(8 * cells);
    gauss.sums = (double*)dev.alloc(8 * 4);
    make_dirs(plan.save_dir);
    gauss.csv = plan.save_dir + "/gauss.csv";
    open_gauss_csv(gauss.csv, dbl, args.restart ? cycle : -1);
  }
  check(tpicb200_prepare(ctx, &st, s_), "startup");
  {
    uint32_t bad = 0;
    check(tpicb200_read_invalid(ctx, &bad, 1, s_), "invalid-counter read");
    if (bad) {
      std::fprintf(stderr, "tpicb200_run: %u nonfinite records at startup\n", bad);
      return 1;
    }
  }
  if (!advance) {
    std::printf("initialized: cycle %lld, %d species, context ready\n", cycle, deck.ns);
    cudaStreamDestroy(stream);
    check(tpicb200_destroy(ctx), "context release");
    return 0;
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
  const int cadence = diagnostics ? plan.diagnostics_cycle : 0;
  const int every = plan.restart_cycle > 0 ? plan.restart_cycle : 0;
  auto record = [&](bool final) {
    if (diagnostics) {
      std::ofstream f(csv, std::ios::app);
      f << row(cycle, deck.dt, final, field, species, deck.ns, initial) << "\n";
    }
    const double t = total_of();
    std::printf("cycle %6lld  total energy %.10e  change %+.3e\n", cycle, t, t - initial);
    std::fflush(stdout);
  };
  // At state `cycle`: finish the open sample, then begin one when due.
  auto gauss_step = [&] {
    if (!gauss.on) return;
    const bool begin = plan.gauss_begins(cycle, last), finish = gauss.begun >= 0;
    if (!begin && !finish) return;
    check(tpicb200_gauss_field(ctx, st.e, gauss.stash, gauss.first, gauss.residual, begin ? 1 : 0, finish ? 1 : 0,
                               finish && !gauss.first_set ? 1 : 0, gauss.sums, s_),
          "Gauss field");
    if (finish) {
      double sums[4];
      cuda(cudaMemcpyAsync(sums, gauss.sums, sizeof(sums), cudaMemcpyDeviceToHost, stream), "Gauss sums");
      cuda(cudaStreamSynchronize(stream), "Gauss sums");
      const double n = double(gauss.cells);
      const double rms[4] = {std::sqrt(sums[0] / n), std::sqrt(sums[1] / n), 0.0, std::sqrt(gauss.charge_sum / n)};
      for (double v : rms)
        if (!std::isfinite(v)) fail("Gauss residual: nonfinite sample");
      const double t = (double(gauss.begun) + 0.5) * deck.dt;
      std::ofstream f(gauss.csv, std::ios::app);
      f << gauss.begun << "," << csv_number(t);
      for (double v : rms) f << "," << csv_number(v);
      f << "\n";
      std::printf("  Gauss residual: cycle %lld t = %e  rms = %e  drift = %e  wall = %e  charge = %e\n",
                  gauss.begun, t, rms[0], rms[1], rms[2], rms[3]);
      std::fflush(stdout);
      gauss.first_set = true;
      gauss.finished = gauss.begun;
      gauss.begun = -1;
    }
    if (begin) {
      check(tpicb200_materialize(ctx, &st, s_), "materialize");
      tpicb200_particles live[TPICB200_MAX_SPECIES];
      for (int s = 0; s < deck.ns; ++s) live[s] = st.slot[s][st.current[s]];
      check(tpicb200_gauss_charge(ctx, deck.ns, live, gauss.stash, gauss.sums, s_), "Gauss charge");
      uint32_t bad = 0;
      check(tpicb200_read_invalid(ctx, &bad, 0, s_), "invalid-counter read");
      if (bad) fail("Gauss residual: invalid records in the sampled state");
      cuda(cudaMemcpyAsync(&gauss.charge_sum, gauss.sums + 3, 8, cudaMemcpyDeviceToHost, stream), "Gauss sums");
      cuda(cudaStreamSynchronize(stream), "Gauss sums");
      gauss.begun = cycle;
    }
  };
  auto snapshots = [&] {
    const bool final = cycle == last;
    const bool fields = plan.fields_due(cycle, final), particles = plan.particles_due(cycle, final);
    if (!fields && !particles) return;
    make_dirs(plan.save_dir);
    check(tpicb200_materialize(ctx, &st, s_), "materialize");
    if (fields)
      write_fields(ctx, st, grid, plan, deck.ns, dbl, cycle, double(cycle) * deck.dt, final, gauss, stream);
    if (particles) write_particles(ctx, st, plan, deck.ns, dbl, cycle, double(cycle) * deck.dt, final, stream);
  };
  if ((cadence && cycle % cadence == 0) || cycle == last) record(cycle == last);
  gauss_step();
  snapshots();
  std::vector<tpicb200_cycle_report> reports;
  while (cycle < last) {
    long long stop = last;
    if (cadence) stop = std::min(stop, (cycle / cadence + 1) * cadence);
    if (every) stop = std::min(stop, (cycle / every + 1) * every);
    for (const int channel : {plan.field_cycle, plan.particles_cycle})
      if (channel > 0) stop = std::min(stop, (cycle / channel + 1) * channel);
    if (gauss.on) {
      if (gauss.begun >= 0) stop = std::min(stop, gauss.begun + 1);
      const long long next = plan.next_gauss_begin(cycle, last);
      if (next >= 0) stop = std::min(stop, next);
    }
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
    gauss_step();
    snapshots();
    if (!std::isfinite(field[0]) || !std::isfinite(field[1])) {
      std::fprintf(stderr, "tpicb200_run: nonfinite field energy\n");
      return 1;
    }
  }
  cudaStreamDestroy(stream);
  check(tpicb200_destroy(ctx), "context release");
  return 0;
}
