// Input decks and analytic initial cases (host code).
//
// The deck reader keeps TPIC's rules (src/config/simulation_parameters.cpp:55-200):
// one `key = value` per line, '#' starts a comment, the last assignment of a
// key wins, a list holds whitespace-separated values of which the first ns
// are used, a boolean is 0, 1, true or false, and a number is read in full.
// It reads the keys of the periodic, one-rank cycle (smoothing included) and of the
// cases built here; it counts the other keys and ignores them.
//
// The cases restate TPIC's analytic startup fields and loading profiles:
//   Uniform    no seed (cases/uniform.hpp);
//   Weibel     B_z = A cos(k x), E_y = -(g/k) A sin(k x)
//              (src/initialization/cases/weibel.cpp:9-40);
//   TwoStream  E_x = -(n_e a / k) sin(k x + phase), electron densities
//              times 1 + a cos(k x + phase) (src/initialization/cases/two_stream.cpp:16-75,
//              cases/two_stream.hpp:14-24);
//   Harris     B_x = B_H tanh((y - Ly/2)/delta) (or the double sheet),
//              a box-scale mode and a Gaussian hump of the out-of-plane
//              potential (src/initialization/cases/harris_sheet.cpp:15-256),
//              sech^2 density of drifting species averaged over the cell's
//              two y nodes (cases/harris_sheet.hpp:68-106).
// Every expression keeps the reference's operation order, so the fields are
// bit-identical to TPIC's on the same host math library.
#include "cases.cuh"
#include "kernels.cuh"

#include <cmath>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace tpicb200 {
namespace {

constexpr double kPi = 3.1415926535897932384626433832795;
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kFourPi = 12.566370614359172953850573533118;

struct DeckError {
  std::string message;
};

std::string trimmed(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  const size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// One value read in full.
bool parse_token(const std::string& text, double& out) {
  std::istringstream in(text);
  in >> out;
  return !in.fail() && (in >> std::ws).eof();
}
bool parse_token(const std::string& text, int& out) {
  std::istringstream in(text);
  in >> out;
  return !in.fail() && (in >> std::ws).eof();
}
bool parse_token(const std::string& text, bool& out) {
  out = text == "1" || text == "true";
  return out || text == "0" || text == "false";
}
bool parse_token(const std::string& text, std::string& out) {
  out = text;
  return true;
}

class Deck {
 public:
  explicit Deck(const char* text) {
    std::istringstream in(text);
    std::string line;
    for (int number = 1; std::getline(in, line); ++number) {
      const std::string content = trimmed(line.substr(0, line.find('#')));
      if (content.empty()) continue;
      const size_t eq = content.find('=');
      const std::string key = trimmed(content.substr(0, eq));
      if (eq == std::string::npos || key.empty())
        throw DeckError{"line " + std::to_string(number) + ": expected 'key = value'"};
      entries_[key] = Entry{trimmed(content.substr(eq + 1)), number, false};
    }
  }
  template <class T> void read_into(const std::string& key, T& target) {
    if (Entry* e = find(key)) target = parse<T>(key, *e);
  }
  template <class T> T required(const std::string& key) {
    Entry* e = find(key);
    if (!e) throw DeckError{"missing required key " + key};
    return parse<T>(key, *e);
  }
  std::string text(const std::string& key) {
    Entry* e = find(key);
    return e ? e->value : std::string();
  }
  bool has(const std::string& key) { return find(key) != nullptr; }
  template <class T> std::vector<T> list(const std::string& key, size_t needed) {
    Entry* e = find(key);
    if (!e) {
      if (needed) throw DeckError{"missing required key " + key};
      return {};
    }
    std::vector<T> values;
    std::istringstream in(e->value);
    for (std::string token; in >> token;) {
      T v{};
      if (!parse_token(token, v))
        throw DeckError{at(*e) + key + " = '" + e->value + "': '" + token + "' is not a valid value"};
      values.push_back(v);
    }
    if (values.size() < needed)
      throw DeckError{at(*e) + key + " lists " + std::to_string(values.size()) + " values, expected at least " +
                      std::to_string(needed)};
    return values;
  }
  int unread() const {
    int n = 0;
    for (const auto& kv : entries_) n += kv.second.read ? 0 : 1;
    return n;
  }

 private:
  struct Entry {
    std::string value;
    int line = 0;
    bool read = false;
  };
  Entry* find(const std::string& key) {
    auto it = entries_.find(key);
    if (it == entries_.end()) return nullptr;
    it->second.read = true;
    return &it->second;
  }
  static std::string at(const Entry& e) { return "line " + std::to_string(e.line) + ": "; }
  template <class T> static T parse(const std::string& key, const Entry& e) {
    T v{};
    if (!parse_token(e.value, v)) throw DeckError{at(e) + key + " = '" + e.value + "' is not a valid value"};
    return v;
  }
  std::map<std::string, Entry> entries_;
};

const char* const kCases[] = {"Uniform", "Weibel", "TwoStream", "GEMHarris", "GEM",
                              "GEMnoPert", "DoubleGEM", "DoubleGEMnoPert", "plasmoidChain"};

bool is_harris(const std::string& name) {
  return name == "GEMHarris" || name == "GEM" || name == "GEMnoPert" || name == "DoubleGEM" ||
         name == "DoubleGEMnoPert" || name == "plasmoidChain";
}

// 2 pi mode / length (initial_case.cpp:59-63).
double mode_wavenumber(int mode, double length) {
  const double k = kTwoPi * static_cast<double>(mode) / length;
  if (!std::isfinite(k) || (mode != 0 && k == 0.0)) throw DeckError{"seed wavenumber is not representable"};
  return k;
}

bool nearly_equal(double a, double b) {
  return std::abs(a - b) <= 1.0e-10 * std::max(1.0, std::max(std::abs(a), std::abs(b)));
}

void require(bool condition, const char* message) {
  if (!condition) throw DeckError{message};
}

// The seed of a Harris sheet (harris_sheet.hpp:13-22): a box-scale mode and
// a Gaussian hump of the out-of-plane potential.
struct HarrisSeed {
  double mode_amplitude = 0, mode_kx = 0, mode_ky = 0;
  double amplitude_x = 0, amplitude_y = 0, width_x = 0, width_y = 0, period_x = 0, period_y = 0;
  double slope_period_x = 0, slope_period_y = 0;
  bool hump() const { return amplitude_x != 0.0 || amplitude_y != 0.0; }
};

// The coefficients prepare_initial_case derives from the deck.
struct Prepared {
  std::string name;
  double wavenumber = 0.0, electric_amplitude = 0.0;  // Weibel, TwoStream
  bool is_double = false;                              // Harris
  HarrisSeed seed;
  bool harris_density[TPICB200_MAX_SPECIES] = {};
  bool density_seed[TPICB200_MAX_SPECIES] = {};        // TwoStream electrons
};

Prepared prepare(const tpicb200_deck& d) {
  Prepared p;
  p.name = std::string(d.case_name, strnlen(d.case_name, TPICB200_CASE_NAME_MAX));
  bool known = false;
  for (const char* c : kCases) known = known || p.name == c;
  if (!known) throw DeckError{"case '" + p.name + "' is not built here"};
  require(d.ns >= 1 && d.ns <= TPICB200_MAX_SPECIES, "ns must be between 1 and 8");
  if (p.name == "Weibel") {
    require(std::isfinite(d.weibel_amplitude) && std::isfinite(d.weibel_growth_rate),
            "WeibelSeedAmplitude and WeibelSeedGrowthRate must be finite");
    require(d.weibel_mode_x >= 0, "WeibelSeedModeX must be non-negative");
    require(d.weibel_amplitude == 0.0 || d.weibel_mode_x > 0,
            "WeibelSeedModeX must be positive for nonzero seed amplitude");
    p.wavenumber = mode_wavenumber(d.weibel_mode_x, d.grid.lx);
    if (d.weibel_amplitude != 0.0) p.electric_amplitude = -(d.weibel_growth_rate / p.wavenumber) * d.weibel_amplitude;
  } else if (p.name == "TwoStream") {
    require(d.two_stream_mode_x >= 0, "TwoStreamSeedModeX must be non-negative");
    require(d.two_stream_mode_x == 0 || 2LL * d.two_stream_mode_x < d.grid.nx,
            "TwoStreamSeedModeX must be below the x-grid Nyquist mode");
    require(std::isfinite(d.two_stream_amplitude) && std::isfinite(d.two_stream_phase),
            "TwoStreamSeedDensityAmplitude and TwoStreamSeedPhase must be finite");
    require(std::abs(d.two_stream_amplitude) < 1.0, "abs(TwoStreamSeedDensityAmplitude) must be less than one");
    require(d.two_stream_amplitude == 0.0 || d.two_stream_mode_x > 0,
            "TwoStreamSeedModeX must be positive for nonzero seed amplitude");
    std::vector<int> electrons;
    int ion = -1;
    for (int s = 0; s < d.ns; ++s) {
      require(d.species[s].rho > 0.0, "TwoStream species rhoINIT must be positive");
      if (d.species[s].qom < 0.0) electrons.push_back(s);
      else ion = s;
    }
    require(d.ns == 3 && electrons.size() == 2 && ion >= 0,
            "TwoStream requires exactly two electron species and one ion species");
    const tpicb200_deck_species& a = d.species[electrons[0]];
    const tpicb200_deck_species& b = d.species[electrons[1]];
    require(nearly_equal(a.rho, b.rho) && nearly_equal(a.qom, b.qom), "TwoStream electron rhoINIT and qom must match");
    require(nearly_equal(a.vth[0], b.vth[0]) && nearly_equal(a.vth[1], b.vth[1]) && nearly_equal(a.vth[2], b.vth[2]),
            "TwoStream electron thermal velocities must match");
    require(a.drift[0] != 0.0 && nearly_equal(a.drift[0], -b.drift[0]),
            "TwoStream electron u0 must be equal and opposite and nonzero");
    const double electron_density = a.rho + b.rho;
    require(nearly_equal(electron_density, d.species[ion].rho),
            "TwoStream ion rhoINIT must equal the sum of electron rhoINIT");
    require(nearly_equal(d.species[ion].drift[0], 0.0), "TwoStream ion drift must be zero");
    for (int s = 0; s < d.ns; ++s) {
      const tpicb200_deck_species& sp = d.species[s];
      require(nearly_equal(sp.drift[1], 0.0) && nearly_equal(sp.drift[2], 0.0), "TwoStream transverse drifts must be zero");
      require(sp.npcel[0] == a.npcel[0] && sp.npcel[1] == a.npcel[1] && sp.npcel[2] == a.npcel[2],
              "TwoStream requires identical particles-per-cell dimensions");
    }
    p.wavenumber = mode_wavenumber(d.two_stream_mode_x, d.grid.lx);
    if (d.two_stream_amplitude != 0.0) {
      p.electric_amplitude = -(electron_density * d.two_stream_amplitude / p.wavenumber);
      require(std::isfinite(p.electric_amplitude), "TwoStream E amplitude is not representable");
    }
    for (int s = 0; s < d.ns; ++s) p.density_seed[s] = d.species[s].qom < 0.0 && d.two_stream_amplitude != 0.0;
  } else if (is_harris(p.name)) {
    require(std::isfinite(d.harris_b0x), "HarrisB0x must be finite");
    require(std::isfinite(d.delta) && d.delta > 0.0, "Harris delta must be finite and positive");
    p.is_double = p.name == "DoubleGEM" || p.name == "DoubleGEMnoPert";
    if (p.name == "GEMHarris") {
      // The seed the GEMHarris keys describe (harris_sheet.cpp:15-45).
      require(std::isfinite(d.pert_gem) && std::isfinite(d.pert_hump) && std::isfinite(d.kx_hump) &&
                  std::isfinite(d.ky_hump),
              "pertGEM, pertHump, kxHump and kyHump must be finite");
      require(std::isfinite(d.deltax_hump) && d.deltax_hump > 0.0 && std::isfinite(d.deltay_hump) &&
                  d.deltay_hump > 0.0,
              "GEMHarris deltaxHump and deltayHump must be finite and positive");
      HarrisSeed& s = p.seed;
      s.mode_amplitude = d.pert_gem;
      s.mode_kx = mode_wavenumber(1, d.grid.lx);
      s.mode_ky = mode_wavenumber(1, d.grid.ly);
      if (d.pert_hump != 0.0) {
        const double kx = d.kx_hump < 0.0 ? kTwoPi / d.grid.lx : d.kx_hump;
        const double ky = d.ky_hump < 0.0 ? .5 * kTwoPi / d.grid.ly : d.ky_hump;
        require(ky != 0.0, "GEMHarris kyHump must be nonzero");
        s.width_x = d.deltax_hump * d.delta;
        s.width_y = d.deltay_hump * d.delta;
        s.amplitude_x = d.pert_hump / (ky * s.width_y);
        s.amplitude_y = d.pert_hump / (ky * s.width_x);
        s.period_x = kPi / (kx * d.delta);
        s.period_y = kPi / (ky * d.delta);
        s.slope_period_x = kPi / (kx * s.width_x);
        s.slope_period_y = kPi / (ky * s.width_y);
      }
    } else if (p.name == "GEM" || p.name == "DoubleGEM") {
      p.seed = HarrisSeed{0.0, 0.0, 0.0, 0.4, 0.4, d.delta, d.delta, 10.0, 10.0, 10.0, 10.0};
    }
    bool electron_seen = false, ion_seen = false;
    for (int s = 0; s < d.ns; ++s) {
      const tpicb200_deck_species& sp = d.species[s];
      if (p.name == "plasmoidChain") {
        bool& seen = sp.qom < 0.0 ? electron_seen : ion_seen;
        p.harris_density[s] = !seen;
        seen = true;
      } else {
        p.harris_density[s] =
            std::abs(sp.drift[0]) > 1.0e-10 || std::abs(sp.drift[1]) > 1.0e-10 || std::abs(sp.drift[2]) > 1.0e-10;
      }
    }
  }
  return p;
}

// The hump of one sheet (harris_sheet.cpp:113-130), in the reference's order.
void add_hump(const HarrisSeed& seed, double x, double y, double center_x, double center_y, double delta,
              double sheet_b0x, double sign, double b[3]) {
  const double xpert = x - center_x;
  const double ypert = y - center_y;
  const double envelope =
      std::exp(-(xpert / seed.width_x) * (xpert / seed.width_x) - (ypert / seed.width_y) * (ypert / seed.width_y));
  const double cos_x = std::cos(kPi * xpert / seed.period_x / delta);
  const double sin_x = std::sin(kPi * xpert / seed.period_x / delta);
  const double cos_y = std::cos(kPi * ypert / seed.period_y / delta);
  const double sin_y = std::sin(kPi * ypert / seed.period_y / delta);
  b[0] += sign * sheet_b0x * seed.amplitude_x * envelope *
          (-cos_x * cos_y * 2.0 * ypert / seed.width_y - cos_x * sin_y * kPi / seed.slope_period_y);
  b[1] += sign * sheet_b0x * seed.amplitude_y * envelope *
          (cos_x * cos_y * 2.0 * xpert / seed.width_x + sin_x * cos_y * kPi / seed.slope_period_x);
}

void case_magnetic(const tpicb200_deck& d, const Prepared& p, double x, double y, double b[3]) {
  b[0] = b[1] = b[2] = 0.0;
  if (p.name == "Weibel") {
    if (d.weibel_amplitude != 0.0) b[2] = d.weibel_amplitude * std::cos(p.wavenumber * x);
  } else if (is_harris(p.name)) {
    const double lx = d.grid.lx, ly = d.grid.ly;
    if (p.is_double) {
      const double bottom = (y - 0.25 * ly) / d.delta;
      const double top = (y - 0.75 * ly) / d.delta;
      b[0] = d.harris_b0x * (-1.0 + std::tanh(bottom) - std::tanh(top));
    } else {
      b[0] = d.harris_b0x * std::tanh((y - 0.5 * ly) / d.delta);
    }
    const HarrisSeed& s = p.seed;
    if (s.mode_amplitude != 0.0) {
      const double xm = x - 0.5 * lx;
      const double ym = y - 0.5 * ly;
      b[0] += -s.mode_amplitude * d.harris_b0x * (lx / ly) * std::cos(s.mode_kx * xm) * std::sin(s.mode_ky * ym);
      b[1] += s.mode_amplitude * d.harris_b0x * std::sin(s.mode_kx * xm) * std::cos(s.mode_ky * ym);
    }
    if (s.hump()) {
      if (p.is_double) {
        add_hump(s, x, y, 0.25 * lx, 0.25 * ly, d.delta, d.harris_b0x, 1.0, b);
        add_hump(s, x, y, 0.75 * lx, 0.75 * ly, d.delta, d.harris_b0x, -1.0, b);
      } else {
        add_hump(s, x, y, 0.5 * lx, 0.5 * ly, d.delta, d.harris_b0x, 1.0, b);
      }
    }
  }
  b[0] += d.b0[0];
  b[1] += d.b0[1];
  b[2] += d.b0[2];
}

void case_electric(const tpicb200_deck& d, const Prepared& p, double x, double e[3]) {
  e[0] = e[1] = e[2] = 0.0;
  if (p.name == "Weibel") {
    if (d.weibel_amplitude != 0.0 && d.weibel_growth_rate != 0.0) e[1] = p.electric_amplitude * std::sin(p.wavenumber * x);
  } else if (p.name == "TwoStream") {
    if (d.two_stream_amplitude != 0.0)
      e[0] = p.electric_amplitude * std::sin(p.wavenumber * x + d.two_stream_phase);
  }
}

int deck_failure(const DeckError& e) { return report_error(TPICB200_INVALID_ARGUMENT, e.message); }

CaseProfile profile_of(const tpicb200_deck& d, const Prepared& p, int s) {
  const tpicb200_deck_species& sp = d.species[s];
  CaseProfile c{};
  c.density = sp.rho / kFourPi;
  for (int a = 0; a < 3; ++a) c.drift[a] = sp.drift[a];
  c.density_seed = p.density_seed[s] ? 1 : 0;
  c.wavenumber = p.wavenumber;
  c.amplitude = d.two_stream_amplitude;
  c.phase = d.two_stream_phase;
  c.harris_density = is_harris(p.name) && p.harris_density[s] ? 1 : 0;
  c.is_double = p.is_double ? 1 : 0;
  c.ly = d.grid.ly;
  c.delta = d.delta;
  c.dy = d.grid.ly / d.grid.ny;
  return c;
}

}  // namespace

int case_profile_of(const tpicb200_deck* deck, int s, CaseProfile* out) {
  if (!deck || !out || s < 0 || s >= deck->ns || s >= TPICB200_MAX_SPECIES)
    return report_error(TPICB200_INVALID_ARGUMENT, "invalid deck or species index");
  try {
    *out = profile_of(*deck, prepare(*deck), s);
    return TPICB200_SUCCESS;
  } catch (const DeckError& err) {
    return deck_failure(err);
  }
}

}  // namespace tpicb200

using namespace tpicb200;

extern "C" int tpicb200_deck_parse(const char* text, tpicb200_deck* out) {
  if (!text || !out) return report_error(TPICB200_INVALID_ARGUMENT, "null deck text or output");
  try {
    Deck cfg(text);
    tpicb200_deck d{};
    d.dt = cfg.required<double>("dt");
    d.ncycles = cfg.required<int>("ncycles");
    d.theta = 1.0;
    cfg.read_into("th", d.theta);
    // Energy-conserving smoothing (config/physics.cpp:65-70; on when
    // SmoothNiter > 0 and Smooth < 1).
    const std::string smoothing = cfg.text("ECSimSmoothing");
    if (!smoothing.empty() && smoothing != "none" && smoothing != "energy_conserving")
      throw DeckError{"ECSimSmoothing = " + smoothing + " (none or energy_conserving)"};
    double smooth = 1.0;
    int smooth_niter = 6;
    cfg.read_into("Smooth", smooth);
    cfg.read_into("SmoothNiter", smooth_niter);
    const std::string op = cfg.text("ECSimSmoothingOperator");
    if (!op.empty() && op != "face7" && op != "binomial27")
      throw DeckError{"ECSimSmoothingOperator = " + op + " (face7 or binomial27)"};
    d.smooth_iterations = 0;
    d.smooth_alpha = 1.0;
    d.smooth_operator = TPICB200_SMOOTH_FACE7;
    if (smoothing == "energy_conserving") {
      if (!std::isfinite(smooth) || smooth < 0 || smooth > 1)
        throw DeckError{"energy-conserving smoothing requires 0 <= Smooth <= 1"};
      if (smooth_niter < 0) throw DeckError{"energy-conserving smoothing requires SmoothNiter >= 0"};
      if (smooth_niter > 0 && smooth < 1) {
        d.smooth_iterations = smooth_niter;
        d.smooth_alpha = smooth;
        d.smooth_operator = op == "binomial27" ? TPICB200_SMOOTH_BINOMIAL27 : TPICB200_SMOOTH_FACE7;
      }
    }
    d.ns = cfg.required<int>("ns");
    if (d.ns < 1 || d.ns > TPICB200_MAX_SPECIES) throw DeckError{"ns must be between 1 and 8"};
    int test_species = 0;
    cfg.read_into("nsTestPart", test_species);
    if (test_species != 0) throw DeckError{"test particles (nsTestPart) are not built here"};
    const size_t ns = size_t(d.ns);
    const auto rho = cfg.list<double>("rhoINIT", ns);
    const auto qom = cfg.list<double>("qom", ns);
    const auto npx = cfg.list<int>("npcelx", ns), npy = cfg.list<int>("npcely", ns), npz = cfg.list<int>("npcelz", ns);
    const auto uth = cfg.list<double>("uth", ns), vth = cfg.list<double>("vth", ns), wth = cfg.list<double>("wth", ns);
    const auto u0 = cfg.list<double>("u0", ns), v0 = cfg.list<double>("v0", ns), w0 = cfg.list<double>("w0", ns);
    const auto center = cfg.list<bool>("CenterInitialVelocity", 0);
    for (size_t s = 0; s < ns; ++s) {
      tpicb200_deck_species& sp = d.species[s];
      sp.rho = rho[s];
      sp.qom = qom[s];
      sp.npcel[0] = npx[s]; sp.npcel[1] = npy[s]; sp.npcel[2] = npz[s];
      sp.vth[0] = uth[s]; sp.vth[1] = vth[s]; sp.vth[2] = wth[s];
      sp.drift[0] = u0[s]; sp.drift[1] = v0[s]; sp.drift[2] = w0[s];
      sp.center_velocity = s < center.size() && center[s] ? 1 : 0;
      if (sp.npcel[0] < 1 || sp.npcel[1] < 1 || sp.npcel[2] < 1)
        throw DeckError{"npcelx, npcely and npcelz must be positive"};
    }
    cfg.read_into("B0x", d.b0[0]);
    cfg.read_into("B0y", d.b0[1]);
    cfg.read_into("B0z", d.b0[2]);
    d.delta = 0.5;
    d.deltax_hump = 8.0;
    d.deltay_hump = 4.0;
    d.kx_hump = -1.0;
    d.ky_hump = -1.0;
    cfg.read_into("delta", d.delta);
    cfg.read_into("HarrisB0x", d.harris_b0x);
    cfg.read_into("pertGEM", d.pert_gem);
    cfg.read_into("pertHump", d.pert_hump);
    cfg.read_into("deltaxHump", d.deltax_hump);
    cfg.read_into("deltayHump", d.deltay_hump);
    cfg.read_into("kxHump", d.kx_hump);
    cfg.read_into("kyHump", d.ky_hump);
    bool ampere = false;
    cfg.read_into("currentFromAmpere", ampere);
    if (ampere) throw DeckError{"currentFromAmpere is not built here"};
    bool varying = false;
    cfg.read_into("spatiallyVaryingThermal", varying);
    cfg.read_into("WeibelSeedModeX", d.weibel_mode_x);
    cfg.read_into("WeibelSeedAmplitude", d.weibel_amplitude);
    cfg.read_into("WeibelSeedGrowthRate", d.weibel_growth_rate);
    cfg.read_into("TwoStreamSeedModeX", d.two_stream_mode_x);
    cfg.read_into("TwoStreamSeedDensityAmplitude", d.two_stream_amplitude);
    cfg.read_into("TwoStreamSeedPhase", d.two_stream_phase);
    d.c = 1.0;
    cfg.read_into("c", d.c);
    d.grid = tpicb200_grid{64, 64, 64, 10.0, 10.0, 10.0};
    cfg.read_into("Lx", d.grid.lx);
    cfg.read_into("Ly", d.grid.ly);
    cfg.read_into("Lz", d.grid.lz);
    cfg.read_into("nxc", d.grid.nx);
    cfg.read_into("nyc", d.grid.ny);
    cfg.read_into("nzc", d.grid.nz);
    // XLEN/YLEN/ZLEN (the rank decomposition) are not read: the whole
    // domain is one rank's here, and a decomposed run is the same physics.
    for (const char* key : {"PERIODICX", "PERIODICY", "PERIODICZ", "PERIODICX_P", "PERIODICY_P", "PERIODICZ_P"}) {
      bool periodic = true;
      cfg.read_into(key, periodic);
      if (!periodic) throw DeckError{std::string(key) + " = false: wall boundaries are not built here"};
    }
    const std::string name = cfg.required<std::string>("Case");
    bool known = false;
    for (const char* c : kCases) known = known || name == c;
    if (!known) throw DeckError{"Case = " + name + " is not built here"};
    if (name.size() >= TPICB200_CASE_NAME_MAX) throw DeckError{"case name too long"};
    std::memcpy(d.case_name, name.c_str(), name.size() + 1);
    bool quiet = false;
    cfg.read_into("QuietStart", quiet);
    d.quiet_start = quiet ? 1 : 0;
    d.gmres_tol = 1e-3;
    cfg.read_into("GMREStol", d.gmres_tol);
    if (!(d.dt > 0.0) || !std::isfinite(d.dt)) throw DeckError{"dt must be positive and finite"};
    if (d.grid.nx < 1 || d.grid.ny < 1 || d.grid.nz < 1 || !(d.grid.lx > 0.0) || !(d.grid.ly > 0.0) ||
        !(d.grid.lz > 0.0))
      throw DeckError{"the grid needs positive cell counts and lengths"};
    (void)prepare(d);  // case admission
    d.ignored_keys = cfg.unread();
    *out = d;
    return TPICB200_SUCCESS;
  } catch (const DeckError& e) {
    return deck_failure(e);
  }
}

extern "C" int tpicb200_case_fields(const tpicb200_deck* deck, long long n, const double* x, const double* y,
                                    const double* z, double* e, double* b) {
  if (!deck || n < 0 || (n > 0 && (!x || !y || !z || !e || !b)))
    return report_error(TPICB200_INVALID_ARGUMENT, "invalid case-field arguments");
  try {
    const Prepared p = prepare(*deck);
    for (long long i = 0; i < n; ++i) {
      if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(z[i]))
        return report_error(TPICB200_OVERFLOW, "case field sample at a nonfinite coordinate");
      double ev[3], bv[3];
      case_electric(*deck, p, x[i], ev);
      case_magnetic(*deck, p, x[i], y[i], bv);
      for (int c = 0; c < 3; ++c) {
        if (!std::isfinite(ev[c]) || !std::isfinite(bv[c]))
          return report_error(TPICB200_OVERFLOW, "case field sample is not finite");
        e[c * n + i] = ev[c];
        b[c * n + i] = bv[c];
      }
    }
    return TPICB200_SUCCESS;
  } catch (const DeckError& err) {
    return deck_failure(err);
  }
}

extern "C" int tpicb200_case_profile(const tpicb200_deck* deck, int s, long long n, const double* x, const double* y,
                                     const double* z, const int* cell_j, double* density, double* multiplier,
                                     double* drift) {
  if (!deck || s < 0 || s >= deck->ns || n < 0 ||
      (n > 0 && (!x || !y || !z || !cell_j || !density || !multiplier || !drift)))
    return report_error(TPICB200_INVALID_ARGUMENT, "invalid case-profile arguments");
  try {
    const Prepared p = prepare(*deck);
    const CaseProfile c = profile_of(*deck, p, s);
    for (long long i = 0; i < n; ++i) {
      double v[3];
      c.evaluate(x[i], y[i], cell_j[i], density[i], multiplier[i], v);
      for (int a = 0; a < 3; ++a) drift[a * n + i] = v[a];
    }
    return TPICB200_SUCCESS;
  } catch (const DeckError& err) {
    return deck_failure(err);
  }
}
