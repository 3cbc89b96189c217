// One species' loading profile of an analytic case, evaluated on the host
// (tpicb200_case_profile) and in the loading kernels from the same source.
//
// TPIC's profiles (include/tpic/initialization/cases/two_stream.hpp:14-24,
// cases/harris_sheet.hpp:68-106): the density starts at rhoINIT/(4 pi) and the
// drift at the deck's (u0, v0, w0);
//   TwoStream electrons: multiplier 1 + a cos(k x + phase);
//   Harris drifting species: density * 0.5 * (shape(y_j) + shape(y_j + dy)),
//     the sech^2 sheet shape at the two y nodes of the particle's cell;
//   double sheet: drift_z * -tanh((y - Ly/2)/delta).
// The charge of a loaded particle is (q_factor * density) * multiplier.
#pragma once

#include <cmath>

namespace tpicb200 {

struct CaseProfile {
  double density;        // rhoINIT / (4 pi)
  double drift[3];       // u0, v0, w0
  int density_seed;      // TwoStream electron density seed
  double wavenumber, amplitude, phase;
  int harris_density;    // sech^2 density of the cell's two y nodes
  int is_double;         // two sheets (at Ly/4 and 3Ly/4)
  double ly, delta, dy;

  __host__ __device__ static double sech_squared(double v) {
    const double ch = cosh(v);
    return 1.0 / (ch * ch);
  }
  __host__ __device__ double sheet_shape(double y) const {
    if (is_double) return sech_squared((y - 0.25 * ly) / delta) + sech_squared((y - 0.75 * ly) / delta);
    return sech_squared((y - 0.5 * ly) / delta);
  }
  // Drift at a physical y (the only coordinate a drift depends on).
  __host__ __device__ void drift_at(double y, double out[3]) const {
    out[0] = drift[0];
    out[1] = drift[1];
    out[2] = drift[2];
    if (is_double) out[2] = out[2] * -tanh((y - 0.5 * ly) / delta);
  }
  // Density, multiplier and drift of a particle at physical (x, y) in a cell
  // whose y index is cell_j (the grid origin is 0).
  __host__ __device__ void evaluate(double x, double y, int cell_j, double& dens, double& mult,
                                    double out_drift[3]) const {
    dens = density;
    mult = 1.0;
    if (density_seed) mult = 1.0 + amplitude * cos(wavenumber * x + phase);
    if (harris_density) {
      const double lower_y = 0.0 + cell_j * dy;
      const double nodes = sheet_shape(lower_y) + sheet_shape(lower_y + dy);
      dens = dens * 0.5 * nodes;
    }
    drift_at(y, out_drift);
  }
};

}  // namespace tpicb200
