// Snapshot output: the output moments of a species on the device, records
// converted to output coordinates on the device, and the VTK XML files of
// TPIC's default engine written on the host.
//
// Output moments (diagnostics/output_moment_deposition_device.hpp:30-107):
// per record the amounts q/V (rho), q/V v (J) and (q/V)(1/qom) v_i v_j (P),
// in FP64, times each nonzero CIC weight, added at the record's cell corners;
// the snapshot writes 4 pi rho (docs/user/output.md, "Moments"). On a fully
// periodic grid the shared-node addition is the corner's wrap onto its
// unique node and the dual volume is the cell volume.
//
// VTK files (src/io/vtk_field_engine.cpp, src/io/vtk_particle_engine.cpp,
// io/detail/vtk_output.hpp): version-1.0 XML with UInt64 headers and raw
// appended data. A field file is Float64 ImageData over the (nx+1)(ny+1)(nz+1)
// node grid, end nodes included, x fastest, components interleaved; a
// particle snapshot is one PolyData piece with the velocity, charge, id and
// species point arrays, the position points and one vertex per point, listed
// by a PPolyData manifest. FieldData carries TimeValue, cycle, final_state
// and the state and precision strings.
#include "kernels.cuh"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <sys/stat.h>

namespace tpicb200 {
namespace {

constexpr double kFourPi = 4.0 * 3.14159265358979323846;

// The output moments of one species (rho scaled by rho_scale: 4 pi for the
// snapshot, 1 for the Gauss-law charge). A record's amounts are checked only
// where they are requested: rho always, J and P when their buffers are given
// (a velocity enters only those).
template <class V>
__global__ void __launch_bounds__(256) output_moments_kernel(Geom g, tpicb200_particles p, double inverse_volume,
                                                           double inverse_qom, double rho_scale,
                                                           double* __restrict__ rho, double* __restrict__ j,
                                                           double* __restrict__ pressure, uint32_t* invalid) {
  const long long unique = (long long)g.nx * g.ny * g.nz;
  const V* u = (const V*)p.u;
  const V* v = (const V*)p.v;
  const V* w = (const V*)p.w;
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < p.count; n += gridDim.x * blockDim.x) {
    const int32_t key = p.cell[n];
    int ci, cj, ck;
    bool ok = key >= 0 && (long long)key < g.bins;
    if (ok) {
      g.decode(key, ci, cj, ck);
      ok = g.interior_cell(ci, cj, ck);
    }
    const double fx = ((const double*)p.rx)[n], fy = ((const double*)p.ry)[n], fz = ((const double*)p.rz)[n];
    ok = ok && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1;
    if (!ok) {
      atomicAdd(invalid, 1u);
      continue;
    }
    const double charge = p.q[n] * inverse_volume;
    const double vx = double(u[n]), vy = double(v[n]), vz = double(w[n]);
    double amount[10];
    amount[0] = charge * rho_scale;
    amount[1] = charge * vx;
    amount[2] = charge * vy;
    amount[3] = charge * vz;
    const double mass = charge * inverse_qom;
    amount[4] = mass * vx * vx;
    amount[5] = mass * vx * vy;
    amount[6] = mass * vx * vz;
    amount[7] = mass * vy * vy;
    amount[8] = mass * vy * vz;
    amount[9] = mass * vz * vz;
    bool finite = isfinite(amount[0]);
#pragma unroll
    for (int c = 1; c < 4; ++c) finite = finite && (!j || isfinite(amount[c]));
#pragma unroll
    for (int c = 4; c < 10; ++c) finite = finite && (!pressure || isfinite(amount[c]));
    if (!finite) {
      atomicAdd(invalid, 1u);
      continue;
    }
    double wt[8];
    cic_weights<double>(fx, fy, fz, wt);
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      if (wt[a] == 0.0) continue;
      const int i = wrap_index(ci + (a & 1), g.nx), jj = wrap_index(cj + ((a >> 1) & 1), g.ny),
                k = wrap_index(ck + ((a >> 2) & 1), g.nz);
      const long long node = i + (long long)g.nx * (jj + (long long)g.ny * k);
      if (rho) atomicAdd(rho + node, amount[0] * wt[a]);
      if (j)
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(j + c * unique + node, amount[1 + c] * wt[a]);
      if (pressure)
#pragma unroll
        for (int c = 0; c < 6; ++c) atomicAdd(pressure + c * unique + node, amount[4 + c] * wt[a]);
    }
  }
}

template <class V>
__global__ void __launch_bounds__(256) output_particles_kernel(Geom g, tpicb200_particles p, double* __restrict__ position,
                                                             double* __restrict__ velocity,
                                                             double* __restrict__ charge, uint32_t* invalid) {
  const V* u = (const V*)p.u;
  const V* v = (const V*)p.v;
  const V* w = (const V*)p.w;
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < p.count; n += gridDim.x * blockDim.x) {
    const int32_t key = p.cell[n];
    int ci = 0, cj = 0, ck = 0;
    bool ok = key >= 0 && (long long)key < g.bins;
    if (ok) {
      g.decode(key, ci, cj, ck);
      ok = g.interior_cell(ci, cj, ck);
    }
    const double f[3] = {((const double*)p.rx)[n], ((const double*)p.ry)[n], ((const double*)p.rz)[n]};
    const double vel[3] = {double(u[n]), double(v[n]), double(w[n])};
    const int cell[3] = {ci, cj, ck};
    const double spacing[3] = {g.dx, g.dy, g.dz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      ok = ok && f[a] >= 0 && f[a] < 1 && isfinite(vel[a]);
      position[3 * (size_t)n + a] = (double(cell[a]) + f[a]) * spacing[a];
      velocity[3 * (size_t)n + a] = vel[a];
    }
    charge[n] = p.q[n];
    if (!ok || !isfinite(p.q[n])) atomicAdd(invalid, 1u);
  }
}

// -- VTK XML ----------------------------------------------------------------

std::string padded(long long value) {
  std::string digits = std::to_string(value);
  return std::string(digits.size() < 6 ? 6 - digits.size() : 0, '0') + digits;
}

std::string number(double x) {
  char buf[40];
  std::snprintf(buf, sizeof(buf), "%.17g", x);
  return buf;
}

void field_data(std::string& xml, int cycle, double time, int final_state, const char* profile, const char* roles) {
  xml += "    <FieldData>\n";
  xml += "      <DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\" format=\"ascii\">" +
         number(time) + "</DataArray>\n";
  xml += "      <DataArray type=\"Int32\" Name=\"cycle\" NumberOfTuples=\"1\" format=\"ascii\">" +
         std::to_string(cycle) + "</DataArray>\n";
  xml += "      <DataArray type=\"UInt8\" Name=\"final_state\" NumberOfTuples=\"1\" format=\"ascii\">" +
         std::string(final_state ? "1" : "0") + "</DataArray>\n";
  // A VTK String array: the ASCII byte values, then a zero terminator.
  auto string_array = [&](const char* name, const char* value) {
    xml += std::string("      <Array type=\"String\" Name=\"") + name + "\" NumberOfTuples=\"1\" format=\"ascii\">";
    for (const char* c = value; *c; ++c) xml += std::to_string(unsigned(static_cast<unsigned char>(*c))) + " ";
    xml += "0</Array>\n";
  };
  string_array("state", final_state ? "final" : "pre_solve");
  string_array("precision_profile", profile ? profile : "");
  string_array("precision_roles", roles ? roles : "");
  xml += "    </FieldData>\n";
}

void file_open(std::string& xml, const char* type) {
  xml += "<?xml version=\"1.0\"?>\n";
  xml += std::string("<VTKFile type=\"") + type + "\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
}

void data_array(std::string& xml, const char* type, const char* name, int components, uint64_t offset) {
  xml += std::string("        <DataArray type=\"") + type + "\" Name=\"" + name + "\" NumberOfComponents=\"" +
         std::to_string(components) + "\" format=\"appended\" offset=\"" + std::to_string(offset) + "\"/>\n";
}

const char kAppendedOpen[] = "  <AppendedData encoding=\"raw\">\n_";
const char kAppendedClose[] = "\n  </AppendedData>\n</VTKFile>\n";

// A file opened for writing: exclusive unless overwrite.
struct File {
  FILE* f = nullptr;
  std::string path;
  bool failed = false;
  File(const std::string& p, int overwrite) : path(p) {
    if (!overwrite) {
      struct stat st;
      if (stat(p.c_str(), &st) == 0) {
        failed = true;
        errno = EEXIST;
        return;
      }
    }
    f = std::fopen(p.c_str(), "wb");
    failed = f == nullptr;
  }
  ~File() {
    if (f) std::fclose(f);
  }
  void write(const void* data, size_t bytes) {
    if (!failed && bytes && std::fwrite(data, 1, bytes, f) != bytes) failed = true;
  }
  void text(const std::string& s) { write(s.data(), s.size()); }
  void value(uint64_t v) { write(&v, sizeof(v)); }
  bool close() {
    if (f && std::fclose(f) != 0) failed = true;
    f = nullptr;
    return !failed;
  }
};

int file_error(const std::string& path) {
  return report_error(TPICB200_BACKEND_FAILURE, "output: cannot write " + path + " (" + std::strerror(errno) + ")");
}

int launch_status(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return TPICB200_SUCCESS;
  return report_error(TPICB200_BACKEND_FAILURE, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

cudaError_t launch_output_moments(int precision, const Geom& g, const tpicb200_particles& p, double qom,
                                  double rho_scale, double* rho, double* j, double* pressure, uint32_t* invalid,
                                  cudaStream_t s) {
  if (p.count == 0) return cudaSuccess;
  const unsigned blocks = grid_for(p.count, 256, 148u * 16u);
  if (precision == TPICB200_PRECISION_DOUBLE)
    output_moments_kernel<double><<<blocks, 256, 0, s>>>(g, p, g.inv_volume, 1.0 / qom, rho_scale, rho, j, pressure,
                                                         invalid);
  else
    output_moments_kernel<float><<<blocks, 256, 0, s>>>(g, p, g.inv_volume, 1.0 / qom, rho_scale, rho, j, pressure,
                                                        invalid);
  count_launches(1);
  return cudaGetLastError();
}

namespace {

// One Float64 array of the node grid (PointData, (nx+1)(ny+1)(nz+1) tuples)
// or of its cells (CellData, nx ny nz tuples) as VTK XML ImageData.
int write_image(bool cells, const char* path, const char* name, int components, const tpicb200_grid* grid,
                const double* values, int cycle, double time, int final_state, const char* profile, const char* roles,
                int overwrite) {
  if (!path || !name || !grid || !values || components < 1)
    return report_error(TPICB200_INVALID_ARGUMENT, "vtk field: null argument or no components");
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return report_error(TPICB200_INVALID_ARGUMENT, "vtk field: empty grid");
  const std::string extent = "0 " + std::to_string(grid->nx) + " 0 " + std::to_string(grid->ny) + " 0 " +
                             std::to_string(grid->nz);
  std::string xml;
  file_open(xml, "ImageData");
  xml += "  <ImageData WholeExtent=\"" + extent + "\" Origin=\"0 0 0\" Spacing=\"" + number(grid->lx / grid->nx) +
         " " + number(grid->ly / grid->ny) + " " + number(grid->lz / grid->nz) + "\">\n";
  field_data(xml, cycle, time, final_state, profile, roles);
  xml += "    <Piece Extent=\"" + extent + "\">\n";
  if (cells) {
    xml += "      <PointData/>\n      <CellData>\n";
    data_array(xml, "Float64", name, components, 0);
    xml += "      </CellData>\n";
  } else {
    xml += "      <PointData>\n";
    data_array(xml, "Float64", name, components, 0);
    xml += "      </PointData>\n      <CellData/>\n";
  }
  xml += "    </Piece>\n  </ImageData>\n";
  xml += kAppendedOpen;
  const int extra = cells ? 0 : 1;
  const uint64_t points = uint64_t(grid->nx + extra) * uint64_t(grid->ny + extra) * uint64_t(grid->nz + extra);
  const uint64_t bytes = points * uint64_t(components) * sizeof(double);
  File f(path, overwrite);
  f.text(xml);
  f.value(bytes);
  f.write(values, bytes);
  f.text(kAppendedClose);
  if (!f.close()) return file_error(path);
  return TPICB200_SUCCESS;
}

}  // namespace
}  // namespace tpicb200

using namespace tpicb200;

extern "C" {

int tpicb200_output_moments(tpicb200_context* ctx, double qom, const tpicb200_particles* p, double* rho, double* j,
                            double* pressure, tpicb200_stream stream) {
  if (!ctx) return report_error(TPICB200_INVALID_ARGUMENT, "null context");
  if (!p) return report_error(TPICB200_INVALID_ARGUMENT, "null particle set");
  if (!std::isfinite(qom) || qom == 0)
    return report_error(TPICB200_INVALID_ARGUMENT, "output moments need a finite nonzero q/m");
  if (p->count == 0 || (!rho && !j && !pressure)) return TPICB200_SUCCESS;
  const cudaError_t e = launch_output_moments(context_options(ctx).precision, context_geom(ctx), *p, qom, kFourPi, rho,
                                              j, pressure, context_invalid(ctx), (cudaStream_t)stream);
  if (e != cudaSuccess)
    return report_error(TPICB200_BACKEND_FAILURE, std::string("output moments launch failed: ") + cudaGetErrorString(e));
  return TPICB200_SUCCESS;
}

int tpicb200_output_particles(tpicb200_context* ctx, const tpicb200_particles* p, double* position, double* velocity,
                              double* charge, tpicb200_stream stream) {
  if (!ctx) return report_error(TPICB200_INVALID_ARGUMENT, "null context");
  if (!p || !position || !velocity || !charge) return report_error(TPICB200_INVALID_ARGUMENT, "null output buffer");
  if (p->count == 0) return TPICB200_SUCCESS;
  const Geom& g = context_geom(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned blocks = grid_for(p->count, 256, 148u * 16u);
  if (context_options(ctx).precision == TPICB200_PRECISION_DOUBLE)
    output_particles_kernel<double><<<blocks, 256, 0, s>>>(g, *p, position, velocity, charge, context_invalid(ctx));
  else
    output_particles_kernel<float><<<blocks, 256, 0, s>>>(g, *p, position, velocity, charge, context_invalid(ctx));
  count_launches(1);
  return launch_status("output particles launch failed");
}

int tpicb200_vtk_write_field(const char* path, const char* name, int components, const tpicb200_grid* grid,
                             const double* values, int cycle, double time, int final_state, const char* profile,
                             const char* roles, int overwrite) {
  return write_image(false, path, name, components, grid, values, cycle, time, final_state, profile, roles, overwrite);
}

int tpicb200_vtk_write_cells(const char* path, const char* name, const tpicb200_grid* grid, const double* values,
                             int cycle, double time, int final_state, const char* profile, const char* roles,
                             int overwrite) {
  return write_image(true, path, name, 1, grid, values, cycle, time, final_state, profile, roles, overwrite);
}

int tpicb200_vtk_write_particles(const char* directory, int cycle, double time, int final_state, const char* profile,
                                 const char* roles, int ns, const tpicb200_vtk_species* species, int overwrite) {
  if (!directory || (ns > 0 && !species) || ns < 0) return report_error(TPICB200_INVALID_ARGUMENT, "vtk particles: bad arguments");
  uint64_t count = 0;
  for (int s = 0; s < ns; ++s) {
    const tpicb200_vtk_species& sp = species[s];
    if (sp.count && (!sp.position || !sp.velocity || !sp.charge || !sp.id))
      return report_error(TPICB200_INVALID_ARGUMENT, "vtk particles: null species array");
    count += sp.count;
  }
  const std::string dir(directory);
  const std::string stem = "particles_t" + padded(cycle);
  const std::string piece = stem + "_r" + padded(0) + ".vtp";
  const uint64_t scalar = count * sizeof(uint64_t);
  // Piece: point data velocity, charge, id, species; points; vertices.
  std::string xml;
  file_open(xml, "PolyData");
  xml += "  <PolyData>\n";
  field_data(xml, cycle, time, final_state, profile, roles);
  xml += "    <Piece NumberOfPoints=\"" + std::to_string(count) + "\" NumberOfVerts=\"" + std::to_string(count) +
         "\" NumberOfLines=\"0\" NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n      <PointData>\n";
  uint64_t offset = 0;
  auto array = [&](const char* type, const char* name, int components) {
    data_array(xml, type, name, components, offset);
    offset += sizeof(uint64_t) + scalar * uint64_t(components);
  };
  array("Float64", "velocity", 3);
  array("Float64", "charge", 1);
  array("UInt64", "id", 1);
  array("UInt64", "species", 1);
  xml += "      </PointData>\n      <CellData/>\n      <Points>\n";
  array("Float64", "position", 3);
  xml += "      </Points>\n      <Verts>\n";
  array("Int64", "connectivity", 1);
  array("Int64", "offsets", 1);
  xml += "      </Verts>\n    </Piece>\n  </PolyData>\n";
  xml += kAppendedOpen;
  const std::string piece_path = dir + "/" + piece;
  {
    File f(piece_path, overwrite);
    f.text(xml);
    f.value(scalar * 3);
    for (int s = 0; s < ns; ++s) f.write(species[s].velocity, species[s].count * 3 * sizeof(double));
    f.value(scalar);
    for (int s = 0; s < ns; ++s) f.write(species[s].charge, species[s].count * sizeof(double));
    f.value(scalar);
    for (int s = 0; s < ns; ++s) f.write(species[s].id, species[s].count * sizeof(uint64_t));
    f.value(scalar);
    std::vector<uint64_t> chunk(4096);
    for (int s = 0; s < ns; ++s) {
      std::fill(chunk.begin(), chunk.end(), species[s].species);
      for (uint64_t start = 0; start < species[s].count; start += chunk.size())
        f.write(chunk.data(), std::min<uint64_t>(chunk.size(), species[s].count - start) * sizeof(uint64_t));
    }
    f.value(scalar * 3);
    for (int s = 0; s < ns; ++s) f.write(species[s].position, species[s].count * 3 * sizeof(double));
    for (uint64_t first = 0; first < 2; ++first) {
      f.value(scalar);
      for (uint64_t start = 0; start < count; start += chunk.size()) {
        const uint64_t n = std::min<uint64_t>(chunk.size(), count - start);
        for (uint64_t i = 0; i < n; ++i) chunk[i] = start + i + first;
        f.write(chunk.data(), n * sizeof(uint64_t));
      }
    }
    f.text(kAppendedClose);
    if (!f.close()) return file_error(piece_path);
  }
  // Manifest.
  std::string m;
  file_open(m, "PPolyData");
  m += "  <PPolyData GhostLevel=\"0\">\n";
  field_data(m, cycle, time, final_state, profile, roles);
  auto parray = [&](const char* type, const char* name, int components) {
    m += std::string("      <PDataArray type=\"") + type + "\" Name=\"" + name + "\" NumberOfComponents=\"" +
         std::to_string(components) + "\"/>\n";
  };
  m += "    <PPointData>\n";
  parray("Float64", "velocity", 3);
  parray("Float64", "charge", 1);
  parray("UInt64", "id", 1);
  parray("UInt64", "species", 1);
  m += "    </PPointData>\n    <PCellData/>\n    <PPoints>\n";
  parray("Float64", "position", 3);
  m += "    </PPoints>\n    <Piece Source=\"" + piece + "\"/>\n  </PPolyData>\n</VTKFile>\n";
  const std::string manifest = dir + "/" + stem + ".pvtp";
  File f(manifest, overwrite);
  f.text(m);
  if (!f.close()) return file_error(manifest);
  return TPICB200_SUCCESS;
}

}  // extern "C"
