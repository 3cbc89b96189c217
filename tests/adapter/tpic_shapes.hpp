// Stand-ins for the TPIC-side types the adapter in INTEGRATION.md uses
// (owners, slots, bins, executor, reports, lpfx::ErrorCode), with the member
// names of TPIC's actions layer, so that the adapter's code compiles against
// include/tpicb200.h in a test. Declarations only: the test compiles the
// adapter, it does not run it.
#pragma once

#include <tpicb200.h>

#include <cstddef>
#include <cstdint>
#include <span>

namespace lpfx {
// include/lpfx/core/error.hpp: the first five values, in order.
enum class ErrorCode { success = 0, invalid_argument, invalid_state, overflow, backend_failure };
}  // namespace lpfx

namespace tpic::simulation {

template <class T> struct DeviceArray {
  T* data();
  const T* data() const;
};

struct ParticleColumns {
  DeviceArray<double>& rx();
  DeviceArray<double>& ry();
  DeviceArray<double>& rz();
  DeviceArray<float>& u();
  DeviceArray<float>& v();
  DeviceArray<float>& w();
  DeviceArray<double>& q();
  DeviceArray<int32_t>& cell();
  DeviceArray<uint64_t>& id();
  std::size_t size() const;
};

enum class SpeciesSlot { first, second };

struct ParticleOwner {
  ParticleColumns& slot(SpeciesSlot s);
};

struct CellBinsOwner {
  uint32_t* counts();
  uint32_t* offsets();
};

struct Species {
  ParticleOwner particles;
  CellBinsOwner bins;
  double qom;
  uint32_t* invalid;
  SpeciesSlot live_slot() const;
  SpeciesSlot idle_slot() const;
  void rotate_slots();
};

struct FieldOwners {
  DeviceArray<float> e, b_cell, b_node, b_node_next, j, mass;
  DeviceArray<double> e_theta;
};

struct Executor {
  CUstream_st* stream() const;
};

struct GmresReport {
  bool converged;
  int iterations;
  double relative_residual;
};

class B200Backend {
 public:
  lpfx::ErrorCode move_and_sort(Species& sp, const FieldOwners& f, const Executor& ex);
  lpfx::ErrorCode deposit(std::span<Species> species, FieldOwners& f, const Executor& ex);
  lpfx::ErrorCode solve(FieldOwners& f, GmresReport& report, const Executor& ex);
  lpfx::ErrorCode cycle_with_tape(tpicb200_state& st, tpicb200_tape& tape, const Executor& ex);
  lpfx::ErrorCode cycle_backward(tpicb200_tape& tape, tpicb200_adjoint& adj, const Executor& ex);

 private:
  tpicb200_context* ctx_ = nullptr;
  int mass_kind_ = 3;
};

}  // namespace tpic::simulation
