// Host-only configuration for compiling the reference's header numerics with
// g++ in the oracle pin harness (no device backend, no profiling, no MPI).
// Written for this harness; the reference generates its own copy with cmake.
#ifndef LPFX_CONFIG_HPP
#define LPFX_CONFIG_HPP
#define LPFX_VERSION_MAJOR 0
#define LPFX_VERSION_MINOR 0
#define LPFX_VERSION_PATCH 0
#define LPFX_CONFIG_PROFILING_NVTX 0
#define LPFX_CONFIG_PROFILING_ROCTX 0
#define LPFX_CONFIG_PROFILING_ROCTX_LEGACY 0
#define LPFX_CONFIG_ENABLE_CRAYPAT 0
#define LPFX_CONFIG_PARTICLE_CAPACITY_HEADROOM_PERCENT 0U
#define LPFX_CONFIG_PARTICLE_CAPACITY_MULTIPLE 1U
#define LPFX_CONFIG_ENABLE_OPENMP 0
#define LPFX_CONFIG_ENABLE_DEVICE_AWARE_MPI 0
#define LPFX_CONFIG_ENABLE_NCCL 0
#define LPFX_CONFIG_ENABLE_RCCL 0
#define LPFX_CONFIG_XCCL_MINIMUM_VERSION 0
#define LPFX_CONFIG_DEVICE_BACKEND_CUDA 0
#define LPFX_CONFIG_DEVICE_BACKEND_HIP 0
#endif
