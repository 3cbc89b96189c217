// Configuration for compiling the reference's device kernels with nvcc in the
// GPU comparator harness (CUDA backend; no profiling, no MPI, no NCCL).
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
#define LPFX_CONFIG_DEVICE_BACKEND_CUDA 1
#define LPFX_CONFIG_DEVICE_BACKEND_HIP 0
#endif
