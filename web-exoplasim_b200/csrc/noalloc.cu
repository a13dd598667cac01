// An allocation-free entry point for the per-planet FP64 global sums.
//
// Some callers cannot allocate device memory at all: a host that runs
// inside another framework's memory pool with cudaMalloc forbidden, an
// embedded runtime that must not grow its footprint after start-up, or a
// caller in the middle of work that may not synchronize the device (which
// cudaMalloc and cudaFree can do). For them this file offers the sums the
// fixer and getiflx reductions compute (the kernel behind exogcm_step's
// fixsum and ice_sums fields) with no allocation: the caller passes the
// inputs and the output, and the kernels' scratch lives in one file-scope
// device array. Unlike the step's reductions, which skip inactive slots (and,
// for getiflx, slots without sea-ice coupling) and leave their outputs as
// they were, this entry point sums every one of `slots` slots it is given.
//
// With CUDA's lazy module loading the array is committed to the device when
// the first call on that device looks up its address, not when the library
// loads: a caller whose footprint must be fixed after start-up makes one
// call during its own start-up.
//
// The scratch is kNoAllocMaxSlots x 256 x 2 doubles (1 MiB). Every GPU that
// loads this library holds it until the process exits. Every call shares it
// and it keeps the last call's values; each call writes every partial it
// later reads, so nothing needs clearing, but calls that overlap on the GPU
// (different streams, or different host threads) race on it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/exogcm.h"

namespace exogcm {
void set_error(const std::string& message);  // engine.cu
}

namespace {

constexpr int kSumThreads = 256;
constexpr int kNoAllocMaxSlots = 256;
constexpr int kMaxDevices = 64;

// Per-slot, per-thread partial sums: [slot][thread][first | second].
static __device__ __align__(256) double g_sum_partials[kNoAllocMaxSlots * kSumThreads * 2];

// Pass 1: thread t of slot s sums points t, t + 256, ... of both fields in
// FP64 (the order of the fused reduction in physics.cu) into the scratch.
__global__ void __launch_bounds__(kSumThreads) k_partials(const float* __restrict__ a, const float* __restrict__ b,
                                                          int points, double* __restrict__ scratch) {
  const int slot = blockIdx.x, t = threadIdx.x;
  double x = 0.0, y = 0.0;
  const size_t base = (size_t)slot * points;
  for (int h = t; h < points; h += kSumThreads) {
    x += (double)a[base + h];
    y += (double)b[base + h];
  }
  scratch[((size_t)slot * kSumThreads + t) * 2] = x;
  scratch[((size_t)slot * kSumThreads + t) * 2 + 1] = y;
}

// Pass 2: the same fixed-order tree over each slot's 256 partials.
__global__ void __launch_bounds__(kSumThreads) k_combine(const double* __restrict__ scratch, int slots,
                                                         float* __restrict__ out) {
  __shared__ double sa[kSumThreads], sb[kSumThreads];
  const int slot = blockIdx.x, t = threadIdx.x;
  sa[t] = scratch[((size_t)slot * kSumThreads + t) * 2];
  sb[t] = scratch[((size_t)slot * kSumThreads + t) * 2 + 1];
  __syncthreads();
  for (int stride = kSumThreads / 2; stride > 0; stride /= 2) {
    if (t < stride) {
      sa[t] += sa[t + stride];
      sb[t] += sb[t + stride];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[slot] = (float)sa[0];
    out[slots + slot] = (float)sb[0];
  }
}

// Device address of the scratch array, looked up once per device under a
// per-device once-flag (host threads may call concurrently). In host code
// g_sum_partials is only a host-side stand-in for the symbol; a kernel must
// be given the address cudaGetSymbolAddress returns for the current device.
// The address belongs to the device's primary context: after a
// cudaDeviceReset the process must reload the library before calling again.
std::once_flag g_scratch_once[kMaxDevices];
double* g_scratch_address[kMaxDevices] = {nullptr};
cudaError_t g_scratch_error[kMaxDevices] = {};

}  // namespace

extern "C" int exogcm_slot_sums_noalloc(const float* first, const float* second, int slots, int points, float* sums,
                                        void* stream) {
  if (!first || !second || !sums) {
    exogcm::set_error("exogcm_slot_sums_noalloc: null pointer");
    return EXOGCM_EINVAL;
  }
  if (slots < 1 || slots > kNoAllocMaxSlots || points < 1) {
    exogcm::set_error("exogcm_slot_sums_noalloc: slots must be 1.." + std::to_string(kNoAllocMaxSlots) +
                      " (the size of its static scratch) and points positive; got slots = " +
                      std::to_string(slots));
    return EXOGCM_EINVAL;
  }
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess || device < 0 || device >= kMaxDevices) {
    exogcm::set_error(std::string("exogcm_slot_sums_noalloc: no usable device: ") + cudaGetErrorString(err));
    return EXOGCM_EDEVICE;
  }
  std::call_once(g_scratch_once[device], [device] {
    void* ptr = nullptr;
    g_scratch_error[device] = cudaGetSymbolAddress(&ptr, g_sum_partials);
    if (g_scratch_error[device] == cudaSuccess) g_scratch_address[device] = static_cast<double*>(ptr);
  });
  double* scratch = g_scratch_address[device];
  if (!scratch) {
    exogcm::set_error(std::string("exogcm_slot_sums_noalloc: scratch address: ") +
                      cudaGetErrorString(g_scratch_error[device]));
    return EXOGCM_EDEVICE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_partials<<<slots, kSumThreads, 0, st>>>(first, second, points, scratch);
  k_combine<<<slots, kSumThreads, 0, st>>>(scratch, slots, sums);
  err = cudaGetLastError();
  if (err != cudaSuccess) {
    exogcm::set_error(std::string("exogcm_slot_sums_noalloc: launch: ") + cudaGetErrorString(err));
    return EXOGCM_EDEVICE;
  }
  return EXOGCM_OK;
}
