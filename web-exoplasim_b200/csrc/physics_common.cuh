// Shared helpers of the column-physics translation units (physics.cu and
// physics_flux.cu): the column prologues, saturation and power helpers, the
// per-level-count dispatch and the one-thread-per-column launcher.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kBlock = 128;

// Asks L2 for a line this thread reads after its first store, so that load
// then hits L2 instead of DRAM (a hint: it moves no data into registers).
__device__ __forceinline__ void prefetch_l2(const float* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Column kernels take the planet constants and per-planet tables as
// __restrict__ parameters: both are read-only during a launch, so the
// compiler may keep their values across the kernel's stores to fields
// instead of reloading them after every store.
#define COLUMN_PROLOGUE                                              \
  pdl_wait();                                                        \
  pdl_release();                                                     \
  const Dims& d = m.d;                                               \
  const int c = blockIdx.x * blockDim.x + threadIdx.x;               \
  if (c >= d.S * d.NHOR) return;                                     \
  const int slot = c / d.NHOR;                                       \
  const int h = c % d.NHOR;                                          \
  const StepParams& P = m.params[slot];                              \
  if (!P.active) return;                                             \
  const PlanetConst& K = pcr[slot];                                  \
  const float* tb = tabr + (size_t)slot * m.to.stride;               \
  const size_t SN = (size_t)d.S * d.NHOR;                            \
  const FieldPtrs& F = m.f;                                          \
  (void)h; (void)K; (void)tb; (void)SN; (void)F; (void)P;

// The same for a kernel that reads its planet's constants inside long
// loops: column kernels run kBlock threads per block over S * NHOR columns,
// and kBlock divides NHOR (2048, 8192 or 18432), so a block's columns
// belong to one slot, whose constants are staged once in shared memory.
#define COLUMN_PROLOGUE_STAGED                                       \
  pdl_wait();                                                        \
  pdl_release();                                                     \
  const Dims& d = m.d;                                               \
  const int slot = blockIdx.x * kBlock / d.NHOR;                     \
  const StepParams& P = m.params[slot];                              \
  if (!P.active) return;                                             \
  __shared__ PlanetConst s_planet;                                   \
  stage_planet(pcr + slot, &s_planet);                               \
  const PlanetConst& K = s_planet;                                   \
  const int c = blockIdx.x * kBlock + threadIdx.x;                   \
  if (c >= d.S * d.NHOR) return;                                     \
  const int h = c - slot * d.NHOR;                                   \
  const float* tb = tabr + (size_t)slot * m.to.stride;               \
  const size_t SN = (size_t)d.S * d.NHOR;                            \
  const FieldPtrs& F = m.f;                                          \
  (void)h; (void)K; (void)tb; (void)SN; (void)F; (void)P;

// Copies one slot's constants into shared memory (all threads of the block
// take part and meet at the barrier).
__device__ __forceinline__ void stage_planet(const PlanetConst* src, PlanetConst* dst) {
  constexpr int n = sizeof(PlanetConst) / sizeof(float);
  const float* a = reinterpret_cast<const float*>(src);
  float* b = reinterpret_cast<float*>(dst);
  for (int i = threadIdx.x; i < n; i += blockDim.x) b[i] = a[i];
  __syncthreads();
}

__device__ __forceinline__ float sat_capped(const PlanetConst& K, float t, float p) {
  return fminf(K.RDBRV * K.RA1 * expf(K.RA2 * (t - K.TMELT) / (t - K.RA4)) / p, K.RDBRV);
}
// The same with IEEE divisions, for the large-scale condensation, whose
// precipitation is the small difference of two iterated states.
__device__ __forceinline__ float sat_capped_rn(const PlanetConst& K, float t, float p) {
  return fminf(__fdiv_rn(K.RDBRV * K.RA1 * expf(__fdiv_rn(K.RA2 * (t - K.TMELT), t - K.RA4)), p), K.RDBRV);
}
__device__ __forceinline__ float sat_divided(const PlanetConst& K, float t, float p) {
  const float q = sat_capped(K, t, p);
  return q / (1.f - K.MOIST * q);
}
// The longwave band fits' base-2 logarithm and power: CUDA's accurate
// log2f and exp2f, or, built with EXOGCM_LWR_FAST_LOG2 / EXOGCM_LWR_FAST_EXP2,
// the special-function unit's lg2.approx / ex2.approx instructions.
__device__ __forceinline__ float fit_log2(float x) {
#ifdef EXOGCM_LWR_FAST_LOG2
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return log2f(x);
#endif
}
__device__ __forceinline__ float fit_exp2(float x) {
#ifdef EXOGCM_LWR_FAST_EXP2
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return exp2f(x);
#endif
}
// x^y for x >= 0 with 0^y = 0: precise_pow (src/model/shared/gpu/math/wgsl/
// precise.wgsl:100-103) is exp(y * log(x)); here exp2(y * log2(x)) with
// CUDA's own exp2f and log2f.
__device__ __forceinline__ float fpow(float x, float y) {
#ifdef EXOGCM_FAST_POW
  float l, r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y * l));
  return x == 0.f ? 0.f : r;
#else
  return x == 0.f ? 0.f : exp2f(y * log2f(x));
#endif
}
// x^n by binary exponentiation, as libgcc's __powisf2 computes x**n.
__device__ __forceinline__ float powi(float x, int n) {
  float base = x;
  unsigned mm = (unsigned)abs(n);
  float result = (mm & 1u) ? x : 1.f;
  mm >>= 1;
  while (mm) {
    base = base * base;
    if (mm & 1u) result = result * base;
    mm >>= 1;
  }
  return n < 0 ? 1.f / result : result;
}

constexpr float kPI = 3.14159265359f;
constexpr float kTWOPI = kPI + kPI;

constexpr int kSumThreads = 256;

inline unsigned nblocks(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

// Implicit vertical diffusion (physics/diffusion/wgsl/implicit.wgsl): the
// tridiagonal solve of one column, for a quantity and for potential
// temperature, with IEEE divisions (the tendencies are small differences of
// the diffused and the old profiles).
template <int NL>
__device__ __forceinline__ void diffuse(const float* ds, float* x, const float* k) {
  float ebs[NL];
  const float ds0 = ds[0];
  ebs[0] = __fdiv_rn(k[0], ds0 + k[0]);
  x[0] = __fdiv_rn(ds0 * x[0], ds0 + k[0]);
#pragma unroll
  for (int l = 1; l < NL - 1; ++l) {
    const float den = ds[l] + k[l] + k[l - 1] * (1.f - ebs[l - 1]);
    ebs[l] = __fdiv_rn(k[l], den);
    x[l] = __fdiv_rn(x[l] * ds[l] + k[l - 1] * x[l - 1], den);
  }
  const float dsn = ds[NL - 1];
  x[NL - 1] = __fdiv_rn(x[NL - 1] * dsn + k[NL - 2] * x[NL - 2], dsn + k[NL - 2] * (1.f - ebs[NL - 2]));
#pragma unroll
  for (int l = NL - 2; l >= 0; --l) x[l] = x[l] + ebs[l] * x[l + 1];
}

template <int NL>
__device__ __forceinline__ void diffuse_potential(const float* ds, float* x, const float* k, const float* skap) {
  float ebs[NL];
  const float ds0 = ds[0];
  ebs[0] = __fdiv_rn(k[0], ds0 + __fdiv_rn(k[0], skap[0]));
  x[0] = __fdiv_rn(ds0 * x[0], ds0 + __fdiv_rn(k[0], skap[0]));
#pragma unroll
  for (int l = 1; l < NL - 1; ++l) {
    const float den = ds[l] + __fdiv_rn(k[l] + k[l - 1] * (1.f - __fdiv_rn(ebs[l - 1], skap[l - 1])), skap[l]);
    ebs[l] = __fdiv_rn(k[l], den);
    x[l] = __fdiv_rn(x[l] * ds[l] + __fdiv_rn(k[l - 1], skap[l - 1]) * x[l - 1], den);
  }
  const int last = NL - 1;
  const float dsn = ds[last];
  x[last] = __fdiv_rn(x[last] * dsn + __fdiv_rn(k[NL - 2] * x[NL - 2], skap[NL - 2]),
                      dsn + __fdiv_rn(k[NL - 2], skap[last]) * (1.f - __fdiv_rn(ebs[NL - 2], skap[NL - 2])));
#pragma unroll
  for (int l = NL - 2; l >= 0; --l) x[l] = x[l] + __fdiv_rn(ebs[l] * x[l + 1], skap[l + 1]);
}


template <template <int> class Launch, typename... A>
void by_levels(int L, A&&... a) {
  if (L == 10)
    Launch<10>::run(a...);
  else if (L == 5)
    Launch<5>::run(a...);
}

// Column kernels begin with COLUMN_PROLOGUE(_STAGED), whose pdl_wait comes
// before any state access, so they start by programmatic dependent launch.
#define COLUMN_LAUNCHER(name, kernel)                                                               \
  template <int NL>                                                                                 \
  struct name {                                                                                     \
    static void run(const Model& m, cudaStream_t st) {                                              \
      pdl_launch(kernel<NL>, nblocks((size_t)m.d.S * m.d.NHOR, kBlock), kBlock, 0, st, m, m.pc, m.tabs); \
    }                                                                                               \
  };

}  // namespace

}  // namespace exogcm
