// Per-planet FP64 global budgets and the device-side monthly-mean
// accumulation of the published snapshot (the reference's page-side
// averager and energy balance, src/model/climate/gcm/averages/index.ts:26-142
// and balance/index.ts, moved next to the state).
//
// On every step a slot publishes, one 256-thread block per slot sums, with a
// fixed order in double precision, the Gaussian-weighted global means of
//   0 surface pressure (the atmosphere's mass, Pa)
//   1 top-of-atmosphere net radiation (W/m^2; snapshot field 16)
//   2 surface net heat flux (W/m^2; snapshot field 17)
//   3 surface temperature (K; snapshot field 0)
//   4 precipitation, convective + large-scale (m/s; snapshot field 5)
//   5 evaporation (m/s, positive upward; snapshot field 18)
//   6 column water vapour (kg/m^2; snapshot field 7)
//   7 the weights' own mean (1 up to rounding: a check)
// and keeps the last values, their running sums and the number of samples.
// The global mean is sum_h w(lat h) f(h) / sum_h w(lat h), the weights the
// FP64 Gaussian weights (summing to 2 per longitude). With averages enabled
// the same step adds every snapshot field of the slot to an FP64 running sum
// (averages/index.ts `add`); exogcm_averages_read returns sum / samples (its
// `close`).
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_budget(Model m) {
  const Dims& d = m.d;
  const int slot = blockIdx.x;
  const StepParams& P = m.params[slot];
  if (!P.active || P.snap[2] == 0.f) return;
  const FieldPtrs& F = m.f;
  const size_t SN = (size_t)d.S * d.NHOR;
  const int NL = d.L;
  double acc[kBudgetQuantities] = {};
  for (int h = threadIdx.x; h < d.NHOR; h += kThreads) {
    const size_t c = (size_t)slot * d.NHOR + h;
    const double w = m.sh.wlat[h / d.NLON];
    const double toa = (double)F.dswfl[c] + (double)F.dlwfl[c];
    const double surf = (double)F.dsmelt[c] * -333700000.0 + (double)F.dswfl[NL * SN + c] +
                        (double)F.dlwfl[NL * SN + c] + (double)F.dshfl[c] + (double)F.dlhfl[c];
    const double q[kBudgetQuantities] = {(double)F.dp[c], toa, surf, (double)F.dt[NL * SN + c],
                                         (double)F.dprc[c] + (double)F.dprl[c], -(double)F.devap[c],
                                         (double)F.dqvi[c], 1.0};
#pragma unroll
    for (int k = 0; k < kBudgetQuantities; ++k) acc[k] += w * q[k];
  }
  __shared__ double red[kBudgetQuantities][kThreads];
#pragma unroll
  for (int k = 0; k < kBudgetQuantities; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int stride = kThreads / 2; stride > 0; stride /= 2) {
    if (threadIdx.x < stride)
#pragma unroll
      for (int k = 0; k < kBudgetQuantities; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double* b = m.budget + (size_t)slot * kBudgetStride;
    const double norm = 2.0 * d.NLON;  // sum of the weights over the grid
    for (int k = 0; k < kBudgetQuantities; ++k) {
      const double v = red[k][0] / norm;
      b[k] = v;
      b[kBudgetQuantities + k] += v;
    }
    b[2 * kBudgetQuantities] += 1.0;
    if (m.avg) b[2 * kBudgetQuantities + 1] += 1.0;
  }
}

// The published snapshot added to the FP64 running sums: one thread per
// point of every snapshot plane of every publishing slot.
__global__ void __launch_bounds__(kThreads) k_average_add(Model m, int planes) {
  const Dims& d = m.d;
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  const size_t per_plane = (size_t)d.S * d.NHOR;
  if (i >= per_plane * planes) return;
  const int slot = (int)((i % per_plane) / d.NHOR);
  const StepParams& P = m.params[slot];
  if (!P.active || P.snap[2] == 0.f) return;
  m.avg[i] += (double)m.f.snapshot[i];
}

}  // namespace

void phy_budget(const Model& m, int snapshot_planes, cudaStream_t st) {
  k_budget<<<m.d.S, kThreads, 0, st>>>(m);
  if (m.avg) {
    const size_t n = (size_t)snapshot_planes * m.d.S * m.d.NHOR;
    k_average_add<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(m, snapshot_planes);
  }
}

}  // namespace exogcm
