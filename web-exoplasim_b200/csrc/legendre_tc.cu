// Inverse Legendre transforms (sp2fc, sp2fcdmu) on the tcgen05 tensor cores:
// engine mode 2 (the optimized path of mode 1 with these two transforms on
// the tensor cores; mode 1 keeps the SIMT latitude-pair kernels, which are
// faster at these sizes because the contraction is bound by staging, not
// arithmetic).
//
// For one zonal wavenumber m the transform of a tile of planes is a GEMM:
//   D[lat][n] = sum over modes t of Q[lat][t] * S[t][n],
// lat over the NLAT Gaussian latitudes (padded to the MMA's 128 rows), t over
// the NTP1 - m modes of m (padded to K steps of 8), n over (plane, re/im).
// The table slice Q is the A operand and the staged coefficients the B
// operand, both K-major without swizzle in shared memory; D accumulates in
// FP32 in tensor memory (TMEM).
//
// Precision: three TF32 products per K step (hi*hi + hi*lo + lo*hi, where
// x = hi + lo and hi is x rounded to TF32) reproduce FP32 to about 2^-21
// relative, well inside the transforms' 1e-5 bound against FP64. The table's
// hi/lo images are built once on the host (exogcm_configure) in the exact
// shared-memory layout; the coefficients are split when staged.
//
// A CTA of 4 warps walks (m, 64-plane tile) items persistently: the threads
// stage A (contiguous image copy) and B (coefficient gather and split), one
// elected thread issues the MMAs and commits them to an mbarrier, and every
// warp reads its 32 TMEM lanes (latitudes) back and writes, per plane, the
// item's contiguous run of latitudes in the m-major Fourier plane. Waits on
// the mbarrier are bounded: on a timeout the CTA records a fault, frees its
// TMEM and stops, and the engine reports the fault after the step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "async_copy.cuh"
#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kTcRows = 128;             // MMA M: latitudes, zero-padded
constexpr int kTcPlanes = 64;            // planes per item
constexpr int kTcN = 2 * kTcPlanes;      // MMA N: (plane, re/im)
constexpr int kTcThreads = 128;          // 4 warps: one per 32 TMEM lanes
constexpr int kTcColumns = 128;          // TMEM columns allocated (>= kTcN, power of 2)
constexpr int kStepFloatsA = kTcRows * 8;  // one K step of A: 128 rows x 8 tf32
constexpr int kStepFloatsB = kTcN * 8;     // one K step of B
constexpr long kWaitLimit = 1L << 22;     // mbarrier polls before a CTA gives up

__device__ __forceinline__ int first_mode(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }

// Offset (floats) of element (row, k) inside one K step of a K-major,
// no-swizzle operand: core matrices of 8 rows x 16 bytes; the two 16-byte
// K halves 128 bytes apart (leading byte offset), 8-row groups 256 bytes
// apart (stride byte offset).
__host__ __device__ __forceinline__ int kmajor_offset(int row, int k) {
  return (row >> 3) * 64 + (k >> 2) * 32 + (row & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100): start address, leading byte
// offset 128, stride byte offset 256 (all >> 4), descriptor version 1,
// no swizzle.
__device__ __forceinline__ uint64_t operand_desc(const void* p) {
  uint64_t d = (uint64_t)((smem_addr(p) >> 4) & 0x3FFF);
  d |= (uint64_t)(128 >> 4) << 16;
  d |= (uint64_t)(256 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor: D F32, A and B TF32, both K-major, N = kTcN,
// M = kTcRows.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(kTcRows >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(smem_addr(mbar)), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive TMEM columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// x rounded to TF32 (nearest, ties away from zero), as a float.
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_tc_inverse(const float* __restrict__ s, float* __restrict__ f, int planes, const float* __restrict__ images,
                 const int* __restrict__ image_at, int* __restrict__ fault, Dims d) {
  extern __shared__ float4 smem_tc[];
  const int ksmax = (d.NTP1 + 7) / 8;
  float* a_hi = reinterpret_cast<float*>(smem_tc);
  float* a_lo = a_hi + ksmax * kStepFloatsA;
  float* b_hi = a_lo + ksmax * kStepFloatsA;
  float* b_lo = b_hi + ksmax * kStepFloatsB;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(b_lo + ksmax * kStepFloatsB);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(kTcColumns));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const size_t plane_floats = (size_t)d.NLAT * d.NFC;
  const int tiles = (planes + kTcPlanes - 1) / kTcPlanes;
  const int items = d.NTP1 * tiles;
  uint32_t parity = 0;
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int m = item % d.NTP1;
    const int p0 = (item / d.NTP1) * kTcPlanes;
    const int np = min(kTcPlanes, planes - p0);
    const int K = d.NTP1 - m, ks = (K + 7) / 8;
    const int w0 = first_mode(m, d.NTP1);
    // A: the table's hi and lo images for m (ks steps each).
    const float* img = images + image_at[m];
    for (int i = threadIdx.x; i < ks * kStepFloatsA / 4; i += blockDim.x) {
      cp_async16(a_hi + 4 * i, img + 4 * i);
      cp_async16(a_lo + 4 * i, img + ks * kStepFloatsA + 4 * i);
    }
    cp_async_commit();
    // B: coefficient (re, im) of plane p, mode t -> rows n = 2p, 2p + 1, K index t.
    for (int i = threadIdx.x; i < kTcPlanes * ks * 8; i += blockDim.x) {
      const int p = i / (ks * 8), t = i - p * (ks * 8);
      float2 v = make_float2(0.f, 0.f);
      if (p < np && t < K) v = *reinterpret_cast<const float2*>(s + (size_t)(p0 + p) * d.NRSP + 2 * (w0 + t));
      const int step = t >> 3, k = t & 7;
      const float hr = tf32_round(v.x), hi_ = tf32_round(v.y);
      const int o0 = step * kStepFloatsB + kmajor_offset(2 * p, k);
      const int o1 = step * kStepFloatsB + kmajor_offset(2 * p + 1, k);
      b_hi[o0] = hr;
      b_lo[o0] = v.x - hr;
      b_hi[o1] = hi_;
      b_lo[o1] = v.y - hi_;
    }
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // staged operands visible to the tensor cores
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (threadIdx.x == 0) {
      for (int step = 0; step < ks; ++step) {
        const uint64_t ah = operand_desc(a_hi + step * kStepFloatsA), al = operand_desc(a_lo + step * kStepFloatsA);
        const uint64_t bh = operand_desc(b_hi + step * kStepFloatsB), bl = operand_desc(b_lo + step * kStepFloatsB);
        mma_tf32(tmem, ah, bh, step > 0 ? 1u : 0u);
        mma_tf32(tmem, ah, bl, 1u);
        mma_tf32(tmem, al, bh, 1u);
      }
      mma_commit(mbar);
    }
    bool done = false;
    for (long i = 0; i < kWaitLimit && !done; ++i) done = mbar_try_wait(mbar, parity);
    parity ^= 1u;
    if (__syncthreads_or(!done)) {
      if (threadIdx.x == 0) atomicExch(fault, 1);
      break;
    }
    fence_after_sync();
    if (warp * 32 < d.NLAT) {
      const int lat = warp * 32 + lane;
#pragma unroll 1
      for (int c = 0; c < kTcN / 32; ++c) {
        float v[32];
        tmem_load32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32), v);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int p = c * 16 + q;
          if (p < np)
            reinterpret_cast<float2*>(f + (size_t)(p0 + p) * plane_floats)[(size_t)m * d.NLAT + lat] =
                make_float2(v[2 * q], v[2 * q + 1]);
        }
      }
    }
    fence_before_sync();
    __syncthreads();  // D and the operands are reused by the next item
  }
  cp_async_wait_all();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcColumns));
}

size_t tc_inverse_smem(const Dims& d) {
  const int ksmax = (d.NTP1 + 7) / 8;
  return (size_t)ksmax * (2 * kStepFloatsA + 2 * kStepFloatsB) * sizeof(float) + 16;
}

}  // namespace

void tc_init() {
  cudaFuncSetAttribute(k_tc_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLegSmemLimit);
}

// Host images of one full-latitude table ([NLAT][NCSP], FP64) for the
// tensor-core inverse: for each m, the hi then the lo image of its K steps,
// laid out as the kernel's A operand. `at[m]` is the float offset of m's
// images; the total length is returned in `at[NTP1]`.
std::vector<float> tc_table_images(const Dims& d, const std::vector<double>& q, std::vector<int>& at) {
  auto round_tf32 = [](float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u = (u + 0x1000u) & ~0x1FFFu;  // nearest, ties away from zero (the magnitude bits)
    float y;
    std::memcpy(&y, &u, 4);
    return y;
  };
  at.assign(d.NTP1 + 1, 0);
  std::vector<float> out;
  for (int m = 0; m < d.NTP1; ++m) {
    const int K = d.NTP1 - m, ks = (K + 7) / 8;
    const int w0 = m * (2 * d.NTP1 - m + 1) / 2;
    at[m] = (int)out.size();
    std::vector<float> hi((size_t)ks * kStepFloatsA, 0.f), lo((size_t)ks * kStepFloatsA, 0.f);
    for (int lat = 0; lat < d.NLAT; ++lat)
      for (int t = 0; t < K; ++t) {
        const double v = q[(size_t)lat * d.NCSP + w0 + t];
        const float h = round_tf32((float)v);
        const float l = round_tf32((float)(v - (double)h));
        const size_t o = (size_t)(t >> 3) * kStepFloatsA + kmajor_offset(lat, t & 7);
        hi[o] = h;
        lo[o] = l;
      }
    out.insert(out.end(), hi.begin(), hi.end());
    out.insert(out.end(), lo.begin(), lo.end());
  }
  at[d.NTP1] = (int)out.size();
  return out;
}

void tc_inverse(const Model& m, const float* s, float* f, int planes, bool derivative, cudaStream_t st) {
  const size_t smem = tc_inverse_smem(m.d);
  const int items = m.d.NTP1 * ((planes + kTcPlanes - 1) / kTcPlanes);
  const int grid = std::min(items, persistent_grid((const void*)k_tc_inverse, kTcThreads, smem));
  k_tc_inverse<<<grid, kTcThreads, smem, st>>>(s, f, planes, derivative ? m.sh.tc_qj : m.sh.tc_qi, m.sh.tc_at,
                                               m.fault, m.d);
}

}  // namespace exogcm
