// The Gauss-Legendre transform family on the tcgen05 tensor cores in split
// precision: engine mode 2 (the optimized path of mode 1 with every Legendre
// contraction here). The reference's shaders are
// src/model/climate/gcm/legendre/wgsl/{inverse,dv2uv,forward,uv2dv,qtend}.wgsl,
// composed by legendre/index.ts:157-330:
//   inverse  sp2fc / sp2fcdmu  f_m(lat)  = sum_n q[lat][mn] s_mn
//   dv2uv                      u, v      from D, zeta (tables qu, qv)
//   forward  fc2sp             s_mn      = sum_pairs q[l][mn] (N +- S)
//   uv2dv / mktend             D, zeta   from u, v (+ kinetic energy, qq)
//   qtend                      flux-form tendency (qe, qc, qm)
//
// For one zonal wavenumber m and a tile of planes every one of them is a
// GEMM whose table operand is fixed and whose data operand is gathered:
//   D[row][col] = sum_k Data[row][k] * Table[col][k]
// with row = (plane, output column c) -- 128 rows, the MMA's M --, col =
// latitude (inverse kinds: N = NLAT) or mode n of m (forward kinds: N = the
// modes rounded up to 16), and k over the table blocks a (qv | qu, qe | qm |
// qq, ...) times the input index: modes of m for the inverse kinds, for the
// forward kinds latitude pairs in two halves, the sum N + S and the
// difference N - S of the northern and southern rows (computed in f32 as the
// shaders do). Each table block multiplies, for each output column c, one
// signed input component (the term table below), so the complex
// multiply-adds of the shaders become one real contraction. Which half a
// mode's table entry sits in follows the parity of n - m, as the shaders'
// north + s * south: the other half's entry is zero.
//
// Precision (split precision, "3xTF32"): every f32 operand x is split into
// hi = x rounded to TF32 and lo = (x - hi) rounded to TF32; the tables are
// split from their FP64 values on the host. Three tcgen05.mma.kind::tf32
// per K step, hi*hi + hi*lo + lo*hi, accumulate in FP32 in tensor memory;
// the dropped lo*lo term is below 2^-22 of the product.
//
// Pipeline (one CTA per SM, persistent over (m, plane tile) items; warp roles):
//   warp 0  producer: TMA (cp.async.bulk.tensor) loads of the raw input rows
//           into a double-buffered raw stage, and cp.async.bulk loads of the
//           table chunks (4 K steps of hi and lo images) into a two-stage
//           ring; every load completes on an mbarrier with a byte count.
//   warps 1-4 converters and epilogue: build the data operand (gather,
//           sign, N +- S, hi/lo split) in the K-major no-swizzle layout for
//           each chunk, then drain the previous item's accumulator
//           (tcgen05.ld, a transpose through shared memory, coalesced
//           stores) while the tensor cores run the current one.
//   warp 5  MMA issuer: one thread issues the MMAs of a chunk as soon as its
//           table and data stages are full, commits them to the stages'
//           "empty" barriers and, after an item's last chunk, to the
//           accumulator's "full" barrier; TMEM holds two accumulators.
// Every tensor map covers this GPU's own memory, and no load uses cluster
// multicast. Every wait on an mbarrier is bounded: a role that gives up sets
// the engine's fault word and an abort flag the other roles poll, the
// producer then waits (bounded) for its loads in flight, the MMA thread for
// its MMAs, and the CTA frees its tensor memory and ends; the engine reports
// the fault after the step.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kRows = 128;        // MMA M: (plane, column) rows of the data operand
constexpr int kThreads = 320;     // warp 0 producer, warps 1-8 converters/epilogue, warp 9 MMA
constexpr int kConv = 256;        // converter threads: two warps per scheduler hide the operand build's latency
constexpr int kMmaWarp = 9;
constexpr int kTmemCols = 256;    // two accumulators of up to 128 columns
constexpr int kStepK = 8;         // K of one tf32 MMA
constexpr int kChunkSteps = 4;    // K steps per pipeline chunk
constexpr int kDataStepFloats = kRows * kStepK;  // one K step of hi (or lo) data operand
constexpr int kMaxTab = 8;        // table stages at most (TcGeom::n_tab of them are used)
constexpr int kNData = 2;         // data operand stages
constexpr long kWaitLimit = 1L << 24;  // mbarrier polls before a role gives up
constexpr size_t kTcSmemLimit = 227 * 1024;  // dynamic shared memory a CTA may ask

// Kinds and their shapes: NR raw input fields, NA table blocks, NC output
// columns per plane (TP = 128 / NC planes per item), FWD forward (K over
// latitude pairs) or inverse (K over modes).
enum Kind : int { INV = 0, DV2UV = 1, FWD = 2, UV2DV = 3, MKTEND = 4, QTEND = 5 };

template <int KIND>
struct Shape {
  static constexpr bool fwd = KIND >= FWD;
  static constexpr int NR = KIND == INV || KIND == FWD ? 1 : KIND == DV2UV || KIND == UV2DV ? 2 : 3;
  static constexpr int NA = KIND == INV || KIND == FWD ? 1 : KIND == DV2UV || KIND == UV2DV ? 2 : 3;
  static constexpr int NC = KIND == INV || KIND == FWD || KIND == QTEND ? 2 : 4;
  static constexpr int TP = kRows / NC;
  static constexpr int NOUT = NC / 2;
};

// Term of table block a for output column c: raw field, component (0 re,
// 1 im), sign; field -1 is a zero term. Inverse kinds read the raw fields in
// the order the launcher passes them: INV {s}, DV2UV {D, zeta}; forward
// kinds FWD {f}, UV2DV/MKTEND {u, v, ke}, QTEND {u, v, x}.
struct Term {
  int field, comp;
  float sign;
};

template <int KIND>
__device__ __forceinline__ Term term(int a, int c) {
  if (KIND == INV || KIND == FWD) return {0, c, 1.f};
  if (KIND == DV2UV) {
    // a0 = qv: U.re += zeta'.re, U.im += zeta.im, V.re -= D.re, V.im -= D.im
    // a1 = qu: U.re += D.im,     U.im -= D.re,    V.re += zeta.im, V.im -= zeta'.re
    // (legendre/wgsl/dv2uv.wgsl: u = sum qv zeta + i qu D, v = sum i qu zeta - qv D)
    if (a == 0) return c == 0 ? Term{1, 0, 1.f} : c == 1 ? Term{1, 1, 1.f} : c == 2 ? Term{0, 0, -1.f} : Term{0, 1, -1.f};
    return c == 0 ? Term{0, 1, 1.f} : c == 1 ? Term{0, 0, -1.f} : c == 2 ? Term{1, 1, 1.f} : Term{1, 0, -1.f};
  }
  if (KIND == UV2DV || KIND == MKTEND) {
    // a0 = qe (difference half for even n - m), a1 = qm (sum half), a2 = qq
    // D.re = -e Vd.re - mq Us.im, D.im = -e Vd.im + mq Us.re,
    // Z.re = e Ud.re - mq Vs.im,  Z.im = e Ud.im + mq Vs.re  (uv2dv.wgsl)
    if (a == 0) return c == 0 ? Term{1, 0, -1.f} : c == 1 ? Term{1, 1, -1.f} : c == 2 ? Term{0, 0, 1.f} : Term{0, 1, 1.f};
    if (a == 1) return c == 0 ? Term{0, 1, -1.f} : c == 1 ? Term{0, 0, 1.f} : c == 2 ? Term{1, 1, -1.f} : Term{1, 0, 1.f};
    return c == 0 ? Term{2, 0, 1.f} : c == 1 ? Term{2, 1, 1.f} : Term{-1, 0, 0.f};
  }
  // QTEND: a0 = qe (Vd), a1 = qc (Xs), a2 = qm (Us):
  // re = e Vd.re + c Xs.re + mq Us.im, im = e Vd.im + c Xs.im - mq Us.re (qtend.wgsl)
  if (a == 0) return c == 0 ? Term{1, 0, 1.f} : Term{1, 1, 1.f};
  if (a == 1) return c == 0 ? Term{2, 0, 1.f} : Term{2, 1, 1.f};
  return c == 0 ? Term{0, 1, 1.f} : Term{0, 0, -1.f};
}

// Half (0: N + S, 1: N - S) table block a takes for modes with even n - m
// (odd n - m take the other): the shaders' north + s * south with
// s = (-1)^(n - m) picks the sum for even and the difference for odd
// (fc2sp), uv2dv's and qtend's e-terms the opposite.
__host__ __device__ constexpr int even_half(int kind, int a) {
  return (kind == UV2DV || kind == MKTEND || kind == QTEND) && a == 0 ? 1 : 0;
}

__host__ __device__ __forceinline__ int first_mode(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }

// Offset (floats) of (row, k) inside one K step of a K-major, no-swizzle
// operand: core matrices of 8 rows x 16 bytes; the two 16-byte K halves 128
// bytes apart (leading byte offset), 8-row groups 256 bytes apart (stride
// byte offset).
__host__ __device__ __forceinline__ int kmajor_offset(int row, int k) {
  return (row >> 3) * 64 + (k >> 2) * 32 + (row & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100): start address, leading byte
// offset 128, stride byte offset 256 (all >> 4), descriptor version 1, no
// swizzle.
__device__ __forceinline__ uint64_t operand_desc(const void* p) {
  uint64_t d = (uint64_t)((smem_addr(p) >> 4) & 0x3FFF);
  d |= (uint64_t)(128 >> 4) << 16;
  d |= (uint64_t)(256 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor: D F32, A and B TF32, both K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(id), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                   smem_addr(mbar)),
               "r"(bytes)
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

// TMA: a 1-D or 2-D tile of a tensor map into shared memory, completing on
// an mbarrier (no multicast; the map covers this GPU's memory).
__device__ __forceinline__ void tma_load_1d(void* dst, const CUtensorMap* map, int x, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(smem_addr(mbar))
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(mbar))
      : "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(mbar))
      : "memory");
}

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

// Per-launch geometry, computed on the host.
struct TcGeom {
  int planes;       // planes of each field
  int tiles;        // plane tiles (TP planes each)
  int items;        // NTP1 * tiles
  int npad_max;     // table rows of the largest m (the table stage's size)
  int raw_floats;   // floats of one raw stage
  int raw_row;      // inverse: floats per staged plane row (a multiple of 32)
  int box;          // inverse: TMA box width in floats (a multiple of 4)
  int out_plane;    // floats per output plane
  float plavor;     // dv2uv: planetary vorticity removed from mode (0, 1)
  int n_tab;        // table stages in the ring (as many as shared memory holds, 2..kMaxTab)
  int raw2d;        // inverse: the planes' rows arrive as one 2-D box (NRSP * 4 a multiple of 16)
};

struct TcMaps {
  CUtensorMap in[3];
};

struct TcOut {
  float* out[2];
  const float* images;  // this kind's table images
  const int* at;        // float offset of m's images, [NTP1 + 1]
};

// Shared memory carve-up (byte offsets from a 128-byte aligned base).
struct TcSmem {
  size_t tab, data, raw, stage, bars, total;
};

__host__ __device__ inline TcSmem tc_smem(int npad_max, int raw_floats, int n_tab) {
  TcSmem s{};
  s.tab = 0;
  const size_t tab_stage = (size_t)kChunkSteps * npad_max * 2 * kStepK * 4;
  s.data = s.tab + n_tab * tab_stage;
  const size_t data_stage = (size_t)kChunkSteps * 2 * kDataStepFloats * 4;
  // raw stages 1024-byte aligned: the forward kinds' tiles arrive with the
  // 128-byte swizzle, whose pattern repeats every 1024 bytes
  s.raw = (s.data + kNData * data_stage + 1023) / 1024 * 1024;
  s.stage = s.raw + 2 * (size_t)raw_floats * 4;
  s.bars = s.stage + (kConv / 32) * 32 * 33 * 4;
  s.total = s.bars + 32 * 8;
  return s;
}

template <int KIND>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_legendre(const __grid_constant__ TcMaps maps, TcOut io, TcGeom g, int* __restrict__ fault, Dims d) {
  using S = Shape<KIND>;
  extern __shared__ unsigned char smem_raw_base[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw_base) + 1023) & ~(uintptr_t)1023);
  const TcSmem L = tc_smem(g.npad_max, g.raw_floats, g.n_tab);
  const int NT = g.n_tab;
  const size_t tab_stage_floats = (size_t)kChunkSteps * g.npad_max * 2 * kStepK;
  const size_t data_stage_floats = (size_t)kChunkSteps * 2 * kDataStepFloats;
  float* tab = reinterpret_cast<float*>(base + L.tab);
  float* dat = reinterpret_cast<float*>(base + L.data);
  float* raw = reinterpret_cast<float*>(base + L.raw);
  float* stage = reinterpret_cast<float*>(base + L.stage);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + L.bars);
  uint64_t* raw_full = bars;          // [2]
  uint64_t* raw_empty = bars + 2;     // [2]
  uint64_t* tab_full = bars + 4;      // [kMaxTab]
  uint64_t* tab_empty = bars + 12;    // [kMaxTab]
  uint64_t* dat_full = bars + 20;     // [kNData]
  uint64_t* dat_empty = bars + 22;    // [kNData]
  uint64_t* acc_full = bars + 24;     // [2]
  uint64_t* acc_empty = bars + 26;    // [2]
  uint64_t* drain = bars + 28;        // MMA drain after an abort
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 29);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 30);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 32) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(raw_full + i, 1);
      mbar_init(raw_empty + i, kConv);
      mbar_init(acc_full + i, 1);
      mbar_init(acc_empty + i, kConv);
    }
    for (int i = 0; i < NT; ++i) {
      mbar_init(tab_full + i, 1);
      mbar_init(tab_empty + i, 1);
    }
    for (int i = 0; i < kNData; ++i) {
      mbar_init(dat_full + i, kConv);
      mbar_init(dat_empty + i, 1);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  // Bounded wait: gives up after kWaitLimit polls or when another role
  // aborted, recording the fault once.
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    for (long i = 0; i < kWaitLimit; ++i) {
      if (mbar_try_wait(bar, parity)) return true;
      if ((i & 255) == 255 && *abort_flag) return false;
    }
    if (!*abort_flag) {
      *abort_flag = 1;
      atomicExch(fault, 1);
    }
    return false;
  };

  const int ntp1 = d.NTP1;
  const int units = S::fwd ? d.NLAT / 32 : 1;
  // K steps of item m: inverse NA * ceil(K_m / 8) in chunks of 4; forward
  // units * NA chunks of 4.
  auto item_m = [&](int item) { return item % ntp1; };
  auto item_p0 = [&](int item) { return (item / ntp1) * S::TP; };
  auto ks_block = [&](int m) { return (ntp1 - m + kStepK - 1) / kStepK; };
  auto chunks_of = [&](int m) {
    return S::fwd ? units * S::NA : (S::NA * ks_block(m) + kChunkSteps - 1) / kChunkSteps;
  };
  auto npad_of = [&](int m) { return S::fwd ? (ntp1 - m + 15) / 16 * 16 : d.NLAT; };

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    uint32_t ri = 0, ti = 0;
    if (lane == 0) {
      bool ok = true;
      for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x) {
        const int m = item_m(item), p0 = item_p0(item);
        const int np = min(S::TP, g.planes - p0);
        const int nchunks = chunks_of(m), npad = npad_of(m);
        const int total_steps = S::fwd ? nchunks * kChunkSteps : S::NA * ks_block(m);
        const float* img = io.images + io.at[m];
        int chunk = 0;
        for (int u = 0; u < units && ok; ++u) {
          const int rb = ri & 1;
          if (!(ok = wait(raw_empty + rb, ((ri >> 1) & 1) ^ 1))) break;
          float* r = raw + (size_t)rb * g.raw_floats;
          if (S::fwd) {
            // per field: the northern 16 latitudes of the unit's pairs, then
            // the southern 16, each a (32 floats x TP planes) box
            const uint32_t bytes = S::NR * 2 * S::TP * 32 * 4;
            const int xn = 2 * (m * d.NLAT + 16 * u), xs = 2 * (m * d.NLAT + d.NLAT - 16 - 16 * u);
            if ((xn & 3) || (xs & 3)) {  // never: NLAT is a multiple of 16
              *abort_flag = 1;
              atomicExch(fault, 2);
              ok = false;
              break;
            }
            mbar_expect_tx(raw_full + rb, bytes);
            for (int f = 0; f < S::NR; ++f) {
              tma_load_2d(r + (size_t)(2 * f) * S::TP * 32, &maps.in[f], xn, p0, raw_full + rb);
              tma_load_2d(r + (size_t)(2 * f + 1) * S::TP * 32, &maps.in[f], xs, p0, raw_full + rb);
            }
          } else {
            // per field and plane: the modes of m, from the 16-byte boundary
            // at or below the first coefficient
            const int w0 = first_mode(m, ntp1);
            if (g.raw2d) {
              // one (box x TP planes) tile per field: every plane's row starts
              // at the same 16-byte boundary below its first coefficient
              mbar_expect_tx(raw_full + rb, (uint32_t)(S::NR * S::TP * g.box * 4));
              for (int f = 0; f < S::NR; ++f)
                tma_load_2d(r + (size_t)f * S::TP * g.raw_row, &maps.in[f], (2 * w0) & ~3, p0, raw_full + rb);
            } else {
              mbar_expect_tx(raw_full + rb, (uint32_t)(S::NR * np * g.box * 4));
              for (int f = 0; f < S::NR; ++f)
                for (int p = 0; p < np; ++p) {
                  const int x = ((p0 + p) * d.NRSP + 2 * w0) & ~3;
                  tma_load_1d(r + ((size_t)f * S::TP + p) * g.raw_row, &maps.in[f], x, raw_full + rb);
                }
            }
          }
          ++ri;
          const int per_unit = S::fwd ? S::NA : nchunks;
          for (int c = 0; c < per_unit && ok; ++c, ++chunk) {
            const int ts = ti % NT;
            if (!(ok = wait(tab_empty + ts, ((ti / NT) & 1) ^ 1))) break;
            const int s0 = chunk * kChunkSteps, ns = min(kChunkSteps, total_steps - s0);
            const uint32_t bytes = (uint32_t)ns * npad * 2 * kStepK * 4;
            mbar_expect_tx(tab_full + ts, bytes);
            bulk_load(tab + ts * tab_stage_floats, img + (size_t)s0 * npad * 2 * kStepK, bytes, tab_full + ts);
            ++ti;
          }
        }
      }
      // Loads in flight land before the CTA ends: wait for the last phase
      // armed on each stage (bounded; loads complete on their own).
      if (*abort_flag) {
        for (uint32_t k = (ri > 2 ? ri - 2 : 0); k < ri; ++k)
          for (long i = 0; i < kWaitLimit && !mbar_try_wait(raw_full + (k & 1), (k >> 1) & 1); ++i) {
          }
        for (uint32_t k = (ti > (uint32_t)NT ? ti - NT : 0); k < ti; ++k)
          for (long i = 0; i < kWaitLimit && !mbar_try_wait(tab_full + k % NT, (k / NT) & 1); ++i) {
          }
      }
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      uint32_t ti = 0, di = 0, ii = 0;
      bool ok = true, issued = false;
      for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x, ++ii) {
        const int m = item_m(item);
        const int nchunks = chunks_of(m), npad = npad_of(m);
        const int total_steps = S::fwd ? nchunks * kChunkSteps : S::NA * ks_block(m);
        const int ab = ii & 1;
        if (!(ok = wait(acc_empty + ab, ((ii >> 1) & 1) ^ 1))) break;
        fence_after_sync();
        const uint32_t dtm = tmem + (uint32_t)(ab * 128);
        const uint32_t id = idesc(npad);
        for (int c = 0; c < nchunks && ok; ++c) {
          const int ts = ti % NT, ds = di % kNData;
          if (!(ok = wait(tab_full + ts, (ti / NT) & 1))) break;
          if (!(ok = wait(dat_full + ds, (di / kNData) & 1))) break;
          fence_after_sync();
          const int ns = min(kChunkSteps, total_steps - c * kChunkSteps);
          const float* tb = tab + ts * tab_stage_floats;
          const float* db = dat + ds * data_stage_floats;
          for (int s = 0; s < ns; ++s) {
            const float* th = tb + (size_t)s * npad * 2 * kStepK;
            const float* tl = th + (size_t)npad * kStepK;
            const float* dh = db + (size_t)s * 2 * kDataStepFloats;
            const float* dl = dh + kDataStepFloats;
            const uint64_t ah = operand_desc(dh), al = operand_desc(dl);
            const uint64_t bh = operand_desc(th), bl = operand_desc(tl);
            mma_tf32(dtm, ah, bh, id, (c > 0 || s > 0) ? 1u : 0u);
            mma_tf32(dtm, ah, bl, id, 1u);
            mma_tf32(dtm, al, bh, id, 1u);
            issued = true;
          }
          mma_commit(tab_empty + ts);
          mma_commit(dat_empty + ds);
          ++ti;
          ++di;
        }
        if (ok) mma_commit(acc_full + ab);
      }
      if (*abort_flag && issued) {
        // MMAs in flight finish before the tensor memory is freed.
        mma_commit(drain);
        for (long i = 0; i < kWaitLimit && !mbar_try_wait(drain, 0); ++i) {
        }
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------ converters and epilogue
    const int t = threadIdx.x - 32;  // 0..255
    const int q = warp & 3;          // TMEM lane quarter of this warp
    const int half = (warp - 1) >> 2;  // the two warps of a quarter drain alternate 32-column slices
    // Each converter thread builds one row's run of four K indices per K
    // step: in the K-major layout (kmajor_offset) the floats 4 t .. 4 t + 3
    // of a step are row (t >> 4) * 8 + (t & 7), K indices 4 ((t >> 3) & 1) +
    // 0..3, so a thread writes one 16-byte hi and one 16-byte lo vector and a
    // warp 512 contiguous bytes. Its row's output column row % NC, and so
    // its term of every table block, is fixed.
    const int row_of_thread = (t >> 4) * 8 + (t & 7);
    const int kg_of_thread = (t >> 3) & 1;
    const int c_of_thread = row_of_thread % S::NC;
    const int p_of_thread = row_of_thread / S::NC;
    float* st = stage + (size_t)(warp - 1) * 32 * 33;
    uint32_t ri = 0, di = 0, ii = 0;
    bool ok = true;
    int prev_item = -1;
    // Drains accumulator ab of item `it`: row n = 32 q + lane holds (plane
    // n / NC, column n % NC); each 32-column slice passes through shared
    // memory so a warp stores each plane's run of 64 floats in 128-byte lines.
    auto epilogue = [&](int it, uint32_t iidx) -> bool {
      const int ab = iidx & 1;
      if (!wait(acc_full + ab, (iidx >> 1) & 1)) return false;
      fence_after_sync();
      const int m = item_m(it), p0 = item_p0(it);
      const int w0 = first_mode(m, ntp1);
      const int ncols = S::fwd ? ntp1 - m : d.NLAT;
      const size_t out_base = S::fwd ? (size_t)2 * w0 : (size_t)2 * m * d.NLAT;
      constexpr int PPW = 32 / S::NC;  // planes per warp
      for (int c0 = 32 * half; c0 < ncols; c0 += 64) {
        float v[32];
        tmem_load32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * 128 + c0), v);
#pragma unroll
        for (int k = 0; k < 32; ++k) st[lane * 33 + k] = v[k];
        __syncwarp();
        const int nvalid = 2 * min(32, ncols - c0);
        for (int pp = 0; pp < PPW; ++pp) {
          const int plane = p0 + q * PPW + pp;
          if (plane >= g.planes) break;
#pragma unroll
          for (int o = 0; o < S::NOUT; ++o) {
            float* dst = io.out[o] + (size_t)plane * g.out_plane + out_base + 2 * c0;
            const int row = pp * S::NC + 2 * o;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int e = lane + 32 * h;
              if (e < nvalid) dst[e] = st[(row + (e & 1)) * 33 + (e >> 1)];
            }
          }
        }
        __syncwarp();
      }
      fence_before_sync();
      mbar_arrive(acc_empty + ab);
      return true;
    };
    for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x, ++ii) {
      const int m = item_m(item), p0 = item_p0(item);
      const int np = min(S::TP, g.planes - p0);
      const int nchunks = chunks_of(m);
      const int K = ntp1 - m, ksb = ks_block(m);
      const int total_steps = S::fwd ? nchunks * kChunkSteps : S::NA * ksb;
      const int w0 = first_mode(m, ntp1);
      int chunk = 0;
      for (int u = 0; u < units && ok; ++u) {
        const int rb = ri & 1;
        if (!(ok = wait(raw_full + rb, (ri >> 1) & 1))) break;
        const float* r = raw + (size_t)rb * g.raw_floats;
        const int per_unit = S::fwd ? S::NA : nchunks;
        for (int cc = 0; cc < per_unit && ok; ++cc, ++chunk) {
          const int ds = di % kNData;
          if (!(ok = wait(dat_empty + ds, ((di / kNData) & 1) ^ 1))) break;
          float* db = dat + ds * data_stage_floats;
          const int s0 = chunk * kChunkSteps, ns = min(kChunkSteps, total_steps - s0);
#pragma unroll
          for (int s = 0; s < kChunkSteps; ++s) {
            if (s >= ns) break;
            float4* dh = reinterpret_cast<float4*>(db + (size_t)s * 2 * kDataStepFloats) + t;
            float4* dl = reinterpret_cast<float4*>(db + (size_t)s * 2 * kDataStepFloats + kDataStepFloats) + t;
            const int gstep = s0 + s;
            const int a = S::fwd ? chunk % S::NA : gstep / ksb;
            const Term tm = term<KIND>(a, c_of_thread);
            const int p = p_of_thread;
            float x[4] = {0.f, 0.f, 0.f, 0.f};
            if (p < np) {
              if (S::fwd) {
                if (tm.field >= 0) {
                  // K indices 8 s + 4 kg + j of the unit's 32: half kk >> 4, pair kk & 15
                  const int kk0 = 8 * s + 4 * kg_of_thread, half = kk0 >> 4, li0 = kk0 & 15;
                  // rows of 32 floats, 16-byte chunks XOR-swizzled by the row
                  // index (the tile's 128-byte swizzle)
                  const int rown = 2 * tm.field * S::TP + p, rows = rown + S::TP;
                  const float* rn = r + (size_t)rown * 32;
                  const float* rs = r + (size_t)rows * 32;
#pragma unroll
                  for (int j = 0; j < 4; ++j) {
                    const int en = 2 * (li0 + j) + tm.comp, es = 2 * (15 - li0 - j) + tm.comp;
                    const float north = rn[(((en >> 2) ^ (rown & 7)) << 2) | (en & 3)];
                    const float south = rs[(((es >> 2) ^ (rows & 7)) << 2) | (es & 3)];
                    x[j] = tm.sign * (half == 0 ? north + south : north - south);
                  }
                }
              } else {
                const int t0 = (gstep % ksb) * kStepK + 4 * kg_of_thread;  // mode n - m of j = 0
                const int off = ((g.raw2d ? 0 : (p0 + p) * d.NRSP) + 2 * w0) & 3;
                const float* rr = r + ((size_t)tm.field * S::TP + p) * g.raw_row + off + tm.comp;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                  const int tmode = t0 + j;
                  float v = tmode < K ? rr[2 * tmode] : 0.f;
                  if (KIND == DV2UV && tm.field == 1 && tm.comp == 0 && m == 0 && tmode == 1) v -= g.plavor;
                  x[j] = tm.sign * v;
                }
              }
            }
            float4 h, l;
            h.x = tf32_round(x[0]);
            h.y = tf32_round(x[1]);
            h.z = tf32_round(x[2]);
            h.w = tf32_round(x[3]);
            l.x = tf32_round(x[0] - h.x);
            l.y = tf32_round(x[1] - h.y);
            l.z = tf32_round(x[2] - h.z);
            l.w = tf32_round(x[3] - h.w);
            *dh = h;
            *dl = l;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
          mbar_arrive(dat_full + ds);
          ++di;
        }
        mbar_arrive(raw_empty + rb);
        ++ri;
      }
      if (!ok) break;
      // drain the previous item while the tensor cores run this one
      if (prev_item >= 0 && !(ok = epilogue(prev_item, ii - 1))) break;
      prev_item = item;
    }
    if (ok && prev_item >= 0) epilogue(prev_item, ii - 1);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// ----------------------------------------------------------------- host

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      throw std::runtime_error("cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// 1-D map over a spectral field of `planes` planes, boxes of `box` floats.
CUtensorMap map_1d(const float* field, size_t floats, int box) {
  CUtensorMap map;
  const cuuint64_t dim[1] = {floats};
  const cuuint64_t stride[1] = {floats * 4};  // unused at rank 1
  const cuuint32_t bdim[1] = {(cuuint32_t)box}, estride[1] = {1};
  if ((reinterpret_cast<uintptr_t>(field) & 15) || (box * 4) % 16 || box > 256)
    throw std::runtime_error("tensor-core transform: bad 1-D map");
  const CUresult r = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 1, const_cast<float*>(field), dim, stride, bdim,
                               estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled (1-D) failed: " + std::to_string((int)r));
  return map;
}

// 2-D map over a field of `planes` planes of `plane_floats` floats, boxes of
// `box` floats x tp planes.
CUtensorMap map_2d(const float* field, int plane_floats, int planes, int box, int tp, bool swizzle = false) {
  CUtensorMap map;
  const cuuint64_t dim[2] = {(cuuint64_t)plane_floats, (cuuint64_t)planes};
  const cuuint64_t stride[1] = {(cuuint64_t)plane_floats * 4};
  const cuuint32_t bdim[2] = {(cuuint32_t)box, (cuuint32_t)tp}, estride[2] = {1, 1};
  if ((reinterpret_cast<uintptr_t>(field) & 15) || stride[0] % 16 || (box * 4) % 16 || box > 256 || tp > 256)
    throw std::runtime_error("tensor-core transform: bad 2-D map");
  if (swizzle && box * 4 != 128) throw std::runtime_error("tensor-core transform: 128-byte swizzle needs 128-byte rows");
  const CUresult r = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(field), dim, stride, bdim,
                               estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                               swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled (2-D) failed: " + std::to_string((int)r));
  return map;
}

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return sms;
}

template <int KIND>
TcGeom geometry(const Dims& d, int planes, float plavor) {
  using S = Shape<KIND>;
  TcGeom g{};
  g.planes = planes;
  g.tiles = (planes + S::TP - 1) / S::TP;
  g.items = d.NTP1 * g.tiles;
  g.npad_max = S::fwd ? (d.NTP1 + 15) / 16 * 16 : d.NLAT;
  g.box = (2 * d.NTP1 + 4 + 3) / 4 * 4;
  // a 2-D box lands as TP rows of `box` floats; per-plane 1-D boxes land on
  // 128-byte row starts
  g.raw2d = !S::fwd && (d.NRSP * 4) % 16 == 0 ? 1 : 0;
  g.raw_row = g.raw2d ? g.box : (g.box + 31) / 32 * 32;
  g.raw_floats = S::fwd ? S::NR * 2 * S::TP * 32 : S::NR * S::TP * g.raw_row;
  g.raw_floats = (g.raw_floats + 31) / 32 * 32;
  g.out_plane = S::fwd ? d.NRSP : d.NLAT * d.NFC;
  g.plavor = plavor;
  // as many table stages as shared memory holds
  g.n_tab = 2;
  while (g.n_tab < kMaxTab && tc_smem(g.npad_max, g.raw_floats, g.n_tab + 1).total + 1024 <= kTcSmemLimit) ++g.n_tab;
  return g;
}

template <int KIND>
size_t smem_bytes(const TcGeom& g) {
  return tc_smem(g.npad_max, g.raw_floats, g.n_tab).total + 1024;
}

template <int KIND>
void launch(const Model& m, const float* const* in, float* out0, float* out1, int planes, int set, float plavor,
            cudaStream_t st) {
  using S = Shape<KIND>;
  const Dims& d = m.d;
  const TcGeom g = geometry<KIND>(d, planes, plavor);
  TcMaps maps{};
  for (int f = 0; f < S::NR; ++f)
    maps.in[f] = S::fwd    ? map_2d(in[f], d.NLAT * d.NFC, planes, 32, S::TP, true)
                 : g.raw2d ? map_2d(in[f], d.NRSP, planes, g.box, S::TP)
                           : map_1d(in[f], (size_t)planes * d.NRSP, g.box);
  TcOut io{};
  io.out[0] = out0;
  io.out[1] = out1;
  io.images = m.sh.tc_img;
  io.at = m.sh.tc_at + (size_t)set * (d.NTP1 + 1);
  const size_t smem = smem_bytes<KIND>(g);
  if (smem > kTcSmemLimit) throw std::runtime_error("tensor-core transform: shared memory over budget");
  const int grid = std::min(g.items, sm_count());
  k_tc_legendre<KIND><<<grid, kThreads, smem, st>>>(maps, io, g, m.fault, d);
}

// Table image sets, in the order of the at[] rows.
enum ImageSet : int { SET_QI = 0, SET_QJ, SET_DV2UV, SET_FC2SP, SET_UV2DV, SET_MKTEND, SET_QTEND, SET_COUNT };

}  // namespace

void tc_init() {
  const int limit = 227 * 1024;
  cudaFuncSetAttribute(k_tc_legendre<INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  cudaFuncSetAttribute(k_tc_legendre<DV2UV>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  cudaFuncSetAttribute(k_tc_legendre<FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  cudaFuncSetAttribute(k_tc_legendre<UV2DV>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  cudaFuncSetAttribute(k_tc_legendre<MKTEND>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  cudaFuncSetAttribute(k_tc_legendre<QTEND>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
}

// Host images of the table operands ([NLAT][NCSP] FP64 tables by name) for
// every kind, m by m, in the kernel's chunk order: each K step holds the hi
// image (npad rows x 8, K-major no-swizzle) then the lo image, hi = the FP64
// value rounded to TF32 and lo = the remainder rounded to TF32. `at` gets
// SET_COUNT rows of NTP1 + 1 float offsets (the last: the row's end).
std::vector<float> tc_table_images(const Dims& d, const std::map<std::string, std::vector<double>>& q,
                                   std::vector<int>& at) {
  auto tf32 = [](double v) {
    float x = (float)v;
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & ~0x1FFFu;  // nearest, ties away from zero
    float y;
    std::memcpy(&y, &u, 4);
    return y;
  };
  const int ntp1 = d.NTP1, JH = d.NLAT / 2;
  std::vector<float> out;
  at.assign((size_t)SET_COUNT * (ntp1 + 1), 0);
  // value(m, a, col, k_in_block): the table entry of block a for output
  // column col (latitude or mode) at K index k of the block.
  struct SetDef {
    int kind;
    std::vector<const std::vector<double>*> tabs;
  };
  const SetDef sets[SET_COUNT] = {
      {INV, {&q.at("qi")}},
      {INV, {&q.at("qj")}},
      {DV2UV, {&q.at("qv"), &q.at("qu")}},
      {FWD, {&q.at("qc")}},
      {UV2DV, {&q.at("qe"), &q.at("qm")}},
      {MKTEND, {&q.at("qe"), &q.at("qm"), &q.at("qq")}},
      {QTEND, {&q.at("qe"), &q.at("qc"), &q.at("qm")}},
  };
  for (int set = 0; set < SET_COUNT; ++set) {
    const SetDef& sd = sets[set];
    const bool fwd = sd.kind >= FWD;
    const int NA = (int)sd.tabs.size();
    for (int m = 0; m < ntp1; ++m) {
      while (out.size() % 4) out.push_back(0.f);
      at[(size_t)set * (ntp1 + 1) + m] = (int)out.size();
      const int K = ntp1 - m, w0 = first_mode(m, ntp1);
      const int npad = fwd ? (K + 15) / 16 * 16 : d.NLAT;
      // the K steps in chunk order, each as (block a, K indices)
      std::vector<std::pair<int, int>> steps;  // (a, step index within the block's K)
      if (fwd) {
        for (int u = 0; u < d.NLAT / 32; ++u)
          for (int a = 0; a < NA; ++a)
            for (int j = 0; j < kChunkSteps; ++j) steps.push_back({a, u * kChunkSteps + j});
      } else {
        const int ksb = (K + kStepK - 1) / kStepK;
        for (int a = 0; a < NA; ++a)
          for (int j = 0; j < ksb; ++j) steps.push_back({a, j});
      }
      for (const auto& sa : steps) {
        const int a = sa.first, j = sa.second;
        std::vector<float> hi((size_t)npad * kStepK, 0.f), lo((size_t)npad * kStepK, 0.f);
        const std::vector<double>& tab = *sd.tabs[a];
        for (int col = 0; col < npad; ++col)
          for (int k = 0; k < kStepK; ++k) {
            double v = 0.0;
            if (fwd) {
              // unit u = j / 4, K index kk of the unit's 32: half, pair
              const int u = j / kChunkSteps, kk = (j % kChunkSteps) * kStepK + k;
              const int half = kk / 16, l = 16 * u + kk % 16;
              const int t = col;
              if (t < K && l < JH && half == (even_half(sd.kind, a) ^ (t & 1)))
                v = tab[(size_t)l * d.NCSP + w0 + t];
            } else {
              const int t = j * kStepK + k, lat = col;
              if (t < K && lat < d.NLAT) v = tab[(size_t)lat * d.NCSP + w0 + t];
            }
            const float h = tf32(v);
            const size_t o = kmajor_offset(col, k);
            hi[o] = h;
            lo[o] = tf32(v - (double)h);
          }
        out.insert(out.end(), hi.begin(), hi.end());
        out.insert(out.end(), lo.begin(), lo.end());
      }
    }
    while (out.size() % 4) out.push_back(0.f);
    at[(size_t)set * (ntp1 + 1) + ntp1] = (int)out.size();
  }
  return out;
}

void tc_inverse(const Model& m, const float* s, float* f, int planes, bool derivative, cudaStream_t st) {
  const float* in[1] = {s};
  launch<INV>(m, in, f, nullptr, planes, derivative ? SET_QJ : SET_QI, 0.f, st);
}

void tc_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
              cudaStream_t st) {
  const float* in[2] = {D, Z};
  launch<DV2UV>(m, in, U, V, planes, SET_DV2UV, plavor, st);
}

void tc_forward(const Model& m, const float* f, float* s, int planes, cudaStream_t st) {
  const float* in[1] = {f};
  launch<FWD>(m, in, s, nullptr, planes, SET_FC2SP, 0.f, st);
}

void tc_uv2dv(const Model& m, const float* u, const float* v, const float* ke, float* D, float* Z, int planes,
              cudaStream_t st) {
  if (ke) {
    const float* in[3] = {u, v, ke};
    launch<MKTEND>(m, in, D, Z, planes, SET_MKTEND, 0.f, st);
  } else {
    const float* in[2] = {u, v};
    launch<UV2DV>(m, in, D, Z, planes, SET_UV2DV, 0.f, st);
  }
}

void tc_qtend(const Model& m, const float* u, const float* v, const float* src, float* out, int planes,
              cudaStream_t st) {
  const float* in[3] = {u, v, src};
  launch<QTEND>(m, in, out, nullptr, planes, SET_QTEND, 0.f, st);
}

}  // namespace exogcm
