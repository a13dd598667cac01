// Longitude transforms as register FFTs, T threads per latitude row (the
// optimized path).
//
// Same results as the truncated DFT of fourier/index.ts:19-36 (gp2fc keeps
// c_m = (1/N) sum_j g_j e^{-i m lambda_j} for m <= NTRU; fc2gp sums
// Re c_0 + 2 Re sum_{m>=1} c_m e^{i m lambda_j}, ignoring Im c_0), computed in
// O(N log N): a real row of N = 2M points is packed as z_n = g_2n + i g_2n+1,
// transformed by an M-point complex FFT, and split into the even/odd halves.
//
// The M-point FFT is the four-step factorisation M = 8 Q (Q = 4, 8, 12 for
// T21, T42, T63): with n = Q p + q and k = k1 + 8 k2,
//   A[q][k1] = sum_p z[Q p + q] w_8^{p k1}          (Q DFT-8s)
//   B[q][k1] = A[q][k1] w_M^{q k1}                  (twiddle)
//   Z[k1 + 8 k2] = sum_q B[q][k1] w_Q^{q k2}        (8 DFT-Qs)
// A row's T threads (consecutive lanes of one warp) each run Q/T DFT-8s and
// 8/T DFT-Qs in registers; B passes between them through shared memory at
// position 9 q + k1, a pitch that keeps every 64-bit access of a half-warp on
// distinct banks. Twiddles come from a table of e^{2 pi i j / N} built in FP64
// on the host and rounded once.
//
// Fourier planes are m-major on this path (coefficient (m, lat) at
// 2 * (m * NLAT + lat)). A block transforms `rows` consecutive latitudes of
// one plane; the chunk's coefficients pass through shared memory
// ([m][pitch]) so that the m-major side is read and written in runs of
// `rows` latitudes.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "fft_core.cuh"
#include "launch.h"

namespace exogcm {

namespace {

using namespace fftcore;

constexpr int kMaxThreads = 512;

// gp2fc: rows of N grid values -> m-major coefficients.
template <int Q>
__global__ void __launch_bounds__(kMaxThreads) k_fft_forward(const float* __restrict__ g, float* __restrict__ c,
                                                             const float2* __restrict__ twg, int nlat, int rows) {
  using Sh = Shape<Q>;
  constexpr int T = Sh::T, N = Sh::N, NTP1 = Sh::NTP1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* twq = tw + N;
  float2* xb = twq + 9 * Q;
  float2* fc = xb + rows * Sh::XP;
  const int pitch = fc_pitch(rows, T);
  const int chunks = nlat / rows;
  const size_t plane = blockIdx.x / chunks;
  const int lat0 = (blockIdx.x % chunks) * rows;
  const int r = threadIdx.x / T, t = threadIdx.x % T;
  // z_n = g_2n + i g_2n+1 for n = Q p + q
  const float2* in = reinterpret_cast<const float2*>(g + (plane * nlat + lat0 + r) * N);
  float2 a[Sh::QT][8];
#pragma unroll
  for (int i = 0; i < Sh::QT; ++i)
#pragma unroll
    for (int p = 0; p < 8; ++p) a[i][p] = in[Q * p + t + T * i];
  load_twiddles<Q>(twg, tw, twq);
  __syncthreads();
  float2* xr = xb + r * Sh::XP;
  float2 b[Sh::KT][Q];
  four_step<Q, -1>(a, b, twq, xr, t);
  // The split needs Z[m] and Z[(M - m) mod M] for m = t + T i. This thread
  // holds Z[t + T j + 8 k2] in b[j][k2], so Z[m] is its own b[i % KT][i / KT];
  // for t > 0 the partner value is b[KT-1-j][Q-1-k2] of lane T - t of the
  // row's group (a shuffle), and for t = 0 it is this thread's own.
  const float inv_n = 1.f / (float)N;
  const int lane = threadIdx.x & 31, src = lane - t + (T - t) % T;
#pragma unroll
  for (int i = 0; i < (NTP1 + T - 1) / T; ++i) {
    constexpr int KT = Sh::KT;
    const int j = i % KT, k2 = i / KT;
    const float2 send = b[KT - 1 - j][Q - 1 - k2];
    float2 partner;
    partner.x = __shfl_sync(0xffffffffu, send.x, src);
    partner.y = __shfl_sync(0xffffffffu, send.y, src);
    if (t == 0) partner = j == 0 ? b[0][(Q - k2) % Q] : b[j][Q - 1 - k2];
    const int m = t + T * i;
    if (m < NTP1) {
      const float2 zm = b[j][k2];
      const float2 zc = conj2(partner);
      const float2 even = make_float2(0.5f * (zm.x + zc.x), 0.5f * (zm.y + zc.y));
      // (zm - zc) / 2i = ((zm - zc).y, -(zm - zc).x) / 2
      const float2 odd = make_float2(0.5f * (zm.y - zc.y), -0.5f * (zm.x - zc.x));
      const float2 gm = cadd(even, cmulc(odd, tw[m]));
      fc[m * pitch + r] = make_float2(gm.x * inv_n, m == 0 ? 0.f : gm.y * inv_n);
    }
  }
  __syncthreads();
  // rows * T threads: thread (m0, lat) writes m = m0, m0 + T, ...
  const int lat = threadIdx.x % rows, m0 = threadIdx.x / rows;
  float2* out = reinterpret_cast<float2*>(c) + plane * nlat * NTP1 + lat0 + lat;
#pragma unroll 4
  for (int m = m0; m < NTP1; m += T) out[(size_t)m * nlat] = fc[m * pitch + lat];
}

// fc2gp: m-major coefficients -> rows of N grid values.
template <int Q>
__global__ void __launch_bounds__(kMaxThreads) k_fft_inverse(const float* __restrict__ c, float* __restrict__ g,
                                                             const float2* __restrict__ twg, int nlat, int rows) {
  using Sh = Shape<Q>;
  constexpr int T = Sh::T, M = Sh::M, N = Sh::N, NTP1 = Sh::NTP1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* twq = tw + N;
  float2* xb = twq + 9 * Q;
  float2* fc = xb + rows * Sh::XP;
  const int pitch = fc_pitch(rows, T);
  const int chunks = nlat / rows;
  const size_t plane = blockIdx.x / chunks;
  const int lat0 = (blockIdx.x % chunks) * rows;
  {
    // rows * T threads: thread (m0, lat) stages m = m0, m0 + T, ... < NTP1;
    // Im c_0 is ignored.
    const int lat = threadIdx.x % rows, m0 = threadIdx.x / rows;
    const float2* src = reinterpret_cast<const float2*>(c) + plane * nlat * NTP1 + lat0 + lat;
#pragma unroll 4
    for (int m = m0; m < NTP1; m += T) {
      float2 v = src[(size_t)m * nlat];
      if (m == 0) v.y = 0.f;
      fc[m * pitch + lat] = v;
    }
  }
  load_twiddles<Q>(twg, tw, twq);
  __syncthreads();
  const int r = threadIdx.x / T, t = threadIdx.x % T;
  float2 a[Sh::QT][8];
#pragma unroll
  for (int i = 0; i < Sh::QT; ++i)
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      // c_k is zero from NTP1 on (k = 0 reads c_M = 0); for most p the
      // bounds are settled at compile time, t being below T
      const int k = Q * p + t + T * i, km = M - k;
      const float2 gk = k < NTP1 ? fc[k * pitch + r] : make_float2(0.f, 0.f);
      const float2 gmk = conj2(km < NTP1 ? fc[km * pitch + r] : make_float2(0.f, 0.f));
      const float2 e = cadd(gk, gmk);
      const float2 o = cmul(csub(gk, gmk), tw[k]);
      a[i][p] = make_float2(e.x - o.y, e.y + o.x);  // e + i o
    }
  float2* xr = xb + r * Sh::XP;
  float2 b[Sh::KT][Q];
  four_step<Q, 1>(a, b, twq, xr, t);
  float2* out = reinterpret_cast<float2*>(g + (plane * nlat + lat0 + r) * N);
#pragma unroll
  for (int j = 0; j < Sh::KT; ++j)
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) out[t + T * j + 8 * k2] = b[j][k2];
}

// Persistent forms of the two kernels (chosen per shape by the autotuner):
// a block loads the twiddles once and loops over chunks `items` = planes x
// chunks apart by the grid size, loading the next chunk's inputs into
// registers while it finishes the current one. Each row's arithmetic is the
// per-chunk kernels', so the results are the same bit for bit.
template <int Q>
__global__ void __launch_bounds__(kMaxThreads) k_fft_forward_persistent(const float* __restrict__ g,
                                                                        float* __restrict__ c,
                                                                        const float2* __restrict__ twg, int nlat,
                                                                        int rows, int items) {
  using Sh = Shape<Q>;
  constexpr int T = Sh::T, N = Sh::N, NTP1 = Sh::NTP1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* twq = tw + N;
  float2* xb = twq + 9 * Q;
  float2* fc = xb + rows * Sh::XP;
  const int pitch = fc_pitch(rows, T);
  const int chunks = nlat / rows;
  const int r = threadIdx.x / T, t = threadIdx.x % T;
  float2 a[Sh::QT][8];
  auto load = [&](int item) {
    const size_t plane = item / chunks;
    const int lat0 = (item % chunks) * rows;
    const float2* in = reinterpret_cast<const float2*>(g + (plane * nlat + lat0 + r) * N);
#pragma unroll
    for (int i = 0; i < Sh::QT; ++i)
#pragma unroll
      for (int p = 0; p < 8; ++p) a[i][p] = in[Q * p + t + T * i];
  };
  int item = blockIdx.x;
  if (item >= items) return;
  load(item);
  load_twiddles<Q>(twg, tw, twq);
  __syncthreads();
  float2* xr = xb + r * Sh::XP;
  const float inv_n = 1.f / (float)N;
  const int lane = threadIdx.x & 31, src = lane - t + (T - t) % T;
  for (; item < items; item += gridDim.x) {
    const size_t plane = item / chunks;
    const int lat0 = (item % chunks) * rows;
    float2 b[Sh::KT][Q];
    four_step<Q, -1>(a, b, twq, xr, t);
    if (item + (int)gridDim.x < items) load(item + gridDim.x);
    // the split of k_fft_forward
#pragma unroll
    for (int i = 0; i < (NTP1 + T - 1) / T; ++i) {
      constexpr int KT = Sh::KT;
      const int j = i % KT, k2 = i / KT;
      const float2 send = b[KT - 1 - j][Q - 1 - k2];
      float2 partner;
      partner.x = __shfl_sync(0xffffffffu, send.x, src);
      partner.y = __shfl_sync(0xffffffffu, send.y, src);
      if (t == 0) partner = j == 0 ? b[0][(Q - k2) % Q] : b[j][Q - 1 - k2];
      const int m = t + T * i;
      if (m < NTP1) {
        const float2 zm = b[j][k2];
        const float2 zc = conj2(partner);
        const float2 even = make_float2(0.5f * (zm.x + zc.x), 0.5f * (zm.y + zc.y));
        const float2 odd = make_float2(0.5f * (zm.y - zc.y), -0.5f * (zm.x - zc.x));
        const float2 gm = cadd(even, cmulc(odd, tw[m]));
        fc[m * pitch + r] = make_float2(gm.x * inv_n, m == 0 ? 0.f : gm.y * inv_n);
      }
    }
    __syncthreads();
    const int lat = threadIdx.x % rows, m0 = threadIdx.x / rows;
    float2* out = reinterpret_cast<float2*>(c) + plane * nlat * NTP1 + lat0 + lat;
#pragma unroll 4
    for (int m = m0; m < NTP1; m += T) out[(size_t)m * nlat] = fc[m * pitch + lat];
    __syncthreads();  // the next chunk's split rewrites fc
  }
}

template <int Q>
__global__ void __launch_bounds__(kMaxThreads) k_fft_inverse_persistent(const float* __restrict__ c,
                                                                        float* __restrict__ g,
                                                                        const float2* __restrict__ twg, int nlat,
                                                                        int rows, int items) {
  using Sh = Shape<Q>;
  constexpr int T = Sh::T, M = Sh::M, N = Sh::N, NTP1 = Sh::NTP1;
  constexpr int KS = (NTP1 + T - 1) / T;  // coefficients a thread stages
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* twq = tw + N;
  float2* xb = twq + 9 * Q;
  float2* fc = xb + rows * Sh::XP;
  const int pitch = fc_pitch(rows, T);
  const int chunks = nlat / rows;
  // rows * T threads: thread (m0, lat) stages m = m0 + T k < NTP1
  const int lat = threadIdx.x % rows, m0 = threadIdx.x / rows;
  float2 v[KS];
  auto load = [&](int item) {
    const size_t plane = item / chunks;
    const int lat0 = (item % chunks) * rows;
    const float2* src = reinterpret_cast<const float2*>(c) + plane * nlat * NTP1 + lat0 + lat;
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const int m = m0 + T * k;
      v[k] = m < NTP1 ? src[(size_t)m * nlat] : make_float2(0.f, 0.f);
    }
  };
  int item = blockIdx.x;
  if (item >= items) return;
  load(item);
  load_twiddles<Q>(twg, tw, twq);
  const int r = threadIdx.x / T, t = threadIdx.x % T;
  float2* xr = xb + r * Sh::XP;
  for (; item < items; item += gridDim.x) {
    const size_t plane = item / chunks;
    const int lat0 = (item % chunks) * rows;
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const int m = m0 + T * k;
      if (m < NTP1) fc[m * pitch + lat] = m == 0 ? make_float2(v[k].x, 0.f) : v[k];  // Im c_0 is ignored
    }
    __syncthreads();
    if (item + (int)gridDim.x < items) load(item + gridDim.x);
    // the row transform of k_fft_inverse
    float2 a[Sh::QT][8];
#pragma unroll
    for (int i = 0; i < Sh::QT; ++i)
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int k = Q * p + t + T * i, km = M - k;
        const float2 gk = k < NTP1 ? fc[k * pitch + r] : make_float2(0.f, 0.f);
        const float2 gmk = conj2(km < NTP1 ? fc[km * pitch + r] : make_float2(0.f, 0.f));
        const float2 e = cadd(gk, gmk);
        const float2 o = cmul(csub(gk, gmk), tw[k]);
        a[i][p] = make_float2(e.x - o.y, e.y + o.x);
      }
    float2 b[Sh::KT][Q];
    four_step<Q, 1>(a, b, twq, xr, t);
    float2* out = reinterpret_cast<float2*>(g + (plane * nlat + lat0 + r) * N);
#pragma unroll
    for (int j = 0; j < Sh::KT; ++j)
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) out[t + T * j + 8 * k2] = b[j][k2];
    __syncthreads();  // the next chunk's staging rewrites fc
  }
}

template <typename K>
void allow_plane_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLegSmemLimit);
}

int q_of(const Dims& d) { return d.NLON / 16; }
int t_of(const Dims& d) { return q_of(d) == 8 ? 8 : 4; }

// One block per resident slot (at most one per chunk), each looping over
// the `items` chunks.
template <typename K>
void launch_persistent(K kernel, const float* in, float* out, const float2* tw, int nlat, int rows, unsigned items,
                       int threads, size_t smem, cudaStream_t st) {
  const unsigned grid = std::min<unsigned>(items, persistent_grid((const void*)kernel, threads, smem));
  kernel<<<grid, threads, smem, st>>>(in, out, tw, nlat, rows, (int)items);
}

}  // namespace

void fft_init() {
  allow_plane_smem(k_fft_forward<4>);
  allow_plane_smem(k_fft_forward<8>);
  allow_plane_smem(k_fft_forward<12>);
  allow_plane_smem(k_fft_inverse<4>);
  allow_plane_smem(k_fft_inverse<8>);
  allow_plane_smem(k_fft_inverse<12>);
  allow_plane_smem(k_fft_forward_persistent<4>);
  allow_plane_smem(k_fft_forward_persistent<8>);
  allow_plane_smem(k_fft_forward_persistent<12>);
  allow_plane_smem(k_fft_inverse_persistent<4>);
  allow_plane_smem(k_fft_inverse_persistent<8>);
  allow_plane_smem(k_fft_inverse_persistent<12>);
}

size_t fft_chunk_smem(const Dims& d, int rows) { return chunk_smem(q_of(d), t_of(d), rows); }

// A chunk is `rows` latitudes (m.tune.fft_rows, a multiple of 8 dividing
// NLAT = 32, 64 or 96), one block of rows * T threads.
bool fft_rows_supported(const Dims& d, int rows) {
  return rows % 8 == 0 && rows <= d.NLAT && d.NLAT % rows == 0 && rows * t_of(d) <= kMaxThreads &&
         fft_chunk_smem(d, rows) <= kLegSmemLimit;
}

void fft_forward(const Model& m, const float* g, float* c, int planes, cudaStream_t st) {
  const float2* tw = reinterpret_cast<const float2*>(m.sh.tw);
  const int rows = m.tune.fft_rows;
  const size_t smem = fft_chunk_smem(m.d, rows);
  const unsigned blocks = planes * (m.d.NLAT / rows);
  const int threads = rows * t_of(m.d);
  if (m.tune.fft_persistent[0]) {
    switch (q_of(m.d)) {
      case 4: return launch_persistent(k_fft_forward_persistent<4>, g, c, tw, m.d.NLAT, rows, blocks, threads, smem, st);
      case 8: return launch_persistent(k_fft_forward_persistent<8>, g, c, tw, m.d.NLAT, rows, blocks, threads, smem, st);
      default:
        return launch_persistent(k_fft_forward_persistent<12>, g, c, tw, m.d.NLAT, rows, blocks, threads, smem, st);
    }
  }
  switch (q_of(m.d)) {
    case 4: k_fft_forward<4><<<blocks, threads, smem, st>>>(g, c, tw, m.d.NLAT, rows); break;
    case 8: k_fft_forward<8><<<blocks, threads, smem, st>>>(g, c, tw, m.d.NLAT, rows); break;
    default: k_fft_forward<12><<<blocks, threads, smem, st>>>(g, c, tw, m.d.NLAT, rows); break;
  }
}

void fft_inverse(const Model& m, const float* c, float* g, int planes, cudaStream_t st) {
  const float2* tw = reinterpret_cast<const float2*>(m.sh.tw);
  const int rows = m.tune.fft_rows;
  const size_t smem = fft_chunk_smem(m.d, rows);
  const unsigned blocks = planes * (m.d.NLAT / rows);
  const int threads = rows * t_of(m.d);
  if (m.tune.fft_persistent[1]) {
    switch (q_of(m.d)) {
      case 4: return launch_persistent(k_fft_inverse_persistent<4>, c, g, tw, m.d.NLAT, rows, blocks, threads, smem, st);
      case 8: return launch_persistent(k_fft_inverse_persistent<8>, c, g, tw, m.d.NLAT, rows, blocks, threads, smem, st);
      default:
        return launch_persistent(k_fft_inverse_persistent<12>, c, g, tw, m.d.NLAT, rows, blocks, threads, smem, st);
    }
  }
  switch (q_of(m.d)) {
    case 4: k_fft_inverse<4><<<blocks, threads, smem, st>>>(c, g, tw, m.d.NLAT, rows); break;
    case 8: k_fft_inverse<8><<<blocks, threads, smem, st>>>(c, g, tw, m.d.NLAT, rows); break;
    default: k_fft_inverse<12><<<blocks, threads, smem, st>>>(c, g, tw, m.d.NLAT, rows); break;
  }
}

}  // namespace exogcm
