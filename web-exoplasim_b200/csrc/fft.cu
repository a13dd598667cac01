// Longitude transforms as warp-per-row real FFTs (the optimized path).
//
// Same results as the truncated DFT of fourier/index.ts:19-36 (gp2fc keeps
// c_m = (1/N) sum_j g_j e^{-i m lambda_j} for m <= NTRU; fc2gp sums
// Re c_0 + 2 Re sum_{m>=1} c_m e^{i m lambda_j}, ignoring Im c_0), computed in
// O(N log N): a real row of N = 2M points is packed as z_n = g_2n + i g_2n+1,
// transformed by an M-point complex FFT, and split into the even/odd halves.
// M = 32 R with R = 1, 2, 3 (T21, T42, T63): each lane of a warp holds the R
// elements n1 + 32 n2 of its row; a radix-R step in registers is followed by
// a 32-point decimation-in-frequency FFT across the lanes (five xor-shuffle
// butterfly stages). Twiddles come from a table of e^{2 pi i j / N} built in
// FP64 on the host and rounded once. Warp shuffles put the bit-reversed FFT
// output back in natural order.
//
// The optimized path stores Fourier planes m-major (coefficient (m, lat) at
// 2 * (m * NLAT + lat)), so that the Legendre transforms on either side
// stream whole runs of latitudes. One block transforms a chunk of `rows`
// consecutive latitudes of one plane: the chunk's coefficients pass through
// shared memory ([m][rows + 1]) between that layout (runs of `rows`
// latitudes per m) and the warps' rows, so both global sides stay
// contiguous. Small chunks give many blocks per SM at different phases, so
// one block's loads overlap another's arithmetic.
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kWarps = 4;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conj2(float2 a) { return make_float2(a.x, -a.y); }

// e^{sign 2 pi i t / N} from the table tw[t] = (cos, sin)(2 pi t / N).
template <int SIGN>
__device__ __forceinline__ float2 twiddle(const float2* tw, int t, int N) {
  float2 w = tw[t % N];
  if (SIGN < 0) w.y = -w.y;
  return w;
}

__device__ __forceinline__ int bitrev5(int x) { return __brev(x) >> 27; }

// In-register M-point FFTs of B rows at once (independent instruction
// streams for the shuffle chains): x[b][r] = z_b[lane + 32 r]; on return
// x[b][k2] holds Z_b[R * bitrev5(lane) + k2].
template <int B, int R, int SIGN>
__device__ __forceinline__ void warp_fft(float2 (&x)[B][R], const float2* tw, int N, int lane) {
  // radix-R step per lane, then the twiddle w_M^{n1 k2}
  if (R == 2) {
    const float2 w = twiddle<SIGN>(tw, 2 * lane, N);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const float2 p = x[b][0], q = x[b][1];
      x[b][0] = cadd(p, q);
      x[b][1] = cmul(csub(p, q), w);
    }
  } else if (R == 3) {
    const float2 w3 = twiddle<SIGN>(tw, N / 3, N);      // e^{sign 2 pi i / 3}
    const float2 w32 = twiddle<SIGN>(tw, 2 * N / 3, N); // e^{sign 4 pi i / 3}
    const float2 t1 = twiddle<SIGN>(tw, 2 * lane, N), t2 = twiddle<SIGN>(tw, 4 * lane, N);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const float2 p = x[b][0], q = x[b][1], u = x[b][2];
      x[b][0] = cadd(cadd(p, q), u);
      x[b][1] = cmul(cadd(cadd(p, cmul(q, w3)), cmul(u, w32)), t1);
      x[b][2] = cmul(cadd(cadd(p, cmul(q, w32)), cmul(u, w3)), t2);
    }
  }
  // 32-point DIF across lanes for each of the R sub-sequences
#pragma unroll
  for (int half = 16; half >= 1; half >>= 1) {
    const bool upper = (lane & half) != 0;
    const float2 w = twiddle<SIGN>(tw, (lane & (half - 1)) * (N / (2 * half)), N);
#pragma unroll
    for (int b = 0; b < B; ++b)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        float2 y;
        y.x = __shfl_xor_sync(0xffffffffu, x[b][r].x, half);
        y.y = __shfl_xor_sync(0xffffffffu, x[b][r].y, half);
        x[b][r] = upper ? cmul(csub(y, x[b][r]), w) : cadd(x[b][r], y);
      }
  }
}

constexpr int kRowsPerWarp = 2;

// After warp_fft lane l holds Z[R * bitrev5(l) + r] in x[r]; this returns
// y[r'] = Z[lane + 32 r'] for the calling lane. Element k sits in lane
// bitrev5(k / R), register k % R: R shuffles of every register, one kept.
template <int R>
__device__ __forceinline__ void natural_order(const float2 (&x)[R], float2 (&y)[R], int lane) {
#pragma unroll
  for (int rp = 0; rp < R; ++rp) {
    const int k = lane + 32 * rp;
    const int src = bitrev5(k / R), reg = k % R;
    float2 v = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float a = __shfl_sync(0xffffffffu, x[r].x, src), b = __shfl_sync(0xffffffffu, x[r].y, src);
      if (reg == r) v = make_float2(a, b);
    }
    y[rp] = v;
  }
}

// Work items are (plane, chunk of `rows` latitudes) pairs, walked by
// persistent blocks: while a block transforms one item, cp.async brings the
// next item's input into the other half of its staging memory.
//
// Inverse staging: the chunk's coefficients [ntp1][rows + 2] (a pitch that
// keeps every 16-byte copy aligned). Forward staging: the chunk's grid rows
// [rows][N] (one contiguous run of the plane), plus one output buffer
// [ntp1][rows + 1] for the m-major write.

__host__ __device__ inline int coef_pitch(int rows) { return rows + 2; }

inline size_t inverse_chunk_smem(int nlon, int rows, int ntp1) {
  return ((size_t)nlon + 2 * (size_t)ntp1 * coef_pitch(rows)) * sizeof(float2);
}

inline size_t forward_chunk_smem(int nlon, int rows, int ntp1) {
  return ((size_t)nlon + (size_t)ntp1 * (rows + 1)) * sizeof(float2);
}

// gp2fc for one plane per block: rows of N grid values -> m-major
// coefficients. A warp transforms kRowsPerWarp rows together.
template <int R>
__global__ void __launch_bounds__(kWarps * 32) k_fft_forward(const float* __restrict__ g, float* __restrict__ c,
                                                             const float2* __restrict__ twg, int nlat, int ntp1,
                                                             int rows) {
  constexpr int M = 32 * R, N = 2 * M, B = kRowsPerWarp;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* fc = tw + N;  // [ntp1][rows + 1]
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twg[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float inv_n = 1.f / (float)N;
  const int chunks = nlat / rows;
  const size_t plane = blockIdx.x / chunks;
  const int lat0 = (blockIdx.x % chunks) * rows;
  for (int row0 = warp * B; row0 < rows; row0 += kWarps * B) {
    float2 x[B][R];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const float2* in = reinterpret_cast<const float2*>(g + (plane * nlat + lat0 + row0 + b) * N);
#pragma unroll
      for (int r = 0; r < R; ++r) x[b][r] = in[lane + 32 * r];
    }
    warp_fft<B, R, -1>(x, tw, N, lane);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      float2 y[R];
      natural_order<R>(x[b], y, lane);
#pragma unroll
      for (int rp = 0; rp < R; ++rp) {
        // Z[m] and Z[(M - m) % M] for m = lane + 32 rp: the second sits in
        // lane 32 - lane, register R - 1 - rp (lane 0: lane 0, register
        // (R - rp) % R).
        const float2 zm = y[rp];
        const float ax = __shfl_sync(0xffffffffu, y[R - 1 - rp].x, (32 - lane) & 31);
        const float ay = __shfl_sync(0xffffffffu, y[R - 1 - rp].y, (32 - lane) & 31);
        const float bx = __shfl_sync(0xffffffffu, y[(R - rp) % R].x, 0);
        const float by = __shfl_sync(0xffffffffu, y[(R - rp) % R].y, 0);
        const float2 zc = lane == 0 ? make_float2(bx, -by) : make_float2(ax, -ay);
        const int m = lane + 32 * rp;
        if (m < ntp1) {
          const float2 even = make_float2(0.5f * (zm.x + zc.x), 0.5f * (zm.y + zc.y));
          // (zm - zc) / 2i = ((zm - zc).y, -(zm - zc).x) / 2
          const float2 odd = make_float2(0.5f * (zm.y - zc.y), -0.5f * (zm.x - zc.x));
          const float2 gm = cadd(even, cmul(twiddle<-1>(tw, m, N), odd));
          fc[m * (rows + 1) + row0 + b] = make_float2(gm.x * inv_n, m == 0 ? 0.f : gm.y * inv_n);
        }
      }
    }
  }
  __syncthreads();
  float2* out = reinterpret_cast<float2*>(c) + plane * nlat * ntp1 + lat0;
  for (int i = threadIdx.x; i < ntp1 * rows; i += blockDim.x) {
    const int m = i / rows, lat = i - m * rows;
    out[(size_t)m * nlat + lat] = fc[m * (rows + 1) + lat];
  }
}

// fc2gp: m-major coefficients -> rows of N grid values, kRowsPerWarp rows
// per warp at once.
template <int R>
__global__ void __launch_bounds__(kWarps * 32) k_fft_inverse(const float* __restrict__ c, float* __restrict__ g,
                                                             const float2* __restrict__ twg, int nlat, int ntp1,
                                                             int rows, int items) {
  constexpr int M = 32 * R, N = 2 * M, B = kRowsPerWarp;
  extern __shared__ float4 sm4[];
  float2* tw = reinterpret_cast<float2*>(sm4);
  float2* fcb = tw + N;  // [2][ntp1][pitch]
  const int pitch = coef_pitch(rows);
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twg[i];
  const int chunks = nlat / rows;
  auto stage = [&](int item, float2* buf) {
    const float2* src =
        reinterpret_cast<const float2*>(c) + (size_t)(item / chunks) * nlat * ntp1 + (item % chunks) * rows;
    const int pieces = rows / 2;
    for (int i = threadIdx.x; i < ntp1 * pieces; i += blockDim.x) {
      const int m = i / pieces, q = i - m * pieces;
      cp_async16(buf + m * pitch + 2 * q, src + (size_t)m * nlat + 2 * q);
    }
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int item = blockIdx.x;
  if (item < items) stage(item, fcb);
  cp_async_commit();
  for (int it = 0; item < items; ++it) {
    const float2* fc = fcb + (size_t)(it & 1) * ntp1 * pitch;
    const int next = item + gridDim.x;
    if (next < items) stage(next, fcb + (size_t)((it + 1) & 1) * ntp1 * pitch);
    cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
    const size_t plane = item / chunks;
    const int lat0 = (item % chunks) * rows;
    for (int row0 = warp * B; row0 < rows; row0 += kWarps * B) {
      float2 x[B][R];
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int row = row0 + b;
        auto coef = [&](int k) {
          float2 v = k < ntp1 ? fc[k * pitch + row] : make_float2(0.f, 0.f);
          if (k == 0) v.y = 0.f;  // Im c_0 is ignored
          return v;
        };
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int k = lane + 32 * r;
          const float2 gk = coef(k);
          const float2 gmk = conj2(coef(M - k));
          const float2 e = cadd(gk, gmk);
          const float2 o = cmul(csub(gk, gmk), twiddle<1>(tw, k, N));
          x[b][r] = make_float2(e.x - o.y, e.y + o.x);  // e + i o
        }
      }
      warp_fft<B, R, 1>(x, tw, N, lane);
#pragma unroll
      for (int b = 0; b < B; ++b) {
        float2 y[R];
        natural_order<R>(x[b], y, lane);
        float2* out = reinterpret_cast<float2*>(g + (plane * nlat + lat0 + row0 + b) * N);
#pragma unroll
        for (int r = 0; r < R; ++r) out[lane + 32 * r] = y[r];
      }
    }
    __syncthreads();  // this staging buffer is reused two items on
    item = next;
  }
  cp_async_wait_all();
}

template <typename K>
void allow_plane_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLegSmemLimit);
}

}  // namespace

void fft_init() {
  allow_plane_smem(k_fft_forward<1>);
  allow_plane_smem(k_fft_forward<2>);
  allow_plane_smem(k_fft_forward<3>);
  allow_plane_smem(k_fft_inverse<1>);
  allow_plane_smem(k_fft_inverse<2>);
  allow_plane_smem(k_fft_inverse<3>);
}

size_t fft_chunk_smem(const Dims& d, int rows) {
  return std::max(inverse_chunk_smem(d.NLON, rows, d.NTP1), forward_chunk_smem(d.NLON, rows, d.NTP1));
}

// A chunk is `rows` latitudes (m.tune.fft_rows, a multiple of
// kWarps * kRowsPerWarp = 8 that divides NLAT = 32, 64 or 96).
template <typename K>
void launch_chunks(K kernel, const void* entry, size_t smem, int items, const float* a, float* b, const Model& m,
                   cudaStream_t st) {
  const int grid = std::min(items, persistent_grid(entry, kWarps * 32, smem));
  kernel<<<grid, kWarps * 32, smem, st>>>(a, b, reinterpret_cast<const float2*>(m.sh.tw), m.d.NLAT, m.d.NTP1,
                                          m.tune.fft_rows, items);
}

void fft_forward(const Model& m, const float* g, float* c, int planes, cudaStream_t st) {
  const float2* tw = reinterpret_cast<const float2*>(m.sh.tw);
  const int rows = m.tune.fft_rows;
  const size_t smem = forward_chunk_smem(m.d.NLON, rows, m.d.NTP1);
  const unsigned blocks = planes * (m.d.NLAT / rows);
  switch (m.d.NLON) {
    case 64: k_fft_forward<1><<<blocks, kWarps * 32, smem, st>>>(g, c, tw, m.d.NLAT, m.d.NTP1, rows); break;
    case 128: k_fft_forward<2><<<blocks, kWarps * 32, smem, st>>>(g, c, tw, m.d.NLAT, m.d.NTP1, rows); break;
    default: k_fft_forward<3><<<blocks, kWarps * 32, smem, st>>>(g, c, tw, m.d.NLAT, m.d.NTP1, rows); break;
  }
}

void fft_inverse(const Model& m, const float* c, float* g, int planes, cudaStream_t st) {
  const int rows = m.tune.fft_rows;
  const size_t smem = inverse_chunk_smem(m.d.NLON, rows, m.d.NTP1);
  const int items = planes * (m.d.NLAT / rows);
  switch (m.d.NLON) {
    case 64: launch_chunks(k_fft_inverse<1>, (const void*)k_fft_inverse<1>, smem, items, c, g, m, st); break;
    case 128: launch_chunks(k_fft_inverse<2>, (const void*)k_fft_inverse<2>, smem, items, c, g, m, st); break;
    default: launch_chunks(k_fft_inverse<3>, (const void*)k_fft_inverse<3>, smem, items, c, g, m, st); break;
  }
}

}  // namespace exogcm
