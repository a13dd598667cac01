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
// FP64 on the host and rounded once. Shared memory reorders the bit-reversed
// FFT output and stages each warp's spectrum.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kWarps = 8;

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

// In-register M-point FFT of the R values x[r] = z[lane + 32 r]; on return
// x[k2] holds Z[R * bitrev5(lane) + k2].
template <int R, int SIGN>
__device__ __forceinline__ void warp_fft(float2 (&x)[R], const float2* tw, int N, int lane) {
  const int M = 32 * R;
  // radix-R step per lane, then the twiddle w_M^{n1 k2}
  if (R == 2) {
    const float2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = cmul(csub(a, b), twiddle<SIGN>(tw, 2 * lane, N));
  } else if (R == 3) {
    const float2 a = x[0], b = x[1], c = x[2];
    const float2 w3 = twiddle<SIGN>(tw, N / 3, N);      // e^{sign 2 pi i / 3}
    const float2 w32 = twiddle<SIGN>(tw, 2 * N / 3, N); // e^{sign 4 pi i / 3}
    x[0] = cadd(cadd(a, b), c);
    x[1] = cmul(cadd(cadd(a, cmul(b, w3)), cmul(c, w32)), twiddle<SIGN>(tw, 2 * lane, N));
    x[2] = cmul(cadd(cadd(a, cmul(b, w32)), cmul(c, w3)), twiddle<SIGN>(tw, 4 * lane, N));
  }
  (void)M;
  // 32-point DIF across lanes for each of the R sub-sequences
#pragma unroll
  for (int half = 16; half >= 1; half >>= 1) {
    const bool upper = (lane & half) != 0;
    const float2 w = twiddle<SIGN>(tw, (lane & (half - 1)) * (N / (2 * half)), N);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 y;
      y.x = __shfl_xor_sync(0xffffffffu, x[r].x, half);
      y.y = __shfl_xor_sync(0xffffffffu, x[r].y, half);
      x[r] = upper ? cmul(csub(y, x[r]), w) : cadd(x[r], y);
    }
  }
}

// gp2fc: rows of N grid values -> rows of NTP1 (re, im) coefficients.
template <int R>
__global__ void __launch_bounds__(kWarps * 32) k_fft_forward(const float* __restrict__ g, float* __restrict__ c,
                                                             int rows, const float2* __restrict__ twg, int ntp1) {
  constexpr int M = 32 * R, N = 2 * M;
  __shared__ float2 tw[N];
  __shared__ float2 zs[kWarps][M];
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twg[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float inv_n = 1.f / (float)N;
  for (int row = blockIdx.x * kWarps + warp; row < rows; row += gridDim.x * kWarps) {
    const float2* in = reinterpret_cast<const float2*>(g + (size_t)row * N);
    float2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = in[lane + 32 * r];
    warp_fft<R, -1>(x, tw, N, lane);
    const int k1 = bitrev5(lane);
#pragma unroll
    for (int r = 0; r < R; ++r) zs[warp][R * k1 + r] = x[r];
    __syncwarp();
    float2* out = reinterpret_cast<float2*>(c + (size_t)row * 2 * ntp1);
    for (int m = lane; m < ntp1; m += 32) {
      const float2 zm = zs[warp][m];
      const float2 zc = conj2(zs[warp][(M - m) % M]);
      const float2 even = make_float2(0.5f * (zm.x + zc.x), 0.5f * (zm.y + zc.y));
      // (zm - zc) / 2i = ((zm - zc).y, -(zm - zc).x) / 2
      const float2 odd = make_float2(0.5f * (zm.y - zc.y), -0.5f * (zm.x - zc.x));
      const float2 gm = cadd(even, cmul(twiddle<-1>(tw, m, N), odd));
      out[m] = make_float2(gm.x * inv_n, m == 0 ? 0.f : gm.y * inv_n);
    }
    __syncwarp();
  }
}

// fc2gp: rows of NTP1 coefficients -> rows of N grid values.
template <int R>
__global__ void __launch_bounds__(kWarps * 32) k_fft_inverse(const float* __restrict__ c, float* __restrict__ g,
                                                             int rows, const float2* __restrict__ twg, int ntp1) {
  constexpr int M = 32 * R, N = 2 * M;
  __shared__ float2 tw[N];
  __shared__ float2 gs[kWarps][M + 1];
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twg[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int row = blockIdx.x * kWarps + warp; row < rows; row += gridDim.x * kWarps) {
    const float2* in = reinterpret_cast<const float2*>(c + (size_t)row * 2 * ntp1);
    for (int m = lane; m <= M; m += 32) {
      float2 v = m < ntp1 ? in[m] : make_float2(0.f, 0.f);
      if (m == 0) v.y = 0.f;  // Im c_0 is ignored
      gs[warp][m] = v;
    }
    __syncwarp();
    float2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int k = lane + 32 * r;
      const float2 gk = gs[warp][k];
      const float2 gmk = conj2(gs[warp][M - k]);
      const float2 e = cadd(gk, gmk);
      const float2 o = cmul(csub(gk, gmk), twiddle<1>(tw, k, N));
      x[r] = make_float2(e.x - o.y, e.y + o.x);  // e + i o
    }
    warp_fft<R, 1>(x, tw, N, lane);
    __syncwarp();
    const int k1 = bitrev5(lane);
#pragma unroll
    for (int r = 0; r < R; ++r) gs[warp][R * k1 + r] = x[r];
    __syncwarp();
    float2* out = reinterpret_cast<float2*>(g + (size_t)row * N);
#pragma unroll
    for (int r = 0; r < R; ++r) out[lane + 32 * r] = gs[warp][lane + 32 * r];
    __syncwarp();
  }
}

inline unsigned fft_blocks(int rows) {
  const int want = (rows + kWarps - 1) / kWarps;
  return (unsigned)(want < 148 * 16 ? want : 148 * 16);
}

}  // namespace

void fft_forward(const Model& m, const float* g, float* c, int planes, cudaStream_t st) {
  const int rows = planes * m.d.NLAT;
  const float2* tw = reinterpret_cast<const float2*>(m.sh.tw);
  switch (m.d.NLON) {
    case 64: k_fft_forward<1><<<fft_blocks(rows), kWarps * 32, 0, st>>>(g, c, rows, tw, m.d.NTP1); break;
    case 128: k_fft_forward<2><<<fft_blocks(rows), kWarps * 32, 0, st>>>(g, c, rows, tw, m.d.NTP1); break;
    default: k_fft_forward<3><<<fft_blocks(rows), kWarps * 32, 0, st>>>(g, c, rows, tw, m.d.NTP1); break;
  }
}

void fft_inverse(const Model& m, const float* c, float* g, int planes, cudaStream_t st) {
  const int rows = planes * m.d.NLAT;
  const float2* tw = reinterpret_cast<const float2*>(m.sh.tw);
  switch (m.d.NLON) {
    case 64: k_fft_inverse<1><<<fft_blocks(rows), kWarps * 32, 0, st>>>(c, g, rows, tw, m.d.NTP1); break;
    case 128: k_fft_inverse<2><<<fft_blocks(rows), kWarps * 32, 0, st>>>(c, g, rows, tw, m.d.NTP1); break;
    default: k_fft_inverse<3><<<fft_blocks(rows), kWarps * 32, 0, st>>>(c, g, rows, tw, m.d.NTP1); break;
  }
}

}  // namespace exogcm
