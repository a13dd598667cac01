// Device code of the longitude FFTs shared by the FFT kernels (fft.cu) and
// the fused spectral-to-grid transforms (spectral_grid.cu): small DFTs in
// registers, the four-step M = 8 Q point FFT of one row by T threads, and
// the twiddle tables. The algorithm is described at the top of fft.cu.
#pragma once

#include <cuda_runtime.h>

namespace exogcm {
namespace fftcore {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conj2(float2 a) { return make_float2(a.x, -a.y); }

// a * (S i)
template <int S>
__device__ __forceinline__ float2 mul_i(float2 a) {
  return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// a * e^{S 2 pi i j / 12} for a compile-time j in 0..6 (cos and sin of
// multiples of 30 degrees).
template <int S, int J>
__device__ __forceinline__ float2 rot12(float2 a) {
  constexpr float c30 = 0.866025403784438647f;
  constexpr float cs[7] = {1.f, c30, 0.5f, 0.f, -0.5f, -c30, -1.f};
  constexpr float sn[7] = {0.f, 0.5f, c30, 1.f, c30, 0.5f, 0.f};
  if (J == 0) return a;
  if (J == 3) return mul_i<S>(a);
  if (J == 6) return make_float2(-a.x, -a.y);
  const float c = cs[J], s = S * sn[J];
  return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

// y_k = sum_p x_p e^{S 2 pi i p k / 4}, in place.
template <int S>
__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
  const float2 c0 = cadd(x0, x2), c1 = csub(x0, x2), d0 = cadd(x1, x3), d1 = mul_i<S>(csub(x1, x3));
  x0 = cadd(c0, d0);
  x2 = csub(c0, d0);
  x1 = cadd(c1, d1);
  x3 = csub(c1, d1);
}

// y_k = sum_p x_p e^{S 2 pi i p k / 3}, in place.
template <int S>
__device__ __forceinline__ void dft3(float2& x0, float2& x1, float2& x2) {
  constexpr float h3 = 0.866025403784438647f;  // sin(60 degrees)
  const float2 s = cadd(x1, x2), d = csub(x1, x2);
  const float2 t = make_float2(x0.x - 0.5f * s.x, x0.y - 0.5f * s.y);
  const float2 r = mul_i<S>(make_float2(h3 * d.x, h3 * d.y));
  x0 = cadd(x0, s);
  x1 = cadd(t, r);
  x2 = csub(t, r);
}

// Radix-2 decimation in frequency onto two DFT-4s; natural-order output.
template <int S>
__device__ __forceinline__ void dft8(float2 (&x)[8]) {
  constexpr float h = 0.707106781186547524f;  // cos(45 degrees)
  float2 a[4], b[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    a[p] = cadd(x[p], x[p + 4]);
    b[p] = csub(x[p], x[p + 4]);
  }
  b[1] = make_float2(h * (b[1].x - S * b[1].y), h * (b[1].y + S * b[1].x));   // * e^{S i pi/4}
  b[2] = mul_i<S>(b[2]);                                                       // * e^{S i pi/2}
  b[3] = make_float2(h * (-b[3].x - S * b[3].y), h * (-b[3].y + S * b[3].x));  // * e^{S 3i pi/4}
  dft4<S>(a[0], a[1], a[2], a[3]);
  dft4<S>(b[0], b[1], b[2], b[3]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[2 * k] = a[k];
    x[2 * k + 1] = b[k];
  }
}

// 12 = 3 x 4 by the same four-step factorisation (n = 4 p + q, k = k1 + 3 k2).
template <int S>
__device__ __forceinline__ void dft12(float2 (&x)[12]) {
  float2 a[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    a[q][0] = x[q];
    a[q][1] = x[4 + q];
    a[q][2] = x[8 + q];
    dft3<S>(a[q][0], a[q][1], a[q][2]);
  }
  a[1][1] = rot12<S, 1>(a[1][1]);
  a[1][2] = rot12<S, 2>(a[1][2]);
  a[2][1] = rot12<S, 2>(a[2][1]);
  a[2][2] = rot12<S, 4>(a[2][2]);
  a[3][1] = rot12<S, 3>(a[3][1]);
  a[3][2] = rot12<S, 6>(a[3][2]);
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    dft4<S>(a[0][k1], a[1][k1], a[2][k1], a[3][k1]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) x[k1 + 3 * k2] = a[k2][k1];
  }
}

template <int Q, int S>
__device__ __forceinline__ void dft_q(float2 (&x)[Q]) {
  if constexpr (Q == 4)
    dft4<S>(x[0], x[1], x[2], x[3]);
  else if constexpr (Q == 8)
    dft8<S>(x);
  else
    dft12<S>(x);
}

// Shared-memory position of Z[k] (k = k1 + 8 k2) and of B[q][k1]: 9 per 8.
__device__ __forceinline__ int zpos(int k) { return k + (k >> 3); }

// Pitch of the [m][pitch] coefficient stage: pitch = 16 / T (mod 16), so
// that a half-warp's 64-bit accesses fc[(t + T i) * pitch + r] fall on
// distinct banks.
__host__ __device__ inline int fc_pitch(int rows, int T) {
  return rows + (((16 / T - rows) % 16) + 16) % 16;
}

template <int Q>
struct Shape {
  static constexpr int M = 8 * Q, N = 2 * M;
  static constexpr int NTP1 = Q == 4 ? 22 : Q == 8 ? 43 : 64;  // T21, T42, T63
  static constexpr int T = Q == 8 ? 8 : 4;                      // threads per row
  static constexpr int QT = Q / T, KT = 8 / T;
  static constexpr int XP = 9 * Q;  // exchange float2s per row
};

// Twiddles, the exchange rows and the coefficient stage of NTP1 rows.
inline size_t chunk_smem(int Q, int T, int rows) {
  const int ntp1 = Q == 4 ? 22 : Q == 8 ? 43 : 64;
  return ((size_t)2 * 8 * Q + 9 * Q + (size_t)rows * 9 * Q + (size_t)ntp1 * fc_pitch(rows, T)) * sizeof(float2);
}

// Twiddle tables into shared memory: tw[j] = e^{2 pi i j / N};
// twq[9 q + k1] = w_M^{q k1}.
template <int Q>
__device__ __forceinline__ void load_twiddles(const float2* __restrict__ twg, float2* tw, float2* twq) {
  using Sh = Shape<Q>;
  for (int i = threadIdx.x; i < Sh::N; i += blockDim.x) tw[i] = twg[i];
  for (int i = threadIdx.x; i < 9 * Q; i += blockDim.x) {
    const int q = i / 9, k1 = i - 9 * q;
    twq[i] = k1 < 8 ? twg[(2 * q * k1) % Sh::N] : make_float2(0.f, 0.f);
  }
}

// Steps two and three of the four-step FFT for one row: a[i] holds the
// DFT-8 input of q = t + T i; on return b[j][k2] = Z[t + T j + 8 k2].
template <int Q, int S>
__device__ __forceinline__ void four_step(float2 (&a)[Shape<Q>::QT][8], float2 (&b)[Shape<Q>::KT][Q],
                                          const float2* twq, float2* xr, int t) {
  using Sh = Shape<Q>;
#pragma unroll
  for (int i = 0; i < Sh::QT; ++i) {
    const int q = t + Sh::T * i;
    dft8<S>(a[i]);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1) {
      const float2 w = twq[9 * q + k1];
      a[i][k1] = S > 0 ? cmul(a[i][k1], w) : cmulc(a[i][k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) xr[9 * q + k1] = a[i][k1];
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < Sh::KT; ++j) {
    const int k1 = t + Sh::T * j;
#pragma unroll
    for (int q = 0; q < Q; ++q) b[j][q] = xr[9 * q + k1];
    dft_q<Q, S>(b[j]);
  }
}


}  // namespace fftcore
}  // namespace exogcm
