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
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kMaxThreads = 512;

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

// gp2fc: rows of N grid values -> m-major coefficients.
template <int Q>
__global__ void __launch_bounds__(kMaxThreads) k_fft_forward(const float* __restrict__ g, float* __restrict__ c,
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
  __syncwarp();
#pragma unroll
  for (int j = 0; j < Sh::KT; ++j)
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) xr[zpos(t + T * j + 8 * k2)] = b[j][k2];
  __syncwarp();
  const float inv_n = 1.f / (float)N;
#pragma unroll
  for (int i = 0; i < (NTP1 + T - 1) / T; ++i) {
    const int m = t + T * i;
    if (m < NTP1) {
      const float2 zm = xr[zpos(m)];
      const float2 zc = conj2(xr[zpos(m == 0 ? 0 : M - m)]);
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

template <typename K>
void allow_plane_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLegSmemLimit);
}

int q_of(const Dims& d) { return d.NLON / 16; }
int t_of(const Dims& d) { return q_of(d) == 8 ? 8 : 4; }

}  // namespace

void fft_init() {
  allow_plane_smem(k_fft_forward<4>);
  allow_plane_smem(k_fft_forward<8>);
  allow_plane_smem(k_fft_forward<12>);
  allow_plane_smem(k_fft_inverse<4>);
  allow_plane_smem(k_fft_inverse<8>);
  allow_plane_smem(k_fft_inverse<12>);
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
  switch (q_of(m.d)) {
    case 4: k_fft_inverse<4><<<blocks, threads, smem, st>>>(c, g, tw, m.d.NLAT, rows); break;
    case 8: k_fft_inverse<8><<<blocks, threads, smem, st>>>(c, g, tw, m.d.NLAT, rows); break;
    default: k_fft_inverse<12><<<blocks, threads, smem, st>>>(c, g, tw, m.d.NLAT, rows); break;
  }
}

}  // namespace exogcm
