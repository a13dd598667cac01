// Legendre transforms of the optimized path (engine mode 1).
//
// The tables are exactly symmetric between the hemispheres: the Gaussian
// latitudes are mirrored (sin at NLAT-1-j is -sin at j), so every table
// entry at latitude NLAT-1-j equals s * (-1)^(n-m) times the entry at j, with
// s = +1 for qi, qc, qm, qq, qu and s = -1 for the derivative tables qj, qe,
// qv (legendre/index.ts:29-109 builds them from one recurrence per
// latitude). Both directions therefore work on latitude pairs:
//
//  * inverse (sp2fc, sp2fcdmu, dv2uv; legendre/wgsl/inverse.wgsl,
//    dv2uv.wgsl): for each plane, pair j and wavenumber m, the even-(n-m)
//    and odd-(n-m) partial sums E, O over the northern table give
//    north = E + O and south = +-(E - O), half the multiply-adds of the
//    full sum over NLAT latitudes;
//  * forward (fc2sp, uv2dv, mktend, qtend; forward.wgsl, uv2dv.wgsl,
//    qtend.wgsl): the shaders already sum latitude pairs (north +- south);
//    here the sums and differences are formed once per (plane, pair, m) in
//    shared memory instead of once per mode, with the shaders' arithmetic
//    in their order, so the results equal the plain path's bit for bit.
//
// Work is tiled as one block per (group of kGroup consecutive wavenumbers,
// tile of planes). The coefficients of a group are contiguous in a spectral
// plane (modes are m-major), and its Fourier outputs are a contiguous chunk
// of every row, so both directions read and write whole sectors. The
// transposed northern tables of the inverse ([mode][pair]) make the table
// reads coalesce across the threads of a warp, which own consecutive pairs.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kGroup = 4;         // zonal wavenumbers per block
constexpr int kRow = 2 * kGroup + 1;  // staged output row: 2 floats per m, padded to an odd stride
constexpr int kForwardThreads = 256;
constexpr size_t kSmemBudget = 100 * 1024;

__device__ __forceinline__ int first_mode(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }
inline int first_mode_host(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }

// Largest number of terms (modes) of one group: the first.
inline int group_terms(const Dims& d) {
  const int m1 = kGroup < d.NTP1 ? kGroup : d.NTP1;
  return first_mode_host(m1, d.NTP1);
}

// ---------------------------------------------------------------- inverse
// KIND 0: f0 = sum over modes of table * s0 (one table, parity `odd`).
// KIND 1: dv2uv: (f0, f1) = (U, V) from (s0, s1) = (D, Z), tables qa = qu
// (even) and qb = qv (odd), plavor taken from vorticity mode w = 1.
// Each thread owns latitude pair j and two planes of the tile.
template <int KIND>
__global__ void k_sym_inverse(const float* __restrict__ s0, const float* __restrict__ s1, float* __restrict__ f0,
                              float* __restrict__ f1, int planes, int tile, const float* __restrict__ qa,
                              const float* __restrict__ qb, int odd, float plavor, Dims d) {
  constexpr int NIN = KIND == 0 ? 1 : 2;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int JH = d.NLAT / 2;
  const int m0 = blockIdx.x * kGroup;
  const int m1 = min(m0 + kGroup, d.NTP1);
  const int w0 = first_mode(m0, d.NTP1);
  const int nt = first_mode(m1, d.NTP1) - w0;
  const int p0 = blockIdx.y * tile;
  const int np = min(tile, planes - p0);
  float2* ss = reinterpret_cast<float2*>(smem);  // [NIN][tile][nt] (re, im)
  float* so = smem + 2 * NIN * tile * nt;        // [NIN][tile][NLAT][kRow]
  for (int k = 0; k < NIN; ++k) {
    const float* src = k == 0 ? s0 : s1;
    for (int i = threadIdx.x; i < np * nt; i += blockDim.x) {
      const int p = i / nt, t = i - p * nt;
      float2 v = *reinterpret_cast<const float2*>(src + (size_t)(p0 + p) * d.NRSP + 2 * (w0 + t));
      if (KIND == 1 && k == 1 && w0 + t == 1) v.x -= plavor;
      ss[(k * tile + p) * nt + t] = v;
    }
  }
  __syncthreads();
  const int j = threadIdx.x % JH;
  const int pa = 2 * (threadIdx.x / JH);  // planes pa, pa + 1 of the tile
  const int south = d.NLAT - 1 - j;
  for (int m = m0; m < m1; ++m) {
    const int mi = m - m0;
    const int toff = first_mode(m, d.NTP1) - w0;
    const int K = d.NTP1 - m;
    const float* ta = qa + (size_t)(w0 + toff) * JH + j;
    if (KIND == 0) {
      const float2* sa = ss + pa * nt + toff;
      const float2* sb = sa + nt;
      float e0r = 0.f, e0i = 0.f, o0r = 0.f, o0i = 0.f, e1r = 0.f, e1i = 0.f, o1r = 0.f, o1i = 0.f;
      int t = 0;
      for (; t + 1 < K; t += 2) {
        const float qe = __ldg(ta + t * JH), qo = __ldg(ta + (t + 1) * JH);
        const float2 a0 = sa[t], a1 = sa[t + 1], b0 = sb[t], b1 = sb[t + 1];
        e0r = fmaf(qe, a0.x, e0r);
        e0i = fmaf(qe, a0.y, e0i);
        e1r = fmaf(qe, b0.x, e1r);
        e1i = fmaf(qe, b0.y, e1i);
        o0r = fmaf(qo, a1.x, o0r);
        o0i = fmaf(qo, a1.y, o0i);
        o1r = fmaf(qo, b1.x, o1r);
        o1i = fmaf(qo, b1.y, o1i);
      }
      if (t < K) {
        const float qe = __ldg(ta + t * JH);
        const float2 a0 = sa[t], b0 = sb[t];
        e0r = fmaf(qe, a0.x, e0r);
        e0i = fmaf(qe, a0.y, e0i);
        e1r = fmaf(qe, b0.x, e1r);
        e1i = fmaf(qe, b0.y, e1i);
      }
      const float sg = odd ? -1.f : 1.f;
      float* r0 = so + (size_t)pa * d.NLAT * kRow + 2 * mi;
      float* r1 = r0 + (size_t)d.NLAT * kRow;
      r0[j * kRow] = e0r + o0r;
      r0[j * kRow + 1] = e0i + o0i;
      r0[south * kRow] = sg * (e0r - o0r);
      r0[south * kRow + 1] = sg * (e0i - o0i);
      r1[j * kRow] = e1r + o1r;
      r1[j * kRow + 1] = e1i + o1i;
      r1[south * kRow] = sg * (e1r - o1r);
      r1[south * kRow + 1] = sg * (e1i - o1i);
    } else {
      const float* tb = qb + (size_t)(w0 + toff) * JH + j;
      // X collects the terms whose table is even at this t (a at even t,
      // b at odd t), Y the others: north = X + Y, south = X - Y.
      float X[2][4] = {}, Y[2][4] = {};
      for (int t = 0; t < K; ++t) {
        const float a = __ldg(ta + t * JH), b = __ldg(tb + t * JH);
#pragma unroll
        for (int pp = 0; pp < 2; ++pp) {
          const float2 D = ss[(pa + pp) * nt + toff + t];
          const float2 Z = ss[(tile + pa + pp) * nt + toff + t];
          const float au[4] = {a * D.y, -a * D.x, a * Z.y, -a * Z.x};
          const float bu[4] = {b * Z.x, b * Z.y, -b * D.x, -b * D.y};
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            if ((t & 1) == 0) {
              X[pp][c] += au[c];
              Y[pp][c] += bu[c];
            } else {
              X[pp][c] += bu[c];
              Y[pp][c] += au[c];
            }
          }
        }
      }
#pragma unroll
      for (int pp = 0; pp < 2; ++pp) {
        float* ru = so + (size_t)(pa + pp) * d.NLAT * kRow + 2 * mi;
        float* rv = ru + (size_t)tile * d.NLAT * kRow;
        ru[j * kRow] = X[pp][0] + Y[pp][0];
        ru[j * kRow + 1] = X[pp][1] + Y[pp][1];
        rv[j * kRow] = X[pp][2] + Y[pp][2];
        rv[j * kRow + 1] = X[pp][3] + Y[pp][3];
        ru[south * kRow] = X[pp][0] - Y[pp][0];
        ru[south * kRow + 1] = X[pp][1] - Y[pp][1];
        rv[south * kRow] = X[pp][2] - Y[pp][2];
        rv[south * kRow + 1] = X[pp][3] - Y[pp][3];
      }
    }
  }
  __syncthreads();
  // Flush: each row gets its group's 2 * (m1 - m0) consecutive floats.
  const int width = 2 * (m1 - m0);
  const int rows = np * d.NLAT;
  for (int k = 0; k < NIN; ++k) {
    float* dst = k == 0 ? f0 : f1;
    const float* src = so + (size_t)k * tile * d.NLAT * kRow;
    for (int i = threadIdx.x; i < rows * width; i += blockDim.x) {
      const int row = i / width, c = i - row * width;
      dst[((size_t)p0 * d.NLAT + row) * d.NFC + 2 * m0 + c] = src[row * kRow + c];
    }
  }
}

// ---------------------------------------------------------------- forward
template <int NIN>
struct SymIn {
  const float* p[NIN];
};

// KIND 0: fc2sp with table q (forward.wgsl).
// KIND 1: uv2dv, in = {u, v}, outputs D, Z (uv2dv.wgsl without the KE term).
// KIND 2: mktend's uv2dv, in = {u, v, ke} (uv2dv.wgsl with HAS_KINETIC).
// KIND 3: qtend, in = {u, v, source} (qtend.wgsl).
// Staged per (input, plane, pair, m): (north + south, north - south) of the
// real and imaginary parts. For mode (m, n) the shader's north + s * south
// with s = (-1)^(m+n) is the sum for even n - m and the difference for odd.
template <int KIND, int NIN>
__global__ void __launch_bounds__(kForwardThreads) k_sym_forward(SymIn<NIN> in, float* __restrict__ out0,
                                                                 float* __restrict__ out1, int planes, int tile,
                                                                 SharedTabs sh, const float* __restrict__ q, Dims d) {
  extern __shared__ float4 pm[];  // [NIN][tile][JH][kGroup]: (sum re, sum im, difference re, difference im)
  const int JH = d.NLAT / 2;
  const int m0 = blockIdx.x * kGroup;
  const int m1 = min(m0 + kGroup, d.NTP1);
  const int gm = m1 - m0;
  const int w0 = first_mode(m0, d.NTP1);
  const int nt = first_mode(m1, d.NTP1) - w0;
  const int p0 = blockIdx.y * tile;
  const int np = min(tile, planes - p0);
  const int plane_floats = d.NLAT * d.NFC;
  for (int k = 0; k < NIN; ++k) {
    const float* src = in.p[k] + (size_t)p0 * plane_floats + 2 * m0;
    for (int i = threadIdx.x; i < np * JH * gm; i += blockDim.x) {
      const int mi = i % gm;
      const int j = (i / gm) % JH;
      const int p = i / (gm * JH);
      const float2 n = *reinterpret_cast<const float2*>(src + (size_t)p * plane_floats + j * d.NFC + 2 * mi);
      const float2 s =
          *reinterpret_cast<const float2*>(src + (size_t)p * plane_floats + (d.NLAT - 1 - j) * d.NFC + 2 * mi);
      pm[((k * tile + p) * JH + j) * kGroup + mi] = make_float4(n.x + s.x, n.y + s.y, n.x - s.x, n.y - s.y);
    }
  }
  __syncthreads();
  for (int o = threadIdx.x; o < np * nt; o += blockDim.x) {
    const int t = o % nt;
    const int p = o / nt;
    const int w = w0 + t;
    const int m = sh.mode_m[w], n = sh.mode_n[w];
    const int mi = m - m0;
    const bool even = ((m + n) & 1) == 0;
    const size_t at = (size_t)(p0 + p) * d.NRSP + 2 * w;
    const float4* A = pm + ((size_t)(0 * tile + p) * JH) * kGroup + mi;
    const float4* B = pm + ((size_t)((NIN > 1 ? 1 : 0) * tile + p) * JH) * kGroup + mi;
    const float4* C = pm + ((size_t)((NIN > 2 ? 2 : 0) * tile + p) * JH) * kGroup + mi;
    if (KIND == 0) {
      float re = 0.f, im = 0.f;
      for (int l = 0; l < JH; ++l) {
        const float qq = __ldg(q + l * d.NCSP + w);
        const float4 f = A[l * kGroup];
        re = fmaf(qq, even ? f.x : f.z, re);
        im = fmaf(qq, even ? f.y : f.w, im);
      }
      out0[at] = re;
      out0[at + 1] = im;
    } else if (KIND == 1 || KIND == 2) {
      float dre = 0.f, dim = 0.f, zre = 0.f, zim = 0.f;
      for (int l = 0; l < JH; ++l) {
        const float e = __ldg(sh.qe + l * d.NCSP + w), mq = __ldg(sh.qm + l * d.NCSP + w);
        const float4 U = A[l * kGroup], V = B[l * kGroup];
        // north - s * south and north + s * south of u and v
        const float dure = even ? U.z : U.x, duim = even ? U.w : U.y;
        const float dvre = even ? V.z : V.x, dvim = even ? V.w : V.y;
        const float sure = even ? U.x : U.z, suim = even ? U.y : U.w;
        const float svre = even ? V.x : V.z, svim = even ? V.y : V.w;
        if (KIND == 2) {
          const float q2 = __ldg(sh.qq + l * d.NCSP + w);
          const float4 Kf = C[l * kGroup];
          dre = dre + q2 * (even ? Kf.x : Kf.z);
          dim = dim + q2 * (even ? Kf.y : Kf.w);
        }
        dre = dre - e * dvre - mq * suim;
        dim = dim - e * dvim + mq * sure;
        zre = zre + e * dure - mq * svim;
        zim = zim + e * duim + mq * svre;
      }
      out0[at] = dre;
      out0[at + 1] = dim;
      out1[at] = zre;
      out1[at + 1] = zim;
    } else {
      float re = 0.f, im = 0.f;
      for (int l = 0; l < JH; ++l) {
        const float e = __ldg(sh.qe + l * d.NCSP + w), c = __ldg(sh.qc + l * d.NCSP + w),
                    mq = __ldg(sh.qm + l * d.NCSP + w);
        const float4 U = A[l * kGroup], V = B[l * kGroup], X = C[l * kGroup];
        re = re + e * (even ? V.z : V.x) + c * (even ? X.x : X.z) + mq * (even ? U.y : U.w);
        im = im + e * (even ? V.w : V.y) + c * (even ? X.y : X.w) - mq * (even ? U.x : U.z);
      }
      out0[at] = re;
      out0[at + 1] = im;
    }
  }
}

// Planes per block: the largest of 32, 16, 8, 4, 2 whose shared memory fits
// the budget (two blocks per SM at most of it).
template <typename F>
int pick_tile(F bytes_for) {
  for (int tile = 32; tile > 2; tile /= 2)
    if (bytes_for(tile) <= kSmemBudget) return tile;
  return 2;
}

size_t inverse_smem(const Dims& d, int nin, int tile) {
  return (size_t)nin * tile * group_terms(d) * 8 + (size_t)nin * tile * d.NLAT * kRow * 4;
}

size_t forward_smem(const Dims& d, int nin, int tile) { return (size_t)nin * tile * (d.NLAT / 2) * kGroup * 16; }

int inverse_tile_for(const Dims& d, int nin) {
  // Threads = pairs * tile / 2; keep blocks at or under 512 threads.
  int tile = pick_tile([&](int t) { return inverse_smem(d, nin, t); });
  while (tile > 2 && (d.NLAT / 2) * tile / 2 > 512) tile /= 2;
  return tile;
}

int forward_tile_for(const Dims& d, int nin) {
  return pick_tile([&](int t) { return forward_smem(d, nin, t); });
}

template <typename K>
void allow_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget);
}

template <int KIND, int NIN>
void launch_sym_forward(const Model& m, SymIn<NIN> in, float* out0, float* out1, int planes, const float* q,
                        cudaStream_t st) {
  const int tile = forward_tile_for(m.d, NIN);
  dim3 grid((m.d.NTP1 + kGroup - 1) / kGroup, (planes + tile - 1) / tile);
  k_sym_forward<KIND, NIN><<<grid, kForwardThreads, forward_smem(m.d, NIN, tile), st>>>(in, out0, out1, planes, tile,
                                                                                      m.sh, q, m.d);
}

}  // namespace

void leg_init() {
  allow_smem(k_sym_inverse<0>);
  allow_smem(k_sym_inverse<1>);
  allow_smem(k_sym_forward<0, 1>);
  allow_smem(k_sym_forward<1, 2>);
  allow_smem(k_sym_forward<2, 3>);
  allow_smem(k_sym_forward<3, 3>);
}

void leg_inverse(const Model& m, const float* s, float* f, int planes, bool derivative, cudaStream_t st) {
  const int tile = inverse_tile_for(m.d, 1);
  dim3 grid((m.d.NTP1 + kGroup - 1) / kGroup, (planes + tile - 1) / tile);
  const int threads = (m.d.NLAT / 2) * tile / 2;
  k_sym_inverse<0><<<grid, threads, inverse_smem(m.d, 1, tile), st>>>(
      s, nullptr, f, nullptr, planes, tile, derivative ? m.sh.qjT : m.sh.qiT, nullptr, derivative ? 1 : 0, 0.f, m.d);
}

void leg_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
               cudaStream_t st) {
  const int tile = inverse_tile_for(m.d, 2);
  dim3 grid((m.d.NTP1 + kGroup - 1) / kGroup, (planes + tile - 1) / tile);
  const int threads = (m.d.NLAT / 2) * tile / 2;
  k_sym_inverse<1><<<grid, threads, inverse_smem(m.d, 2, tile), st>>>(D, Z, U, V, planes, tile, m.sh.quT, m.sh.qvT,
                                                                      0, plavor, m.d);
}

void leg_forward(const Model& m, const float* f, float* s, int planes, const float* q, cudaStream_t st) {
  SymIn<1> in{{f}};
  launch_sym_forward<0, 1>(m, in, s, nullptr, planes, q, st);
}

void leg_uv2dv(const Model& m, const float* u, const float* v, const float* ke, float* D, float* Z, int planes,
               cudaStream_t st) {
  if (ke) {
    SymIn<3> in{{u, v, ke}};
    launch_sym_forward<2, 3>(m, in, D, Z, planes, nullptr, st);
  } else {
    SymIn<2> in{{u, v}};
    launch_sym_forward<1, 2>(m, in, D, Z, planes, nullptr, st);
  }
}

void leg_qtend(const Model& m, const float* u, const float* v, const float* src, float* out, int planes,
               cudaStream_t st) {
  SymIn<3> in{{u, v, src}};
  launch_sym_forward<3, 3>(m, in, out, nullptr, planes, nullptr, st);
}

}  // namespace exogcm
