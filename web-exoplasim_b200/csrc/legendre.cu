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
// Fourier planes are m-major on this path (coefficient (m, lat) at
// 2 * (m * NLAT + lat)), so an output wavenumber of the inverse is one
// contiguous run of latitudes, written by the threads that own consecutive
// latitude pairs (north run ascending, south run descending), and the
// forward transform reads such runs. Work is tiled as one block per (group
// of consecutive wavenumbers, tile of planes): a group's coefficients are
// contiguous in a spectral plane (modes are m-major) and a group's table
// slice is contiguous in the transposed northern tables ([mode][pair]), so
// both are staged in shared memory by contiguous loads.
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kForwardThreads = 256;
constexpr size_t kSmemBudget = kLegSmemLimit;

__device__ __forceinline__ int first_mode(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }
inline int first_mode_host(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }

// Terms (modes) of the first, largest group of `group` wavenumbers.
inline int group_terms(const Dims& d, int group) {
  const int m1 = group < d.NTP1 ? group : d.NTP1;
  return first_mode_host(m1, d.NTP1);
}

// ---------------------------------------------------------------- inverse
// KIND 0: f0 = sum over modes of table * s0 (one table, parity `odd`).
// KIND 1: dv2uv: (f0, f1) = (U, V) from (s0, s1) = (D, Z), tables qa = qu
// (even) and qb = qv (odd), plavor taken from vorticity mode w = 1.
// Persistent blocks walk the (wavenumber group, plane tile) items; while a
// block computes one item, cp.async brings the next item's coefficients
// and table slice into the other half of its shared memory, so staging
// latency overlaps arithmetic. Each thread owns latitude pair j and two
// planes of the tile.
template <int KIND>
__global__ void k_sym_inverse(const float* __restrict__ s0, const float* __restrict__ s1, float* __restrict__ f0,
                              float* __restrict__ f1, int planes, int tile, int group, int ntmax, int buf_floats,
                              const float* __restrict__ qa, const float* __restrict__ qb, int odd, float plavor,
                              Dims d) {
  constexpr int NIN = KIND == 0 ? 1 : 2;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int JH = d.NLAT / 2;
  const int ngroups = (d.NTP1 + group - 1) / group;
  const int items = ngroups * ((planes + tile - 1) / tile);
  const size_t plane_floats = (size_t)d.NLAT * d.NFC;
  // One buffer: [NIN][nt][tile] (re, im) term-major coefficients, then the
  // [NIN tables][nt][JH] table slice at a fixed 16-byte aligned offset.
  const int qs_at = 2 * NIN * ntmax * tile;
  auto stage = [&](int item, float* buf) {
    const int m0 = (item % ngroups) * group, p0 = (item / ngroups) * tile;
    const int m1 = min(m0 + group, d.NTP1);
    const int w0 = first_mode(m0, d.NTP1), nt = first_mode(m1, d.NTP1) - w0;
    const int np = min(tile, planes - p0);
    float* qs = buf + qs_at;
    for (int i = threadIdx.x; i < nt * JH / 4; i += blockDim.x) {
      cp_async16(qs + 4 * i, qa + (size_t)w0 * JH + 4 * i);
      if (KIND == 1) cp_async16(qs + nt * JH + 4 * i, qb + (size_t)w0 * JH + 4 * i);
    }
    float2* ss = reinterpret_cast<float2*>(buf);
    for (int k = 0; k < NIN; ++k) {
      const float* src = k == 0 ? s0 : s1;
      for (int i = threadIdx.x; i < np * nt; i += blockDim.x) {
        const int p = i / nt, t = i - p * nt;
        cp_async8(ss + ((size_t)k * nt + t) * tile + p, src + (size_t)(p0 + p) * d.NRSP + 2 * (w0 + t));
      }
    }
  };
  int item = blockIdx.x;
  if (item < items) stage(item, smem);
  cp_async_commit();
  for (int it = 0; item < items; ++it) {
    float* buf = smem + (size_t)(it & 1) * buf_floats;
    const int next = item + gridDim.x;
    if (next < items) stage(next, smem + (size_t)((it + 1) & 1) * buf_floats);
    cp_async_commit();
    cp_async_wait_one();  // this item's copies have landed (the next item's may be in flight)
    __syncthreads();
    const int m0 = (item % ngroups) * group, p0 = (item / ngroups) * tile;
    const int m1 = min(m0 + group, d.NTP1);
    const int w0 = first_mode(m0, d.NTP1), nt = first_mode(m1, d.NTP1) - w0;
    const int np = min(tile, planes - p0);
    float2* ss = reinterpret_cast<float2*>(buf);
    const float* qs = buf + qs_at;
    if (KIND == 1 && w0 <= 1 && 1 < w0 + nt) {
      // vorticity mode w = 1 (real part) without plavor
      for (int p = threadIdx.x; p < np; p += blockDim.x) ss[((size_t)nt + (1 - w0)) * tile + p].x -= plavor;
      __syncthreads();
    }
    const int j = threadIdx.x % JH;
    const int pa = 2 * (threadIdx.x / JH);  // planes pa, pa + 1 of the tile
    const int south = d.NLAT - 1 - j;
    const bool has_a = pa < np, has_b = pa + 1 < np;
    float2* outa0 = reinterpret_cast<float2*>(f0 + (size_t)(p0 + pa) * plane_floats);
    float2* outb0 = outa0 + plane_floats / 2;
    for (int m = m0; m < m1; ++m) {
      const int toff = first_mode(m, d.NTP1) - w0;
      const int K = d.NTP1 - m;
      const float* qc = qs + toff * JH + j;
      const float4* sc = reinterpret_cast<const float4*>(ss + (size_t)toff * tile + pa);
      const int step4 = tile / 2;  // float4 stride between terms
      const size_t rn = (size_t)m * d.NLAT + j, rs = (size_t)m * d.NLAT + south;
      if (KIND == 0) {
        float4 e = make_float4(0.f, 0.f, 0.f, 0.f), o = e;  // (re a, im a, re b, im b)
        int t = 0;
        for (; t + 1 < K; t += 2) {
          const float qe = qc[t * JH], qo = qc[(t + 1) * JH];
          const float4 ve = sc[t * step4], vo = sc[(t + 1) * step4];
          e.x = fmaf(qe, ve.x, e.x);
          e.y = fmaf(qe, ve.y, e.y);
          e.z = fmaf(qe, ve.z, e.z);
          e.w = fmaf(qe, ve.w, e.w);
          o.x = fmaf(qo, vo.x, o.x);
          o.y = fmaf(qo, vo.y, o.y);
          o.z = fmaf(qo, vo.z, o.z);
          o.w = fmaf(qo, vo.w, o.w);
        }
        if (t < K) {
          const float qe = qc[t * JH];
          const float4 ve = sc[t * step4];
          e.x = fmaf(qe, ve.x, e.x);
          e.y = fmaf(qe, ve.y, e.y);
          e.z = fmaf(qe, ve.z, e.z);
          e.w = fmaf(qe, ve.w, e.w);
        }
        const float sg = odd ? -1.f : 1.f;
        if (has_a) {
          outa0[rn] = make_float2(e.x + o.x, e.y + o.y);
          outa0[rs] = make_float2(sg * (e.x - o.x), sg * (e.y - o.y));
        }
        if (has_b) {
          outb0[rn] = make_float2(e.z + o.z, e.w + o.w);
          outb0[rs] = make_float2(sg * (e.z - o.z), sg * (e.w - o.w));
        }
      } else {
        const float* qd = qc + nt * JH;
        const float4* zc = sc + (size_t)nt * step4;
        // Term t's contribution to u and v: a(t) * (dim, -dre, zim, -zre)
        // + b(t) * (zre, zim, -dre, -dim); the even-t a part and odd-t b
        // part go to X, the rest to Y: north = X + Y, south = X - Y.
        float X[2][4] = {}, Y[2][4] = {};
        auto add = [&](float (*acc_a)[4], float (*acc_b)[4], float a, float b, int t) {
          const float4 D = sc[t * step4], Z = zc[t * step4];
          const float2 Dp[2] = {make_float2(D.x, D.y), make_float2(D.z, D.w)};
          const float2 Zp[2] = {make_float2(Z.x, Z.y), make_float2(Z.z, Z.w)};
#pragma unroll
          for (int pp = 0; pp < 2; ++pp) {
            acc_a[pp][0] = fmaf(a, Dp[pp].y, acc_a[pp][0]);
            acc_a[pp][1] = fmaf(-a, Dp[pp].x, acc_a[pp][1]);
            acc_a[pp][2] = fmaf(a, Zp[pp].y, acc_a[pp][2]);
            acc_a[pp][3] = fmaf(-a, Zp[pp].x, acc_a[pp][3]);
            acc_b[pp][0] = fmaf(b, Zp[pp].x, acc_b[pp][0]);
            acc_b[pp][1] = fmaf(b, Zp[pp].y, acc_b[pp][1]);
            acc_b[pp][2] = fmaf(-b, Dp[pp].x, acc_b[pp][2]);
            acc_b[pp][3] = fmaf(-b, Dp[pp].y, acc_b[pp][3]);
          }
        };
        int t = 0;
        for (; t + 1 < K; t += 2) {
          add(X, Y, qc[t * JH], qd[t * JH], t);
          add(Y, X, qc[(t + 1) * JH], qd[(t + 1) * JH], t + 1);
        }
        if (t < K) add(X, Y, qc[t * JH], qd[t * JH], t);
        float2* outa1 = reinterpret_cast<float2*>(f1 + (size_t)(p0 + pa) * plane_floats);
        float2* outb1 = outa1 + plane_floats / 2;
        if (has_a) {
          outa0[rn] = make_float2(X[0][0] + Y[0][0], X[0][1] + Y[0][1]);
          outa0[rs] = make_float2(X[0][0] - Y[0][0], X[0][1] - Y[0][1]);
          outa1[rn] = make_float2(X[0][2] + Y[0][2], X[0][3] + Y[0][3]);
          outa1[rs] = make_float2(X[0][2] - Y[0][2], X[0][3] - Y[0][3]);
        }
        if (has_b) {
          outb0[rn] = make_float2(X[1][0] + Y[1][0], X[1][1] + Y[1][1]);
          outb0[rs] = make_float2(X[1][0] - Y[1][0], X[1][1] - Y[1][1]);
          outb1[rn] = make_float2(X[1][2] + Y[1][2], X[1][3] + Y[1][3]);
          outb1[rs] = make_float2(X[1][2] - Y[1][2], X[1][3] - Y[1][3]);
        }
      }
    }
    __syncthreads();  // this buffer is restaged two items on
    item = next;
  }
  cp_async_wait_all();
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
// Staged per (input, plane, m, pair): (north + south, north - south) of the
// real and imaginary parts, read from the m-major planes as contiguous runs
// of latitudes, and the group's table slices ([table][pair][term]). For mode
// (m, n) the shader's north + s * south with s = (-1)^(m+n) is the sum for
// even n - m and the difference for odd. A thread owns one term (mode) for
// kFwdPlanes planes, so every table value it loads serves all of them.
constexpr int kFwdTile = 8;    // planes per block
constexpr int kFwdPlanes = 4;  // planes per thread

template <int KIND>
struct FwdTables {
  static constexpr int N = KIND == 0 ? 1 : KIND == 3 ? 3 : KIND == 2 ? 3 : 2;
};

template <int KIND, int NIN>
__global__ void __launch_bounds__(kForwardThreads) k_sym_forward(SymIn<NIN> in, float* __restrict__ out0,
                                                                 float* __restrict__ out1, int planes, int group,
                                                                 SharedTabs sh, const float* __restrict__ q, Dims d) {
  constexpr int NTAB = FwdTables<KIND>::N;
  extern __shared__ float4 pm[];  // [NIN][kFwdTile][group][JH], then the tables
  const int JH = d.NLAT / 2;
  const int m0 = blockIdx.x * group;
  const int m1 = min(m0 + group, d.NTP1);
  const int gm = m1 - m0;
  const int w0 = first_mode(m0, d.NTP1);
  const int nt = first_mode(m1, d.NTP1) - w0;
  const int p0 = blockIdx.y * kFwdTile;
  const int np = min(kFwdTile, planes - p0);
  const size_t plane_floats = (size_t)d.NLAT * d.NFC;
  float* tab = reinterpret_cast<float*>(pm + (size_t)NIN * kFwdTile * group * JH);  // [NTAB][JH][nt]
  // Tables in KIND order: 0: q; 1: qe, qm; 2: qe, qm, qq; 3: qe, qc, qm.
  const float* tsrc[3] = {KIND == 0 ? q : sh.qe, KIND == 3 ? sh.qc : sh.qm, KIND == 2 ? sh.qq : sh.qm};
#pragma unroll
  for (int k = 0; k < NTAB; ++k)
    for (int i = threadIdx.x; i < JH * nt; i += blockDim.x) {
      const int l = i / nt, t = i - l * nt;
      tab[(k * JH + l) * nt + t] = __ldg(tsrc[k] + (size_t)l * d.NCSP + w0 + t);
    }
  for (int k = 0; k < NIN; ++k) {
    for (int i = threadIdx.x; i < kFwdTile * gm * JH; i += blockDim.x) {
      const int j = i % JH;
      const int mi = (i / JH) % gm;
      const int p = i / (JH * gm);
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (p < np) {
        const float2* row = reinterpret_cast<const float2*>(in.p[k] + (size_t)(p0 + p) * plane_floats) +
                            (size_t)(m0 + mi) * d.NLAT;
        const float2 n = row[j], s = row[d.NLAT - 1 - j];
        v = make_float4(n.x + s.x, n.y + s.y, n.x - s.x, n.y - s.y);
      }
      pm[((k * kFwdTile + p) * group + mi) * JH + j] = v;
    }
  }
  __syncthreads();
  constexpr int NPG = kFwdTile / kFwdPlanes;
  for (int o = threadIdx.x; o < nt * NPG; o += blockDim.x) {
    const int t = o % nt;
    const int pg = o / nt;
    const int w = w0 + t;
    const int m = sh.mode_m[w], n = sh.mode_n[w];
    const int mi = m - m0;
    const bool even = ((m + n) & 1) == 0;
    const float* tq = tab + t;
    // pm row of input k, plane p of this thread's group, at pair l: pin(k, pp)[l]
    auto pin = [&](int k, int pp) { return pm + ((size_t)(k * kFwdTile + pg * kFwdPlanes + pp) * group + mi) * JH; };
    float r0[kFwdPlanes] = {}, r1[kFwdPlanes] = {}, r2[kFwdPlanes] = {}, r3[kFwdPlanes] = {};
    for (int l = 0; l < JH; ++l) {
      const float qa = tq[l * nt];
      const float qb = NTAB > 1 ? tq[(JH + l) * nt] : 0.f;
      const float qc = NTAB > 2 ? tq[(2 * JH + l) * nt] : 0.f;
#pragma unroll
      for (int pp = 0; pp < kFwdPlanes; ++pp) {
        if (KIND == 0) {
          const float4 f = pin(0, pp)[l];
          r0[pp] = fmaf(qa, even ? f.x : f.z, r0[pp]);
          r1[pp] = fmaf(qa, even ? f.y : f.w, r1[pp]);
        } else if (KIND == 1 || KIND == 2) {
          const float e = qa, mq = qb;
          const float4 U = pin(0, pp)[l], V = pin(NIN > 1 ? 1 : 0, pp)[l];
          // north - s * south and north + s * south of u and v
          const float dure = even ? U.z : U.x, duim = even ? U.w : U.y;
          const float dvre = even ? V.z : V.x, dvim = even ? V.w : V.y;
          const float sure = even ? U.x : U.z, suim = even ? U.y : U.w;
          const float svre = even ? V.x : V.z, svim = even ? V.y : V.w;
          if (KIND == 2) {
            const float q2 = qc;
            const float4 Kf = pin(NIN > 2 ? 2 : 0, pp)[l];
            r0[pp] = r0[pp] + q2 * (even ? Kf.x : Kf.z);
            r1[pp] = r1[pp] + q2 * (even ? Kf.y : Kf.w);
          }
          r0[pp] = r0[pp] - e * dvre - mq * suim;
          r1[pp] = r1[pp] - e * dvim + mq * sure;
          r2[pp] = r2[pp] + e * dure - mq * svim;
          r3[pp] = r3[pp] + e * duim + mq * svre;
        } else {
          const float e = qa, c = qb, mq = qc;
          const float4 U = pin(0, pp)[l], V = pin(NIN > 1 ? 1 : 0, pp)[l], X = pin(NIN > 2 ? 2 : 0, pp)[l];
          r0[pp] = r0[pp] + e * (even ? V.z : V.x) + c * (even ? X.x : X.z) + mq * (even ? U.y : U.w);
          r1[pp] = r1[pp] + e * (even ? V.w : V.y) + c * (even ? X.y : X.w) - mq * (even ? U.x : U.z);
        }
      }
    }
#pragma unroll
    for (int pp = 0; pp < kFwdPlanes; ++pp) {
      const int p = pg * kFwdPlanes + pp;
      if (p >= np) break;
      const size_t at = (size_t)(p0 + p) * d.NRSP + 2 * w;
      out0[at] = r0[pp];
      out0[at + 1] = r1[pp];
      if (KIND == 1 || KIND == 2) {
        out1[at] = r2[pp];
        out1[at + 1] = r3[pp];
      }
    }
  }
}

// Floats of one staging buffer of the inverse (a 16-byte multiple); a
// block holds two.
size_t inverse_buffer_floats(const Dims& d, int nin, int group, int tile) {
  const size_t nt = group_terms(d, group);
  const size_t f = (size_t)2 * nin * nt * tile + (size_t)nin * nt * (d.NLAT / 2);
  return (f + 3) / 4 * 4;
}

size_t inverse_smem(const Dims& d, int nin, int group, int tile) {
  return 2 * inverse_buffer_floats(d, nin, group, tile) * sizeof(float);
}

// Forward: kFwdTile planes per block; the group of wavenumbers is tuned.
size_t forward_smem(const Dims& d, int nin, int ntab, int group) {
  return (size_t)nin * kFwdTile * group * (d.NLAT / 2) * 16 + (size_t)ntab * (d.NLAT / 2) * group_terms(d, group) * 4;
}

template <typename K>
void allow_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget);
}

template <int KIND, int NIN>
void launch_sym_forward(const Model& m, SymIn<NIN> in, float* out0, float* out1, int planes, const float* q,
                        cudaStream_t st) {
  constexpr int NTAB = FwdTables<KIND>::N;
  const int group = m.tune.fwd_group[KIND];
  dim3 grid((m.d.NTP1 + group - 1) / group, (planes + kFwdTile - 1) / kFwdTile);
  k_sym_forward<KIND, NIN><<<grid, kForwardThreads, forward_smem(m.d, NIN, NTAB, group), st>>>(
      in, out0, out1, planes, group, m.sh, q, m.d);
}

}  // namespace

// The persistent grid: resident blocks per SM for a launch shape, times
// the SM count.
int persistent_grid(const void* kernel, int threads, size_t smem) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  return sms * (per_sm > 0 ? per_sm : 1);
}

void leg_init() {
  allow_smem(k_sym_inverse<0>);
  allow_smem(k_sym_inverse<1>);
  allow_smem(k_sym_forward<0, 1>);
  allow_smem(k_sym_forward<1, 2>);
  allow_smem(k_sym_forward<2, 3>);
  allow_smem(k_sym_forward<3, 3>);
}

template <int KIND>
void launch_inverse(const Model& m, const float* s0, const float* s1, float* f0, float* f1, int planes,
                    const float* qa, const float* qb, int odd, float plavor, cudaStream_t st) {
  const int nin = KIND == 0 ? 1 : 2;
  const int group = m.tune.inv_group[KIND], tile = m.tune.inv_tile[KIND];
  const int threads = (m.d.NLAT / 2) * tile / 2;
  const size_t smem = inverse_smem(m.d, nin, group, tile);
  const int items = ((m.d.NTP1 + group - 1) / group) * ((planes + tile - 1) / tile);
  const int grid = std::min(items, persistent_grid((const void*)k_sym_inverse<KIND>, threads, smem));
  k_sym_inverse<KIND><<<grid, threads, smem, st>>>(s0, s1, f0, f1, planes, tile, group, group_terms(m.d, group),
                                                   (int)inverse_buffer_floats(m.d, nin, group, tile), qa, qb, odd,
                                                   plavor, m.d);
}

void leg_inverse(const Model& m, const float* s, float* f, int planes, bool derivative, cudaStream_t st) {
  launch_inverse<0>(m, s, nullptr, f, nullptr, planes, derivative ? m.sh.qjT : m.sh.qiT, nullptr,
                    derivative ? 1 : 0, 0.f, st);
}

void leg_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
               cudaStream_t st) {
  launch_inverse<1>(m, D, Z, U, V, planes, m.sh.quT, m.sh.qvT, 0, plavor, st);
}

// Shared memory a tuning asks of each transform kernel, and the default
// tuning: the largest wavenumber groups that fit about 48 KB (inverse) and
// 60 KB (forward), 16-plane inverse tiles (32 at T21) and 16-latitude FFT
// chunks. The autotuner times the shapes that fit kLegSmemLimit.
size_t leg_inverse_smem(const Dims& d, int kind, int group, int tile) {
  return inverse_smem(d, kind == 0 ? 1 : 2, group, tile);
}

size_t leg_forward_smem(const Dims& d, int kind, int group) {
  const int nin = kind == 0 ? 1 : kind == 1 ? 2 : 3;
  const int ntab = kind == 0 ? 1 : kind == 1 ? 2 : 3;
  return forward_smem(d, nin, ntab, group);
}

Tuning default_tuning(const Dims& d) {
  Tuning t{};
  t.fft_rows = 16;
  for (int k = 0; k < 2; ++k) {
    t.inv_tile[k] = d.NLAT == 32 ? 32 : 16;
    t.inv_group[k] = 1;
    for (int g = 4; g > 1; g /= 2)
      if (leg_inverse_smem(d, k, g, t.inv_tile[k]) <= 48 * 1024) {
        t.inv_group[k] = g;
        break;
      }
  }
  for (int k = 0; k < 4; ++k) {
    t.fwd_group[k] = 1;
    for (int g = 4; g > 1; g /= 2)
      if (leg_forward_smem(d, k, g) <= 60 * 1024) {
        t.fwd_group[k] = g;
        break;
      }
  }
  return t;
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
