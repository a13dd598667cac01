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
// forward transform reads such runs. The inverse's work items are (group
// of consecutive wavenumbers, tile of planes): a group's coefficients are
// contiguous in a spectral plane (modes are m-major) and a group's table
// slice is contiguous in the transposed northern tables ([mode][pair]), so
// both are staged in shared memory by contiguous loads. The forward's
// blocks own wavenumber pairs (see k_sym_forward).
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

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
    // A thread owns pair j and PPT consecutive planes of the tile (2 for
    // sp2fc; 4 for dv2uv, whose 16 multiply-adds per term and plane pair
    // otherwise leave the loads a third of the issued instructions).
    constexpr int PPT = KIND == 0 ? 2 : 4;
    const int j = threadIdx.x % JH;
    const int pa = PPT * (threadIdx.x / JH);
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
        float X[PPT][4] = {}, Y[PPT][4] = {};
        auto add = [&](float (*acc_a)[4], float (*acc_b)[4], float a, float b, int t) {
          float2 Dp[PPT], Zp[PPT];
#pragma unroll
          for (int h = 0; h < PPT / 2; ++h) {
            const float4 D = sc[t * step4 + h], Z = zc[t * step4 + h];
            Dp[2 * h] = make_float2(D.x, D.y);
            Dp[2 * h + 1] = make_float2(D.z, D.w);
            Zp[2 * h] = make_float2(Z.x, Z.y);
            Zp[2 * h + 1] = make_float2(Z.z, Z.w);
          }
#pragma unroll
          for (int pp = 0; pp < PPT; ++pp) {
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
#pragma unroll
        for (int pp = 0; pp < PPT; ++pp) {
          if (pa + pp >= np) break;
          float2* u = reinterpret_cast<float2*>(f0 + (size_t)(p0 + pa + pp) * plane_floats);
          float2* v = reinterpret_cast<float2*>(f1 + (size_t)(p0 + pa + pp) * plane_floats);
          u[rn] = make_float2(X[pp][0] + Y[pp][0], X[pp][1] + Y[pp][1]);
          u[rs] = make_float2(X[pp][0] - Y[pp][0], X[pp][1] - Y[pp][1]);
          v[rn] = make_float2(X[pp][2] + Y[pp][2], X[pp][3] + Y[pp][3]);
          v[rs] = make_float2(X[pp][2] - Y[pp][2], X[pp][3] - Y[pp][3]);
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
//
// A block owns the wavenumber pair (g, NTP1 - 1 - g), or the middle
// wavenumber alone: NTP1 + 1 modes for every pair, so blocks carry equal
// work. Its table slices ([table][pair][mode]) are staged once, and it then
// walks a range of planes in tiles of TP. While one tile is computed, the
// next tile's inputs are fetched into registers; they are stored as
// (north + south, north - south) of the real and imaginary parts per
// (input, plane, wavenumber, pair). For mode (m, n) the shaders'
// north + s * south with s = (-1)^(m+n) is the sum for even n - m and the
// difference for odd. A thread owns one mode for TP / 4 planes, so each
// table value it loads serves all of them. Every mode's sum runs over the
// pairs in the shaders' order and expression, so the results equal the
// plain path's bit for bit, whatever the tiling.
template <int KIND>
struct FwdTables {
  static constexpr int N = KIND == 0 ? 1 : KIND == 3 ? 3 : KIND == 2 ? 3 : 2;
};

template <int JH, int TP>
struct FwdShape {
  static constexpr int NLAT = 2 * JH;
  static constexpr int NTP1 = JH == 16 ? 22 : JH == 32 ? 43 : 64;  // T21, T42, T63
  static constexpr int NT = NTP1 + 1;                               // modes of a wavenumber pair
  static constexpr int GROUPS = (NTP1 + 1) / 2;
  static constexpr int PP = TP / 4;                                 // planes per thread
  static constexpr int THREADS = (4 * NT + 31) / 32 * 32;           // (mode, plane quarter) tasks
  static constexpr int ROW = JH + 1;                                // float4s per staged row, padded
};

// NB staging buffers: with two, the next tile is stored while the current
// one is read; with one, a barrier separates them and the block needs about
// half the shared memory, so more blocks share an SM (the autotuner picks).
template <int KIND, int NIN, int JH, int TP, int NB>
__global__ void __launch_bounds__(FwdShape<JH, TP>::THREADS)
    k_sym_forward(SymIn<NIN> in, float* __restrict__ out0, float* __restrict__ out1, int planes, int per_block,
                  SharedTabs sh, const float* __restrict__ q, int ncsp) {
  using S = FwdShape<JH, TP>;
  constexpr int NTAB = FwdTables<KIND>::N;
  constexpr int NLAT = S::NLAT, NTP1 = S::NTP1, NT = S::NT, PP = S::PP, ROW = S::ROW;
  constexpr size_t PLANE = (size_t)NLAT * 2 * NTP1;  // floats of a Fourier plane
  constexpr int CONV = NIN * TP * 2 * ROW;            // float4s of one staged tile
  extern __shared__ float4 fsm[];
  float* tab = reinterpret_cast<float*>(fsm);           // [NTAB][JH][NT]
  float4* conv = fsm + (NTAB * JH * NT + 3) / 4;        // [NB][NIN][TP][2][ROW]
  const int g = blockIdx.x % S::GROUPS;
  const int pbeg = (blockIdx.x / S::GROUPS) * per_block;
  const int pend = min(planes, pbeg + per_block);
  const int ma = g, mb = NTP1 - 1 - g;
  const bool pair = mb != ma;
  const int Ka = NTP1 - ma;
  const int nt = pair ? NT : Ka;
  const int wa = first_mode(ma, NTP1), wb = first_mode(mb, NTP1);

  // Fetch: element e = ((k * TP + p) * 2 + mi) * JH + l of a tile, the
  // north and south values of pair l.
  constexpr int E = NIN * TP * 2 * JH;
  constexpr int R = (E + S::THREADS - 1) / S::THREADS;
  float2 rn[R], rs[R];
  auto fetch = [&](int tile) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int e = threadIdx.x + i * S::THREADS;
      const int l = e % JH, mi = (e / JH) % 2, p = (e / (2 * JH)) % TP, k = e / (2 * JH * TP);
      const int plane = tile + p;
      float2 a = make_float2(0.f, 0.f), b = a;
      if (e < E && plane < pend && (mi == 0 || pair)) {
        const float* base = k == 0 ? in.p[0] : k == 1 ? in.p[NIN > 1 ? 1 : 0] : in.p[NIN > 2 ? 2 : 0];
        const float2* row =
            reinterpret_cast<const float2*>(base + (size_t)plane * PLANE) + (size_t)(mi ? mb : ma) * NLAT;
        a = row[l];
        b = row[NLAT - 1 - l];
      }
      rn[i] = a;
      rs[i] = b;
    }
  };
  auto store = [&](float4* buf) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int e = threadIdx.x + i * S::THREADS;
      if (e < E) {
        const int l = e % JH, row = e / JH;
        const float2 n = rn[i], so = rs[i];
        buf[row * ROW + l] = make_float4(n.x + so.x, n.y + so.y, n.x - so.x, n.y - so.y);
      }
    }
  };

  fetch(pbeg);
  // Tables in KIND order: 0: q; 1: qe, qm; 2: qe, qm, qq; 3: qe, qc, qm.
#pragma unroll
  for (int k = 0; k < NTAB; ++k) {
    const float* src = k == 0 ? (KIND == 0 ? q : sh.qe) : k == 1 ? (KIND == 3 ? sh.qc : sh.qm)
                                                                 : (KIND == 2 ? sh.qq : sh.qm);
    for (int i = threadIdx.x; i < JH * NT; i += S::THREADS) {
      const int t = i % NT, l = i / NT;
      const int w = t < Ka ? wa + t : wb + (t - Ka);
      tab[k * JH * NT + i] = t < nt ? __ldg(src + (size_t)l * ncsp + w) : 0.f;
    }
  }
  store(conv);
  __syncthreads();

  // This thread's task: mode t of the block, planes pq * PP .. of each tile.
  const int t = threadIdx.x % nt, pq = threadIdx.x / nt;
  const bool active = pq < 4;
  const int mi = t < Ka ? 0 : 1;
  const int toff = mi ? t - Ka : t;  // n - m
  const int w = (mi ? wb : wa) + toff;
  const bool even = (toff & 1) == 0;
  const float* tq = tab + t;
  int it = 0;
  for (int tile = pbeg; tile < pend; tile += TP, ++it) {
    const float4* cur = conv + (NB == 2 ? (it & 1) * CONV : 0);
    const int next = tile + TP;
    if (next < pend) fetch(next);
    if (active) {
      // staged row of input k, plane pp of this thread's planes, at pair l: pin(k, pp)[l]
      auto pin = [&](int k, int pp) { return cur + ((k * TP + pq * PP + pp) * 2 + mi) * ROW; };
      // the (sum) or (difference) half of a staged float4 as one float2:
      // half(k, pp, 0)[2 l] is (re, im) of north + south, half(k, pp, 1)[2 l] of north - south
      auto half = [&](int k, int pp, int h) { return reinterpret_cast<const float2*>(pin(k, pp)) + h; };
      const int hs = even ? 0 : 1;  // the half the shaders' north + s * south selects
      float r0[PP] = {}, r1[PP] = {}, r2[PP] = {}, r3[PP] = {};
#pragma unroll 4
      for (int l = 0; l < JH; ++l) {
        const float qa = tq[l * NT];
        const float qb = NTAB > 1 ? tq[(JH + l) * NT] : 0.f;
        const float qc = NTAB > 2 ? tq[(2 * JH + l) * NT] : 0.f;
#pragma unroll
        for (int pp = 0; pp < PP; ++pp) {
          if (KIND == 0) {
            const float2 f = half(0, pp, hs)[2 * l];
            r0[pp] = fmaf(qa, f.x, r0[pp]);
            r1[pp] = fmaf(qa, f.y, r1[pp]);
          } else if (KIND == 1 || KIND == 2) {
            const float e = qa, mq = qb;
            // north + s * south (Us, Vs) and north - s * south (Ud, Vd) of u and v
            const float2 Us = half(0, pp, hs)[2 * l], Ud = half(0, pp, 1 - hs)[2 * l];
            const float2 Vs = half(NIN > 1 ? 1 : 0, pp, hs)[2 * l], Vd = half(NIN > 1 ? 1 : 0, pp, 1 - hs)[2 * l];
            if (KIND == 2) {
              const float q2 = qc;
              const float2 Ks = half(NIN > 2 ? 2 : 0, pp, hs)[2 * l];
              r0[pp] = r0[pp] + q2 * Ks.x;
              r1[pp] = r1[pp] + q2 * Ks.y;
            }
            r0[pp] = r0[pp] - e * Vd.x - mq * Us.y;
            r1[pp] = r1[pp] - e * Vd.y + mq * Us.x;
            r2[pp] = r2[pp] + e * Ud.x - mq * Vs.y;
            r3[pp] = r3[pp] + e * Ud.y + mq * Vs.x;
          } else {
            const float e = qa, c = qb, mq = qc;
            // V's difference and X's and U's sums for even n - m, the other halves for odd
            const float2 U = half(0, pp, hs)[2 * l], V = half(NIN > 1 ? 1 : 0, pp, 1 - hs)[2 * l],
                         X = half(NIN > 2 ? 2 : 0, pp, hs)[2 * l];
            r0[pp] = r0[pp] + e * V.x + c * X.x + mq * U.y;
            r1[pp] = r1[pp] + e * V.y + c * X.y - mq * U.x;
          }
        }
      }
#pragma unroll
      for (int pp = 0; pp < PP; ++pp) {
        const int plane = tile + pq * PP + pp;
        if (plane < pend) {
          const size_t at = (size_t)plane * (2 * ncsp) + 2 * w;
          *reinterpret_cast<float2*>(out0 + at) = make_float2(r0[pp], r1[pp]);
          if (KIND == 1 || KIND == 2) *reinterpret_cast<float2*>(out1 + at) = make_float2(r2[pp], r3[pp]);
        }
      }
    }
    if (NB == 2) {
      if (next < pend) store(conv + ((it + 1) & 1) * CONV);
    } else if (next < pend) {
      __syncthreads();
      store(conv);
    }
    __syncthreads();
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

// Forward: the table slices of a wavenumber pair and NB staged tiles.
template <int KIND, int NIN, int JH, int TP, int NB = 2>
size_t forward_smem() {
  using S = FwdShape<JH, TP>;
  return ((size_t)(FwdTables<KIND>::N * JH * S::NT + 3) / 4 + NB * (size_t)NIN * TP * 2 * S::ROW) * sizeof(float4);
}

template <typename K>
void allow_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget);
}

template <int KIND, int NIN, int JH, int TP, int NB>
void launch_forward_shape(const Model& m, SymIn<NIN> in, float* out0, float* out1, int planes, const float* q,
                          cudaStream_t st) {
  using S = FwdShape<JH, TP>;
  const auto kernel = k_sym_forward<KIND, NIN, JH, TP, NB>;
  const size_t smem = forward_smem<KIND, NIN, JH, TP, NB>();
  // Blocks per wavenumber pair: enough for every SM's resident blocks, in
  // whole tiles of planes.
  const int tiles = (planes + TP - 1) / TP;
  const int target = persistent_grid((const void*)kernel, S::THREADS, smem);
  const int splits = std::max(1, std::min(tiles, (target + S::GROUPS - 1) / S::GROUPS));
  const int per_tiles = (tiles + splits - 1) / splits;
  const int blocks = S::GROUPS * ((tiles + per_tiles - 1) / per_tiles);
  kernel<<<blocks, S::THREADS, smem, st>>>(in, out0, out1, planes, per_tiles * TP, m.sh, q, m.d.NCSP);
}

template <int KIND, int NIN>
void launch_sym_forward(const Model& m, SymIn<NIN> in, float* out0, float* out1, int planes, const float* q,
                        cudaStream_t st) {
  const bool big = m.tune.fwd_tile[KIND] == 16, one = m.tune.fwd_buffers[KIND] == 1;
#define EXOGCM_FWD(JH)                                                                         \
  (big ? (one ? launch_forward_shape<KIND, NIN, JH, 16, 1>(m, in, out0, out1, planes, q, st)  \
              : launch_forward_shape<KIND, NIN, JH, 16, 2>(m, in, out0, out1, planes, q, st)) \
       : (one ? launch_forward_shape<KIND, NIN, JH, 8, 1>(m, in, out0, out1, planes, q, st)   \
              : launch_forward_shape<KIND, NIN, JH, 8, 2>(m, in, out0, out1, planes, q, st)))
  switch (m.d.NLAT) {
    case 32: EXOGCM_FWD(16); break;
    case 64: EXOGCM_FWD(32); break;
    default: EXOGCM_FWD(48); break;
  }
#undef EXOGCM_FWD
}

template <int KIND, int NIN>
size_t forward_smem_for(const Dims& d, int tile) {
  const bool big = tile == 16;
  switch (d.NLAT) {
    case 32: return big ? forward_smem<KIND, NIN, 16, 16>() : forward_smem<KIND, NIN, 16, 8>();
    case 64: return big ? forward_smem<KIND, NIN, 32, 16>() : forward_smem<KIND, NIN, 32, 8>();
    default: return big ? forward_smem<KIND, NIN, 48, 16>() : forward_smem<KIND, NIN, 48, 8>();
  }
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

template <int KIND, int NIN, int NB>
void allow_forward_smem_nb() {
  allow_smem(k_sym_forward<KIND, NIN, 16, 8, NB>);
  allow_smem(k_sym_forward<KIND, NIN, 16, 16, NB>);
  allow_smem(k_sym_forward<KIND, NIN, 32, 8, NB>);
  allow_smem(k_sym_forward<KIND, NIN, 32, 16, NB>);
  allow_smem(k_sym_forward<KIND, NIN, 48, 8, NB>);
  allow_smem(k_sym_forward<KIND, NIN, 48, 16, NB>);
}

template <int KIND, int NIN>
void allow_forward_smem() {
  allow_forward_smem_nb<KIND, NIN, 1>();
  allow_forward_smem_nb<KIND, NIN, 2>();
}

void leg_init() {
  allow_smem(k_sym_inverse<0>);
  allow_smem(k_sym_inverse<1>);
  allow_forward_smem<0, 1>();
  allow_forward_smem<1, 2>();
  allow_forward_smem<2, 3>();
  allow_forward_smem<3, 3>();
}

template <int KIND>
void launch_inverse(const Model& m, const float* s0, const float* s1, float* f0, float* f1, int planes,
                    const float* qa, const float* qb, int odd, float plavor, cudaStream_t st) {
  const int nin = KIND == 0 ? 1 : 2;
  const int group = m.tune.inv_group[KIND], tile = m.tune.inv_tile[KIND];
  const int threads = (m.d.NLAT / 2) * tile / (KIND == 0 ? 2 : 4);
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
// tuning: the largest inverse wavenumber groups that fit about 48 KB,
// 16-plane inverse tiles (32 at T21), 8-plane forward tiles and 16-latitude
// FFT chunks. The autotuner times the shapes that fit kLegSmemLimit.
size_t leg_inverse_smem(const Dims& d, int kind, int group, int tile) {
  return inverse_smem(d, kind == 0 ? 1 : 2, group, tile);
}

size_t leg_forward_smem(const Dims& d, int kind, int tile) {
  switch (kind) {
    case 0: return forward_smem_for<0, 1>(d, tile);
    case 1: return forward_smem_for<1, 2>(d, tile);
    case 2: return forward_smem_for<2, 3>(d, tile);
    default: return forward_smem_for<3, 3>(d, tile);
  }
}

Tuning default_tuning(const Dims& d) {
  Tuning t{};
  t.fft_rows = 16;
  t.fft_persistent[0] = t.fft_persistent[1] = 0;
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
    t.fwd_tile[k] = 8;
    t.fwd_buffers[k] = 2;
  }
  t.sp2gp_planes = 2;
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
