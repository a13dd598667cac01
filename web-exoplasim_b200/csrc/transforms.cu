// Longitude (Fourier) and latitude (Gauss-Legendre) transforms, batched over
// every plane of every planet slot, in plain FP32 on the CUDA cores.
//
// Semantics follow the reference's WGSL transforms
// (src/model/climate/gcm/fourier/wgsl/*.wgsl, legendre/wgsl/*.wgsl): the
// longitude transforms are the truncated DFT with the f64-built tables of
// fourier/index.ts:19-36 (c_m = (1/N) sum_j g_j e^{-i m lambda_j} for
// m <= NTRU, and its inverse that ignores Im c_0), and the Legendre sums run
// over latitude pairs with the (m + n)-parity folding of legmod's
// single-process branch. Each kernel stages what its threads share in shared
// memory: the DFT tables and a tile of rows, or a tile of spectral or Fourier
// planes, so each table element read from L2 serves a whole tile.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kThreads = 256;

// ---------------------------------------------------------------- DFTs
// gp2fc: rows of NLON grid values -> rows of NFC (re, im) coefficients.
__global__ void __launch_bounds__(kThreads) k_dft_forward(const float* __restrict__ g,
                                                          float* __restrict__ c, int rows,
                                                          const float* __restrict__ tab, int nlon,
                                                          int nfc, int rows_per_block) {
  extern __shared__ float smem[];
  float* ts = smem;               // [nlon][nfc]
  float* gs = smem + nlon * nfc;  // [rows_per_block][nlon]
  const int row0 = blockIdx.x * rows_per_block;
  const int nrows = min(rows_per_block, rows - row0);
  for (int i = threadIdx.x; i < nlon * nfc; i += blockDim.x) ts[i] = tab[i];
  for (int i = threadIdx.x; i < nrows * nlon; i += blockDim.x) gs[i] = g[(size_t)row0 * nlon + i];
  __syncthreads();
  for (int o = threadIdx.x; o < nrows * nfc; o += blockDim.x) {
    const int r = o / nfc, k = o % nfc;
    const float* gr = gs + r * nlon;
    float s = 0.f;
    for (int j = 0; j < nlon; ++j) s = fmaf(ts[j * nfc + k], gr[j], s);
    c[(size_t)(row0 + r) * nfc + k] = s;
  }
}

// fc2gp: rows of NFC coefficients -> rows of NLON grid values.
__global__ void __launch_bounds__(kThreads) k_dft_inverse(const float* __restrict__ c,
                                                          float* __restrict__ g, int rows,
                                                          const float* __restrict__ tab, int nlon,
                                                          int nfc, int rows_per_block) {
  extern __shared__ float smem[];
  float* ts = smem;               // [nfc][nlon]
  float* cs = smem + nlon * nfc;  // [rows_per_block][nfc]
  const int row0 = blockIdx.x * rows_per_block;
  const int nrows = min(rows_per_block, rows - row0);
  for (int i = threadIdx.x; i < nlon * nfc; i += blockDim.x) ts[i] = tab[i];
  for (int i = threadIdx.x; i < nrows * nfc; i += blockDim.x) cs[i] = c[(size_t)row0 * nfc + i];
  __syncthreads();
  for (int o = threadIdx.x; o < nrows * nlon; o += blockDim.x) {
    const int r = o / nlon, j = o % nlon;
    const float* cr = cs + r * nfc;
    float s = 0.f;
    for (int k = 0; k < nfc; ++k) s = fmaf(ts[k * nlon + j], cr[k], s);
    g[(size_t)(row0 + r) * nlon + j] = s;
  }
}

// gpmt: d/dlambda in Fourier space, (re, im) * i m (fourier/wgsl/dlambda.wgsl).
__global__ void k_dlambda(const float* __restrict__ a, float* __restrict__ b, int n, int ntp1, int nfc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = i % ntp1;
  const size_t at = (size_t)(i / ntp1) * nfc + 2 * m;
  const float re = a[at], im = a[at + 1];
  b[at] = -im * (float)m;
  b[at + 1] = re * (float)m;
}

// The same on the optimized path's m-major Fourier planes (coefficient
// (m, lat) at 2 * (m * NLAT + lat)).
__global__ void k_dlambda_m_major(const float* __restrict__ a, float* __restrict__ b, int n, int nlat, int ntp1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = (i / nlat) % ntp1;
  const size_t at = 2 * (size_t)i;
  const float re = a[at], im = a[at + 1];
  b[at] = -im * (float)m;
  b[at + 1] = re * (float)m;
}

// ---------------------------------------------------------------- Legendre
// Inverse transforms (sp2fc, sp2fcdmu, dv2uv): output (plane, lat, m) sums
// modes n = m..NTRU of its plane. A block stages a tile of spectral planes
// and the table rows of a tile of latitudes in shared memory (coalesced
// loads, reused by every plane), and each thread computes wavenumbers j and
// NTRU - j together so every thread sums NTRU + 2 terms.
constexpr int kInvPlanes = 4;

struct InvTile {
  int lats;    // latitudes per block
  size_t smem; // bytes
};

InvTile inverse_tile(const Dims& d, int tables, int inputs) {
  const size_t budget = 160 * 1024;
  for (int lats = 16; lats >= 2; lats /= 2) {
    const size_t smem = (size_t)inputs * kInvPlanes * d.NRSP * 4 + (size_t)tables * lats * d.NCSP * 4;
    if (smem <= budget && d.NLAT % lats == 0) return {lats, smem};
  }
  return {1, (size_t)inputs * kInvPlanes * d.NRSP * 4 + (size_t)tables * d.NCSP * 4};
}

__device__ __forceinline__ int mode_first(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }

__global__ void __launch_bounds__(kThreads) k_leg_inverse(const float* __restrict__ s, float* __restrict__ f,
                                                          int planes, const float* __restrict__ q, Dims d,
                                                          int lats) {
  extern __shared__ float smem[];
  float* sp = smem;                        // [kInvPlanes][NRSP]
  float* qs = smem + kInvPlanes * d.NRSP;  // [lats][NCSP]
  const int p0 = blockIdx.x * kInvPlanes;
  const int np = min(kInvPlanes, planes - p0);
  const int lat0 = blockIdx.y * lats;
  for (int i = threadIdx.x; i < np * d.NRSP; i += blockDim.x) sp[i] = s[(size_t)p0 * d.NRSP + i];
  for (int i = threadIdx.x; i < lats * d.NCSP; i += blockDim.x) qs[i] = q[(size_t)lat0 * d.NCSP + i];
  __syncthreads();
  const int pairs = (d.NTP1 + 1) / 2;
  for (int o = threadIdx.x; o < np * lats * pairs; o += blockDim.x) {
    const int j = o % pairs;
    const int lat = (o / pairs) % lats;
    const int p = o / (pairs * lats);
    const float* spp = sp + p * d.NRSP;
    const float* qr = qs + lat * d.NCSP;
    float* out = f + ((size_t)(p0 + p) * d.NLAT + lat0 + lat) * d.NFC;
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      const int m = half == 0 ? j : d.T - j;
      if (half == 1 && m == j) break;
      const int first = mode_first(m, d.NTP1);
      float re = 0.f, im = 0.f;
      for (int w = first; w < first + d.NTP1 - m; ++w) {
        const float qq = qr[w];
        re = fmaf(qq, spp[2 * w], re);
        im = fmaf(qq, spp[2 * w + 1], im);
      }
      out[2 * m] = re;
      out[2 * m + 1] = im;
    }
  }
}

// dv2uv: winds at every latitude from spectral divergence and vorticity,
// with plavor removed from vorticity mode w = 1 (legendre/wgsl/dv2uv.wgsl).
__global__ void __launch_bounds__(kThreads) k_dv2uv(const float* __restrict__ D, const float* __restrict__ Z,
                                                    float* __restrict__ U, float* __restrict__ V, int planes,
                                                    const float* __restrict__ qu, const float* __restrict__ qv,
                                                    float plavor, Dims d, int lats) {
  extern __shared__ float smem[];
  float* sp = smem;                                 // [kInvPlanes][2][NRSP]
  float* qus = smem + 2 * kInvPlanes * d.NRSP;      // [lats][NCSP]
  float* qvs = qus + (size_t)lats * d.NCSP;         // [lats][NCSP]
  const int p0 = blockIdx.x * kInvPlanes;
  const int np = min(kInvPlanes, planes - p0);
  const int lat0 = blockIdx.y * lats;
  for (int i = threadIdx.x; i < np * d.NRSP; i += blockDim.x) {
    const int p = i / d.NRSP, k = i % d.NRSP;
    sp[(2 * p) * d.NRSP + k] = D[(size_t)p0 * d.NRSP + i];
    float z = Z[(size_t)p0 * d.NRSP + i];
    if (k == 2) z -= plavor;  // w == 1, real part
    sp[(2 * p + 1) * d.NRSP + k] = z;
  }
  for (int i = threadIdx.x; i < lats * d.NCSP; i += blockDim.x) {
    qus[i] = qu[(size_t)lat0 * d.NCSP + i];
    qvs[i] = qv[(size_t)lat0 * d.NCSP + i];
  }
  __syncthreads();
  const int pairs = (d.NTP1 + 1) / 2;
  for (int o = threadIdx.x; o < np * lats * pairs; o += blockDim.x) {
    const int j = o % pairs;
    const int lat = (o / pairs) % lats;
    const int p = o / (pairs * lats);
    const float* dd = sp + (2 * p) * d.NRSP;
    const float* zz = sp + (2 * p + 1) * d.NRSP;
    const float* qur = qus + lat * d.NCSP;
    const float* qvr = qvs + lat * d.NCSP;
    const size_t row = ((size_t)(p0 + p) * d.NLAT + lat0 + lat) * d.NFC;
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      const int m = half == 0 ? j : d.T - j;
      if (half == 1 && m == j) break;
      const int first = mode_first(m, d.NTP1);
      float ure = 0.f, uim = 0.f, vre = 0.f, vim = 0.f;
      for (int w = first; w < first + d.NTP1 - m; ++w) {
        const float a = qur[w], b = qvr[w];
        const float zre = zz[2 * w], zim = zz[2 * w + 1], dre = dd[2 * w], dim = dd[2 * w + 1];
        ure = ure + b * zre + a * dim;
        uim = uim + b * zim - a * dre;
        vre = vre + a * zim - b * dre;
        vim = vim - a * zre - b * dim;
      }
      U[row + 2 * m] = ure;
      U[row + 2 * m + 1] = uim;
      V[row + 2 * m] = vre;
      V[row + 2 * m + 1] = vim;
    }
  }
}

// Forward transforms: each output (plane, mode w) sums latitude pairs of its
// plane's Fourier coefficients at wavenumber m; a block stages kFwdPlanes
// Fourier planes of each input.
template <int NIN>
struct FwdIn {
  const float* p[NIN];
};

// kind 0: fc2sp with table q (legendre/wgsl/forward.wgsl).
// kind 1: uv2dv, in = {u, v}, outputs D, Z (uv2dv.wgsl without the KE term).
// kind 2: mktend's uv2dv, in = {u, v, ke} (uv2dv.wgsl with HAS_KINETIC).
// kind 3: qtend, in = {u, v, source} (qtend.wgsl).
template <int KIND, int NIN>
__global__ void __launch_bounds__(kThreads) k_leg_forward(FwdIn<NIN> in, float* __restrict__ out0,
                                                          float* __restrict__ out1, int planes,
                                                          int planes_per_block, SharedTabs sh,
                                                          const float* __restrict__ q, Dims d) {
  extern __shared__ float fs[];  // [NIN][planes_per_block][NLAT * NFC]
  const int plane_floats = d.NLAT * d.NFC;
  const int p0 = blockIdx.x * planes_per_block;
  const int np = min(planes_per_block, planes - p0);
  for (int k = 0; k < NIN; ++k)
    for (int i = threadIdx.x; i < np * plane_floats; i += blockDim.x)
      fs[(size_t)k * planes_per_block * plane_floats + i] = in.p[k][(size_t)p0 * plane_floats + i];
  __syncthreads();
  const int half = d.NLAT / 2;
  for (int o = threadIdx.x; o < np * d.NCSP; o += blockDim.x) {
    const int w = o % d.NCSP;
    const int p = o / d.NCSP;
    const int m = sh.mode_m[w], n = sh.mode_n[w];
    const float s = ((m + n) & 1) == 0 ? 1.f : -1.f;
    const size_t at = (size_t)(p0 + p) * d.NRSP + 2 * w;
    if (KIND == 0) {
      const float* fp = fs + p * plane_floats + 2 * m;
      float re = 0.f, im = 0.f;
      for (int l = 0; l < half; ++l) {
        const float qq = q[l * d.NCSP + w];
        const float* north = fp + l * d.NFC;
        const float* south = fp + (d.NLAT - 1 - l) * d.NFC;
        re = fmaf(qq, north[0] + s * south[0], re);
        im = fmaf(qq, north[1] + s * south[1], im);
      }
      out0[at] = re;
      out0[at + 1] = im;
    } else if (KIND == 1 || KIND == 2) {
      const float* U = fs + p * plane_floats + 2 * m;
      const float* V = U + (size_t)planes_per_block * plane_floats;
      const float* K = V + (size_t)planes_per_block * plane_floats;
      float dre = 0.f, dim = 0.f, zre = 0.f, zim = 0.f;
      for (int l = 0; l < half; ++l) {
        const int north = l * d.NFC, south = (d.NLAT - 1 - l) * d.NFC;
        const float e = sh.qe[l * d.NCSP + w], mq = sh.qm[l * d.NCSP + w];
        const float dure = U[north] - s * U[south], duim = U[north + 1] - s * U[south + 1];
        const float dvre = V[north] - s * V[south], dvim = V[north + 1] - s * V[south + 1];
        const float sure = U[north] + s * U[south], suim = U[north + 1] + s * U[south + 1];
        const float svre = V[north] + s * V[south], svim = V[north + 1] + s * V[south + 1];
        if (KIND == 2) {
          const float q2 = sh.qq[l * d.NCSP + w];
          dre = dre + q2 * (K[north] + s * K[south]);
          dim = dim + q2 * (K[north + 1] + s * K[south + 1]);
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
      const float* U = fs + p * plane_floats + 2 * m;
      const float* V = U + (size_t)planes_per_block * plane_floats;
      const float* X = V + (size_t)planes_per_block * plane_floats;
      float re = 0.f, im = 0.f;
      for (int l = 0; l < half; ++l) {
        const int north = l * d.NFC, south = (d.NLAT - 1 - l) * d.NFC;
        const float e = sh.qe[l * d.NCSP + w], c = sh.qc[l * d.NCSP + w], mq = sh.qm[l * d.NCSP + w];
        re = re + e * (V[north] - s * V[south]) + c * (X[north] + s * X[south]) +
             mq * (U[north + 1] + s * U[south + 1]);
        im = im + e * (V[north + 1] - s * V[south + 1]) + c * (X[north + 1] + s * X[south + 1]) -
             mq * (U[north] + s * U[south]);
      }
      out0[at] = re;
      out0[at + 1] = im;
    }
  }
}

int forward_planes_per_block(const Dims& d, int nin) {
  const int plane_bytes = d.NLAT * d.NFC * 4;
  const int budget = 96 * 1024;
  int ppb = budget / (plane_bytes * nin);
  return ppb < 1 ? 1 : (ppb > 8 ? 8 : ppb);
}

// Dynamic shared memory above 48 KB needs an opt-in per kernel; tr_init sets
// it once for every transform kernel before any launch or graph capture.
constexpr int kMaxDynamicSmem = 200 * 1024;
template <typename K>
void allow_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
}

template <int KIND, int NIN>
void launch_forward(const Model& m, FwdIn<NIN> in, float* out0, float* out1, int planes, const float* q,
                    cudaStream_t st) {
  const int ppb = forward_planes_per_block(m.d, NIN);
  const size_t smem = (size_t)NIN * ppb * m.d.NLAT * m.d.NFC * sizeof(float);
  auto kernel = k_leg_forward<KIND, NIN>;
  const int blocks = (planes + ppb - 1) / ppb;
  kernel<<<blocks, kThreads, smem, st>>>(in, out0, out1, planes, ppb, m.sh, q, m.d);
}

int dft_rows_per_block(const Dims& d) { return d.NLAT == 96 ? 24 : 32; }

}  // namespace

void tr_init() {
  leg_init();
  tc_init();
  fft_init();
  grid_init();
  allow_smem(k_dft_forward);
  allow_smem(k_dft_inverse);
  allow_smem(k_leg_inverse);
  allow_smem(k_dv2uv);
  allow_smem(k_leg_forward<0, 1>);
  allow_smem(k_leg_forward<1, 2>);
  allow_smem(k_leg_forward<2, 3>);
  allow_smem(k_leg_forward<3, 3>);
}

void tr_fourier_forward(const Model& m, const float* g, float* c, int planes, cudaStream_t st) {
  if (m.mode >= 1) return fft_forward(m, g, c, planes, st);
  const int rows = planes * m.d.NLAT;
  const int rpb = dft_rows_per_block(m.d);
  const size_t smem = ((size_t)m.d.NLON * m.d.NFC + (size_t)rpb * m.d.NLON) * sizeof(float);
  k_dft_forward<<<(rows + rpb - 1) / rpb, kThreads, smem, st>>>(g, c, rows, m.sh.fwd, m.d.NLON, m.d.NFC, rpb);
}

void tr_fourier_inverse(const Model& m, const float* c, float* g, int planes, cudaStream_t st) {
  if (m.mode >= 1) return fft_inverse(m, c, g, planes, st);
  const int rows = planes * m.d.NLAT;
  const int rpb = dft_rows_per_block(m.d);
  const size_t smem = ((size_t)m.d.NLON * m.d.NFC + (size_t)rpb * m.d.NFC) * sizeof(float);
  k_dft_inverse<<<(rows + rpb - 1) / rpb, kThreads, smem, st>>>(c, g, rows, m.sh.inv, m.d.NLON, m.d.NFC, rpb);
}

void tr_dlambda(const Model& m, const float* a, float* b, int planes, cudaStream_t st) {
  const int n = planes * m.d.NLAT * m.d.NTP1;
  if (m.mode >= 1) {
    k_dlambda_m_major<<<(n + 255) / 256, 256, 0, st>>>(a, b, n, m.d.NLAT, m.d.NTP1);
    return;
  }
  k_dlambda<<<(n + 255) / 256, 256, 0, st>>>(a, b, n, m.d.NTP1, m.d.NFC);
}

void tr_sp2gp(const Model& m, const float* s, float* f, float* g, int planes, const float* q, cudaStream_t st) {
  if (m.mode == 1 && (q == m.sh.qi || q == m.sh.qj)) return grid_sp2gp(m, s, f, g, planes, q == m.sh.qj, st);
  tr_legendre_inverse(m, s, f, planes, q, st);
  tr_fourier_inverse(m, f, g, planes, st);
}

void tr_legendre_inverse(const Model& m, const float* s, float* f, int planes, const float* q,
                         cudaStream_t st) {
  if (m.mode >= 1 && (q == m.sh.qi || q == m.sh.qj)) {
    if (m.mode == 2) return tc_inverse(m, s, f, planes, q == m.sh.qj, st);
    return leg_inverse(m, s, f, planes, q == m.sh.qj, st);
  }
  const InvTile t = inverse_tile(m.d, 1, 1);
  dim3 grid((planes + kInvPlanes - 1) / kInvPlanes, m.d.NLAT / t.lats);
  k_leg_inverse<<<grid, kThreads, t.smem, st>>>(s, f, planes, q, m.d, t.lats);
}

void tr_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
              cudaStream_t st) {
  if (m.mode == 2) return tc_dv2uv(m, D, Z, U, V, planes, plavor, st);
  if (m.mode >= 1) return leg_dv2uv(m, D, Z, U, V, planes, plavor, st);
  const InvTile t = inverse_tile(m.d, 2, 2);
  dim3 grid((planes + kInvPlanes - 1) / kInvPlanes, m.d.NLAT / t.lats);
  k_dv2uv<<<grid, kThreads, t.smem, st>>>(D, Z, U, V, planes, m.sh.qu, m.sh.qv, plavor, m.d, t.lats);
}

void tr_legendre_forward(const Model& m, const float* f, float* s, int planes, const float* q,
                         cudaStream_t st) {
  if (m.mode == 2 && q == m.sh.qc) return tc_forward(m, f, s, planes, st);
  if (m.mode >= 1) return leg_forward(m, f, s, planes, q, st);
  FwdIn<1> in{{f}};
  launch_forward<0, 1>(m, in, s, nullptr, planes, q, st);
}

void tr_uv2dv(const Model& m, const float* u, const float* v, const float* ke, float* D, float* Z, int planes,
              cudaStream_t st) {
  if (m.mode == 2) return tc_uv2dv(m, u, v, ke, D, Z, planes, st);
  if (m.mode >= 1) return leg_uv2dv(m, u, v, ke, D, Z, planes, st);
  if (ke) {
    FwdIn<3> in{{u, v, ke}};
    launch_forward<2, 3>(m, in, D, Z, planes, nullptr, st);
  } else {
    FwdIn<2> in{{u, v}};
    launch_forward<1, 2>(m, in, D, Z, planes, nullptr, st);
  }
}

void tr_qtend(const Model& m, const float* u, const float* v, const float* src, float* out, int planes,
              cudaStream_t st) {
  if (m.mode == 2) return tc_qtend(m, u, v, src, out, planes, st);
  if (m.mode >= 1) return leg_qtend(m, u, v, src, out, planes, st);
  FwdIn<3> in{{u, v, src}};
  launch_forward<3, 3>(m, in, out, nullptr, planes, nullptr, st);
}

}  // namespace exogcm
