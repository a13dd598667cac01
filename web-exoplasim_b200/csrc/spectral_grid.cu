// Inverse spectral transforms fused with the longitude FFT (optimized path):
// spectral plane -> grid plane in one kernel, so that the Fourier
// coefficients between sp2fc (legendre/wgsl/inverse.wgsl) and fc2gp
// (fourier/wgsl/inverse.wgsl) stay in shared memory instead of making a
// round trip through HBM.
//
// A block owns JR = 8 latitude pairs (16 rows of every plane) and walks a
// range of planes two (or four) at a time. Its slice of the northern table is
// copied in once (16-byte asynchronous copies of a slice laid out in HBM as
// it sits in shared memory), pair-major ([pair][mode]): a row pitch of 4
// (mod 32) banks and each
// wavenumber's modes starting at a position of residue u (mod 4), for the
// wavenumber pair u that reads them, put the 32 lanes of a warp (8 pairs x 4
// wavenumber pairs) on 32 distinct banks. Per plane pair:
//  1. Legendre: thread (wavenumber pair u, latitude pair jj) sums the modes of
//     wavenumbers u and NTP1 - 1 - u for both planes: even-(n-m) and
//     odd-(n-m) partial sums E, O in the order of the unfused latitude-pair
//     kernel (legendre.cu), north = E + O, south = s (E - O). The Fourier
//     coefficients go to the FFT's coefficient stage [plane][m][row].
//  2. FFT: the 32 rows of the pair, T threads per row, the four-step FFT of
//     fft.cu; rows are written to the grid plane.
// The next pair's spectral coefficients are fetched into registers during
// step 2, and the spectral stage shares its memory with the FFT's exchange
// rows. Results equal the unfused kernels' bit for bit. When the model asks
// to keep the Fourier fields (stage replay), step 1 also writes them in the
// path's m-major layout.
#include <cuda_runtime.h>

#include <algorithm>

#include "async_copy.cuh"
#include "common.cuh"
#include "fft_core.cuh"
#include "launch.h"

namespace exogcm {

// A block's slice of the northern table: JR latitude pairs, each a row of
// grid_table_pitch floats holding every mode, wavenumber m's modes from
// position grid_table_positions()[m]. The slices are laid out so in HBM
// once per resolution (grid_table_layout), and a block copies its slice
// into shared memory as it stands.
constexpr int kGridPairs = 8;

__host__ __device__ __forceinline__ int mode_start(int m, int ntp1) { return m * (2 * ntp1 - m + 1) / 2; }

// Row pitch: every mode plus up to 3 floats of alignment gap per wavenumber,
// rounded to 4 (mod 32) banks.
__host__ __device__ constexpr int grid_table_pitch(int ntp1) {
  return ntp1 * (ntp1 + 1) / 2 + 3 * ntp1 + ((((4 - (ntp1 * (ntp1 + 1) / 2 + 3 * ntp1)) % 32) + 32) % 32);
}

// m is read by wavenumber pair u = m (m < (NTP1 + 1) / 2) or u = NTP1 - 1 - m,
// and its modes start at a position of residue u (mod 4).
__host__ __device__ __forceinline__ void grid_table_positions(int ntp1, int* pos) {
  const int groups = (ntp1 + 1) / 2;
  int at = 0;
  for (int m = 0; m < ntp1; ++m) {
    const int u = m < groups ? m : ntp1 - 1 - m;
    at += ((u - at) % 4 + 4) % 4;
    pos[m] = at;
    at += ntp1 - m;
  }
}

std::vector<float> grid_table_layout(const Dims& d, const std::vector<double>& qT) {
  const int JH = d.NLAT / 2, chunks = JH / kGridPairs, TP = grid_table_pitch(d.NTP1);
  std::vector<int> pos(d.NTP1);
  grid_table_positions(d.NTP1, pos.data());
  std::vector<float> out((size_t)chunks * kGridPairs * TP, 0.f);
  for (int c = 0; c < chunks; ++c)
    for (int jj = 0; jj < kGridPairs; ++jj) {
      float* row = out.data() + ((size_t)c * kGridPairs + jj) * TP;
      for (int m = 0, w = 0; m < d.NTP1; ++m)
        for (int k = 0; k < d.NTP1 - m; ++k, ++w) row[pos[m] + k] = (float)qT[(size_t)w * JH + c * kGridPairs + jj];
    }
  return out;
}

namespace {

using namespace fftcore;

template <int Q, int PPASS = 2>
struct GridShape {
  using F = Shape<Q>;
  static constexpr int M = F::M, N = F::N, NTP1 = F::NTP1, T = F::T;
  static constexpr int NLAT = M, JH = M / 2;
  static constexpr int NCSP = NTP1 * (NTP1 + 1) / 2;
  static constexpr int JR = kGridPairs;   // latitude pairs per block
  static constexpr int ROWS = 2 * JR;     // rows of a plane
  static constexpr int PP = PPASS;        // planes per pass (2 or 4)
  static constexpr int NPAIR = PP / 2;    // plane pairs per pass
  static constexpr int FROWS = PP * ROWS; // FFT rows per pass
  static constexpr int THREADS = FROWS * T;
  static constexpr int GROUPS = (NTP1 + 1) / 2;
  static constexpr int TASKS = GROUPS * JR * NPAIR;
  static constexpr int TP = grid_table_pitch(NTP1);                // table row pitch, 4 (mod 32)
  static_assert((JR * TP) % 4 == 0, "a table slice is whole 16-byte chunks");
  static constexpr int PITCH = (ROWS + (((16 / T - ROWS) % 16) + 16) % 16);
  static constexpr int FC = NTP1 * PITCH;  // float2s of one plane's coefficient stage
  static constexpr int SPEC = NPAIR * NCSP;  // float4s of the spectral stage ([pair][mode], two planes each)
  static constexpr int XB = FROWS * 9 * Q;   // float2s of the FFT exchange rows
  static constexpr int SHARED = (2 * SPEC > XB ? 2 * SPEC : XB);  // float2s of the union
  static constexpr int R = (SPEC + THREADS - 1) / THREADS;        // spectral float4s per thread
  static_assert((N + 9 * Q + PP * FC) % 2 == 0, "the spectral stage must start 16-byte aligned");
  static_assert((N + 9 * Q + PP * FC + SHARED) % 2 == 0, "the table slice must start 16-byte aligned");
  static size_t smem() {
    return ((size_t)N + 9 * Q + (size_t)PP * FC + SHARED) * sizeof(float2) + (size_t)JR * TP * sizeof(float) +
           (size_t)NTP1 * sizeof(int);
  }
};

// Grid row of stage row rr of the block starting at pair j0: rows 0..JR-1
// are the northern latitudes j0.., rows JR..2JR-1 the southern ones in
// ascending order (NLAT - 2 JR - j0 + rr).
template <typename G>
__device__ __forceinline__ int stage_lat(int rr, int j0) {
  return rr < G::JR ? j0 + rr : G::NLAT - 2 * G::JR - j0 + rr;
}

// PP planes per pass: 2, or 4 (twice the threads and stages per block, the
// table slice and the barriers shared by twice the planes; the autotuner picks).
template <int Q, int PP>
__global__ void __launch_bounds__(GridShape<Q, PP>::THREADS)
    k_sp2gp(const float* __restrict__ s, float* __restrict__ f, float* __restrict__ g, int planes, int per_block,
            const float* __restrict__ qT, const float2* __restrict__ twg, int odd,
            int keep) {
  using G = GridShape<Q, PP>;
  constexpr int T = G::T, M = G::M, N = G::N, NTP1 = G::NTP1, JR = G::JR, JH = G::JH, TP = G::TP;
  constexpr int NLAT = G::NLAT, ROWS = G::ROWS, PITCH = G::PITCH, NCSP = G::NCSP, R = G::R;
  constexpr size_t SPLANE = 2 * (size_t)NCSP;              // floats of a spectral plane (NRSP)
  constexpr size_t FPLANE = (size_t)NLAT * 2 * NTP1;       // floats of a Fourier plane
  constexpr size_t GPLANE = (size_t)NLAT * N;              // floats of a grid plane
  extern __shared__ float4 smem4[];
  float2* tw = reinterpret_cast<float2*>(smem4);
  float2* twq = tw + N;
  float2* fc = twq + 9 * Q;               // [PP][NTP1][PITCH]
  float2* shared = fc + G::PP * G::FC;    // spectral stage [NPAIR][NCSP] float4, or the FFT exchange rows
  float4* spec = reinterpret_cast<float4*>(shared);
  float2* xb = shared;
  float* tab = reinterpret_cast<float*>(shared + G::SHARED);  // [JR][TP]
  int* tpos = reinterpret_cast<int*>(tab + JR * TP);           // [NTP1] first position of m's modes
  const int chunks = JH / JR;
  const int j0 = (blockIdx.x % chunks) * JR;
  const int pbeg = (blockIdx.x / chunks) * per_block;
  const int pend = min(planes, pbeg + per_block);

  // Spectral coefficients of the pass's plane pairs (p + 2k, p + 2k + 1)
  // as (re a, im a, re b, im b), pair-major.
  float4 rs[R];
  auto fetch = [&](int p) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int e = threadIdx.x + i * G::THREADS;
      const int pair = e / NCSP, w = e - pair * NCSP;
      const int pa = p + 2 * pair;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e < G::SPEC && pa < pend) {
        const float2 x = reinterpret_cast<const float2*>(s + (size_t)pa * SPLANE)[w];
        const float2 y = pa + 1 < pend ? reinterpret_cast<const float2*>(s + (size_t)(pa + 1) * SPLANE)[w]
                                       : make_float2(0.f, 0.f);
        v = make_float4(x.x, x.y, y.x, y.y);
      }
      rs[i] = v;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int e = threadIdx.x + i * G::THREADS;
      if (e < G::SPEC) spec[e] = rs[i];
    }
  };

  {
    // the block's table slice, laid out in HBM as it sits here
    const float4* src = reinterpret_cast<const float4*>(qT + (size_t)(j0 / JR) * JR * TP);
    float4* dst = reinterpret_cast<float4*>(tab);
    for (int i = threadIdx.x; i < JR * TP / 4; i += G::THREADS) cp_async16(dst + i, src + i);
    cp_async_commit();
  }
  if (pbeg < pend) fetch(pbeg);
  load_twiddles<Q>(twg, tw, twq);
  if (threadIdx.x == 0) grid_table_positions(NTP1, tpos);
  store();
  cp_async_wait_all();
  __syncthreads();

  const float sg = odd ? -1.f : 1.f;
  const int r = threadIdx.x / T, t = threadIdx.x % T;  // FFT row and lane
  const int pr = r / ROWS, rr = r - pr * ROWS;         // plane of the pass, stage row
  const int lat = stage_lat<G>(rr, j0);
  for (int p = pbeg; p < pend; p += G::PP) {
    // 1. Legendre sums into the coefficient stage.
    for (int task = threadIdx.x; task < G::TASKS; task += G::THREADS) {
      const int pair = task / (G::GROUPS * JR), rest = task - pair * (G::GROUPS * JR);
      const int u = rest / JR, jj = rest - u * JR;
#pragma unroll 1
      for (int side = 0; side < 2; ++side) {
        const int m = side == 0 ? u : NTP1 - 1 - u;
        if (side == 1 && m == u) break;
        const int w0 = mode_start(m, NTP1), K = NTP1 - m;
        const float* qc = tab + jj * TP + tpos[m];
        const float4* sc = spec + pair * NCSP + w0;
        float4 e = make_float4(0.f, 0.f, 0.f, 0.f), o = e;  // (re a, im a, re b, im b)
        int k = 0;
#pragma unroll 2
        for (; k + 1 < K; k += 2) {
          const float qe = qc[k], qo = qc[k + 1];
          const float4 ve = sc[k], vo = sc[k + 1];
          e.x = fmaf(qe, ve.x, e.x);
          e.y = fmaf(qe, ve.y, e.y);
          e.z = fmaf(qe, ve.z, e.z);
          e.w = fmaf(qe, ve.w, e.w);
          o.x = fmaf(qo, vo.x, o.x);
          o.y = fmaf(qo, vo.y, o.y);
          o.z = fmaf(qo, vo.z, o.z);
          o.w = fmaf(qo, vo.w, o.w);
        }
        if (k < K) {
          const float qe = qc[k];
          const float4 ve = sc[k];
          e.x = fmaf(qe, ve.x, e.x);
          e.y = fmaf(qe, ve.y, e.y);
          e.z = fmaf(qe, ve.z, e.z);
          e.w = fmaf(qe, ve.w, e.w);
        }
        float2* fa = fc + (2 * pair) * G::FC + m * PITCH;
        float2* fb = fa + G::FC;
        const int rn = jj, rsouth = ROWS - 1 - jj;
        fa[rn] = make_float2(e.x + o.x, e.y + o.y);
        fa[rsouth] = make_float2(sg * (e.x - o.x), sg * (e.y - o.y));
        fb[rn] = make_float2(e.z + o.z, e.w + o.w);
        fb[rsouth] = make_float2(sg * (e.z - o.z), sg * (e.w - o.w));
      }
    }
    __syncthreads();
    if (keep) {
      for (int i = threadIdx.x; i < G::PP * NTP1 * ROWS; i += G::THREADS) {
        const int q = i / (NTP1 * ROWS), rem = i - q * NTP1 * ROWS, m = rem / ROWS, row = rem - m * ROWS;
        if (p + q < pend)
          reinterpret_cast<float2*>(f + (size_t)(p + q) * FPLANE)[(size_t)m * NLAT + stage_lat<G>(row, j0)] =
              fc[q * G::FC + m * PITCH + row];
      }
    }
    const int next = p + G::PP;
    if (next < pend) fetch(next);
    // 2. FFT of the pass's rows (the exchange rows reuse the spectral stage).
    const float2* fr = fc + pr * G::FC;
    float2 a[G::F::QT][8];
#pragma unroll
    for (int i = 0; i < G::F::QT; ++i)
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = Q * q + t + T * i, km = M - k;
        float2 gk = k < NTP1 ? fr[k * PITCH + rr] : make_float2(0.f, 0.f);
        if (k == 0) gk.y = 0.f;  // Im c_0 is ignored
        const float2 gmk = conj2(km < NTP1 ? fr[km * PITCH + rr] : make_float2(0.f, 0.f));
        const float2 ev = cadd(gk, gmk);
        const float2 ov = cmul(csub(gk, gmk), tw[k]);
        a[i][q] = make_float2(ev.x - ov.y, ev.y + ov.x);  // e + i o
      }
    float2 b[G::F::KT][Q];
    four_step<Q, 1>(a, b, twq, xb + r * G::F::XP, t);
    if (p + pr < pend) {
      float2* out = reinterpret_cast<float2*>(g + (size_t)(p + pr) * GPLANE + (size_t)lat * N);
#pragma unroll
      for (int j = 0; j < G::F::KT; ++j)
#pragma unroll
        for (int k2 = 0; k2 < Q; ++k2) out[t + T * j + 8 * k2] = b[j][k2];
    }
    __syncthreads();
    if (next < pend) {
      store();
      __syncthreads();
    }
  }
}

template <int Q, int PP>
void launch_sp2gp(const Model& m, const float* s, float* f, float* g, int planes, const float* qT, int odd,
                  cudaStream_t st) {
  using G = GridShape<Q, PP>;
  const size_t smem = G::smem();
  const int chunks = G::JH / G::JR;
  const int passes = (planes + PP - 1) / PP;
  const int target = persistent_grid((const void*)k_sp2gp<Q, PP>, G::THREADS, smem);
  const int splits = std::max(1, std::min(passes, (target + chunks - 1) / chunks));
  const int per_passes = (passes + splits - 1) / splits;
  const int blocks = chunks * ((passes + per_passes - 1) / per_passes);
  k_sp2gp<Q, PP><<<blocks, G::THREADS, smem, st>>>(s, f, g, planes, PP * per_passes, qT,
                                                    reinterpret_cast<const float2*>(m.sh.tw), odd, m.keep_fourier);
}

template <int Q, int PP>
void allow_sp2gp_smem() {
  cudaFuncSetAttribute(k_sp2gp<Q, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GridShape<Q, PP>::smem());
}

}  // namespace

void grid_init() {
  allow_sp2gp_smem<4, 2>();
  allow_sp2gp_smem<8, 2>();
  allow_sp2gp_smem<12, 2>();
  allow_sp2gp_smem<4, 4>();
  allow_sp2gp_smem<8, 4>();
  allow_sp2gp_smem<12, 4>();
}

size_t grid_sp2gp_smem(const Dims& d, int planes_per_pass) {
  const bool four = planes_per_pass == 4;
  switch (d.NLON) {
    case 64: return four ? GridShape<4, 4>::smem() : GridShape<4, 2>::smem();
    case 128: return four ? GridShape<8, 4>::smem() : GridShape<8, 2>::smem();
    default: return four ? GridShape<12, 4>::smem() : GridShape<12, 2>::smem();
  }
}

void grid_sp2gp(const Model& m, const float* s, float* f, float* g, int planes, bool derivative, cudaStream_t st) {
  const float* qT = derivative ? m.sh.qjG : m.sh.qiG;
  const int odd = derivative ? 1 : 0;
  const bool four = m.tune.sp2gp_planes == 4;
  switch (m.d.NLON) {
    case 64:
      four ? launch_sp2gp<4, 4>(m, s, f, g, planes, qT, odd, st) : launch_sp2gp<4, 2>(m, s, f, g, planes, qT, odd, st);
      break;
    case 128:
      four ? launch_sp2gp<8, 4>(m, s, f, g, planes, qT, odd, st) : launch_sp2gp<8, 2>(m, s, f, g, planes, qT, odd, st);
      break;
    default:
      four ? launch_sp2gp<12, 4>(m, s, f, g, planes, qT, odd, st)
           : launch_sp2gp<12, 2>(m, s, f, g, planes, qT, odd, st);
      break;
  }
}

}  // namespace exogcm
