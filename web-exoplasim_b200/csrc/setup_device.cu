// The set-up's heavy FP64 loops on the device: legini with the filters, the
// grid -> spectral analysis of the initial state and orography, and makebm's
// LU inverses. Every kernel keeps the host loop's order of operations
// (setup.cpp) and this file is compiled with -fmad=false, so a device result
// equals the host's bit for bit (FP64 division and square root are IEEE
// round-to-nearest on both).
//
//   legini   legendre/index.ts:29-136   one thread per (latitude, zonal m)
//   analyse  fourier/index.ts:95-115    one block per (plane, latitude row),
//            legendre/index.ts:334-361  then one thread per (plane, mode, part)
//   makebm   dynamics/setup/index.ts:154-239  one thread per (phase, degree)
#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <string>

#include "setup.h"

namespace exogcm {
namespace {

constexpr int kMaxLevels = 10;
constexpr int kTables = 8;  // qi qj qc qe qm qq qu qv, then the unfiltered qc

void cuda_ok(cudaError_t err, const char* what) {
  if (err != cudaSuccess) throw std::runtime_error(std::string("set-up device: ") + what + ": " + cudaGetErrorString(err));
}

// First compact mode index of zonal wavenumber m (modes ordered m-major,
// n = m..T within each m).
__host__ __device__ inline int mode_base(int m, int T) { return m * (T + 1) - m * (m - 1) / 2; }

// legendre/index.ts:29-108 for the column (lat, m). The diagonal chain
// f1m/f2m runs from m' = 1 to m in the host's order; the n recurrence keeps
// the two previous P values in registers. Writes the eight filtered tables
// tabs[t][lat][mode] (t in qi qj qc qe qm qq qu qv) and the unfiltered qc at
// tabs[8].
__global__ void k_legini(const double* __restrict__ sines, const double* __restrict__ weights,
                         const double* __restrict__ g2s, const double* __restrict__ s2g, int T, int nlat,
                         double* __restrict__ tabs) {
  const int lat = blockIdx.x, m = threadIdx.x;
  if (lat >= nlat || m > T) return;
  const int modes = (T + 1) * (T + 2) / 2;
  const size_t plane = (size_t)nlat * modes;
  const double sin = sines[lat], weight = weights[lat];
  const double cos2 = 1 - sin * sin, wocs = weight / cos2;
  const int base = mode_base(m, T);
  const int last = modes - 1;  // the mode (T, T)

  auto emit = [&](int n, double p, double d) {
    const int w = base + (n - m);
    const double invdeg = n > 0 ? 1.0 / ((double)n * (n + 1)) : 0.0;
    const size_t at = (size_t)lat * modes + w;
    const double vi = p, vj = d, vc = p * weight, vu = p * invdeg * m, vv = d * invdeg, ve = d * wocs;
    const double vq = p * wocs * n * (n + 1) * 0.5, vm = p * wocs * m;
    const double fg = g2s[n], fs = s2g[n];
    tabs[0 * plane + at] = vi * fs;
    tabs[1 * plane + at] = vj * fs;
    tabs[2 * plane + at] = vc * fg;
    tabs[3 * plane + at] = ve * fg;
    tabs[4 * plane + at] = vm * fg;
    tabs[5 * plane + at] = vq * fg;
    tabs[6 * plane + at] = vu * fs;
    tabs[7 * plane + at] = vv * fs;
    tabs[8 * plane + at] = vc;
  };

  // P(m, m) and P(m, m + 1), and the derivative of P(m, m).
  double f1m = sqrt(1.5), f2m = 0;
  double p_mm, p_next = 0;
  for (int k = 1; k <= m; ++k) {
    f2m = -f1m * sqrt(cos2 / (k + k));
    f1m = f2m * sqrt((double)(k + k + 3));
  }
  double d_mm = 0;
  if (m == 0) {
    p_mm = sqrt(0.5);
    p_next = f1m * sin;
    d_mm = 0;
  } else {
    p_mm = f2m;
    if (base < last) {
      p_next = f1m * sin;
      d_mm = -m * f2m * sin;
    }
  }
  if (m == T) {  // one mode in the column; it is the last mode overall
    emit(T, p_mm, -T * sin * p_mm);
    return;
  }
  const double m2 = (double)m * m;
  // prev2 = P(m, n - 2), prev1 = P(m, n - 1); the derivative of n - 1 is
  // known once P(m, n) is.
  double prev2 = p_mm, prev1 = p_next;
  double d_prev2 = d_mm;  // derivative of P(m, n - 2), pending emission
  int n = m + 2;
  for (; n <= T; ++n) {
    const double z1 = sqrt(((double)(n - 1) * (n - 1) - m2) / (4.0 * (n - 1) * (n - 1) - 1));
    const double z2 = sin * prev1 - z1 * prev2;
    const double pn = z2 * sqrt((4.0 * n * n - 1) / ((double)n * n - m2));
    const double d_prev1 = (1 - n) * z2 + n * z1 * prev2;
    emit(n - 2, prev2, d_prev2);
    prev2 = prev1;
    prev1 = pn;
    d_prev2 = d_prev1;
  }
  // Here prev2 = P(m, T - 1) with its derivative d_prev2, prev1 = P(m, T).
  emit(T - 1, prev2, d_prev2);
  double d_last;
  if (base + (T - m) < last) {
    const double z3 = sqrt(((double)T * T - m2) / (4.0 * T * T - 1));
    d_last = -T * sin * prev1 + (T + T + 1) * prev2 * z3;
  } else {
    d_last = -T * sin * prev1;
  }
  emit(T, prev1, d_last);
}

// fourier/index.ts:95-115: four[plane][row][c] = sum over j ascending of
// grid[plane][row][j] * fwd[j][c]. One block per (plane, row), one thread
// per coefficient.
__global__ void k_analyse_fourier(const double* __restrict__ grids, const double* __restrict__ fwd, int nlon,
                                  int nfc, int rows, double* __restrict__ four) {
  extern __shared__ double g[];
  const size_t row = blockIdx.x;
  for (int j = threadIdx.x; j < nlon; j += blockDim.x) g[j] = grids[row * nlon + j];
  __syncthreads();
  for (int c = threadIdx.x; c < nfc; c += blockDim.x) {
    double acc = 0;
    for (int j = 0; j < nlon; ++j) acc += g[j] * fwd[(size_t)j * nfc + c];
    four[row * nfc + c] = acc;
  }
}

// legendre/index.ts:334-361: sp[plane][2w + part] = sum over the northern
// latitudes l ascending of qc(l, w) * (north + sign * south) * g2s[n].
__global__ void k_analyse_legendre(const double* __restrict__ four, const double* __restrict__ qc,
                                   const double* __restrict__ g2s, const int* __restrict__ mm,
                                   const int* __restrict__ nn, int nlat, int nfc, int modes, int planes,
                                   double* __restrict__ sp) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)planes * 2 * modes) return;
  const int plane = (int)(i / (2 * modes)), r = (int)(i % (2 * modes));
  const int w = r >> 1, part = r & 1, m = mm[w], n = nn[w];
  const double sign = (m + n) % 2 == 0 ? 1 : -1;
  const double* f = four + (size_t)plane * nlat * nfc;
  double acc = 0;
  for (int l = 0; l < nlat / 2; ++l) {
    const double row = f[(size_t)l * nfc + 2 * m + part] + sign * f[(size_t)(nlat - 1 - l) * nfc + 2 * m + part];
    acc = acc + qc[(size_t)l * modes + w] * row * g2s[n];
  }
  sp[i] = acc;
}

// dynamics/setup/index.ts:154-211 (ludcmp with implicit partial pivoting,
// then lubksb on each unit column), column-major a(i, j) = a[j * n + i], for
// the matrix base + diag(1 / (degree (degree + 1))).
__global__ void k_makebm(const double* __restrict__ bases, int n, int T, double* __restrict__ bm1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * T) return;
  const int phase = t / T, degree = t % T + 1;
  double a[kMaxLevels * kMaxLevels], scale[kMaxLevels], b[kMaxLevels];
  int index[kMaxLevels];
  const double* base = bases + (size_t)phase * n * n;
  for (int i = 0; i < n * n; ++i) a[i] = base[i];
  for (int l = 0; l < n; ++l) a[l * n + l] += 1.0 / ((double)degree * (degree + 1));
#define A(i, j) a[(j) * n + (i)]
  for (int i = 0; i < n; ++i) {
    double largest = 0;
    for (int j = 0; j < n; ++j) largest = fmax(largest, fabs(A(i, j)));
    scale[i] = 1 / largest;
  }
  for (int j = 0; j < n; ++j) {
    for (int i = 1; i < j; ++i) {
      double dot = 0;
      for (int k = 0; k < i; ++k) dot += A(i, k) * A(k, j);
      A(i, j) -= dot;
    }
    double largest = 0;
    int pivot = j;
    for (int i = j; i < n; ++i) {
      if (j > 0) {
        double dot = 0;
        for (int k = 0; k < j; ++k) dot += A(i, k) * A(k, j);
        A(i, j) -= dot;
      }
      const double size = scale[i] * fabs(A(i, j));
      if (size >= largest) {
        pivot = i;
        largest = size;
      }
    }
    if (j != pivot) {
      for (int k = 0; k < n; ++k) {
        const double s = A(pivot, k);
        A(pivot, k) = A(j, k);
        A(j, k) = s;
      }
      scale[pivot] = scale[j];
    }
    index[j] = pivot;
    if (A(j, j) == 0) A(j, j) = 5e-324;
    for (int i = j + 1; i < n; ++i) A(i, j) /= A(j, j);
  }
  double* out = bm1 + ((size_t)phase * T + (degree - 1)) * n * n;
  for (int column = 0; column < n; ++column) {
    for (int i = 0; i < n; ++i) b[i] = 0;
    b[column] = 1;
    int first = -1;
    for (int i = 0; i < n; ++i) {
      const int li = index[i];
      double sum = b[li];
      b[li] = b[i];
      if (first >= 0) {
        for (int j = first; j < i; ++j) sum -= A(i, j) * b[j];
      } else if (sum != 0) {
        first = i;
      }
      b[i] = sum;
    }
    for (int i = n - 1; i >= 0; --i) {
      double sum = b[i];
      for (int j = i + 1; j < n; ++j) sum -= A(i, j) * b[j];
      b[i] = sum / A(i, i);
    }
    for (int i = 0; i < n; ++i) out[(size_t)column * n + i] = b[i];
  }
#undef A
}

// Device buffers that grow on demand, a pinned staging area and a stream of
// its own, so set-up kernels run beside batches stepping on the engine's.
class CudaSetupDevice final : public SetupDevice {
 public:
  CudaSetupDevice() {
    cuda_ok(cudaGetDevice(&device_), "device");
    cuda_ok(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  }
  ~CudaSetupDevice() override {
    if (stream_) cudaStreamDestroy(stream_);
    for (void* p : {(void*)dev_, (void*)tab_dev_, (void*)mn_dev_}) cudaFree(p);
    cudaFreeHost(pinned_);
  }

  void legini(const Vec& sines, const Vec& weights, int T, const Vec& g2s, const Vec& s2g,
              std::map<std::string, Vec>& q, Vec& qc_unfiltered) override {
    const int nlat = (int)sines.size(), modes = (T + 1) * (T + 2) / 2;
    const size_t plane = (size_t)nlat * modes;
    // inputs: sines, weights, g2s, s2g; output: 9 tables
    const size_t in = 2 * (size_t)nlat + 2 * (size_t)(T + 1);
    double* d = device_doubles(in + (kTables + 1) * plane);
    double* h = pinned_doubles(std::max(in, (kTables + 1) * plane));
    std::memcpy(h, sines.data(), nlat * sizeof(double));
    std::memcpy(h + nlat, weights.data(), nlat * sizeof(double));
    std::memcpy(h + 2 * nlat, g2s.data(), (T + 1) * sizeof(double));
    std::memcpy(h + 2 * nlat + T + 1, s2g.data(), (T + 1) * sizeof(double));
    cuda_ok(cudaMemcpyAsync(d, h, in * sizeof(double), cudaMemcpyHostToDevice, stream_), "legini inputs");
    double* tabs = d + in;
    k_legini<<<nlat, T + 1, 0, stream_>>>(d, d + nlat, d + 2 * nlat, d + 2 * nlat + T + 1, T, nlat, tabs);
    cuda_ok(cudaGetLastError(), "legini launch");
    cuda_ok(cudaMemcpyAsync(h, tabs, (kTables + 1) * plane * sizeof(double), cudaMemcpyDeviceToHost, stream_),
            "legini tables");
    cuda_ok(cudaStreamSynchronize(stream_), "legini");
    const char* names[kTables] = {"qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv"};
    for (int t = 0; t < kTables; ++t) q[names[t]] = Vec(h + t * plane, h + (t + 1) * plane);
    qc_unfiltered.assign(h + kTables * plane, h + (kTables + 1) * plane);
    // Keep this resolution's analysis tables resident.
    bind_tables(T, nlat, qc_unfiltered, g2s, nullptr);
  }

  void analyse(const SharedSetup& sh, const double* grids, int planes, double* spectra) override {
    const int T = sh.truncation, nlat = sh.nlat, nlon = sh.nlon, nfc = 2 * (T + 1);
    const int modes = (T + 1) * (T + 2) / 2;
    bind_tables(T, nlat, sh.qc_unfiltered, sh.g2s, &sh.fwd);
    const size_t points = (size_t)nlat * nlon, grid = (size_t)planes * points;
    const size_t four = (size_t)planes * nlat * nfc, spec = (size_t)planes * 2 * modes;
    double* d = device_doubles(grid + four + spec);
    double* h = pinned_doubles(std::max(grid, spec));
    std::memcpy(h, grids, grid * sizeof(double));
    cuda_ok(cudaMemcpyAsync(d, h, grid * sizeof(double), cudaMemcpyHostToDevice, stream_), "analyse grids");
    const int threads = nfc <= 64 ? 64 : 128;
    k_analyse_fourier<<<planes * nlat, threads, nlon * sizeof(double), stream_>>>(d, tab_fwd_, nlon, nfc,
                                                                                 planes * nlat, d + grid);
    cuda_ok(cudaGetLastError(), "analyse fourier launch");
    const int blocks = (int)((spec + 127) / 128);
    k_analyse_legendre<<<blocks, 128, 0, stream_>>>(d + grid, tab_qc_, tab_g2s_, mn_dev_, mn_dev_ + modes, nlat,
                                                    nfc, modes, planes, d + grid + four);
    cuda_ok(cudaGetLastError(), "analyse legendre launch");
    cuda_ok(cudaMemcpyAsync(h, d + grid + four, spec * sizeof(double), cudaMemcpyDeviceToHost, stream_),
            "analyse spectra");
    cuda_ok(cudaStreamSynchronize(stream_), "analyse");
    std::memcpy(spectra, h, spec * sizeof(double));
  }

  void makebm(const double* base, int n, int T, double* bm1) override {
    if (n < 1 || n > kMaxLevels) throw std::invalid_argument("makebm: levels must be 1..10");
    const size_t in = 4 * (size_t)n * n, out = 4 * (size_t)T * n * n;
    double* d = device_doubles(in + out);
    double* h = pinned_doubles(std::max(in, out));
    std::memcpy(h, base, in * sizeof(double));
    cuda_ok(cudaMemcpyAsync(d, h, in * sizeof(double), cudaMemcpyHostToDevice, stream_), "makebm bases");
    k_makebm<<<(4 * T + 63) / 64, 64, 0, stream_>>>(d, n, T, d + in);
    cuda_ok(cudaGetLastError(), "makebm launch");
    cuda_ok(cudaMemcpyAsync(h, d + in, out * sizeof(double), cudaMemcpyDeviceToHost, stream_), "makebm inverses");
    cuda_ok(cudaStreamSynchronize(stream_), "makebm");
    std::memcpy(bm1, h, out * sizeof(double));
  }

 private:
  double* device_doubles(size_t count) {
    if (count > dev_cap_) {
      cuda_ok(cudaStreamSynchronize(stream_), "grow");
      cudaFree(dev_);
      dev_ = nullptr;
      cuda_ok(cudaMalloc(&dev_, count * sizeof(double)), "device buffer");
      dev_cap_ = count;
    }
    return dev_;
  }
  double* pinned_doubles(size_t count) {
    if (count > pinned_cap_) {
      cuda_ok(cudaStreamSynchronize(stream_), "grow");
      cudaFreeHost(pinned_);
      pinned_ = nullptr;
      cuda_ok(cudaMallocHost(&pinned_, count * sizeof(double)), "pinned buffer");
      pinned_cap_ = count;
    }
    return pinned_;
  }
  // The analysis tables of one resolution: qc unfiltered, g2s, the mode
  // indices and (once given) the forward Fourier table, resident on the
  // device until the resolution changes.
  void bind_tables(int T, int nlat, const Vec& qc, const Vec& g2s, const Vec* fwd) {
    if (T != tab_T_ || nlat != tab_nlat_ || g2s != tab_g2s_host_) {
      const int modes = (T + 1) * (T + 2) / 2, nlon = 2 * nlat, nfc = 2 * (T + 1);
      const size_t count = (size_t)nlat * modes + (T + 1) + (size_t)nlon * nfc;
      cuda_ok(cudaStreamSynchronize(stream_), "rebind");
      cudaFree(tab_dev_);
      cudaFree(mn_dev_);
      tab_dev_ = nullptr;
      mn_dev_ = nullptr;
      cuda_ok(cudaMalloc(&tab_dev_, count * sizeof(double)), "analysis tables");
      cuda_ok(cudaMalloc(&mn_dev_, 2 * modes * sizeof(int)), "mode indices");
      tab_qc_ = tab_dev_;
      tab_g2s_ = tab_qc_ + (size_t)nlat * modes;
      tab_fwd_ = tab_g2s_ + (T + 1);
      std::vector<int> mn(2 * modes);
      int w = 0;
      for (int m = 0; m <= T; ++m)
        for (int n = m; n <= T; ++n, ++w) {
          mn[w] = m;
          mn[modes + w] = n;
        }
      cuda_ok(cudaMemcpy(tab_qc_, qc.data(), qc.size() * sizeof(double), cudaMemcpyHostToDevice), "qc");
      cuda_ok(cudaMemcpy(tab_g2s_, g2s.data(), g2s.size() * sizeof(double), cudaMemcpyHostToDevice), "g2s");
      cuda_ok(cudaMemcpy(mn_dev_, mn.data(), mn.size() * sizeof(int), cudaMemcpyHostToDevice), "mode indices");
      tab_T_ = T;
      tab_nlat_ = nlat;
      tab_g2s_host_ = g2s;
      fwd_bound_ = false;
    }
    if (fwd && !fwd_bound_) {
      cuda_ok(cudaMemcpy(tab_fwd_, fwd->data(), fwd->size() * sizeof(double), cudaMemcpyHostToDevice), "fwd");
      fwd_bound_ = true;
    }
  }

  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  double* dev_ = nullptr;
  size_t dev_cap_ = 0;
  double* pinned_ = nullptr;
  size_t pinned_cap_ = 0;
  double* tab_dev_ = nullptr;
  double *tab_qc_ = nullptr, *tab_g2s_ = nullptr, *tab_fwd_ = nullptr;
  int* mn_dev_ = nullptr;
  int tab_T_ = -1, tab_nlat_ = -1;
  Vec tab_g2s_host_;
  bool fwd_bound_ = false;
};

}  // namespace

std::unique_ptr<SetupDevice> make_setup_device() { return std::make_unique<CudaSetupDevice>(); }

}  // namespace exogcm
