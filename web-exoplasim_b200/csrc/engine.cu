// The batched GCM engine behind the C ABI of include/exogcm.h.
//
// Mirrors the reference's engine plumbing (src/model/climate/gcm/):
//   configure  -> SETUP.state/schedule + STEPPER.context + LAYOUT.write
//                 (setup/index.ts:434-477, stepper/index.ts:94-118)
//   step       -> STEPPER.values + STEPPER.batch (stepper/index.ts:203-334):
//                 the step's kernels in master's order
//                 (stepper/index.ts:148-161, dynamics/index.ts:171-344)
//   readback   -> LAYOUT.read (layout/index.ts:73-108)
//   checkpoint -> RESTART.encode/decode (checkpoint/restart/index.ts:11-75)
// for S planet slots at once. One device arena holds every field as
// [plane][slot][points]; a batch of K steps is one CUDA graph whose step k
// reads its per-slot host values at params + k * S.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/exogcm.h"
#include "common.cuh"
#include "launch.h"
#include "setup.h"

using namespace exogcm;

namespace {

thread_local std::string g_error;

}  // namespace

namespace exogcm {
void set_error(const std::string& message) { g_error = message; }
}  // namespace exogcm

namespace {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(EXOGCM_EDEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

struct FieldInfo {
  std::string name;
  char shape;
  int count;
  size_t plane;   // floats per plane per slot
  size_t offset;  // floats from the arena base
};

struct Slot {
  bool active = false;
  long step = 0;
  int carbon_step = 0;
  int startup_left = 0;
  long published = -1;
  long stop = -1;  // model step at which the slot stops (-1: never)
  double deltsec[4] = {0}, delt[4] = {0};
  Calendar cal{};
  bool storm = false;  // NSTORMDIAG > 0: hurricanestep runs for this slot
};

constexpr int kMaxBatch = 64;
constexpr int kInFlight = 2;  // batches exogcm_step_async keeps submitted

}  // namespace

struct exogcm_engine {
  Dims d{};
  int mode = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  std::vector<FieldInfo> fields;
  std::map<std::string, size_t> field_index;
  float* arena = nullptr;
  size_t arena_floats = 0;
  FieldPtrs fp{};
  // shared tables
  bool shared_ready = false;
  int filter_kind = -1, filter_gp = -1, filter_sp = -1;
  float* shared_buf = nullptr;
  int* mode_buf = nullptr;
  SharedTabs sh{};
  // per-slot tables and constants
  TabOffsets to{};
  std::vector<std::pair<std::string, int>> tab_list;
  float* tabs = nullptr;
  PlanetConst* pc = nullptr;
  StepParams* params = nullptr;   // device [kMaxBatch][S]
  StepParams* hparams = nullptr;  // pinned host [1 + kInFlight][kMaxBatch][S]: row 0 for synchronous calls
  // Batches submitted by exogcm_step_async and not yet retired, oldest first
  // (the reference's worker keeps IN_FLIGHT = 2 batches submitted,
  // runner/webgpu/gcm.worker.ts:215-225). Batch b uploads its step values
  // from its own pinned row 1 + b, so the host never overwrites values a
  // queued copy has yet to read, and copies the device fault word into its
  // own pinned int before recording its end event.
  struct Batch {
    cudaEvent_t start = nullptr, end = nullptr, done = nullptr;
    int* fault_host = nullptr;
  };
  Batch batch[kInFlight];
  std::deque<int> pending;
  double* sums = nullptr;
  double* budget = nullptr;  // [S][kBudgetStride] FP64 budgets (budget.cu)
  double* avg = nullptr;     // FP64 running sums of the snapshot field, when averages are enabled
  double* wlat64 = nullptr;  // FP64 Gaussian weights [NLAT]
  int* flags = nullptr;
  int* fault = nullptr;  // device word: a kernel gave up a bounded wait
  // overlapped snapshot copies (exogcm_snapshots_begin/wait)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t snap_staged = nullptr, snap_copied = nullptr;
  float* snap_stage = nullptr;  // device copy of the snapshot field
  bool copy_pending = false;
  std::vector<Slot> slots;
  std::map<int, cudaGraphExec_t> graphs;
  std::map<int, cudaGraph_t> graph_templates;  // the captured K-step graphs (child nodes of group graphs)
  Tuning tune{};
  SharedSetup shared_setup;  // host copy of the shared tables (set-up of later planets)
  // FP64 set-up loops on this device (setup_device.cu), created at the first
  // configure; exogcm_setup_on_device(e, 0) moves them to the host.
  std::unique_ptr<SetupDevice> setup_device;
  bool setup_on_device = true;
  float* upload_stage = nullptr;  // pinned floats: one planet's fields and tables on their way in
  size_t upload_stage_floats = 0;

  Model model(int k) const {
    Model m{};
    m.d = d;
    m.f = fp;
    m.sh = sh;
    m.to = to;
    m.tabs = tabs;
    m.pc = pc;
    m.params = params + (size_t)k * d.S;
    m.sums = sums;
    m.budget = budget;
    m.avg = avg;
    m.flags = flags;
    m.fault = fault;
    m.mode = mode;
    m.tune = tune;
    m.keep_fourier = 0;
    m.zero_gdt = 0;
    m.storm = 0;
    for (const Slot& s : slots) m.storm |= s.storm ? 1 : 0;
    return m;
  }
};

namespace {

size_t plane_floats(const Dims& d, char shape) {
  switch (shape) {
    case 'S': return d.NRSP;
    case 'F': return (size_t)d.NLAT * d.NFC;
    case 'G': return d.NHOR;
    default: return 1;
  }
}

void layout(exogcm_engine* e) {
  const Dims& d = e->d;
  const int L = d.L, H = d.L + 1, P = d.P;
  (void)L;
  (void)H;
  (void)P;
  size_t off = 0;
  // Every field starts on a 256-byte boundary (vector loads in the FFTs need
  // at least 8-byte aligned rows whatever the slot count).
#define EXOGCM_ADD_FIELD(name, shape, cnt)                                            \
  {                                                                                   \
    off = (off + 63) / 64 * 64;                                                       \
    FieldInfo fi{#name, #shape[0], (int)(cnt), plane_floats(d, #shape[0]), off};      \
    e->field_index[#name] = e->fields.size();                                         \
    e->fields.push_back(fi);                                                          \
    off += fi.plane * fi.count * d.S;                                                 \
  }
  {
    const int L = d.L;
    EXOGCM_FIELDS(EXOGCM_ADD_FIELD)
  }
#undef EXOGCM_ADD_FIELD
  e->arena_floats = off;
}

void bind_fields(exogcm_engine* e) {
#define EXOGCM_BIND(name, shape, count) e->fp.name = e->arena + e->fields[e->field_index[#name]].offset;
  EXOGCM_FIELDS(EXOGCM_BIND)
#undef EXOGCM_BIND
}

void table_layout(exogcm_engine* e) {
  const int L = e->d.L, NTRU = e->d.T, NRSP = e->d.NRSP;
  int off = 0;
#define EXOGCM_TAB(name, count)                  \
  e->to.name = off;                              \
  e->tab_list.push_back({#name, (int)(count)});  \
  off += (int)(count);
  EXOGCM_PTABLES(EXOGCM_TAB)
#undef EXOGCM_TAB
  e->to.stride = (off + 31) / 32 * 32;
}

const FieldInfo& field(exogcm_engine* e, const char* name) {
  auto it = e->field_index.find(name ? name : "");
  if (it == e->field_index.end()) throw Error(EXOGCM_EINVAL, std::string("no state field ") + (name ? name : "(null)"));
  return e->fields[it->second];
}

void check_slot(exogcm_engine* e, int slot) {
  if (slot < 0 || slot >= e->d.S) throw Error(EXOGCM_EINVAL, "slot out of range");
}

// Copies between a host array [count][plane] and one slot's planes.
// The optimized path keeps Fourier planes m-major, [m][lat] (re, im) pairs,
// where the reference (and the plain path) keeps them [lat][m]. Host copies
// always see the reference's layout.
void fourier_to_m_major(const Dims& d, const float* src, float* dst, int planes) {
  for (int p = 0; p < planes; ++p) {
    const float* a = src + (size_t)p * d.NLAT * d.NFC;
    float* b = dst + (size_t)p * d.NLAT * d.NFC;
    for (int lat = 0; lat < d.NLAT; ++lat)
      for (int m = 0; m < d.NTP1; ++m) {
        b[2 * ((size_t)m * d.NLAT + lat)] = a[(size_t)lat * d.NFC + 2 * m];
        b[2 * ((size_t)m * d.NLAT + lat) + 1] = a[(size_t)lat * d.NFC + 2 * m + 1];
      }
  }
}

void fourier_from_m_major(const Dims& d, const float* src, float* dst, int planes) {
  for (int p = 0; p < planes; ++p) {
    const float* b = src + (size_t)p * d.NLAT * d.NFC;
    float* a = dst + (size_t)p * d.NLAT * d.NFC;
    for (int lat = 0; lat < d.NLAT; ++lat)
      for (int m = 0; m < d.NTP1; ++m) {
        a[(size_t)lat * d.NFC + 2 * m] = b[2 * ((size_t)m * d.NLAT + lat)];
        a[(size_t)lat * d.NFC + 2 * m + 1] = b[2 * ((size_t)m * d.NLAT + lat) + 1];
      }
  }
}

void copy_field(exogcm_engine* e, const FieldInfo& fi, int slot, void* host, bool to_device) {
  float* base = e->arena + fi.offset + (size_t)slot * fi.plane;
  const size_t pitch = fi.plane * e->d.S * sizeof(float);
  const size_t width = fi.plane * sizeof(float);
  const bool m_major = e->mode >= 1 && fi.shape == 'F';
  std::vector<float> staged;
  void* h = host;
  if (m_major) {
    staged.resize(fi.plane * fi.count);
    if (to_device) fourier_to_m_major(e->d, static_cast<const float*>(host), staged.data(), fi.count);
    h = staged.data();
  }
  if (to_device)
    check(cudaMemcpy2DAsync(base, pitch, h, width, width, fi.count, cudaMemcpyHostToDevice, e->stream),
          "write field");
  else
    check(cudaMemcpy2DAsync(h, width, base, pitch, width, fi.count, cudaMemcpyDeviceToHost, e->stream),
          "read field");
  check(cudaStreamSynchronize(e->stream), "field copy");
  if (m_major && !to_device) fourier_from_m_major(e->d, staged.data(), static_cast<float*>(host), fi.count);
}

void upload_shared(exogcm_engine* e, const SharedSetup& s) {
  const Dims& d = e->d;
  std::vector<float> buf;
  auto put = [&](const Vec& v) {
    size_t at = buf.size();
    for (double x : v) buf.push_back((float)x);
    while (buf.size() % 32) buf.push_back(0.f);
    return at;
  };
  const size_t fwd = put(s.fwd), inv = put(s.inv);
  size_t q[8];
  const char* names[8] = {"qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv"};
  for (int i = 0; i < 8; ++i) q[i] = put(s.q.at(names[i]));
  Vec zgw(d.NHOR), rcsq(d.NHOR), cola(d.NLAT), nindex(d.NRSP);
  for (int h = 0; h < d.NHOR; ++h) {
    const double sn = s.sines[h / d.NLON];
    zgw[h] = s.weights[h / d.NLON];
    rcsq[h] = 1 / (1 - sn * sn);
  }
  for (int l = 0; l < d.NLAT; ++l) cola[l] = std::sqrt(1 - s.sines[l] * s.sines[l]);
  std::vector<int> mm(d.NCSP), nn(d.NCSP);
  {
    int w = 0, r = 0;
    for (int m = 0; m <= d.T; ++m)
      for (int n = m; n <= d.T; ++n) {
        mm[w] = m;
        nn[w] = n;
        ++w;
        nindex[r] = nindex[r + 1] = n;
        r += 2;
      }
  }
  Vec tw(2 * (size_t)d.NLON);
  for (int j = 0; j < d.NLON; ++j) {
    tw[2 * j] = std::cos(2 * M_PI * j / d.NLON);
    tw[2 * j + 1] = std::sin(2 * M_PI * j / d.NLON);
  }
  const size_t izgw = put(zgw), ircsq = put(rcsq), isid = put(s.sines), icola = put(cola), inidx = put(nindex);
  const size_t itw = put(tw);
  // Transposed northern halves of qi, qj, qu, qv ([mode][pair]).
  size_t qt[4];
  std::vector<float> grid_tables[2];
  const char* tnames[4] = {"qi", "qj", "qu", "qv"};
  for (int i = 0; i < 4; ++i) {
    const Vec& q = s.q.at(tnames[i]);
    const int JH = d.NLAT / 2;
    Vec t((size_t)d.NCSP * JH);
    for (int j = 0; j < JH; ++j)
      for (int w = 0; w < d.NCSP; ++w) t[(size_t)w * JH + j] = q[(size_t)j * d.NCSP + w];
    qt[i] = put(t);
    if (i < 2 && e->mode == 1) grid_tables[i] = grid_table_layout(d, t);
  }
  // Tensor-core transforms (mode 2): hi/lo images of every table operand per m.
  std::vector<int> tc_at;
  const std::vector<float> img = e->mode == 2 ? tc_table_images(d, s.q, tc_at) : std::vector<float>();
  if (tc_at.empty()) tc_at.assign(1, 0);
  auto put_floats = [&](const std::vector<float>& v) {
    while (buf.size() % 32) buf.push_back(0.f);
    const size_t at = buf.size();
    buf.insert(buf.end(), v.begin(), v.end());
    return at;
  };
  const size_t itc = put_floats(img);
  const size_t igi = put_floats(grid_tables[0]), igj = put_floats(grid_tables[1]);
  check(cudaMalloc(&e->shared_buf, buf.size() * sizeof(float)), "shared tables");
  check(cudaMemcpy(e->shared_buf, buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice), "shared tables");
  check(cudaMalloc(&e->mode_buf, (2 * d.NCSP + tc_at.size()) * sizeof(int)), "mode tables");
  check(cudaMemcpy(e->mode_buf, mm.data(), d.NCSP * sizeof(int), cudaMemcpyHostToDevice), "mode tables");
  check(cudaMemcpy(e->mode_buf + d.NCSP, nn.data(), d.NCSP * sizeof(int), cudaMemcpyHostToDevice), "mode tables");
  check(cudaMemcpy(e->mode_buf + 2 * d.NCSP, tc_at.data(), tc_at.size() * sizeof(int), cudaMemcpyHostToDevice),
        "mode tables");
  float* b = e->shared_buf;
  e->sh.fwd = b + fwd;
  e->sh.inv = b + inv;
  e->sh.qi = b + q[0];
  e->sh.qj = b + q[1];
  e->sh.qc = b + q[2];
  e->sh.qe = b + q[3];
  e->sh.qm = b + q[4];
  e->sh.qq = b + q[5];
  e->sh.qu = b + q[6];
  e->sh.qv = b + q[7];
  e->sh.zgw = b + izgw;
  check(cudaMalloc(&e->wlat64, d.NLAT * sizeof(double)), "FP64 weights");
  check(cudaMemcpy(e->wlat64, s.weights.data(), d.NLAT * sizeof(double), cudaMemcpyHostToDevice), "FP64 weights");
  e->sh.wlat = e->wlat64;
  e->sh.rcsq = b + ircsq;
  e->sh.sid = b + isid;
  e->sh.cola = b + icola;
  e->sh.nindex = b + inidx;
  e->sh.tw = b + itw;
  e->sh.qiT = b + qt[0];
  e->sh.qjT = b + qt[1];
  e->sh.quT = b + qt[2];
  e->sh.qvT = b + qt[3];
  e->sh.qiG = b + igi;
  e->sh.qjG = b + igj;
  e->sh.tc_img = b + itc;
  e->sh.tc_at = e->mode_buf + 2 * d.NCSP;
  e->sh.mode_m = e->mode_buf;
  e->sh.mode_n = e->mode_buf + d.NCSP;
  e->shared_ready = true;
}

// ---------------------------------------------------------------- the step
void stage_gridpointa(const Model& m, cudaStream_t st) {
  const Dims& d = m.d;
  const FieldPtrs& F = m.f;
  const int LP = d.L * d.S, SP = d.S;
  tr_dv2uv(m, F.sd, F.sz, F.fgu, F.fgv, LP, 1.63299310207f, st);
  tr_legendre_inverse(m, F.sp, F.fgp, SP, m.sh.qi, st);
  tr_dlambda(m, F.fgp, F.fgpmt, SP, st);
  tr_fourier_inverse(m, F.fgu, F.gu, LP, st);
  tr_fourier_inverse(m, F.fgv, F.gv, LP, st);
  tr_sp2gp(m, F.st, F.fgt, F.gt, LP, m.sh.qi, st);
  tr_sp2gp(m, F.sd, F.fgd, F.gd, LP, m.sh.qi, st);
  tr_sp2gp(m, F.sz, F.fgz, F.gz, LP, m.sh.qi, st);
  tr_sp2gp(m, F.sp, F.fgpj, F.gpj, SP, m.sh.qj, st);
  tr_fourier_inverse(m, F.fgpmt, F.gpmt, SP, st);
  tr_fourier_inverse(m, F.fgp, F.gp, SP, st);
  tr_sp2gp(m, F.sq, F.fgq, F.gq, LP, m.sh.qi, st);
  dyn_calcgp(m, st);
  tr_fourier_forward(m, F.gtn, F.fgtn, LP, st);
  tr_fourier_forward(m, F.gqn, F.fgqn, LP, st);
  tr_fourier_forward(m, F.gut, F.fgut, LP, st);
  tr_fourier_forward(m, F.gvt, F.fgvt, LP, st);
  tr_fourier_forward(m, F.guz, F.fguz, LP, st);
  tr_fourier_forward(m, F.gvz, F.fgvz, LP, st);
  tr_fourier_forward(m, F.gke, F.fgke, LP, st);
  tr_fourier_forward(m, F.gvpp, F.fgvpp, SP, st);
  tr_fourier_forward(m, F.guq, F.fguq, LP, st);
  tr_fourier_forward(m, F.gvq, F.fgvq, LP, st);
  tr_legendre_forward(m, F.fgvpp, F.spt, SP, m.sh.qc, st);
  tr_uv2dv(m, F.fgvz, F.fguz, F.fgke, F.sdt, F.szt, LP, st);
  tr_qtend(m, F.fgut, F.fgvt, F.fgtn, F.stt, LP, st);
  tr_qtend(m, F.fguq, F.fgvq, F.fgqn, F.sqt, LP, st);
}

void stage_physics_in(const Model& m, cudaStream_t st) {
  const Dims& d = m.d;
  const FieldPtrs& F = m.f;
  const int LP = d.L * d.S, SP = d.S;
  tr_dv2uv(m, F.sd, F.sz, F.fgu, F.fgv, LP, 1.63299310207f, st);
  tr_fourier_inverse(m, F.fgu, F.gu, LP, st);
  tr_fourier_inverse(m, F.fgv, F.gv, LP, st);
  tr_sp2gp(m, F.st, F.fgt, F.gt, LP, m.sh.qi, st);
  tr_sp2gp(m, F.sp, F.fgp, F.gp, SP, m.sh.qi, st);
  tr_sp2gp(m, F.sq, F.fgq, F.gq, LP, m.sh.qi, st);
  dyn_physics_in(m, st);
}

void stage_precipitation(const Model& m, cudaStream_t st) {
  const int LP = m.d.L * m.d.S;
  tr_sp2gp(m, m.f.sqt, m.f.fdqt, m.f.dqt, LP, m.sh.qi, st);
  phy_precipitation_columns(m, st);
}

void stage_physics_out(const Model& m, cudaStream_t st) {
  const int LP = m.d.L * m.d.S;
  const FieldPtrs& F = m.f;
  dyn_physics_out(m, st);
  tr_fourier_forward(m, F.gtdt, F.fgtdt, LP, st);
  tr_fourier_forward(m, F.gudt, F.fgudt, LP, st);
  tr_fourier_forward(m, F.gvdt, F.fgvdt, LP, st);
  tr_fourier_forward(m, F.gqdt, F.fgqdt, LP, st);
  tr_legendre_forward(m, F.fgtdt, F.stt, LP, m.sh.qc, st);
  tr_legendre_forward(m, F.fgqdt, F.sqt, LP, m.sh.qc, st);
  tr_uv2dv(m, F.fgudt, F.fgvdt, nullptr, F.sdt, F.szt, LP, st);
}

void stage_spectrald(const Model& m, cudaStream_t st) {
  const int LP = m.d.L * m.d.S;
  const FieldPtrs& F = m.f;
  const float plavor = 1.63299310207f;
  dyn_spectrald_diffusion(m, st);
  tr_dv2uv(m, F.sdp, F.szp, F.fzu, F.fzv, LP, plavor, st);
  tr_fourier_inverse(m, F.fzu, F.zu, LP, st);
  tr_fourier_inverse(m, F.fzv, F.zv, LP, st);
  tr_dv2uv(m, F.zdsdp1, F.zdszp1, F.fzdu, F.fzdv, LP, 0.f, st);
  tr_fourier_inverse(m, F.fzdu, F.zdu, LP, st);
  tr_fourier_inverse(m, F.fzdv, F.zdv, LP, st);
  dyn_mkdheat(m, 1, st);
  tr_fourier_forward(m, F.zdtdt, F.fzdtdt, LP, st);
  tr_legendre_forward(m, F.fzdtdt, F.zstt1, LP, m.sh.qc, st);
  tr_dv2uv(m, F.zdsdp2, F.zdszp2, F.fzdu, F.fzdv, LP, 0.f, st);
  tr_fourier_inverse(m, F.fzdu, F.zdu, LP, st);
  tr_fourier_inverse(m, F.fzdv, F.zdv, LP, st);
  dyn_mkdheat(m, 2, st);
  tr_fourier_forward(m, F.zdekin, F.fzdekin, LP, st);
  tr_legendre_forward(m, F.fzdekin, F.zsdef, LP, m.sh.qc, st);
  dyn_mean_mode(m, F.zsdef, st);
  tr_sp2gp(m, F.zsdef, F.fzdekin, F.zdekin, LP, m.sh.qi, st);
  dyn_mkdheat(m, 3, st);
  tr_fourier_forward(m, F.zdtdt, F.fzdtdt, LP, st);
  tr_legendre_forward(m, F.fzdtdt, F.zstt2, LP, m.sh.qc, st);
  dyn_spectrald_update(m, st);
}

void run_stage(const Model& m, const std::string& s, cudaStream_t st) {
  if (s == "gridpointa") stage_gridpointa(m, st);
  else if (s == "spectrala") dyn_spectrala(m, st);
  else if (s == "physics_in") stage_physics_in(m, st);
  else if (s == "fixer") phy_fixer(m, st);
  else if (s == "surface_flux") phy_surface_flux(m, st);
  else if (s == "radiation") phy_radiation(m, st);
  else if (s == "precipitation") stage_precipitation(m, st);
  else if (s == "surface") phy_surface(m, st);
  else if (s == "carbon") phy_carbon(m, st);
  else if (s == "storm") phy_storm(m, st);
  else if (s == "physics_out") stage_physics_out(m, st);
  else if (s == "spectrald") stage_spectrald(m, st);
  else if (s == "pack") phy_pack(m, st);
  else throw Error(EXOGCM_EINVAL, "unknown stage " + s);
}

// master's step order (stepper/index.ts:148-161).
// The physics between the per-planet reductions runs as column kernels,
// fused where that measured faster (physics.cu); exogcm_run_stage runs the
// same routines stage by stage, unfused.
void full_step(const Model& m, cudaStream_t st) {
  stage_gridpointa(m, st);
  dyn_spectrala(m, st);
  stage_physics_in(m, st);
  phy_fused_through_radiation(m, st);
  tr_sp2gp(m, m.f.sqt, m.f.fdqt, m.f.dqt, m.d.L * m.d.S, m.sh.qi, st);  // precipitation's dqt
  phy_fused_precipitation_to_carbon(m, st);
  phy_storm(m, st);
  stage_physics_out(m, st);
  stage_spectrald(m, st);
  phy_pack(m, st);
  phy_budget(m, m.d.P, st);
}

// The host values of one slot's next step; advances the slot's counters when
// `advance` (stepper/index.ts:281-334 with the start-up schedule of
// runner/webgpu/gcm.worker.ts:137-153: start-up steps at the start step's
// date with halved timesteps, no filter and no icestep).
StepParams next_params(Slot& s, int publish_every, bool advance) {
  StepParams p{};
  if (!s.active) return p;
  if (s.stop >= 0 && s.startup_left == 0 && s.step >= s.stop) return p;  // finished: kernels skip the slot
  const int phase = s.startup_left;
  p.phase = phase;
  p.active = 1;
  p.delt = (float)s.delt[phase];
  p.delt2 = (float)(s.delt[phase] + s.delt[phase]);
  p.deltsec = (float)s.deltsec[phase];
  p.deltsec2 = (float)(s.deltsec[phase] + s.deltsec[phase]);
  p.filter = phase == 0 ? 1.f : 0.f;
  p.coupled = phase == 0 ? 1.f : 0.f;
  const StepValues v = step_values(s.cal, s.step, s.carbon_step);
  for (int i = 0; i < 5; ++i) p.rad[i] = (float)v.rad[i];
  for (int i = 0; i < 7; ++i) p.surf[i] = (float)v.surf[i];
  p.carbon = (float)v.carbon;
  p.snap[0] = (float)s.step;
  p.snap[1] = (float)s.cal.output_window_steps;
  const bool publish = phase == 0 && publish_every > 0 && s.step % publish_every == 0;
  p.snap[2] = publish ? 1.f : 0.f;
  if (advance) {
    s.carbon_step = v.next_carbon_step;
    if (publish) s.published = s.step;
    if (phase > 0)
      s.startup_left--;
    else
      s.step++;
  }
  return p;
}

cudaGraphExec_t batch_graph(exogcm_engine* e, int K) {
  auto it = e->graphs.find(K);
  if (it != e->graphs.end()) return it->second;
  cudaGraph_t graph;
  check(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed), "capture");
  for (int k = 0; k < K; ++k) full_step(e->model(k), e->stream);
  check(cudaStreamEndCapture(e->stream, &graph), "capture end");
  cudaGraphExec_t exec;
  check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
  e->graph_templates[K] = graph;
  e->graphs[K] = exec;
  return exec;
}

// The slot's table block [to.stride] in float, into `block`.
void fill_slot_tables(exogcm_engine* e, const PlanetSetup& ps, float* block) {
  std::fill(block, block + e->to.stride, 0.f);
  int off = 0;
  for (auto& t : e->tab_list) {
    auto it = ps.tables.find(t.first);
    if (it == ps.tables.end()) throw Error(EXOGCM_EINVAL, "set-up lacks table " + t.first);
    const Vec& v = it->second;
    for (int i = 0; i < t.second && i < (int)v.size(); ++i) block[off + i] = (float)v[i];
    off += t.second;
  }
}

// Queues the slot's table block (filled by fill_slot_tables into pinned
// `block`) and its constants on the engine's stream; the caller synchronises.
void upload_slot_tables(exogcm_engine* e, int slot, const PlanetSetup& ps, float* block) {
  check(cudaMemcpyAsync(e->tabs + (size_t)slot * e->to.stride, block, e->to.stride * sizeof(float),
                        cudaMemcpyHostToDevice, e->stream),
        "slot tables");
  PlanetConst pc{};
#define EXOGCM_SET_CONST(n)                                                    \
  {                                                                            \
    auto c = ps.consts.find(#n);                                               \
    if (c == ps.consts.end()) throw Error(EXOGCM_EINVAL, "set-up lacks " #n);  \
    pc.n = (float)c->second;                                                   \
  }
  EXOGCM_CONSTS(EXOGCM_SET_CONST)
#undef EXOGCM_SET_CONST
  // The constants ride in the staging area after the table block.
  PlanetConst* staged = reinterpret_cast<PlanetConst*>(block + e->to.stride);
  *staged = pc;
  check(cudaMemcpyAsync(e->pc + slot, staged, sizeof(pc), cudaMemcpyHostToDevice, e->stream), "slot constants");
}

void zero_slot(exogcm_engine* e, int slot) {
  for (auto& fi : e->fields) {
    float* base = e->arena + fi.offset + (size_t)slot * fi.plane;
    check(cudaMemset2DAsync(base, fi.plane * e->d.S * sizeof(float), 0, fi.plane * sizeof(float), fi.count,
                            e->stream),
          "zero slot");
  }
}

template <typename F>
int guard(F&& f) {
  try {
    f();
    return EXOGCM_OK;
  } catch (const Error& err) {
    g_error = err.what();
    return err.code;
  } catch (const std::invalid_argument& err) {
    g_error = err.what();
    return EXOGCM_EINVAL;
  } catch (const std::bad_alloc&) {
    g_error = "host allocation failed";
    return EXOGCM_ENOMEM;
  } catch (const std::exception& err) {
    g_error = err.what();
    return EXOGCM_EDEVICE;
  }
}

// ---------------------------------------------------------------- checkpoint
const char kMagic[] = "GCM-WEBGPU-STATE\n";

std::string header_json(exogcm_engine* e, long step, int carbon_step) {
  std::string s = "{\"fields\":[";
  for (size_t i = 0; i < e->fields.size(); ++i) {
    const FieldInfo& fi = e->fields[i];
    if (i) s += ",";
    s += "[\"" + fi.name + "\"," + std::to_string(fi.plane * fi.count) + "]";
  }
  s += "],\"step\":" + std::to_string(step) + ",\"carbonStep\":" + std::to_string(carbon_step) + "}";
  return s;
}

long json_number(const std::string& s, const char* key) {
  const std::string k = std::string("\"") + key + "\":";
  const size_t at = s.find(k);
  if (at == std::string::npos) throw Error(EXOGCM_ELAYOUT, std::string("checkpoint header lacks ") + key);
  return std::stol(s.substr(at + k.size()));
}

}  // namespace

// ================================================================= C ABI
namespace {

// Scratch of the autotuner: events for the timed launches and, when the
// batch's state is larger than L2, a buffer whose overwrite evicts L2.
struct TuneScratch {
  static constexpr int kReps = 5;
  cudaEvent_t ev[2 * kReps] = {};
  void* flush = nullptr;
  size_t flush_bytes = 0;
  TuneScratch(size_t state_bytes) {
    for (auto& v : ev) check(cudaEventCreate(&v), "event");
    int dev = 0, l2 = 0;
    check(cudaGetDevice(&dev), "device");
    check(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev), "L2 size");
    if (state_bytes > (size_t)l2) {
      flush_bytes = 2 * (size_t)l2;
      check(cudaMalloc(&flush, flush_bytes), "autotune flush buffer");
    }
  }
  ~TuneScratch() {
    for (auto& v : ev)
      if (v) cudaEventDestroy(v);
    if (flush) cudaFree(flush);
  }
};

// Times each transform kernel of the optimized path over the launch shapes
// it supports and keeps the fastest: full-level launches over every slot,
// one warm-up and five timed launches per shape (CUDA events on the
// engine's stream around each launch). When the batch's state exceeds L2,
// as in a step, L2 is overwritten before each timed launch, so that shapes
// are judged on HBM-resident inputs. A burst of launches first brings the
// clocks up, so that the order of the candidates does not bias the pick.
// Runs once, at the first configure, before any slot holds state; the
// shapes change how work is split, not any result.
void autotune(exogcm_engine* e) {
  const Dims& d = e->d;
  const int LP = d.L * d.S, JH = d.NLAT / 2;
  const FieldPtrs& F = e->fp;
  Tuning& t = e->tune;
  TuneScratch x(e->arena_floats * sizeof(float));
  auto time = [&](const std::function<void(const Model&)>& launch) {
    const Model m = e->model(0);
    launch(m);
    for (int r = 0; r < TuneScratch::kReps; ++r) {
      if (x.flush) check(cudaMemsetAsync(x.flush, r, x.flush_bytes, e->stream), "flush");
      check(cudaEventRecord(x.ev[2 * r], e->stream), "event");
      launch(m);
      check(cudaEventRecord(x.ev[2 * r + 1], e->stream), "event");
    }
    check(cudaStreamSynchronize(e->stream), "autotune");
    float total = 0.f;
    for (int r = 0; r < TuneScratch::kReps; ++r) {
      float ms = 0.f;
      check(cudaEventElapsedTime(&ms, x.ev[2 * r], x.ev[2 * r + 1]), "event time");
      total += ms;
    }
    return total;
  };
  {
    const Model m = e->model(0);
    auto now = [] { return std::chrono::steady_clock::now(); };
    const auto start = now();
    while (now() - start < std::chrono::milliseconds(50)) {
      for (int r = 0; r < 20; ++r) tr_fourier_inverse(m, F.fgu, F.gu, LP, e->stream);
      check(cudaStreamSynchronize(e->stream), "autotune warm-up");
    }
  }
  {
    float best = 1e30f;
    int pick = t.fft_rows;
    for (int rows : {8, 16, 32, 48, 64, 96}) {
      if (!fft_rows_supported(d, rows)) continue;
      t.fft_rows = rows;
      const float ms = time([&](const Model& m) {
        tr_fourier_inverse(m, F.fgu, F.gu, LP, e->stream);
        tr_fourier_forward(m, F.gtn, F.fgtn, LP, e->stream);
      });
      if (ms < best) best = ms, pick = rows;
    }
    t.fft_rows = pick;
    // per direction: one block per chunk, or persistent blocks looping over chunks
    for (int dir = 0; dir < 2; ++dir) {
      float ms[2];
      for (int form = 0; form < 2; ++form) {
        t.fft_persistent[dir] = form;
        ms[form] = time([&](const Model& m) {
          if (dir == 0)
            tr_fourier_forward(m, F.gtn, F.fgtn, LP, e->stream);
          else
            tr_fourier_inverse(m, F.fgu, F.gu, LP, e->stream);
        });
      }
      t.fft_persistent[dir] = ms[1] < ms[0] ? 1 : 0;
    }
  }
  for (int k = 0; k < 2; ++k) {
    float best = 1e30f;
    int pg = t.inv_group[k], pt = t.inv_tile[k];
    for (int group : {1, 2, 4})
      for (int tile : {8, 16, 32}) {
        if (JH * tile / 2 > 1024 || leg_inverse_smem(d, k, group, tile) > kLegSmemLimit) continue;
        t.inv_group[k] = group;
        t.inv_tile[k] = tile;
        const float ms = time([&](const Model& m) {
          if (k == 0)
            tr_legendre_inverse(m, F.st, F.fgt, LP, m.sh.qi, e->stream);
          else
            tr_dv2uv(m, F.sd, F.sz, F.fgu, F.fgv, LP, 0.f, e->stream);
        });
        if (ms < best) best = ms, pg = group, pt = tile;
      }
    t.inv_group[k] = pg;
    t.inv_tile[k] = pt;
  }
  for (int k = 0; k < 4; ++k) {
    float best = 1e30f;
    int pick = t.fwd_tile[k], pick_buffers = t.fwd_buffers[k];
    for (int shape = 0; shape < 4; ++shape) {
      const int tile = shape & 1 ? 16 : 8, buffers = shape & 2 ? 1 : 2;
      if (leg_forward_smem(d, k, tile) > kLegSmemLimit) continue;
      t.fwd_tile[k] = tile;
      t.fwd_buffers[k] = buffers;
      const float ms = time([&](const Model& m) {
        if (k == 0)
          tr_legendre_forward(m, F.fgtdt, F.zstt1, LP, m.sh.qc, e->stream);
        else if (k == 1)
          tr_uv2dv(m, F.fgudt, F.fgvdt, nullptr, F.sdt, F.szt, LP, e->stream);
        else if (k == 2)
          tr_uv2dv(m, F.fgvz, F.fguz, F.fgke, F.zdsdp1, F.zdszp1, LP, e->stream);
        else
          tr_qtend(m, F.fgut, F.fgvt, F.fgtn, F.zstt2, LP, e->stream);
      });
      if (ms < best) best = ms, pick = tile, pick_buffers = buffers;
    }
    t.fwd_tile[k] = pick;
    t.fwd_buffers[k] = pick_buffers;
  }
  {
    float best = 1e30f;
    int pick = t.sp2gp_planes;
    for (int pp : {2, 4}) {
      if (grid_sp2gp_smem(d, pp) > kLegSmemLimit) continue;
      t.sp2gp_planes = pp;
      const float ms = time([&](const Model& m) { tr_sp2gp(m, F.st, F.fgt, F.gt, LP, m.sh.qi, e->stream); });
      if (ms < best) best = ms, pick = pp;
    }
    t.sp2gp_planes = pick;
  }
}

// Group graphs (exogcm_group_step): one instantiated graph per list of
// (engine, steps), whose nodes are the engines' K-step batch graphs as
// child graphs. Engines being destroyed drop the group graphs they are in.
std::mutex g_group_mutex;
std::map<std::vector<std::pair<const exogcm_engine*, int>>, cudaGraphExec_t> g_group_graphs;

void drop_group_graphs(const exogcm_engine* e) {
  std::lock_guard<std::mutex> lock(g_group_mutex);
  for (auto it = g_group_graphs.begin(); it != g_group_graphs.end();) {
    bool has = false;
    for (const auto& m : it->first) has = has || m.first == e;
    if (has) {
      cudaGraphExecDestroy(it->second);
      it = g_group_graphs.erase(it);
    } else {
      ++it;
    }
  }
}

// Destroys the engine's captured batch graphs (and the group graphs holding
// them) so the next batch captures them again with the current Model.
void drop_graphs(exogcm_engine* e) {
  drop_group_graphs(e);
  for (auto& g : e->graphs) cudaGraphExecDestroy(g.second);
  for (auto& g : e->graph_templates) cudaGraphDestroy(g.second);
  e->graphs.clear();
  e->graph_templates.clear();
}

// Retires the oldest batch in flight once its stream has passed it:
// blocking waits for it, otherwise a batch not yet done is left alone and
// false returned. Reports a fault word a tensor-core transform set.
bool retire_oldest(exogcm_engine* e, bool blocking) {
  if (e->pending.empty()) return false;
  exogcm_engine::Batch& B = e->batch[e->pending.front()];
  if (blocking) {
    check(cudaEventSynchronize(B.done), "step");
  } else {
    const cudaError_t q = cudaEventQuery(B.done);
    if (q == cudaErrorNotReady) return false;
    check(q, "step");
  }
  e->pending.pop_front();
  check(cudaEventElapsedTime(&e->last_ms, B.start, B.end), "event time");
  if (*B.fault_host) {
    *B.fault_host = 0;
    throw Error(EXOGCM_EDEVICE, "a tensor-core transform gave up waiting for its MMAs; this step's results are invalid");
  }
  return true;
}

// Every call other than exogcm_step_async/poll/wait first retires the batches
// in flight: they read and write host slot state and device memory the
// batches use, through copies that do not order with the engine's stream.
void retire_all(exogcm_engine* e) {
  while (!e->pending.empty()) retire_oldest(e, true);
}

}  // namespace

extern "C" {

int exogcm_last_error(char* buffer, size_t size) {
  if (!buffer || size == 0) return EXOGCM_EINVAL;
  std::snprintf(buffer, size, "%s", g_error.c_str());
  return EXOGCM_OK;
}

int exogcm_create(int truncation, int levels, int slots, int mode, exogcm_engine** out) {
  return guard([&] {
    if (!out) throw Error(EXOGCM_EINVAL, "null engine pointer");
    *out = nullptr;
    if (truncation != 21 && truncation != 42 && truncation != 63)
      throw Error(EXOGCM_EINVAL, "truncation must be 21, 42 or 63");
    if (levels != 5 && levels != 10) throw Error(EXOGCM_EINVAL, "levels must be 5 or 10");
    if (slots < 1 || slots > 4096) throw Error(EXOGCM_EINVAL, "slots must be 1..4096");
    if (mode < 0 || mode > 2)
      throw Error(EXOGCM_EINVAL, "mode must be 0 (plain FP32), 1 (optimized) or 2 (optimized, tensor-core sp2fc)");
    auto e = std::make_unique<exogcm_engine>();
    e->d = make_dims(truncation, levels, slots);
    e->mode = mode;
    e->tune = default_tuning(e->d);
    check(cudaGetDevice(&e->device), "device");
    layout(e.get());
    table_layout(e.get());
    if (cudaMalloc(&e->arena, e->arena_floats * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(EXOGCM_ENOMEM, "device memory for the state arena (" +
                                     std::to_string(e->arena_floats * 4 / (1 << 20)) + " MiB) not available");
    }
    check(cudaMemset(e->arena, 0, e->arena_floats * sizeof(float)), "arena clear");
    bind_fields(e.get());
    check(cudaMalloc(&e->tabs, (size_t)slots * e->to.stride * sizeof(float)), "slot tables");
    check(cudaMemset(e->tabs, 0, (size_t)slots * e->to.stride * sizeof(float)), "slot tables");
    check(cudaMalloc(&e->pc, slots * sizeof(PlanetConst)), "constants");
    check(cudaMemset(e->pc, 0, slots * sizeof(PlanetConst)), "constants");
    check(cudaMalloc(&e->params, (size_t)kMaxBatch * slots * sizeof(StepParams)), "params");
    check(cudaMemset(e->params, 0, (size_t)kMaxBatch * slots * sizeof(StepParams)), "params");
    check(cudaMallocHost(&e->hparams, (size_t)(1 + kInFlight) * kMaxBatch * slots * sizeof(StepParams)),
          "pinned params");
    for (auto& b : e->batch) {
      check(cudaEventCreate(&b.start), "event");
      check(cudaEventCreate(&b.end), "event");
      check(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming), "event");
      check(cudaMallocHost(&b.fault_host, sizeof(int)), "pinned fault word");
      *b.fault_host = 0;
    }
    check(cudaMalloc(&e->budget, (size_t)slots * kBudgetStride * sizeof(double)), "budgets");
    check(cudaMemset(e->budget, 0, (size_t)slots * kBudgetStride * sizeof(double)), "budgets");
    check(cudaMalloc(&e->sums, (size_t)slots * 4 * sizeof(double)), "sums");
    check(cudaMemset(e->sums, 0, (size_t)slots * 4 * sizeof(double)), "sums");
    check(cudaMalloc(&e->flags, slots * sizeof(int)), "flags");
    check(cudaMemset(e->flags, 0, slots * sizeof(int)), "flags");
    check(cudaMalloc(&e->fault, sizeof(int)), "fault word");
    check(cudaMemset(e->fault, 0, sizeof(int)), "fault word");
    check(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "stream");
    check(cudaEventCreate(&e->ev0), "event");
    check(cudaEventCreate(&e->ev1), "event");
    tr_init();
    e->slots.resize(slots);
    *out = e.release();
  });
}

void exogcm_destroy(exogcm_engine* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->copy_stream) {
    cudaStreamSynchronize(e->copy_stream);
    cudaStreamDestroy(e->copy_stream);
  }
  if (e->snap_staged) cudaEventDestroy(e->snap_staged);
  if (e->snap_copied) cudaEventDestroy(e->snap_copied);
  cudaFree(e->snap_stage);
  drop_group_graphs(e);
  for (auto& g : e->graphs) cudaGraphExecDestroy(g.second);
  for (auto& g : e->graph_templates) cudaGraphDestroy(g.second);
  cudaFree(e->arena);
  cudaFree(e->shared_buf);
  cudaFree(e->mode_buf);
  cudaFree(e->tabs);
  cudaFree(e->pc);
  cudaFree(e->params);
  cudaFreeHost(e->hparams);
  cudaFree(e->sums);
  cudaFree(e->budget);
  cudaFree(e->avg);
  cudaFree(e->wlat64);
  cudaFree(e->flags);
  cudaFree(e->fault);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  for (auto& b : e->batch) {
    if (b.start) cudaEventDestroy(b.start);
    if (b.end) cudaEventDestroy(b.end);
    if (b.done) cudaEventDestroy(b.done);
    cudaFreeHost(b.fault_host);
  }
  if (e->stream) cudaStreamDestroy(e->stream);
  e->setup_device.reset();
  cudaFreeHost(e->upload_stage);
  delete e;
}

namespace {
// Process-wide caches for the set-up of a new engine: the shared FP64 tables
// of a resolution and filter setting, and the autotuned launch shapes of an
// engine shape on a device (the shapes change no result). An elastic server
// creating blocks of a resolution it served before pays neither again.
std::mutex g_setup_cache_mutex;
std::map<std::tuple<int, int, int, int>, SharedSetup> g_shared_cache;
std::map<std::tuple<int, int, int, int, int>, Tuning> g_tuning_cache;

SharedSetup cached_shared(int T, int kind, int gp, int sp, SetupDevice* dev) {
  const auto key = std::make_tuple(T, kind, gp, sp);
  {
    std::lock_guard<std::mutex> lock(g_setup_cache_mutex);
    auto it = g_shared_cache.find(key);
    if (it != g_shared_cache.end()) return it->second;
  }
  SharedSetup sh = build_shared(T, kind, gp, sp, dev);
  std::lock_guard<std::mutex> lock(g_setup_cache_mutex);
  return g_shared_cache.emplace(key, std::move(sh)).first->second;
}

void cached_autotune(exogcm_engine* e) {
  const auto key = std::make_tuple(e->device, e->d.T, e->d.L, e->d.S, e->mode);
  {
    std::lock_guard<std::mutex> lock(g_setup_cache_mutex);
    auto it = g_tuning_cache.find(key);
    if (it != g_tuning_cache.end()) {
      e->tune = it->second;
      return;
    }
  }
  autotune(e);
  std::lock_guard<std::mutex> lock(g_setup_cache_mutex);
  g_tuning_cache[key] = e->tune;
}
}  // namespace

int exogcm_configure(exogcm_engine* e, int slot, const exogcm_planet* planet, const exogcm_boundary* boundary) {
  return guard([&] {
    if (!e || !planet || !boundary) throw Error(EXOGCM_EINVAL, "null argument");
    check_slot(e, slot);
    if (planet->truncation != e->d.T || planet->levels != e->d.L)
      throw Error(EXOGCM_EINVAL, "planet resolution differs from the engine's");
    SetupDevice* dev = nullptr;
    if (e->setup_on_device) {
      if (!e->setup_device) e->setup_device = make_setup_device();
      dev = e->setup_device.get();
    }
    if (!e->shared_ready) {
      retire_all(e);
      e->shared_setup = cached_shared(e->d.T, planet->filter_kind, planet->filter_gp, planet->filter_sp, dev);
      upload_shared(e, e->shared_setup);
      if (e->mode >= 1) cached_autotune(e);
      e->filter_kind = planet->filter_kind;
      e->filter_gp = planet->filter_gp;
      e->filter_sp = planet->filter_sp;
    } else if (planet->filter_kind != e->filter_kind || planet->filter_gp != e->filter_gp ||
               planet->filter_sp != e->filter_sp) {
      throw Error(EXOGCM_EINVAL, "planets of one engine share the physics filter setting");
    }
    // The host set-up runs while batches already submitted step on the
    // device; the slot's upload waits for them.
    PlanetSetup ps = build_planet(*planet, *boundary, e->shared_setup, dev);
    // Every field and the slot's tables go through one pinned staging area,
    // converted to float (Fourier fields to the m-major layout) before the
    // in-flight batches are retired, then copied with one synchronisation.
    size_t need = e->to.stride + (sizeof(PlanetConst) + sizeof(float) - 1) / sizeof(float);
    for (auto& kv : ps.state) {
      const FieldInfo& fi = field(e, kv.first.c_str());
      if (kv.second.size() != fi.plane * fi.count)
        throw Error(EXOGCM_EINVAL, "set-up field " + kv.first + " has the wrong size");
      need += fi.plane * fi.count;
    }
    if (need > e->upload_stage_floats) {
      retire_all(e);
      check(cudaStreamSynchronize(e->stream), "staging");
      cudaFreeHost(e->upload_stage);
      e->upload_stage = nullptr;
      e->upload_stage_floats = 0;
      check(cudaMallocHost(&e->upload_stage, need * sizeof(float)), "pinned staging");
      e->upload_stage_floats = need;
    }
    float* stage = e->upload_stage;
    std::vector<std::pair<const FieldInfo*, float*>> staged;
    std::vector<float> plain;
    for (auto& kv : ps.state) {
      const FieldInfo& fi = field(e, kv.first.c_str());
      const size_t n = fi.plane * fi.count;
      if (e->mode >= 1 && fi.shape == 'F') {
        plain.assign(kv.second.begin(), kv.second.end());
        fourier_to_m_major(e->d, plain.data(), stage, fi.count);
      } else {
        for (size_t i = 0; i < n; ++i) stage[i] = (float)kv.second[i];
      }
      staged.push_back({&fi, stage});
      stage += n;
    }
    fill_slot_tables(e, ps, stage);
    retire_all(e);
    zero_slot(e, slot);
    for (auto& f : staged) {
      const FieldInfo& fi = *f.first;
      float* base = e->arena + fi.offset + (size_t)slot * fi.plane;
      check(cudaMemcpy2DAsync(base, fi.plane * e->d.S * sizeof(float), f.second, fi.plane * sizeof(float),
                              fi.plane * sizeof(float), fi.count, cudaMemcpyHostToDevice, e->stream),
            "write field");
    }
    upload_slot_tables(e, slot, ps, stage);
    check(cudaMemsetAsync(e->flags + slot, 0, sizeof(int), e->stream), "flags");
    check(cudaMemsetAsync(e->budget + (size_t)slot * kBudgetStride, 0, kBudgetStride * sizeof(double), e->stream),
          "budgets");
    if (e->avg)
      check(cudaMemset2DAsync(e->avg + (size_t)slot * e->d.NHOR, e->d.S * e->d.NHOR * sizeof(double), 0,
                              e->d.NHOR * sizeof(double), e->d.P, e->stream),
            "averages");
    bool storm_before = false;
    for (const Slot& o : e->slots) storm_before = storm_before || o.storm;
    Slot& s = e->slots[slot];
    s = Slot{};
    s.active = true;
    s.storm = ps.consts.at("NSTORMDIAG") > 0;
    s.step = ps.start_step;
    s.carbon_step = 0;
    s.startup_left = ps.nkits;
    for (int k = 0; k < 4; ++k) {
      s.deltsec[k] = ps.deltsec[k];
      s.delt[k] = ps.delt[k];
    }
    s.cal = ps.cal;
    bool storm_after = false;
    for (const Slot& o : e->slots) storm_after = storm_after || o.storm;
    // The batch graphs hold whether the storm diagnostics launch.
    if (storm_after != storm_before) drop_graphs(e);
    check(cudaStreamSynchronize(e->stream), "configure");
  });
}

namespace {
int setup_preview(const exogcm_planet* planet, const exogcm_boundary* boundary, const char* name, double* values,
                  size_t* count, bool on_device) {
  return guard([&] {
    if (!planet || !boundary || !name || !count) throw Error(EXOGCM_EINVAL, "null argument");
    std::unique_ptr<SetupDevice> dev;
    if (on_device) dev = make_setup_device();
    const SharedSetup sh =
        build_shared(planet->truncation, planet->filter_kind, planet->filter_gp, planet->filter_sp, dev.get());
    const PlanetSetup ps = build_planet(*planet, *boundary, sh, dev.get());
    const std::string n(name);
    const size_t colon = n.find(':');
    if (colon == std::string::npos) throw Error(EXOGCM_EINVAL, "name needs a kind: prefix");
    const std::string kind = n.substr(0, colon), key = n.substr(colon + 1);
    Vec out;
    if (kind == "state") {
      auto it = ps.state.find(key);
      if (it == ps.state.end()) throw Error(EXOGCM_EINVAL, "no initial field " + key);
      out = it->second;
    } else if (kind == "table") {
      auto it = ps.tables.find(key);
      if (it == ps.tables.end()) throw Error(EXOGCM_EINVAL, "no table " + key);
      out = it->second;
    } else if (kind == "const") {
      auto it = ps.consts.find(key);
      if (it == ps.consts.end()) throw Error(EXOGCM_EINVAL, "no constant " + key);
      out = {it->second};
    } else if (kind == "shared") {
      if (key == "fwd") out = sh.fwd;
      else if (key == "inv") out = sh.inv;
      else if (key == "sines") out = sh.sines;
      else if (key == "weights") out = sh.weights;
      else {
        auto it = sh.q.find(key);
        if (it == sh.q.end()) throw Error(EXOGCM_EINVAL, "no shared table " + key);
        out = it->second;
      }
    } else if (kind == "calendar") {
      const long step = std::stol(key);
      const StepValues v = step_values(ps.cal, step, 0);
      out.assign(v.rad, v.rad + 5);
      out.insert(out.end(), v.surf, v.surf + 7);
      out.push_back(v.carbon);
      out.push_back(v.next_carbon_step);
      out.push_back((double)ps.start_step);
      out.push_back(ps.nkits);
    } else {
      throw Error(EXOGCM_EINVAL, "unknown kind " + kind);
    }
    if (values) {
      if (*count < out.size()) throw Error(EXOGCM_EINVAL, "buffer too small");
      std::copy(out.begin(), out.end(), values);
    }
    *count = out.size();
  });
}
}  // namespace

int exogcm_setup_preview(const exogcm_planet* planet, const exogcm_boundary* boundary, const char* name,
                         double* values, size_t* count) {
  return setup_preview(planet, boundary, name, values, count, false);
}

int exogcm_setup_preview_device(const exogcm_planet* planet, const exogcm_boundary* boundary, const char* name,
                                double* values, size_t* count) {
  return setup_preview(planet, boundary, name, values, count, true);
}

int exogcm_slot_date(exogcm_engine* e, int slot, long step, int* date) {
  return guard([&] {
    if (!e || !date) throw Error(EXOGCM_EINVAL, "null argument");
    check_slot(e, slot);
    const Slot& s = e->slots[slot];
    if (!s.active && s.cal.steps_per_day == 0) throw Error(EXOGCM_ESTATE, "slot was never configured");
    calendar_date(s.cal, step < 0 ? s.step : step, date);
  });
}

int exogcm_setup_on_device(exogcm_engine* e, int enable) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    e->setup_on_device = enable != 0;
  });
}

int exogcm_release(exogcm_engine* e, int slot) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    check_slot(e, slot);
    e->slots[slot].active = false;
    e->slots[slot].published = -1;
  });
}

int exogcm_step_async(exogcm_engine* e, int steps, int publish_every) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    if (steps < 1 || steps > kMaxBatch) throw Error(EXOGCM_EINVAL, "steps must be 1..64");
    if (publish_every < 1 || steps > publish_every)
      throw Error(EXOGCM_EINVAL, "publish_every must be >= steps so each slot publishes at most once");
    if (!e->shared_ready) throw Error(EXOGCM_ESTATE, "no slot configured");
    // A third batch waits for the oldest to finish (IN_FLIGHT = 2).
    while ((int)e->pending.size() >= kInFlight) retire_oldest(e, true);
    int b = 0;
    while (std::find(e->pending.begin(), e->pending.end(), b) != e->pending.end()) ++b;
    exogcm_engine::Batch& B = e->batch[b];
    const int S = e->d.S;
    StepParams* rows = e->hparams + (size_t)(1 + b) * kMaxBatch * S;
    for (int s = 0; s < S; ++s) e->slots[s].published = -1;
    for (int k = 0; k < steps; ++k)
      for (int s = 0; s < S; ++s) rows[(size_t)k * S + s] = next_params(e->slots[s], publish_every, true);
    check(cudaMemcpyAsync(e->params, rows, (size_t)steps * S * sizeof(StepParams), cudaMemcpyHostToDevice,
                          e->stream),
          "params upload");
    cudaGraphExec_t g = batch_graph(e, steps);
    check(cudaEventRecord(B.start, e->stream), "event");
    check(cudaGraphLaunch(g, e->stream), "graph launch");
    check(cudaEventRecord(B.end, e->stream), "event");
    phy_finite_check(e->model(steps - 1), e->stream);
    check(cudaMemcpyAsync(B.fault_host, e->fault, sizeof(int), cudaMemcpyDeviceToHost, e->stream), "fault word");
    check(cudaMemsetAsync(e->fault, 0, sizeof(int), e->stream), "fault word");
    // start/end bracket the graph alone (the step time); done marks the
    // fault word's arrival in host memory, after which the batch retires.
    check(cudaEventRecord(B.done, e->stream), "event");
    e->pending.push_back(b);
  });
}

int exogcm_poll(exogcm_engine* e, int* done) {
  return guard([&] {
    if (!e || !done) throw Error(EXOGCM_EINVAL, "null argument");
    while (!e->pending.empty() && retire_oldest(e, false)) {
    }
    *done = e->pending.empty() ? 1 : 0;
  });
}

int exogcm_wait(exogcm_engine* e) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
  });
}

int exogcm_step(exogcm_engine* e, int steps, int publish_every) {
  const int rc = exogcm_step_async(e, steps, publish_every);
  if (rc != EXOGCM_OK) return rc;
  return exogcm_wait(e);
}

int exogcm_group_step(exogcm_engine** engines, int count, const int* steps, int publish_every, float* ms) {
  return guard([&] {
    if (!engines || !steps || count < 1) throw Error(EXOGCM_EINVAL, "null argument or empty group");
    std::vector<std::pair<const exogcm_engine*, int>> key;
    for (int i = 0; i < count; ++i) {
      exogcm_engine* e = engines[i];
      if (!e) throw Error(EXOGCM_EINVAL, "null engine in group");
      if (steps[i] < 1 || steps[i] > kMaxBatch) throw Error(EXOGCM_EINVAL, "steps must be 1..64");
      if (publish_every < 1 || steps[i] > publish_every)
        throw Error(EXOGCM_EINVAL, "publish_every must be >= steps so each slot publishes at most once");
      if (!e->shared_ready) throw Error(EXOGCM_ESTATE, "an engine of the group has no slot configured");
      if (e->device != engines[0]->device) throw Error(EXOGCM_EINVAL, "engines of a group share one device");
      for (const auto& k : key)
        if (k.first == e) throw Error(EXOGCM_EINVAL, "an engine appears twice in the group");
      key.push_back({e, steps[i]});
      retire_all(e);
    }
    exogcm_engine* lead = engines[0];
    cudaStream_t st = lead->stream;
    // Each engine's step values, uploaded to its own parameter block; its
    // K-step graph (captured once) becomes a child node of the group graph.
    for (int i = 0; i < count; ++i) {
      exogcm_engine* e = engines[i];
      const int S = e->d.S;
      for (int s = 0; s < S; ++s) e->slots[s].published = -1;
      for (int k = 0; k < steps[i]; ++k)
        for (int s = 0; s < S; ++s) e->hparams[(size_t)k * S + s] = next_params(e->slots[s], publish_every, true);
      check(cudaMemcpyAsync(e->params, e->hparams, (size_t)steps[i] * S * sizeof(StepParams),
                            cudaMemcpyHostToDevice, st),
            "params upload");
      batch_graph(e, steps[i]);
    }
    cudaGraphExec_t exec = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_group_mutex);
      auto it = g_group_graphs.find(key);
      if (it != g_group_graphs.end()) exec = it->second;
    }
    if (!exec) {
      cudaGraph_t parent;
      check(cudaGraphCreate(&parent, 0), "group graph");
      for (int i = 0; i < count; ++i) {
        cudaGraphNode_t node;
        check(cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, engines[i]->graph_templates.at(steps[i])),
              "group graph child");
      }
      check(cudaGraphInstantiate(&exec, parent, 0), "group graph instantiate");
      cudaGraphDestroy(parent);
      std::lock_guard<std::mutex> lock(g_group_mutex);
      g_group_graphs[key] = exec;
    }
    check(cudaEventRecord(lead->ev0, st), "event");
    check(cudaGraphLaunch(exec, st), "group graph launch");
    check(cudaEventRecord(lead->ev1, st), "event");
    for (int i = 0; i < count; ++i) phy_finite_check(engines[i]->model(steps[i] - 1), st);
    check(cudaStreamSynchronize(st), "group step");
    float t = 0.f;
    check(cudaEventElapsedTime(&t, lead->ev0, lead->ev1), "event time");
    if (ms) *ms = t;
    for (int i = 0; i < count; ++i) {
      int fault = 0;
      check(cudaMemcpy(&fault, engines[i]->fault, sizeof(int), cudaMemcpyDeviceToHost), "fault word");
      if (fault) {
        check(cudaMemset(engines[i]->fault, 0, sizeof(int)), "fault word");
        throw Error(EXOGCM_EDEVICE, "a tensor-core transform gave up waiting for its MMAs; this step's results are invalid");
      }
      engines[i]->last_ms = t;
    }
  });
}

int exogcm_budgets(exogcm_engine* e, int slot, double* last, double* mean, long* samples, int reset) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    check_slot(e, slot);
    double b[kBudgetStride];
    check(cudaMemcpy(b, e->budget + (size_t)slot * kBudgetStride, sizeof(b), cudaMemcpyDeviceToHost), "budgets");
    const double n = b[2 * kBudgetQuantities];
    for (int k = 0; k < kBudgetQuantities; ++k) {
      if (last) last[k] = b[k];
      if (mean) mean[k] = n > 0 ? b[kBudgetQuantities + k] / n : 0.0;
    }
    if (samples) *samples = (long)n;
    if (reset) {
      check(cudaMemset(e->budget + (size_t)slot * kBudgetStride + kBudgetQuantities, 0,
                       (kBudgetQuantities + 1) * sizeof(double)),
            "budgets");
    }
  });
}

int exogcm_averages_enable(exogcm_engine* e, int enable) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    const size_t n = (size_t)e->d.P * e->d.S * e->d.NHOR;
    if (enable && !e->avg) {
      if (cudaMalloc(&e->avg, n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        e->avg = nullptr;
        throw Error(EXOGCM_ENOMEM, "device memory for the averages (" + std::to_string(n * 8 >> 20) + " MiB)");
      }
      check(cudaMemset(e->avg, 0, n * sizeof(double)), "averages");
      for (int s = 0; s < e->d.S; ++s)
        check(cudaMemset(e->budget + (size_t)s * kBudgetStride + 2 * kBudgetQuantities + 1, 0, sizeof(double)),
              "averages");
    } else if (!enable && e->avg) {
      check(cudaStreamSynchronize(e->stream), "averages");
      cudaFree(e->avg);
      e->avg = nullptr;
    } else {
      return;
    }
    // The batch graphs hold the averages pointer: capture them again.
    drop_graphs(e);
  });
}

int exogcm_averages_read(exogcm_engine* e, int slot, float* mean, size_t count, long* samples, int reset) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    check_slot(e, slot);
    if (!e->avg) throw Error(EXOGCM_ESTATE, "averages are not enabled");
    const size_t per = (size_t)e->d.P * e->d.NHOR;
    if (mean && count != per) throw Error(EXOGCM_EINVAL, "averages buffer size mismatch (snapshot planes x points)");
    double n = 0;
    check(cudaMemcpy(&n, e->budget + (size_t)slot * kBudgetStride + 2 * kBudgetQuantities + 1, sizeof(double),
                     cudaMemcpyDeviceToHost),
          "averages");
    if (samples) *samples = (long)n;
    std::vector<double> row(e->d.NHOR);
    for (int pl = 0; pl < e->d.P; ++pl) {
      double* src = e->avg + ((size_t)pl * e->d.S + slot) * e->d.NHOR;
      if (mean) {
        check(cudaMemcpy(row.data(), src, e->d.NHOR * sizeof(double), cudaMemcpyDeviceToHost), "averages");
        for (int h = 0; h < e->d.NHOR; ++h) mean[(size_t)pl * e->d.NHOR + h] = n > 0 ? (float)(row[h] / n) : 0.f;
      }
      if (reset) check(cudaMemset(src, 0, e->d.NHOR * sizeof(double)), "averages");
    }
    if (reset)
      check(cudaMemset(e->budget + (size_t)slot * kBudgetStride + 2 * kBudgetQuantities + 1, 0, sizeof(double)),
            "averages");
  });
}

int exogcm_read_snapshot(exogcm_engine* e, int slot, float* values, size_t count, long* step) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    check_slot(e, slot);
    const long pub = e->slots[slot].published;
    if (step) *step = pub;
    if (!values || pub < 0) return;
    const FieldInfo& fi = field(e, "snapshot");
    if (count != fi.plane * fi.count) throw Error(EXOGCM_EINVAL, "snapshot buffer size mismatch");
    copy_field(e, fi, slot, values, false);
  });
}

int exogcm_snapshots_begin(exogcm_engine* e, float* values, size_t count) {
  return guard([&] {
    if (!e || !values) throw Error(EXOGCM_EINVAL, "null argument");
    // Batches in flight are not waited for: the staging copy below is queued
    // on the engine's stream behind the last submitted batch, so it takes the
    // snapshot that batch leaves while the host goes on submitting.
    const FieldInfo& fi = field(e, "snapshot");
    const size_t n = fi.plane * fi.count * e->d.S;
    if (count != n) throw Error(EXOGCM_EINVAL, "snapshot buffer size mismatch (planes x slots x points)");
    if (e->copy_pending) {
      check(cudaEventSynchronize(e->snap_copied), "previous snapshot copy");
      e->copy_pending = false;
    }
    // Each resource is created on its own test, so a call after a failed
    // set-up (say, the staging allocation) retries what is missing instead of
    // copying through a null staging buffer.
    if (!e->copy_stream)
      check(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking), "copy stream");
    if (!e->snap_staged) check(cudaEventCreateWithFlags(&e->snap_staged, cudaEventDisableTiming), "event");
    if (!e->snap_copied) check(cudaEventCreateWithFlags(&e->snap_copied, cudaEventDisableTiming), "event");
    if (!e->snap_stage) check(cudaMalloc(&e->snap_stage, n * sizeof(float)), "snapshot staging");
    // The device copy runs on the engine's stream, so the next step's graph
    // (queued after it) may overwrite the field while the host copy drains
    // the staging buffer on the copy stream.
    check(cudaMemcpyAsync(e->snap_stage, e->arena + fi.offset, n * sizeof(float), cudaMemcpyDeviceToDevice,
                          e->stream),
          "snapshot staging");
    check(cudaEventRecord(e->snap_staged, e->stream), "event");
    check(cudaStreamWaitEvent(e->copy_stream, e->snap_staged, 0), "copy stream wait");
    check(cudaMemcpyAsync(values, e->snap_stage, n * sizeof(float), cudaMemcpyDeviceToHost, e->copy_stream),
          "snapshot copy");
    check(cudaEventRecord(e->snap_copied, e->copy_stream), "event");
    e->copy_pending = true;
  });
}

int exogcm_snapshots_wait(exogcm_engine* e) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    if (!e->copy_pending) return;
    check(cudaEventSynchronize(e->snap_copied), "snapshot copy");
    e->copy_pending = false;
  });
}

int exogcm_set_stop(exogcm_engine* e, int slot, long step) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    retire_all(e);
    check_slot(e, slot);
    e->slots[slot].stop = step;
  });
}

int exogcm_slot_info(exogcm_engine* e, int slot, long* step, int* startup_left, int* active) {
  return guard([&] {
    if (!e) throw Error(EXOGCM_EINVAL, "null engine");
    check_slot(e, slot);
    if (step) *step = e->slots[slot].step;
    if (startup_left) *startup_left = e->slots[slot].startup_left;
    if (active) *active = e->slots[slot].active ? 1 : 0;
  });
}

int exogcm_field_size(exogcm_engine* e, const char* name, size_t* count) {
  return guard([&] {
    if (!e || !count) throw Error(EXOGCM_EINVAL, "null argument");
    const FieldInfo& fi = field(e, name);
    *count = fi.plane * fi.count;
  });
}

int exogcm_read_field(exogcm_engine* e, int slot, const char* name, float* values, size_t count) {
  return guard([&] {
    if (!e || !values) throw Error(EXOGCM_EINVAL, "null argument");
    retire_all(e);
    check_slot(e, slot);
    const FieldInfo& fi = field(e, name);
    if (count != fi.plane * fi.count) throw Error(EXOGCM_EINVAL, std::string(name) + ": wrong value count");
    copy_field(e, fi, slot, values, false);
  });
}

int exogcm_write_field(exogcm_engine* e, int slot, const char* name, const float* values, size_t count) {
  return guard([&] {
    if (!e || !values) throw Error(EXOGCM_EINVAL, "null argument");
    retire_all(e);
    check_slot(e, slot);
    const FieldInfo& fi = field(e, name);
    if (count != fi.plane * fi.count) throw Error(EXOGCM_EINVAL, std::string(name) + ": wrong value count");
    copy_field(e, fi, slot, const_cast<float*>(values), true);
  });
}

int exogcm_read_table(exogcm_engine* e, int slot, const char* name, float* values, size_t count) {
  return guard([&] {
    if (!e || !values || !name) throw Error(EXOGCM_EINVAL, "null argument");
    retire_all(e);
    check_slot(e, slot);
    int off = 0;
    for (auto& t : e->tab_list) {
      if (t.first == name) {
        if ((int)count != t.second) throw Error(EXOGCM_EINVAL, "table size mismatch");
        check(cudaMemcpy(values, e->tabs + (size_t)slot * e->to.stride + off, count * sizeof(float),
                         cudaMemcpyDeviceToHost),
              "read table");
        return;
      }
      off += t.second;
    }
    throw Error(EXOGCM_EINVAL, std::string("no table ") + name);
  });
}

int exogcm_checkpoint_save(exogcm_engine* e, int slot, void** buffer, size_t* size) {
  return guard([&] {
    if (!e || !buffer || !size) throw Error(EXOGCM_EINVAL, "null argument");
    retire_all(e);
    check_slot(e, slot);
    const Slot& s = e->slots[slot];
    if (!s.active) throw Error(EXOGCM_ESTATE, "slot is not running");
    if (s.startup_left > 0) throw Error(EXOGCM_ESTATE, "slot is still in its start-up steps");
    const std::string json = header_json(e, s.step, s.carbon_step);
    const size_t mlen = sizeof(kMagic) - 1;
    const size_t start = (mlen + 4 + json.size() + 3) / 4 * 4;
    size_t floats = 0;
    for (auto& fi : e->fields) floats += fi.plane * fi.count;
    const size_t total = start + floats * 4;
    unsigned char* out = static_cast<unsigned char*>(std::calloc(total, 1));
    if (!out) throw Error(EXOGCM_ENOMEM, "checkpoint buffer");
    std::memcpy(out, kMagic, mlen);
    const uint32_t len = (uint32_t)json.size();
    std::memcpy(out + mlen, &len, 4);  // little-endian hosts
    std::memcpy(out + mlen + 4, json.data(), json.size());
    float* data = reinterpret_cast<float*>(out + start);
    try {
      for (auto& fi : e->fields) {
        copy_field(e, fi, slot, data, false);
        data += fi.plane * fi.count;
      }
    } catch (...) {
      std::free(out);
      throw;
    }
    *buffer = out;
    *size = total;
  });
}

int exogcm_checkpoint_load(exogcm_engine* e, int slot, const void* buffer, size_t size) {
  return guard([&] {
    if (!e || !buffer) throw Error(EXOGCM_EINVAL, "null argument");
    retire_all(e);
    check_slot(e, slot);
    Slot& s = e->slots[slot];
    if (!s.active) throw Error(EXOGCM_ESTATE, "configure the slot before loading a checkpoint");
    const unsigned char* in = static_cast<const unsigned char*>(buffer);
    const size_t mlen = sizeof(kMagic) - 1;
    if (size < mlen + 4 || std::memcmp(in, kMagic, mlen) != 0)
      throw Error(EXOGCM_ELAYOUT, "This checkpoint was not saved by the WebGPU model");
    uint32_t len;
    std::memcpy(&len, in + mlen, 4);
    if (mlen + 4 + (size_t)len > size) throw Error(EXOGCM_ELAYOUT, "truncated checkpoint header");
    const std::string json(reinterpret_cast<const char*>(in + mlen + 4), len);
    const std::string expected = header_json(e, 0, 0);
    const size_t cut = expected.find("],\"step\"");
    if (json.compare(0, cut, expected, 0, cut) != 0)
      throw Error(EXOGCM_ELAYOUT, "This checkpoint's model state does not match this version of the model");
    const long step = json_number(json, "step");
    const long carbon = json_number(json, "carbonStep");
    const size_t start = (mlen + 4 + len + 3) / 4 * 4;
    size_t floats = 0;
    for (auto& fi : e->fields) floats += fi.plane * fi.count;
    if (start + floats * 4 != size) throw Error(EXOGCM_ELAYOUT, "checkpoint data size does not match its header");
    std::vector<float> buf;
    const unsigned char* data = in + start;
    for (auto& fi : e->fields) {
      const size_t n = fi.plane * fi.count;
      buf.resize(n);
      std::memcpy(buf.data(), data, n * 4);
      copy_field(e, fi, slot, buf.data(), true);
      data += n * 4;
    }
    s.step = step;
    s.carbon_step = (int)carbon;
    s.startup_left = 0;
    s.published = -1;
  });
}

void exogcm_free(void* buffer) { std::free(buffer); }

int exogcm_unstable(exogcm_engine* e, int* flags, int n) {
  return guard([&] {
    if (!e || !flags || n != e->d.S) throw Error(EXOGCM_EINVAL, "flags must hold one int per slot");
    retire_all(e);
    check(cudaMemcpy(flags, e->flags, n * sizeof(int), cudaMemcpyDeviceToHost), "flags");
  });
}

int exogcm_run_stage(exogcm_engine* e, const char* stage) {
  return guard([&] {
    if (!e || !stage) throw Error(EXOGCM_EINVAL, "null argument");
    retire_all(e);
    if (!e->shared_ready) throw Error(EXOGCM_ESTATE, "no slot configured");
    const int S = e->d.S;
    // A replayed step publishes (main loop), so the pack stage writes the
    // snapshot the replay compares.
    for (int s = 0; s < S; ++s) {
      Slot copy = e->slots[s];
      e->hparams[s] = next_params(copy, 1, false);
    }
    check(cudaMemcpyAsync(e->params, e->hparams, S * sizeof(StepParams), cudaMemcpyHostToDevice, e->stream),
          "params");
    // Stage replay compares every field, so the fused transforms also write
    // the Fourier fields they pass through, and physics_in zeroes the grid
    // tendencies.
    Model m = e->model(0);
    m.keep_fourier = 1;
    m.zero_gdt = 1;
    run_stage(m, stage, e->stream);
    check(cudaGetLastError(), "stage launch");
    check(cudaStreamSynchronize(e->stream), "stage");
  });
}

int exogcm_last_step_ms(exogcm_engine* e, float* ms) {
  return guard([&] {
    if (!e || !ms) throw Error(EXOGCM_EINVAL, "null argument");
    *ms = e->last_ms;
  });
}

int exogcm_time_kernel(exogcm_engine* e, const char* kernel, int reps, float* ms, double* bytes) {
  return guard([&] {
    if (!e || !kernel || !ms || reps < 1) throw Error(EXOGCM_EINVAL, "bad argument");
    retire_all(e);
    if (!e->shared_ready) throw Error(EXOGCM_ESTATE, "no slot configured");
    const Dims& d = e->d;
    const int S = d.S;
    for (int s = 0; s < S; ++s) {
      Slot copy = e->slots[s];
      e->hparams[s] = next_params(copy, 1 << 30, false);
    }
    check(cudaMemcpyAsync(e->params, e->hparams, S * sizeof(StepParams), cudaMemcpyHostToDevice, e->stream),
          "params");
    const Model m = e->model(0);
    const FieldPtrs& F = m.f;
    const int LP = d.L * S;
    const double grid = (double)d.NHOR * 4, four = (double)d.NLAT * d.NFC * 4, spec = (double)d.NRSP * 4;
    const double cols = (double)S * d.NHOR;
    const std::string k(kernel);
    std::function<void()> launch;
    double b = 0;
    const double L = d.L;
    if (k == "fourier_forward") {
      launch = [&] { tr_fourier_forward(m, F.gtn, F.fgtn, LP, e->stream); };
      b = LP * (grid + four);
    } else if (k == "fourier_inverse") {
      launch = [&] { tr_fourier_inverse(m, F.fgu, F.gu, LP, e->stream); };
      b = LP * (four + grid);
    } else if (k == "fourier_forward_per_chunk" || k == "fourier_forward_persistent" ||
               k == "fourier_inverse_per_chunk" || k == "fourier_inverse_persistent") {
      // an FFT in a fixed form whatever the tuning chose
      const bool forward = k.compare(0, 15, "fourier_forward") == 0;
      const int form = k.size() > 10 && k.compare(k.size() - 10, 10, "persistent") == 0 ? 1 : 0;
      launch = [&, forward, form] {
        Model mp = m;
        mp.tune.fft_persistent[forward ? 0 : 1] = form;
        if (forward)
          tr_fourier_forward(mp, F.gtn, F.fgtn, LP, e->stream);
        else
          tr_fourier_inverse(mp, F.fgu, F.gu, LP, e->stream);
      };
      b = LP * (grid + four);
    } else if (k == "legendre_forward") {
      launch = [&] { tr_legendre_forward(m, F.fgtdt, F.zstt1, LP, m.sh.qc, e->stream); };
      b = LP * (four + spec);
    } else if (k == "sp2gp") {
      // fused sp2fc + fc2gp: the spectral plane in, the grid plane out
      launch = [&] { tr_sp2gp(m, F.st, F.fgt, F.gt, LP, m.sh.qi, e->stream); };
      b = LP * (spec + grid);
    } else if (k == "sp2gp_planes2" || k == "sp2gp_planes4") {
      // the fused transform at a fixed number of planes per pass
      const int pp = k == "sp2gp_planes4" ? 4 : 2;
      if (grid_sp2gp_smem(d, pp) > kLegSmemLimit) throw Error(EXOGCM_EINVAL, "shape needs too much shared memory");
      launch = [&, pp] {
        Model mp = m;
        mp.tune.sp2gp_planes = pp;
        tr_sp2gp(mp, F.st, F.fgt, F.gt, LP, mp.sh.qi, e->stream);
      };
      b = LP * (spec + grid);
    } else if (k == "legendre_inverse") {
      launch = [&] { tr_legendre_inverse(m, F.st, F.fgt, LP, m.sh.qi, e->stream); };
      b = LP * (spec + four);
    } else if (k == "dv2uv") {
      launch = [&] { tr_dv2uv(m, F.sd, F.sz, F.fgu, F.fgv, LP, 1.63299310207f, e->stream); };
      b = LP * 2 * (spec + four);
    } else if (k == "uv2dv") {
      launch = [&] { tr_uv2dv(m, F.fgvz, F.fguz, F.fgke, F.zdsdp1, F.zdszp1, LP, e->stream); };
      b = LP * (3 * four + 2 * spec);
    } else if (k == "qtend") {
      launch = [&] { tr_qtend(m, F.fgut, F.fgvt, F.fgtn, F.zstt2, LP, e->stream); };
      b = LP * (3 * four + spec);
    } else if (k == "calcgp") {
      launch = [&] { dyn_calcgp(m, e->stream); };
      b = cols * 4 * (6.0 * d.L + 3 + 12.0 * d.L + 2);
    } else if (k == "spectrala") {
      launch = [&] { dyn_spectrala(m, e->stream); };
      b = (double)S * d.NRSP * 4 * (6.0 * d.L + 3 + 14.0 * d.L + 3);
    } else if (k == "mkdheat") {
      // stage 1: dq, u, v, du, dv per level and dp in; dtdt out
      launch = [&] { dyn_mkdheat(m, 1, e->stream); };
      b = cols * 4 * (6.0 * d.L + 1);
    } else if (k == "physics_in") {
      // gp, u, v, t, q in; dp, the dimensional u, v, t, q and the surface
      // level of the zeroed dimensional tendencies out
      launch = [&] { dyn_physics_in(m, e->stream); };
      b = cols * 4 * (4.0 * d.L + 1 + 1 + 4.0 * d.L + 4);
    } else if (k == "physics_out") {
      // four physics tendencies, the fixer's gqdt and dp in; four tendencies out
      launch = [&] { dyn_physics_out(m, e->stream); };
      b = cols * 4 * (5.0 * d.L + 1 + 4.0 * d.L);
    } else {
      // Column kernels: compulsory reads + writes per column, in floats.
      const std::map<std::string, double> per_column = {
          {"vdiff", 8 * L + 4},                              // t, q, u, v, surflx's tendencies in; 4 tendencies out
          {"swr", 5 * L + 7 + 3 * (L + 1) + 3},              // dcc, dql, dq, dt, dqo3 + surface in; 3 fluxes + albedos out
          {"lwr_radstep", 7 * L + 4 + 4 * (L + 1) + 4 * L},  // t, q, o3, co2, clouds, sw flux, dtdt in; 4 fluxes + 4 rates out
          {"kuo", 5 * L + 3 + 6 * L + 1},                    // dqt, q, t and tendencies in; tendencies, rain, cloud levels out
          {"rain_column", 12 * L + 4 + 6 * L + 8},
          // the full step's other column kernels and its fused ones (timed
          // for the fusion choice; no byte count)
          {"fixer_apply", 0}, {"surflx", 0}, {"solang_mko3", 0}, {"mkdca", 0}, {"soil", 0}, {"land_surface", 0},
          {"sea_ice", 0}, {"sea", 0}, {"carbon", 0}, {"storm", 0}, {"fused_fixer_flux_solang", 0},
          {"fused_kuo_mkdca", 0},
          {"fused_rain_soil", 0}, {"fused_land_seaice", 0}, {"fused_sea_carbon", 0},
      };
      auto it = per_column.find(k);
      if (it == per_column.end()) throw Error(EXOGCM_EINVAL, "unknown kernel " + k);
      launch = [&] {
        if (!phy_launch_one(m, k, e->stream)) throw Error(EXOGCM_EINVAL, "unknown kernel " + k);
      };
      b = cols * 4 * it->second;
    }
    launch();  // warm
    check(cudaEventRecord(e->ev0, e->stream), "event");
    for (int r = 0; r < reps; ++r) launch();
    check(cudaEventRecord(e->ev1, e->stream), "event");
    check(cudaStreamSynchronize(e->stream), "time kernel");
    float total = 0;
    check(cudaEventElapsedTime(&total, e->ev0, e->ev1), "event time");
    *ms = total / reps;
    if (bytes) *bytes = b;
  });
}

int exogcm_tuning(exogcm_engine* e, int* values, int count) {
  return guard([&] {
    if (!e || !values || count < 9) throw Error(EXOGCM_EINVAL, "need room for 9 values");
    const Tuning& t = e->tune;
    const int v[16] = {t.fft_rows,       t.inv_group[0],   t.inv_tile[0],      t.inv_group[1],
                       t.inv_tile[1],    t.fwd_tile[0],    t.fwd_tile[1],      t.fwd_tile[2],
                       t.fwd_tile[3],    t.fwd_buffers[0], t.fwd_buffers[1],   t.fwd_buffers[2],
                       t.fwd_buffers[3], t.sp2gp_planes,   t.fft_persistent[0], t.fft_persistent[1]};
    std::copy(v, v + std::min(count, 16), values);
  });
}

int exogcm_graph_launches(exogcm_engine* e, int steps, size_t* launches) {
  return guard([&] {
    if (!e || !launches || steps < 1 || steps > kMaxBatch) throw Error(EXOGCM_EINVAL, "bad argument");
    cudaGraph_t graph;
    check(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed), "capture");
    for (int k = 0; k < steps; ++k) full_step(e->model(k), e->stream);
    check(cudaStreamEndCapture(e->stream, &graph), "capture end");
    size_t n = 0;
    check(cudaGraphGetNodes(graph, nullptr, &n), "graph nodes");
    cudaGraphDestroy(graph);
    *launches = n;
  });
}

int exogcm_device_field(exogcm_engine* e, const char* name, void** pointer, size_t* floats) {
  return guard([&] {
    if (!e || !pointer) throw Error(EXOGCM_EINVAL, "null argument");
    const FieldInfo& fi = field(e, name);
    *pointer = e->arena + fi.offset;
    if (floats) *floats = fi.plane * fi.count * e->d.S;
  });
}

void* exogcm_stream(exogcm_engine* e) { return e ? (void*)e->stream : nullptr; }

}  // extern "C"
