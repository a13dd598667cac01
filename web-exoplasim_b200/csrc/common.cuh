// Device-side data layout shared by every kernel of the batched GCM step.
//
// HBM layout. A batch holds S planet slots of one resolution (T, L). Every
// state field is stored [plane][slot][plane floats], where a field's planes
// are its levels (or climatology months, or table entries). So level l of
// slot s of a grid field f is f[(l * S + s) * NHOR + h]: with the column
// index c = s * NHOR + h the whole batch is one grid of S * NHOR columns and
// the column kernels index it exactly as the reference indexes one planet
// (state[field + l * NHOR + h], src/model/climate/gcm/kernel/index.ts). The
// same holds for spectral fields (S * NRSP coefficients per level) and
// Fourier fields (S * NLAT rows of NFC per level). Transforms see each field
// as count * S contiguous planes.
//
// Per-planet values: PlanetConst (scalars) indexed by slot, and a block of
// per-planet tables (PlaneTabs offsets) at tabs + slot * tab_stride.
// Per-step values (the reference's CPU-written radiation_step, surface_step,
// carbon_step, snapshot_step slots and the start-up phase) are StepParams,
// indexed [step in batch][slot].
#pragma once
#include <cstddef>
#include <cstdint>

#include "fields.h"

namespace exogcm {


// Programmatic dependent launch. A kernel started by pdl_launch may become
// resident while the kernel before it on the stream drains: it calls
// pdl_wait() before its first access to any state an earlier kernel writes
// (that returns once those kernels have finished and their stores are
// visible), and pdl_release() to let the kernel after it start the same way.
// In a kernel launched the ordinary way both return at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Per-planet global budgets (budget.cu): quantities per published step.
constexpr int kBudgetQuantities = 8;
constexpr int kBudgetStride = 2 * kBudgetQuantities + 2;  // last[8], sums[8], samples, averaged samples

constexpr int NLSOIL = 5;  // landmod's soil layers
constexpr int MONTHS = 14; // climatology months with December before and January after

struct Dims {
  int T, L, NLAT, NLON, NHOR, NTP1, NCSP, NRSP, NFC, NLEV, NLEM, NLEP, P;
  int S;  // planet slots in the batch
};

inline Dims make_dims(int truncation, int levels, int slots) {
  Dims d{};
  d.T = truncation;
  d.L = levels;
  d.NLAT = truncation == 21 ? 32 : truncation == 42 ? 64 : truncation == 63 ? 96 : 0;
  d.NLON = 2 * d.NLAT;
  d.NHOR = d.NLAT * d.NLON;
  d.NTP1 = truncation + 1;
  d.NCSP = d.NTP1 * (d.NTP1 + 1) / 2;
  d.NRSP = 2 * d.NCSP;
  d.NFC = 2 * d.NTP1;
  d.NLEV = levels;
  d.NLEM = levels - 1;
  d.NLEP = levels + 1;
  d.P = 51 + 5 * levels;
  d.S = slots;
  return d;
}

struct PlanetConst {
#define EXOGCM_DECLARE_CONST(n) float n;
  EXOGCM_CONSTS(EXOGCM_DECLARE_CONST)
#undef EXOGCM_DECLARE_CONST
};

// One step's host-computed values for one slot (stepper/index.ts:281-334)
// and its timestep phase (setup/index.ts:44-49: halved per start-up step).
struct StepParams {
  float delt, delt2, deltsec, deltsec2;
  float filter;   // leapfrog filter on (main loop)
  float coupled;  // icestep coupled (main loop)
  int phase;      // bm1 block: 0 main loop, k = start-up steps still to run
  int active;     // slot holds a running planet
  float rad[5];   // radiation_step
  float surf[7];  // surface_step
  float carbon;   // carbon_step
  float snap[3];  // snapshot_step
};

struct FieldPtrs {
#define EXOGCM_DECLARE_FIELD(name, shape, count) float* name;
  EXOGCM_FIELDS(EXOGCM_DECLARE_FIELD)
#undef EXOGCM_DECLARE_FIELD
};

struct TabOffsets {
#define EXOGCM_DECLARE_TAB(name, count) int name;
  EXOGCM_PTABLES(EXOGCM_DECLARE_TAB)
#undef EXOGCM_DECLARE_TAB
  int stride;
};

// Tables every slot of a batch shares (one resolution, one filter setting).
struct SharedTabs {
  const float* fwd;    // fourier_forward [NLON][NFC]
  const float* inv;    // fourier_inverse [NFC][NLON]
  const float* qi;     // legendre_q* [NLAT][NCSP], filtered
  const float* qj;
  const float* qc;
  const float* qe;
  const float* qm;
  const float* qq;
  const float* qu;
  const float* qv;
  const float* zgw;    // Gaussian weight per point [NHOR]
  const double* wlat;  // Gaussian weight per latitude in FP64 [NLAT] (the budgets' global means)
  const float* rcsq;   // 1 / cos^2(latitude) per point [NHOR]
  const float* sid;    // sin(latitude) [NLAT]
  const float* cola;   // cos(latitude) [NLAT]
  const float* nindex; // total wavenumber per real coefficient [NRSP]
  const int* mode_m;   // zonal wavenumber m of mode w [NCSP]
  const int* mode_n;   // total wavenumber n of mode w [NCSP]
  const float* tw;     // e^{2 pi i j / NLON} as (cos, sin) pairs [NLON][2], for the FFTs
  // Northern halves of the inverse tables, transposed to [NCSP][NLAT / 2]
  // for the optimized path's latitude-pair transforms.
  const float* qiT;
  const float* qjT;
  const float* quT;
  const float* qvT;
  // qiT and qjT again as the fused inverse transform's per-block slices
  // ([chunk of 8 latitude pairs][pair][padded mode row], grid_table_layout).
  const float* qiG;
  const float* qjG;
  // Tensor-core (mode 2) table operands: per image set (qi, qj, dv2uv,
  // fc2sp, uv2dv, mktend, qtend) and m, the hi and lo TF32 images of the
  // tables in the MMA's shared-memory layout, at float offset
  // tc_at[set * (NTP1 + 1) + m] of tc_img.
  const float* tc_img;
  const int* tc_at;
};

// Launch shapes of the optimized path's transforms, measured per engine by
// the autotuner among the shapes each kernel supports. They change how work
// is split over blocks, never the order of any sum, so results do not
// depend on them.
struct Tuning {
  int fft_rows;      // latitudes per FFT block (a multiple of 8 dividing NLAT)
  int fft_persistent[2];  // FFT blocks loop over chunks (1) or take one each (0): [0] forward, [1] inverse
  int inv_group[2];  // wavenumbers per inverse Legendre block: [0] sp2fc, [1] dv2uv
  int inv_tile[2];   // planes per inverse Legendre block (even)
  int fwd_tile[4];   // planes per forward Legendre tile (8 or 16), by kind
  int fwd_buffers[4];  // staging buffers of a forward Legendre block (1 or 2), by kind
  int sp2gp_planes;    // planes per pass of the fused inverse transform (2 or 4)
};

// Everything a step kernel can reach.
struct Model {
  Dims d;
  FieldPtrs f;
  SharedTabs sh;
  TabOffsets to;
  const float* tabs;         // per-slot table blocks [S][to.stride]
  const PlanetConst* pc;     // [S]
  const StepParams* params;  // [S] for the step being run
  double* sums;              // FP64 per-slot reductions scratch [S][4]
  double* budget;            // FP64 per-slot budgets [S][kBudgetStride]: last values, running sums, samples
  double* avg;               // FP64 running sums of the published snapshot fields, or null (averages off)
  int* flags;                // per-slot status flags [S]
  int* fault;                // nonzero after a kernel gave up a bounded wait
  int mode;                  // 0 plain path, 1 optimized path (FFTs, latitude-pair Legendre, m-major Fourier),
                             // 2 optimized path with every Legendre transform on the tensor cores
                             // (split precision)
  Tuning tune;               // optimized path launch shapes
  int keep_fourier;          // optimized path: fused transforms also write the Fourier fields they pass through
  // physics_in zeroes the grid tendencies gudt, gvdt, gtdt, gqdt and the
  // dimensional ones dudt, dvdt, dtdt, dqdt. The fixer first raises gqdt and
  // physics_out completes the four grid ones; surflx first raises the
  // lowest level of the dimensional ones and vdiff then updates every
  // level. Within a full step (zero_gdt = 0) physics_in leaves all but the
  // dimensional ones' surface level alone, and those kernels take the
  // zeros as values instead of reading them (the fixer writes gqdt as
  // 0 + its increment, physics_out gudt, gvdt, gtdt as its increment + 0,
  // surflx its level as 0 + its increment; vdiff reads only that level):
  // the values the zeroed fields give. Single-stage replay compares every
  // field after each stage, so there (zero_gdt = 1) the kernels zero and
  // read them as the reference does.
  int zero_gdt;
  int storm;  // some slot runs the storm-climatology diagnostics (NSTORMDIAG > 0)
};

}  // namespace exogcm
