// Host-side launchers of the step's kernels (one call each, all slots).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace exogcm {

// transforms.cu
void tr_init();
void tr_fourier_forward(const Model& m, const float* g, float* c, int planes, cudaStream_t st);
void tr_fourier_inverse(const Model& m, const float* c, float* g, int planes, cudaStream_t st);
void tr_dlambda(const Model& m, const float* a, float* b, int planes, cudaStream_t st);
void tr_legendre_inverse(const Model& m, const float* s, float* f, int planes, const float* q, cudaStream_t st);
// sp2fc then fc2gp of one field: f is the Fourier field between them (on the
// optimized path written only when m.keep_fourier), g the grid field.
void tr_sp2gp(const Model& m, const float* s, float* f, float* g, int planes, const float* q, cudaStream_t st);
void tr_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
              cudaStream_t st);
void tr_legendre_forward(const Model& m, const float* f, float* s, int planes, const float* q, cudaStream_t st);
void tr_uv2dv(const Model& m, const float* u, const float* v, const float* ke, float* D, float* Z, int planes,
              cudaStream_t st);
void tr_qtend(const Model& m, const float* u, const float* v, const float* src, float* out, int planes,
              cudaStream_t st);

// legendre.cu (optimized path)
constexpr size_t kLegSmemLimit = 200 * 1024;  // dynamic shared memory the transform kernels may ask
void leg_init();
// Resident blocks of `kernel` per SM for a launch shape, times the SM count.
int persistent_grid(const void* kernel, int threads, size_t smem);
size_t leg_inverse_smem(const Dims& d, int kind, int group, int tile);
size_t leg_forward_smem(const Dims& d, int kind, int tile);
Tuning default_tuning(const Dims& d);
void leg_inverse(const Model& m, const float* s, float* f, int planes, bool derivative, cudaStream_t st);
void leg_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
               cudaStream_t st);
void leg_forward(const Model& m, const float* f, float* s, int planes, const float* q, cudaStream_t st);
void leg_uv2dv(const Model& m, const float* u, const float* v, const float* ke, float* D, float* Z, int planes,
               cudaStream_t st);
void leg_qtend(const Model& m, const float* u, const float* v, const float* src, float* out, int planes,
               cudaStream_t st);

// legendre_tc.cu (mode 2: the Legendre transforms on the tensor cores, split precision)
void tc_init();
std::vector<float> tc_table_images(const Dims& d, const std::map<std::string, std::vector<double>>& q,
                                   std::vector<int>& at);
void tc_inverse(const Model& m, const float* s, float* f, int planes, bool derivative, cudaStream_t st);
void tc_dv2uv(const Model& m, const float* D, const float* Z, float* U, float* V, int planes, float plavor,
              cudaStream_t st);
void tc_forward(const Model& m, const float* f, float* s, int planes, cudaStream_t st);
void tc_uv2dv(const Model& m, const float* u, const float* v, const float* ke, float* D, float* Z, int planes,
              cudaStream_t st);
void tc_qtend(const Model& m, const float* u, const float* v, const float* src, float* out, int planes,
              cudaStream_t st);

// fft.cu (optimized path; Fourier planes m-major)
void fft_init();
// The northern table (transposed, [mode][pair]) as the fused inverse
// transform's blocks hold it: per chunk of 8 latitude pairs, one padded row
// of modes per pair.
std::vector<float> grid_table_layout(const Dims& d, const std::vector<double>& qT);
// Shared memory of the fused inverse transform at 2 or 4 planes per pass.
size_t grid_sp2gp_smem(const Dims& d, int planes_per_pass);
void grid_init();
void grid_sp2gp(const Model& m, const float* s, float* f, float* g, int planes, bool derivative, cudaStream_t st);
size_t fft_chunk_smem(const Dims& d, int rows);
bool fft_rows_supported(const Dims& d, int rows);
void fft_forward(const Model& m, const float* g, float* c, int planes, cudaStream_t st);
void fft_inverse(const Model& m, const float* c, float* g, int planes, cudaStream_t st);

// dynamics.cu
void dyn_calcgp(const Model& m, cudaStream_t st);
void dyn_spectrala(const Model& m, cudaStream_t st);
void dyn_spectrald_diffusion(const Model& m, cudaStream_t st);
void dyn_mkdheat(const Model& m, int stage, cudaStream_t st);
void dyn_mean_mode(const Model& m, float* target, cudaStream_t st);
void dyn_spectrald_update(const Model& m, cudaStream_t st);
void dyn_physics_in(const Model& m, cudaStream_t st);
void dyn_physics_out(const Model& m, cudaStream_t st);

// physics_flux.cu (IEEE division): fixer apply, surface fluxes, vdiff, solang/mko3
void phy_fixer_apply(const Model& m, cudaStream_t st);
void phy_solang_mko3(const Model& m, cudaStream_t st);
void phy_fused_fixer_flux_solang(const Model& m, cudaStream_t st);
bool phy_flux_launch_one(const Model& m, const std::string& kernel, cudaStream_t st);

// physics.cu
void phy_fixer(const Model& m, cudaStream_t st);
void phy_surface_flux(const Model& m, cudaStream_t st);
void phy_radiation(const Model& m, cudaStream_t st);
void phy_precipitation_columns(const Model& m, cudaStream_t st);
void phy_surface(const Model& m, cudaStream_t st);
void phy_carbon(const Model& m, cudaStream_t st);
// hurricanestep (physics/storm/wgsl/storm.wgsl), for slots with NSTORMDIAG > 0.
void phy_storm(const Model& m, cudaStream_t st);
// The full step's fused physics (see physics.cu): fixer through radiation,
// and (after the precipitation transform) precipitation through carbon.
void phy_fused_through_radiation(const Model& m, cudaStream_t st);
void phy_fused_precipitation_to_carbon(const Model& m, cudaStream_t st);
void phy_pack(const Model& m, cudaStream_t st);

// budget.cu: per-slot FP64 global budgets and the snapshot's running sums
void phy_budget(const Model& m, int snapshot_planes, cudaStream_t st);
void phy_finite_check(const Model& m, cudaStream_t st);
// One named column kernel of the physics (for timing); false if unknown.
bool phy_launch_one(const Model& m, const std::string& kernel, cudaStream_t st);

}  // namespace exogcm
