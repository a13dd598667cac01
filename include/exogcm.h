/*
 * exogcm: a B200-native ExoPlaSim spectral-GCM timestep behind a C ABI.
 *
 * This header is the drop-in boundary for the engine interface of
 * ryoung48/web-exoplasim (paths relative to src/model/climate/gcm/):
 *   - GCM_RUNNER.start / GcmRunRequest / GcmRun (runner/index.ts:61-78,
 *     runner/types.ts:47-74) drive an engine through configure, step, field
 *     readback and checkpoint; a host (the TypeScript runner through N-API,
 *     or any FFI) calls the functions below for those four operations.
 *   - Every function returns 0 on success or a negative EXOGCM_E* code;
 *     exogcm_last_error() gives the message (the reference's worker reports
 *     failures as strings through `fail`, runner/webgpu/gcm.worker.ts:48-51).
 *   - An engine is used from one host thread at a time. It owns one CUDA
 *     stream and all device memory; buffers passed in are caller-owned.
 *
 * An engine holds `slots` planets of one resolution (truncation T, L levels)
 * that step together in one batched launch sequence; slots are configured,
 * stepped, read and released independently (continuous batching).
 */
#ifndef EXOGCM_H
#define EXOGCM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EXOGCM_OK 0
#define EXOGCM_EINVAL (-1)     /* invalid argument */
#define EXOGCM_ENOMEM (-2)     /* device or host allocation failed (admission) */
#define EXOGCM_EUNSTABLE (-3)  /* a slot's state became non-finite */
#define EXOGCM_ELAYOUT (-4)    /* checkpoint does not match this layout */
#define EXOGCM_EDEVICE (-5)    /* CUDA error */
#define EXOGCM_ESTATE (-6)     /* call not valid in the slot's state */

typedef struct exogcm_engine exogcm_engine;

/* A planet's configuration: the GcmConfig fields the reference turns into
 * namelist edits (namelist/index.ts:40-182, types.ts:28-62), with the
 * atmosphere already resolved to a pressure, gas constant and CO2. */
typedef struct exogcm_planet {
  int truncation;                /* 21, 42 or 63 */
  int levels;                    /* 5 or 10 */
  double radius_earth;           /* planet radius in Earth radii */
  double gravity;                /* m/s^2 */
  double flux;                   /* stellar flux, W/m^2 */
  double eccentricity;
  double obliquity_deg;
  int fixed_orbit;               /* 1: orbit as given (NFIXORB = 1) */
  int keplerian;                 /* NGENKEPLERIAN */
  int synchronous;               /* tidally locked (NFIXED) */
  double substellar_longitude_deg;
  double ocean_depth_m;          /* slab ocean mixed-layer depth */
  double year_days;
  double rotation_period_days;
  double timestep_minutes;
  double pressure_bar;
  double gas_constant;           /* J/(kg K) */
  double co2_ppm;
  int ozone;
  int wet_soil;
  int vegetation;                /* 0, 1 or 2 */
  double initial_growth;
  int glaciers;                  /* glacier model on */
  double glacier_min_depth_m;
  double glacier_initial_height_m;
  int filter_gp;                 /* physics filter on grid-to-spectral sums */
  int filter_sp;                 /* physics filter on spectral-to-grid sums */
  int filter_kind;               /* NFILTER: 0 none, 1 Cesaro, 2 exp, 3 Landau-Hoskins, 4 */
  double soil_depth_scale;
  double star_temperature_k;     /* 0: no stellar-spectrum albedo split */
  int storm_diagnostics;         /* NSTORMDIAG: storm-climatology fields each step (GcmConfig.stormclim) */
  double storm_ckcd;             /* CKCD, Ck/Cd; 0: 0.9 */
  double storm_vithresh;         /* VITHRESH, ventilation threshold; 0: 0.145 */
} exogcm_planet;

/* Boundary and initial fields on the Gaussian grid (NLAT x 2 NLAT points,
 * north first), as the reference's .sra inputs (setup/surface/index.ts). */
typedef struct exogcm_boundary {
  const double* land_mask;   /* code 172, NHOR values; required */
  const double* orography;   /* code 129 surface geopotential (m^2/s^2), NHOR; or NULL */
  const double* sst;         /* code 169, 1 or 12 monthly fields; or NULL */
  int sst_months;
  const double* ice_cover;   /* code 210, 1 or 12 monthly fields; or NULL */
  int ice_cover_months;
  const double* t_init;      /* initial temperature (K) [levels][NHOR]; required */
  const double* q_init;      /* initial specific humidity [levels][NHOR]; required */
} exogcm_boundary;

/* Message of the last failed call on this thread. */
int exogcm_last_error(char* buffer, size_t size);

/* Creates an engine of `slots` planet slots at T`truncation` L`levels` on
 * the current CUDA device (STEPPER.context, stepper/index.ts:94-118).
 * `mode` 0: the plain path (truncated-DFT longitude transforms and one thread
 * per Legendre output, as the reference's shaders); 1: the optimized path
 * (warp-shuffle FFTs, latitude-pair Legendre transforms on m-major Fourier
 * planes); 2: the optimized path with every Legendre transform (sp2fc,
 * sp2fcdmu, dv2uv, fc2sp, uv2dv/mktend, qtend) as tcgen05 tensor-core
 * contractions in split precision (3xTF32, FP32 accumulation; within 1e-5 of
 * FP64, about 3x a sequential-f32 sum's error). All compute in FP32 and share
 * the physics. */
int exogcm_create(int truncation, int levels, int slots, int mode, exogcm_engine** engine);
void exogcm_destroy(exogcm_engine* engine);

/* Set-up of one slot in FP64 and upload of its tables and initial state
 * (SETUP.state / SETUP.schedule, setup/index.ts:434-477; LAYOUT.write,
 * layout/index.ts:66-71). The slot then runs the reference's start-up steps
 * before its main loop. The heavy FP64 loops (the Legendre tables of the
 * engine's first planet, legendre/index.ts:29-136; the grid -> spectral
 * analysis of the orography and the initial temperature and humidity,
 * legendre/index.ts:334-361; makebm's LU inverses,
 * dynamics/setup/index.ts:154-239) run on the engine's device on a stream
 * of their own, beside batches already stepping, unless
 * exogcm_setup_on_device(engine, 0) moved them to the host; both give the
 * same numbers bit for bit. */
int exogcm_configure(exogcm_engine* engine, int slot, const exogcm_planet* planet,
                     const exogcm_boundary* boundary);

/* Chooses where exogcm_configure runs its heavy FP64 set-up loops: on the
 * engine's device (enable != 0, the default) or on the host. */
int exogcm_setup_on_device(exogcm_engine* engine, int enable);

/* Runs the FP64 set-up of exogcm_configure on the host only and returns one
 * of its arrays, with no device involved (a dry run of configure). `name`
 * is "state:<field>" (initial state, reference layout), "table:<name>"
 * (per-planet constant table; bm1 holds the four timestep phases),
 * "const:<NAME>" (one kernel constant), "shared:<q|fwd|inv|sines|weights>"
 * (resolution tables; q* are the filtered Legendre tables) or
 * "calendar:<step>" (that step's 16 host values: radiation_step[5],
 * surface_step[7], carbon flag, next carbon counter from 0, start step,
 * start-up steps). `*count` returns the array length; values may be NULL. */
int exogcm_setup_preview(const exogcm_planet* planet, const exogcm_boundary* boundary, const char* name,
                         double* values, size_t* count);

/* exogcm_setup_preview with the heavy FP64 loops on the current device, as
 * exogcm_configure runs them (needs a GPU). */
int exogcm_setup_preview_device(const exogcm_planet* planet, const exogcm_boundary* boundary, const char* name,
                                double* values, size_t* count);

/* Frees a slot for another planet (continuous batching). */
int exogcm_release(exogcm_engine* engine, int slot);

/* Runs `steps` model steps for every active slot (STEPPER.batch,
 * stepper/index.ts:203-276): per-step CPU values computed on the host,
 * uploaded once, then the whole batch as one CUDA graph. A slot whose step
 * number is a multiple of `publish_every` packs its snapshot on that step.
 * `steps` must not exceed `publish_every` so a slot publishes at most once.
 * Returns when the batch is done (exogcm_step_async + exogcm_wait). */
int exogcm_step(exogcm_engine* engine, int steps, int publish_every);

/* Submits the same batch and returns at once: the mapAsync-style pipelining
 * of the reference's worker, which keeps IN_FLIGHT = 2 batches submitted
 * (runner/webgpu/gcm.worker.ts:215-225, pump/submit :285-346). At most two
 * batches are in flight; a third call waits for the oldest. While batches
 * are in flight the engine accepts only exogcm_step_async, exogcm_poll,
 * exogcm_wait, exogcm_snapshots_begin, exogcm_slot_info and the query calls;
 * every other call first waits for them (exogcm_configure computes the new planet's host set-up
 * before it waits, so that work overlaps the device's). */
int exogcm_step_async(exogcm_engine* engine, int steps, int publish_every);

/* *done = 1 when no batch is in flight, else 0; never blocks. Retires
 * every finished batch (exogcm_last_step_ms then reports the latest), and
 * returns EXOGCM_EDEVICE if one of them reported a device fault. */
int exogcm_poll(exogcm_engine* engine, int* done);

/* Blocks until every submitted batch is done. */
int exogcm_wait(exogcm_engine* engine);

/* Steps several engines, of any resolutions, together: engine i runs
 * steps[i] model steps (each as exogcm_step would), all as ONE launch of a
 * CUDA graph whose nodes are the engines' captured batch graphs, so the
 * batches of a mixed-resolution ensemble (128 T21 L5 + 96 T42 L10 + 32 T63
 * L10 planets, say) run concurrently from one submission. Engines must be
 * distinct and on one device; the group graph is instantiated once per
 * (engines, steps) list and reused. Returns when every batch is done; *ms
 * (may be NULL) receives the device time of the launch. No counterpart in
 * the reference, whose worker steps one planet per device
 * (runner/webgpu/gcm.worker.ts:215-346). */
int exogcm_group_step(exogcm_engine** engines, int count, const int* steps, int publish_every, float* ms);

/* Per-planet global budgets in FP64, computed on the device on every step a
 * slot publishes (the quantities of the reference's yearly energy balance,
 * averages/index.ts:31-49 and balance/index.ts, plus the mass and water
 * budgets): Gaussian-weighted global means of [0] surface pressure (Pa, the
 * atmosphere's mass), [1] top-of-atmosphere net radiation (W/m^2), [2]
 * surface net heat flux (W/m^2), [3] surface temperature (K), [4]
 * precipitation (m/s), [5] evaporation (m/s), [6] column water vapour
 * (kg/m^2), [7] the weights' mean (1). `last` (8 doubles, may be NULL) gets
 * the last publishing step's values, `mean` (may be NULL) the mean over the
 * `*samples` publishing steps since configure or the last reset; `reset`
 * clears the means. */
int exogcm_budgets(exogcm_engine* engine, int slot, double* last, double* mean, long* samples, int reset);

/* Monthly means on the device (averages/index.ts:85-103 `add`/`close`):
 * with averages enabled, every publishing step adds the slot's snapshot
 * fields to FP64 running sums (snapshot planes x slots x NHOR doubles of
 * device memory). exogcm_averages_read returns, per slot, their mean over
 * the `*samples` publishing steps since the last reset as floats
 * [plane][point] (count = snapshot planes x NHOR; `mean` may be NULL), and
 * `reset` starts the next month. Enabling or disabling recaptures the
 * engine's batch graphs. */
int exogcm_averages_enable(exogcm_engine* engine, int enable);
int exogcm_averages_read(exogcm_engine* engine, int slot, float* mean, size_t count, long* samples, int reset);

/* Calendar date of model step `step` for a slot's planet (calendar/date/
 * index.ts:43-80; step < 0: the slot's current step): date[5] = year, month,
 * day, hour, minute. The date a snapshot or checkpoint carries
 * (types.ts GcmDate). */
int exogcm_slot_date(exogcm_engine* engine, int slot, long step, int* date);

/* Snapshot of a slot published during the last exogcm_step (the 101/76
 * fields of snapshot/index.ts, each NHOR values): returns the step it was
 * taken at in *step, or -1 when the slot did not publish. `values` may be
 * NULL to query only. */
int exogcm_read_snapshot(exogcm_engine* engine, int slot, float* values, size_t count, long* step);

/* Starts copying every slot's snapshot field, as the last submitted batch
 * (exogcm_step or exogcm_step_async) leaves it, into `values` (count =
 * snapshot planes x slots x NHOR floats, laid out [plane][slot][point] as on
 * the device) and returns at once without waiting for batches in flight:
 * the copy to the host runs on a stream of its own, from a device-side copy
 * queued on the engine's stream behind that batch, so the next batches
 * compute while it drains. Use
 * pinned host memory for `values` to get that overlap. Only slots that
 * published in that step hold a new snapshot (see exogcm_read_snapshot). A
 * second call waits for the first copy; exogcm_snapshots_wait waits for the
 * last one. There is no counterpart in the reference, whose worker maps one
 * staging buffer per snapshot (stepper/index.ts:254-265). */
int exogcm_snapshots_begin(exogcm_engine* engine, float* values, size_t count);
int exogcm_snapshots_wait(exogcm_engine* engine);

/* Stops a slot at model step `step`: later steps of a batch leave the slot
 * untouched (its kernels skip it), so a run ends exactly on its last step
 * whatever the batch length. A negative step removes the limit. */
int exogcm_set_stop(exogcm_engine* engine, int slot, long step);

/* Per-slot model step counter and start-up steps still to run. */
int exogcm_slot_info(exogcm_engine* engine, int slot, long* step, int* startup_left, int* active);

/* Field readback / write by the reference's state field names
 * (LAYOUT.read / LAYOUT.write), one slot at a time, f32. */
int exogcm_field_size(exogcm_engine* engine, const char* name, size_t* count);
int exogcm_read_field(exogcm_engine* engine, int slot, const char* name, float* values, size_t count);
int exogcm_write_field(exogcm_engine* engine, int slot, const char* name, const float* values, size_t count);

/* Per-slot constant table readback (f32 as the kernels read it). */
int exogcm_read_table(exogcm_engine* engine, int slot, const char* name, float* values, size_t count);

/* Checkpoint of one slot in the reference's restart format
 * (checkpoint/restart/index.ts:11-75: magic, JSON header with field names
 * and counts, step and carbon counter, then every field's f32 values).
 * Save returns a library-owned buffer released with exogcm_free. Load
 * rejects a checkpoint whose field list does not match (EXOGCM_ELAYOUT). */
int exogcm_checkpoint_save(exogcm_engine* engine, int slot, void** buffer, size_t* size);
int exogcm_checkpoint_load(exogcm_engine* engine, int slot, const void* buffer, size_t size);
void exogcm_free(void* buffer);

/* Per-slot instability flags (1 = non-finite state seen since the last
 * clear); the reference stops with "model became unstable at step N"
 * (runner/webgpu/gcm.worker.ts:317-323). */
int exogcm_unstable(exogcm_engine* engine, int* flags, int slots);

/* Runs one named stage of the step for every active slot at its current
 * step without advancing it: gridpointa, spectrala, physics_in, fixer,
 * surface_flux, radiation, precipitation, surface, carbon, physics_out,
 * spectrald, pack. For per-routine replay tests (the reference's
 * scripts/exoplasim-webgpu/verify-dynamics.mjs). */
int exogcm_run_stage(exogcm_engine* engine, const char* stage);

/* Device time of the last exogcm_step in milliseconds (CUDA events). */
int exogcm_last_step_ms(exogcm_engine* engine, float* ms);

/* Launches one of the step's kernels `reps` times on the current state of
 * every slot and returns its mean device time per launch in *ms (CUDA events
 * on the engine's stream), with the algorithmic bytes one launch moves in
 * *bytes. Kernels: "fourier_forward", "fourier_inverse" (FFTs on the
 * optimized path, DFTs on the plain one; "fourier_forward_per_chunk",
 * "fourier_forward_persistent" and the same for "fourier_inverse" run the
 * FFT in that form whatever the tuning chose), "legendre_forward",
 * "legendre_inverse", "sp2gp" (the fused inverse Legendre transform and FFT
 * of the optimized path; "sp2gp_planes2" and "sp2gp_planes4" run it at 2
 * or 4 planes per pass whatever the tuning chose), "dv2uv", "uv2dv", "qtend", "calcgp", "spectrala",
 * "mkdheat" (its first stage), "physics_in", "physics_out", and the single
 * column kernels "vdiff", "swr", "lwr_radstep", "kuo", "rain_column". The
 * launches change the state; use it for measurement only. */
int exogcm_time_kernel(exogcm_engine* engine, const char* kernel, int reps, float* ms, double* bytes);

/* Launch shapes the autotuner chose for the optimized path's transforms at
 * the engine's first configure (plain path: the defaults; an engine of a
 * shape - device, truncation, levels, slots, mode - the process tuned
 * before reuses that choice, as it reuses the shared FP64 tables of a
 * resolution): values[0] FFT
 * latitudes per block; [1], [2] sp2fc wavenumbers and planes per block;
 * [3], [4] the same for dv2uv; [5..8] forward Legendre planes per tile
 * for fc2sp, uv2dv, mktend's uv2dv and qtend; [9..12] (when count >= 13)
 * the staging buffers of those forward blocks (1 or 2); [13] (when count >=
 * 14) the planes per pass of the fused inverse transform (2 or 4); [14],
 * [15] (when count >= 16) 1 where the forward / inverse FFT runs as
 * persistent blocks looping over latitude chunks, 0 for one block per
 * chunk. `count` must be at least 9.
 * The shapes split work differently but leave every result unchanged. */
int exogcm_tuning(exogcm_engine* engine, int* values, int count);

/* Kernel launches in the CUDA graph of a `steps`-step batch. */
int exogcm_graph_launches(exogcm_engine* engine, int steps, size_t* launches);

/* Allocation-free per-slot FP64 sums (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory: a host embedded in another
 * framework's memory pool where cudaMalloc is not allowed, a runtime whose
 * device footprint is fixed after start-up, or code that must not trigger
 * the device synchronization cudaMalloc/cudaFree can cause. It computes what
 * the step's fixer and getiflx reductions compute: for each of `slots`
 * planets, the sums of `points` values of `first` and of `second`
 * (device arrays [slots][points], the layout exogcm_device_field gives for a
 * one-level grid field), in double precision with a fixed order, written as
 * floats to the device array `sums` [2][slots] (first sums, then second).
 * Every slot given is summed: unlike the step's reductions it does not skip
 * inactive or uncoupled slots.
 * It calls no allocator: its scratch is a static device array sized for at
 * most 256 slots (1 MiB, held on every GPU that loads the library until the
 * process exits); larger `slots` are rejected with EXOGCM_EINVAL. The first
 * call on a device looks up that array's device address, which also commits
 * the array to the device under CUDA's lazy module loading: a caller with a
 * fixed footprint makes that first call during its own start-up, and before
 * any stream capture. After a cudaDeviceReset, reload the library. Every
 * call shares the scratch and keeps the last call's contents; calls that
 * overlap on the GPU race. `stream` is a cudaStream_t (NULL: the legacy
 * default stream). */
int exogcm_slot_sums_noalloc(const float* first, const float* second, int slots, int points, float* sums,
                             void* stream);

/* Raw device pointer of a field (slot-major layout [plane][slot][points])
 * and the engine's CUDA stream, for in-process hosts that keep inputs
 * resident. */
int exogcm_device_field(exogcm_engine* engine, const char* name, void** pointer, size_t* floats);
void* exogcm_stream(exogcm_engine* engine);

/* ---------------------------------------------------------------- server
 * A batched server above the engine calls: continuous batching of many planet
 * runs on the current device. It has no counterpart in the reference, whose
 * page runs one planet per worker (runner/webgpu/gcm.worker.ts); it runs many
 * the way that worker runs one. Runs of one resolution share engines
 * ("blocks" of slots) created within one device-byte budget by their per-slot
 * footprint and destroyed when empty and another resolution needs the room;
 * each run stops exactly at its last step, so its result does not depend on
 * what else ran. One server is used from one host thread at a time. */
typedef struct exogcm_server exogcm_server;

typedef struct exogcm_server_options {
  double budget_bytes; /* device bytes the blocks' state may take */
  int block_slots;     /* slots of a T21 L5 block; fewer at larger resolutions, by footprint */
  int chunk_steps;     /* model steps per batch of a block (1..64) */
  int mode;            /* engine mode of every block (exogcm_create) */
} exogcm_server_options;

#define EXOGCM_REQUEST_QUEUED 0
#define EXOGCM_REQUEST_RUNNING 1
#define EXOGCM_REQUEST_FINISHED 2
#define EXOGCM_REQUEST_FAILED 3   /* unstable ("model became unstable"), or its set-up failed */
#define EXOGCM_REQUEST_REJECTED 4 /* one block of its resolution exceeds the budget */

int exogcm_server_create(const exogcm_server_options* options, exogcm_server** server);
void exogcm_server_destroy(exogcm_server* server);

/* Queues a run of `steps` main-loop model steps (after the start-up steps)
 * of a planet; the planet and its boundary arrays are copied. */
int exogcm_server_submit(exogcm_server* server, const exogcm_planet* planet, const exogcm_boundary* boundary,
                         long steps, long* request);

/* One scheduling round: submits a batch of chunk_steps for every block with
 * running runs (exogcm_step_async), admits queued runs into free slots or
 * new blocks while those batches run, waits for them and collects the runs
 * that finished or became unstable. `*active` returns the runs queued or
 * running (may be NULL). */
int exogcm_server_pump(exogcm_server* server, int* active);

/* A run's status (EXOGCM_REQUEST_*) and main-loop steps done. */
int exogcm_server_poll(exogcm_server* server, long request, int* status, long* steps_done);

/* A finished run's final spectral prognostic field ("st", "sz", "sd", "sq"
 * or "sp"; reference layout, `count` its exogcm_field_size). */
int exogcm_server_result(exogcm_server* server, long request, const char* field, float* values, size_t count);

/* Forgets a finished, failed or rejected run and its result. */
int exogcm_server_release(exogcm_server* server, long request);

#ifdef __cplusplus
}
#endif

#endif /* EXOGCM_H */
