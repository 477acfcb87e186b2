/*
 * tlm_b200.h -- C ABI of the B200-native SCN TLM time step.
 *
 * Drop-in replacement for the time loop behind smilima/EMSolver's
 * TlmSolver (TlmSolver.h:202-264, the IFieldSolver implementation at
 * TlmSolver.h:148-192). Every entry point below names the reference
 * interface it stands in for. Plain C types only: no CUDA or C++ types cross
 * this boundary, so cgo / JNI / ctypes / C++ can bind it directly.
 *
 * Conventions
 *  - Every call returns a tlm_status; TLM_OK is 0. On failure the handle's
 *    message (tlm_last_error) says why; failures before a handle exists go
 *    to the thread's message (tlm_last_error(NULL)).
 *  - The library owns all device state. Input arrays are copied during the
 *    call. Output arrays are caller-allocated with a stated capacity; the
 *    number of valid elements is written to *n_out.
 *  - A handle is not re-entrant: one thread drives it. tlm_request_stop,
 *    tlm_current_step, tlm_current_energy, tlm_is_running and
 *    tlm_is_finished may be called from any thread at any time, which is
 *    how the reference's UI polls a solver running on a worker thread
 *    (MainUnit.cpp:991, :1453).
 *  - There is no CPU fallback. If the CUDA device or the kernels are not
 *    usable the call fails with TLM_ENODEV / TLM_ECUDA.
 *
 * Cell indexing is the reference's VoxelGridSpec::cellIndex
 * (Geometry.h:91-94): cell = (k*ny + j)*nx + i. Link-pulse slots follow the
 * reference's portOf (TlmSolver.cpp:19-29): slot = axis*4 + side*2 + pol.
 */
#ifndef TLM_B200_H
#define TLM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TLM_API __attribute__((visibility("default")))
#else
#define TLM_API
#endif

typedef enum tlm_status {
    TLM_OK = 0,
    TLM_EINVAL = 1,    /* bad argument or inconsistent inputs */
    TLM_ENOMEM = 2,    /* HBM admission refused or allocation failed */
    TLM_ECUDA = 3,     /* CUDA runtime / kernel error */
    TLM_ETIMEOUT = 4,  /* a bounded device wait ran out */
    TLM_ESTOPPED = 5,  /* run ended early by tlm_request_stop */
    TLM_ESTATE = 6,    /* call not valid in the handle's current state */
    TLM_ENODEV = 7,    /* no usable CUDA device / kernels not loadable */
    TLM_EBUSY = 8      /* the handle is running on another thread */
} tlm_status;

/* Material ids of the map (TlmSolver.h:59): 0 air, 1 PEC, id >= 2 a
 * dielectric whose properties are table[id - 2]. */
enum { TLM_MAT_AIR = 0, TLM_MAT_PEC = 1, TLM_MAT_DIEL0 = 2 };

/* WaveformType (TlmSolver.h:70) plus TLM_WAVE_TABLE: per-step source values
 * supplied by tlm_set_source_table (the harness-side waveform hook). */
typedef enum tlm_waveform {
    TLM_WAVE_CW_RAMPED = 0,
    TLM_WAVE_GAUSSIAN_SINE = 1,
    TLM_WAVE_GAUSSIAN_PULSE = 2,
    TLM_WAVE_TABLE = 3
} tlm_waveform;

/* Pulse storage. Scatter arithmetic is FP32 for F32/BF16/F16/BFP16 and FP64
 * for F64 (the on-device FP64 oracle mode). BF16/F16 store pulse/scale.
 * BFP16 is block floating point at 16 bits per pulse: each aligned group of
 * 4 x-neighbours of one link plane shares an 8-bit exponent and keeps a
 * 14-bit signed mantissa per pulse (13 bits below the group maximum). */
typedef enum tlm_storage {
    TLM_STORE_F32 = 0,
    TLM_STORE_BF16 = 1,
    TLM_STORE_F16 = 2,
    TLM_STORE_F64 = 3,
    TLM_STORE_BFP16 = 4
} tlm_storage;

/* VoxelGridSpec (Geometry.h:85-113). */
typedef struct tlm_grid {
    int nx, ny, nz;
    float origin[3];
    float dl;
} tlm_grid;

/* MatProps (TlmSolver.h:61-65). */
typedef struct tlm_matprops {
    float epsr;
    float sigma;
} tlm_matprops;

/* TlmConfig (TlmSolver.h:113-123) and the B200 extensions after it. */
typedef struct tlm_config {
    float f0;            /* excitation / analysis frequency (Hz) */
    int waveform;        /* tlm_waveform */
    int total_steps;     /* tlm_run stops here */
    int settle_steps;    /* the Js and Huygens DFTs start at this step */
    float boundary_rho;  /* outer-face reflection coefficient */
    int huy_offset;      /* Huygens box inset in cells (>= 2 enables the box;
                            needs surface_monitors) */
    int use_gpu;         /* ignored: this library always runs on the GPU */
    int record_every;    /* record a playback frame every N steps (0 = off) */
    /* --- extensions --- */
    int storage;         /* tlm_storage */
    float pulse_scale;   /* BF16/F16 per-grid scale (0 = choose from sources) */
    int steps_per_launch;/* steps per monitor window; 0 = default (64) */
    int kernel_variant;  /* thread-tile shape of the step kernel; 0 = default
                            (tlm_kernel_variants lists the others) */
    int rounding;        /* 16-bit storage: 0 round to nearest, 1 stochastic */
    int general_tiles;   /* 1: every tile runs the general step body (no
                            interior-tile fast path); results are identical,
                            the switch exists to cross-check the two bodies */
    int surface_monitors;/* 1: record the reference's PEC-surface currents
                            (|Js| per face and its DFT at f0) and, with
                            huy_offset >= 2, the Huygens-box phasors that the
                            far field needs. One extra small launch per step;
                            not available for handles driven by a batch */
    int no_staging;      /* 1: FP32 interior tiles load their pulses directly
                            instead of through shared-memory stages filled by
                            bulk copies; results are identical */
    int stage_wait_us;   /* staged tiles: the consumers give up waiting for a
                            stage's bulk copies (the producer for a stage to
                            be released) after this many microseconds and the
                            step fails with TLM_ECUDA; 0 = default (about 2 s),
                            < 0 = at the first poll that finds the stage not
                            ready (exercises the error path). The producer
                            always lets the copies it issued land */
    int near_field;      /* FP16/BF16 storage: radius r in cells of the
                            near-field box, the bounding box of the PEC cells
                            and port cells grown by r (0 = none). Box cells
                            keep the FP32 residual of their stored pulses
                            beside them (4 B more per pulse, read and written
                            in the box only) and step as FP32 storage would;
                            the rest of the grid is stored in 16 bits. The box
                            is fixed when the first step (or tlm_set_pulses)
                            prepares the grid */
} tlm_config;

typedef struct tlm_solver *tlm_handle;

/* ---- lifetime ------------------------------------------------------- */

/* Version string of the library. */
TLM_API const char *tlm_version(void);

/* Fill *cfg with TlmConfig's defaults (TlmSolver.h:113-123). */
TLM_API void tlm_config_default(tlm_config *cfg);

/* Replaces `new TlmSolver()` (TlmSolver.cpp:245-250): binds a handle to a
 * CUDA device and creates its stream. */
TLM_API tlm_status tlm_create(tlm_handle *out, int device);

/* Replaces `delete solver` (TlmSolver.cpp:253-256). */
TLM_API tlm_status tlm_destroy(tlm_handle h);

/* Message of the last failure on h (NULL: of the calling thread). */
TLM_API const char *tlm_last_error(tlm_handle h);

/* ---- setup (TlmSolver::setup, TlmSolver.cpp:259-304) ---------------- */

/* Copies the material map (n_cells = nx*ny*nz bytes) and the dielectric
 * table, derives yhat = 4*(max(1,epsr)-1) and ghat = max(0,sigma)*dl*eta0
 * per table entry, zeroes all pulse state, clears ports/probes/sources and
 * allocates device memory (refused with TLM_ENOMEM if it would not fit).
 * Unlike the reference, a material id >= 2 without a table entry is
 * rejected (TLM_EINVAL) instead of reading past the table. */
TLM_API tlm_status tlm_setup(tlm_handle h, const tlm_grid *grid, const uint8_t *mat,
                             size_t n_cells, const tlm_matprops *table, int n_table,
                             const tlm_config *cfg);

/* TlmSolver::addPort (TlmSolver.cpp:362-374). Cells that are not air (or
 * out of range) are dropped silently, as in the reference. *out_idx gets
 * the port index. A port whose current loop (the 4 transverse linear-index
 * neighbours of its middle cell, TlmSolver.cpp:687-698) would read outside
 * the grid is refused with TLM_EINVAL; the reference reads out of bounds. */
TLM_API tlm_status tlm_add_port(tlm_handle h, const uint64_t *cells, int n_cells,
                                int pol_axis, float amp, int *out_idx);

/* TlmSolver::addPlaneWave (TlmSolver.cpp:394-407). */
TLM_API tlm_status tlm_add_plane_wave(tlm_handle h, int prop_axis, int plane_index,
                                      int pol_axis, float amp);

/* Append soft sources one cell at a time: the reference's SourceCell list
 * (TlmSolver.h:72-77, filled by addPlaneWave). For callers that hold that
 * list, e.g. a RunGpuTlm seam (GpuTlm.h:15). Non-air cells are dropped. */
TLM_API tlm_status tlm_add_source_cells(tlm_handle h, const uint64_t *cells, int n_cells,
                                        int pol_axis, float amp);

/* TlmSolver::addProbe (TlmSolver.cpp:377-391): *out_idx = -1 when the world
 * point is outside the grid (status TLM_OK, like the reference). */
TLM_API tlm_status tlm_add_probe(tlm_handle h, float x, float y, float z, int *out_idx);

/* Probe at a cell given by its indices (no world-position rounding). */
TLM_API tlm_status tlm_add_probe_cell(tlm_handle h, int i, int j, int k, int *out_idx);

/* Per-step source values for TLM_WAVE_TABLE (steps past the table get 0).
 * Stands in for TlmSolver::waveformValue (TlmSolver.cpp:410-436). */
TLM_API tlm_status tlm_set_source_table(tlm_handle h, const float *sv, int n_steps);

/* Frequencies (Hz) of the on-device FP64 running DFT of every port's V and
 * I records: V(f) = sum_n v[n] exp(-j 2 pi f n dt), the transform the
 * reference computes after the run from the float records
 * (SelfTest.cpp:182-195, MainUnit.cpp:1830-1846). Call before stepping. */
TLM_API tlm_status tlm_set_port_dft(tlm_handle h, const double *freqs_hz, int n_freq);

/* ---- time loop -------------------------------------------------------- */

/* Advance n_steps time steps (TlmSolver::step, TlmSolver.cpp:485-513, once
 * per step: inject, monitors, scatter, connect) and wait for the device. */
TLM_API tlm_status tlm_step(tlm_handle h, int n_steps);

/* Same, without waiting: the work is queued on the handle's stream.
 * Results are visible after tlm_sync (or any getter, which syncs). */
TLM_API tlm_status tlm_step_async(tlm_handle h, int n_steps);
TLM_API tlm_status tlm_sync(tlm_handle h);

/* TlmSolver::run (TlmSolver.cpp:439-464): steps from the current step to
 * total_steps, checking the stop flag between launch windows. Returns
 * TLM_ESTOPPED if tlm_request_stop ended it early; calling it again resumes
 * from the current step, as runCpu does. */
TLM_API tlm_status tlm_run(tlm_handle h);

/* TlmSolver::requestStop / currentStep / currentEnergy / isRunning /
 * isFinished / totalSteps / timestep (TlmSolver.h:219-234). Thread-safe. */
TLM_API tlm_status tlm_request_stop(tlm_handle h);
TLM_API int tlm_current_step(tlm_handle h);
TLM_API float tlm_current_energy(tlm_handle h);
TLM_API int tlm_is_running(tlm_handle h);
TLM_API int tlm_is_finished(tlm_handle h);
TLM_API int tlm_total_steps(tlm_handle h);
TLM_API tlm_status tlm_timestep(tlm_handle h, float *dt);
/* grid() (TlmSolver.h:171, 229): the grid given to tlm_setup. */
TLM_API tlm_status tlm_get_grid(tlm_handle h, tlm_grid *grid);

/* ---- results ------------------------------------------------------- */

TLM_API int tlm_probe_count(tlm_handle h);
/* TlmSolver::probe(i) (TlmSolver.h:260): the E series, one value per step. */
TLM_API tlm_status tlm_get_probe(tlm_handle h, int idx, float *ex, float *ey, float *ez,
                                 int cap, int *n_out);
TLM_API tlm_status tlm_get_probe_f64(tlm_handle h, int idx, double *ex, double *ey,
                                     double *ez, int cap, int *n_out);
TLM_API tlm_status tlm_get_probe_cell(tlm_handle h, int idx, uint64_t *cell);

TLM_API int tlm_port_count(tlm_handle h);
/* TlmSolver::ports()[i].vRec / iRec (TlmSolver.h:81-87). */
TLM_API tlm_status tlm_get_port(tlm_handle h, int idx, float *v, float *i, int cap,
                                int *n_out);
TLM_API tlm_status tlm_get_port_f64(tlm_handle h, int idx, double *v, double *i, int cap,
                                    int *n_out);
/* Gap cells kept by tlm_add_port (air cells only, in the caller's order). */
TLM_API tlm_status tlm_get_port_cells(tlm_handle h, int idx, uint64_t *cells, int cap,
                                      int *n_out);
/* FP64 running DFT of port idx at the tlm_set_port_dft frequencies. */
TLM_API tlm_status tlm_get_port_dft(tlm_handle h, int idx, double *v_re, double *v_im,
                                    double *i_re, double *i_im, int cap, int *n_out);

/* TlmSolver::getEnergyHistory (TlmSolver.cpp:793-799): sum of the squares
 * of all link pulses every 16 steps, accumulated in FP64. vals (float, as
 * the reference) and/or vals64 may be NULL. */
TLM_API tlm_status tlm_get_energy_history(tlm_handle h, int *steps, float *vals,
                                          double *vals64, int cap, int *n_out);

/* Incident pulses in the reference's AoS layout (cell*12 + slot), i.e. the
 * reference's V after the last completed step; float or double. */
TLM_API tlm_status tlm_get_pulses(tlm_handle h, float *out, size_t cap);
TLM_API tlm_status tlm_get_pulses_f64(tlm_handle h, double *out, size_t cap);
/* Overwrite the incident pulses (snapshot restore / test set-up). */
TLM_API tlm_status tlm_set_pulses(tlm_handle h, const float *in, size_t n);
/* Stub pulses (cell*3 + j; zeros when the grid has no dielectric). */
TLM_API tlm_status tlm_get_stubs(tlm_handle h, float *out, size_t cap);
/* Device copies of the material map and the yhat / ghat tables. */
TLM_API tlm_status tlm_get_materials(tlm_handle h, uint8_t *out, size_t cap);
TLM_API tlm_status tlm_get_tables(tlm_handle h, float *yhat, float *ghat, int cap,
                                  int *n_out);

/* TlmSolver::waveformValue (TlmSolver.cpp:410-436) for a grid of cell size
 * dl: the source value the step kernels inject at step n (FP32 modes).
 * Host-only; needs no device. */
TLM_API tlm_status tlm_waveform_value(int waveform, float f0, float dl, int n, float *out);

/* ---- known-answer tests run on the device --------------------------- */

/* TlmSolver::ScatterUnitarityError / DielScatterUnitarityError
 * (TlmSolver.cpp:116-169), evaluated with the device scatter functions. */
TLM_API tlm_status tlm_scatter_unitarity_error(int device, float *err);
TLM_API tlm_status tlm_stub_unitarity_error(int device, float epsr, float *err);

/* ---- batched execution of many grids -------------------------------- */

/* No single counterpart in the reference, whose UI runs one TlmSolver at a
 * time (MainUnit.cpp:872-991). A batch advances many handles -- each set up
 * as usual with tlm_setup / tlm_add_port / tlm_add_probe ... -- with one
 * kernel launch per step for all of them (per storage mode and tile shape),
 * in windows of steps_per_launch steps captured as CUDA graphs. Each member
 * runs from its current step to its own total_steps and stops there. While
 * attached, a handle is stepped only by its batch (tlm_step/tlm_run on it
 * return TLM_ESTATE); its results are read with the ordinary getters and are
 * bitwise those it would get stepped alone. */
typedef struct tlm_batch_s *tlm_batch;

typedef struct tlm_batch_tuning {
    int kernel_variant;    /* step-kernel tile shape (see tlm_kernel_variants) */
    int steps_per_launch;  /* steps per window (graph) */
    int blocks_per_sm;     /* resident step-kernel blocks per SM, 0 = all that fit */
    int use_graphs;        /* 1: replay windows as CUDA graphs */
    int overlap;           /* 1: an FP32 group's general tiles (wire, port, probes,
                              partial tiles) step on a second stream, one block
                              per SM, beside its staged tiles; 0: before them.
                              Measured on B200: equal or up to 8 % faster for a
                              batch of one 192^3 grid, whose general tiles are
                              few; 1.24 -> 1.63 ms per step for the batched
                              dipoles, whose wire tiles are 11 % */
    double ms_per_step;    /* autotuner: measured time per step of the batch */
} tlm_batch_tuning;

TLM_API tlm_status tlm_batch_create(tlm_batch *out, int device);
/* Detaches every member (the handles stay valid) and frees the batch. */
TLM_API tlm_status tlm_batch_destroy(tlm_batch b);
TLM_API tlm_status tlm_batch_attach(tlm_batch b, tlm_handle h);
TLM_API tlm_status tlm_batch_detach(tlm_batch b, tlm_handle h);
/* Attached handles, and those not yet at their total_steps. */
TLM_API int tlm_batch_size(tlm_batch b);
TLM_API int tlm_batch_active(tlm_batch b);
/* Advance every member by up to n_steps (none past its total_steps) and
 * wait for the device. */
TLM_API tlm_status tlm_batch_step(tlm_batch b, int n_steps);
/* Advance until every member has reached its total_steps. */
TLM_API tlm_status tlm_batch_run(tlm_batch b);
/* Queue one window (steps_per_launch steps) without waiting, so the caller
 * can prepare new members while the GPU works; *n_steps gets the window
 * length (0 when no member is active). Follow with tlm_batch_sync before
 * attaching, detaching or reading members. */
TLM_API tlm_status tlm_batch_launch_window(tlm_batch b, int *n_steps);
TLM_API tlm_status tlm_batch_sync(tlm_batch b);
TLM_API tlm_status tlm_batch_set_tuning(tlm_batch b, const tlm_batch_tuning *t);
TLM_API tlm_status tlm_batch_get_tuning(tlm_batch b, tlm_batch_tuning *t);
/* Time trial_windows windows of 100 steps of every tile shape (then, for
 * the best shape, the general tiles beside the staged ones instead of before
 * them, and windows of 50 and 200 steps) on the batch's own members, keep
 * the fastest, and rewind every member to step 0 (fields zero). Call before the
 * first step. Results are cached per (GPU, storage modes, size class), in
 * the file named by TLM_AUTOTUNE_CACHE when that variable is set. */
TLM_API tlm_status tlm_batch_autotune(tlm_batch b, int trial_windows, tlm_batch_tuning *out);
TLM_API tlm_status tlm_batch_get_stream(tlm_batch b, void **stream);

/* ---- continuous-batching request server ------------------------------ */

/* No counterpart in the reference (a desktop application running one solve
 * at a time). Requests are complete solves; a worker thread admits queued
 * requests (by default the least work -- padded cells x steps -- first)
 * while their device footprint fits the HBM budget and the running cells
 * stay within a cap that keeps the GPU saturated, keeps their state resident
 * on the GPU, advances all running requests together in a batch one window
 * at a time, and retires each at its total_steps. Requests that arrive while
 * others run join the batch at the next window. Each result equals the same
 * solve run alone with tlm_setup/tlm_run. */
typedef struct tlm_server_s *tlm_server;

enum { TLM_REQ_QUEUED = 0, TLM_REQ_RUNNING = 1, TLM_REQ_DONE = 2, TLM_REQ_FAILED = 3,
       TLM_REQ_CANCELLED = 4 };

typedef struct tlm_request {
    tlm_grid grid;
    const uint8_t *mat;             /* n_cells = nx*ny*nz material ids */
    size_t n_cells;
    const tlm_matprops *table;      /* n_table dielectric entries */
    int n_table;
    tlm_config cfg;                 /* waveform, total_steps, rho, storage ... */
    const float *source_table;      /* for TLM_WAVE_TABLE, n_source values */
    int n_source;
    int n_ports;                    /* ports: cells concatenated, count per port */
    const uint64_t *port_cells;
    const int *port_ncells;
    const int *port_pol;
    const float *port_amp;
    int n_probes;                   /* probes: i,j,k per probe */
    const int *probe_ijk;
    int n_freq;                     /* port DFT frequencies (Hz) */
    const double *freqs;
} tlm_request;

typedef struct tlm_server_stats_t {
    long long completed, failed, cancelled, queued, running;
    double latency_p50_s, latency_p99_s, latency_mean_s;  /* submit -> done */
    double solves_per_s;            /* completed / (last completion - start) */
    size_t hbm_used_bytes, hbm_budget_bytes;
    long long windows;
    double busy_s;                  /* time spent stepping */
    double gpu_window_s;            /* device time of the windows (events) */
    double setup_s, retire_s;       /* host set-up of admitted requests (during
                                       windows) / read-out and release of
                                       finished ones (between windows) */
    double mean_running_cells;      /* padded cells running, mean over windows */
} tlm_server_stats_t;

/* hbm_budget_bytes 0 = 80% of the device's free memory; steps_per_launch 0
 * = 64 (the admission / retirement granularity). */
TLM_API tlm_status tlm_server_create(tlm_server *out, int device, size_t hbm_budget_bytes,
                                     int steps_per_launch);
/* Admission order: TLM_SERVE_LEAST_WORK (default: the queued request with
 * the fewest padded cells x steps first, so short solves are not held up
 * behind long ones) or TLM_SERVE_ARRIVAL (first come, first served);
 * max_running_cells caps the padded cells of the running requests (0 = no
 * cap; default 8 Mi), above which queued requests wait rather than slow
 * every running one down. The first request always runs. Requests of
 * solo_cells padded cells or more (0 = none; default 1 Mi) do not join the
 * batch: large grids fill the GPU alone, so they are stepped window by
 * window on their own stream by the single-grid kernels, beside the batch. */
enum { TLM_SERVE_ARRIVAL = 0, TLM_SERVE_LEAST_WORK = 1 };
TLM_API tlm_status tlm_server_set_policy(tlm_server s, int order, long long max_running_cells,
                                         long long solo_cells);
/* Stops the worker; queued and running requests end CANCELLED. */
TLM_API tlm_status tlm_server_destroy(tlm_server s);
/* Copies the request and queues it; TLM_ENOMEM if it can never fit. */
TLM_API tlm_status tlm_server_submit(tlm_server s, const tlm_request *req, uint64_t *id);
TLM_API tlm_status tlm_server_poll(tlm_server s, uint64_t id, int *state);
/* Wait until the request ends (timeout_s < 0: no limit); TLM_ETIMEOUT if it
 * has not ended in time. */
TLM_API tlm_status tlm_server_wait(tlm_server s, uint64_t id, double timeout_s, int *state);
TLM_API tlm_status tlm_server_cancel(tlm_server s, uint64_t id);
/* FP64 DFT of a finished request's port (and its latency). */
TLM_API tlm_status tlm_server_result(tlm_server s, uint64_t id, int port, double *v_re,
                                     double *v_im, double *i_re, double *i_im, int cap,
                                     int *n_freq, double *latency_s);
TLM_API tlm_status tlm_server_port_records(tlm_server s, uint64_t id, int port, float *v,
                                           float *i, int cap, int *n_out);
/* Forget a finished request (frees its results). */
TLM_API tlm_status tlm_server_release(tlm_server s, uint64_t id);
TLM_API tlm_status tlm_server_stats(tlm_server s, tlm_server_stats_t *out);
/* Device bytes a request holds while it runs (what admission counts). */
TLM_API tlm_status tlm_request_footprint(const tlm_request *req, size_t *bytes);

/* ---- surface monitors, cut plane, frames, far field ----------------- */

/* TlmSolver::faces() (TlmSolver.h:237; built by BuildPecSurfaceFaces,
 * Geometry.cpp:402-436): faces between a PEC cell and a non-PEC neighbour, in
 * the reference's order. Per face: the neighbour's linear cell index, the
 * normal axis, the side (+1: the neighbour is on the + side) and the face
 * centre (3 floats). Any output may be NULL; *n = face count. Empty unless
 * tlm_config.surface_monitors = 1. */
TLM_API tlm_status tlm_get_surface_faces(tlm_handle h, uint64_t *air_cells, int *axis, int *sign,
                                         float *centers, int cap, int *n);
/* getJsInstant (TlmSolver.cpp:926-930): |Js| per face at the last step. */
TLM_API tlm_status tlm_get_js_instant(tlm_handle h, float *out, int cap, int *n);
/* getJsDft after finalizeDft (TlmSolver.cpp:467-481, 950-957): per face
 * 2/samples * |(Re1, Im1, Re2, Im2)| of the DFT at f0 over the steps from
 * settle_steps on; re/im (2 per face) are the raw accumulators (jsDftRe/Im).
 * Any output may be NULL. */
TLM_API tlm_status tlm_get_js_dft(tlm_handle h, float *magnitude, float *re, float *im, int cap, int *n,
                                  int *samples);
/* The Huygens box (TlmSolver::buildHuygens, TlmSolver.cpp:310-348): air cells
 * inset huy_offset cells, per face the cell, normal axis, outward sign and
 * position relative to the domain centre (3 floats). */
TLM_API tlm_status tlm_get_huygens_faces(tlm_handle h, uint64_t *cells, int *axis, int *out_sign, float *pos,
                                         int cap, int *n);
/* The Huygens phasors (huyDft, TlmSolver.cpp:652-675): 8 floats per face,
 * E1 re/im, E2 re/im, eta0*H1 re/im, eta0*H2 re/im. */
TLM_API tlm_status tlm_get_huygens_dft(tlm_handle h, float *acc8, int cap, int *n, int *samples);
/* setFieldPlane (TlmSolver.cpp:961-966): |E| over the plane normal to axis
 * (-1 = off) at index, computed every second step. Between steps only. */
TLM_API tlm_status tlm_set_field_plane(tlm_handle h, int axis, int index);
/* getFieldPlane (TlmSolver.cpp:969-982): n1 x n2 floats (n1 along the first
 * remaining axis); TLM_ESTATE if no plane has been computed. */
TLM_API tlm_status tlm_get_field_plane(tlm_handle h, float *out, size_t cap, int *axis, int *index, int *n1,
                                       int *n2);
/* frameCount / getFrame (TlmSolver.cpp:933-947): one frame every
 * record_every steps with |Js| per face and the latest cut plane (if any). */
TLM_API tlm_status tlm_frame_count(tlm_handle h, int *n);
TLM_API tlm_status tlm_get_frame(tlm_handle h, int idx, int *step, float *js, int js_cap, float *plane,
                                 size_t plane_cap, int *axis, int *index, int *n1, int *n2);
/* computeFarField (ComputeFarFieldFromHuygens, TlmSolver.cpp:805-916): the
 * radiation intensity U over n_theta x n_phi directions (theta 0..pi, phi
 * 0..2pi inclusive, U may be NULL), its maximum, the directivity and the
 * peak direction, from the Huygens phasors at f0. Sums run in FP64 on the
 * device, so U agrees with the reference's FP32 sums to their rounding, not
 * bitwise. TLM_ESTATE without Huygens data. */
TLM_API tlm_status tlm_compute_far_field(tlm_handle h, int n_theta, int n_phi, float *U, float *u_max,
                                         float *directivity, float *peak_theta_deg, float *peak_phi_deg);

/* ---- one grid split into z-slabs over several solvers ------------------ */

/* No single counterpart in the reference: its z-slab worker threads
 * (TlmSolver.cpp:174-240, 516-613) split one grid in one address space;
 * here each slab is its own solver (one per GPU) and the slabs trade the
 * z-directed link pulses that cross their shared faces once per step.
 *
 * A slab's handle is set up on its planes plus one ghost plane on each side
 * that has a neighbouring slab (the neighbour's boundary plane, with its true
 * material), then tlm_set_slab(h, ghost_lo, ghost_hi) before the first step.
 * Ghost planes are stepped but excluded from the energy; probes and ports
 * (with their current loops) must lie in the slab's own planes (TLM_EINVAL at
 * the first step otherwise); sources may lie anywhere, since only the owning
 * slab's copy of a plane reaches the results. Not with surface monitors,
 * frames or batches; F16/BF16 need an explicit pulse_scale shared by all
 * slabs. Between two tlm_step_async(h, 1) calls, exchange:
 *   tlm_halo_pack(h, send_lo, send_hi)     this slab's first and last own
 *                                          planes' outgoing z pulses,
 *   send_lo to the slab below / send_hi to the slab above, receive theirs,
 *   tlm_halo_unpack(h, recv_lo, recv_hi)   into the ghost planes.
 * Buffers are device memory of tlm_halo_bytes each (NULL on a side without
 * a ghost plane); copies are queued on the handle's stream (tlm_get_stream).
 * Stepped this way every pulse of the own planes, every probe and port
 * record is bitwise what the undivided grid gives; energies add up. */
TLM_API tlm_status tlm_set_slab(tlm_handle h, int ghost_lo, int ghost_hi);
TLM_API tlm_status tlm_halo_bytes(tlm_handle h, size_t *bytes);
TLM_API tlm_status tlm_halo_pack(tlm_handle h, void *send_lo, void *send_hi);
TLM_API tlm_status tlm_halo_unpack(tlm_handle h, const void *recv_lo, const void *recv_hi);
/* The same exchange overlapped with the step, in two calls per step:
 *   tlm_slab_step_begin(h, send_lo, send_hi)   steps the tiles of the own
 *       planes next to a ghost plane, then packs their outgoing halo on the
 *       halo stream (tlm_get_halo_stream);
 *   the caller trades the messages on the halo stream (NCCL send/recv);
 *   tlm_slab_step_end(h, recv_lo, recv_hi)     unpacks the received halo on
 *       the halo stream while the other own planes step on the handle's
 *       stream; the next step waits for the unpack.
 * Ghost planes are not stepped. Steps are grouped into the handle's launch
 * windows (records, DFT and energy once per window); tlm_slab_flush closes
 * a partial window and must precede any other stepping of the handle or
 * reading its records. Results are bitwise those of tlm_step with
 * tlm_halo_pack/unpack, and of the undivided grid. */
TLM_API tlm_status tlm_slab_step_begin(tlm_handle h, void *send_lo, void *send_hi);
TLM_API tlm_status tlm_slab_step_end(tlm_handle h, const void *recv_lo, const void *recv_hi);
TLM_API tlm_status tlm_slab_flush(tlm_handle h);
TLM_API tlm_status tlm_get_halo_stream(tlm_handle h, void **stream);

/* ---- one step over caller-owned device memory, no allocation -------- */

/* No counterpart in the reference. For callers that may not allocate device
 * memory: a host application that reserves the GPU's memory in its own pool
 * and hands this library only buffers it owns, or a time-critical loop that
 * must not pay the device-wide synchronisation cudaMalloc/cudaFree can
 * cause. It advances one FP32 step over planes the caller owns and calls no
 * cudaMalloc, cudaFree or other allocating routine.
 *
 * Layout (all pointers are device pointers): px = nx rounded up to a
 * multiple of 8, P = px*ny*nz; plane s (0..11, slot axis*4 + side*2 + pol)
 * starts at element s*P; node (i,j,k) is element (k*ny + j)*px + i.
 * mat has P bytes, padding columns (i >= nx) must be TLM_MAT_PEC and their
 * pulses zero. in_planes holds the reflected pulses of the previous step
 * (or, with input_is_incident != 0, incident pulses such as the reference's
 * V re-laid out); out_planes (12*P floats, not aliasing in_planes) receives
 * the reflected pulses of this step: pass it as in_planes of the next call.
 * stubs: 3 planes read and written on dielectric nodes. yhat/ghat: n_diel
 * entries, one per dielectric id (id - 2); with n_diel > 0 stubs, yhat and
 * ghat must all be given (else TLM_EINVAL), with n_diel = 0 they may be NULL.
 * The tables are copied into a static table of all 254 dielectric ids whose
 * entries past n_diel are NaN: a node whose id is 2 + n_diel or more steps to
 * NaN pulses, and nothing past the caller's buffers is read. No sources or
 * monitors.
 * energy_out (NULL to skip): the FP64 sum of the squares of all incident
 * link pulses of this step. Planes 16-byte aligned, mat 4-byte aligned.
 * Work is queued on `stream` (a cudaStream_t, NULL = default stream).
 *
 * Limits and sharing: its only scratch, one FP64 energy partial per thread
 * block and the padded dielectric table, is a fixed 514 KiB of static device
 * arrays that every GPU loading this library holds until the process exits;
 * grids above 67,108,864 padded nodes are rejected with TLM_EINVAL. The
 * first call on a device looks up those arrays' device addresses
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call shares the arrays, so calls that overlap on the GPU (other
 * streams, other threads) race: serialise them. Each call rewrites the table
 * and the partials it uses; nothing needs clearing. The bounds-checked build
 * of the library (libtlm_b200_checked.so) waits for the step and returns
 * TLM_ECUDA if any index fell outside its buffer.
 * Errors: status code, message in tlm_last_error(NULL). */
TLM_API tlm_status tlm_step_planes_noalloc(const float *in_planes, float *out_planes,
                                           float *stubs, const uint8_t *mat, const float *yhat,
                                           const float *ghat, int n_diel, int nx, int ny, int nz,
                                           float rho, int input_is_incident, double *energy_out,
                                           void *stream);

/* ---- bench / integration helpers ------------------------------------ */

/* Number of step-kernel tile shapes for a storage mode (valid values of
 * tlm_config.kernel_variant are 0 .. n-1) and, for one of them, the nodes
 * per thread and the minimum resident blocks per SM it is compiled for. */
TLM_API int tlm_kernel_variants(int storage);
TLM_API tlm_status tlm_kernel_variant_info(int storage, int variant, int *nodes_per_thread,
                                           int *min_blocks_per_sm);

/* The near-field box (tlm_config.near_field) fixed when the grid was
 * prepared: box[0..2] its first cell (i, j, k), box[3..5] its extent in
 * cells; all zero when the handle has none (or is not prepared yet). */
TLM_API tlm_status tlm_near_field_box(tlm_handle h, int box[6]);

/* The handle's CUDA stream (cudaStream_t) for event timing by the caller. */
TLM_API tlm_status tlm_get_stream(tlm_handle h, void **stream);
/* Bytes of device memory the handle holds. */
TLM_API tlm_status tlm_device_bytes(tlm_handle h, size_t *bytes);
/* Kernel timing: when enabled, the kernels of every step are bracketed by
 * CUDA events on the handle's stream; tlm_kernel_time returns the summed
 * duration and the number of timed steps since the last enable. */
TLM_API tlm_status tlm_set_kernel_timing(tlm_handle h, int enable);
TLM_API tlm_status tlm_kernel_time(tlm_handle h, double *ms, long long *launches);
/* Kernels one step launches (the FP32 step of large grids runs its staged
 * interior tiles and the remaining tiles as two kernels; surface monitors add
 * one); the window epilogue every steps_per_launch steps is not counted. */
TLM_API tlm_status tlm_step_launches(tlm_handle h, int *per_step);

#ifdef __cplusplus
}
#endif

#endif /* TLM_B200_H */
