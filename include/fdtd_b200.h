/* fdtd_b200.h -- C ABI of the B200 Yee FDTD solver, the second time-domain
 * solver behind the reference's IFieldSolver interface (FdtdSolver.h).
 *
 * Same conventions as tlm_b200.h: plain C types, int status codes
 * (tlm_status) with a per-handle message, caller-owned inputs copied at
 * setup, caller-allocated outputs with capacities, device state owned by the
 * library, no CPU fallback. Grids, materials and the configuration use the
 * TLM types (the reference shares them: FdtdSolver::setup takes the same
 * VoxelGridSpec, MatProps and TlmConfig).
 *
 * Fields live in the reference's Yee layouts (FdtdSolver.h:63-86):
 *   Ex[nx][ny+1][nz+1], Ey[nx+1][ny][nz+1], Ez[nx+1][ny+1][nz],
 *   Hx[nx+1][ny][nz],   Hy[nx][ny+1][nz],   Hz[nx][ny][nz+1]
 * (x fastest), FP32. With the same inputs every field value, record and
 * surface monitor is bitwise the reference's CPU solver; the energy history
 * is an FP64 sum in another order (relative 1e-6). */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include "tlm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdtd_solver *fdtd_handle;

/* Replaces `new FdtdSolver()` (FdtdSolver.cpp:25-31). */
TLM_API tlm_status fdtd_create(fdtd_handle *out, int device);
TLM_API tlm_status fdtd_destroy(fdtd_handle h);
TLM_API const char *fdtd_last_error(fdtd_handle h);

/* FdtdSolver::setup (FdtdSolver.cpp:81-132): dt = 0.99 dl / (c0 sqrt 3),
 * per-edge PEC masks and lossy-dielectric coefficients averaged over the 4
 * cells around each edge, Mur boundary. Uses cfg->f0, waveform,
 * total_steps, settle_steps, huy_offset, record_every, surface_monitors
 * (1: PEC-surface currents and, with huy_offset >= 2, the Huygens box). */
TLM_API tlm_status fdtd_setup(fdtd_handle h, const tlm_grid *grid, const uint8_t *mat, size_t n_cells,
                              const tlm_matprops *table, int n_table, const tlm_config *cfg);
/* addPort (FdtdSolver.cpp:282-295): gap cells (non-air dropped) carrying a
 * soft E source on their 4 pol-axis edges; V = -sum E dl, I by the Ampere
 * loop around the middle cell. Refused (TLM_EINVAL) if that loop leaves the
 * grid (the reference reads out of bounds there). */
TLM_API tlm_status fdtd_add_port(fdtd_handle h, const uint64_t *cells, int n_cells, int pol_axis, float amp,
                                 int *idx);
/* addPlaneWave (FdtdSolver.cpp:315-329). */
TLM_API tlm_status fdtd_add_plane_wave(fdtd_handle h, int prop_axis, int plane_index, int pol_axis, float amp);
/* addProbe (FdtdSolver.cpp:298-312): cell-centred E at a world point;
 * *idx = -1 outside the grid. */
TLM_API tlm_status fdtd_add_probe(fdtd_handle h, float x, float y, float z, int *idx);
/* Per-step source values in place of the configured waveform. */
TLM_API tlm_status fdtd_set_source_table(fdtd_handle h, const float *values, int n);

/* FdtdSolver::step (FdtdSolver.cpp:401-446) n times: inject, monitors,
 * H update, E update with Mur boundaries. */
TLM_API tlm_status fdtd_step(fdtd_handle h, int n_steps);
/* run (FdtdSolver.cpp:361-380): steps up to total_steps. */
TLM_API tlm_status fdtd_run(fdtd_handle h);
TLM_API int fdtd_current_step(fdtd_handle h);
/* The CUDA stream (cudaStream_t) the handle's work is queued on. */
TLM_API tlm_status fdtd_get_stream(fdtd_handle h, void **stream);
TLM_API float fdtd_timestep(fdtd_handle h);
/* The grid given to fdtd_setup. */
TLM_API tlm_status fdtd_get_grid(fdtd_handle h, tlm_grid *grid);

/* Field component `which` (0..5 = Ex Ey Ez Hx Hy Hz) in its Yee layout;
 * *n = its length. */
TLM_API tlm_status fdtd_get_field(fdtd_handle h, int which, float *out, size_t cap, size_t *n);
/* Probe and port records (FieldProbe / TlmPort, TlmSolver.h:81-141). */
TLM_API tlm_status fdtd_get_probe(fdtd_handle h, int idx, float *ex, float *ey, float *ez, int cap, int *n);
TLM_API tlm_status fdtd_get_port(fdtd_handle h, int idx, float *v, float *i, int cap, int *n);
/* getEnergyHistory (FdtdSolver.cpp:947-952): sum E^2 + eta0^2 sum H^2 every
 * 16 steps (FP64 sum; vals as float, vals64 as double, either may be NULL). */
TLM_API tlm_status fdtd_get_energy_history(fdtd_handle h, int *steps, float *vals, double *vals64, int cap,
                                           int *n);

/* Surface monitors, cut plane, frames, far field: the same meaning as the
 * tlm_* functions of the same names (TlmSolver.h:237-245 and
 * FdtdSolver.cpp:673-881: Js from eta0*H at the face cell, Huygens from the
 * cell-centred E and eta0*H, plane |E| times dl, PEC cells included). */
TLM_API tlm_status fdtd_get_surface_faces(fdtd_handle h, uint64_t *air_cells, int *axis, int *sign,
                                          float *centers, int cap, int *n);
TLM_API tlm_status fdtd_get_js_instant(fdtd_handle h, float *out, int cap, int *n);
TLM_API tlm_status fdtd_get_js_dft(fdtd_handle h, float *magnitude, float *re, float *im, int cap, int *n,
                                   int *samples);
TLM_API tlm_status fdtd_get_huygens_faces(fdtd_handle h, uint64_t *cells, int *axis, int *out_sign, float *pos,
                                          int cap, int *n);
TLM_API tlm_status fdtd_get_huygens_dft(fdtd_handle h, float *acc8, int cap, int *n, int *samples);
TLM_API tlm_status fdtd_set_field_plane(fdtd_handle h, int axis, int index);
TLM_API tlm_status fdtd_get_field_plane(fdtd_handle h, float *out, size_t cap, int *axis, int *index, int *n1,
                                        int *n2);
TLM_API tlm_status fdtd_frame_count(fdtd_handle h, int *n);
TLM_API tlm_status fdtd_get_frame(fdtd_handle h, int idx, int *step, float *js, int js_cap, float *plane,
                                  size_t plane_cap, int *axis, int *index, int *n1, int *n2);
TLM_API tlm_status fdtd_compute_far_field(fdtd_handle h, int n_theta, int n_phi, float *U, float *u_max,
                                          float *directivity, float *peak_theta_deg, float *peak_phi_deg);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_B200_H */
