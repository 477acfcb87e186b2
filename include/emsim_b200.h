/* emsim_b200.h -- C ABI of the .emsim project file: the reference's on-disk
 * format for a simulation's settings, scene, displayed results, plots and
 * recorded playback (ProjectIO.h / ProjectIO.cpp, format version 2).
 *
 * A document (emsim_doc) holds one project in memory. emsim_load reads any
 * version 1 or 2 file the reference writes and emsim_save writes version 2
 * files the reference's LoadProject reads; a loaded document saves back to
 * the same bytes. emsim_from_tlm / emsim_from_fdtd fill a document's result
 * and playback sections from a solver handle the way the reference's main
 * window does before saving, so served results and recorded frames can be
 * opened in the reference application.
 *
 * Conventions: tlm_status codes (tlm_b200.h) with a per-document message
 * (emsim_last_error). Getters return views (pointers into the document)
 * that stay valid until the document is changed or freed; setters copy the
 * caller's arrays. Vectors are 3 floats (x, y, z). */
#ifndef EMSIM_B200_H
#define EMSIM_B200_H

#include "tlm_b200.h"
#include "fdtd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct emsim_doc emsim_doc;

/* SurfaceFace (Geometry.h:141-147). */
typedef struct emsim_face {
    int32_t air_cell;   /* linear index of the non-PEC cell beside the face */
    float center[3];    /* world position of the face centre */
    int8_t axis;        /* normal axis 0..2 */
    int8_t sign;        /* +1: the air cell is on the + side */
} emsim_face;

/* Toolbar state of ProjectData (ProjectIO.h:48-52). */
typedef struct emsim_toolbar {
    int solver, excitation, waveform, currents, db_range;
    int gpu, show_model, db_scale, plane_on, mesh_on;  /* stored as bytes */
} emsim_toolbar;

/* ProjObject (ProjectIO.h:16-28); parameters through emsim_*_object_param. */
typedef struct emsim_object {
    int kind;
    const char *name;
    float position[3], rot_deg[3];
    int dielectric;
    float epsr, sigma;
    double design_freq_hz;
    int is_stl;
    uint32_t n_stl_verts;     /* floats (3 per vertex) */
    const float *stl_verts;
    uint32_t n_stl_idx;
    const int32_t *stl_idx;
    uint32_t n_params;        /* getter only */
} emsim_object;

/* FarFieldData (TlmSolver.h:103-110). */
typedef struct emsim_pattern {
    int n_theta, n_phi;
    uint32_t n_u;
    const float *U;
    float u_max, directivity, peak_theta_deg, peak_phi_deg;
} emsim_pattern;

/* GLResult (GLView.h:15-36): the displayed result snapshot. */
typedef struct emsim_result {
    uint32_t n_faces;
    const emsim_face *faces;
    uint32_t n_face_vals;
    const float *face_vals;
    float face_dl;
    uint32_t n_tri_v;           /* vectors */
    const float *tri_v;
    uint32_t n_tri_idx;
    const int32_t *tri_idx;
    uint32_t n_tri_mag;
    const float *tri_mag;
    uint32_t n_wire_pts;        /* vectors */
    const float *wire_pts;
    uint32_t n_wire_mag;
    const float *wire_mag;
    int has_plane;
    tlm_grid plane_grid;
    int plane_axis, plane_index, plane_n1, plane_n2;
    uint32_t n_plane_vals;
    const float *plane_vals;
    int has_pattern;
    emsim_pattern pattern;
    float pat_center[3];
    float pat_scale;
    float domain_lo[3], domain_hi[3];
    int domain_visible;
    uint32_t n_probe_markers;   /* vectors */
    const float *probe_markers;
} emsim_result;

/* ProjCurve (ProjectIO.h:31). */
typedef struct emsim_curve {
    const char *name;
    uint32_t color;
    uint32_t n_x;
    const double *x;
    uint32_t n_y;
    const double *y;
} emsim_curve;

/* VizFrame (TlmSolver.h:126-132). */
typedef struct emsim_frame {
    int step;
    int plane_axis, plane_index, plane_n1, plane_n2;
    uint32_t n_js;
    const float *js;
    uint32_t n_plane;
    const float *plane;
} emsim_frame;

/* Empty project (ProjectData defaults). */
TLM_API tlm_status emsim_new(emsim_doc **out);
/* LoadProject (ProjectIO.cpp:194-248): on failure *out is NULL, the status
 * is TLM_EINVAL (TLM_ENOMEM when the file cannot be opened) and err holds the
 * reference's message ("cannot open file", "not an EMSIM project file",
 * "unsupported project version", "corrupt settings", "corrupt object list",
 * "corrupt plot data", "corrupt curve data", "corrupt playback data", "file
 * truncated or corrupt"). */
TLM_API tlm_status emsim_load(const char *path, emsim_doc **out, char *err, size_t err_cap);
/* SaveProject (ProjectIO.cpp:137-191): always format version 2. */
TLM_API tlm_status emsim_save(emsim_doc *d, const char *path);
TLM_API void emsim_free(emsim_doc *d);
TLM_API const char *emsim_last_error(emsim_doc *d);
/* Format version of the file the document was loaded from (2 for new). */
TLM_API int emsim_file_version(emsim_doc *d);

/* Settings rows (key, value strings). */
TLM_API int emsim_setting_count(emsim_doc *d);
TLM_API tlm_status emsim_get_setting(emsim_doc *d, int i, const char **key, const char **value);
TLM_API tlm_status emsim_add_setting(emsim_doc *d, const char *key, const char *value);
TLM_API tlm_status emsim_clear_settings(emsim_doc *d);

TLM_API tlm_status emsim_get_toolbar(emsim_doc *d, emsim_toolbar *out);
TLM_API tlm_status emsim_set_toolbar(emsim_doc *d, const emsim_toolbar *t);

/* Scene objects. */
TLM_API int emsim_object_count(emsim_doc *d);
TLM_API tlm_status emsim_get_object(emsim_doc *d, int i, emsim_object *out);
TLM_API tlm_status emsim_get_object_param(emsim_doc *d, int i, int p, const char **name, double *value);
TLM_API tlm_status emsim_add_object(emsim_doc *d, const emsim_object *o, int *idx);
TLM_API tlm_status emsim_add_object_param(emsim_doc *d, int i, const char *name, double value);
TLM_API tlm_status emsim_clear_objects(emsim_doc *d);

/* Displayed result. emsim_result_default fills GLResult's defaults (no
 * arrays, plane axis -1, pattern scale 1, empty domain box). */
TLM_API void emsim_result_default(emsim_result *r);
TLM_API tlm_status emsim_get_result(emsim_doc *d, emsim_result *out);
TLM_API tlm_status emsim_set_result(emsim_doc *d, const emsim_result *r);

/* Plot pages and their curves. */
TLM_API int emsim_page_count(emsim_doc *d);
TLM_API tlm_status emsim_get_page(emsim_doc *d, int i, const char **title, const char **x_label,
                                  const char **y_label, int *n_curves);
TLM_API tlm_status emsim_get_curve(emsim_doc *d, int page, int c, emsim_curve *out);
TLM_API tlm_status emsim_add_page(emsim_doc *d, const char *title, const char *x_label, const char *y_label,
                                  int *idx);
TLM_API tlm_status emsim_add_curve(emsim_doc *d, int page, const emsim_curve *c);
TLM_API tlm_status emsim_clear_pages(emsim_doc *d);

/* Playback (ProjPlayback, ProjectIO.h:36-44). emsim_set_playback marks it
 * valid and drops any frames; emsim_clear_playback marks it invalid. */
TLM_API tlm_status emsim_get_playback(emsim_doc *d, int *valid, tlm_grid *grid, float *dt,
                                      const emsim_face **faces, uint32_t *n_faces, uint32_t *n_frames);
TLM_API tlm_status emsim_set_playback(emsim_doc *d, const tlm_grid *grid, float dt, const emsim_face *faces,
                                      uint32_t n_faces);
TLM_API tlm_status emsim_get_frame(emsim_doc *d, uint32_t i, emsim_frame *out);
TLM_API tlm_status emsim_add_frame(emsim_doc *d, const emsim_frame *f);
TLM_API tlm_status emsim_clear_playback(emsim_doc *d);

/* What emsim_from_tlm / emsim_from_fdtd put in the document. */
typedef struct emsim_capture {
    int js_dft;          /* 1: face values = |Js| DFT at f0 (getJsDft, the
                            "DFT" display of a finished run); 0: |Js| now */
    int n_theta, n_phi;  /* > 0: compute the far-field pattern and store it */
    int playback;        /* 1: store the recorded frames as playback */
} emsim_capture;

/* The result and playback a finished run leaves in the reference's main
 * window (MainUnit.cpp:1025-1057, 2026-2043, 2275-2302): the PEC-surface
 * faces with |Js| (surface_monitors = 1), the cut plane if one was computed,
 * the pattern centred on the grid with radius 0.45 min(n) dl, the domain box
 * of the grid (shown), and, with record_every > 0, every recorded frame with
 * the grid, dt and faces. Other sections of the document are unchanged. */
TLM_API tlm_status emsim_from_tlm(emsim_doc *d, tlm_handle h, const emsim_capture *c);
TLM_API tlm_status emsim_from_fdtd(emsim_doc *d, fdtd_handle h, const emsim_capture *c);

#ifdef __cplusplus
}
#endif

#endif /* EMSIM_B200_H */
