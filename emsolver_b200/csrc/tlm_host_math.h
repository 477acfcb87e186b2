// tlm_host_math.h -- host scalar math that must match the reference bit for bit.
#pragma once

#include <cstddef>
#include <cstdint>

namespace tlmh {
float eta0_f32();
float timestep_f32(float dl);
double timestep_f64(float dl);
float waveform_f32(int type, float f0, float dt, int n);
double waveform_f64(int type, float f0, double dt, int n);
void tables_f32(const float *epsr, const float *sigma, int n, float dl, float *yhat,
                float *ghat);
void tables_f64(const float *epsr, const float *sigma, int n, float dl, double *yhat,
                double *ghat);
float probe_scale_f32(float dl);
float fdtd_dt(float dl);
float fdtd_cmur(float dt, float dl);
float fdtd_cb0(float dt, float dl);
float fdtd_ch(float dt, float dl);
void fdtd_edge_coef(float eAcc, float sAcc, int cnt, float dt, float dl, float *ca, float *cb);
void dft_phase_f32(float f0, float dt, int n, float *c, float *s);
void dft_phase_f64(float f0, double dt, int n, double *c, double *s);
double probe_scale_f64(float dl);
void cell_of(const float origin[3], float dl, float x, float y, float z, int *i, int *j, int *k);
// copy n bytes and return the largest
uint8_t copy_max_u8(const uint8_t *src, uint8_t *dst, size_t n);
} // namespace tlmh
