// tlm_host_math.cpp -- host-side scalar math that must round exactly like the
// reference's CPU solver: time step, source waveforms and the per-material
// stub tables. Compiled by g++ with -O2 -ffp-contract=off (no FMA
// contraction, like the reference built for x86-64 without -march) so the
// FP32 results are bitwise those of TlmSolver.cpp. The FP64 variants feed the
// on-device FP64 mode and use the same float constants promoted to double.
#include "tlm_host_math.h"

#include <algorithm>
#include <cmath>

namespace tlmh {

// Constants as the reference declares them (TlmSolver.cpp:15-16).
static const float kC0 = 299792458.0f;
static const float kEta0 = 376.730313f;
static const double kPiD = 3.14159265358979323846;

float eta0_f32() { return kEta0; }

// dt = dl / (2 c0) (TlmSolver.cpp:268).
float timestep_f32(float dl) { return dl / (2.0f * kC0); }
double timestep_f64(float dl) { return (double)dl / (2.0 * (double)kC0); }

// Source waveforms at t = n*dt (TlmSolver.cpp:410-436):
//  0 CW with a raised-cosine ramp over 3 periods,
//  1 Gaussian-windowed sine, tau = 2/f0, delay 3 tau,
//  2 Gaussian pulse, tau = 0.5/f0, delay 3 tau.
template <class T> static T waveformT(int type, float f0in, T dt, int n)
{
    const T pi = (T)kPiD;
    const T f0 = (T)f0in;
    T t = (T)n * dt;
    T w = (T)2 * pi * f0;
    if (type == 0)
    {
        T ramp = (T)3 / f0;
        T r = (t < ramp) ? (T)0.5 * ((T)1 - std::cos(pi * t / ramp)) : (T)1;
        return r * std::sin(w * t);
    }
    if (type == 1)
    {
        T tau = (T)2 / f0, t0 = (T)3 * tau;
        T u = (t - t0) / tau;
        return std::exp(-u * u) * std::sin(w * (t - t0));
    }
    T tau = (T)0.5 / f0, t0 = (T)3 * tau;
    T u = (t - t0) / tau;
    return std::exp(-u * u);
}

float waveform_f32(int type, float f0, float dt, int n) { return waveformT<float>(type, f0, dt, n); }
double waveform_f64(int type, float f0, double dt, int n)
{
    return waveformT<double>(type, f0, dt, n);
}

// Stub tables (TlmSolver.cpp:270-276): yhat = 4 (max(1, er) - 1),
// ghat = (max(0, sigma) * dl) * eta0.
void tables_f32(const float *epsr, const float *sigma, int n, float dl, float *yhat,
                float *ghat)
{
    for (int t = 0; t < n; ++t)
    {
        yhat[t] = 4.0f * (std::max(1.0f, epsr[t]) - 1.0f);
        ghat[t] = std::max(0.0f, sigma[t]) * dl * kEta0;
    }
}
void tables_f64(const float *epsr, const float *sigma, int n, float dl, double *yhat,
                double *ghat)
{
    for (int t = 0; t < n; ++t)
    {
        yhat[t] = 4.0 * (std::max(1.0, (double)epsr[t]) - 1.0);
        ghat[t] = std::max(0.0, (double)sigma[t]) * (double)dl * (double)kEta0;
    }
}

// Probe scale -1/dl (TlmSolver.cpp:709).
// Phase of the surface-monitor DFT at step n (TlmSolver.cpp:619-620):
// 2 pi f0 (n dt), then its cosine and sine.
void dft_phase_f32(float f0, float dt, int n, float *c, float *s)
{
    const float phase = 2.0f * (float)kPiD * f0 * ((float)n * dt);
    *c = std::cos(phase);
    *s = std::sin(phase);
}
void dft_phase_f64(float f0, double dt, int n, double *c, double *s)
{
    const double phase = 2.0 * kPiD * (double)f0 * ((double)n * dt);
    *c = std::cos(phase);
    *s = std::sin(phase);
}

// Yee FDTD constants (FdtdSolver.cpp:15-18, 88-89, 143, 452): Courant-limited
// time step, first-order Mur coefficient, air E update and H update factors.
static const float kEps0 = 8.8541878128e-12f;
static const float kMu0 = 1.25663706212e-6f;
float fdtd_dt(float dl) { return 0.99f * dl / (kC0 * std::sqrt(3.0f)); }
float fdtd_cmur(float dt, float dl) { return (kC0 * dt - dl) / (kC0 * dt + dl); }
float fdtd_cb0(float dt, float dl) { return dt / (kEps0 * dl); }
float fdtd_ch(float dt, float dl) { return dt / (kMu0 * dl); }
// Lossy-dielectric E coefficients of one edge from the sums of (1 + (epsr -
// 1)) and sigma over its cnt in-grid neighbour cells (FdtdSolver.cpp:193-206).
void fdtd_edge_coef(float eAcc, float sAcc, int cnt, float dt, float dl, float *ca, float *cb)
{
    const float epsr = eAcc / cnt;
    const float sigma = sAcc / cnt;
    const float eps = kEps0 * std::max(1.0f, epsr);
    const float lf = sigma * dt / (2.0f * eps);
    *ca = (1.0f - lf) / (1.0f + lf);
    *cb = (dt / (eps * dl)) / (1.0f + lf);
}

float probe_scale_f32(float dl) { return -1.0f / dl; }
double probe_scale_f64(float dl) { return -1.0 / (double)dl; }

// Cell containing a world point, floor((p - origin)/dl) in float
// (Geometry.h:107-112).
void cell_of(const float origin[3], float dl, float x, float y, float z, int *i, int *j, int *k)
{
    *i = (int)std::floor((x - origin[0]) / dl);
    *j = (int)std::floor((y - origin[1]) / dl);
    *k = (int)std::floor((z - origin[2]) / dl);
}

} // namespace tlmh

namespace tlmh {
// Copy n material ids and return the largest: one pass over the caller's map
// instead of a scan and a copy. Sixteen running maxima side by side, so that
// the compiler keeps them in one vector register (a byte-wise max per 16
// bytes) instead of one dependent max per byte.
__attribute__((optimize("tree-vectorize"))) uint8_t copy_max_u8(const uint8_t *__restrict src,
                                                                 uint8_t *__restrict dst, size_t n)
{
    uint8_t m[16] = {};
    size_t i = 0;
    for (; i + 16 <= n; i += 16)
        for (int l = 0; l < 16; ++l)
        {
            const uint8_t v = src[i + l];
            dst[i + l] = v;
            m[l] = m[l] > v ? m[l] : v;
        }
    uint8_t r = 0;
    for (int l = 0; l < 16; ++l) r = r > m[l] ? r : m[l];
    for (; i < n; ++i)
    {
        dst[i] = src[i];
        r = r > src[i] ? r : src[i];
    }
    return r;
}
} // namespace tlmh
