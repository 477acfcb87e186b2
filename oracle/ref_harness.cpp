// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// Drives the reference's own CPU TLM solver, compiled unmodified from
// TlmSolver.cpp + Geometry.cpp of smilima/EMSolver, through a small C ABI so
// that tests, golden-vector generation and the CPU baseline leg of the bench
// can call it from Python (ctypes). Nothing in the product links this file.
//
// Access to the solver's private state uses the reference's own hook:
// TlmSolver declares `friend class GpuTlm;` (TlmSolver.h:267). This file
// defines that class (the reference's GpuTlm.cpp, the OpenGL path, is not
// compiled), and supplies RunGpuTlm (GpuTlm.h:15) returning false, which is
// what the reference does on a machine without an OpenGL 4.3 device.
#include "TlmSolver.h"
#include "GpuTlm.h"

#include <cstdint>
#include <cstring>
#include <string>
#include <thread>

bool RunGpuTlm(TlmSolver &, std::string &msg)
{
    msg = "OpenGL compute path not built (headless reference build)";
    return false;
}

class GpuTlm
{
public:
    // One reference time step with a caller-supplied source value instead of
    // waveformValue(n): the injection of TlmSolver::step (TlmSolver.cpp:487-505)
    // followed by the reference's own private monitors/scatter/connect.
    static void stepWithSource(TlmSolver &s, int n, float sv)
    {
        for (const auto &src : s.sources)
            inject(s, src.cell, src.polAxis, src.amp, sv);
        for (const auto &p : s.portList)
            for (size_t c : p.cells)
                inject(s, c, p.polAxis, p.amp, sv);
        s.monitors(n);
        s.scatter();
        s.connect();
        s.curStep = n + 1;
    }
    static void step(TlmSolver &s, int n)
    {
        s.step(n);
        s.curStep = n + 1;
    }
    static float waveform(const TlmSolver &s, int n) { return s.waveformValue(n); }
    static const std::vector<float> &V(const TlmSolver &s) { return s.V; }
    static std::vector<float> &Vmut(TlmSolver &s) { return s.V; }
    static const std::vector<float> &Vs(const TlmSolver &s) { return s.Vs; }
    static const std::vector<float> &yhat(const TlmSolver &s) { return s.yhat; }
    static const std::vector<float> &ghat(const TlmSolver &s) { return s.ghat; }
    static int threads(const TlmSolver &s) { return s.pool->threadCount(); }
    static const std::vector<TlmPort> &ports(const TlmSolver &s) { return s.portList; }
    static const std::vector<float> &jsDftRe(const TlmSolver &s) { return s.jsDftRe; }
    static const std::vector<float> &jsDftIm(const TlmSolver &s) { return s.jsDftIm; }
    static int dftSamples(const TlmSolver &s) { return s.dftSamples; }
    static const std::vector<HuyFace> &huyFaces(const TlmSolver &s) { return s.huyFaces; }
    static const std::vector<float> &huyDft(const TlmSolver &s) { return s.huyDft; }
    static int huySamples(const TlmSolver &s) { return s.huySamples; }
    static void finalizeDft(TlmSolver &s) { s.finalizeDft(); }

private:
    // Soft source: q = 0.5*amp*sv onto the two link pulses of polarisation
    // polAxis on each of the two axes orthogonal to it. Slot numbering is the
    // reference's axis*4 + side*2 + pol, pol = index of polAxis in the
    // axis's transverse pair {(1,2),(0,2),(0,1)}.
    static void inject(TlmSolver &s, size_t cell, int polAxis, float amp, float sv)
    {
        static const int tpair[3][2] = { {1, 2}, {0, 2}, {0, 1} };
        float q = 0.5f * amp * sv;
        float *vp = &s.V[cell * 12];
        for (int axis = 0; axis < 3; ++axis)
        {
            if (axis == polAxis)
                continue;
            int pol = (polAxis == tpair[axis][0]) ? 0 : 1;
            vp[axis * 4 + 0 * 2 + pol] += q;
            vp[axis * 4 + 1 * 2 + pol] += q;
        }
    }
};

extern "C" {

void *ref_create(void) { return new TlmSolver(); }
void ref_destroy(void *h) { delete static_cast<TlmSolver *>(h); }

int ref_setup_ex(void *h, int nx, int ny, int nz, float ox, float oy, float oz,
                 float dl, const uint8_t *mat, const float *epsr,
                 const float *sigma, int ntab, float f0, int waveform,
                 int totalSteps, int settleSteps, float rho, int huyOffset,
                 int recordEvery);

int ref_setup(void *h, int nx, int ny, int nz, float ox, float oy, float oz,
              float dl, const uint8_t *mat, const float *epsr,
              const float *sigma, int ntab, float f0, int waveform,
              int totalSteps, int settleSteps, float rho)
{
    return ref_setup_ex(h, nx, ny, nz, ox, oy, oz, dl, mat, epsr, sigma, ntab, f0,
                        waveform, totalSteps, settleSteps, rho, 0, 0);
}

int ref_setup_ex(void *h, int nx, int ny, int nz, float ox, float oy, float oz,
                 float dl, const uint8_t *mat, const float *epsr,
                 const float *sigma, int ntab, float f0, int waveform,
                 int totalSteps, int settleSteps, float rho, int huyOffset,
                 int recordEvery)
{
    TlmSolver *s = static_cast<TlmSolver *>(h);
    VoxelGridSpec g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.origin = Vec3(ox, oy, oz);
    g.dl = dl;
    size_t n = (size_t)nx * ny * nz;
    std::vector<uint8_t> m(mat, mat + n);
    std::vector<MatProps> tab(ntab);
    for (int i = 0; i < ntab; ++i)
    {
        tab[i].epsr = epsr[i];
        tab[i].sigma = sigma[i];
    }
    TlmConfig cfg;
    cfg.f0 = f0;
    cfg.waveform = (WaveformType)waveform;
    cfg.totalSteps = totalSteps;
    cfg.settleSteps = settleSteps;
    cfg.boundaryRho = rho;
    cfg.huyOffset = huyOffset;
    cfg.useGpu = false;
    cfg.recordEvery = recordEvery;
    s->setup(g, std::move(m), std::move(tab), cfg);
    return 0;
}

int ref_add_port(void *h, const uint64_t *cells, int n, int pol, float amp)
{
    std::vector<size_t> c(cells, cells + n);
    return static_cast<TlmSolver *>(h)->addPort(c, pol, amp);
}

int ref_add_probe(void *h, float x, float y, float z)
{
    return static_cast<TlmSolver *>(h)->addProbe(Vec3(x, y, z));
}

void ref_add_plane_wave(void *h, int propAxis, int planeIndex, int polAxis, float amp)
{
    static_cast<TlmSolver *>(h)->addPlaneWave(propAxis, planeIndex, polAxis, amp);
}

void ref_step(void *h, int n) { GpuTlm::step(*static_cast<TlmSolver *>(h), n); }
void ref_step_sv(void *h, int n, float sv)
{
    GpuTlm::stepWithSource(*static_cast<TlmSolver *>(h), n, sv);
}
void ref_steps(void *h, int n0, int count)
{
    TlmSolver *s = static_cast<TlmSolver *>(h);
    for (int n = n0; n < n0 + count; ++n)
        GpuTlm::step(*s, n);
}
void ref_steps_sv(void *h, int n0, int count, const float *sv)
{
    TlmSolver *s = static_cast<TlmSolver *>(h);
    for (int i = 0; i < count; ++i)
        GpuTlm::stepWithSource(*s, n0 + i, sv[i]);
}
void ref_run(void *h) { static_cast<TlmSolver *>(h)->run(); }

float ref_waveform(void *h, int n) { return GpuTlm::waveform(*static_cast<TlmSolver *>(h), n); }
float ref_dt(void *h) { return static_cast<TlmSolver *>(h)->timestep(); }
int ref_threads(void *h) { return GpuTlm::threads(*static_cast<TlmSolver *>(h)); }
int ref_current_step(void *h) { return static_cast<TlmSolver *>(h)->currentStep(); }
float ref_current_energy(void *h) { return static_cast<TlmSolver *>(h)->currentEnergy(); }

size_t ref_get_pulses(void *h, float *out, size_t cap)
{
    const auto &v = GpuTlm::V(*static_cast<TlmSolver *>(h));
    size_t n = v.size() < cap ? v.size() : cap;
    if (out && n) std::memcpy(out, v.data(), n * sizeof(float));
    return v.size();
}
size_t ref_set_pulses(void *h, const float *in, size_t n)
{
    auto &v = GpuTlm::Vmut(*static_cast<TlmSolver *>(h));
    if (n != v.size()) return 0;
    std::memcpy(v.data(), in, n * sizeof(float));
    return n;
}
size_t ref_get_stubs(void *h, float *out, size_t cap)
{
    const auto &v = GpuTlm::Vs(*static_cast<TlmSolver *>(h));
    size_t n = v.size() < cap ? v.size() : cap;
    if (out && n) std::memcpy(out, v.data(), n * sizeof(float));
    return v.size();
}
int ref_get_tables(void *h, float *yhat, float *ghat, int cap)
{
    const TlmSolver &s = *static_cast<TlmSolver *>(h);
    const auto &y = GpuTlm::yhat(s);
    const auto &g = GpuTlm::ghat(s);
    int n = (int)y.size();
    for (int i = 0; i < n && i < cap; ++i) { yhat[i] = y[i]; ghat[i] = g[i]; }
    return n;
}

int ref_probe_count(void *h) { return static_cast<TlmSolver *>(h)->probeCount(); }
int ref_get_probe(void *h, int idx, float *ex, float *ey, float *ez, int cap,
                  uint64_t *cell)
{
    const FieldProbe &p = static_cast<TlmSolver *>(h)->probe(idx);
    int n = (int)p.ez.size();
    for (int i = 0; i < n && i < cap; ++i)
    {
        ex[i] = p.ex[i]; ey[i] = p.ey[i]; ez[i] = p.ez[i];
    }
    if (cell) *cell = p.cell;
    return n;
}
int ref_port_count(void *h) { return (int)GpuTlm::ports(*static_cast<TlmSolver *>(h)).size(); }
int ref_get_port(void *h, int idx, float *v, float *i, int cap, uint64_t *cells, int cellCap,
                 int *ncells)
{
    const TlmPort &p = GpuTlm::ports(*static_cast<TlmSolver *>(h))[idx];
    int n = (int)p.vRec.size();
    for (int t = 0; t < n && t < cap; ++t) { v[t] = p.vRec[t]; i[t] = p.iRec[t]; }
    if (ncells) *ncells = (int)p.cells.size();
    for (int t = 0; cells && t < (int)p.cells.size() && t < cellCap; ++t) cells[t] = p.cells[t];
    return n;
}
int ref_energy_history(void *h, int *steps, float *vals, int cap)
{
    std::vector<int> st;
    std::vector<float> va;
    static_cast<TlmSolver *>(h)->getEnergyHistory(st, va);
    int n = (int)st.size();
    for (int t = 0; t < n && t < cap; ++t) { steps[t] = st[t]; vals[t] = va[t]; }
    return n;
}

// ---- surface monitors: Js faces, Huygens box, cut plane, frames, far field
int ref_surface_faces(void *h, uint64_t *cells, int *axis, int *sign, float *center, int cap)
{
    const auto &f = static_cast<TlmSolver *>(h)->faces();
    for (int t = 0; t < (int)f.size() && t < cap; ++t)
    {
        if (cells) cells[t] = (uint64_t)f[t].airCell;
        if (axis) axis[t] = f[t].axis;
        if (sign) sign[t] = f[t].sign;
        if (center) { center[3 * t] = f[t].center.x; center[3 * t + 1] = f[t].center.y; center[3 * t + 2] = f[t].center.z; }
    }
    return (int)f.size();
}
int ref_js_instant(void *h, float *out, int cap)
{
    std::vector<float> v;
    static_cast<TlmSolver *>(h)->getJsInstant(v);
    for (int t = 0; t < (int)v.size() && t < cap; ++t) out[t] = v[t];
    return (int)v.size();
}
// Raw Js DFT accumulators, and the magnitudes of the reference's own
// finalizeDft (which run() calls after the last step).
int ref_js_dft(void *h, float *re, float *im, float *mag, int cap, int *samples)
{
    TlmSolver &s = *static_cast<TlmSolver *>(h);
    const auto &r = GpuTlm::jsDftRe(s);
    const auto &i = GpuTlm::jsDftIm(s);
    for (int t = 0; t < (int)r.size() && t / 2 < cap; ++t) { if (re) re[t] = r[t]; if (im) im[t] = i[t]; }
    if (mag)
    {
        GpuTlm::finalizeDft(s);
        std::vector<float> m;
        s.getJsDft(m);
        for (int t = 0; t < (int)m.size() && t < cap; ++t) mag[t] = m[t];
    }
    if (samples) *samples = GpuTlm::dftSamples(s);
    return (int)(r.size() / 2);
}
int ref_huygens_faces(void *h, uint64_t *cells, int *axis, int *outSign, float *pos, int cap)
{
    const auto &f = GpuTlm::huyFaces(*static_cast<TlmSolver *>(h));
    for (int t = 0; t < (int)f.size() && t < cap; ++t)
    {
        if (cells) cells[t] = (uint64_t)f[t].cell;
        if (axis) axis[t] = f[t].axis;
        if (outSign) outSign[t] = f[t].outSign;
        if (pos) { pos[3 * t] = f[t].pos.x; pos[3 * t + 1] = f[t].pos.y; pos[3 * t + 2] = f[t].pos.z; }
    }
    return (int)f.size();
}
int ref_huygens_dft(void *h, float *acc, int cap, int *samples)
{
    const TlmSolver &s = *static_cast<TlmSolver *>(h);
    const auto &a = GpuTlm::huyDft(s);
    for (int t = 0; t < (int)a.size() && t / 8 < cap; ++t) acc[t] = a[t];
    if (samples) *samples = GpuTlm::huySamples(s);
    return (int)(a.size() / 8);
}
void ref_set_field_plane(void *h, int axis, int index)
{
    static_cast<TlmSolver *>(h)->setFieldPlane(axis, index);
}
int ref_field_plane(void *h, float *out, size_t cap, int *axis, int *index, int *n1, int *n2)
{
    std::vector<float> v;
    if (!static_cast<TlmSolver *>(h)->getFieldPlane(v, *axis, *index, *n1, *n2)) return -1;
    for (size_t t = 0; t < v.size() && t < cap; ++t) out[t] = v[t];
    return 0;
}
int ref_frame_count(void *h) { return static_cast<TlmSolver *>(h)->frameCount(); }
int ref_get_frame(void *h, int idx, int *step, float *js, int jsCap, float *plane, size_t planeCap,
                  int *axis, int *pidx, int *n1, int *n2)
{
    VizFrame fr;
    if (!static_cast<TlmSolver *>(h)->getFrame(idx, fr)) return -1;
    *step = fr.step;
    for (int t = 0; t < (int)fr.js.size() && t < jsCap; ++t) js[t] = fr.js[t];
    for (size_t t = 0; t < fr.plane.size() && t < planeCap; ++t) plane[t] = fr.plane[t];
    *axis = fr.planeAxis;
    *pidx = fr.planeIdx;
    *n1 = fr.planeN1;
    *n2 = fr.planeN2;
    return (int)fr.plane.size();
}
int ref_far_field(void *h, int nTheta, int nPhi, float *U, float *uMax, float *directivity,
                  float *peakTheta, float *peakPhi)
{
    FarFieldData d;
    if (!static_cast<TlmSolver *>(h)->computeFarField(d, nTheta, nPhi)) return -1;
    for (size_t t = 0; t < d.U.size(); ++t) U[t] = d.U[t];
    *uMax = d.uMax;
    *directivity = d.directivity;
    *peakTheta = d.peakThetaDeg;
    *peakPhi = d.peakPhiDeg;
    return 0;
}

float ref_scatter_unitarity(void) { return TlmSolver::ScatterUnitarityError(); }
float ref_diel_unitarity(float epsr) { return TlmSolver::DielScatterUnitarityError(epsr); }
unsigned ref_hw_concurrency(void) { return std::thread::hardware_concurrency(); }

} // extern "C"
