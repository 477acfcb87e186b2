// ref_fdtd_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// Drives the reference's own Yee FDTD solver (FdtdSolver.cpp of
// smilima/EMSolver, compiled unmodified) through a small C ABI for tests,
// golden-vector generation and the bench's CPU baseline. Nothing in the
// product links this file.
//
// The reference's GPU seam for this solver is the friend function
// `bool RunGpuFdtd(FdtdSolver&, std::string&)` (FdtdSolver.h:9, GpuFdtd.h).
// This file defines it (the OpenGL GpuFdtd.cpp is not compiled) and uses its
// friend access to run one private step with a caller-chosen source value and
// to read the private fields and monitor accumulators. The reference's run()
// only calls it when config.useGpu is set, which setup here never does.
#include "FdtdSolver.h"
#include "GpuFdtd.h"

#include <cstdint>
#include <cstring>
#include <string>

namespace {

enum Op { kNone, kStep, kStepSv, kField, kJsRaw, kHuy, kFinalize, kDt };
struct Request
{
    Op op = kNone;
    int n = 0, count = 0;
    const float *sv = nullptr;
    int which = 0;
    float *out = nullptr;
    size_t cap = 0;
    size_t size = 0;
    float *re = nullptr, *im = nullptr;
    int samples = 0;
    uint64_t *cells = nullptr;
    int *axis = nullptr, *sign = nullptr;
    float *pos = nullptr;
};
thread_local Request g_req;

} // namespace

// Friend of FdtdSolver: performs the pending request with access to its
// private members.
bool RunGpuFdtd(FdtdSolver &s, std::string &msg)
{
    Request &r = g_req;
    switch (r.op)
    {
    case kStep:
        for (int i = 0; i < r.count; ++i)
        {
            s.step(r.n + i);
            s.curStep = r.n + i + 1;
        }
        break;
    case kStepSv:
        // FdtdSolver::step (FdtdSolver.cpp:401-446) with sv[i] instead of
        // waveformValue(n): the same injection onto the cell's 4 edges.
        for (int i = 0; i < r.count; ++i)
        {
            const int n = r.n + i;
            const float sv = r.sv[i];
            auto inject = [&](size_t cell, int polAxis, float amp) {
                int ci = (int)(cell % s.g.nx);
                int cj = (int)((cell / s.g.nx) % s.g.ny);
                int ck = (int)(cell / ((size_t)s.g.nx * s.g.ny));
                float q = -0.25f * amp * sv;
                if (polAxis == 0)
                {
                    if (s.mEx[s.iEx(ci, cj, ck)]) s.Ex[s.iEx(ci, cj, ck)] += q;
                    if (s.mEx[s.iEx(ci, cj + 1, ck)]) s.Ex[s.iEx(ci, cj + 1, ck)] += q;
                    if (s.mEx[s.iEx(ci, cj, ck + 1)]) s.Ex[s.iEx(ci, cj, ck + 1)] += q;
                    if (s.mEx[s.iEx(ci, cj + 1, ck + 1)]) s.Ex[s.iEx(ci, cj + 1, ck + 1)] += q;
                }
                else if (polAxis == 1)
                {
                    if (s.mEy[s.iEy(ci, cj, ck)]) s.Ey[s.iEy(ci, cj, ck)] += q;
                    if (s.mEy[s.iEy(ci + 1, cj, ck)]) s.Ey[s.iEy(ci + 1, cj, ck)] += q;
                    if (s.mEy[s.iEy(ci, cj, ck + 1)]) s.Ey[s.iEy(ci, cj, ck + 1)] += q;
                    if (s.mEy[s.iEy(ci + 1, cj, ck + 1)]) s.Ey[s.iEy(ci + 1, cj, ck + 1)] += q;
                }
                else
                {
                    if (s.mEz[s.iEz(ci, cj, ck)]) s.Ez[s.iEz(ci, cj, ck)] += q;
                    if (s.mEz[s.iEz(ci + 1, cj, ck)]) s.Ez[s.iEz(ci + 1, cj, ck)] += q;
                    if (s.mEz[s.iEz(ci, cj + 1, ck)]) s.Ez[s.iEz(ci, cj + 1, ck)] += q;
                    if (s.mEz[s.iEz(ci + 1, cj + 1, ck)]) s.Ez[s.iEz(ci + 1, cj + 1, ck)] += q;
                }
            };
            for (const auto &src : s.sources) inject(src.cell, src.polAxis, src.amp);
            for (const auto &p : s.portList)
                for (size_t c : p.cells) inject(c, p.polAxis, p.amp);
            s.monitors(n);
            s.updateH();
            s.applyMur();
            s.curStep = n + 1;
        }
        break;
    case kField:
    {
        const std::vector<float> *v[6] = { &s.Ex, &s.Ey, &s.Ez, &s.Hx, &s.Hy, &s.Hz };
        const std::vector<float> &a = *v[r.which];
        r.size = a.size();
        if (r.out) std::memcpy(r.out, a.data(), std::min(r.cap, a.size()) * sizeof(float));
        break;
    }
    case kJsRaw:
        r.size = s.jsDftRe.size() / 2;
        for (size_t t = 0; t < s.jsDftRe.size() && t / 2 < r.cap; ++t)
        {
            if (r.re) r.re[t] = s.jsDftRe[t];
            if (r.im) r.im[t] = s.jsDftIm[t];
        }
        r.samples = s.dftSamples;
        break;
    case kHuy:
        r.size = s.huyFaces.size();
        for (size_t f = 0; f < s.huyFaces.size() && f < r.cap; ++f)
        {
            if (r.cells) r.cells[f] = (uint64_t)s.huyFaces[f].cell;
            if (r.axis) r.axis[f] = s.huyFaces[f].axis;
            if (r.sign) r.sign[f] = s.huyFaces[f].outSign;
            if (r.pos)
            {
                r.pos[3 * f] = s.huyFaces[f].pos.x;
                r.pos[3 * f + 1] = s.huyFaces[f].pos.y;
                r.pos[3 * f + 2] = s.huyFaces[f].pos.z;
            }
            if (r.out)
                for (int q = 0; q < 8; ++q) r.out[8 * f + q] = s.huyDft[8 * f + q];
        }
        r.samples = s.huySamples;
        break;
    case kFinalize:
        s.finalizeDft();
        break;
    default:
        msg = "no request";
        return false;
    }
    r.op = kNone;
    return true;
}

namespace {

bool run(FdtdSolver *s, Request r)
{
    g_req = r;
    std::string msg;
    return RunGpuFdtd(*s, msg);
}

} // namespace

extern "C" {

void *fdr_create(void) { return new FdtdSolver(); }
void fdr_destroy(void *h) { delete static_cast<FdtdSolver *>(h); }

int fdr_setup(void *h, int nx, int ny, int nz, float ox, float oy, float oz, float dl, const uint8_t *mat,
              const float *epsr, const float *sigma, int ntab, float f0, int waveform, int totalSteps,
              int settleSteps, int huyOffset, int recordEvery)
{
    FdtdSolver *s = static_cast<FdtdSolver *>(h);
    VoxelGridSpec g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
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
    cfg.huyOffset = huyOffset;
    cfg.useGpu = false;
    cfg.recordEvery = recordEvery;
    s->setup(g, std::move(m), std::move(tab), cfg);
    return 0;
}
int fdr_add_port(void *h, const uint64_t *cells, int n, int pol, float amp)
{
    std::vector<size_t> c(cells, cells + n);
    return static_cast<FdtdSolver *>(h)->addPort(c, pol, amp);
}
int fdr_add_probe(void *h, float x, float y, float z)
{
    return static_cast<FdtdSolver *>(h)->addProbe(Vec3(x, y, z));
}
void fdr_add_plane_wave(void *h, int prop, int plane, int pol, float amp)
{
    static_cast<FdtdSolver *>(h)->addPlaneWave(prop, plane, pol, amp);
}
void fdr_steps(void *h, int n0, int count)
{
    Request r;
    r.op = kStep;
    r.n = n0;
    r.count = count;
    run(static_cast<FdtdSolver *>(h), r);
}
void fdr_steps_sv(void *h, int n0, int count, const float *sv)
{
    Request r;
    r.op = kStepSv;
    r.n = n0;
    r.count = count;
    r.sv = sv;
    run(static_cast<FdtdSolver *>(h), r);
}
void fdr_run(void *h) { static_cast<FdtdSolver *>(h)->run(); }
float fdr_dt(void *h) { return static_cast<FdtdSolver *>(h)->timestep(); }
int fdr_current_step(void *h) { return static_cast<FdtdSolver *>(h)->currentStep(); }

// Field component `which` (0..5 = Ex Ey Ez Hx Hy Hz) in the reference's
// Yee layout; returns its length.
size_t fdr_get_field(void *h, int which, float *out, size_t cap)
{
    Request r;
    r.op = kField;
    r.which = which;
    r.out = out;
    r.cap = cap;
    run(static_cast<FdtdSolver *>(h), r);
    return g_req.size;
}
int fdr_get_probe(void *h, int idx, float *ex, float *ey, float *ez, int cap)
{
    const FieldProbe &p = static_cast<FdtdSolver *>(h)->probe(idx);
    int n = (int)p.ez.size();
    for (int i = 0; i < n && i < cap; ++i)
    {
        ex[i] = p.ex[i];
        ey[i] = p.ey[i];
        ez[i] = p.ez[i];
    }
    return n;
}
int fdr_get_port(void *h, int idx, float *v, float *i, int cap)
{
    const TlmPort &p = static_cast<FdtdSolver *>(h)->ports()[idx];
    int n = (int)p.vRec.size();
    for (int t = 0; t < n && t < cap; ++t)
    {
        v[t] = p.vRec[t];
        i[t] = p.iRec[t];
    }
    return n;
}
int fdr_energy_history(void *h, int *steps, float *vals, int cap)
{
    std::vector<int> st;
    std::vector<float> va;
    static_cast<FdtdSolver *>(h)->getEnergyHistory(st, va);
    int n = (int)st.size();
    for (int t = 0; t < n && t < cap; ++t)
    {
        steps[t] = st[t];
        vals[t] = va[t];
    }
    return n;
}

// ---- surface monitors (same shapes as the TLM harness)
int fdr_surface_faces(void *h, uint64_t *cells, int *axis, int *sign, float *center, int cap)
{
    const auto &f = static_cast<FdtdSolver *>(h)->faces();
    for (int t = 0; t < (int)f.size() && t < cap; ++t)
    {
        if (cells) cells[t] = (uint64_t)f[t].airCell;
        if (axis) axis[t] = f[t].axis;
        if (sign) sign[t] = f[t].sign;
        if (center)
        {
            center[3 * t] = f[t].center.x;
            center[3 * t + 1] = f[t].center.y;
            center[3 * t + 2] = f[t].center.z;
        }
    }
    return (int)f.size();
}
int fdr_js_instant(void *h, float *out, int cap)
{
    std::vector<float> v;
    static_cast<FdtdSolver *>(h)->getJsInstant(v);
    for (int t = 0; t < (int)v.size() && t < cap; ++t) out[t] = v[t];
    return (int)v.size();
}
int fdr_js_dft(void *h, float *re, float *im, float *mag, int cap, int *samples)
{
    FdtdSolver *s = static_cast<FdtdSolver *>(h);
    Request r;
    r.op = kJsRaw;
    r.re = re;
    r.im = im;
    r.cap = (size_t)cap;
    run(s, r);
    const int n = (int)g_req.size;
    if (samples) *samples = g_req.samples;
    if (mag)
    {
        Request f;
        f.op = kFinalize;
        run(s, f);
        std::vector<float> m;
        s->getJsDft(m);
        for (int t = 0; t < (int)m.size() && t < cap; ++t) mag[t] = m[t];
    }
    return n;
}
int fdr_huygens_faces(void *h, uint64_t *cells, int *axis, int *outSign, float *pos, int cap)
{
    Request r;
    r.op = kHuy;
    r.cells = cells;
    r.axis = axis;
    r.sign = outSign;
    r.pos = pos;
    r.cap = (size_t)cap;
    run(static_cast<FdtdSolver *>(h), r);
    return (int)g_req.size;
}
int fdr_huygens_dft(void *h, float *acc, int cap, int *samples)
{
    Request r;
    r.op = kHuy;
    r.out = acc;
    r.cap = (size_t)cap;
    run(static_cast<FdtdSolver *>(h), r);
    if (samples) *samples = g_req.samples;
    return (int)g_req.size;
}
void fdr_set_field_plane(void *h, int axis, int index)
{
    static_cast<FdtdSolver *>(h)->setFieldPlane(axis, index);
}
int fdr_field_plane(void *h, float *out, size_t cap, int *axis, int *index, int *n1, int *n2)
{
    std::vector<float> v;
    if (!static_cast<FdtdSolver *>(h)->getFieldPlane(v, *axis, *index, *n1, *n2)) return -1;
    for (size_t t = 0; t < v.size() && t < cap; ++t) out[t] = v[t];
    return 0;
}
int fdr_frame_count(void *h) { return static_cast<FdtdSolver *>(h)->frameCount(); }
int fdr_get_frame(void *h, int idx, int *step, float *js, int jsCap, float *plane, size_t planeCap, int *axis,
                  int *pidx, int *n1, int *n2)
{
    VizFrame fr;
    if (!static_cast<FdtdSolver *>(h)->getFrame(idx, fr)) return -1;
    *step = fr.step;
    for (int t = 0; t < (int)fr.js.size() && t < jsCap; ++t) js[t] = fr.js[t];
    for (size_t t = 0; t < fr.plane.size() && t < planeCap; ++t) plane[t] = fr.plane[t];
    *axis = fr.planeAxis;
    *pidx = fr.planeIdx;
    *n1 = fr.planeN1;
    *n2 = fr.planeN2;
    return (int)fr.plane.size();
}
int fdr_far_field(void *h, int nTheta, int nPhi, float *U, float *uMax, float *directivity, float *peakTheta,
                  float *peakPhi)
{
    FarFieldData d;
    if (!static_cast<FdtdSolver *>(h)->computeFarField(d, nTheta, nPhi)) return -1;
    for (size_t t = 0; t < d.U.size(); ++t) U[t] = d.U[t];
    *uMax = d.uMax;
    *directivity = d.directivity;
    *peakTheta = d.peakThetaDeg;
    *peakPhi = d.peakPhiDeg;
    return 0;
}

} // extern "C"
