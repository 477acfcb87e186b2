// ref_emsim_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// Drives the reference's own project writer and reader (SaveProject /
// LoadProject, ProjectIO.cpp of smilima/EMSolver, compiled unmodified) so
// that the tests can check the library's .emsim code byte for byte against
// them. Nothing in the product links this file.
//
// ProjectIO.h includes the VCL viewport header GLView.h only for the plain
// struct GLResult; the recipe in oracle/Makefile defines that header's guard
// and force-includes a header holding GLResult extracted from the reference's
// GLView.h at build time, so no VCL or OpenGL code is involved.
#include "ProjectIO.h"

#include <cstdint>
#include <cstring>
#include <string>

namespace {

std::wstring widen(const char *p)
{
    std::wstring w;
    for (; *p; ++p) w.push_back((wchar_t)(unsigned char)*p);
    return w;
}

void copyErr(const std::string &e, char *err, int cap)
{
    if (!err || cap <= 0) return;
    std::strncpy(err, e.c_str(), (size_t)cap - 1);
    err[cap - 1] = 0;
}

// Small deterministic generator for the sample project.
struct Lcg
{
    uint32_t s;
    float f() { s = s * 1664525u + 1013904223u; return (float)(s >> 8) * (1.0f / 16777216.0f) - 0.5f; }
    int i(int n) { s = s * 1664525u + 1013904223u; return (int)((s >> 8) % (uint32_t)n); }
};

Vec3 v3(Lcg &g) { return Vec3(g.f() * 10.0f, g.f() * 10.0f, g.f() * 10.0f); }

SurfaceFace face(Lcg &g, int k)
{
    SurfaceFace f{};  // value-initialised: the two padding bytes are zero
    f.airCell = 1000 * k + g.i(997);
    f.center = v3(g);
    f.axis = (int8_t)(k % 3);
    f.sign = (int8_t)((k & 1) ? -1 : 1);
    return f;
}

} // namespace

extern "C" {

// LoadProject(in) and, on success, SaveProject(out). Returns 1 when both
// succeed, 0 when loading fails (err = the reference's message), -1 when
// saving fails.
int ref_emsim_resave(const char *in, const char *out, char *err, int cap)
{
    ProjectData d;
    std::string e;
    if (!LoadProject(widen(in), d, e))
    {
        copyErr(e, err, cap);
        return 0;
    }
    return SaveProject(widen(out), d) ? 1 : -1;
}

// SaveProject of a sample project with every section filled from `seed`
// (settings, toolbar, an antenna with parameters, an STL object, a result
// with faces, triangle and wire currents, a plane and a pattern, two plot
// pages, and playback frames when with_playback is set).
int ref_emsim_write_sample(const char *path, int seed, int with_playback)
{
    Lcg g{ (uint32_t)seed * 2654435761u + 17u };
    ProjectData d;
    const int ns = 2 + seed % 3;
    for (int i = 0; i < ns; ++i)
        d.settings.emplace_back("key" + std::to_string(i), "value " + std::to_string(i * seed));
    d.solverIdx = seed % 5;
    d.excitationIdx = 1 + seed % 2;
    d.waveformIdx = seed % 3;
    d.currentsIdx = 2;
    d.dbRangeIdx = seed % 4;
    d.gpu = seed & 1;
    d.showModel = (seed >> 1) & 1;
    d.dbScale = true;
    d.planeOn = (seed >> 2) & 1;
    d.meshOn = false;

    ProjObject a;
    a.kind = 3 + seed % 4;
    a.name = "dipole " + std::to_string(seed);
    a.position = v3(g);
    a.rotDeg = v3(g);
    a.dielectric = seed & 1;
    a.epsr = 2.5f + g.f();
    a.sigma = 0.01f * (g.f() + 0.5f);
    a.designFreqHz = 1.5e9 + 1e6 * seed;
    a.params = { { "length", 0.1 + 0.01 * seed }, { "gap", 0.002 }, { "radius", 1e-3 * (1 + seed % 3) } };
    d.objects.push_back(a);
    ProjObject s;
    s.kind = 0;
    s.name = "mesh.stl";
    s.isStl = true;
    for (int i = 0; i < 12; ++i) s.stlVerts.push_back(g.f());
    s.stlIdx = { 0, 1, 2, 0, 2, 3 };
    d.objects.push_back(s);

    GLResult &r = d.result;
    const int nf = 4 + seed % 5;
    for (int k = 0; k < nf; ++k) r.faces.push_back(face(g, k));
    for (int k = 0; k < nf; ++k) r.faceVals.push_back(g.f() + 0.5f);
    r.faceDl = 1e-3f * (1 + seed % 4);
    for (int k = 0; k < 4; ++k) r.triV.push_back(v3(g));
    r.triIdx = { 0, 1, 2, 1, 3, 2 };
    r.triMag = { g.f(), g.f() };
    r.wirePts = { v3(g), v3(g) };
    r.wireMag = { g.f() };
    r.hasPlane = true;
    r.planeGrid.nx = 5 + seed % 3;
    r.planeGrid.ny = 6;
    r.planeGrid.nz = 7;
    r.planeGrid.origin = v3(g);
    r.planeGrid.dl = 2e-3f;
    r.planeAxis = seed % 3;
    r.planeIdx = 2;
    r.planeN1 = 3;
    r.planeN2 = 2;
    for (int k = 0; k < 6; ++k) r.planeVals.push_back(g.f());
    r.hasPattern = true;
    r.pattern.nTheta = 3;
    r.pattern.nPhi = 4;
    for (int k = 0; k < 12; ++k) r.pattern.U.push_back(g.f() + 0.5f);
    r.pattern.uMax = 0.9f;
    r.pattern.directivity = 1.64f;
    r.pattern.peakThetaDeg = 90.0f;
    r.pattern.peakPhiDeg = 45.0f;
    r.patCenter = v3(g);
    r.patScale = 0.3f;
    r.domain.grow(v3(g));
    r.domain.grow(v3(g));
    r.domainVisible = true;
    r.probeMarkers = { v3(g) };

    for (int p = 0; p < 2; ++p)
    {
        ProjPage pg;
        pg.title = "page " + std::to_string(p);
        pg.xLabel = "f (GHz)";
        pg.yLabel = p ? "|S11| (dB)" : "Z (ohm)";
        for (int c = 0; c <= p; ++c)
        {
            ProjCurve cv;
            cv.name = "curve " + std::to_string(c);
            cv.color = 0x00ff0000u >> (8 * c);
            for (int k = 0; k < 5 + c; ++k)
            {
                cv.x.push_back(0.5 + 0.1 * k);
                cv.y.push_back((double)g.f());
            }
            pg.curves.push_back(cv);
        }
        d.pages.push_back(pg);
    }

    if (with_playback)
    {
        d.playback.valid = true;
        d.playback.grid = r.planeGrid;
        d.playback.dt = 1.9e-12f;
        d.playback.faces = r.faces;
        for (int i = 0; i < 3; ++i)
        {
            VizFrame fr;
            fr.step = 10 * (i + 1);
            for (int k = 0; k < nf; ++k) fr.js.push_back(g.f() + 0.5f);
            if (i != 1)
            {
                fr.planeAxis = r.planeAxis;
                fr.planeIdx = 2;
                fr.planeN1 = 3;
                fr.planeN2 = 2;
                for (int k = 0; k < 6; ++k) fr.plane.push_back(g.f());
            }
            d.playback.frames.push_back(fr);
        }
    }
    return SaveProject(widen(path), d) ? 1 : 0;
}

// LoadProject(path) and a summary of what it read: out[0..11] = version-
// independent counts (settings, objects, result faces, face values, plane
// values, pattern U, pages, curves on page 0, playback valid, playback faces,
// frames, js values of frame 0). Returns 1, or 0 with err on failure.
int ref_emsim_summary(const char *path, int64_t *out, char *err, int cap)
{
    ProjectData d;
    std::string e;
    if (!LoadProject(widen(path), d, e))
    {
        copyErr(e, err, cap);
        return 0;
    }
    out[0] = (int64_t)d.settings.size();
    out[1] = (int64_t)d.objects.size();
    out[2] = (int64_t)d.result.faces.size();
    out[3] = (int64_t)d.result.faceVals.size();
    out[4] = (int64_t)d.result.planeVals.size();
    out[5] = (int64_t)d.result.pattern.U.size();
    out[6] = (int64_t)d.pages.size();
    out[7] = d.pages.empty() ? 0 : (int64_t)d.pages[0].curves.size();
    out[8] = d.playback.valid ? 1 : 0;
    out[9] = (int64_t)d.playback.faces.size();
    out[10] = (int64_t)d.playback.frames.size();
    out[11] = d.playback.frames.empty() ? 0 : (int64_t)d.playback.frames[0].js.size();
    return 1;
}

} // extern "C"
