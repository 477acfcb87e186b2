// emsim_io.cpp -- the .emsim project file (format version 2) behind the C ABI
// of emsim_b200.h: an in-memory document, its byte-exact serialisation, and
// the capture of a solver's result and playback into it.
//
// The file is the reference's (ProjectIO.cpp): an 8-byte magic "EMSIM" + 3
// zero bytes, a uint32 version, then the sections in a fixed order. Scalars
// are little-endian images of the reference's types; a string is a uint32
// length and its bytes; an array is a uint32 element count and the packed
// elements; flags are single bytes. Records that the reference writes as raw
// struct images keep those layouts here:
//   VoxelGridSpec 28 B (int nx, ny, nz; float origin[3]; float dl),
//   SurfaceFace   20 B (int32 cell; float centre[3]; int8 axis, sign; 2 pad),
//   Vec3 12 B, Aabb 24 B (lo, hi).
// The face padding bytes read from a file are kept, so a loaded document
// saves back to the same bytes; faces made through the API carry zero pads.
#include "emsim_b200.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

namespace {

const char kMagic[8] = { 'E', 'M', 'S', 'I', 'M', 0, 0, 0 };
const uint32_t kVersion = 2;

struct Vec { float v[3] = { 0.0f, 0.0f, 0.0f }; };

struct Face
{
    int32_t cell = 0;
    float c[3] = { 0.0f, 0.0f, 0.0f };
    int8_t axis = 0, sign = 0;
    uint8_t pad[2] = { 0, 0 };
};

struct Grid
{
    int32_t n[3] = { 0, 0, 0 };
    float origin[3] = { 0.0f, 0.0f, 0.0f };
    float dl = 1e-3f;
};

struct Object
{
    int32_t kind = 0;
    std::string name;
    Vec pos, rot;
    bool diel = false;
    float epsr = 4.0f, sigma = 0.0f;
    double freq = 1e9;
    bool stl = false;
    std::vector<float> verts;
    std::vector<int32_t> idx;
    std::vector<std::pair<std::string, double>> params;
};

struct Result
{
    std::vector<Face> faces;
    std::vector<float> faceVals;
    float faceDl = 0.0f;
    std::vector<Vec> triV;
    std::vector<int32_t> triIdx;
    std::vector<float> triMag;
    std::vector<Vec> wirePts;
    std::vector<float> wireMag;
    bool hasPlane = false;
    Grid planeGrid;
    int32_t planeAxis = -1, planeIdx = 0, planeN1 = 0, planeN2 = 0;
    std::vector<float> planeVals;
    bool hasPattern = false;
    int32_t nTheta = 0, nPhi = 0;
    std::vector<float> U;
    float uMax = 0.0f, directivity = 0.0f, peakTheta = 0.0f, peakPhi = 0.0f;
    Vec patCenter;
    float patScale = 1.0f;
    Vec lo, hi;
    bool domainVisible = false;
    std::vector<Vec> probeMarkers;
    Result()
    {
        for (int a = 0; a < 3; ++a)
        {
            lo.v[a] = 1e30f;
            hi.v[a] = -1e30f;
        }
    }
};

struct Curve
{
    std::string name;
    uint32_t color = 0;
    std::vector<double> x, y;
};
struct Page
{
    std::string title, xLabel, yLabel;
    std::vector<Curve> curves;
};
struct Frame
{
    int32_t step = 0, axis = -1, idx = 0, n1 = 0, n2 = 0;
    std::vector<float> js, plane;
};

struct Project
{
    std::vector<std::pair<std::string, std::string>> settings;
    int32_t solver = 0, excitation = 0, waveform = 0, currents = 1, dbRange = 2;
    bool gpu = false, showModel = true, dbScale = true, planeOn = false, meshOn = false;
    std::vector<Object> objects;
    Result result;
    std::vector<Page> pages;
    bool pbValid = false;
    Grid pbGrid;
    float pbDt = 0.0f;
    std::vector<Face> pbFaces;
    std::vector<Frame> frames;
};

// ---- writing (SaveProject, ProjectIO.cpp:137-191) ------------------------
struct Out
{
    std::vector<uint8_t> b;
    void raw(const void *p, size_t n)
    {
        const uint8_t *q = static_cast<const uint8_t *>(p);
        b.insert(b.end(), q, q + n);
    }
    void u8(bool v) { b.push_back(v ? 1 : 0); }
    void i32(int32_t v) { raw(&v, 4); }
    void u32(uint32_t v) { raw(&v, 4); }
    void f32(float v) { raw(&v, 4); }
    void f64(double v) { raw(&v, 8); }
    void str(const std::string &s)
    {
        u32((uint32_t)s.size());
        raw(s.data(), s.size());
    }
    template <class T> void arr(const std::vector<T> &v)
    {
        u32((uint32_t)v.size());
        if (!v.empty()) raw(v.data(), v.size() * sizeof(T));
    }
    void vec(const Vec &v) { raw(v.v, 12); }
    void vecs(const std::vector<Vec> &v)
    {
        u32((uint32_t)v.size());
        for (const Vec &x : v) vec(x);
    }
    void grid(const Grid &g)
    {
        raw(g.n, 12);
        raw(g.origin, 12);
        f32(g.dl);
    }
    void faces(const std::vector<Face> &v)
    {
        u32((uint32_t)v.size());
        for (const Face &f : v)
        {
            i32(f.cell);
            raw(f.c, 12);
            raw(&f.axis, 1);
            raw(&f.sign, 1);
            raw(f.pad, 2);
        }
    }
};

void writeProject(Out &w, const Project &d)
{
    w.raw(kMagic, 8);
    w.u32(kVersion);
    w.u32((uint32_t)d.settings.size());
    for (const auto &kv : d.settings)
    {
        w.str(kv.first);
        w.str(kv.second);
    }
    w.i32(d.solver);
    w.i32(d.excitation);
    w.i32(d.waveform);
    w.i32(d.currents);
    w.i32(d.dbRange);
    w.u8(d.gpu);
    w.u8(d.showModel);
    w.u8(d.dbScale);
    w.u8(d.planeOn);
    w.u8(d.meshOn);
    w.u32((uint32_t)d.objects.size());
    for (const Object &o : d.objects)
    {
        w.i32(o.kind);
        w.str(o.name);
        w.vec(o.pos);
        w.vec(o.rot);
        w.u8(o.diel);
        w.f32(o.epsr);
        w.f32(o.sigma);
        w.f64(o.freq);
        w.u8(o.stl);
        w.arr(o.verts);
        w.arr(o.idx);
        w.u32((uint32_t)o.params.size());
        for (const auto &p : o.params)
        {
            w.str(p.first);
            w.f64(p.second);
        }
    }
    // GLResult (ProjectIO.cpp:83-98)
    const Result &r = d.result;
    w.faces(r.faces);
    w.arr(r.faceVals);
    w.f32(r.faceDl);
    w.vecs(r.triV);
    w.arr(r.triIdx);
    w.arr(r.triMag);
    w.vecs(r.wirePts);
    w.arr(r.wireMag);
    w.u8(r.hasPlane);
    w.grid(r.planeGrid);
    w.i32(r.planeAxis);
    w.i32(r.planeIdx);
    w.i32(r.planeN1);
    w.i32(r.planeN2);
    w.arr(r.planeVals);
    w.u8(r.hasPattern);
    w.i32(r.nTheta);
    w.i32(r.nPhi);
    w.arr(r.U);
    w.f32(r.uMax);
    w.f32(r.directivity);
    w.f32(r.peakTheta);
    w.f32(r.peakPhi);
    w.vec(r.patCenter);
    w.f32(r.patScale);
    w.vec(r.lo);
    w.vec(r.hi);
    w.u8(r.domainVisible);
    w.vecs(r.probeMarkers);
    w.u32((uint32_t)d.pages.size());
    for (const Page &pg : d.pages)
    {
        w.str(pg.title);
        w.str(pg.xLabel);
        w.str(pg.yLabel);
        w.u32((uint32_t)pg.curves.size());
        for (const Curve &c : pg.curves)
        {
            w.str(c.name);
            w.u32(c.color);
            w.arr(c.x);
            w.arr(c.y);
        }
    }
    w.u8(d.pbValid);
    if (d.pbValid)
    {
        w.grid(d.pbGrid);
        w.f32(d.pbDt);
        w.faces(d.pbFaces);
        w.u32((uint32_t)d.frames.size());
        for (const Frame &f : d.frames)  // VizFrame (ProjectIO.cpp:120-125)
        {
            w.i32(f.step);
            w.i32(f.axis);
            w.i32(f.idx);
            w.i32(f.n1);
            w.i32(f.n2);
            w.arr(f.js);
            w.arr(f.plane);
        }
    }
}

// ---- reading (LoadProject, ProjectIO.cpp:194-248) ------------------------
// A short read stores the bytes that remain (as fread does) and fails; every
// later read fails too, so a count cut off by the end of the file is tested
// by its partial value exactly as the reference tests it. The limits and
// messages are the reference's. An element count larger than the bytes left
// fails before anything is allocated.
struct In
{
    const uint8_t *p;
    size_t n, at = 0;
    bool ok = true;
    bool raw(void *dst, size_t k)
    {
        if (!ok) return false;
        if (n - at < k)
        {
            std::memcpy(dst, p + at, n - at);
            at = n;
            ok = false;
            return false;
        }
        std::memcpy(dst, p + at, k);
        at += k;
        return true;
    }
    template <class T> void pod(T &v) { raw(&v, sizeof(T)); }
    void flag(bool &b)
    {
        uint8_t v = 0;
        if (raw(&v, 1)) b = v != 0;
    }
    std::string str()
    {
        uint32_t k = 0;
        pod(k);
        std::string s;
        if (ok && k < 200000000u && k <= n - at)
        {
            s.assign(reinterpret_cast<const char *>(p + at), k);
            at += k;
        }
        else
            ok = false;
        return s;
    }
    bool count(uint32_t &k, size_t elem)
    {
        k = 0;
        pod(k);
        if (ok && (size_t)k * elem < 4000000000u && (size_t)k * elem <= n - at) return true;
        ok = false;
        return false;
    }
    template <class T> void arr(std::vector<T> &v)
    {
        uint32_t k;
        if (!count(k, sizeof(T))) return;
        v.resize(k);
        if (k) raw(v.data(), (size_t)k * sizeof(T));
    }
    void vec(Vec &v) { raw(v.v, 12); }
    void vecs(std::vector<Vec> &v)
    {
        uint32_t k;
        if (!count(k, 12)) return;
        v.resize(k);
        for (Vec &x : v) vec(x);
    }
    void grid(Grid &g)
    {
        uint8_t b[28];
        if (!raw(b, 28)) return;
        std::memcpy(g.n, b, 12);
        std::memcpy(g.origin, b + 12, 12);
        std::memcpy(&g.dl, b + 24, 4);
    }
    void faces(std::vector<Face> &v)
    {
        uint32_t k;
        if (!count(k, 20)) return;
        v.resize(k);
        for (Face &f : v)
        {
            uint8_t b[20];
            if (!raw(b, 20)) return;
            std::memcpy(&f.cell, b, 4);
            std::memcpy(f.c, b + 4, 12);
            std::memcpy(&f.axis, b + 16, 1);
            std::memcpy(&f.sign, b + 17, 1);
            std::memcpy(f.pad, b + 18, 2);
        }
    }
};

// Returns "" on success, else the reference's message.
std::string readProject(In &r, Project &d, uint32_t &ver)
{
    char magic[8];
    r.raw(magic, 8);
    if (!r.ok || std::memcmp(magic, kMagic, 8) != 0) return "not an EMSIM project file";
    ver = 0;
    r.pod(ver);
    if (ver < 1 || ver > kVersion) return "unsupported project version";
    d = Project();
    uint32_t ns = 0;
    r.pod(ns);
    if (ns > 1000) return "corrupt settings";
    d.settings.resize(ns);
    for (auto &kv : d.settings)
    {
        kv.first = r.str();
        kv.second = r.str();
    }
    r.pod(d.solver);
    r.pod(d.excitation);
    r.pod(d.waveform);
    r.pod(d.currents);
    r.pod(d.dbRange);
    uint8_t b[5] = { 0, 0, 0, 0, 0 };
    r.raw(b, 5);
    d.gpu = b[0] != 0;
    d.showModel = b[1] != 0;
    d.dbScale = b[2] != 0;
    d.planeOn = b[3] != 0;
    d.meshOn = b[4] != 0;
    uint32_t no = 0;
    r.pod(no);
    if (no > 100000) return "corrupt object list";
    d.objects.resize(no);
    for (Object &o : d.objects)
    {
        r.pod(o.kind);
        o.name = r.str();
        r.vec(o.pos);
        r.vec(o.rot);
        r.flag(o.diel);
        r.pod(o.epsr);
        r.pod(o.sigma);
        r.pod(o.freq);
        r.flag(o.stl);
        r.arr(o.verts);
        r.arr(o.idx);
        uint32_t np = 0;
        r.pod(np);
        if (np > 100000)
            r.ok = false;
        else if (r.ok)
        {
            o.params.resize(np);
            for (auto &kv : o.params)
            {
                kv.first = r.str();
                r.pod(kv.second);
            }
        }
    }
    Result &g = d.result;
    r.faces(g.faces);
    r.arr(g.faceVals);
    r.pod(g.faceDl);
    r.vecs(g.triV);
    r.arr(g.triIdx);
    r.arr(g.triMag);
    r.vecs(g.wirePts);
    r.arr(g.wireMag);
    r.flag(g.hasPlane);
    r.grid(g.planeGrid);
    r.pod(g.planeAxis);
    r.pod(g.planeIdx);
    r.pod(g.planeN1);
    r.pod(g.planeN2);
    r.arr(g.planeVals);
    r.flag(g.hasPattern);
    r.pod(g.nTheta);
    r.pod(g.nPhi);
    r.arr(g.U);
    r.pod(g.uMax);
    r.pod(g.directivity);
    r.pod(g.peakTheta);
    r.pod(g.peakPhi);
    r.vec(g.patCenter);
    r.pod(g.patScale);
    r.vec(g.lo);
    r.vec(g.hi);
    r.flag(g.domainVisible);
    r.vecs(g.probeMarkers);
    uint32_t npg = 0;
    r.pod(npg);
    if (npg > 1000) return "corrupt plot data";
    d.pages.resize(npg);
    for (Page &pg : d.pages)
    {
        pg.title = r.str();
        pg.xLabel = r.str();
        pg.yLabel = r.str();
        uint32_t nc = 0;
        r.pod(nc);
        if (nc > 1000) return "corrupt curve data";
        pg.curves.resize(nc);
        for (Curve &c : pg.curves)
        {
            c.name = r.str();
            r.pod(c.color);
            r.arr(c.x);
            r.arr(c.y);
        }
    }
    if (ver >= 2)
    {
        uint8_t hpb = 0;
        r.pod(hpb);
        if (hpb)
        {
            d.pbValid = true;
            r.grid(d.pbGrid);
            r.pod(d.pbDt);
            r.faces(d.pbFaces);
            uint32_t nf = 0;
            r.pod(nf);
            if (nf > 10000000u) return "corrupt playback data";
            // every frame holds at least 28 bytes: a count beyond the file
            // fails here instead of allocating
            if (r.ok && (size_t)nf * 28 > r.n - r.at)
                r.ok = false;
            else
            {
                d.frames.resize(nf);
                for (Frame &f : d.frames)
                {
                    r.pod(f.step);
                    r.pod(f.axis);
                    r.pod(f.idx);
                    r.pod(f.n1);
                    r.pod(f.n2);
                    r.arr(f.js);
                    r.arr(f.plane);
                }
            }
        }
    }
    if (!r.ok) return "file truncated or corrupt";
    return "";
}

Face toFace(const emsim_face &f)
{
    Face o;
    o.cell = f.air_cell;
    std::memcpy(o.c, f.center, 12);
    o.axis = f.axis;
    o.sign = f.sign;
    return o;
}
Grid toGrid(const tlm_grid &g)
{
    Grid o;
    o.n[0] = g.nx;
    o.n[1] = g.ny;
    o.n[2] = g.nz;
    std::memcpy(o.origin, g.origin, 12);
    o.dl = g.dl;
    return o;
}
tlm_grid fromGrid(const Grid &g)
{
    tlm_grid o;
    o.nx = g.n[0];
    o.ny = g.n[1];
    o.nz = g.n[2];
    std::memcpy(o.origin, g.origin, 12);
    o.dl = g.dl;
    return o;
}
std::vector<Vec> toVecs(const float *p, uint32_t n)
{
    std::vector<Vec> v(p ? n : 0);
    for (uint32_t i = 0; i < v.size(); ++i) std::memcpy(v[i].v, p + 3 * (size_t)i, 12);
    return v;
}
template <class T> std::vector<T> toVec(const T *p, uint32_t n)
{
    return p ? std::vector<T>(p, p + n) : std::vector<T>();
}

} // namespace

struct emsim_doc
{
    Project p;
    uint32_t fileVersion = kVersion;
    std::string err;
    std::vector<emsim_face> faceView, pbFaceView;  // views handed out by getters
    tlm_status fail(tlm_status s, const std::string &m)
    {
        err = m;
        return s;
    }
};

namespace {

void faceViews(const std::vector<Face> &in, std::vector<emsim_face> &out)
{
    out.resize(in.size());
    for (size_t i = 0; i < in.size(); ++i)
    {
        emsim_face &f = out[i];
        f.air_cell = in[i].cell;
        std::memcpy(f.center, in[i].c, 12);
        f.axis = in[i].axis;
        f.sign = in[i].sign;
    }
}

const float *vecData(const std::vector<Vec> &v) { return v.empty() ? nullptr : v[0].v; }

// Solver access shared by emsim_from_tlm and emsim_from_fdtd.
struct Source
{
    tlm_status (*grid)(void *, tlm_grid *);
    tlm_status (*dt)(void *, float *);
    tlm_status (*faces)(void *, uint64_t *, int *, int *, float *, int, int *);
    tlm_status (*jsNow)(void *, float *, int, int *);
    tlm_status (*jsDft)(void *, float *, float *, float *, int, int *, int *);
    tlm_status (*plane)(void *, float *, size_t, int *, int *, int *, int *);
    tlm_status (*frameCount)(void *, int *);
    tlm_status (*frame)(void *, int, int *, float *, int, float *, size_t, int *, int *, int *, int *);
    tlm_status (*farField)(void *, int, int, float *, float *, float *, float *, float *);
};

tlm_status capture(emsim_doc *d, void *h, const Source &s, const emsim_capture *c, const char *(*errOf)(void *))
{
    if (!d) return TLM_EINVAL;
    if (!h || !c) return d->fail(TLM_EINVAL, "null solver handle or capture options");
    auto solverErr = [&](tlm_status st) { return d->fail(st, std::string("solver: ") + errOf(h)); };
    tlm_grid g;
    tlm_status st = s.grid(h, &g);
    if (st != TLM_OK) return solverErr(st);
    Result r;
    // surface currents (MainUnit.cpp:1033-1045)
    int nf = 0;
    if ((st = s.faces(h, nullptr, nullptr, nullptr, nullptr, 0, &nf)) != TLM_OK) return solverErr(st);
    std::vector<Face> faces(nf);
    if (nf > 0)
    {
        std::vector<uint64_t> cells(nf);
        std::vector<int> axis(nf), sign(nf);
        std::vector<float> ctr(3 * (size_t)nf);
        if ((st = s.faces(h, cells.data(), axis.data(), sign.data(), ctr.data(), nf, &nf)) != TLM_OK)
            return solverErr(st);
        for (int f = 0; f < nf; ++f)
        {
            faces[f].cell = (int32_t)cells[f];
            std::memcpy(faces[f].c, &ctr[3 * (size_t)f], 12);
            faces[f].axis = (int8_t)axis[f];
            faces[f].sign = (int8_t)sign[f];
        }
        std::vector<float> vals(nf);
        int n = 0, samples = 0;
        st = c->js_dft ? s.jsDft(h, vals.data(), nullptr, nullptr, nf, &n, &samples) : s.jsNow(h, vals.data(), nf, &n);
        if (st != TLM_OK) return solverErr(st);
        r.faces = faces;
        r.faceVals = vals;
    }
    r.faceDl = g.dl;
    // cut plane (MainUnit.cpp:1047-1054)
    int axis = -1, index = 0, n1 = 0, n2 = 0;
    if (s.plane(h, nullptr, 0, &axis, &index, &n1, &n2) == TLM_OK && n1 > 0 && n2 > 0)
    {
        r.planeVals.resize((size_t)n1 * n2);
        if ((st = s.plane(h, r.planeVals.data(), r.planeVals.size(), &axis, &index, &n1, &n2)) != TLM_OK)
            return solverErr(st);
        r.hasPlane = true;
        r.planeGrid = toGrid(g);
        r.planeAxis = axis;
        r.planeIdx = index;
        r.planeN1 = n1;
        r.planeN2 = n2;
    }
    // far-field pattern (MainUnit.cpp:2030-2043)
    if (c->n_theta > 0 && c->n_phi > 0)
    {
        r.U.resize((size_t)c->n_theta * c->n_phi);
        st = s.farField(h, c->n_theta, c->n_phi, r.U.data(), &r.uMax, &r.directivity, &r.peakTheta, &r.peakPhi);
        if (st != TLM_OK) return solverErr(st);
        r.hasPattern = true;
        r.nTheta = c->n_theta;
        r.nPhi = c->n_phi;
        const float ext[3] = { g.nx * g.dl, g.ny * g.dl, g.nz * g.dl };
        for (int a = 0; a < 3; ++a) r.patCenter.v[a] = g.origin[a] + ext[a] * 0.5f;
        r.patScale = 0.45f * std::min(std::min(g.nx, g.ny), g.nz) * g.dl;
    }
    // domain box of the grid, shown (MainUnit.cpp:980-983)
    {
        const float ext[3] = { g.nx * g.dl, g.ny * g.dl, g.nz * g.dl };
        for (int a = 0; a < 3; ++a)
        {
            const float p0 = g.origin[a], p1 = g.origin[a] + ext[a];
            r.lo.v[a] = std::min(std::min(r.lo.v[a], p0), p1);
            r.hi.v[a] = std::max(std::max(r.hi.v[a], p0), p1);
        }
        r.domainVisible = true;
    }
    // playback (MainUnit.cpp:2279-2295)
    std::vector<Frame> frames;
    float dt = 0.0f;
    int nfr = 0;
    if (c->playback)
    {
        if ((st = s.frameCount(h, &nfr)) != TLM_OK) return solverErr(st);
        if (nfr > 0 && (st = s.dt(h, &dt)) != TLM_OK) return solverErr(st);
        frames.resize(nfr);
        for (int i = 0; i < nfr; ++i)
        {
            Frame &f = frames[i];
            if ((st = s.frame(h, i, &f.step, nullptr, 0, nullptr, 0, &f.axis, &f.idx, &f.n1, &f.n2)) != TLM_OK)
                return solverErr(st);
            f.js.resize(nf);
            if (f.axis >= 0) f.plane.resize((size_t)f.n1 * f.n2);
            if ((st = s.frame(h, i, &f.step, f.js.data(), nf, f.plane.empty() ? nullptr : f.plane.data(),
                              f.plane.size(), &f.axis, &f.idx, &f.n1, &f.n2)) != TLM_OK)
                return solverErr(st);
        }
    }
    d->p.result = std::move(r);
    if (c->playback && nfr > 0)
    {
        d->p.pbValid = true;
        d->p.pbGrid = toGrid(g);
        d->p.pbDt = dt;
        d->p.pbFaces = faces;
        d->p.frames = std::move(frames);
    }
    return TLM_OK;
}

#define DOC_CHECK(d)                                                                                             \
    do                                                                                                           \
    {                                                                                                            \
        if (!(d)) return TLM_EINVAL;                                                                             \
    } while (0)

} // namespace

extern "C" {

tlm_status emsim_new(emsim_doc **out)
{
    if (!out) return TLM_EINVAL;
    *out = new (std::nothrow) emsim_doc();
    return *out ? TLM_OK : TLM_ENOMEM;
}

tlm_status emsim_load(const char *path, emsim_doc **out, char *err, size_t err_cap)
{
    auto setErr = [&](const char *m) {
        if (err && err_cap)
        {
            std::strncpy(err, m, err_cap - 1);
            err[err_cap - 1] = 0;
        }
    };
    if (!out || !path)
    {
        setErr("null path or output");
        return TLM_EINVAL;
    }
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f)
    {
        setErr("cannot open file");
        return TLM_ENOMEM;
    }
    std::vector<uint8_t> bytes;
    uint8_t buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + k);
    std::fclose(f);
    emsim_doc *d = new (std::nothrow) emsim_doc();
    if (!d)
    {
        setErr("out of host memory");
        return TLM_ENOMEM;
    }
    In r{ bytes.data(), bytes.size() };
    uint32_t ver = 0;
    std::string e;
    try
    {
        e = readProject(r, d->p, ver);
    }
    catch (const std::bad_alloc &)
    {
        e = "file truncated or corrupt";
    }
    if (!e.empty())
    {
        delete d;
        setErr(e.c_str());
        return TLM_EINVAL;
    }
    d->fileVersion = ver;
    setErr("");
    *out = d;
    return TLM_OK;
}

tlm_status emsim_save(emsim_doc *d, const char *path)
{
    DOC_CHECK(d);
    if (!path) return d->fail(TLM_EINVAL, "null path");
    Out w;
    writeProject(w, d->p);
    FILE *f = std::fopen(path, "wb");
    if (!f) return d->fail(TLM_EINVAL, std::string("cannot write ") + path);
    const bool ok = std::fwrite(w.b.data(), 1, w.b.size(), f) == w.b.size();
    if (std::fclose(f) != 0 || !ok) return d->fail(TLM_EINVAL, std::string("write to ") + path + " failed");
    return TLM_OK;
}

void emsim_free(emsim_doc *d) { delete d; }
const char *emsim_last_error(emsim_doc *d) { return d ? d->err.c_str() : "null document"; }
int emsim_file_version(emsim_doc *d) { return d ? (int)d->fileVersion : 0; }

// ---- settings, toolbar ---------------------------------------------------
int emsim_setting_count(emsim_doc *d) { return d ? (int)d->p.settings.size() : 0; }
tlm_status emsim_get_setting(emsim_doc *d, int i, const char **key, const char **value)
{
    DOC_CHECK(d);
    if (i < 0 || i >= (int)d->p.settings.size()) return d->fail(TLM_EINVAL, "no such setting");
    if (key) *key = d->p.settings[i].first.c_str();
    if (value) *value = d->p.settings[i].second.c_str();
    return TLM_OK;
}
tlm_status emsim_add_setting(emsim_doc *d, const char *key, const char *value)
{
    DOC_CHECK(d);
    if (!key || !value) return d->fail(TLM_EINVAL, "null key or value");
    if (d->p.settings.size() >= 1000) return d->fail(TLM_EINVAL, "a project holds at most 1000 settings");
    d->p.settings.emplace_back(key, value);
    return TLM_OK;
}
tlm_status emsim_clear_settings(emsim_doc *d)
{
    DOC_CHECK(d);
    d->p.settings.clear();
    return TLM_OK;
}
tlm_status emsim_get_toolbar(emsim_doc *d, emsim_toolbar *t)
{
    DOC_CHECK(d);
    if (!t) return d->fail(TLM_EINVAL, "null output");
    const Project &p = d->p;
    *t = emsim_toolbar{ p.solver, p.excitation, p.waveform, p.currents, p.dbRange,
                        p.gpu,    p.showModel,  p.dbScale,  p.planeOn,  p.meshOn };
    return TLM_OK;
}
tlm_status emsim_set_toolbar(emsim_doc *d, const emsim_toolbar *t)
{
    DOC_CHECK(d);
    if (!t) return d->fail(TLM_EINVAL, "null toolbar");
    Project &p = d->p;
    p.solver = t->solver;
    p.excitation = t->excitation;
    p.waveform = t->waveform;
    p.currents = t->currents;
    p.dbRange = t->db_range;
    p.gpu = t->gpu != 0;
    p.showModel = t->show_model != 0;
    p.dbScale = t->db_scale != 0;
    p.planeOn = t->plane_on != 0;
    p.meshOn = t->mesh_on != 0;
    return TLM_OK;
}

// ---- objects -------------------------------------------------------------
int emsim_object_count(emsim_doc *d) { return d ? (int)d->p.objects.size() : 0; }
tlm_status emsim_get_object(emsim_doc *d, int i, emsim_object *o)
{
    DOC_CHECK(d);
    if (!o || i < 0 || i >= (int)d->p.objects.size()) return d->fail(TLM_EINVAL, "no such object");
    const Object &s = d->p.objects[i];
    o->kind = s.kind;
    o->name = s.name.c_str();
    std::memcpy(o->position, s.pos.v, 12);
    std::memcpy(o->rot_deg, s.rot.v, 12);
    o->dielectric = s.diel;
    o->epsr = s.epsr;
    o->sigma = s.sigma;
    o->design_freq_hz = s.freq;
    o->is_stl = s.stl;
    o->n_stl_verts = (uint32_t)s.verts.size();
    o->stl_verts = s.verts.empty() ? nullptr : s.verts.data();
    o->n_stl_idx = (uint32_t)s.idx.size();
    o->stl_idx = s.idx.empty() ? nullptr : s.idx.data();
    o->n_params = (uint32_t)s.params.size();
    return TLM_OK;
}
tlm_status emsim_get_object_param(emsim_doc *d, int i, int p, const char **name, double *value)
{
    DOC_CHECK(d);
    if (i < 0 || i >= (int)d->p.objects.size() || p < 0 || p >= (int)d->p.objects[i].params.size())
        return d->fail(TLM_EINVAL, "no such object parameter");
    if (name) *name = d->p.objects[i].params[p].first.c_str();
    if (value) *value = d->p.objects[i].params[p].second;
    return TLM_OK;
}
tlm_status emsim_add_object(emsim_doc *d, const emsim_object *o, int *idx)
{
    DOC_CHECK(d);
    if (!o) return d->fail(TLM_EINVAL, "null object");
    if (d->p.objects.size() >= 100000) return d->fail(TLM_EINVAL, "a project holds at most 100000 objects");
    Object s;
    s.kind = o->kind;
    s.name = o->name ? o->name : "";
    std::memcpy(s.pos.v, o->position, 12);
    std::memcpy(s.rot.v, o->rot_deg, 12);
    s.diel = o->dielectric != 0;
    s.epsr = o->epsr;
    s.sigma = o->sigma;
    s.freq = o->design_freq_hz;
    s.stl = o->is_stl != 0;
    s.verts = toVec(o->stl_verts, o->n_stl_verts);
    s.idx = toVec(o->stl_idx, o->n_stl_idx);
    d->p.objects.push_back(std::move(s));
    if (idx) *idx = (int)d->p.objects.size() - 1;
    return TLM_OK;
}
tlm_status emsim_add_object_param(emsim_doc *d, int i, const char *name, double value)
{
    DOC_CHECK(d);
    if (i < 0 || i >= (int)d->p.objects.size() || !name) return d->fail(TLM_EINVAL, "no such object or null name");
    if (d->p.objects[i].params.size() >= 100000) return d->fail(TLM_EINVAL, "at most 100000 parameters");
    d->p.objects[i].params.emplace_back(name, value);
    return TLM_OK;
}
tlm_status emsim_clear_objects(emsim_doc *d)
{
    DOC_CHECK(d);
    d->p.objects.clear();
    return TLM_OK;
}

// ---- result --------------------------------------------------------------
void emsim_result_default(emsim_result *r)
{
    if (!r) return;
    std::memset(r, 0, sizeof *r);
    r->plane_axis = -1;
    r->plane_grid.dl = 1e-3f;
    r->pat_scale = 1.0f;
    for (int a = 0; a < 3; ++a)
    {
        r->domain_lo[a] = 1e30f;
        r->domain_hi[a] = -1e30f;
    }
}
tlm_status emsim_get_result(emsim_doc *d, emsim_result *o)
{
    DOC_CHECK(d);
    if (!o) return d->fail(TLM_EINVAL, "null output");
    const Result &r = d->p.result;
    faceViews(r.faces, d->faceView);
    o->n_faces = (uint32_t)r.faces.size();
    o->faces = d->faceView.empty() ? nullptr : d->faceView.data();
    o->n_face_vals = (uint32_t)r.faceVals.size();
    o->face_vals = r.faceVals.empty() ? nullptr : r.faceVals.data();
    o->face_dl = r.faceDl;
    o->n_tri_v = (uint32_t)r.triV.size();
    o->tri_v = vecData(r.triV);
    o->n_tri_idx = (uint32_t)r.triIdx.size();
    o->tri_idx = r.triIdx.empty() ? nullptr : r.triIdx.data();
    o->n_tri_mag = (uint32_t)r.triMag.size();
    o->tri_mag = r.triMag.empty() ? nullptr : r.triMag.data();
    o->n_wire_pts = (uint32_t)r.wirePts.size();
    o->wire_pts = vecData(r.wirePts);
    o->n_wire_mag = (uint32_t)r.wireMag.size();
    o->wire_mag = r.wireMag.empty() ? nullptr : r.wireMag.data();
    o->has_plane = r.hasPlane;
    o->plane_grid = fromGrid(r.planeGrid);
    o->plane_axis = r.planeAxis;
    o->plane_index = r.planeIdx;
    o->plane_n1 = r.planeN1;
    o->plane_n2 = r.planeN2;
    o->n_plane_vals = (uint32_t)r.planeVals.size();
    o->plane_vals = r.planeVals.empty() ? nullptr : r.planeVals.data();
    o->has_pattern = r.hasPattern;
    o->pattern.n_theta = r.nTheta;
    o->pattern.n_phi = r.nPhi;
    o->pattern.n_u = (uint32_t)r.U.size();
    o->pattern.U = r.U.empty() ? nullptr : r.U.data();
    o->pattern.u_max = r.uMax;
    o->pattern.directivity = r.directivity;
    o->pattern.peak_theta_deg = r.peakTheta;
    o->pattern.peak_phi_deg = r.peakPhi;
    std::memcpy(o->pat_center, r.patCenter.v, 12);
    o->pat_scale = r.patScale;
    std::memcpy(o->domain_lo, r.lo.v, 12);
    std::memcpy(o->domain_hi, r.hi.v, 12);
    o->domain_visible = r.domainVisible;
    o->n_probe_markers = (uint32_t)r.probeMarkers.size();
    o->probe_markers = vecData(r.probeMarkers);
    return TLM_OK;
}
tlm_status emsim_set_result(emsim_doc *d, const emsim_result *s)
{
    DOC_CHECK(d);
    if (!s) return d->fail(TLM_EINVAL, "null result");
    Result r;
    if (s->faces)
        for (uint32_t i = 0; i < s->n_faces; ++i) r.faces.push_back(toFace(s->faces[i]));
    r.faceVals = toVec(s->face_vals, s->n_face_vals);
    r.faceDl = s->face_dl;
    r.triV = toVecs(s->tri_v, s->n_tri_v);
    r.triIdx = toVec(s->tri_idx, s->n_tri_idx);
    r.triMag = toVec(s->tri_mag, s->n_tri_mag);
    r.wirePts = toVecs(s->wire_pts, s->n_wire_pts);
    r.wireMag = toVec(s->wire_mag, s->n_wire_mag);
    r.hasPlane = s->has_plane != 0;
    r.planeGrid = toGrid(s->plane_grid);
    r.planeAxis = s->plane_axis;
    r.planeIdx = s->plane_index;
    r.planeN1 = s->plane_n1;
    r.planeN2 = s->plane_n2;
    r.planeVals = toVec(s->plane_vals, s->n_plane_vals);
    r.hasPattern = s->has_pattern != 0;
    r.nTheta = s->pattern.n_theta;
    r.nPhi = s->pattern.n_phi;
    r.U = toVec(s->pattern.U, s->pattern.n_u);
    r.uMax = s->pattern.u_max;
    r.directivity = s->pattern.directivity;
    r.peakTheta = s->pattern.peak_theta_deg;
    r.peakPhi = s->pattern.peak_phi_deg;
    std::memcpy(r.patCenter.v, s->pat_center, 12);
    r.patScale = s->pat_scale;
    std::memcpy(r.lo.v, s->domain_lo, 12);
    std::memcpy(r.hi.v, s->domain_hi, 12);
    r.domainVisible = s->domain_visible != 0;
    r.probeMarkers = toVecs(s->probe_markers, s->n_probe_markers);
    d->p.result = std::move(r);
    return TLM_OK;
}

// ---- pages ---------------------------------------------------------------
int emsim_page_count(emsim_doc *d) { return d ? (int)d->p.pages.size() : 0; }
tlm_status emsim_get_page(emsim_doc *d, int i, const char **title, const char **x_label, const char **y_label,
                          int *n_curves)
{
    DOC_CHECK(d);
    if (i < 0 || i >= (int)d->p.pages.size()) return d->fail(TLM_EINVAL, "no such page");
    const Page &pg = d->p.pages[i];
    if (title) *title = pg.title.c_str();
    if (x_label) *x_label = pg.xLabel.c_str();
    if (y_label) *y_label = pg.yLabel.c_str();
    if (n_curves) *n_curves = (int)pg.curves.size();
    return TLM_OK;
}
tlm_status emsim_get_curve(emsim_doc *d, int page, int c, emsim_curve *o)
{
    DOC_CHECK(d);
    if (!o || page < 0 || page >= (int)d->p.pages.size() || c < 0 || c >= (int)d->p.pages[page].curves.size())
        return d->fail(TLM_EINVAL, "no such curve");
    const Curve &s = d->p.pages[page].curves[c];
    o->name = s.name.c_str();
    o->color = s.color;
    o->n_x = (uint32_t)s.x.size();
    o->x = s.x.empty() ? nullptr : s.x.data();
    o->n_y = (uint32_t)s.y.size();
    o->y = s.y.empty() ? nullptr : s.y.data();
    return TLM_OK;
}
tlm_status emsim_add_page(emsim_doc *d, const char *title, const char *x_label, const char *y_label, int *idx)
{
    DOC_CHECK(d);
    if (d->p.pages.size() >= 1000) return d->fail(TLM_EINVAL, "a project holds at most 1000 plot pages");
    Page pg;
    pg.title = title ? title : "";
    pg.xLabel = x_label ? x_label : "";
    pg.yLabel = y_label ? y_label : "";
    d->p.pages.push_back(std::move(pg));
    if (idx) *idx = (int)d->p.pages.size() - 1;
    return TLM_OK;
}
tlm_status emsim_add_curve(emsim_doc *d, int page, const emsim_curve *c)
{
    DOC_CHECK(d);
    if (!c || page < 0 || page >= (int)d->p.pages.size()) return d->fail(TLM_EINVAL, "no such page or null curve");
    if (d->p.pages[page].curves.size() >= 1000) return d->fail(TLM_EINVAL, "a page holds at most 1000 curves");
    Curve s;
    s.name = c->name ? c->name : "";
    s.color = c->color;
    s.x = toVec(c->x, c->n_x);
    s.y = toVec(c->y, c->n_y);
    d->p.pages[page].curves.push_back(std::move(s));
    return TLM_OK;
}
tlm_status emsim_clear_pages(emsim_doc *d)
{
    DOC_CHECK(d);
    d->p.pages.clear();
    return TLM_OK;
}

// ---- playback ------------------------------------------------------------
tlm_status emsim_get_playback(emsim_doc *d, int *valid, tlm_grid *grid, float *dt, const emsim_face **faces,
                              uint32_t *n_faces, uint32_t *n_frames)
{
    DOC_CHECK(d);
    faceViews(d->p.pbFaces, d->pbFaceView);
    if (valid) *valid = d->p.pbValid;
    if (grid) *grid = fromGrid(d->p.pbGrid);
    if (dt) *dt = d->p.pbDt;
    if (faces) *faces = d->pbFaceView.empty() ? nullptr : d->pbFaceView.data();
    if (n_faces) *n_faces = (uint32_t)d->p.pbFaces.size();
    if (n_frames) *n_frames = (uint32_t)d->p.frames.size();
    return TLM_OK;
}
tlm_status emsim_set_playback(emsim_doc *d, const tlm_grid *grid, float dt, const emsim_face *faces,
                              uint32_t n_faces)
{
    DOC_CHECK(d);
    if (!grid || (n_faces && !faces)) return d->fail(TLM_EINVAL, "null grid or faces");
    d->p.pbValid = true;
    d->p.pbGrid = toGrid(*grid);
    d->p.pbDt = dt;
    d->p.pbFaces.clear();
    for (uint32_t i = 0; i < n_faces; ++i) d->p.pbFaces.push_back(toFace(faces[i]));
    d->p.frames.clear();
    return TLM_OK;
}
tlm_status emsim_get_frame(emsim_doc *d, uint32_t i, emsim_frame *o)
{
    DOC_CHECK(d);
    if (!o || i >= d->p.frames.size()) return d->fail(TLM_EINVAL, "no such frame");
    const Frame &f = d->p.frames[i];
    o->step = f.step;
    o->plane_axis = f.axis;
    o->plane_index = f.idx;
    o->plane_n1 = f.n1;
    o->plane_n2 = f.n2;
    o->n_js = (uint32_t)f.js.size();
    o->js = f.js.empty() ? nullptr : f.js.data();
    o->n_plane = (uint32_t)f.plane.size();
    o->plane = f.plane.empty() ? nullptr : f.plane.data();
    return TLM_OK;
}
tlm_status emsim_add_frame(emsim_doc *d, const emsim_frame *f)
{
    DOC_CHECK(d);
    if (!f) return d->fail(TLM_EINVAL, "null frame");
    if (!d->p.pbValid) return d->fail(TLM_ESTATE, "emsim_set_playback has not been called");
    if (d->p.frames.size() >= 10000000u) return d->fail(TLM_EINVAL, "a project holds at most 10^7 frames");
    Frame s;
    s.step = f->step;
    s.axis = f->plane_axis;
    s.idx = f->plane_index;
    s.n1 = f->plane_n1;
    s.n2 = f->plane_n2;
    s.js = toVec(f->js, f->n_js);
    s.plane = toVec(f->plane, f->n_plane);
    d->p.frames.push_back(std::move(s));
    return TLM_OK;
}
tlm_status emsim_clear_playback(emsim_doc *d)
{
    DOC_CHECK(d);
    d->p.pbValid = false;
    d->p.pbGrid = Grid();
    d->p.pbDt = 0.0f;
    d->p.pbFaces.clear();
    d->p.frames.clear();
    return TLM_OK;
}

// ---- capture from a solver -----------------------------------------------
tlm_status emsim_from_tlm(emsim_doc *d, tlm_handle h, const emsim_capture *c)
{
    Source s;
    s.grid = [](void *x, tlm_grid *g) { return tlm_get_grid((tlm_handle)x, g); };
    s.dt = [](void *x, float *dt) { return tlm_timestep((tlm_handle)x, dt); };
    s.faces = [](void *x, uint64_t *a, int *b, int *c2, float *e, int cap, int *n) {
        return tlm_get_surface_faces((tlm_handle)x, a, b, c2, e, cap, n);
    };
    s.jsNow = [](void *x, float *o, int cap, int *n) { return tlm_get_js_instant((tlm_handle)x, o, cap, n); };
    s.jsDft = [](void *x, float *m, float *re, float *im, int cap, int *n, int *ns) {
        return tlm_get_js_dft((tlm_handle)x, m, re, im, cap, n, ns);
    };
    s.plane = [](void *x, float *o, size_t cap, int *a, int *i, int *n1, int *n2) {
        return tlm_get_field_plane((tlm_handle)x, o, cap, a, i, n1, n2);
    };
    s.frameCount = [](void *x, int *n) { return tlm_frame_count((tlm_handle)x, n); };
    s.frame = [](void *x, int i, int *st, float *js, int jc, float *pl, size_t pc, int *a, int *ix, int *n1,
                 int *n2) { return tlm_get_frame((tlm_handle)x, i, st, js, jc, pl, pc, a, ix, n1, n2); };
    s.farField = [](void *x, int nt, int np, float *U, float *um, float *dir, float *pt, float *pp) {
        return tlm_compute_far_field((tlm_handle)x, nt, np, U, um, dir, pt, pp);
    };
    return capture(d, h, s, c, [](void *x) { return tlm_last_error((tlm_handle)x); });
}

tlm_status emsim_from_fdtd(emsim_doc *d, fdtd_handle h, const emsim_capture *c)
{
    Source s;
    s.grid = [](void *x, tlm_grid *g) { return fdtd_get_grid((fdtd_handle)x, g); };
    s.dt = [](void *x, float *dt) {
        *dt = fdtd_timestep((fdtd_handle)x);
        return (tlm_status)TLM_OK;
    };
    s.faces = [](void *x, uint64_t *a, int *b, int *c2, float *e, int cap, int *n) {
        return fdtd_get_surface_faces((fdtd_handle)x, a, b, c2, e, cap, n);
    };
    s.jsNow = [](void *x, float *o, int cap, int *n) { return fdtd_get_js_instant((fdtd_handle)x, o, cap, n); };
    s.jsDft = [](void *x, float *m, float *re, float *im, int cap, int *n, int *ns) {
        return fdtd_get_js_dft((fdtd_handle)x, m, re, im, cap, n, ns);
    };
    s.plane = [](void *x, float *o, size_t cap, int *a, int *i, int *n1, int *n2) {
        return fdtd_get_field_plane((fdtd_handle)x, o, cap, a, i, n1, n2);
    };
    s.frameCount = [](void *x, int *n) { return fdtd_frame_count((fdtd_handle)x, n); };
    s.frame = [](void *x, int i, int *st, float *js, int jc, float *pl, size_t pc, int *a, int *ix, int *n1,
                 int *n2) { return fdtd_get_frame((fdtd_handle)x, i, st, js, jc, pl, pc, a, ix, n1, n2); };
    s.farField = [](void *x, int nt, int np, float *U, float *um, float *dir, float *pt, float *pp) {
        return fdtd_compute_far_field((fdtd_handle)x, nt, np, U, um, dir, pt, pp);
    };
    return capture(d, h, s, c, [](void *x) { return fdtd_last_error((fdtd_handle)x); });
}

} // extern "C"
