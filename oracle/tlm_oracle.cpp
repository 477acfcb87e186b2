// tlm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A single-threaded CPU restatement of the reference's symmetrical-condensed-
// node (SCN) TLM time step (smilima/EMSolver, TlmSolver.cpp), templated on the
// arithmetic type:
//   * real = float  must agree BITWISE with the reference's own CPU step
//     (compiled headless under oracle/_ref). The float arithmetic below keeps
//     the reference's operation order and is compiled with -ffp-contract=off,
//     like the reference on x86-64 without -march.
//   * real = double is the FP64 oracle that the reduced-precision pulse
//     storage modes are measured against.
// Only tests/, the smoke check and the bench's CPU-baseline leg load this
// library, and only as the checker; the product never calls it.
//
// Structure (deliberately not the reference's in-place loops): the state is
// the incident pulse array `inc` (same AoS layout as the reference's V:
// cell*12 + slot), one step computes inject -> monitors -> scatter into a
// separate `refl` array -> connect back into `inc` as a pure gather.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// Physical constants exactly as the reference declares them (float literals,
// TlmSolver.cpp:15-16); the FP64 oracle promotes the same float values so that
// both solve the same discrete problem.
const float kC0f = 299792458.0f;
const float kEta0f = 376.730313f;
const double kPi = 3.14159265358979323846;

enum { kAir = 0, kPec = 1, kDiel0 = 2 };   // TlmSolver.h:59

// Slot numbering of the 12 link pulses (TlmSolver.cpp:19-29): a link on
// `axis`, face `side` (0 = -, 1 = +), carrying the E component `field`,
// lives in slot axis*4 + side*2 + (field is the first of the axis's two
// transverse axes ? 0 : 1). Transverse pairs: x:(y,z) y:(x,z) z:(x,y).
inline int firstTransverse(int axis) { return axis == 0 ? 1 : 0; }
inline int secondTransverse(int axis) { return axis == 2 ? 1 : 2; }
inline int slot(int axis, int side, int field)
{
    return axis * 4 + side * 2 + (field == firstTransverse(axis) ? 0 : 1);
}

// Node voltage of polarisation j from the four links that carry E_j
// (TlmSolver.cpp:46-52): 0.5 * (((a- + a+) + b-) + b+), a < b the two axes
// other than j.
template <class T> inline T nodeVoltage(const T *v, int j)
{
    int a = (j == 0) ? 1 : 0;
    int b = (j == 2) ? 1 : 2;
    return T(0.5) * (v[slot(a, 0, j)] + v[slot(a, 1, j)] + v[slot(b, 0, j)] +
                     v[slot(b, 1, j)]);
}

// Link-line circulation about axis k (TlmSolver.cpp:33-42): with (p, q) the
// cyclic pair for which e_p x e_q = e_k,
// 0.5 * (((v[p,-,q] - v[p,+,q]) - v[q,-,p]) + v[q,+,p]).
template <class T> inline T circulation(const T *v, int k)
{
    int p = (k + 1) % 3, q = (k + 2) % 3;
    return T(0.5) * (v[slot(p, 0, q)] - v[slot(p, 1, q)] - v[slot(q, 0, p)] +
                     v[slot(q, 1, p)]);
}

// Reflected pulses from node quantities (TlmSolver.cpp:59-76, field form):
// out[i,s,j] = (Vj +/- ZI_k) - in[i,1-s,j], k the third axis. The sign is +
// when (j follows i cyclically) == (s is the + face). The reference writes
// Vj + sg*ZI_k with sg = +/-1; multiplying by +/-1 is exact and
// x + (-y) == x - y in IEEE arithmetic, so both forms round identically.
template <class T>
inline void reflectLinks(const T *in, const T Vn[3], const T ZI[3], T *out)
{
    for (int i = 0; i < 3; ++i)
        for (int s = 0; s < 2; ++s)
            for (int t = 0; t < 2; ++t)
            {
                int j = t == 0 ? firstTransverse(i) : secondTransverse(i);
                int k = 3 - i - j;
                bool plus = ((j == (i + 1) % 3) == (s == 1));
                T base = plus ? (Vn[j] + ZI[k]) : (Vn[j] - ZI[k]);
                out[i * 4 + s * 2 + t] = base - in[slot(i, 1 - s, j)];
            }
}

template <class T> inline void scatterAir(const T *in, T *out)
{
    T Vn[3], ZI[3];
    for (int j = 0; j < 3; ++j) Vn[j] = nodeVoltage(in, j);
    for (int k = 0; k < 3; ++k) ZI[k] = circulation(in, k);
    reflectLinks(in, Vn, ZI, out);
}

// Stub-loaded node (TlmSolver.cpp:78-113): three open-circuit permittivity
// stubs of normalised admittance yh and a shunt loss gh;
// Vj = (2 * (sum4 + yh*vs_j)) / ((4 + yh) + gh), links reflect as in air,
// and each stub's reflected pulse Vj - vs_j returns next step.
template <class T>
inline void scatterStub(const T *in, T *vs, T yh, T gh, T *out)
{
    T Vn[3], ZI[3];
    T den = T(4) + yh + gh;
    for (int j = 0; j < 3; ++j)
    {
        int a = (j == 0) ? 1 : 0;
        int b = (j == 2) ? 1 : 2;
        T sum4 = in[slot(a, 0, j)] + in[slot(a, 1, j)] + in[slot(b, 0, j)] +
                 in[slot(b, 1, j)];
        T load = yh * vs[j];
        Vn[j] = (T(2) * (sum4 + load)) / den;
    }
    for (int k = 0; k < 3; ++k) ZI[k] = circulation(in, k);
    reflectLinks(in, Vn, ZI, out);
    for (int j = 0; j < 3; ++j) vs[j] = Vn[j] - vs[j];
}

struct Port
{
    std::vector<size_t> cells;
    int pol = 2;
    float amp = 1.0f;
    std::vector<double> v, i;
};
struct Probe
{
    size_t cell = 0;
    std::vector<double> ex, ey, ez;
};
struct Source
{
    size_t cell;
    int pol;
    float amp;
};

class OracleBase
{
public:
    virtual ~OracleBase() {}
    virtual int setup(int nx, int ny, int nz, float ox, float oy, float oz, float dl,
                      const uint8_t *mat, const float *epsr, const float *sigma,
                      int ntab, float f0, int waveform, int total, int settle,
                      float rho) = 0;
    virtual int addPort(const uint64_t *cells, int n, int pol, float amp) = 0;
    virtual int addProbe(float x, float y, float z) = 0;
    virtual void addPlaneWave(int prop, int plane, int pol, float amp) = 0;
    virtual double waveform(int n) const = 0;
    virtual void step(int n, bool haveSv, double sv) = 0;
    virtual size_t getPulses(double *out, size_t cap) const = 0;
    virtual size_t setPulses(const double *in, size_t n) = 0;
    virtual size_t getStubs(double *out, size_t cap) const = 0;
    virtual int getTables(double *y, double *g, int cap) const = 0;
    virtual int probeCount() const = 0;
    virtual int getProbe(int idx, double *ex, double *ey, double *ez, int cap,
                         uint64_t *cell) const = 0;
    virtual int portCount() const = 0;
    virtual int getPort(int idx, double *v, double *i, int cap) const = 0;
    virtual int energyHistory(int *steps, double *vals, int cap) const = 0;
    virtual double dt() const = 0;
    // surface monitors (TlmSolver.cpp:303-348, 616-675, 715-763, 805-916)
    virtual int configureSurface(int huyOffset, int recordEvery) = 0;
    virtual void setFieldPlane(int axis, int index) = 0;
    virtual int surfaceFaces(uint64_t *cells, int *axis, int *sign, float *center, int cap) const = 0;
    virtual int jsInstant(double *out, int cap) const = 0;
    virtual int jsDft(double *re, double *im, double *mag, int cap, int *samples) const = 0;
    virtual int huygensFaces(uint64_t *cells, int *axis, int *outSign, float *pos, int cap) const = 0;
    virtual int huygensDft(double *acc, int cap, int *samples) const = 0;
    virtual int fieldPlane(double *out, size_t cap, int *axis, int *index, int *n1, int *n2) const = 0;
    virtual int frameCount() const = 0;
    virtual int getFrame(int idx, int *step, double *js, int jsCap, double *plane, size_t planeCap,
                         int *axis, int *pidx, int *n1, int *n2) const = 0;
    virtual int farField(int nTheta, int nPhi, double *U, double *uMax, double *directivity,
                         double *peakTheta, double *peakPhi) const = 0;
};

template <class T> class Oracle : public OracleBase
{
public:
    int setup(int nx_, int ny_, int nz_, float ox, float oy, float oz, float dl_,
              const uint8_t *mat_, const float *epsr, const float *sigma, int ntab,
              float f0_, int waveform_, int total, int settle, float rho_) override
    {
        if (nx_ <= 0 || ny_ <= 0 || nz_ <= 0) return -1;
        nx = nx_; ny = ny_; nz = nz_;
        origin[0] = ox; origin[1] = oy; origin[2] = oz;
        dl = dl_;
        f0 = f0_;
        wave = waveform_;
        totalSteps = total;
        settleSteps = settle;
        rho = T(rho_);
        n = (size_t)nx * ny * nz;
        mat.assign(mat_, mat_ + n);
        // setup tables (TlmSolver.cpp:268-283)
        timeStep = T(dl) / (T(2) * T(kC0f));
        yhat.clear();
        ghat.clear();
        for (int t = 0; t < ntab; ++t)
        {
            T er = T(epsr[t]), sg = T(sigma[t]);
            yhat.push_back(T(4) * (std::max(T(1), er) - T(1)));
            ghat.push_back(std::max(T(0), sg) * T(dl) * T(kEta0f));
        }
        bool anyDiel = false;
        for (uint8_t m : mat)
        {
            if (m >= kDiel0)
            {
                anyDiel = true;
                if ((int)(m - kDiel0) >= ntab) return -2;   // id without a table entry
            }
        }
        inc.assign(n * 12, T(0));
        refl.assign(n * 12, T(0));
        stubs.assign(anyDiel ? n * 3 : 0, T(0));
        ports.clear();
        probes.clear();
        sources.clear();
        energySteps.clear();
        energyVals.clear();
        huyOffset = 0;
        recordEvery = 0;
        planeAxis = -1;
        planeIndex = 0;
        buildSurfaceFaces();
        buildHuygens();
        return 0;
    }

    // Huygens box inset and playback-frame period (TlmConfig::huyOffset,
    // recordEvery, TlmSolver.h:120-122); rebuilds the Huygens face list.
    int configureSurface(int huyOffset_, int recordEvery_) override
    {
        huyOffset = huyOffset_;
        recordEvery = recordEvery_;
        buildHuygens();
        return 0;
    }
    void setFieldPlane(int axis, int index) override
    {
        planeAxis = axis;
        planeIndex = index;
    }

    // Lumped port (TlmSolver.cpp:362-374): cells that are out of range or not
    // air are dropped silently, as the reference does.
    int addPort(const uint64_t *cells, int cnt, int pol, float amp) override
    {
        Port p;
        p.pol = pol;
        p.amp = amp;
        for (int t = 0; t < cnt; ++t)
            if (cells[t] < n && mat[cells[t]] == kAir) p.cells.push_back(cells[t]);
        // The current loop reads the 4 transverse linear-index neighbours of
        // the middle gap cell; the reference does not check them
        // (TlmSolver.cpp:687-698). A port whose loop would leave the array is
        // refused here (-1), the same rule the product applies.
        if (!p.cells.empty())
        {
            const size_t stride[3] = { 1, (size_t)nx, (size_t)nx * ny };
            size_t c = p.cells[p.cells.size() / 2];
            size_t s1 = stride[(pol + 1) % 3], s2 = stride[(pol + 2) % 3];
            if (c + s1 >= n || c < s1 || c + s2 >= n || c < s2) return -1;
        }
        ports.push_back(p);
        return (int)ports.size() - 1;
    }

    // E probe at a world point (TlmSolver.cpp:377-391, Geometry.h:107-112):
    // floor((p - origin)/dl) per axis in float, -1 outside the grid.
    int addProbe(float x, float y, float z) override
    {
        float p[3] = { x, y, z };
        int c[3];
        int dims[3] = { nx, ny, nz };
        for (int a = 0; a < 3; ++a)
        {
            c[a] = (int)std::floor((p[a] - origin[a]) / dl);
            if (c[a] < 0 || c[a] >= dims[a]) return -1;
        }
        Probe pr;
        pr.cell = ((size_t)c[2] * ny + c[1]) * nx + c[0];
        probes.push_back(pr);
        return (int)probes.size() - 1;
    }

    // Plane-wave soft source over the air cells of one plane
    // (TlmSolver.cpp:394-407), in the reference's cell order.
    void addPlaneWave(int prop, int plane, int pol, float amp) override
    {
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                {
                    int co[3] = { i, j, k };
                    if (co[prop] != plane) continue;
                    size_t c = ((size_t)k * ny + j) * nx + i;
                    if (mat[c] == kAir) sources.push_back({ c, pol, amp });
                }
    }

    // Source waveforms (TlmSolver.cpp:410-436).
    double waveform(int step) const override
    {
        T t = T(step) * timeStep;
        T pi = T(kPi);
        T F = T(f0);
        T w = T(2) * pi * F;
        switch (wave)
        {
        case 0:
        {
            T Tr = T(3) / F;
            T r = (t < Tr) ? T(0.5) * (T(1) - std::cos(pi * t / Tr)) : T(1);
            return (double)(r * std::sin(w * t));
        }
        case 1:
        {
            T tau = T(2) / F, t0 = T(3) * tau;
            T u = (t - t0) / tau;
            return (double)(std::exp(-u * u) * std::sin(w * (t - t0)));
        }
        default:
        {
            T tau = T(0.5) / F, t0 = T(3) * tau;
            T u = (t - t0) / tau;
            return (double)std::exp(-u * u);
        }
        }
    }

    void step(int stepIndex, bool haveSv, double svIn) override
    {
        T sv = haveSv ? T(svIn) : T(waveform(stepIndex));
        // 1. soft sources: plane-wave cells first, then port cells, each in
        //    registration order (TlmSolver.cpp:487-505).
        for (const Source &s : sources) inject(s.cell, s.pol, s.amp, sv);
        for (const Port &p : ports)
            for (size_t c : p.cells) inject(c, p.pol, p.amp, sv);
        // 2. monitors on the incident pulses after injection.
        sample(stepIndex);
        // 3. scatter every non-PEC node into `refl` (TlmSolver.cpp:516-548).
        for (size_t c = 0; c < n; ++c)
        {
            const T *in = &inc[c * 12];
            T *out = &refl[c * 12];
            uint8_t m = mat[c];
            if (m == kPec)
            {
                std::fill(out, out + 12, T(0));
                continue;
            }
            if (m >= kDiel0 && !stubs.empty())
                scatterStub(in, &stubs[c * 3], yhat[m - kDiel0], ghat[m - kDiel0], out);
            else
                scatterAir(in, out);
        }
        // 4. connect as a gather (TlmSolver.cpp:551-613): the pulse arriving
        //    at face (a, s) of node c is the neighbour's reflected pulse on
        //    its opposite face; -own reflected pulse if the neighbour is PEC;
        //    rho * own at the outer boundary. PEC nodes keep zero pulses.
        const long long stride[3] = { 1, nx, (long long)nx * ny };
        const int dims[3] = { nx, ny, nz };
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                {
                    size_t c = ((size_t)k * ny + j) * nx + i;
                    T *dst = &inc[c * 12];
                    if (mat[c] == kPec)
                    {
                        std::fill(dst, dst + 12, T(0));
                        continue;
                    }
                    const int co[3] = { i, j, k };
                    for (int a = 0; a < 3; ++a)
                        for (int s = 0; s < 2; ++s)
                        {
                            int q = co[a] + (s ? 1 : -1);
                            for (int t = 0; t < 2; ++t)
                            {
                                int sl = a * 4 + s * 2 + t;
                                T own = refl[c * 12 + sl];
                                if (q < 0 || q >= dims[a])
                                    dst[sl] = rho * own;
                                else
                                {
                                    size_t nb = c + (size_t)((s ? 1 : -1) * stride[a]);
                                    if (mat[nb] == kPec)
                                        dst[sl] = -own;
                                    else
                                        dst[sl] = refl[nb * 12 + a * 4 + (1 - s) * 2 + t];
                                }
                            }
                        }
                }
    }

    size_t getPulses(double *out, size_t cap) const override
    {
        for (size_t t = 0; t < inc.size() && t < cap; ++t) out[t] = (double)inc[t];
        return inc.size();
    }
    size_t setPulses(const double *in, size_t cnt) override
    {
        if (cnt != inc.size()) return 0;
        for (size_t t = 0; t < cnt; ++t) inc[t] = T(in[t]);
        return cnt;
    }
    size_t getStubs(double *out, size_t cap) const override
    {
        for (size_t t = 0; t < stubs.size() && t < cap; ++t) out[t] = (double)stubs[t];
        return stubs.size();
    }
    int getTables(double *y, double *g, int cap) const override
    {
        for (size_t t = 0; t < yhat.size() && (int)t < cap; ++t)
        {
            y[t] = (double)yhat[t];
            g[t] = (double)ghat[t];
        }
        return (int)yhat.size();
    }
    int probeCount() const override { return (int)probes.size(); }
    int getProbe(int idx, double *ex, double *ey, double *ez, int cap,
                 uint64_t *cell) const override
    {
        if (idx < 0 || idx >= (int)probes.size()) return -1;
        const Probe &p = probes[idx];
        for (size_t t = 0; t < p.ez.size() && (int)t < cap; ++t)
        {
            ex[t] = p.ex[t]; ey[t] = p.ey[t]; ez[t] = p.ez[t];
        }
        if (cell) *cell = p.cell;
        return (int)p.ez.size();
    }
    int portCount() const override { return (int)ports.size(); }
    int getPort(int idx, double *v, double *i, int cap) const override
    {
        if (idx < 0 || idx >= (int)ports.size()) return -1;
        const Port &p = ports[idx];
        for (size_t t = 0; t < p.v.size() && (int)t < cap; ++t)
        {
            v[t] = p.v[t]; i[t] = p.i[t];
        }
        return (int)p.v.size();
    }
    int energyHistory(int *steps, double *vals, int cap) const override
    {
        for (size_t t = 0; t < energySteps.size() && (int)t < cap; ++t)
        {
            steps[t] = energySteps[t];
            vals[t] = energyVals[t];
        }
        return (int)energySteps.size();
    }
    double dt() const override { return (double)timeStep; }

    int surfaceFaces(uint64_t *cells, int *axis, int *sign, float *center, int cap) const override
    {
        for (int f = 0; f < (int)surf.size() && f < cap; ++f)
        {
            if (cells) cells[f] = surf[f].airCell;
            if (axis) axis[f] = surf[f].axis;
            if (sign) sign[f] = surf[f].sign;
            if (center)
                for (int a = 0; a < 3; ++a) center[f * 3 + a] = surf[f].center[a];
        }
        return (int)surf.size();
    }
    int jsInstant(double *out, int cap) const override
    {
        for (int f = 0; f < (int)jsInst.size() && f < cap; ++f) out[f] = (double)jsInst[f];
        return (int)jsInst.size();
    }
    // Raw accumulators and the magnitude finalizeDft would produce
    // (TlmSolver.cpp:467-481): 2/dftSamples * |(Re1, Im1, Re2, Im2)|.
    int jsDft(double *re, double *im, double *mag, int cap, int *samples) const override
    {
        const int nf = (int)surf.size();
        for (int f = 0; f < nf && f < cap; ++f)
        {
            if (re) { re[2 * f] = (double)jsRe[2 * f]; re[2 * f + 1] = (double)jsRe[2 * f + 1]; }
            if (im) { im[2 * f] = (double)jsIm[2 * f]; im[2 * f + 1] = (double)jsIm[2 * f + 1]; }
            if (mag)
            {
                T m = T(0);
                if (dftSamples > 0)
                {
                    T norm = T(2) / T(dftSamples);
                    T r1 = jsRe[2 * f], i1 = jsIm[2 * f], r2 = jsRe[2 * f + 1], i2 = jsIm[2 * f + 1];
                    m = norm * std::sqrt(r1 * r1 + i1 * i1 + r2 * r2 + i2 * i2);
                }
                mag[f] = (double)m;
            }
        }
        if (samples) *samples = dftSamples;
        return nf;
    }
    int huygensFaces(uint64_t *cells, int *axis, int *outSign, float *pos, int cap) const override
    {
        for (int f = 0; f < (int)huy.size() && f < cap; ++f)
        {
            if (cells) cells[f] = huy[f].cell;
            if (axis) axis[f] = huy[f].axis;
            if (outSign) outSign[f] = huy[f].outSign;
            if (pos)
                for (int a = 0; a < 3; ++a) pos[f * 3 + a] = huy[f].pos[a];
        }
        return (int)huy.size();
    }
    int huygensDft(double *acc, int cap, int *samples) const override
    {
        for (size_t t = 0; t < huyAcc.size() && (int)(t / 8) < cap; ++t) acc[t] = (double)huyAcc[t];
        if (samples) *samples = huySamples;
        return (int)huy.size();
    }
    int fieldPlane(double *out, size_t cap, int *axis, int *index, int *n1, int *n2) const override
    {
        if (planeAxis < 0 || planeBuf.empty()) return -1;
        for (size_t t = 0; t < planeBuf.size() && t < cap; ++t) out[t] = (double)planeBuf[t];
        *axis = planeAxis;
        *index = planeIndex;
        *n1 = planeN1;
        *n2 = planeN2;
        return 0;
    }
    int frameCount() const override { return (int)frames.size(); }
    int getFrame(int idx, int *step, double *js, int jsCap, double *plane, size_t planeCap, int *axis,
                 int *pidx, int *n1, int *n2) const override
    {
        if (idx < 0 || idx >= (int)frames.size()) return -1;
        const Frame &fr = frames[idx];
        *step = fr.step;
        for (int f = 0; f < (int)fr.js.size() && f < jsCap; ++f) js[f] = (double)fr.js[f];
        for (size_t t = 0; t < fr.plane.size() && t < planeCap; ++t) plane[t] = (double)fr.plane[t];
        *axis = fr.axis;
        *pidx = fr.idx;
        *n1 = fr.n1;
        *n2 = fr.n2;
        return (int)fr.plane.size();
    }

    // Near-to-far-field transform of the Huygens phasors at f0
    // (ComputeFarFieldFromHuygens, TlmSolver.cpp:805-916): equivalent
    // currents J' = n x (eta0 H), M = -(n x E) per face, radiation vectors
    // summed face by face with e^{+j k0 r.pos}, U = |L_phi + N_theta|^2 +
    // |L_theta - N_phi|^2 over a theta/phi grid, directivity by the
    // trapezoidal rule in FP64.
    int farField(int nTheta, int nPhi, double *U, double *uMax, double *directivity,
                 double *peakTheta, double *peakPhi) const override
    {
        if (huy.empty() || huySamples == 0 || nTheta < 2 || nPhi < 2) return -1;
        const T pi = T(kPi);
        const T k0 = T(2) * pi * T(f0) / T(kC0f);
        const int nh = (int)huy.size();
        struct Cur
        {
            T pos[3], jRe[3], jIm[3], mRe[3], mIm[3];
        };
        std::vector<Cur> fc(nh);
        for (int f = 0; f < nh; ++f)
        {
            const T *a = &huyAcc[(size_t)f * 8];
            const int ax = huy[f].axis;
            const int t1 = firstTransverse(ax), t2 = secondTransverse(ax);
            const T sa = (ax == 1) ? T(-1) : T(1);
            const T sg = T(huy[f].outSign);
            Cur &q = fc[f];
            for (int c = 0; c < 3; ++c)
            {
                q.pos[c] = T(huy[f].pos[c]);
                q.jRe[c] = q.jIm[c] = q.mRe[c] = q.mIm[c] = T(0);
            }
            q.jRe[t2] = sg * sa * a[4];
            q.jIm[t2] = sg * sa * a[5];
            q.jRe[t1] = -sg * sa * a[6];
            q.jIm[t1] = -sg * sa * a[7];
            q.mRe[t2] = -sg * sa * a[0];
            q.mIm[t2] = -sg * sa * a[1];
            q.mRe[t1] = sg * sa * a[2];
            q.mIm[t1] = sg * sa * a[3];
        }
        std::vector<T> u((size_t)nTheta * nPhi);
        for (int ti = 0; ti < nTheta; ++ti)
        {
            const T th = pi * T(ti) / T(nTheta - 1);
            const T st = std::sin(th), ct = std::cos(th);
            for (int pj = 0; pj < nPhi; ++pj)
            {
                const T ph = T(2) * pi * T(pj) / T(nPhi - 1);
                const T cp = std::cos(ph), sp = std::sin(ph);
                const T rh[3] = { st * cp, st * sp, ct };
                const T th3[3] = { ct * cp, ct * sp, -st };
                const T ph3[2] = { -sp, cp };
                T NtR = 0, NtI = 0, NpR = 0, NpI = 0, LtR = 0, LtI = 0, LpR = 0, LpI = 0;
                for (int f = 0; f < nh; ++f)
                {
                    const Cur &q = fc[f];
                    const T pha = k0 * (rh[0] * q.pos[0] + rh[1] * q.pos[1] + rh[2] * q.pos[2]);
                    const T c = std::cos(pha), sn = std::sin(pha);
                    const T jtR = q.jRe[0] * th3[0] + q.jRe[1] * th3[1] + q.jRe[2] * th3[2];
                    const T jtI = q.jIm[0] * th3[0] + q.jIm[1] * th3[1] + q.jIm[2] * th3[2];
                    const T jpR = q.jRe[0] * ph3[0] + q.jRe[1] * ph3[1];
                    const T jpI = q.jIm[0] * ph3[0] + q.jIm[1] * ph3[1];
                    const T mtR = q.mRe[0] * th3[0] + q.mRe[1] * th3[1] + q.mRe[2] * th3[2];
                    const T mtI = q.mIm[0] * th3[0] + q.mIm[1] * th3[1] + q.mIm[2] * th3[2];
                    const T mpR = q.mRe[0] * ph3[0] + q.mRe[1] * ph3[1];
                    const T mpI = q.mIm[0] * ph3[0] + q.mIm[1] * ph3[1];
                    NtR += jtR * c - jtI * sn;
                    NtI += jtR * sn + jtI * c;
                    NpR += jpR * c - jpI * sn;
                    NpI += jpR * sn + jpI * c;
                    LtR += mtR * c - mtI * sn;
                    LtI += mtR * sn + mtI * c;
                    LpR += mpR * c - mpI * sn;
                    LpI += mpR * sn + mpI * c;
                }
                const T aR = LpR + NtR, aI = LpI + NtI;
                const T bR = LtR - NpR, bI = LtI - NpI;
                u[(size_t)ti * nPhi + pj] = aR * aR + aI * aI + bR * bR + bI * bI;
            }
        }
        T um = T(0);
        int iMax = 0;
        double prad = 0.0;
        const T dTh = pi / T(nTheta - 1);
        const T dPh = T(2) * pi / T(nPhi - 1);
        for (int ti = 0; ti < nTheta; ++ti)
        {
            const T th = pi * T(ti) / T(nTheta - 1);
            const T wTh = (ti == 0 || ti == nTheta - 1) ? T(0.5) : T(1);
            for (int pj = 0; pj < nPhi; ++pj)
            {
                const T wPh = (pj == 0 || pj == nPhi - 1) ? T(0.5) : T(1);
                const T v = u[(size_t)ti * nPhi + pj];
                if (v > um)
                {
                    um = v;
                    iMax = ti * nPhi + pj;
                }
                prad += (double)v * std::sin(th) * wTh * wPh * dTh * dPh;
            }
        }
        for (size_t t = 0; t < u.size(); ++t) U[t] = (double)u[t];
        *uMax = (double)um;
        *directivity = prad > 0 ? (double)(T)(4.0 * kPi * (double)um / prad) : 0.0;
        *peakTheta = (double)(T(180) * T(iMax / nPhi) / T(nTheta - 1));
        *peakPhi = (double)(T(360) * T(iMax % nPhi) / T(nPhi - 1));
        return 0;
    }

private:
    struct SurfFace
    {
        size_t airCell;
        int axis, sign;
        float center[3];
    };
    struct HuyFaceO
    {
        size_t cell;
        int axis, outSign;
        float pos[3];
    };
    struct Frame
    {
        int step = 0;
        std::vector<T> js, plane;
        int axis = -1, idx = 0, n1 = 0, n2 = 0;
    };

    // Cell centre origin + (i + 0.5) dl per axis in float (Geometry.h:100-105).
    void cellCenter(int i, int j, int k, float c[3]) const
    {
        c[0] = origin[0] + ((float)i + 0.5f) * dl;
        c[1] = origin[1] + ((float)j + 0.5f) * dl;
        c[2] = origin[2] + ((float)k + 0.5f) * dl;
    }

    // Faces between a PEC cell and a non-PEC neighbour, in the order of the
    // reference's scan (Geometry.cpp:402-436): cells in linear order, then
    // axis, then side -1 before +1.
    void buildSurfaceFaces()
    {
        surf.clear();
        const long long stride[3] = { 1, nx, (long long)nx * ny };
        const int dims[3] = { nx, ny, nz };
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                {
                    const size_t c = ((size_t)k * ny + j) * nx + i;
                    if (mat[c] != kPec) continue;
                    const int co[3] = { i, j, k };
                    for (int a = 0; a < 3; ++a)
                        for (int sd = -1; sd <= 1; sd += 2)
                        {
                            const int q = co[a] + sd;
                            if (q < 0 || q >= dims[a]) continue;
                            const size_t nb = c + (size_t)((long long)sd * stride[a]);
                            if (mat[nb] == kPec) continue;
                            SurfFace f;
                            f.airCell = nb;
                            f.axis = a;
                            f.sign = sd;
                            cellCenter(i, j, k, f.center);
                            f.center[a] = f.center[a] + (float)sd * dl * 0.5f;
                            surf.push_back(f);
                        }
                }
        jsInst.assign(surf.size(), T(0));
        jsRe.assign(surf.size() * 2, T(0));
        jsIm.assign(surf.size() * 2, T(0));
        dftSamples = 0;
    }

    // Huygens box faces, `huyOffset` cells inside the domain, air cells only,
    // in the reference's order (TlmSolver.cpp:310-348): x faces over (k, j),
    // then y faces over (k, i), then z faces over (j, i), low face first.
    void buildHuygens()
    {
        huy.clear();
        huyAcc.clear();
        huySamples = 0;
        const int o = huyOffset;
        if (o < 2) return;
        const int nn[3] = { nx, ny, nz };
        if (2 * o + 2 >= nn[0] || 2 * o + 2 >= nn[1] || 2 * o + 2 >= nn[2]) return;
        float dom[3];
        const float half[3] = { ((float)nx * dl) * 0.5f, ((float)ny * dl) * 0.5f, ((float)nz * dl) * 0.5f };
        for (int a = 0; a < 3; ++a) dom[a] = origin[a] + half[a];
        auto add = [&](int i, int j, int k, int axis, int outSign) {
            const size_t c = ((size_t)k * ny + j) * nx + i;
            if (mat[c] != kAir) return;
            HuyFaceO f;
            f.cell = c;
            f.axis = axis;
            f.outSign = outSign;
            float cc[3];
            cellCenter(i, j, k, cc);
            for (int a = 0; a < 3; ++a) f.pos[a] = cc[a] - dom[a];
            huy.push_back(f);
        };
        const int x0 = o, x1 = nn[0] - 1 - o, y0 = o, y1 = nn[1] - 1 - o, z0 = o, z1 = nn[2] - 1 - o;
        for (int k = z0; k <= z1; ++k)
            for (int j = y0; j <= y1; ++j)
            {
                add(x0, j, k, 0, -1);
                add(x1, j, k, 0, +1);
            }
        for (int k = z0; k <= z1; ++k)
            for (int i = x0; i <= x1; ++i)
            {
                add(i, y0, k, 1, -1);
                add(i, y1, k, 1, +1);
            }
        for (int j = y0; j <= y1; ++j)
            for (int i = x0; i <= x1; ++i)
            {
                add(i, j, z0, 2, -1);
                add(i, j, z1, 2, +1);
            }
        huyAcc.assign(huy.size() * 8, T(0));
    }

    // Surface monitors of one step on the incident pulses after injection
    // (TlmSolver.cpp:616-675, 715-763).
    void surfaceMonitors(int stepIndex)
    {
        const bool doDft = stepIndex >= settleSteps;
        const T phase = T(2) * T(kPi) * T(f0) * (T(stepIndex) * timeStep);
        const T cph = std::cos(phase), sph = std::sin(phase);
        for (size_t f = 0; f < surf.size(); ++f)
        {
            const T *vp = &inc[surf[f].airCell * 12];
            const int t1 = firstTransverse(surf[f].axis), t2 = secondTransverse(surf[f].axis);
            const T h1 = circulation(vp, t1), h2 = circulation(vp, t2);
            jsInst[f] = std::sqrt(h1 * h1 + h2 * h2);
            if (doDft)
            {
                jsRe[f * 2] += h1 * cph;
                jsIm[f * 2] -= h1 * sph;
                jsRe[f * 2 + 1] += h2 * cph;
                jsIm[f * 2 + 1] -= h2 * sph;
            }
        }
        if (doDft) ++dftSamples;
        if (doDft && !huy.empty())
        {
            for (size_t f = 0; f < huy.size(); ++f)
            {
                const T *vp = &inc[huy[f].cell * 12];
                const int t1 = firstTransverse(huy[f].axis), t2 = secondTransverse(huy[f].axis);
                const T e1 = -nodeVoltage(vp, t1), e2 = -nodeVoltage(vp, t2);
                const T m1 = -circulation(vp, t1), m2 = -circulation(vp, t2);
                T *acc = &huyAcc[f * 8];
                acc[0] += e1 * cph;
                acc[1] -= e1 * sph;
                acc[2] += e2 * cph;
                acc[3] -= e2 * sph;
                acc[4] += m1 * cph;
                acc[5] -= m1 * sph;
                acc[6] += m2 * cph;
                acc[7] -= m2 * sph;
            }
            ++huySamples;
        }
        // |E| cut plane every second step
        if (planeAxis >= 0 && (stepIndex % 2) == 0)
        {
            const int nn[3] = { nx, ny, nz };
            const int pa = planeAxis;
            const int a1 = (pa == 0) ? 1 : 0, a2 = (pa == 2) ? 1 : 2;
            planeN1 = nn[a1];
            planeN2 = nn[a2];
            planeBuf.assign((size_t)planeN1 * planeN2, T(0));
            const int idx = std::min(std::max(planeIndex, 0), nn[pa] - 1);
            for (int q2 = 0; q2 < planeN2; ++q2)
                for (int q1 = 0; q1 < planeN1; ++q1)
                {
                    int co[3];
                    co[pa] = idx;
                    co[a1] = q1;
                    co[a2] = q2;
                    const size_t c = ((size_t)co[2] * ny + co[1]) * nx + co[0];
                    if (mat[c] == kPec) continue;
                    const T *vp = &inc[c * 12];
                    T e2 = T(0);
                    for (int j = 0; j < 3; ++j)
                    {
                        const T vj = nodeVoltage(vp, j);
                        e2 += vj * vj;
                    }
                    planeBuf[(size_t)q2 * planeN1 + q1] = std::sqrt(e2);
                }
        }
        if (recordEvery > 0 && (stepIndex % recordEvery) == 0)
        {
            Frame fr;
            fr.step = stepIndex;
            fr.js = jsInst;
            if (planeAxis >= 0 && !planeBuf.empty())
            {
                fr.plane = planeBuf;
                fr.axis = planeAxis;
                fr.idx = planeIndex;
                fr.n1 = planeN1;
                fr.n2 = planeN2;
            }
            frames.push_back(std::move(fr));
        }
    }

    void inject(size_t c, int pol, float amp, T sv)
    {
        T q = T(0.5) * T(amp) * sv;
        T *v = &inc[c * 12];
        for (int a = 0; a < 3; ++a)
        {
            if (a == pol) continue;
            v[slot(a, 0, pol)] += q;
            v[slot(a, 1, pol)] += q;
        }
    }

    // Monitors (TlmSolver.cpp:677-713, 766-789).
    void sample(int stepIndex)
    {
        surfaceMonitors(stepIndex);
        const long long stride[3] = { 1, nx, (long long)nx * ny };
        for (Port &p : ports)
        {
            T vSum = T(0);
            for (size_t c : p.cells) vSum += nodeVoltage(&inc[c * 12], p.pol);
            T cur = T(0);
            if (!p.cells.empty())
            {
                // Ampere loop through the 4 transverse neighbours of the middle
                // gap cell: I = (-2 * zi) / eta0 with
                // zi = ZI_t2(+t1) - ZI_t2(-t1) - ZI_t1(+t2) + ZI_t1(-t2),
                // t1 x t2 = pol. Neighbours are plain linear-index offsets, as
                // in the reference; addPort has checked that they are in range.
                size_t c = p.cells[p.cells.size() / 2];
                int t1 = (p.pol + 1) % 3, t2 = (p.pol + 2) % 3;
                size_t s1 = (size_t)stride[t1], s2 = (size_t)stride[t2];
                T zi = T(0);
                zi += circulation(&inc[(c + s1) * 12], t2);
                zi -= circulation(&inc[(c - s1) * 12], t2);
                zi -= circulation(&inc[(c + s2) * 12], t1);
                zi += circulation(&inc[(c - s2) * 12], t1);
                cur = (T(-2) * zi) / T(kEta0f);
            }
            p.v.push_back((double)vSum);
            p.i.push_back((double)cur);
        }
        T inv = T(-1) / T(dl);
        for (Probe &pr : probes)
        {
            const T *v = &inc[pr.cell * 12];
            pr.ex.push_back((double)(inv * nodeVoltage(v, 0)));
            pr.ey.push_back((double)(inv * nodeVoltage(v, 1)));
            pr.ez.push_back((double)(inv * nodeVoltage(v, 2)));
        }
        if ((stepIndex & 15) == 0)
        {
            double e = 0.0;
            for (size_t t = 0; t < inc.size(); ++t) e += (double)inc[t] * (double)inc[t];
            energySteps.push_back(stepIndex);
            energyVals.push_back(e);
        }
    }
    int nx = 0, ny = 0, nz = 0;
    float origin[3] = { 0, 0, 0 };
    float dl = 1e-3f, f0 = 1e9f;
    int wave = 0, totalSteps = 0, settleSteps = 0;
    T rho = T(0), timeStep = T(0);
    size_t n = 0;
    std::vector<uint8_t> mat;
    std::vector<T> yhat, ghat, inc, refl, stubs;
    std::vector<Port> ports;
    std::vector<Probe> probes;
    std::vector<Source> sources;
    std::vector<int> energySteps;
    std::vector<double> energyVals;
    int huyOffset = 0, recordEvery = 0;
    int planeAxis = -1, planeIndex = 0, planeN1 = 0, planeN2 = 0;
    std::vector<SurfFace> surf;
    std::vector<HuyFaceO> huy;
    std::vector<T> jsInst, jsRe, jsIm, huyAcc, planeBuf;
    int dftSamples = 0, huySamples = 0;
    std::vector<Frame> frames;
};

// Unitarity known-answer tests (TlmSolver.cpp:116-169): build the scattering
// matrix column by column from unit excitations and return max |S^T W S - W|.
template <class T> T scatterUnitarityError()
{
    T S[12][12];
    for (int c = 0; c < 12; ++c)
    {
        T in[12] = {}, out[12];
        in[c] = T(1);
        scatterAir(in, out);
        for (int r = 0; r < 12; ++r) S[r][c] = out[r];
    }
    T worst = T(0);
    for (int a = 0; a < 12; ++a)
        for (int b = 0; b < 12; ++b)
        {
            T dot = T(0);
            for (int r = 0; r < 12; ++r) dot += S[r][a] * S[r][b];
            worst = std::max(worst, (T)std::fabs(dot - (a == b ? T(1) : T(0))));
        }
    return worst;
}

template <class T> T stubUnitarityError(T epsr)
{
    const int np = 15;
    T yh = T(4) * (epsr - T(1));
    T W[np], S[np][np];
    for (int t = 0; t < np; ++t) W[t] = t < 12 ? T(1) : yh;
    for (int c = 0; c < np; ++c)
    {
        T in[12] = {}, vs[3] = {}, out[12];
        if (c < 12) in[c] = T(1); else vs[c - 12] = T(1);
        scatterStub(in, vs, yh, T(0), out);
        for (int r = 0; r < 12; ++r) S[r][c] = out[r];
        for (int r = 0; r < 3; ++r) S[12 + r][c] = vs[r];
    }
    T worst = T(0);
    for (int a = 0; a < np; ++a)
        for (int b = 0; b < np; ++b)
        {
            T dot = T(0);
            for (int r = 0; r < np; ++r) dot += W[r] * S[r][a] * S[r][b];
            worst = std::max(worst, (T)std::fabs(dot - (a == b ? W[a] : T(0))));
        }
    return worst;
}

} // namespace

extern "C" {

void *orc_create(int fp64)
{
    if (fp64) return static_cast<OracleBase *>(new Oracle<double>());
    return static_cast<OracleBase *>(new Oracle<float>());
}
void orc_destroy(void *h) { delete static_cast<OracleBase *>(h); }
int orc_setup(void *h, int nx, int ny, int nz, float ox, float oy, float oz, float dl,
              const uint8_t *mat, const float *epsr, const float *sigma, int ntab,
              float f0, int waveform, int total, int settle, float rho)
{
    return static_cast<OracleBase *>(h)->setup(nx, ny, nz, ox, oy, oz, dl, mat, epsr,
                                               sigma, ntab, f0, waveform, total,
                                               settle, rho);
}
int orc_add_port(void *h, const uint64_t *cells, int n, int pol, float amp)
{
    return static_cast<OracleBase *>(h)->addPort(cells, n, pol, amp);
}
int orc_add_probe(void *h, float x, float y, float z)
{
    return static_cast<OracleBase *>(h)->addProbe(x, y, z);
}
void orc_add_plane_wave(void *h, int prop, int plane, int pol, float amp)
{
    static_cast<OracleBase *>(h)->addPlaneWave(prop, plane, pol, amp);
}
double orc_waveform(void *h, int n) { return static_cast<OracleBase *>(h)->waveform(n); }
double orc_dt(void *h) { return static_cast<OracleBase *>(h)->dt(); }
void orc_steps(void *h, int n0, int count, const double *sv)
{
    OracleBase *o = static_cast<OracleBase *>(h);
    for (int t = 0; t < count; ++t) o->step(n0 + t, sv != nullptr, sv ? sv[t] : 0.0);
}
size_t orc_get_pulses(void *h, double *out, size_t cap)
{
    return static_cast<OracleBase *>(h)->getPulses(out, cap);
}
size_t orc_set_pulses(void *h, const double *in, size_t n)
{
    return static_cast<OracleBase *>(h)->setPulses(in, n);
}
size_t orc_get_stubs(void *h, double *out, size_t cap)
{
    return static_cast<OracleBase *>(h)->getStubs(out, cap);
}
int orc_get_tables(void *h, double *y, double *g, int cap)
{
    return static_cast<OracleBase *>(h)->getTables(y, g, cap);
}
int orc_probe_count(void *h) { return static_cast<OracleBase *>(h)->probeCount(); }
int orc_get_probe(void *h, int idx, double *ex, double *ey, double *ez, int cap,
                  uint64_t *cell)
{
    return static_cast<OracleBase *>(h)->getProbe(idx, ex, ey, ez, cap, cell);
}
int orc_port_count(void *h) { return static_cast<OracleBase *>(h)->portCount(); }
int orc_get_port(void *h, int idx, double *v, double *i, int cap)
{
    return static_cast<OracleBase *>(h)->getPort(idx, v, i, cap);
}
int orc_energy_history(void *h, int *steps, double *vals, int cap)
{
    return static_cast<OracleBase *>(h)->energyHistory(steps, vals, cap);
}
int orc_configure_surface(void *h, int huy_offset, int record_every)
{
    return static_cast<OracleBase *>(h)->configureSurface(huy_offset, record_every);
}
void orc_set_field_plane(void *h, int axis, int index)
{
    static_cast<OracleBase *>(h)->setFieldPlane(axis, index);
}
int orc_surface_faces(void *h, uint64_t *cells, int *axis, int *sign, float *center, int cap)
{
    return static_cast<OracleBase *>(h)->surfaceFaces(cells, axis, sign, center, cap);
}
int orc_js_instant(void *h, double *out, int cap)
{
    return static_cast<OracleBase *>(h)->jsInstant(out, cap);
}
int orc_js_dft(void *h, double *re, double *im, double *mag, int cap, int *samples)
{
    return static_cast<OracleBase *>(h)->jsDft(re, im, mag, cap, samples);
}
int orc_huygens_faces(void *h, uint64_t *cells, int *axis, int *out_sign, float *pos, int cap)
{
    return static_cast<OracleBase *>(h)->huygensFaces(cells, axis, out_sign, pos, cap);
}
int orc_huygens_dft(void *h, double *acc, int cap, int *samples)
{
    return static_cast<OracleBase *>(h)->huygensDft(acc, cap, samples);
}
int orc_field_plane(void *h, double *out, size_t cap, int *axis, int *index, int *n1, int *n2)
{
    return static_cast<OracleBase *>(h)->fieldPlane(out, cap, axis, index, n1, n2);
}
int orc_frame_count(void *h) { return static_cast<OracleBase *>(h)->frameCount(); }
int orc_get_frame(void *h, int idx, int *step, double *js, int js_cap, double *plane, size_t plane_cap,
                  int *axis, int *pidx, int *n1, int *n2)
{
    return static_cast<OracleBase *>(h)->getFrame(idx, step, js, js_cap, plane, plane_cap, axis, pidx, n1,
                                                  n2);
}
int orc_far_field(void *h, int n_theta, int n_phi, double *U, double *u_max, double *directivity,
                  double *peak_theta, double *peak_phi)
{
    return static_cast<OracleBase *>(h)->farField(n_theta, n_phi, U, u_max, directivity, peak_theta,
                                                  peak_phi);
}
double orc_scatter_unitarity(int fp64)
{
    return fp64 ? scatterUnitarityError<double>() : (double)scatterUnitarityError<float>();
}
double orc_stub_unitarity(int fp64, double epsr)
{
    return fp64 ? stubUnitarityError<double>(epsr)
                : (double)stubUnitarityError<float>((float)epsr);
}

} // extern "C"
