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
        return 0;
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

private:
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
