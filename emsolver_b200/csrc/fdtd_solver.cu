// fdtd_solver.cu -- Yee FDTD time step on sm_100a (the reference's second
// time-domain solver, FdtdSolver.cpp), behind the C ABI of fdtd_b200.h.
//
// One step (FdtdSolver::step, FdtdSolver.cpp:401-446):
//   1. soft sources on E edges (per-edge thread applying its contributions in
//      the reference's source order, so edges shared by several source cells
//      add up exactly as the sequential loop does);
//   2. monitors on the current fields (ports, probes, surface currents,
//      Huygens phasors, cut plane; energy every 16 steps);
//   3. H update over all H components;
//   4. Mur snapshot of the two outermost layers of every tangential E
//      component, E update of the interior edges (PEC masks, lossy
//      coefficients), then the first-order Mur boundary in two launches whose
//      order reproduces the reference's six face passes (edges shared by two
//      faces end with the later pass's value).
// Fields use the reference's Yee layouts (x fastest), so every update is a
// coalesced row sweep; all arithmetic is FP32 in the reference's operation
// order (the library is compiled with --fmad=false), hence bitwise results.
#include "fdtd_b200.h"
#include "tlm_b200.h"
#include "tlm_internal.h"

#include "tlm_host_math.h"
#include "tlm_device.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

using tlmi::SurfaceState;

namespace fdk {

struct Dims
{
    int nx, ny, nz;
    __host__ __device__ long long iEx(int i, int j, int k) const { return ((long long)k * (ny + 1) + j) * nx + i; }
    __host__ __device__ long long iEy(int i, int j, int k) const { return ((long long)k * ny + j) * (nx + 1) + i; }
    __host__ __device__ long long iEz(int i, int j, int k) const
    {
        return ((long long)k * (ny + 1) + j) * (nx + 1) + i;
    }
    __host__ __device__ long long iHx(int i, int j, int k) const { return ((long long)k * ny + j) * (nx + 1) + i; }
    __host__ __device__ long long iHy(int i, int j, int k) const { return ((long long)k * (ny + 1) + j) * nx + i; }
    __host__ __device__ long long iHz(int i, int j, int k) const { return ((long long)k * ny + j) * nx + i; }
    // 32-bit forms for the update sweeps: setup refuses grids whose
    // (nx+1)(ny+1)(nz+1) index box reaches 2^31, so every component fits.
    __device__ int jEx(int i, int j, int k) const { return (k * (ny + 1) + j) * nx + i; }
    __device__ int jEy(int i, int j, int k) const { return (k * ny + j) * (nx + 1) + i; }
    __device__ int jEz(int i, int j, int k) const { return (k * (ny + 1) + j) * (nx + 1) + i; }
    __device__ int jHx(int i, int j, int k) const { return (k * ny + j) * (nx + 1) + i; }
    __device__ int jHy(int i, int j, int k) const { return (k * (ny + 1) + j) * nx + i; }
    __device__ int jHz(int i, int j, int k) const { return (k * ny + j) * nx + i; }
};

struct Fields
{
    float *E[3], *H[3];
    const uint8_t *mE[3];        // 1 = free edge, 0 = PEC
    const float *ca[3], *cb[3];  // lossy coefficients (nullptr: air everywhere)
};

// ---- cell-centred averages (FdtdSolver.cpp:42-79) -------------------------
__device__ __forceinline__ float ecAt(const Fields &f, const Dims &d, int i, int j, int k, int c)
{
    if (c == 0)
        return 0.25f * (((f.E[0][d.iEx(i, j, k)] + f.E[0][d.iEx(i, j + 1, k)]) + f.E[0][d.iEx(i, j, k + 1)]) +
                        f.E[0][d.iEx(i, j + 1, k + 1)]);
    if (c == 1)
        return 0.25f * (((f.E[1][d.iEy(i, j, k)] + f.E[1][d.iEy(i + 1, j, k)]) + f.E[1][d.iEy(i, j, k + 1)]) +
                        f.E[1][d.iEy(i + 1, j, k + 1)]);
    return 0.25f * (((f.E[2][d.iEz(i, j, k)] + f.E[2][d.iEz(i + 1, j, k)]) + f.E[2][d.iEz(i, j + 1, k)]) +
                    f.E[2][d.iEz(i + 1, j + 1, k)]);
}
__device__ __forceinline__ float hcAt(const Fields &f, const Dims &d, int i, int j, int k, int c)
{
    if (c == 0) return 0.5f * (f.H[0][d.iHx(i, j, k)] + f.H[0][d.iHx(i + 1, j, k)]);
    if (c == 1) return 0.5f * (f.H[1][d.iHy(i, j, k)] + f.H[1][d.iHy(i, j + 1, k)]);
    return 0.5f * (f.H[2][d.iHz(i, j, k)] + f.H[2][d.iHz(i, j, k + 1)]);
}

// ---- 1. soft sources ----------------------------------------------------
// Edge e (code: component * 2^60 + field index) receives amps[off[e]..off[e+1])
// in source order: E += (-0.25 amp) sv each (FdtdSolver.cpp:404-437).
__global__ void injectKernel(Fields f, const long long *__restrict__ edge, const int *__restrict__ off,
                             const float *__restrict__ amps, int nedges, float sv)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nedges) return;
    const long long code = edge[e];
    const int c = (int)(code >> 60);
    const long long idx = code & ((1LL << 60) - 1);
    float *E = c == 0 ? f.E[0] : c == 1 ? f.E[1] : f.E[2];
    float v = E[idx];
    for (int t = off[e]; t < off[e + 1]; ++t) v = v + (-0.25f * amps[t]) * sv;
    E[idx] = v;
}

// ---- 2. monitors ----------------------------------------------------------
struct MonArgs
{
    Fields f;
    Dims d;
    float dl, eta0;
    int step;
    // ports: cells of port p at cells[poff[p] .. poff[p+1]), middle cell pmid[p]
    int nports;
    const int *poff;
    const long long *pcells;
    const int *ppol;
    float *vrec, *irec;  // [step][nports]
    // probes
    int nprobes;
    const long long *probeCell;
    float *prec;         // [step][nprobes][3]
    // surface faces: code = cell * 8 + axis * 2 + (sign < 0)
    int njs;
    const long long *jsCode;
    float *jsInst, *jsAcc;
    int nhuy;
    const long long *huyCode;
    float *huyAcc;
    int doDft;
    float cph, sph;
    int planeAxis, planeIndex, planeN1, planeN2;
    float *plane;
};

__device__ __forceinline__ void cellCo(long long c, const Dims &d, int co[3])
{
    co[0] = (int)(c % d.nx);
    co[1] = (int)((c / d.nx) % d.ny);
    co[2] = (int)(c / ((long long)d.nx * d.ny));
}

__global__ void __launch_bounds__(256) monitorKernel(const MonArgs a)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const Fields &f = a.f;
    const Dims &d = a.d;
    if (t < a.nports)
    {
        // FdtdSolver.cpp:753-781
        const int p = (int)t;
        const int pol = a.ppol[p];
        float vSum = 0.0f;
        for (int q = a.poff[p]; q < a.poff[p + 1]; ++q)
        {
            int co[3];
            cellCo(a.pcells[q], d, co);
            vSum += -ecAt(f, d, co[0], co[1], co[2], pol) * a.dl;
        }
        float iVal = 0.0f;
        if (a.poff[p + 1] > a.poff[p])
        {
            const int mid = a.poff[p] + (a.poff[p + 1] - a.poff[p]) / 2;
            int co[3];
            cellCo(a.pcells[mid], d, co);
            const int t1 = (pol + 1) % 3, t2 = (pol + 2) % 3;
            int d1[3] = { 0, 0, 0 }, d2[3] = { 0, 0, 0 };
            d1[t1] = 1;
            d2[t2] = 1;
            iVal = 2.0f * a.dl *
                   (((hcAt(f, d, co[0] + d1[0], co[1] + d1[1], co[2] + d1[2], t2) -
                      hcAt(f, d, co[0] - d1[0], co[1] - d1[1], co[2] - d1[2], t2)) -
                     hcAt(f, d, co[0] + d2[0], co[1] + d2[1], co[2] + d2[2], t1)) +
                    hcAt(f, d, co[0] - d2[0], co[1] - d2[1], co[2] - d2[2], t1));
        }
        a.vrec[(long long)a.step * a.nports + p] = vSum;
        a.irec[(long long)a.step * a.nports + p] = iVal;
        return;
    }
    t -= a.nports;
    if (t < a.nprobes)
    {
        int co[3];
        cellCo(a.probeCell[t], d, co);
        float *o = a.prec + ((long long)a.step * a.nprobes + t) * 3;
        const float ex = ecAt(f, d, co[0], co[1], co[2], 0), ey = ecAt(f, d, co[0], co[1], co[2], 1);
        const float ez = ecAt(f, d, co[0], co[1], co[2], 2);
        o[0] = ex;
        o[1] = ey;
        o[2] = ez;
        return;
    }
    t -= a.nprobes;
    if (t < a.njs)
    {
        // FdtdSolver.cpp:703-721: eta0 H at the face cell
        const long long code = a.jsCode[t];
        int co[3];
        cellCo(code >> 3, d, co);
        const int ax = (int)((code >> 1) & 3);
        const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
        const float h1 = a.eta0 * hcAt(f, d, co[0], co[1], co[2], t1);
        const float h2 = a.eta0 * hcAt(f, d, co[0], co[1], co[2], t2);
        a.jsInst[t] = sqrtf(h1 * h1 + h2 * h2);
        if (a.doDft)
        {
            float *acc = a.jsAcc + t * 4;
            acc[0] = acc[0] + h1 * a.cph;
            acc[1] = acc[1] - h1 * a.sph;
            acc[2] = acc[2] + h2 * a.cph;
            acc[3] = acc[3] - h2 * a.sph;
        }
        return;
    }
    t -= a.njs;
    const int nh = a.doDft ? a.nhuy : 0;
    if (t < nh)
    {
        // FdtdSolver.cpp:729-748: cell-centred E and eta0 H
        const long long code = a.huyCode[t];
        int co[3];
        cellCo(code >> 3, d, co);
        const int ax = (int)((code >> 1) & 3);
        const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
        const float e1 = ecAt(f, d, co[0], co[1], co[2], t1), e2 = ecAt(f, d, co[0], co[1], co[2], t2);
        const float m1 = a.eta0 * hcAt(f, d, co[0], co[1], co[2], t1);
        const float m2 = a.eta0 * hcAt(f, d, co[0], co[1], co[2], t2);
        float *acc = a.huyAcc + t * 8;
        acc[0] = acc[0] + e1 * a.cph;
        acc[1] = acc[1] - e1 * a.sph;
        acc[2] = acc[2] + e2 * a.cph;
        acc[3] = acc[3] - e2 * a.sph;
        acc[4] = acc[4] + m1 * a.cph;
        acc[5] = acc[5] - m1 * a.sph;
        acc[6] = acc[6] + m2 * a.cph;
        acc[7] = acc[7] - m2 * a.sph;
        return;
    }
    t -= nh;
    const long long np = a.planeAxis >= 0 ? (long long)a.planeN1 * a.planeN2 : 0;
    if (t < np)
    {
        // FdtdSolver.cpp:790-813: |E| dl over the plane, PEC cells included
        const int q1 = (int)(t % a.planeN1), q2 = (int)(t / a.planeN1);
        const int pa = a.planeAxis, a1 = pa == 0 ? 1 : 0, a2 = pa == 2 ? 1 : 2;
        int co[3];
        co[pa] = a.planeIndex;
        co[a1] = q1;
        co[a2] = q2;
        const float ex = ecAt(f, d, co[0], co[1], co[2], 0);
        const float ey = ecAt(f, d, co[0], co[1], co[2], 1);
        const float ez = ecAt(f, d, co[0], co[1], co[2], 2);
        a.plane[t] = sqrtf(ex * ex + ey * ey + ez * ez) * a.dl;
    }
}

// Energy (FdtdSolver.cpp:836-870): sum E^2 + eta0^2 sum H^2 in FP64, block
// partials in a fixed order. Every component is swept as 16-byte vectors
// (device allocations are 256-byte aligned), four in flight per thread.
__device__ __forceinline__ double sumSquares(const float *arr, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const float4 *a4 = reinterpret_cast<const float4 *>(arr);
    const long long n4 = n >> 2;
    double acc = 0.0;
#pragma unroll 4
    for (long long i = t0; i < n4; i += stride)
    {
        const float4 v = a4[i];
        const double x = v.x, y = v.y, z = v.z, w = v.w;
        acc += ((x * x + y * y) + z * z) + w * w;
    }
    const long long r = (n4 << 2) + t0;
    if (r < n)
    {
        const double x = arr[r];
        acc += x * x;
    }
    return acc;
}
__global__ void __launch_bounds__(256) energyPartialKernel(Fields f, long long nE0, long long nE1, long long nE2,
                                                           long long nH0, long long nH1, long long nH2,
                                                           double eta2, double *part)
{
    __shared__ double red[8];
    const double se = (sumSquares(f.E[0], nE0) + sumSquares(f.E[1], nE1)) + sumSquares(f.E[2], nE2);
    const double sh = (sumSquares(f.H[0], nH0) + sumSquares(f.H[1], nH1)) + sumSquares(f.H[2], nH2);
    double s = se + sh * eta2;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}
__global__ void __launch_bounds__(256) energyFinalKernel(const double *part, int n, double *out)
{
    __shared__ double red[8];
    double t = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) t += part[b];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        *out = s;
    }
}

// ---- Mur boundary state ----------------------------------------------------
// Face planes: 0 x-faces Ey, 1 x-faces Ez, 2 y-faces Ex, 3 y-faces Ez,
// 4 z-faces Ex, 5 z-faces Ey. Plane position (q1, q2) over the two other
// axes; layers 0, 1, N-1, N along the face normal (N = grid size on it).
struct Mur
{
    int n1[6], n2[6];
    long long off[6];  // start of each plane's 4 layers in `snap`
    float *snap;
    float cMur;
};
__device__ __forceinline__ long long murIndex(const Dims &d, int F, int L, int q1, int q2)
{
    switch (F)
    {
    case 0: return d.iEy(L, q1, q2);
    case 1: return d.iEz(L, q1, q2);
    case 2: return d.iEx(q1, L, q2);
    case 3: return d.iEz(q1, L, q2);
    case 4: return d.iEx(q1, q2, L);
    default: return d.iEy(q1, q2, L);
    }
}
__device__ __forceinline__ float *murField(const Fields &f, int F)
{
    return (F == 0 || F == 5) ? f.E[1] : (F == 1 || F == 3) ? f.E[2] : f.E[0];
}
__device__ __forceinline__ int murN(const Dims &d, int F) { return F < 2 ? d.nx : F < 4 ? d.ny : d.nz; }

// A flat item index over planes [F0, F0 + NP) resolved to its plane F, the
// position (q1, q2), and that position's first layer in `snap` (with the
// layer stride pl). Unrolled so that the plane tables stay in parameter space.
struct MurAt
{
    int F, q1, q2;
    long long pl;
    float *s;
};
template <int F0, int NP>
__device__ __forceinline__ bool murItem(const Mur &m, long long t, MurAt *a)
{
    bool found = false;
#pragma unroll
    for (int p = F0; p < F0 + NP; ++p)
    {
        const long long n = (long long)m.n1[p] * m.n2[p];
        if (!found)
        {
            if (t < n)
            {
                found = true;
                a->F = p;
                a->q1 = (int)(t % m.n1[p]);
                a->q2 = (int)(t / m.n1[p]);
                a->pl = n;
                a->s = m.snap + m.off[p] + (long long)a->q2 * m.n1[p] + a->q1;
            }
            else
                t -= n;
        }
    }
    return found;
}

// Copy of layers 0, 1, N-1, N of every face plane, taken before the E
// update (it runs as extra blocks of the H update, which leaves E unchanged).
__device__ __forceinline__ void murSnapItem(const Fields &f, const Dims &d, const Mur &m, long long t)
{
    MurAt a;
    if (!murItem<0, 6>(m, t, &a)) return;
    const int N = murN(d, a.F);
    const float *E = murField(f, a.F);
    const float e0 = E[murIndex(d, a.F, 0, a.q1, a.q2)], e1 = E[murIndex(d, a.F, 1, a.q1, a.q2)];
    const float e2 = E[murIndex(d, a.F, N - 1, a.q1, a.q2)], e3 = E[murIndex(d, a.F, N, a.q1, a.q2)];
    a.s[0] = e0;
    a.s[a.pl] = e1;
    a.s[2 * a.pl] = e2;
    a.s[3 * a.pl] = e3;
}

// ---- 3. H update (FdtdSolver.cpp:449-484) and the Mur snapshot ------------
// One thread per Yee cell (i, j, k) of the (nx+1) x (ny+1) x (nz+1) index
// box, flattened (x fastest) so that no block is padded per row.
struct Box
{
    unsigned total;
    tlmk::FastDiv divX, divY;  // by nx + 1 and ny + 1
};
__device__ __forceinline__ bool boxCell(const Box &b, const Dims &d, int *i, int *j, int *k)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.total) return false;
    const unsigned r = tlmk::fastDiv(t, b.divX);
    *i = (int)(t - r * (unsigned)(d.nx + 1));
    const unsigned kk = tlmk::fastDiv(r, b.divY);
    *j = (int)(r - kk * (unsigned)(d.ny + 1));
    *k = (int)kk;
    return true;
}

// Every load of the thread is issued before its first store (the three H
// components share E operands: 9 distinct E loads and 3 H loads), so one
// memory round trip covers the cell. Operation order per component is the
// reference's.
__global__ void __launch_bounds__(256) updateHKernel(Fields f, Dims d, Box b, float ch, Mur m, unsigned hBlocks)
{
    if (blockIdx.x >= hBlocks)
    {
        murSnapItem(f, d, m, (long long)(blockIdx.x - hBlocks) * blockDim.x + threadIdx.x);
        return;
    }
    int i, j, k;
    if (!boxCell(b, d, &i, &j, &k)) return;
    const float *__restrict__ Ex = f.E[0];
    const float *__restrict__ Ey = f.E[1];
    const float *__restrict__ Ez = f.E[2];
    const bool ax = j < d.ny && k < d.nz, ay = i < d.nx && k < d.nz, az = i < d.nx && j < d.ny;
    float hx = 0.f, hy = 0.f, hz = 0.f;
    float ez0 = 0.f, ezj = 0.f, ezi = 0.f, ey0 = 0.f, eyk = 0.f, eyi = 0.f, ex0 = 0.f, exk = 0.f, exj = 0.f;
    const int qx = ax ? d.jHx(i, j, k) : 0, qy = ay ? d.jHy(i, j, k) : 0, qz = az ? d.jHz(i, j, k) : 0;
    if (ax)
    {
        hx = f.H[0][qx];
        ezj = Ez[d.jEz(i, j + 1, k)];
        eyk = Ey[d.jEy(i, j, k + 1)];
    }
    if (ay)
    {
        hy = f.H[1][qy];
        exk = Ex[d.jEx(i, j, k + 1)];
        ezi = Ez[d.jEz(i + 1, j, k)];
    }
    if (az)
    {
        hz = f.H[2][qz];
        eyi = Ey[d.jEy(i + 1, j, k)];
        exj = Ex[d.jEx(i, j + 1, k)];
    }
    if (ax || ay) ez0 = Ez[d.jEz(i, j, k)];
    if (ax || az) ey0 = Ey[d.jEy(i, j, k)];
    if (ay || az) ex0 = Ex[d.jEx(i, j, k)];
    if (ax) f.H[0][qx] = hx - ch * ((ezj - ez0) - (eyk - ey0));
    if (ay) f.H[1][qy] = hy - ch * ((exk - ex0) - (ezi - ez0));
    if (az) f.H[2][qz] = hz - ch * ((eyi - ey0) - (exj - ex0));
}

// E update of the interior edges (FdtdSolver.cpp:487-555). As for H, all
// loads (masks, 6 distinct H values shared by the three components, the
// edges' own E and lossy coefficients) come before the stores.
__global__ void __launch_bounds__(256) updateEKernel(Fields f, Dims d, Box b, float cb0)
{
    int i, j, k;
    if (!boxCell(b, d, &i, &j, &k)) return;
    const float *__restrict__ Hx = f.H[0];
    const float *__restrict__ Hy = f.H[1];
    const float *__restrict__ Hz = f.H[2];
    const bool ix = i >= 1 && i < d.nx, jy = j >= 1 && j < d.ny, kz = k >= 1 && k < d.nz;
    const bool ax = i < d.nx && jy && kz, ay = ix && j < d.ny && kz, az = ix && jy && k < d.nz;
    const bool lossy = f.ca[0] != nullptr;
    const int qx = ax ? d.jEx(i, j, k) : 0, qy = ay ? d.jEy(i, j, k) : 0, qz = az ? d.jEz(i, j, k) : 0;
    uint8_t mx = 0, my = 0, mz = 0;
    float ex = 0.f, ey = 0.f, ez = 0.f, cax = 0.f, cbx = 0.f, cay = 0.f, cby = 0.f, caz = 0.f, cbz = 0.f;
    float hz0 = 0.f, hzj = 0.f, hzi = 0.f, hy0 = 0.f, hyk = 0.f, hyi = 0.f, hx0 = 0.f, hxk = 0.f, hxj = 0.f;
    if (ax)
    {
        mx = f.mE[0][qx];
        ex = f.E[0][qx];
        hzj = Hz[d.jHz(i, j - 1, k)];
        hyk = Hy[d.jHy(i, j, k - 1)];
        if (lossy)
        {
            cax = f.ca[0][qx];
            cbx = f.cb[0][qx];
        }
    }
    if (ay)
    {
        my = f.mE[1][qy];
        ey = f.E[1][qy];
        hxk = Hx[d.jHx(i, j, k - 1)];
        hzi = Hz[d.jHz(i - 1, j, k)];
        if (lossy)
        {
            cay = f.ca[1][qy];
            cby = f.cb[1][qy];
        }
    }
    if (az)
    {
        mz = f.mE[2][qz];
        ez = f.E[2][qz];
        hyi = Hy[d.jHy(i - 1, j, k)];
        hxj = Hx[d.jHx(i, j - 1, k)];
        if (lossy)
        {
            caz = f.ca[2][qz];
            cbz = f.cb[2][qz];
        }
    }
    if (ax || ay) hz0 = Hz[d.jHz(i, j, k)];
    if (ax || az) hy0 = Hy[d.jHy(i, j, k)];
    if (ay || az) hx0 = Hx[d.jHx(i, j, k)];
    if (ax)
    {
        const float curl = (hz0 - hzj) - (hy0 - hyk);
        f.E[0][qx] = !mx ? 0.0f : lossy ? cax * ex + cbx * curl : ex + cb0 * curl;
    }
    if (ay)
    {
        const float curl = (hx0 - hxk) - (hz0 - hzi);
        f.E[1][qy] = !my ? 0.0f : lossy ? cay * ey + cby * curl : ey + cb0 * curl;
    }
    if (az)
    {
        const float curl = (hy0 - hyi) - (hx0 - hxj);
        f.E[2][qz] = !mz ? 0.0f : lossy ? caz * ez + cbz * curl : ez + cb0 * curl;
    }
}

// Mur on planes [F0, F0 + 3): per plane position the low face, then the high
// face (FdtdSolver.cpp:624-670): E_b = E_1(old) + cMur (E_1(new) - E_b(old)).
template <int F0>
__global__ void murApplyKernel(Fields f, Dims d, Mur m)
{
    MurAt a;
    if (!murItem<F0, 3>(m, (long long)blockIdx.x * blockDim.x + threadIdx.x, &a)) return;
    const int N = murN(d, a.F);
    float *E = murField(f, a.F);
    const long long b0 = murIndex(d, a.F, 0, a.q1, a.q2), b1 = murIndex(d, a.F, 1, a.q1, a.q2);
    const long long bN = murIndex(d, a.F, N, a.q1, a.q2), bN1 = murIndex(d, a.F, N - 1, a.q1, a.q2);
    const float s0 = a.s[0], s1 = a.s[a.pl], s2 = a.s[2 * a.pl], s3 = a.s[3 * a.pl];
    const float e1 = E[b1], eN1 = E[bN1];
    E[b0] = s1 + m.cMur * (e1 - s0);
    E[bN] = s2 + m.cMur * (eN1 - s3);
}

} // namespace fdk

// ---------------------------------------------------------------------------
struct fdtd_solver
{
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    std::string err;
    bool configured = false;
    tlm_grid g{};
    tlm_config cfg{};
    std::vector<uint8_t> mat;
    std::vector<tlm_matprops> table;
    fdk::Dims d{};
    float dt = 0, cMur = 0, cb0 = 0, ch = 0;
    bool haveDiel = false;
    long long len[6] = {};       // Ex Ey Ez Hx Hy Hz lengths
    void *dField[6] = {};
    uint8_t *dMask[3] = {};
    std::vector<uint8_t> hMask[3];  // host copies of the PEC masks (source edges)
    float *dCa[3] = {}, *dCb[3] = {};
    fdk::Mur mur{};
    // sources
    struct Src
    {
        uint64_t cell;
        int pol;
        float amp;
    };
    std::vector<Src> planeSources;
    struct Port
    {
        std::vector<uint64_t> cells;
        int pol;
        float amp;
    };
    std::vector<Port> ports;
    std::vector<uint64_t> probeCells;
    std::vector<float> svTable;
    bool prepared = false;
    long long *dEdge = nullptr;
    int *dEdgeOff = nullptr;
    float *dAmps = nullptr;
    int nEdges = 0;
    int *dPoff = nullptr, *dPpol = nullptr;
    long long *dPcells = nullptr, *dProbe = nullptr;
    float *dVrec = nullptr, *dIrec = nullptr, *dPrec = nullptr;
    double *dEhist = nullptr, *dEpart = nullptr;
    long long recCap = 0;
    int nEpart = 0;
    SurfaceState surf;
    int curStep = 0;
    std::vector<void *> allocs;

    bool maskHost(int c, long long idx) const { return hMask[c][(size_t)idx] != 0; }
    tlm_status fail(tlm_status s, const std::string &m)
    {
        err = m;
        return s;
    }
    tlm_status cuda(cudaError_t e, const char *what)
    {
        if (e == cudaSuccess) return TLM_OK;
        cudaGetLastError();
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? TLM_ENOMEM : TLM_ECUDA;
    }
};

namespace {

thread_local std::string g_fdtdErr;

#define FD_TRY(x)                                                                                                      \
    do                                                                                                                 \
    {                                                                                                                  \
        tlm_status s_ = (x);                                                                                           \
        if (s_ != TLM_OK) return s_;                                                                                   \
    } while (0)
#define FD_CU(h, call) FD_TRY((h)->cuda((call), #call))

struct Guard
{
    int prev = -1;
    explicit Guard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Guard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

template <class T> tlm_status alloc(fdtd_solver *h, T **p, size_t bytes)
{
    void *q = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&q, std::max<size_t>(bytes, 1), h->pool, h->stream);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return h->fail(TLM_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    *p = static_cast<T *>(q);
    return TLM_OK;
}
template <class T> void release(fdtd_solver *h, T *&p)
{
    if (p) cudaFreeAsync((void *)p, h->stream);
    p = nullptr;
}

void freeMonitors(fdtd_solver *h)
{
    release(h, h->dEdge);
    release(h, h->dEdgeOff);
    release(h, h->dAmps);
    release(h, h->dPoff);
    release(h, h->dPpol);
    release(h, h->dPcells);
    release(h, h->dProbe);
    release(h, h->dVrec);
    release(h, h->dIrec);
    release(h, h->dPrec);
    release(h, h->dEhist);
    release(h, h->dEpart);
    SurfaceState &s = h->surf;
    release(h, s.dJsNode);
    release(h, s.dHuyNode);
    release(h, s.dJsInst);
    release(h, s.dJsAcc);
    release(h, s.dHuyAcc);
    release(h, s.dPlane);
    release(h, s.dFrames);
    s.planeCap = 0;
    s.planeValid = false;
    s.framesCap = s.framesUsed = 0;
    s.frames.clear();
    h->recCap = 0;
    h->prepared = false;
}

void freeAll(fdtd_solver *h)
{
    freeMonitors(h);
    for (int c = 0; c < 6; ++c) release(h, h->dField[c]);
    for (int c = 0; c < 3; ++c)
    {
        release(h, h->dMask[c]);
        release(h, h->dCa[c]);
        release(h, h->dCb[c]);
    }
    release(h, h->mur.snap);
}

tlm_status ready(fdtd_solver *h)
{
    if (!h)
    {
        g_fdtdErr = "null handle";
        return TLM_EINVAL;
    }
    if (!h->configured) return h->fail(TLM_ESTATE, "fdtd_setup has not been called");
    return TLM_OK;
}

float sourceValue(const fdtd_solver *h, int n)
{
    if (h->cfg.waveform == TLM_WAVE_TABLE) return (n >= 0 && n < (int)h->svTable.size()) ? h->svTable[n] : 0.0f;
    return tlmh::waveform_f32(h->cfg.waveform, h->cfg.f0, h->dt, n);
}

tlm_status ensureRecords(fdtd_solver *h, long long need)
{
    if (need <= h->recCap) return TLM_OK;
    long long cap = std::max<long long>(need, std::max<long long>(h->cfg.total_steps, 64));
    cap = std::max(cap, h->recCap * 2);
    const int np = std::max<int>((int)h->ports.size(), 1), nr = std::max<int>((int)h->probeCells.size(), 1);
    float *v = nullptr, *i = nullptr, *p = nullptr;
    double *e = nullptr;
    FD_TRY(alloc(h, &v, (size_t)cap * np * 4));
    FD_TRY(alloc(h, &i, (size_t)cap * np * 4));
    FD_TRY(alloc(h, &p, (size_t)cap * nr * 3 * 4));
    FD_TRY(alloc(h, &e, (size_t)(cap / 16 + 2) * 8));
    if (h->recCap > 0)
    {
        FD_CU(h, cudaMemcpyAsync(v, h->dVrec, (size_t)h->recCap * np * 4, cudaMemcpyDeviceToDevice, h->stream));
        FD_CU(h, cudaMemcpyAsync(i, h->dIrec, (size_t)h->recCap * np * 4, cudaMemcpyDeviceToDevice, h->stream));
        FD_CU(h, cudaMemcpyAsync(p, h->dPrec, (size_t)h->recCap * nr * 12, cudaMemcpyDeviceToDevice, h->stream));
        FD_CU(h, cudaMemcpyAsync(e, h->dEhist, (size_t)(h->recCap / 16 + 2) * 8, cudaMemcpyDeviceToDevice,
                                 h->stream));
    }
    release(h, h->dVrec);
    release(h, h->dIrec);
    release(h, h->dPrec);
    release(h, h->dEhist);
    h->dVrec = v;
    h->dIrec = i;
    h->dPrec = p;
    h->dEhist = e;
    h->recCap = cap;
    return TLM_OK;
}

// Source edges in CSR form: every E edge a source cell drives, with its
// amplitudes in the reference's order (plane-wave cells, then port cells).
tlm_status prepare(fdtd_solver *h)
{
    if (h->prepared) return TLM_OK;
    freeMonitors(h);
    const fdk::Dims &d = h->d;
    std::map<long long, std::vector<float>> edges;  // per edge, amplitudes in source order
    auto add = [&](uint64_t cell, int pol, float amp) {
        const int i = (int)(cell % d.nx), j = (int)((cell / d.nx) % d.ny), k = (int)(cell / ((uint64_t)d.nx * d.ny));
        long long idx[4];
        if (pol == 0)
        {
            idx[0] = d.iEx(i, j, k); idx[1] = d.iEx(i, j + 1, k); idx[2] = d.iEx(i, j, k + 1); idx[3] = d.iEx(i, j + 1, k + 1);
        }
        else if (pol == 1)
        {
            idx[0] = d.iEy(i, j, k); idx[1] = d.iEy(i + 1, j, k); idx[2] = d.iEy(i, j, k + 1); idx[3] = d.iEy(i + 1, j, k + 1);
        }
        else
        {
            idx[0] = d.iEz(i, j, k); idx[1] = d.iEz(i + 1, j, k); idx[2] = d.iEz(i, j + 1, k); idx[3] = d.iEz(i + 1, j + 1, k);
        }
        for (int e = 0; e < 4; ++e)
            if (h->maskHost(pol, idx[e])) edges[((long long)pol << 60) | idx[e]].push_back(amp);
    };
    for (const auto &s : h->planeSources) add(s.cell, s.pol, s.amp);
    for (const auto &p : h->ports)
        for (uint64_t c : p.cells) add(c, p.pol, p.amp);
    std::vector<long long> code;
    std::vector<int> off(1, 0);
    std::vector<float> amps;
    for (const auto &kv : edges)
    {
        code.push_back(kv.first);
        amps.insert(amps.end(), kv.second.begin(), kv.second.end());
        off.push_back((int)amps.size());
    }
    h->nEdges = (int)code.size();
    if (h->nEdges)
    {
        FD_TRY(alloc(h, &h->dEdge, code.size() * 8));
        FD_TRY(alloc(h, &h->dEdgeOff, off.size() * 4));
        FD_TRY(alloc(h, &h->dAmps, amps.size() * 4));
        FD_CU(h, cudaMemcpyAsync(h->dEdge, code.data(), code.size() * 8, cudaMemcpyHostToDevice, h->stream));
        FD_CU(h, cudaMemcpyAsync(h->dEdgeOff, off.data(), off.size() * 4, cudaMemcpyHostToDevice, h->stream));
        FD_CU(h, cudaMemcpyAsync(h->dAmps, amps.data(), amps.size() * 4, cudaMemcpyHostToDevice, h->stream));
    }
    // ports and probes
    const int np = (int)h->ports.size();
    std::vector<int> poff(np + 1, 0), ppol(std::max(np, 1), 0);
    std::vector<long long> pcells;
    for (int p = 0; p < np; ++p)
    {
        for (uint64_t c : h->ports[p].cells) pcells.push_back((long long)c);
        poff[p + 1] = (int)pcells.size();
        ppol[p] = h->ports[p].pol;
    }
    if (pcells.empty()) pcells.push_back(0);
    std::vector<long long> probes(h->probeCells.begin(), h->probeCells.end());
    if (probes.empty()) probes.push_back(0);
    FD_TRY(alloc(h, &h->dPoff, poff.size() * 4));
    FD_TRY(alloc(h, &h->dPpol, ppol.size() * 4));
    FD_TRY(alloc(h, &h->dPcells, pcells.size() * 8));
    FD_TRY(alloc(h, &h->dProbe, probes.size() * 8));
    FD_CU(h, cudaMemcpyAsync(h->dPoff, poff.data(), poff.size() * 4, cudaMemcpyHostToDevice, h->stream));
    FD_CU(h, cudaMemcpyAsync(h->dPpol, ppol.data(), ppol.size() * 4, cudaMemcpyHostToDevice, h->stream));
    FD_CU(h, cudaMemcpyAsync(h->dPcells, pcells.data(), pcells.size() * 8, cudaMemcpyHostToDevice, h->stream));
    FD_CU(h, cudaMemcpyAsync(h->dProbe, probes.data(), probes.size() * 8, cudaMemcpyHostToDevice, h->stream));
    // surface faces
    SurfaceState &s = h->surf;
    auto upload = [&](long long **dst, const std::vector<uint64_t> &cells, const std::vector<int> &axis,
                      const std::vector<int> *sign) -> tlm_status {
        if (cells.empty()) return TLM_OK;
        std::vector<long long> c(cells.size());
        for (size_t f = 0; f < cells.size(); ++f)
            c[f] = (long long)cells[f] * 8 + axis[f] * 2 + ((sign && (*sign)[f] < 0) ? 1 : 0);
        FD_TRY(alloc(h, dst, c.size() * 8));
        FD_CU(h, cudaMemcpyAsync(*dst, c.data(), c.size() * 8, cudaMemcpyHostToDevice, h->stream));
        FD_CU(h, cudaStreamSynchronize(h->stream));
        return TLM_OK;
    };
    FD_TRY(upload(&s.dJsNode, s.jsCell, s.jsAxis, nullptr));
    FD_TRY(upload(&s.dHuyNode, s.huyCell, s.huyAxis, &s.huySign));
    const size_t nj = s.jsCell.size(), nh = s.huyCell.size();
    if (nj)
    {
        FD_TRY(alloc(h, (float **)&s.dJsInst, nj * 4));
        FD_TRY(alloc(h, (float **)&s.dJsAcc, nj * 16));
        FD_CU(h, cudaMemsetAsync(s.dJsInst, 0, nj * 4, h->stream));
        FD_CU(h, cudaMemsetAsync(s.dJsAcc, 0, nj * 16, h->stream));
    }
    if (nh)
    {
        FD_TRY(alloc(h, (float **)&s.dHuyAcc, nh * 32));
        FD_CU(h, cudaMemsetAsync(s.dHuyAcc, 0, nh * 32, h->stream));
    }
    h->nEpart = 148 * 4;
    FD_TRY(alloc(h, &h->dEpart, (size_t)h->nEpart * 8));
    FD_TRY(ensureRecords(h, std::max(h->cfg.total_steps, 1)));
    FD_CU(h, cudaStreamSynchronize(h->stream));
    h->prepared = true;
    return TLM_OK;
}

tlm_status launchStep(fdtd_solver *h, int n)
{
    const fdk::Dims &d = h->d;
    fdk::Fields f;
    for (int c = 0; c < 3; ++c)
    {
        f.E[c] = static_cast<float *>(h->dField[c]);
        f.H[c] = static_cast<float *>(h->dField[3 + c]);
        f.mE[c] = h->dMask[c];
        f.ca[c] = h->dCa[c];
        f.cb[c] = h->dCb[c];
    }
    const float sv = sourceValue(h, n);
    // 1. soft sources
    if (h->nEdges)
        fdk::injectKernel<<<(h->nEdges + 255) / 256, 256, 0, h->stream>>>(f, h->dEdge, h->dEdgeOff, h->dAmps,
                                                                         h->nEdges, sv);
    // 2. monitors
    SurfaceState &s = h->surf;
    const int nj = (int)s.jsCell.size(), nhuy = (int)s.huyCell.size();
    const bool doDft = n >= h->cfg.settle_steps;
    const bool doPlane = s.planeAxis >= 0 && (n % 2) == 0;
    int n1 = 0, n2 = 0;
    if (doPlane)
    {
        const int dims[3] = { d.nx, d.ny, d.nz };
        n1 = dims[s.planeAxis == 0 ? 1 : 0];
        n2 = dims[s.planeAxis == 2 ? 1 : 2];
        if ((size_t)n1 * n2 > s.planeCap)
        {
            release(h, s.dPlane);
            FD_TRY(alloc(h, (float **)&s.dPlane, (size_t)n1 * n2 * 4));
            s.planeCap = (size_t)n1 * n2;
        }
    }
    fdk::MonArgs a;
    a.f = f;
    a.d = d;
    a.dl = h->g.dl;
    a.eta0 = tlmh::eta0_f32();
    a.step = n;
    a.nports = (int)h->ports.size();
    a.poff = h->dPoff;
    a.pcells = h->dPcells;
    a.ppol = h->dPpol;
    a.vrec = h->dVrec;
    a.irec = h->dIrec;
    a.nprobes = (int)h->probeCells.size();
    a.probeCell = h->dProbe;
    a.prec = h->dPrec;
    a.njs = nj;
    a.jsCode = s.dJsNode;
    a.jsInst = static_cast<float *>(s.dJsInst);
    a.jsAcc = static_cast<float *>(s.dJsAcc);
    a.nhuy = nhuy;
    a.huyCode = s.dHuyNode;
    a.huyAcc = static_cast<float *>(s.dHuyAcc);
    a.doDft = doDft ? 1 : 0;
    a.cph = a.sph = 0.0f;
    if (doDft && (nj || nhuy)) tlmh::dft_phase_f32(h->cfg.f0, h->dt, n, &a.cph, &a.sph);
    a.planeAxis = doPlane ? s.planeAxis : -1;
    a.planeIndex = doPlane ? std::min(std::max(s.planeIndex, 0),
                                      (s.planeAxis == 0 ? d.nx : s.planeAxis == 1 ? d.ny : d.nz) - 1)
                           : 0;
    a.planeN1 = n1;
    a.planeN2 = n2;
    a.plane = static_cast<float *>(s.dPlane);
    const long long items = (long long)a.nports + a.nprobes + nj + (doDft ? nhuy : 0) + (doPlane ? (long long)n1 * n2 : 0);
    if (items > 0) fdk::monitorKernel<<<(unsigned)((items + 255) / 256), 256, 0, h->stream>>>(a);
    if (doPlane)
    {
        s.planeValid = true;
        s.planeAxisDone = s.planeAxis;
        s.planeIndexDone = a.planeIndex;
        s.planeN1 = n1;
        s.planeN2 = n2;
    }
    if ((n & 15) == 0)
    {
        const double eta = (double)tlmh::eta0_f32();
        fdk::energyPartialKernel<<<h->nEpart, 256, 0, h->stream>>>(f, h->len[0], h->len[1], h->len[2], h->len[3],
                                                                  h->len[4], h->len[5], eta * eta, h->dEpart);
        fdk::energyFinalKernel<<<1, 256, 0, h->stream>>>(h->dEpart, h->nEpart, h->dEhist + n / 16);
    }
    if (h->cfg.record_every > 0 && (n % h->cfg.record_every) == 0)
    {
        const bool withPlane = s.planeAxis >= 0 && s.planeValid;
        const size_t np = withPlane ? (size_t)s.planeN1 * s.planeN2 : 0;
        const size_t need = s.framesUsed + nj + np;
        if (need > s.framesCap)
        {
            const size_t cap = std::max(need, s.framesCap * 2 + 1024);
            float *dn = nullptr;
            FD_TRY(alloc(h, &dn, cap * 4));
            if (s.framesUsed)
                FD_CU(h, cudaMemcpyAsync(dn, s.dFrames, s.framesUsed * 4, cudaMemcpyDeviceToDevice, h->stream));
            release(h, s.dFrames);
            s.dFrames = dn;
            s.framesCap = cap;
        }
        float *base = static_cast<float *>(s.dFrames) + s.framesUsed;
        if (nj) FD_CU(h, cudaMemcpyAsync(base, s.dJsInst, nj * 4, cudaMemcpyDeviceToDevice, h->stream));
        if (np) FD_CU(h, cudaMemcpyAsync(base + nj, s.dPlane, np * 4, cudaMemcpyDeviceToDevice, h->stream));
        SurfaceState::Frame fr;
        fr.step = n;
        fr.hasPlane = withPlane ? 1 : 0;
        fr.axis = withPlane ? s.planeAxisDone : -1;
        fr.index = withPlane ? s.planeIndexDone : 0;
        fr.n1 = withPlane ? s.planeN1 : 0;
        fr.n2 = withPlane ? s.planeN2 : 0;
        fr.off = s.framesUsed;
        s.frames.push_back(fr);
        s.framesUsed = need;
    }
    // 3. H, 4. Mur snapshot, E, Mur
    fdk::Box box;
    box.total = (unsigned)((long long)(d.nx + 1) * (d.ny + 1) * (d.nz + 1));
    box.divX = tlmk::makeFastDiv((unsigned)(d.nx + 1));
    box.divY = tlmk::makeFastDiv((unsigned)(d.ny + 1));
    const unsigned grid = (box.total + 255) / 256;
    long long snapItems = 0;
    for (int F = 0; F < 6; ++F) snapItems += (long long)h->mur.n1[F] * h->mur.n2[F];
    const unsigned snapBlocks = (unsigned)((snapItems + 255) / 256);
    fdk::updateHKernel<<<grid + snapBlocks, 256, 0, h->stream>>>(f, d, box, h->ch, h->mur, grid);
    fdk::updateEKernel<<<grid, 256, 0, h->stream>>>(f, d, box, h->cb0);
    long long aItems = 0, bItems = 0;
    for (int F = 0; F < 3; ++F) aItems += (long long)h->mur.n1[F] * h->mur.n2[F];
    for (int F = 3; F < 6; ++F) bItems += (long long)h->mur.n1[F] * h->mur.n2[F];
    fdk::murApplyKernel<0><<<(unsigned)((aItems + 255) / 256), 256, 0, h->stream>>>(f, d, h->mur);
    fdk::murApplyKernel<3><<<(unsigned)((bItems + 255) / 256), 256, 0, h->stream>>>(f, d, h->mur);
    return h->cuda(cudaGetLastError(), "FDTD step launch");
}

} // namespace

extern "C" {

tlm_status fdtd_create(fdtd_handle *out, int device)
{
    if (!out)
    {
        g_fdtdErr = "null output";
        return TLM_EINVAL;
    }
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        g_fdtdErr = "no CUDA device";
        return TLM_ENODEV;
    }
    if (device < 0 || device >= count)
    {
        g_fdtdErr = "no such device";
        return TLM_EINVAL;
    }
    fdtd_solver *h = new fdtd_solver();
    h->device = device;
    Guard g(device);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    {
        cudaGetLastError();
        delete h;
        g_fdtdErr = "stream creation failed";
        return TLM_ECUDA;
    }
    h->pool = tlmi::devicePool(device);
    if (!h->pool)
    {
        cudaStreamDestroy(h->stream);
        delete h;
        g_fdtdErr = "memory pool unavailable";
        return TLM_ECUDA;
    }
    *out = h;
    return TLM_OK;
}

tlm_status fdtd_destroy(fdtd_handle h)
{
    if (!h) return TLM_OK;
    {
        Guard g(h->device);
        cudaStreamSynchronize(h->stream);
        freeAll(h);
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
    }
    delete h;
    return TLM_OK;
}

const char *fdtd_last_error(fdtd_handle h) { return h ? h->err.c_str() : g_fdtdErr.c_str(); }

tlm_status fdtd_setup(fdtd_handle h, const tlm_grid *grid, const uint8_t *mat, size_t n_cells,
                      const tlm_matprops *table, int n_table, const tlm_config *cfg)
{
    if (!h)
    {
        g_fdtdErr = "null handle";
        return TLM_EINVAL;
    }
    if (!grid || !mat || !cfg || (n_table > 0 && !table) || n_table < 0)
        return h->fail(TLM_EINVAL, "null grid, material map, table or config");
    if (grid->nx < 2 || grid->ny < 2 || grid->nz < 2) return h->fail(TLM_EINVAL, "grid must be at least 2 cells per axis");
    if ((long long)(grid->nx + 1) * (grid->ny + 1) * (grid->nz + 1) >= (1LL << 31))
        return h->fail(TLM_EINVAL, "grid too large");
    if (!(grid->dl > 0.0f)) return h->fail(TLM_EINVAL, "dl must be positive");
    const size_t n = (size_t)grid->nx * grid->ny * grid->nz;
    if (n_cells != n) return h->fail(TLM_EINVAL, "material map does not match the grid");
    for (size_t c = 0; c < n; ++c)
        if (mat[c] >= TLM_MAT_DIEL0 && (int)(mat[c] - TLM_MAT_DIEL0) >= n_table)
            return h->fail(TLM_EINVAL, "material id without a table entry");
    if (cfg->waveform < 0 || cfg->waveform > TLM_WAVE_TABLE) return h->fail(TLM_EINVAL, "unknown waveform");
    if (cfg->record_every < 0 || cfg->huy_offset < 0) return h->fail(TLM_EINVAL, "negative record_every or huy_offset");
    Guard gd(h->device);
    cudaStreamSynchronize(h->stream);
    freeAll(h);
    h->configured = false;
    h->g = *grid;
    h->cfg = *cfg;
    h->mat.assign(mat, mat + n);
    h->table.assign(table, table + n_table);
    h->d = fdk::Dims{ grid->nx, grid->ny, grid->nz };
    const fdk::Dims &d = h->d;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    h->dt = tlmh::fdtd_dt(grid->dl);
    h->cMur = tlmh::fdtd_cmur(h->dt, grid->dl);
    h->cb0 = tlmh::fdtd_cb0(h->dt, grid->dl);
    h->ch = tlmh::fdtd_ch(h->dt, grid->dl);
    h->haveDiel = false;
    for (size_t c = 0; c < n; ++c)
        if (mat[c] >= TLM_MAT_DIEL0)
        {
            h->haveDiel = true;
            break;
        }
    h->len[0] = (long long)nx * (ny + 1) * (nz + 1);
    h->len[1] = (long long)(nx + 1) * ny * (nz + 1);
    h->len[2] = (long long)(nx + 1) * (ny + 1) * nz;
    h->len[3] = (long long)(nx + 1) * ny * nz;
    h->len[4] = (long long)nx * (ny + 1) * nz;
    h->len[5] = (long long)nx * ny * (nz + 1);
    // per-edge classification (FdtdSolver.cpp:135-231)
    std::vector<float> ca[3], cb[3];
    for (int c = 0; c < 3; ++c)
    {
        h->hMask[c].assign((size_t)h->len[c], 1);
        if (h->haveDiel)
        {
            ca[c].assign((size_t)h->len[c], 1.0f);
            cb[c].assign((size_t)h->len[c], h->cb0);
        }
    }
    const int ext[3][3] = { { nx, ny + 1, nz + 1 }, { nx + 1, ny, nz + 1 }, { nx + 1, ny + 1, nz } };
    for (int axis = 0; axis < 3; ++axis)
    {
        const int t1 = axis == 0 ? 1 : 0, t2 = axis == 2 ? 1 : 2;
        for (int k = 0; k < ext[axis][2]; ++k)
            for (int j = 0; j < ext[axis][1]; ++j)
                for (int i = 0; i < ext[axis][0]; ++i)
                {
                    const long long q = axis == 0 ? d.iEx(i, j, k) : axis == 1 ? d.iEy(i, j, k) : d.iEz(i, j, k);
                    bool pec = false;
                    float eAcc = 0.0f, sAcc = 0.0f;
                    int cnt = 0;
                    for (int d1 = -1; d1 <= 0; ++d1)
                        for (int d2 = -1; d2 <= 0; ++d2)
                        {
                            int co[3] = { i, j, k };
                            co[t1] += d1;
                            co[t2] += d2;
                            if (co[0] < 0 || co[1] < 0 || co[2] < 0 || co[0] >= nx || co[1] >= ny || co[2] >= nz)
                                continue;
                            const uint8_t m = mat[((size_t)co[2] * ny + co[1]) * nx + co[0]];
                            float e1 = 1.0f, s1 = 0.0f;
                            if (m == TLM_MAT_PEC)
                                pec = true;
                            else if (m >= TLM_MAT_DIEL0)
                            {
                                e1 += table[m - TLM_MAT_DIEL0].epsr - 1.0f;
                                s1 += table[m - TLM_MAT_DIEL0].sigma;
                            }
                            eAcc += e1;
                            sAcc += s1;
                            ++cnt;
                        }
                    if (pec)
                    {
                        h->hMask[axis][(size_t)q] = 0;
                        if (h->haveDiel)
                        {
                            ca[axis][(size_t)q] = 0.0f;
                            cb[axis][(size_t)q] = 0.0f;
                        }
                        continue;
                    }
                    if (h->haveDiel && cnt > 0)
                        tlmh::fdtd_edge_coef(eAcc, sAcc, cnt, h->dt, grid->dl, &ca[axis][(size_t)q],
                                             &cb[axis][(size_t)q]);
                }
    }
    size_t need = 0;
    for (int c = 0; c < 6; ++c) need += (size_t)h->len[c] * 4;
    for (int c = 0; c < 3; ++c) need += (size_t)h->len[c] * (h->haveDiel ? 9 : 1);
    if (need + ((size_t)256 << 20) > tlmi::poolAvailable(h->device))
        return h->fail(TLM_ENOMEM, "grid needs " + std::to_string(need >> 20) + " MiB of HBM");
    for (int c = 0; c < 6; ++c)
    {
        FD_TRY(alloc(h, &h->dField[c], (size_t)h->len[c] * 4));
        if (reinterpret_cast<uintptr_t>(h->dField[c]) & 15)  // the energy sweep reads 16-byte vectors
            return h->fail(TLM_ECUDA, "field allocation not 16-byte aligned");
        FD_CU(h, cudaMemsetAsync(h->dField[c], 0, (size_t)h->len[c] * 4, h->stream));
    }
    for (int c = 0; c < 3; ++c)
    {
        FD_TRY(alloc(h, &h->dMask[c], (size_t)h->len[c]));
        FD_CU(h, cudaMemcpyAsync(h->dMask[c], h->hMask[c].data(), (size_t)h->len[c], cudaMemcpyHostToDevice,
                                 h->stream));
        if (h->haveDiel)
        {
            FD_TRY(alloc(h, &h->dCa[c], (size_t)h->len[c] * 4));
            FD_TRY(alloc(h, &h->dCb[c], (size_t)h->len[c] * 4));
            FD_CU(h, cudaMemcpyAsync(h->dCa[c], ca[c].data(), (size_t)h->len[c] * 4, cudaMemcpyHostToDevice, h->stream));
            FD_CU(h, cudaMemcpyAsync(h->dCb[c], cb[c].data(), (size_t)h->len[c] * 4, cudaMemcpyHostToDevice, h->stream));
        }
    }
    // Mur planes: x faces (Ey, Ez), y faces (Ex, Ez), z faces (Ex, Ey)
    const int n1[6] = { ny, ny + 1, nx, nx + 1, nx, nx + 1 };
    const int n2[6] = { nz + 1, nz, nz + 1, nz, ny + 1, ny };
    long long total = 0;
    for (int F = 0; F < 6; ++F)
    {
        h->mur.n1[F] = n1[F];
        h->mur.n2[F] = n2[F];
        h->mur.off[F] = total;
        total += 4LL * n1[F] * n2[F];
    }
    h->mur.cMur = h->cMur;
    FD_TRY(alloc(h, &h->mur.snap, (size_t)total * 4));
    FD_CU(h, cudaMemsetAsync(h->mur.snap, 0, (size_t)total * 4, h->stream));
    FD_CU(h, cudaStreamSynchronize(h->stream));
    h->planeSources.clear();
    h->ports.clear();
    h->probeCells.clear();
    h->svTable.clear();
    h->surf = SurfaceState();
    tlmi::buildFaceLists(nx, ny, nz, grid->origin, grid->dl, mat, cfg->surface_monitors != 0, cfg->huy_offset,
                         h->surf);
    h->curStep = 0;
    h->prepared = false;
    h->configured = true;
    return TLM_OK;
}

tlm_status fdtd_add_port(fdtd_handle h, const uint64_t *cells, int n_cells, int pol_axis, float amp, int *idx)
{
    FD_TRY(ready(h));
    if (h->curStep > 0) return h->fail(TLM_ESTATE, "ports must be added before the first step");
    if (pol_axis < 0 || pol_axis > 2 || n_cells < 0 || (n_cells > 0 && !cells))
        return h->fail(TLM_EINVAL, "bad port");
    fdtd_solver::Port p;
    p.pol = pol_axis;
    p.amp = amp;
    for (int t = 0; t < n_cells; ++t)
        if (cells[t] < h->mat.size() && h->mat[cells[t]] == TLM_MAT_AIR) p.cells.push_back(cells[t]);
    if (!p.cells.empty())
    {
        const uint64_t c = p.cells[p.cells.size() / 2];
        int co[3] = { (int)(c % h->d.nx), (int)((c / h->d.nx) % h->d.ny), (int)(c / ((uint64_t)h->d.nx * h->d.ny)) };
        const int dims[3] = { h->d.nx, h->d.ny, h->d.nz };
        for (int a : { (pol_axis + 1) % 3, (pol_axis + 2) % 3 })
            if (co[a] < 1 || co[a] > dims[a] - 2)
                return h->fail(TLM_EINVAL, "the port's current loop leaves the grid");
    }
    h->ports.push_back(p);
    h->prepared = false;
    if (idx) *idx = (int)h->ports.size() - 1;
    return TLM_OK;
}

tlm_status fdtd_add_plane_wave(fdtd_handle h, int prop_axis, int plane_index, int pol_axis, float amp)
{
    FD_TRY(ready(h));
    if (h->curStep > 0) return h->fail(TLM_ESTATE, "sources must be added before the first step");
    if (prop_axis < 0 || prop_axis > 2 || pol_axis < 0 || pol_axis > 2) return h->fail(TLM_EINVAL, "bad axis");
    for (int k = 0; k < h->d.nz; ++k)
        for (int j = 0; j < h->d.ny; ++j)
            for (int i = 0; i < h->d.nx; ++i)
            {
                const int co[3] = { i, j, k };
                if (co[prop_axis] != plane_index) continue;
                const size_t c = ((size_t)k * h->d.ny + j) * h->d.nx + i;
                if (h->mat[c] == TLM_MAT_AIR) h->planeSources.push_back({ c, pol_axis, amp });
            }
    h->prepared = false;
    return TLM_OK;
}

tlm_status fdtd_add_probe(fdtd_handle h, float x, float y, float z, int *idx)
{
    FD_TRY(ready(h));
    if (h->curStep > 0) return h->fail(TLM_ESTATE, "probes must be added before the first step");
    int i, j, k;
    tlmh::cell_of(h->g.origin, h->g.dl, x, y, z, &i, &j, &k);
    if (i < 0 || j < 0 || k < 0 || i >= h->d.nx || j >= h->d.ny || k >= h->d.nz)
    {
        if (idx) *idx = -1;
        return TLM_OK;
    }
    h->probeCells.push_back(((uint64_t)k * h->d.ny + j) * h->d.nx + i);
    h->prepared = false;
    if (idx) *idx = (int)h->probeCells.size() - 1;
    return TLM_OK;
}

tlm_status fdtd_set_source_table(fdtd_handle h, const float *values, int n)
{
    FD_TRY(ready(h));
    if (n < 0 || (n > 0 && !values)) return h->fail(TLM_EINVAL, "bad source table");
    h->svTable.assign(values, values + n);
    h->cfg.waveform = TLM_WAVE_TABLE;
    return TLM_OK;
}

tlm_status fdtd_step(fdtd_handle h, int n_steps)
{
    FD_TRY(ready(h));
    if (n_steps < 0) return h->fail(TLM_EINVAL, "n_steps must be >= 0");
    Guard gd(h->device);
    FD_TRY(prepare(h));
    FD_TRY(ensureRecords(h, (long long)h->curStep + n_steps));
    for (int t = 0; t < n_steps; ++t)
    {
        FD_TRY(launchStep(h, h->curStep));
        ++h->curStep;
    }
    FD_CU(h, cudaStreamSynchronize(h->stream));
    return TLM_OK;
}

tlm_status fdtd_run(fdtd_handle h)
{
    FD_TRY(ready(h));
    return fdtd_step(h, std::max(0, h->cfg.total_steps - h->curStep));
}

int fdtd_current_step(fdtd_handle h) { return h ? h->curStep : 0; }
tlm_status fdtd_get_stream(fdtd_handle h, void **stream)
{
    if (!h || !stream)
    {
        g_fdtdErr = "null handle or output";
        return TLM_EINVAL;
    }
    *stream = (void *)h->stream;
    return TLM_OK;
}
float fdtd_timestep(fdtd_handle h) { return h ? h->dt : 0.0f; }

tlm_status fdtd_get_grid(fdtd_handle h, tlm_grid *grid)
{
    FD_TRY(ready(h));
    if (!grid) return h->fail(TLM_EINVAL, "null output");
    *grid = h->g;
    return TLM_OK;
}

tlm_status fdtd_get_field(fdtd_handle h, int which, float *out, size_t cap, size_t *n)
{
    FD_TRY(ready(h));
    if (which < 0 || which > 5) return h->fail(TLM_EINVAL, "which must be 0..5 (Ex Ey Ez Hx Hy Hz)");
    if (n) *n = (size_t)h->len[which];
    if (!out) return TLM_OK;
    if (cap < (size_t)h->len[which]) return h->fail(TLM_EINVAL, "output smaller than the field");
    Guard gd(h->device);
    FD_CU(h, cudaStreamSynchronize(h->stream));
    FD_CU(h, cudaMemcpy(out, h->dField[which], (size_t)h->len[which] * 4, cudaMemcpyDeviceToHost));
    return TLM_OK;
}

tlm_status fdtd_get_probe(fdtd_handle h, int idx, float *ex, float *ey, float *ez, int cap, int *n)
{
    FD_TRY(ready(h));
    const int nr = (int)h->probeCells.size();
    if (idx < 0 || idx >= nr) return h->fail(TLM_EINVAL, "no such probe");
    const int steps = h->curStep;
    if (n) *n = steps;
    const int m = std::min(steps, cap);
    if (m <= 0 || !h->dPrec) return TLM_OK;
    Guard gd(h->device);
    std::vector<float> all((size_t)m * nr * 3);
    FD_CU(h, cudaMemcpy(all.data(), h->dPrec, all.size() * 4, cudaMemcpyDeviceToHost));
    for (int t = 0; t < m; ++t)
    {
        if (ex) ex[t] = all[((size_t)t * nr + idx) * 3];
        if (ey) ey[t] = all[((size_t)t * nr + idx) * 3 + 1];
        if (ez) ez[t] = all[((size_t)t * nr + idx) * 3 + 2];
    }
    return TLM_OK;
}

tlm_status fdtd_get_port(fdtd_handle h, int idx, float *v, float *i, int cap, int *n)
{
    FD_TRY(ready(h));
    const int np = (int)h->ports.size();
    if (idx < 0 || idx >= np) return h->fail(TLM_EINVAL, "no such port");
    const int steps = h->curStep;
    if (n) *n = steps;
    const int m = std::min(steps, cap);
    if (m <= 0 || !h->dVrec) return TLM_OK;
    Guard gd(h->device);
    std::vector<float> vv((size_t)m * np), ii((size_t)m * np);
    FD_CU(h, cudaMemcpy(vv.data(), h->dVrec, vv.size() * 4, cudaMemcpyDeviceToHost));
    FD_CU(h, cudaMemcpy(ii.data(), h->dIrec, ii.size() * 4, cudaMemcpyDeviceToHost));
    for (int t = 0; t < m; ++t)
    {
        if (v) v[t] = vv[(size_t)t * np + idx];
        if (i) i[t] = ii[(size_t)t * np + idx];
    }
    return TLM_OK;
}

tlm_status fdtd_get_energy_history(fdtd_handle h, int *steps, float *vals, double *vals64, int cap, int *n)
{
    FD_TRY(ready(h));
    const int ne = h->curStep > 0 ? (h->curStep - 1) / 16 + 1 : 0;
    if (n) *n = ne;
    const int m = std::min(ne, cap);
    if (m <= 0 || !h->dEhist) return TLM_OK;
    Guard gd(h->device);
    std::vector<double> buf(m);
    FD_CU(h, cudaMemcpy(buf.data(), h->dEhist, (size_t)m * 8, cudaMemcpyDeviceToHost));
    for (int t = 0; t < m; ++t)
    {
        if (steps) steps[t] = 16 * t;
        if (vals) vals[t] = (float)buf[t];
        if (vals64) vals64[t] = buf[t];
    }
    return TLM_OK;
}

// ---- surface monitors, cut plane, frames, far field -----------------------
tlm_status fdtd_get_surface_faces(fdtd_handle h, uint64_t *air_cells, int *axis, int *sign, float *centers, int cap,
                                  int *n)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    const int nf = (int)s.jsCell.size();
    if (n) *n = nf;
    for (int f = 0; f < nf && f < cap; ++f)
    {
        if (air_cells) air_cells[f] = s.jsCell[f];
        if (axis) axis[f] = s.jsAxis[f];
        if (sign) sign[f] = s.jsSign[f];
        if (centers) std::memcpy(centers + 3 * f, &s.jsCenter[3 * f], 12);
    }
    return TLM_OK;
}

static int fdtdSamples(const fdtd_solver *h) { return std::max(0, h->curStep - std::max(h->cfg.settle_steps, 0)); }

tlm_status fdtd_get_js_instant(fdtd_handle h, float *out, int cap, int *n)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    const int nf = (int)s.jsCell.size();
    if (n) *n = nf;
    if (!out || cap <= 0 || nf == 0) return TLM_OK;
    if (!s.dJsInst)
    {
        std::fill(out, out + std::min(nf, cap), 0.0f);
        return TLM_OK;
    }
    Guard gd(h->device);
    FD_CU(h, cudaStreamSynchronize(h->stream));
    std::vector<float> t(nf);
    FD_CU(h, cudaMemcpy(t.data(), s.dJsInst, (size_t)nf * 4, cudaMemcpyDeviceToHost));
    std::copy(t.begin(), t.begin() + std::min(nf, cap), out);
    return TLM_OK;
}

tlm_status fdtd_get_js_dft(fdtd_handle h, float *magnitude, float *re, float *im, int cap, int *n, int *samples)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    const int nf = (int)s.jsCell.size();
    const int ns = nf ? fdtdSamples(h) : 0;
    if (n) *n = nf;
    if (samples) *samples = ns;
    if (nf == 0 || cap <= 0) return TLM_OK;
    std::vector<float> acc((size_t)nf * 4, 0.0f);
    if (s.dJsAcc)
    {
        Guard gd(h->device);
        FD_CU(h, cudaStreamSynchronize(h->stream));
        FD_CU(h, cudaMemcpy(acc.data(), s.dJsAcc, acc.size() * 4, cudaMemcpyDeviceToHost));
    }
    for (int f = 0; f < nf && f < cap; ++f)
    {
        const float r1 = acc[4 * f], i1 = acc[4 * f + 1], r2 = acc[4 * f + 2], i2 = acc[4 * f + 3];
        if (re) { re[2 * f] = r1; re[2 * f + 1] = r2; }
        if (im) { im[2 * f] = i1; im[2 * f + 1] = i2; }
        if (magnitude)
        {
            float m = 0.0f;
            if (ns > 0)
            {
                const float norm = 2.0f / (float)ns;
                m = norm * std::sqrt(r1 * r1 + i1 * i1 + r2 * r2 + i2 * i2);
            }
            magnitude[f] = m;
        }
    }
    return TLM_OK;
}

tlm_status fdtd_get_huygens_faces(fdtd_handle h, uint64_t *cells, int *axis, int *out_sign, float *pos, int cap,
                                  int *n)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    const int nh = (int)s.huyCell.size();
    if (n) *n = nh;
    for (int f = 0; f < nh && f < cap; ++f)
    {
        if (cells) cells[f] = s.huyCell[f];
        if (axis) axis[f] = s.huyAxis[f];
        if (out_sign) out_sign[f] = s.huySign[f];
        if (pos) std::memcpy(pos + 3 * f, &s.huyPos[3 * f], 12);
    }
    return TLM_OK;
}

tlm_status fdtd_get_huygens_dft(fdtd_handle h, float *acc8, int cap, int *n, int *samples)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    const int nh = (int)s.huyCell.size();
    if (n) *n = nh;
    if (samples) *samples = nh ? fdtdSamples(h) : 0;
    if (!acc8 || nh == 0 || cap <= 0) return TLM_OK;
    const int m = std::min(nh, cap);
    if (!s.dHuyAcc)
    {
        std::fill(acc8, acc8 + (size_t)m * 8, 0.0f);
        return TLM_OK;
    }
    Guard gd(h->device);
    FD_CU(h, cudaStreamSynchronize(h->stream));
    FD_CU(h, cudaMemcpy(acc8, s.dHuyAcc, (size_t)m * 32, cudaMemcpyDeviceToHost));
    return TLM_OK;
}

tlm_status fdtd_set_field_plane(fdtd_handle h, int axis, int index)
{
    FD_TRY(ready(h));
    if (axis < -1 || axis > 2) return h->fail(TLM_EINVAL, "plane axis must be -1 (off), 0, 1 or 2");
    h->surf.planeAxis = axis;
    h->surf.planeIndex = index;
    return TLM_OK;
}

tlm_status fdtd_get_field_plane(fdtd_handle h, float *out, size_t cap, int *axis, int *index, int *n1, int *n2)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    if (s.planeAxis < 0 || !s.planeValid) return h->fail(TLM_ESTATE, "no field plane has been computed");
    const size_t np = (size_t)s.planeN1 * s.planeN2;
    if (axis) *axis = s.planeAxisDone;
    if (index) *index = s.planeIndexDone;
    if (n1) *n1 = s.planeN1;
    if (n2) *n2 = s.planeN2;
    if (!out) return TLM_OK;
    if (cap < np) return h->fail(TLM_EINVAL, "output holds fewer values than the plane");
    Guard gd(h->device);
    FD_CU(h, cudaStreamSynchronize(h->stream));
    FD_CU(h, cudaMemcpy(out, s.dPlane, np * 4, cudaMemcpyDeviceToHost));
    return TLM_OK;
}

tlm_status fdtd_frame_count(fdtd_handle h, int *n)
{
    FD_TRY(ready(h));
    if (!n) return h->fail(TLM_EINVAL, "null output");
    *n = (int)h->surf.frames.size();
    return TLM_OK;
}

tlm_status fdtd_get_frame(fdtd_handle h, int idx, int *step, float *js, int js_cap, float *plane, size_t plane_cap,
                          int *axis, int *index, int *n1, int *n2)
{
    FD_TRY(ready(h));
    const SurfaceState &s = h->surf;
    if (idx < 0 || idx >= (int)s.frames.size()) return h->fail(TLM_EINVAL, "no such frame");
    const SurfaceState::Frame &fr = s.frames[idx];
    const int nj = (int)s.jsCell.size();
    const size_t np = fr.hasPlane ? (size_t)fr.n1 * fr.n2 : 0;
    if (step) *step = fr.step;
    if (axis) *axis = fr.axis;
    if (index) *index = fr.index;
    if (n1) *n1 = fr.n1;
    if (n2) *n2 = fr.n2;
    Guard gd(h->device);
    FD_CU(h, cudaStreamSynchronize(h->stream));
    const float *base = static_cast<const float *>(s.dFrames) + fr.off;
    if (js && nj && js_cap > 0)
        FD_CU(h, cudaMemcpy(js, base, (size_t)std::min(nj, js_cap) * 4, cudaMemcpyDeviceToHost));
    if (plane && np)
    {
        if (plane_cap < np) return h->fail(TLM_EINVAL, "plane output holds fewer values than the frame's plane");
        FD_CU(h, cudaMemcpy(plane, base + nj, np * 4, cudaMemcpyDeviceToHost));
    }
    return TLM_OK;
}

tlm_status fdtd_compute_far_field(fdtd_handle h, int n_theta, int n_phi, float *U, float *u_max, float *directivity,
                                  float *peak_theta_deg, float *peak_phi_deg)
{
    FD_TRY(ready(h));
    if (n_theta < 2 || n_phi < 2) return h->fail(TLM_EINVAL, "need at least 2 theta and 2 phi samples");
    const SurfaceState &s = h->surf;
    const int nh = (int)s.huyCell.size();
    if (nh == 0 || fdtdSamples(h) == 0 || !s.dHuyAcc)
        return h->fail(TLM_ESTATE, "no Huygens phasors recorded (surface_monitors, huy_offset >= 2, "
                                   "steps past settle_steps)");
    Guard gd(h->device);
    FD_CU(h, cudaStreamSynchronize(h->stream));
    tlmi::FarField out;
    std::string err;
    const tlm_status st = tlmi::farFieldTransform(h->stream, h->pool, false, s.dHuyAcc, s.dHuyNode, s.huyPos.data(),
                                                  nh, h->cfg.f0, n_theta, n_phi, U, out, err);
    if (st != TLM_OK) return h->fail(st, err);
    if (u_max) *u_max = out.uMax;
    if (directivity) *directivity = out.directivity;
    if (peak_theta_deg) *peak_theta_deg = out.peakTheta;
    if (peak_phi_deg) *peak_phi_deg = out.peakPhi;
    return TLM_OK;
}

} // extern "C"
