// tlm_surface.cu -- surface monitors of the TLM step and the far field.
//
// The reference's monitors beyond ports, probes and energy
// (TlmSolver::monitors, TlmSolver.cpp:616-675 and 715-763):
//   * PEC-surface currents: for every face between a PEC cell and a non-PEC
//     neighbour (Geometry.cpp:402-436), the circulations ZI of the two
//     tangential axes at the neighbour (|Js| = sqrt(h1^2 + h2^2) each step,
//     and a running DFT at f0 from settle_steps on);
//   * Huygens-box phasors: on the air cells of a box inset huy_offset cells
//     (TlmSolver.cpp:310-348), running DFTs of -V_t and -ZI_t of the two
//     tangential axes, input of the near-to-far-field transform;
//   * the |E| cut plane (every second step) and playback frames.
// Each runs on the incident pulses after injection of step n. Those are not
// stored (the state between steps is the reflected pulses), so the monitor
// kernel recomputes them for the cells it needs from the same input buffer
// the step kernel of step n reads: the gather of connect, then the soft
// sources of the cell in the reference's order. Every accumulator belongs to
// one thread and is updated in step order in the storage's real type, so
// FP32 results are bitwise the reference's.
//
// The far field (ComputeFarFieldFromHuygens, TlmSolver.cpp:805-916) is one
// block per direction summing the faces' radiation vectors in FP64.
#include "tlm_b200.h"
#include "tlm_internal.h"

#include "tlm_host_math.h"
#include "tlm_step_kernel.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

using namespace tlmi;

namespace tlmk {

template <class S> struct SurfaceArgs
{
    using R = typename Traits<S>::R;
    const S *in;            // state before step n (reflected pulses, or incident if `incident`)
    int incident;
    const uint8_t *mat;
    long long P;
    int nx, ny, nz, px;
    R rho, scale;
    const SpecEntry *spec;  // node-sorted sources and samples
    int nspec;
    R sv;                   // source value of step n
    // PEC-surface faces
    const long long *jsNode;  // face code: padded node * 8 + axis * 2 + (normal sign < 0)
    int njs;
    R *jsInst;              // |Js| per face
    R *jsAcc;               // per face: Re1 Im1 Re2 Im2
    // Huygens faces
    const long long *huyNode;
    int nhuy;
    R *huyAcc;              // per face: E1 re/im, E2 re/im, eta0 H1 re/im, eta0 H2 re/im
    int doDft;
    R cph, sph;
    // cut plane
    int planeAxis, planeIndex, planeN1, planeN2;
    R *plane;
};

// The 12 incident pulses of node `node` (cell i, j, k) at step n: the gather
// of connect (TlmSolver.cpp:551-613) from the reflected pulses of step n-1,
// then the soft sources of the node (TlmSolver.cpp:487-505).
template <class S>
__device__ void incidentAt(const SurfaceArgs<S> &a, long long node, int i, int j, int k,
                           typename Traits<S>::R (&inc)[12])
{
    using R = typename Traits<S>::R;
    const long long stride[3] = { 1, a.px, (long long)a.px * a.ny };
    const int co[3] = { i, j, k };
    const int dims[3] = { a.nx, a.ny, a.nz };
#pragma unroll
    for (int s = 0; s < 12; ++s)
    {
        const R own = loadOne<S>(a.in, s * a.P + node, a.scale);
        if (a.incident)
        {
            inc[s] = own;
            continue;
        }
        const int ax = s >> 2, side = (s >> 1) & 1;
        const int q = co[ax] + (side ? 1 : -1);
        if (q < 0 || q >= dims[ax])
            inc[s] = a.rho * own;
        else
        {
            const long long nb = node + (side ? stride[ax] : -stride[ax]);
            inc[s] = (a.mat[nb] == kPec) ? -own : loadOne<S>(a.in, (s ^ 2) * a.P + nb, a.scale);
        }
    }
    // soft sources of this node, in the order the step kernel applies them
    int lo = 0, hi = a.nspec;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (a.spec[mid].node < node) lo = mid + 1; else hi = mid;
    }
    for (int e = lo; e < a.nspec && a.spec[e].node == node; ++e)
    {
        const SpecEntry se = a.spec[e];
        if (se.kind != kInject) continue;
        const R qv = (R(0.5) * R(se.amp)) * a.sv;
#pragma unroll
        for (int s = 0; s < 12; ++s)
            if ((s >> 2) != se.arg && fieldOfSlot(s) == se.arg) inc[s] = inc[s] + qv;
    }
}

__device__ __forceinline__ void cellOfNode(long long node, int px, int ny, int *i, int *j, int *k)
{
    const long long r = node / px;
    *i = (int)(node - r * px);
    *j = (int)(r % ny);
    *k = (int)(r / ny);
}

template <class S> __global__ void __launch_bounds__(256) surfaceMonitorKernel(const SurfaceArgs<S> a)
{
    using R = typename Traits<S>::R;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = a.doDft ? a.nhuy : 0;
    const long long nplane = a.planeAxis >= 0 ? (long long)a.planeN1 * a.planeN2 : 0;
    R inc[12];
    if (t < a.njs)
    {
        // TlmSolver.cpp:632-646
        const long long code = a.jsNode[t];
        const long long node = code >> 3;
        const int ax = (int)((code >> 1) & 3);
        int i, j, k;
        cellOfNode(node, a.px, a.ny, &i, &j, &k);
        incidentAt<S>(a, node, i, j, k, inc);
        const R h1 = circulation(inc, ax == 0 ? 1 : 0), h2 = circulation(inc, ax == 2 ? 1 : 2);
        a.jsInst[t] = sqrt(h1 * h1 + h2 * h2);
        if (a.doDft)
        {
            R *acc = a.jsAcc + t * 4;
            acc[0] = acc[0] + h1 * a.cph;
            acc[1] = acc[1] - h1 * a.sph;
            acc[2] = acc[2] + h2 * a.cph;
            acc[3] = acc[3] - h2 * a.sph;
        }
        return;
    }
    long long u = t - a.njs;
    if (u < nh)
    {
        // TlmSolver.cpp:660-671: E_t ~ -V_t, eta0 H_t ~ -ZI_t
        const long long code = a.huyNode[u];
        const long long node = code >> 3;
        const int ax = (int)((code >> 1) & 3);
        int i, j, k;
        cellOfNode(node, a.px, a.ny, &i, &j, &k);
        incidentAt<S>(a, node, i, j, k, inc);
        const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
        const R e1 = -nodeVoltage(inc, t1), e2 = -nodeVoltage(inc, t2);
        const R m1 = -circulation(inc, t1), m2 = -circulation(inc, t2);
        R *acc = a.huyAcc + u * 8;
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
    u -= nh;
    if (u < nplane)
    {
        // TlmSolver.cpp:716-743: |E| = sqrt(V_x^2 + V_y^2 + V_z^2), 0 on PEC
        const int q1 = (int)(u % a.planeN1), q2 = (int)(u / a.planeN1);
        const int pa = a.planeAxis;
        const int a1 = pa == 0 ? 1 : 0, a2 = pa == 2 ? 1 : 2;
        int co[3];
        co[pa] = a.planeIndex;
        co[a1] = q1;
        co[a2] = q2;
        const long long node = ((long long)co[2] * a.ny + co[1]) * a.px + co[0];
        R v = R(0);
        if (a.mat[node] != kPec)
        {
            incidentAt<S>(a, node, co[0], co[1], co[2], inc);
            R e2 = R(0);
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
            {
                const R vj = nodeVoltage(inc, jj);
                e2 = e2 + vj * vj;
            }
            v = sqrt(e2);
        }
        a.plane[u] = v;
    }
}

// Far field: block d = direction (theta index d / nPhi, phi index d % nPhi).
// Per face the equivalent currents J' = n x (eta0 H), M = -(n x E) in world
// components (TlmSolver.cpp:829-848), projected on theta/phi and summed with
// e^{+j k0 r.pos} into N and L (TlmSolver.cpp:860-890); sums in FP64 with a
// fixed-order block reduction. U = |L_phi + N_theta|^2 + |L_theta - N_phi|^2.
template <class R>
__global__ void __launch_bounds__(256)
    farFieldKernel(const R *__restrict__ acc, const long long *__restrict__ code, const float *__restrict__ pos,
                   int nh, R k0, int nTheta, int nPhi, R *__restrict__ U)
{
    __shared__ double red[8][8];
    const int d = blockIdx.x;
    const int ti = d / nPhi, pj = d % nPhi;
    const R pi = R(3.14159265358979323846);
    const R th = pi * R(ti) / R(nTheta - 1);
    const R ph = R(2) * pi * R(pj) / R(nPhi - 1);
    const R st = sin(th), ct = cos(th), cp = cos(ph), sp = sin(ph);
    const R rh[3] = { st * cp, st * sp, ct };
    const R tv[3] = { ct * cp, ct * sp, -st };
    const R pv[2] = { -sp, cp };
    double s[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };  // Nt, Np, Lt, Lp (re, im)
    for (int f = threadIdx.x; f < nh; f += blockDim.x)
    {
        const R *a = acc + (long long)f * 8;
        const int ax = (int)((code[f] >> 1) & 3);
        const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
        const R sa = ax == 1 ? R(-1) : R(1);
        const R sg = (code[f] & 1) ? R(-1) : R(1);  // outward normal sign
        R jR[3] = { 0, 0, 0 }, jI[3] = { 0, 0, 0 }, mR[3] = { 0, 0, 0 }, mI[3] = { 0, 0, 0 };
        jR[t2] = sg * sa * a[4];
        jI[t2] = sg * sa * a[5];
        jR[t1] = -sg * sa * a[6];
        jI[t1] = -sg * sa * a[7];
        mR[t2] = -sg * sa * a[0];
        mI[t2] = -sg * sa * a[1];
        mR[t1] = sg * sa * a[2];
        mI[t1] = sg * sa * a[3];
        const R px = R(pos[3 * f]), py = R(pos[3 * f + 1]), pz = R(pos[3 * f + 2]);
        const R pha = k0 * (rh[0] * px + rh[1] * py + rh[2] * pz);
        const double c = (double)cos(pha), sn = (double)sin(pha);
        const double jt[2] = { (double)(jR[0] * tv[0] + jR[1] * tv[1] + jR[2] * tv[2]),
                               (double)(jI[0] * tv[0] + jI[1] * tv[1] + jI[2] * tv[2]) };
        const double jp[2] = { (double)(jR[0] * pv[0] + jR[1] * pv[1]), (double)(jI[0] * pv[0] + jI[1] * pv[1]) };
        const double mt[2] = { (double)(mR[0] * tv[0] + mR[1] * tv[1] + mR[2] * tv[2]),
                               (double)(mI[0] * tv[0] + mI[1] * tv[1] + mI[2] * tv[2]) };
        const double mp[2] = { (double)(mR[0] * pv[0] + mR[1] * pv[1]), (double)(mI[0] * pv[0] + mI[1] * pv[1]) };
        s[0] += jt[0] * c - jt[1] * sn;
        s[1] += jt[0] * sn + jt[1] * c;
        s[2] += jp[0] * c - jp[1] * sn;
        s[3] += jp[0] * sn + jp[1] * c;
        s[4] += mt[0] * c - mt[1] * sn;
        s[5] += mt[0] * sn + mt[1] * c;
        s[6] += mp[0] * c - mp[1] * sn;
        s[7] += mp[0] * sn + mp[1] * c;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
        for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
    {
#pragma unroll
        for (int q = 0; q < 8; ++q) red[warp][q] = s[q];
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            for (int q = 0; q < 8; ++q) t[q] += red[w][q];
        const double aR = t[6] + t[0], aI = t[7] + t[1];
        const double bR = t[4] - t[2], bI = t[5] - t[3];
        U[d] = (R)(aR * aR + aI * aI + bR * bR + bI * bI);
    }
}

} // namespace tlmk

namespace tlmi {

namespace {

size_t realSize(const tlm_solver *h) { return realBytes(h->storage); }

} // namespace

// Face lists in the reference's order: PEC faces by the scan of
// BuildPecSurfaceFaces (Geometry.cpp:402-436; cell, then axis, then side -1
// before +1), Huygens faces by TlmSolver::buildHuygens (TlmSolver.cpp:310-348;
// x faces over (k, j), y faces over (k, i), z faces over (j, i), low first).
void buildFaceLists(int nx, int ny, int nz, const float origin[3], float dl, const uint8_t *mat, bool surfaceOn,
                    int huyOffset, SurfaceState &s)
{
    s.jsCell.clear();
    s.jsAxis.clear();
    s.jsSign.clear();
    s.jsCenter.clear();
    s.huyCell.clear();
    s.huyAxis.clear();
    s.huySign.clear();
    s.huyPos.clear();
    if (!surfaceOn) return;
    auto center = [&](int i, int j, int k, float c[3]) {
        // origin + (i + 0.5) dl per axis, in float (Geometry.h:100-105)
        c[0] = origin[0] + ((float)i + 0.5f) * dl;
        c[1] = origin[1] + ((float)j + 0.5f) * dl;
        c[2] = origin[2] + ((float)k + 0.5f) * dl;
    };
    const long long stride[3] = { 1, nx, (long long)nx * ny };
    const int dims[3] = { nx, ny, nz };
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
            {
                const size_t c = ((size_t)k * ny + j) * nx + i;
                if (mat[c] != tlmk::kPec) continue;
                const int co[3] = { i, j, k };
                for (int a = 0; a < 3; ++a)
                    for (int sd = -1; sd <= 1; sd += 2)
                    {
                        const int q = co[a] + sd;
                        if (q < 0 || q >= dims[a]) continue;
                        const size_t nb = c + (size_t)((long long)sd * stride[a]);
                        if (mat[nb] == tlmk::kPec) continue;
                        float cc[3];
                        center(i, j, k, cc);
                        cc[a] = cc[a] + (float)sd * dl * 0.5f;
                        s.jsCell.push_back(nb);
                        s.jsAxis.push_back(a);
                        s.jsSign.push_back(sd);
                        s.jsCenter.insert(s.jsCenter.end(), cc, cc + 3);
                    }
            }
    const int o = huyOffset;
    if (o < 2 || 2 * o + 2 >= nx || 2 * o + 2 >= ny || 2 * o + 2 >= nz) return;
    const float half[3] = { ((float)nx * dl) * 0.5f, ((float)ny * dl) * 0.5f, ((float)nz * dl) * 0.5f };
    float dom[3];
    for (int a = 0; a < 3; ++a) dom[a] = origin[a] + half[a];
    auto add = [&](int i, int j, int k, int axis, int outSign) {
        const size_t c = ((size_t)k * ny + j) * nx + i;
        if (mat[c] != tlmk::kAir) return;
        float cc[3];
        center(i, j, k, cc);
        s.huyCell.push_back(c);
        s.huyAxis.push_back(axis);
        s.huySign.push_back(outSign);
        for (int a = 0; a < 3; ++a) s.huyPos.push_back(cc[a] - dom[a]);
    };
    const int x0 = o, x1 = nx - 1 - o, y0 = o, y1 = ny - 1 - o, z0 = o, z1 = nz - 1 - o;
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
}

void buildSurfaceLists(tlm_solver *h)
{
    buildFaceLists(h->nx, h->ny, h->nz, h->g.origin, h->g.dl, h->mat.data(), h->cfg.surface_monitors != 0,
                   h->cfg.huy_offset, h->surf);
}

bool surfaceActive(const tlm_solver *h)
{
    const SurfaceState &s = h->surf;
    return !s.jsCell.empty() || !s.huyCell.empty() || s.planeAxis >= 0 || h->cfg.record_every > 0;
}

void freeSurface(tlm_solver *h)
{
    SurfaceState &s = h->surf;
    devFree(h, s.dJsNode);
    devFree(h, s.dHuyNode);
    devFree(h, s.dJsInst);
    devFree(h, s.dJsAcc);
    devFree(h, s.dHuyAcc);
    devFree(h, s.dPlane);
    devFree(h, s.dFrames);
    s.planeCap = 0;
    s.planeValid = false;
    s.framesCap = s.framesUsed = 0;
    s.frames.clear();
}

// Upload the face lists and zero the accumulators (before the first step).
tlm_status prepareSurface(tlm_solver *h)
{
    SurfaceState &s = h->surf;
    const size_t r = realSize(h);
    auto upload = [&](long long **dst, const std::vector<uint64_t> &cells, const std::vector<int> &axis,
                      const std::vector<int> *sign) -> tlm_status {
        if (cells.empty()) return TLM_OK;
        std::vector<long long> code(cells.size());
        for (size_t f = 0; f < cells.size(); ++f)
            code[f] = paddedNode(h, cells[f]) * 8 + axis[f] * 2 + ((sign && (*sign)[f] < 0) ? 1 : 0);
        TLM_TRY(devAlloc(h, dst, code.size() * sizeof(long long)));
        TLM_CU(h, cudaMemcpyAsync(*dst, code.data(), code.size() * sizeof(long long), cudaMemcpyHostToDevice,
                                  h->stream));
        TLM_CU(h, cudaStreamSynchronize(h->stream));
        return TLM_OK;
    };
    TLM_TRY(upload(&s.dJsNode, s.jsCell, s.jsAxis, nullptr));
    TLM_TRY(upload(&s.dHuyNode, s.huyCell, s.huyAxis, &s.huySign));
    const size_t nj = s.jsCell.size(), nh = s.huyCell.size();
    if (nj)
    {
        TLM_TRY(devAlloc(h, &s.dJsInst, nj * r));
        TLM_TRY(devAlloc(h, &s.dJsAcc, nj * 4 * r));
    }
    if (nh) TLM_TRY(devAlloc(h, &s.dHuyAcc, nh * 8 * r));
    return rewindSurface(h);
}

tlm_status rewindSurface(tlm_solver *h)
{
    SurfaceState &s = h->surf;
    const size_t r = realSize(h);
    const size_t nj = s.jsCell.size(), nh = s.huyCell.size();
    if (s.dJsInst) TLM_CU(h, cudaMemsetAsync(s.dJsInst, 0, nj * r, h->stream));
    if (s.dJsAcc) TLM_CU(h, cudaMemsetAsync(s.dJsAcc, 0, nj * 4 * r, h->stream));
    if (s.dHuyAcc) TLM_CU(h, cudaMemsetAsync(s.dHuyAcc, 0, nh * 8 * r, h->stream));
    s.planeValid = false;
    s.frames.clear();
    s.framesUsed = 0;
    return TLM_OK;
}

namespace {

template <class S> tlm_status launchSurfaceT(tlm_solver *h, int n)
{
    using R = typename tlmk::Traits<S>::R;
    SurfaceState &s = h->surf;
    const int nj = (int)s.jsCell.size(), nh = (int)s.huyCell.size();
    const bool doDft = n >= h->cfg.settle_steps;
    const bool doPlane = s.planeAxis >= 0 && (n % 2) == 0;
    int n1 = 0, n2 = 0;
    if (doPlane)
    {
        const int dims[3] = { h->nx, h->ny, h->nz };
        n1 = dims[s.planeAxis == 0 ? 1 : 0];
        n2 = dims[s.planeAxis == 2 ? 1 : 2];
        const size_t need = (size_t)n1 * n2;
        if (need > s.planeCap)
        {
            devFree(h, s.dPlane);
            TLM_TRY(devAlloc(h, &s.dPlane, need * sizeof(R)));
            s.planeCap = need;
        }
    }
    const long long items = (long long)nj + (doDft ? nh : 0) + (doPlane ? (long long)n1 * n2 : 0);
    if (items > 0)
    {
        tlmk::SurfaceArgs<S> a;
        a.in = static_cast<const S *>(h->dPulses[h->curBuf]);
        a.incident = h->stateIncident ? 1 : 0;
        a.mat = h->dMat;
        a.P = h->P;
        a.nx = h->nx;
        a.ny = h->ny;
        a.nz = h->nz;
        a.px = h->px;
        a.rho = (R)h->cfg.boundary_rho;
        a.scale = (R)h->scale;
        a.spec = h->dSpec;
        a.nspec = h->dSpec ? h->specCount : 0;
        a.sv = (R)sourceValue(h, n);
        a.jsNode = s.dJsNode;
        a.njs = nj;
        a.jsInst = static_cast<R *>(s.dJsInst);
        a.jsAcc = static_cast<R *>(s.dJsAcc);
        a.huyNode = s.dHuyNode;
        a.nhuy = nh;
        a.huyAcc = static_cast<R *>(s.dHuyAcc);
        a.doDft = doDft ? 1 : 0;
        a.cph = a.sph = R(0);
        if ((nj || nh) && doDft)
        {
            // the DFT phase of step n, computed on the host like the reference
            if (h->storage == TLM_STORE_F64)
            {
                double c, sn;
                tlmh::dft_phase_f64(h->cfg.f0, h->dt64, n, &c, &sn);
                a.cph = (R)c;
                a.sph = (R)sn;
            }
            else
            {
                float c, sn;
                tlmh::dft_phase_f32(h->cfg.f0, h->dt32, n, &c, &sn);
                a.cph = (R)c;
                a.sph = (R)sn;
            }
        }
        a.planeAxis = doPlane ? s.planeAxis : -1;
        a.planeIndex = doPlane ? std::min(std::max(s.planeIndex, 0), (s.planeAxis == 0 ? h->nx : s.planeAxis == 1 ? h->ny : h->nz) - 1) : 0;
        a.planeN1 = n1;
        a.planeN2 = n2;
        a.plane = static_cast<R *>(s.dPlane);
        const long long blocks = (items + 255) / 256;
        tlmk::surfaceMonitorKernel<S><<<(unsigned)blocks, 256, 0, h->stream>>>(a);
        TLM_CU(h, cudaGetLastError());
        if (doPlane)
        {
            s.planeValid = true;
            s.planeAxisDone = s.planeAxis;
            s.planeIndexDone = a.planeIndex;
            s.planeN1 = n1;
            s.planeN2 = n2;
        }
    }
    // playback frame (TlmSolver.cpp:746-762): |Js| and the latest cut plane
    if (h->cfg.record_every > 0 && (n % h->cfg.record_every) == 0)
    {
        const bool withPlane = s.planeAxis >= 0 && s.planeValid;
        const size_t np = withPlane ? (size_t)s.planeN1 * s.planeN2 : 0;
        const size_t need = s.framesUsed + nj + np;
        if (need > s.framesCap)
        {
            const size_t cap = std::max(need, s.framesCap * 2 + 1024);
            void *d = nullptr;
            TLM_TRY(devAlloc(h, &d, cap * sizeof(R)));
            if (s.framesUsed)
                TLM_CU(h, cudaMemcpyAsync(d, s.dFrames, s.framesUsed * sizeof(R), cudaMemcpyDeviceToDevice,
                                          h->stream));
            devFree(h, s.dFrames);
            s.dFrames = d;
            s.framesCap = cap;
        }
        R *base = static_cast<R *>(s.dFrames) + s.framesUsed;
        if (nj) TLM_CU(h, cudaMemcpyAsync(base, s.dJsInst, nj * sizeof(R), cudaMemcpyDeviceToDevice, h->stream));
        if (np) TLM_CU(h, cudaMemcpyAsync(base + nj, s.dPlane, np * sizeof(R), cudaMemcpyDeviceToDevice, h->stream));
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
    return TLM_OK;
}

} // namespace

tlm_status launchSurface(tlm_solver *h, int n)
{
    switch (h->storage)
    {
    case TLM_STORE_F64: return launchSurfaceT<double>(h, n);
    case TLM_STORE_BF16: return launchSurfaceT<__nv_bfloat16>(h, n);
    case TLM_STORE_F16: return launchSurfaceT<__half>(h, n);
    case TLM_STORE_BFP16: return launchSurfaceT<tlmk::Bfp4>(h, n);
    default: return launchSurfaceT<float>(h, n);
    }
}

} // namespace tlmi

namespace tlmi {

// Near-to-far-field transform of the Huygens phasors on the device (one block
// per direction, FP64 sums), then the reference's directivity and peak
// search on the host (TlmSolver.cpp:893-915). `f64`: the phasors are double.
tlm_status farFieldTransform(cudaStream_t stream, cudaMemPool_t pool, bool f64, const void *dAcc,
                             const long long *dCode, const float *hostPos, int nh, float f0, int n_theta,
                             int n_phi, float *U, FarField &out, std::string &err)
{
    const int nd = n_theta * n_phi;
    float *dPos = nullptr;
    void *dU = nullptr;
    const size_t r = f64 ? 8 : 4;
    cudaError_t e = cudaMallocFromPoolAsync((void **)&dPos, (size_t)nh * 3 * sizeof(float), pool, stream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&dU, (size_t)nd * r, pool, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dPos, hostPos, (size_t)nh * 3 * sizeof(float), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
    {
        if (f64)
        {
            const double k0 = 2.0 * 3.14159265358979323846 * (double)f0 / (double)299792458.0f;
            tlmk::farFieldKernel<double><<<nd, 256, 0, stream>>>(static_cast<const double *>(dAcc), dCode, dPos,
                                                                 nh, k0, n_theta, n_phi,
                                                                 static_cast<double *>(dU));
        }
        else
        {
            const float k0 = 2.0f * (float)3.14159265358979323846 * f0 / 299792458.0f;
            tlmk::farFieldKernel<float><<<nd, 256, 0, stream>>>(static_cast<const float *>(dAcc), dCode, dPos, nh,
                                                                k0, n_theta, n_phi, static_cast<float *>(dU));
        }
        e = cudaGetLastError();
    }
    std::vector<float> u(nd);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess)
    {
        if (f64)
        {
            std::vector<double> t(nd);
            e = cudaMemcpy(t.data(), dU, (size_t)nd * 8, cudaMemcpyDeviceToHost);
            for (int i = 0; i < nd; ++i) u[i] = (float)t[i];
        }
        else
            e = cudaMemcpy(u.data(), dU, (size_t)nd * 4, cudaMemcpyDeviceToHost);
    }
    if (dPos) cudaFreeAsync(dPos, stream);
    if (dU) cudaFreeAsync(dU, stream);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        err = std::string("far-field transform: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? TLM_ENOMEM : TLM_ECUDA;
    }
    const float pi = (float)3.14159265358979323846;
    float um = 0.0f;
    int iMax = 0;
    double prad = 0.0;
    const float dTh = pi / (float)(n_theta - 1);
    const float dPh = 2.0f * pi / (float)(n_phi - 1);
    for (int ti = 0; ti < n_theta; ++ti)
    {
        const float th = pi * (float)ti / (float)(n_theta - 1);
        const float wTh = (ti == 0 || ti == n_theta - 1) ? 0.5f : 1.0f;
        for (int pj = 0; pj < n_phi; ++pj)
        {
            const float wPh = (pj == 0 || pj == n_phi - 1) ? 0.5f : 1.0f;
            const float v = u[(size_t)ti * n_phi + pj];
            if (v > um)
            {
                um = v;
                iMax = ti * n_phi + pj;
            }
            prad += (double)v * std::sin(th) * wTh * wPh * dTh * dPh;
        }
    }
    if (U) std::copy(u.begin(), u.end(), U);
    out.uMax = um;
    out.directivity = prad > 0 ? (float)(4.0 * 3.14159265358979323846 * um / prad) : 0.0f;
    out.peakTheta = 180.0f * (float)(iMax / n_phi) / (float)(n_theta - 1);
    out.peakPhi = 360.0f * (float)(iMax % n_phi) / (float)(n_phi - 1);
    return TLM_OK;
}

} // namespace tlmi

namespace {

// Device buffer of the storage's real type -> host floats.
tlm_status realsToHost(tlm_solver *h, const void *d, size_t count, float *out)
{
    if (!count) return TLM_OK;
    if (h->storage == TLM_STORE_F64)
    {
        std::vector<double> t(count);
        TLM_CU(h, cudaMemcpy(t.data(), d, count * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < count; ++i) out[i] = (float)t[i];
    }
    else
        TLM_CU(h, cudaMemcpy(out, d, count * 4, cudaMemcpyDeviceToHost));
    return TLM_OK;
}

int samplesOf(const tlm_solver *h)
{
    const int settle = std::max(h->cfg.settle_steps, 0);
    return std::max(0, h->curStep - settle);
}

} // namespace

extern "C" {

tlm_status tlm_get_surface_faces(tlm_handle h, uint64_t *air_cells, int *axis, int *sign, float *centers,
                                 int cap, int *n_out)
{
    TLM_TRY(checkReady(h));
    const SurfaceState &s = h->surf;
    const int n = (int)s.jsCell.size();
    if (n_out) *n_out = n;
    for (int f = 0; f < n && f < cap; ++f)
    {
        if (air_cells) air_cells[f] = s.jsCell[f];
        if (axis) axis[f] = s.jsAxis[f];
        if (sign) sign[f] = s.jsSign[f];
        if (centers) std::memcpy(centers + 3 * f, &s.jsCenter[3 * f], 3 * sizeof(float));
    }
    return TLM_OK;
}

tlm_status tlm_get_js_instant(tlm_handle h, float *out, int cap, int *n_out)
{
    TLM_TRY(checkReady(h));
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    const SurfaceState &s = h->surf;
    const int n = (int)s.jsCell.size();
    if (n_out) *n_out = n;
    if (!out || cap <= 0 || n == 0) return TLM_OK;
    if (!s.dJsInst)
    {
        std::fill(out, out + std::min(n, cap), 0.0f);
        return TLM_OK;
    }
    std::vector<float> t(n);
    TLM_TRY(realsToHost(h, s.dJsInst, n, t.data()));
    std::copy(t.begin(), t.begin() + std::min(n, cap), out);
    return TLM_OK;
}

tlm_status tlm_get_js_dft(tlm_handle h, float *magnitude, float *re, float *im, int cap, int *n_out,
                          int *samples)
{
    TLM_TRY(checkReady(h));
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    const SurfaceState &s = h->surf;
    const int n = (int)s.jsCell.size();
    const int ns = s.jsCell.empty() ? 0 : samplesOf(h);
    if (n_out) *n_out = n;
    if (samples) *samples = ns;
    if (n == 0 || cap <= 0) return TLM_OK;
    std::vector<float> acc((size_t)n * 4, 0.0f);
    if (s.dJsAcc) TLM_TRY(realsToHost(h, s.dJsAcc, (size_t)n * 4, acc.data()));
    for (int f = 0; f < n && f < cap; ++f)
    {
        const float r1 = acc[4 * f], i1 = acc[4 * f + 1], r2 = acc[4 * f + 2], i2 = acc[4 * f + 3];
        if (re)
        {
            re[2 * f] = r1;
            re[2 * f + 1] = r2;
        }
        if (im)
        {
            im[2 * f] = i1;
            im[2 * f + 1] = i2;
        }
        if (magnitude)
        {
            // finalizeDft (TlmSolver.cpp:467-481)
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

tlm_status tlm_get_huygens_faces(tlm_handle h, uint64_t *cells, int *axis, int *out_sign, float *pos, int cap,
                                 int *n_out)
{
    TLM_TRY(checkReady(h));
    const SurfaceState &s = h->surf;
    const int n = (int)s.huyCell.size();
    if (n_out) *n_out = n;
    for (int f = 0; f < n && f < cap; ++f)
    {
        if (cells) cells[f] = s.huyCell[f];
        if (axis) axis[f] = s.huyAxis[f];
        if (out_sign) out_sign[f] = s.huySign[f];
        if (pos) std::memcpy(pos + 3 * f, &s.huyPos[3 * f], 3 * sizeof(float));
    }
    return TLM_OK;
}

tlm_status tlm_get_huygens_dft(tlm_handle h, float *acc8, int cap, int *n_out, int *samples)
{
    TLM_TRY(checkReady(h));
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    const SurfaceState &s = h->surf;
    const int n = (int)s.huyCell.size();
    if (n_out) *n_out = n;
    if (samples) *samples = n ? samplesOf(h) : 0;
    if (!acc8 || n == 0 || cap <= 0) return TLM_OK;
    const int m = std::min(n, cap);
    if (!s.dHuyAcc)
    {
        std::fill(acc8, acc8 + (size_t)m * 8, 0.0f);
        return TLM_OK;
    }
    return realsToHost(h, s.dHuyAcc, (size_t)m * 8, acc8);
}

tlm_status tlm_set_field_plane(tlm_handle h, int axis, int index)
{
    TLM_TRY(checkReady(h));
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch");
    if (axis < -1 || axis > 2) return h->fail(TLM_EINVAL, "plane axis must be -1 (off), 0, 1 or 2");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    h->surf.planeAxis = axis;
    h->surf.planeIndex = index;
    return TLM_OK;
}

tlm_status tlm_get_field_plane(tlm_handle h, float *out, size_t cap, int *axis, int *index, int *n1, int *n2)
{
    TLM_TRY(checkReady(h));
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    const SurfaceState &s = h->surf;
    if (s.planeAxis < 0 || !s.planeValid) return h->fail(TLM_ESTATE, "no field plane has been computed");
    const size_t n = (size_t)s.planeN1 * s.planeN2;
    if (axis) *axis = s.planeAxisDone;
    if (index) *index = s.planeIndexDone;
    if (n1) *n1 = s.planeN1;
    if (n2) *n2 = s.planeN2;
    if (!out) return TLM_OK;
    if (cap < n) return h->fail(TLM_EINVAL, "output holds fewer values than the plane");
    return realsToHost(h, s.dPlane, n, out);
}

tlm_status tlm_frame_count(tlm_handle h, int *n)
{
    TLM_TRY(checkReady(h));
    if (!n) return h->fail(TLM_EINVAL, "null output");
    *n = (int)h->surf.frames.size();
    return TLM_OK;
}

tlm_status tlm_get_frame(tlm_handle h, int idx, int *step, float *js, int js_cap, float *plane, size_t plane_cap,
                         int *axis, int *index, int *n1, int *n2)
{
    TLM_TRY(checkReady(h));
    const SurfaceState &s = h->surf;
    if (idx < 0 || idx >= (int)s.frames.size()) return h->fail(TLM_EINVAL, "no such frame");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    const SurfaceState::Frame &fr = s.frames[idx];
    const int nj = (int)s.jsCell.size();
    const size_t np = fr.hasPlane ? (size_t)fr.n1 * fr.n2 : 0;
    if (step) *step = fr.step;
    if (axis) *axis = fr.axis;
    if (index) *index = fr.index;
    if (n1) *n1 = fr.n1;
    if (n2) *n2 = fr.n2;
    const size_t r = realBytes(h->storage);
    const char *base = static_cast<const char *>(s.dFrames) + fr.off * r;
    if (js && nj)
    {
        std::vector<float> t(nj);
        TLM_TRY(realsToHost(h, base, nj, t.data()));
        std::copy(t.begin(), t.begin() + std::min(nj, std::max(js_cap, 0)), js);
    }
    if (plane && np)
    {
        if (plane_cap < np) return h->fail(TLM_EINVAL, "plane output holds fewer values than the frame's plane");
        TLM_TRY(realsToHost(h, base + (size_t)nj * r, np, plane));
    }
    return TLM_OK;
}

tlm_status tlm_compute_far_field(tlm_handle h, int n_theta, int n_phi, float *U, float *u_max,
                                 float *directivity, float *peak_theta_deg, float *peak_phi_deg)
{
    TLM_TRY(checkReady(h));
    if (n_theta < 2 || n_phi < 2) return h->fail(TLM_EINVAL, "need at least 2 theta and 2 phi samples");
    const SurfaceState &s = h->surf;
    const int nh = (int)s.huyCell.size();
    if (nh == 0 || samplesOf(h) == 0 || !s.dHuyAcc)
        return h->fail(TLM_ESTATE, "no Huygens phasors recorded (surface_monitors, huy_offset >= 2, "
                                   "steps past settle_steps)");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    FarField out;
    std::string err;
    const tlm_status st = farFieldTransform(h->stream, h->pool, h->storage == TLM_STORE_F64, s.dHuyAcc,
                                            s.dHuyNode, s.huyPos.data(), nh, h->cfg.f0, n_theta, n_phi, U,
                                            out, err);
    if (st != TLM_OK) return h->fail(st, err);
    if (u_max) *u_max = out.uMax;
    if (directivity) *directivity = out.directivity;
    if (peak_theta_deg) *peak_theta_deg = out.peakTheta;
    if (peak_phi_deg) *peak_phi_deg = out.peakPhi;
    return TLM_OK;
}

} // extern "C"
