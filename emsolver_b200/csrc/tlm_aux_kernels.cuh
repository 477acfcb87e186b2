// tlm_aux_kernels.cuh -- small kernels around the step kernel:
//  * windowEpilogue: once per launch window, turns the per-step monitor
//    samples into the reference's port V/I and probe E records, advances the
//    FP64 running DFT of every port, and reduces the block energy partials
//    in a fixed order (deterministic) into the energy history;
//  * incidentToAos / aosToIncident / stubsToAos: state import and export in
//    the reference's AoS layout (cell*12 + slot, cell*3 + j);
//  * unitarityKernel: the reference's scatter known-answer tests evaluated
//    with the device scatter functions.
#pragma once

#include "tlm_step_kernel.cuh"

namespace tlmk {

template <class R> struct EpilogueArgs
{
    const R *samples;       // [w][nsamp][6]: V_x V_y V_z ZI_x ZI_y ZI_z
    int nsamp;
    int w;                  // steps in this window
    long long base;         // absolute index of the window's first step
    int nports;
    const int *port_off;    // [nports+1] into port_slots
    const int *port_slots;  // sample slot of each kept gap cell, in order
    const int *port_pol;    // E axis of each port
    const int *port_nb;     // [nports][4] sample slots of the current loop
    int nprobes;
    const int *probe_slot;
    R probe_scale;          // -1/dl
    R eta0;
    double *vrec, *irec;    // [step][nports]
    double *prec;           // [step][nprobes][3]
    int nfreq;
    const double *wdt;      // 2*pi*f*dt per DFT frequency
    double *dft;            // [nports][nfreq][4]: Vre Vim Ire Iim
    const double *epart;    // [n_e][nblocks]
    int nblocks;
    int n_e;                // energy steps in this window
    long long e_first;      // absolute index of the first energy step
    double *ehist;          // [step/16]
    double *elatest;        // last energy value (polled by the host)
};

// Body of the window epilogue for one grid; run by one block (any size up to
// 512 threads); `red` holds blockDim.x/32 doubles of shared memory.
template <class R> __device__ __forceinline__ void epilogueBody(const EpilogueArgs<R> &a, double *red)
{
    const int nent = a.nports + a.nprobes;
    const long long total = (long long)a.w * nent;
    // 1. records (TlmSolver.cpp:677-713), float arithmetic in the
    //    reference's order: V = sum of V_pol over the gap cells;
    //    I = (-2 * zi) / eta0, zi = ZI_t2(+t1) - ZI_t2(-t1) - ZI_t1(+t2) + ZI_t1(-t2).
    for (long long idx = threadIdx.x; idx < total; idx += blockDim.x)
    {
        const int i = (int)(idx / nent), e = (int)(idx % nent);
        const long long n = a.base + i;
        const R *smp = a.samples + (long long)i * a.nsamp * 6;
        if (e < a.nports)
        {
            const int p = e, pol = a.port_pol[p];
            R vSum = R(0);
            for (int c = a.port_off[p]; c < a.port_off[p + 1]; ++c)
                vSum = vSum + smp[a.port_slots[c] * 6 + pol];
            R cur = R(0);
            const int *nb = a.port_nb + p * 4;
            if (nb[0] >= 0)
            {
                const int t1 = (pol + 1) % 3, t2 = (pol + 2) % 3;
                R zi = R(0);
                zi = zi + smp[nb[0] * 6 + 3 + t2];
                zi = zi - smp[nb[1] * 6 + 3 + t2];
                zi = zi - smp[nb[2] * 6 + 3 + t1];
                zi = zi + smp[nb[3] * 6 + 3 + t1];
                cur = (R(-2) * zi) / a.eta0;
            }
            a.vrec[n * a.nports + p] = (double)vSum;
            a.irec[n * a.nports + p] = (double)cur;
        }
        else
        {
            const int pr = e - a.nports;
            const R *s = smp + a.probe_slot[pr] * 6;
            double *d = a.prec + (n * a.nprobes + pr) * 3;
            d[0] = (double)(a.probe_scale * s[0]);
            d[1] = (double)(a.probe_scale * s[1]);
            d[2] = (double)(a.probe_scale * s[2]);
        }
    }
    __syncthreads();
    // 2. FP64 running DFT: X(f) += x[n] exp(-j w n). The phasor is a
    //    function of the absolute step alone -- seeded exactly with sincos at
    //    every multiple of 64 and rotated by exp(-j w) in between -- so the
    //    result does not depend on how the steps were split into windows.
    for (int idx = threadIdx.x; idx < a.nports * a.nfreq; idx += blockDim.x)
    {
        const int p = idx / a.nfreq, f = idx % a.nfreq;
        const double w = a.wdt[f];
        double c, s, cw, sw;
        sincos(w, &sw, &cw);
        const long long n0 = a.base / 64 * 64;
        sincos(w * (double)n0, &s, &c);
        for (long long n = n0; n < a.base; ++n)
        {
            const double c2 = c * cw - s * sw;
            s = s * cw + c * sw;
            c = c2;
        }
        double *acc = a.dft + ((long long)p * a.nfreq + f) * 4;
        double vr = acc[0], vi = acc[1], ir = acc[2], ii = acc[3];
        for (int i = 0; i < a.w; ++i)
        {
            const long long n = a.base + i;
            if (n % 64 == 0) sincos(w * (double)n, &s, &c);
            const double v = a.vrec[n * a.nports + p], cu = a.irec[n * a.nports + p];
            vr += v * c;
            vi -= v * s;
            ir += cu * c;
            ii -= cu * s;
            const double c2 = c * cw - s * sw;
            s = s * cw + c * sw;
            c = c2;
        }
        acc[0] = vr;
        acc[1] = vi;
        acc[2] = ir;
        acc[3] = ii;
    }
    // 3. energy history (TlmSolver.cpp:766-789), fixed-order FP64 reduction.
    for (int e = 0; e < a.n_e; ++e)
    {
        double s = 0.0;
        for (int b = threadIdx.x; b < a.nblocks; b += blockDim.x)
            s += a.epart[(long long)e * a.nblocks + b];
        const double tot = blockSumDouble(s, red);
        if (threadIdx.x == 0)
        {
            const long long n = a.e_first + 16LL * e;
            a.ehist[n / 16] = tot;
            *a.elatest = tot;
        }
        __syncthreads();
    }
}

template <class R> __global__ void __launch_bounds__(512) windowEpilogue(const EpilogueArgs<R> a)
{
    __shared__ double red[16];
    epilogueBody(a, red);
}

// Connect applied to a reflected state: the incident pulses the next step
// would see, in the reference's AoS layout (the reference's V). Nodes of the
// near-field box `nb` (none when nb.lo_in is null) see their sources
// completed by the residuals, as the step does.
template <class S, class O>
__global__ void incidentToAos(const S *__restrict__ refl, const uint8_t *__restrict__ mat, long long P,
                              int nx, int ny, int nz, int px, typename Traits<S>::R rho,
                              typename Traits<S>::R scale, O *__restrict__ out, NearBox nb)
{
    using R = typename Traits<S>::R;
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(c % nx);
        const int j = (int)((c / nx) % ny);
        const int k = (int)(c / ((long long)nx * ny));
        const long long node = ((long long)k * ny + j) * px + i;
        O *dst = out + c * 12;
        if (mat[node] == kPec)
        {
            for (int s = 0; s < 12; ++s) dst[s] = O(0);
            continue;
        }
        const int co[3] = { i, j, k };
        const int dims[3] = { nx, ny, nz };
        const long long st[3] = { 1, px, (long long)px * ny };
        const bool inBox = nb.lo_in != nullptr && nb.at(i, j, k) >= 0;
        for (int s = 0; s < 12; ++s)
        {
            const int ax = s >> 2, side = (s >> 1) & 1;
            const int qn = co[ax] + (side ? 1 : -1);
            R own = loadOne<S>(refl, s * P + node, scale);
            if (inBox) own += nb.lo_in[s * nb.bP + nb.at(i, j, k)] * scale;  // residuals: storage units
            R v;
            if (qn < 0 || qn >= dims[ax])
                v = rho * own;
            else
            {
                const long long nbr = node + (side ? st[ax] : -st[ax]);
                if (mat[nbr] == kPec)
                    v = -own;
                else
                {
                    v = loadOne<S>(refl, (s ^ 2) * P + nbr, scale);
                    if (inBox)
                    {
                        int c2[3] = { i, j, k };
                        c2[ax] = qn;
                        const long long b = nb.at(c2[0], c2[1], c2[2]);
                        if (b >= 0) v += nb.lo_in[(s ^ 2) * nb.bP + b] * scale;
                    }
                }
            }
            dst[s] = (O)v;
        }
    }
}

// Incident planes (state written by tlm_set_pulses) -> AoS; near-field box
// nodes completed by their residuals.
template <class S, class O>
__global__ void planesToAos(const S *__restrict__ planes, long long P, int nx, int ny, int nz, int px,
                            typename Traits<S>::R scale, O *__restrict__ out, NearBox nb)
{
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(c % nx);
        const int j = (int)((c / nx) % ny);
        const int k = (int)(c / ((long long)nx * ny));
        const long long node = ((long long)k * ny + j) * px + i;
        const long long b = nb.lo_in != nullptr ? nb.at(i, j, k) : -1;
        for (int s = 0; s < 12; ++s)
        {
            typename Traits<S>::R v = loadOne<S>(planes, s * P + node, scale);
            if (b >= 0) v += nb.lo_in[s * nb.bP + b] * scale;  // residuals: storage units
            out[c * 12 + s] = (O)v;
        }
    }
}

// Incident AoS state -> incident planes (PEC and padding nodes get 0), one
// aligned group of 4 nodes per thread iteration (the unit of every storage
// type, block floating point included). Near-field box nodes (nb.lo_out
// non-null) also get the residual of their rounded value.
template <class S, class I>
__global__ void aosToIncident(const I *__restrict__ in, const uint8_t *__restrict__ mat, long long P,
                              int nx, int ny, int nz, int px, typename Traits<S>::R inv_scale,
                              S *__restrict__ planes, NearBox nb)
{
    using R = typename Traits<S>::R;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < P / 4;
         g += (long long)gridDim.x * blockDim.x)
    {
        const long long node0 = g * 4;
        const int i0 = (int)(node0 % px);
        const long long r = node0 / px;
        const int j = (int)(r % ny), k = (int)(r / ny);
        for (int s = 0; s < 12; ++s)
        {
            R v[4];
            for (int c = 0; c < 4; ++c)
            {
                const int i = i0 + c;
                const bool real = i < nx && k < nz && mat[node0 + c] != kPec;
                const long long cell = ((long long)k * ny + j) * nx + i;
                v[c] = real ? (R)in[cell * 12 + s] : R(0);
            }
            storeVec<S, 4>(planes, s * P + node0, v, inv_scale, false, 0u, s);
            if constexpr (Traits<S>::kScaled)
            {
                if (nb.lo_out != nullptr)
                    for (int c = 0; c < 4; ++c)
                    {
                        const long long b = nb.at(i0 + c, j, k);
                        if (b >= 0)  // in storage units, like the step kernels' residuals
                        {
                            const R u = v[c] * inv_scale;
                            nb.lo_out[s * nb.bP + b] = u - decodeRaw(encodeRaw<S>(u));
                        }
                    }
            }
        }
    }
}

// Stub planes (storage units) -> AoS, times `scale`.
template <class R, class O>
__global__ void stubsToAos(const R *__restrict__ stub, long long P, int nx, int ny, int nz, int px,
                           O *__restrict__ out, R scale)
{
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(c % nx);
        const int j = (int)((c / nx) % ny);
        const int k = (int)(c / ((long long)nx * ny));
        const long long node = ((long long)k * ny + j) * px + i;
        for (int s = 0; s < 3; ++s) out[c * 3 + s] = (O)(stub[s * P + node] * scale);
    }
}

template <class R>
__global__ void aosToStubs(const R *__restrict__ in, long long P, int nx, int ny, int nz, int px,
                           R *__restrict__ stub)
{
    for (long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x; node < P;
         node += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(node % px);
        const long long r = node / px;
        const int j = (int)(r % ny), k = (int)(r / ny);
        const bool real = i < nx && k < nz;
        const long long c = ((long long)k * ny + j) * nx + i;
        for (int s = 0; s < 3; ++s) stub[s * P + node] = real ? in[c * 3 + s] : R(0);
    }
}

// Material map in the reference's cell order -> the padded layout (row pitch
// px, padding columns PEC), one padded node per thread.
static __global__ void padMaterial(const uint8_t *__restrict__ raw, int nx, int px, long long rows,
                            uint8_t *__restrict__ out)
{
    const long long P = rows * px;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < P;
         n += (long long)gridDim.x * blockDim.x)
    {
        const long long r = n / px;
        const int i = (int)(n - r * px);
        out[n] = i < nx ? raw[r * nx + i] : (uint8_t)kPec;
    }
}

// The material part of the step kernel's tile flags (tiles of T consecutive
// padded nodes, T a multiple of 32): kTileGeneral when a node of the tile is
// PEC or has a PEC neighbour inside the grid, kTileDiel when it holds a
// dielectric node; padding columns count for neither. Bits 8 and up of a
// tile's word count its dielectric nodes. One padded node per thread; the
// 32 nodes of a warp lie in one tile, so one lane ORs the warp's flags into
// that tile's word and adds its count.
static __global__ void materialTileFlags(const uint8_t *__restrict__ mat, int nx, int ny, int nz, int px, long long T,
                                  unsigned *__restrict__ flags)
{
    const long long sy = px, sz = (long long)px * ny, P = sz * nz;
    for (long long base = blockIdx.x * (long long)blockDim.x; base < P; base += (long long)gridDim.x * blockDim.x)
    {
        const long long n = base + threadIdx.x;
        unsigned f = 0;
        if (n < P)
        {
            const long long r = n / px;
            const int i = (int)(n - r * px);
            const int j = (int)(r % ny), k = (int)(r / ny);
            if (i < nx)
            {
                const uint8_t m = mat[n];
                if (m >= kDiel0) f |= kTileDiel;
                bool g = m == kPec;
                g = g || (i > 0 && mat[n - 1] == kPec) || (i < nx - 1 && mat[n + 1] == kPec);
                g = g || (j > 0 && mat[n - sy] == kPec) || (j < ny - 1 && mat[n + sy] == kPec);
                g = g || (k > 0 && mat[n - sz] == kPec) || (k < nz - 1 && mat[n + sz] == kPec);
                if (g) f |= kTileGeneral;
            }
        }
        const unsigned nd = __popc(__ballot_sync(0xffffffffu, (f & kTileDiel) != 0));
        f = __reduce_or_sync(0xffffffffu, f);
        const long long n0 = base + (threadIdx.x & ~31u);
        if ((threadIdx.x & 31) == 0 && f != 0 && n0 < P) atomicOr(&flags[n0 / T], f);
        // stub-loaded nodes of the tile, counted above the flag byte
        if ((threadIdx.x & 31) == 0 && nd != 0 && n0 < P) atomicAdd(&flags[n0 / T], nd << 8);
    }
}

// Unitarity KATs (TlmSolver.cpp:116-169): max |S^T W S - W| with W = 1 on
// the 12 links and yh on the 3 stubs (stub case).
static __global__ void unitarityKernel(float epsr, int withStubs, float *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int np = withStubs ? 15 : 12;
    const float yh = 4.0f * (epsr - 1.0f);
    float S[15][15];
    for (int c = 0; c < np; ++c)
    {
        float in[12], out[12], vs[3] = { 0.0f, 0.0f, 0.0f };
        for (int r = 0; r < 12; ++r) in[r] = 0.0f;
        if (c < 12) in[c] = 1.0f; else vs[c - 12] = 1.0f;
        if (withStubs)
            scatterStub(in, vs, yh, 0.0f, out);
        else
            scatterAir(in, out);
        for (int r = 0; r < 12; ++r) S[r][c] = out[r];
        if (withStubs)
            for (int r = 0; r < 3; ++r) S[12 + r][c] = vs[r];
    }
    float worst = 0.0f;
    for (int a = 0; a < np; ++a)
        for (int b = 0; b < np; ++b)
        {
            float dot = 0.0f;
            for (int r = 0; r < np; ++r)
            {
                const float w = r < 12 ? 1.0f : yh;
                dot += (withStubs ? w * S[r][a] : S[r][a]) * S[r][b];
            }
            const float want = (a == b) ? (a < 12 ? 1.0f : yh) : 0.0f;
            worst = fmaxf(worst, fabsf(dot - want));
        }
    *err = worst;
}

} // namespace tlmk
