// tlm_solver.cu -- C ABI (include/tlm_b200.h) over the fused SCN TLM kernels.
//
// The handle mirrors TlmSolver's life cycle (TlmSolver.h:202-264):
// setup -> add ports / probes / plane waves -> step or run -> read records.
// All device state is owned here; there is no CPU execution path.
#include "tlm_b200.h"
#include "tlm_internal.h"

#include "tlm_aux_kernels.cuh"
#include "tlm_host_math.h"
#include "tlm_step_kernel.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

using tlmk::kBlock;
using tlmk::kPadX;
using tlmk::SpecEntry;
using namespace tlmi;

namespace {

thread_local std::string g_threadError;

const char *kVersion = "tlm_b200 0.1.0 (sm_100a)";

// Smallest power of two >= v (a power of two maps to itself).
float pow2Ceil(float v)
{
    if (!(v > 0.0f) || !std::isfinite(v)) return 1.0f;
    int e = 0;
    const float m = std::frexp(v, &e);  // v = m * 2^e, m in [0.5, 1)
    return m == 0.5f ? v : std::ldexp(1.0f, e);
}

} // namespace

// Lets other translation units of the library report a failure of a call
// that has no handle through tlm_last_error(NULL).
void tlmSetThreadError(const std::string &m) { g_threadError = m; }
namespace tlmi {
void setThreadError(const std::string &m) { g_threadError = m; }
} // namespace tlmi


namespace tlmi {





void freeMonitors(tlm_solver *h)
{
    freeSurface(h);
    devFree(h, h->dSpec);
    devFree(h, h->dTile);
    devFree(h, h->dTileFlags);
    devFree(h, h->dStaged);
    devFree(h, h->dListed);
    h->nStaged = h->nListed = 0;
    devFree(h, h->dSamples);
    devFree(h, h->dEpart);
    devFree(h, h->dPortOff);
    devFree(h, h->dPortSlots);
    devFree(h, h->dPortPol);
    devFree(h, h->dPortNb);
    devFree(h, h->dProbeSlot);
    devFree(h, h->dVrec);
    devFree(h, h->dIrec);
    devFree(h, h->dPrec);
    devFree(h, h->dEhist);
    devFree(h, h->dWdt);
    devFree(h, h->dDft);
    devFree(h, h->dLo[0]);
    devFree(h, h->dLo[1]);
    h->nearBox = tlmk::NearBox{};
    devFree(h, h->dSlabB);
    devFree(h, h->dSlabI);
    devFree(h, h->dSlabS);
    h->nSlabB = h->nSlabI = h->nSlabS = 0;
    h->slabLists = false;
    h->recCap = 0;
    h->prepared = false;
}

void freeAll(tlm_solver *h)
{
    freeMonitors(h);
    devFree(h, h->dSv);
    h->svCount = 0;
    devFree(h, h->dPulses[0]);
    devFree(h, h->dPulses[1]);
    devFree(h, h->dStub);
    devFree(h, h->dMat);
    devFree(h, h->dYhat);
    devFree(h, h->dGhat);
    h->devBytes = 0;
}

bool busy(tlm_solver *h) { return h->running.load(); }

// ---- source values ----------------------------------------------------
double sourceValue(const tlm_solver *h, int n)
{
    if (h->cfg.waveform == TLM_WAVE_TABLE)
        return (n >= 0 && n < (int)h->svTable.size()) ? (double)h->svTable[n] : 0.0;
    if (h->storage == TLM_STORE_F64)
        return tlmh::waveform_f64(h->cfg.waveform, h->cfg.f0, h->dt64, n);
    return (double)tlmh::waveform_f32(h->cfg.waveform, h->cfg.f0, h->dt32, n);
}

// Padded node index of a reference linear cell index.
long long paddedNode(const tlm_solver *h, uint64_t cell)
{
    const long long i = (long long)(cell % (uint64_t)h->nx);
    const long long r = (long long)(cell / (uint64_t)h->nx);
    return r * h->px + i;
}

// Per-tile flags of the step kernel (tlmk::kTileGeneral, tlmk::kTileDiel):
// a tile is general when it is the partial last tile, holds a source or
// monitor entry (tileBegin ranges), or holds a node that is PEC or next to a
// PEC node.
// The near-field box (tlm_config.near_field = r > 0, FP16/BF16 storage):
// the bounding box of the PEC cells and port cells grown by r cells on every
// side and clipped to the grid; none (bP = 0) without such cells.
tlmk::NearBox nearBoxOf(const tlm_solver *h)
{
    tlmk::NearBox b{};
    const int r = h->cfg.near_field;
    if (r <= 0 || (h->storage != TLM_STORE_F16 && h->storage != TLM_STORE_BF16)) return b;
    int lo[3] = { h->nx, h->ny, h->nz }, hi[3] = { -1, -1, -1 };
    auto take = [&](long long i, long long j, long long k) {
        const long long c[3] = { i, j, k };
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = (int)std::min<long long>(lo[a], c[a]);
            hi[a] = (int)std::max<long long>(hi[a], c[a]);
        }
    };
    for (int k = 0; k < h->nz; ++k)
        for (int j = 0; j < h->ny; ++j)
        {
            const uint8_t *row = h->mat.data() + ((size_t)k * h->ny + j) * h->nx;
            for (int i = 0; i < h->nx; ++i)
                if (row[i] == tlmk::kPec) take(i, j, k);
        }
    for (const PortInfo &p : h->ports)
        for (uint64_t c : p.cells)
            take((long long)(c % (uint64_t)h->nx), (long long)(c / (uint64_t)h->nx % (uint64_t)h->ny),
                 (long long)(c / ((uint64_t)h->nx * h->ny)));
    if (hi[0] < 0) return b;
    const int n[3] = { h->nx, h->ny, h->nz };
    for (int a = 0; a < 3; ++a)
    {
        lo[a] = std::max(lo[a] - r, 0);
        hi[a] = std::min(hi[a] + r, n[a] - 1);
    }
    b.x0 = lo[0];
    b.y0 = lo[1];
    b.z0 = lo[2];
    b.nx = hi[0] - lo[0] + 1;
    b.ny = hi[1] - lo[1] + 1;
    b.nz = hi[2] - lo[2] + 1;
    b.bP = (long long)b.nx * b.ny * b.nz;
    return b;
}

std::vector<uint8_t> tileFlags(const tlm_solver *h, const std::vector<int> &tileBegin,
                               const std::vector<unsigned> &matFlags)
{
    const long long T = (long long)kBlock * h->V;
    const int nb = h->nblocks;
    std::vector<uint8_t> f((size_t)nb, h->cfg.general_tiles ? tlmk::kTileGeneral : 0);
    // PEC and dielectric flags from the device pass over the material map,
    // and whether at most a quarter of the tile's nodes are stub-loaded
    for (int b = 0; b < nb; ++b)
    {
        const unsigned mf = matFlags[(size_t)b];
        f[(size_t)b] |= (uint8_t)mf;
        if ((mf & tlmk::kTileDiel) && (long long)(mf >> 8) * tlmk::kStubSparseDiv <= T)
            f[(size_t)b] |= tlmk::kTileStubSparse;
    }
    if (h->nquads % kBlock) f[(size_t)nb - 1] |= tlmk::kTileGeneral;
    // outer y and z faces: the first and last plane, the first and last row
    // of every plane
    const long long planeN = (long long)h->px * h->ny;
    auto markRange = [&](long long n0, long long n1) {
        for (long long t = n0 / T; t * T < n1 && t < nb; ++t) f[(size_t)t] |= tlmk::kTileEdge;
    };
    markRange(0, planeN);
    markRange((long long)(h->nz - 1) * planeN, (long long)h->nz * planeN);
    for (int k = 0; k < h->nz; ++k)
    {
        markRange((long long)k * planeN, (long long)k * planeN + h->px);
        markRange((long long)k * planeN + (long long)(h->ny - 1) * h->px, (long long)(k + 1) * planeN);
    }
    for (int b = 0; b < nb; ++b)
        if (tileBegin[b + 1] > tileBegin[b]) f[(size_t)b] |= tlmk::kTileGeneral;
    // near-field box: the tiles over each of its rows
    const tlmk::NearBox &nb3 = h->nearBox;
    if (nb3.bP > 0)
        for (int k = nb3.z0; k < nb3.z0 + nb3.nz; ++k)
            for (int j = nb3.y0; j < nb3.y0 + nb3.ny; ++j)
            {
                const long long r0 = ((long long)k * h->ny + j) * h->px;
                for (long long t = (r0 + nb3.x0) / T; t * T < r0 + nb3.x0 + nb3.nx && t < nb; ++t)
                    f[(size_t)t] |= tlmk::kTileGeneral | tlmk::kTileNear;
            }
    return f;
}

// The material part of the tile flags, computed on the device from the
// padded material map (tlmk::materialTileFlags) and read back.
tlm_status materialFlags(tlm_solver *h, std::vector<unsigned> &out)
{
    out.assign((size_t)h->nblocks, 0u);
    unsigned *d = nullptr;
    TLM_TRY(tmpAlloc(h, &d, out.size() * sizeof(unsigned)));
    cudaError_t e = cudaMemsetAsync(d, 0, out.size() * sizeof(unsigned), h->stream);
    if (e == cudaSuccess)
    {
        tlmk::materialTileFlags<<<std::max(1, std::min(h->nblocks * h->V, 148 * 16)), 256, 0, h->stream>>>(
            h->dMat, h->nx, h->ny, h->nz, h->px, (long long)kBlock * h->V, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out.data(), d, out.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFreeAsync(d, h->stream);
    return h->cuda(e, "tile flags from the material map");
}

// Build the device tables of sources and monitors once, before the first
// step: the node-sorted entry list, per-block ranges, sample slots, port
// and probe descriptors, records and DFT accumulators.
// A slab's ghost planes are copies of the neighbours' planes whose pulses
// are only correct on the faces the halo exchange rewrites: nothing may be
// monitored there (sources are harmless: the owning slab injects them).
tlm_status checkSlabMonitors(tlm_solver *h)
{
    if (!h->ghostLo && !h->ghostHi) return TLM_OK;
    const long long plane = (long long)h->nx * h->ny;
    auto ghost = [&](long long cell) {
        const long long k = cell / plane;
        return (h->ghostLo && k == 0) || (h->ghostHi && k == h->nz - 1);
    };
    for (uint64_t c : h->probeCells)
        if (ghost((long long)c)) return h->fail(TLM_EINVAL, "a probe lies in a ghost plane of the slab");
    for (const PortInfo &p : h->ports)
    {
        for (uint64_t c : p.cells)
            if (ghost((long long)c)) return h->fail(TLM_EINVAL, "a port cell lies in a ghost plane of the slab");
        if (!p.cells.empty())
            for (int t = 0; t < 4; ++t)
                if (ghost(p.nb[t]))
                    return h->fail(TLM_EINVAL, "a port's current loop reaches a ghost plane of the slab");
    }
    return TLM_OK;
}

// The staged kernel's shape per storage type: FP32 stages tiles of 2 nodes
// per thread in 3 stages, FP16/BF16 tiles of 4 nodes per thread (the same 2
// KB per plane segment) in 2 stages (3 would not leave room for 2 blocks per
// SM); both run 2 blocks per SM.
template <class S> struct StagedShape
{
    static constexpr int V = 2, kStages = tlmk::kStages;
};
template <> struct StagedShape<__half>
{
    static constexpr int V = 4, kStages = 2;
};
template <> struct StagedShape<__nv_bfloat16>
{
    static constexpr int V = 4, kStages = 2;
};
template <class S> constexpr int stagedSmem()
{
    return StagedShape<S>::kStages * tlmk::Stage<S, StagedShape<S>::V>::kBytes;
}

template <class S> tlm_status stagedAttributes(tlm_solver *h)
{
    TLM_TRY(h->cuda(cudaFuncSetAttribute(tlmk::stepKernelStaged<S, StagedShape<S>::V, StagedShape<S>::kStages>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, stagedSmem<S>()),
                    "cudaFuncSetAttribute(stepKernelStaged)"));
    if constexpr (tlmk::kSparseStubs<S>)
        TLM_TRY(h->cuda(cudaFuncSetAttribute(
                            tlmk::stepKernelStaged<S, StagedShape<S>::V, StagedShape<S>::kStages, 2, true>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, stagedSmem<S>()),
                        "cudaFuncSetAttribute(stepKernelStaged)"));
    return TLM_OK;
}

// FP32 with 2 nodes per thread (the default shape): interior tiles go to the
// staged kernel, the others (PEC, sources, monitors, the partial last tile)
// to the list kernel, both launched every step (tlm_config.no_staging = 1: the single
// step kernel as before). The 16-bit storage types keep the single step
// kernel: staged, or with their interior tiles in a kernel of their own
// beside the list kernel, they measured slower.
tlm_status prepareStaging(tlm_solver *h, const std::vector<uint8_t> &flags)
{
    h->nStaged = h->nListed = 0;
    h->sparseStaged = false;
    h->stagedTiles.clear();
    h->listedTiles.clear();
    h->edgeTiles.clear();
    const bool f32 = h->storage == TLM_STORE_F32 && h->V == 2;
    const bool half = (h->storage == TLM_STORE_F16 || h->storage == TLM_STORE_BF16) && h->V == 4;
    if (!(f32 || half) || h->cfg.no_staging || !shapeOf(h->storage, h->variant).select) return TLM_OK;
    // staged lists hold packed entries (tile and flags, tlmk::packStagedEntry)
    std::vector<int> staged, listed, edge;
    for (int t = 0; t < h->nblocks; ++t)
    {
        const uint8_t f = flags[(size_t)t];
        if (f & tlmk::kTileGeneral)
            listed.push_back(t);
        else if (f & tlmk::kTileEdge)
        {
            listed.push_back(t);
            edge.push_back(tlmk::packStagedEntry(t, f));
        }
        else
            staged.push_back(tlmk::packStagedEntry(t, f));
    }
    // interior tiles on an outer face cost the producer more (their segments
    // come in runs); alone on the device they run in the list kernel, which
    // overlaps the staged one, while a batch stages them too (edgeTiles)
    h->edgeTiles = edge;
    std::sort(listed.begin(), listed.end());
    if (staged.empty()) return TLM_OK;
    if (half)
    {
        // 16-bit tiles with stub-loaded nodes stage 12 KB of FP32 stubs
        // beside 26 KB of pulses: with more than a quarter of them, the
        // single kernel measured faster (192^3 heterogeneous: 0.1142 ms staged
        // against 0.1056; the 384x384x256 dipole: 0.3436 against 0.359)
        size_t diel = 0;
        // (counting the sparse ones, which stage none: with them left out,
        // the 192^3 heterogeneous grid took the staged kernel and measured
        // 0.1086 ms against 0.1045)
        for (int e : staged) diel += (tlmk::entryFlags(e) & tlmk::kTileDiel) != 0;
        if (4 * diel > staged.size())
        {
            h->edgeTiles.clear();
            return TLM_OK;
        }
    }
    int sms = 0;
    TLM_CU(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    if (h->storage == TLM_STORE_F16)
        TLM_TRY(stagedAttributes<__half>(h));
    else if (h->storage == TLM_STORE_BF16)
        TLM_TRY(stagedAttributes<__nv_bfloat16>(h));
    else
        TLM_TRY(stagedAttributes<float>(h));
    if (!h->side)
    {
        TLM_CU(h, cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        TLM_CU(h, cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming));
        TLM_CU(h, cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming));
    }
    TLM_TRY(devAlloc(h, &h->dStaged, staged.size() * sizeof(int)));
    TLM_CU(h, cudaMemcpyAsync(h->dStaged, staged.data(), staged.size() * sizeof(int), cudaMemcpyHostToDevice,
                              h->stream));
    if (!listed.empty())
    {
        TLM_TRY(devAlloc(h, &h->dListed, listed.size() * sizeof(int)));
        TLM_CU(h, cudaMemcpyAsync(h->dListed, listed.data(), listed.size() * sizeof(int), cudaMemcpyHostToDevice,
                                  h->stream));
    }
    h->nStaged = (int)staged.size();
    for (int e : staged) h->sparseStaged |= (tlmk::entryFlags(e) & tlmk::kTileStubSparse) != 0;
    h->nListed = (int)listed.size();
    h->stagedTiles = std::move(staged);
    h->listedTiles = std::move(listed);
    h->stagedGrid = std::min(h->nStaged, 2 * sms);
    return TLM_OK;
}

tlm_status prepare(tlm_solver *h)
{
    if (h->prepared) return TLM_OK;
    TLM_TRY(checkSlabMonitors(h));
    freeMonitors(h);
    // unique monitored nodes -> sample slots
    std::vector<long long> monNodes;
    for (uint64_t c : h->probeCells) monNodes.push_back(paddedNode(h, c));
    for (const PortInfo &p : h->ports)
    {
        for (uint64_t c : p.cells) monNodes.push_back(paddedNode(h, c));
        if (!p.cells.empty())
            for (int t = 0; t < 4; ++t) monNodes.push_back(paddedNode(h, (uint64_t)p.nb[t]));
    }
    std::sort(monNodes.begin(), monNodes.end());
    monNodes.erase(std::unique(monNodes.begin(), monNodes.end()), monNodes.end());
    h->nsamp = (int)monNodes.size();
    auto slotOf = [&](uint64_t cell) {
        long long nd = paddedNode(h, cell);
        return (int)(std::lower_bound(monNodes.begin(), monNodes.end(), nd) - monNodes.begin());
    };

    // entries: plane-wave sources, then port cells (the reference's injection
    // order), then one sample per monitored node; stable-sorted by node.
    std::vector<SpecEntry> ents;
    for (const SourceInfo &s : h->sources)
        ents.push_back({ paddedNode(h, s.cell), tlmk::kInject, s.pol, s.amp, 0 });
    for (const PortInfo &p : h->ports)
        for (uint64_t c : p.cells) ents.push_back({ paddedNode(h, c), tlmk::kInject, p.pol, p.amp, 0 });
    for (int sidx = 0; sidx < h->nsamp; ++sidx)
        ents.push_back({ monNodes[sidx], tlmk::kSample, sidx, 0.0f, 0 });
    std::stable_sort(ents.begin(), ents.end(),
                     [](const SpecEntry &a, const SpecEntry &b) { return a.node < b.node; });
    std::vector<int> tile(h->nblocks + 1, 0);
    {
        size_t e = 0;
        const long long perBlock = (long long)kBlock * h->V;
        for (int b = 0; b <= h->nblocks; ++b)
        {
            const long long start = (long long)b * perBlock;
            while (e < ents.size() && ents[e].node < start) ++e;
            tile[b] = (int)e;
        }
    }
    h->nearBox = nearBoxOf(h);
    if (h->nearBox.bP > 0)
        for (int b = 0; b < 2; ++b)
        {
            const size_t bytes = (size_t)12 * h->nearBox.bP * sizeof(float);
            TLM_TRY(devAlloc(h, &h->dLo[b], bytes));
            TLM_CU(h, cudaMemsetAsync(h->dLo[b], 0, bytes, h->stream));
        }
    {
        std::vector<unsigned> mf;
        TLM_TRY(materialFlags(h, mf));
        const std::vector<uint8_t> flags = tileFlags(h, tile, mf);
        h->tileFlagsHost = flags;
        TLM_TRY(devAlloc(h, &h->dTileFlags, flags.size()));
        TLM_CU(h, cudaMemcpyAsync(h->dTileFlags, flags.data(), flags.size(), cudaMemcpyHostToDevice,
                                  h->stream));
        TLM_TRY(prepareStaging(h, flags));
    }
    h->specCount = (int)ents.size();
    if (!ents.empty())
    {
        TLM_TRY(devAlloc(h, &h->dSpec, ents.size() * sizeof(SpecEntry)));
        TLM_CU(h, cudaMemcpyAsync(h->dSpec, ents.data(), ents.size() * sizeof(SpecEntry),
                                  cudaMemcpyHostToDevice, h->stream));
        TLM_TRY(devAlloc(h, &h->dTile, tile.size() * sizeof(int)));
        TLM_CU(h, cudaMemcpyAsync(h->dTile, tile.data(), tile.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, h->stream));
    }
    const size_t rb = realBytes(h->storage);
    TLM_TRY(devAlloc(h, &h->dSamples, (size_t)h->window * std::max(h->nsamp, 1) * 6 * rb));
    TLM_TRY(devAlloc(h, &h->dEpart, (size_t)(h->window / 16 + 1) * h->nblocks * sizeof(double)));

    // port / probe descriptors
    const int np = (int)h->ports.size();
    std::vector<int> off(np + 1, 0), slots, pol(np), nb(np * 4, -1);
    for (int p = 0; p < np; ++p)
    {
        const PortInfo &pi = h->ports[p];
        for (uint64_t c : pi.cells) slots.push_back(slotOf(c));
        off[p + 1] = (int)slots.size();
        pol[p] = pi.pol;
        if (!pi.cells.empty())
            for (int t = 0; t < 4; ++t) nb[p * 4 + t] = slotOf((uint64_t)pi.nb[t]);
    }
    std::vector<int> pslot;
    for (uint64_t c : h->probeCells) pslot.push_back(slotOf(c));
    if (slots.empty()) slots.push_back(0);
    if (pslot.empty()) pslot.push_back(0);
    if (np == 0)
    {
        pol.push_back(0);
        nb.assign(4, -1);
    }
    TLM_TRY(devAlloc(h, &h->dPortOff, off.size() * sizeof(int)));
    TLM_TRY(devAlloc(h, &h->dPortSlots, slots.size() * sizeof(int)));
    TLM_TRY(devAlloc(h, &h->dPortPol, pol.size() * sizeof(int)));
    TLM_TRY(devAlloc(h, &h->dPortNb, nb.size() * sizeof(int)));
    TLM_TRY(devAlloc(h, &h->dProbeSlot, pslot.size() * sizeof(int)));
    TLM_CU(h, cudaMemcpyAsync(h->dPortOff, off.data(), off.size() * sizeof(int),
                              cudaMemcpyHostToDevice, h->stream));
    TLM_CU(h, cudaMemcpyAsync(h->dPortSlots, slots.data(), slots.size() * sizeof(int),
                              cudaMemcpyHostToDevice, h->stream));
    TLM_CU(h, cudaMemcpyAsync(h->dPortPol, pol.data(), pol.size() * sizeof(int),
                              cudaMemcpyHostToDevice, h->stream));
    TLM_CU(h, cudaMemcpyAsync(h->dPortNb, nb.data(), nb.size() * sizeof(int),
                              cudaMemcpyHostToDevice, h->stream));
    TLM_CU(h, cudaMemcpyAsync(h->dProbeSlot, pslot.data(), pslot.size() * sizeof(int),
                              cudaMemcpyHostToDevice, h->stream));
    // DFT
    const int nf = (int)h->dftFreqs.size();
    if (nf > 0 && np > 0)
    {
        std::vector<double> wdt(nf);
        const double dt = h->storage == TLM_STORE_F64 ? h->dt64 : (double)h->dt32;
        for (int f = 0; f < nf; ++f) wdt[f] = 2.0 * 3.14159265358979323846 * h->dftFreqs[f] * dt;
        TLM_TRY(devAlloc(h, &h->dWdt, nf * sizeof(double)));
        TLM_CU(h, cudaMemcpyAsync(h->dWdt, wdt.data(), nf * sizeof(double), cudaMemcpyHostToDevice,
                                  h->stream));
        TLM_TRY(devAlloc(h, &h->dDft, (size_t)np * nf * 4 * sizeof(double)));
        TLM_CU(h, cudaMemsetAsync(h->dDft, 0, (size_t)np * nf * 4 * sizeof(double), h->stream));
    }
    TLM_TRY(prepareSurface(h));
    h->prepared = true;
    return TLM_OK;
}

// Grow the step-major record arrays to hold `need` steps.
tlm_status ensureRecords(tlm_solver *h, long long need)
{
    if (need <= h->recCap) return TLM_OK;
    long long cap = std::max<long long>(need, std::max<long long>(h->cfg.total_steps, 64));
    cap = std::max(cap, h->recCap * 2);
    const int np = std::max<int>((int)h->ports.size(), 1);
    const int nr = std::max<int>((int)h->probeCells.size(), 1);
    double *v = nullptr, *i = nullptr, *p = nullptr, *e = nullptr;
    TLM_TRY(devAlloc(h, &v, (size_t)cap * np * sizeof(double)));
    TLM_TRY(devAlloc(h, &i, (size_t)cap * np * sizeof(double)));
    TLM_TRY(devAlloc(h, &p, (size_t)cap * nr * 3 * sizeof(double)));
    TLM_TRY(devAlloc(h, &e, (size_t)(cap / 16 + 2) * sizeof(double)));
    if (h->recCap > 0)
    {
        TLM_CU(h, cudaMemcpyAsync(v, h->dVrec, (size_t)h->recCap * np * sizeof(double),
                                  cudaMemcpyDeviceToDevice, h->stream));
        TLM_CU(h, cudaMemcpyAsync(i, h->dIrec, (size_t)h->recCap * np * sizeof(double),
                                  cudaMemcpyDeviceToDevice, h->stream));
        TLM_CU(h, cudaMemcpyAsync(p, h->dPrec, (size_t)h->recCap * nr * 3 * sizeof(double),
                                  cudaMemcpyDeviceToDevice, h->stream));
        TLM_CU(h, cudaMemcpyAsync(e, h->dEhist, (size_t)(h->recCap / 16 + 2) * sizeof(double),
                                  cudaMemcpyDeviceToDevice, h->stream));
        TLM_CU(h, cudaStreamSynchronize(h->stream));
        devFree(h, h->dVrec);
        devFree(h, h->dIrec);
        devFree(h, h->dPrec);
        devFree(h, h->dEhist);
    }
    h->dVrec = v;
    h->dIrec = i;
    h->dPrec = p;
    h->dEhist = e;
    h->recCap = cap;
    return TLM_OK;
}

// Kernel view of the near-field box for a step that reads pulse buffer `cur`.
tlmk::NearBox nearArgs(const tlm_solver *h, int cur)
{
    tlmk::NearBox b = h->nearBox;
    b.lo_in = b.bP > 0 ? h->dLo[cur] : nullptr;
    b.lo_out = b.bP > 0 ? h->dLo[cur ^ 1] : nullptr;
    return b;
}

// Launch the step kernel in the tile shape `variant` of the storage type
// (the shape tables of tlm_internal.h).
template <class S>
void launchShaped(const tlmk::StepArgs<S> &a, int variant, bool incident, int nblocks, cudaStream_t st)
{
    withShape<S>(variant, [&](auto V, auto MINB, auto SEL) {
        if (incident)
            tlmk::stepKernelShaped<S, V(), MINB(), true, SEL()><<<nblocks, kBlock, 0, st>>>(a);
        else
            tlmk::stepKernelShaped<S, V(), MINB(), false, SEL()><<<nblocks, kBlock, 0, st>>>(a);
    });
}

// The step kernels' arguments for step n, the i-th of its launch window
// (records of the window's first energy step eFirst), reading buffer curBuf.
template <class S> tlmk::StepArgs<S> stepArgs(const tlm_solver *h, int n, int i, long long eFirst)
{
    using R = typename tlmk::Traits<S>::R;
    tlmk::StepArgs<S> a;
    a.in = static_cast<const S *>(h->dPulses[h->curBuf]);
    a.out = static_cast<S *>(h->dPulses[h->curBuf ^ 1]);
    a.stub = static_cast<R *>(h->dStub);
    a.mat = h->dMat;
    a.yhat = static_cast<const R *>(h->dYhat);
    a.ghat = static_cast<const R *>(h->dGhat);
    a.P = h->P;
    a.nquads = h->nquads;
    a.nx = h->nx;
    a.ny = h->ny;
    a.nz = h->nz;
    a.px = h->px;
    a.nq = h->nq;
    a.div_nq = tlmk::makeFastDiv((unsigned)h->nq);
    a.div_ny = tlmk::makeFastDiv((unsigned)h->ny);
    a.rho = (R)h->cfg.boundary_rho;
    a.scale = (R)h->scale;
    a.inv_scale = (R)(1.0f / h->scale);
    a.tile_begin = h->dTile;
    a.spec = h->dSpec;
    a.tile_flags = h->dTileFlags;
    a.neg_zero = -0.0f;
    a.sv = (R)sourceValue(h, n) * (R)(1.0f / h->scale);  // in storage units
    a.samples = static_cast<R *>(h->dSamples) + (size_t)i * h->nsamp * 6;
    a.epart = (n % 16 == 0) ? h->dEpart + (size_t)((n - eFirst) / 16) * h->nblocks : nullptr;
    const long long planeNodes = (long long)h->ny * h->px;
    a.e_lo = h->ghostLo ? planeNodes : 0;
    a.e_hi = h->ghostHi ? (long long)(h->nz - 1) * planeNodes : LLONG_MAX;
    a.fault = h->dFault;
    a.stage_wait_ns = h->cfg.stage_wait_us > 0   ? (unsigned long long)h->cfg.stage_wait_us * 1000ull
                      : h->cfg.stage_wait_us < 0 ? 0ull
                                                 : tlmk::kStageWaitNs;
    a.near = nearArgs(h, h->curBuf);
    a.round_seed = tlmk::mix32((unsigned)n * 0x9E3779B9u + 0x7f4a7c15u);
    a.stochastic = h->cfg.rounding == 1 ? 1 : 0;
    return a;
}

template <class S> tlm_status launchStep(tlm_solver *h, int n, int i, long long eFirst)
{
    const tlmk::StepArgs<S> a = stepArgs<S>(h, n, i, eFirst);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (h->timing)
    {
        while (h->evs.size() < h->evUsed + 2)
        {
            cudaEvent_t ev;
            TLM_CU(h, cudaEventCreate(&ev));
            h->evs.push_back(ev);
        }
        e0 = h->evs[h->evUsed];
        e1 = h->evs[h->evUsed + 1];
        h->evUsed += 2;
        TLM_CU(h, cudaEventRecord(e0, h->stream));
    }
    if (surfaceActive(h)) TLM_TRY(launchSurface(h, n));  // reads the same input buffer, first
    if constexpr (std::is_same<S, float>::value)
    {
        if (h->nStaged > 0 && !h->stateIncident)
        {
            // the listed tiles run beside the staged ones (disjoint outputs,
            // the same input), on the side stream between a fork and a join
            if (h->nListed > 0)
            {
                TLM_CU(h, cudaEventRecord(h->evFork, h->stream));
                TLM_CU(h, cudaStreamWaitEvent(h->side, h->evFork, 0));
                tlmk::stepKernelList<S, 2, 4, true><<<h->nListed, kBlock, 0, h->side>>>(a, h->dListed);
                TLM_CU(h, cudaEventRecord(h->evJoin, h->side));
            }
            if (h->sparseStaged)
                tlmk::stepKernelStaged<S, 2, tlmk::kStages, 2, true>
                    <<<h->stagedGrid, tlmk::kStagedThreads, tlmk::kStages * tlmk::Stage<S>::kBytes, h->stream>>>(
                        a, h->dStaged, h->nStaged);
            else
                tlmk::stepKernelStaged<S, 2><<<h->stagedGrid, tlmk::kStagedThreads,
                                               tlmk::kStages * tlmk::Stage<S>::kBytes, h->stream>>>(a, h->dStaged,
                                                                                                     h->nStaged);
            if (h->nListed > 0) TLM_CU(h, cudaStreamWaitEvent(h->stream, h->evJoin, 0));
        }
        else
            launchShaped<S>(a, h->variant, h->stateIncident, h->nblocks, h->stream);
    }
    else if constexpr (std::is_same<S, __half>::value || std::is_same<S, __nv_bfloat16>::value)
    {
        if (h->nStaged > 0 && !h->stateIncident)
        {
            // as FP32: the listed tiles beside the staged ones
            if (h->nListed > 0)
            {
                TLM_CU(h, cudaEventRecord(h->evFork, h->stream));
                TLM_CU(h, cudaStreamWaitEvent(h->side, h->evFork, 0));
                tlmk::stepKernelList<S, 4, 3, true><<<h->nListed, kBlock, 0, h->side>>>(a, h->dListed);
                TLM_CU(h, cudaEventRecord(h->evJoin, h->side));
            }
            tlmk::stepKernelStaged<S, 4, StagedShape<S>::kStages>
                <<<h->stagedGrid, tlmk::kStagedThreads, stagedSmem<S>(), h->stream>>>(a, h->dStaged, h->nStaged);
            if (h->nListed > 0) TLM_CU(h, cudaStreamWaitEvent(h->stream, h->evJoin, 0));
        }
        else
            launchShaped<S>(a, h->variant, h->stateIncident, h->nblocks, h->stream);
    }
    else
        launchShaped<S>(a, h->variant, h->stateIncident, h->nblocks, h->stream);
    TLM_CU(h, cudaGetLastError());
    if (h->timing) TLM_CU(h, cudaEventRecord(e1, h->stream));
    h->stateIncident = false;
    h->curBuf ^= 1;
    return TLM_OK;
}

template <class R> tlm_status launchEpilogue(tlm_solver *h, long long base, int w, long long eFirst,
                                             int nE)
{
    tlmk::EpilogueArgs<R> a;
    a.samples = static_cast<const R *>(h->dSamples);
    a.nsamp = h->nsamp;
    a.w = w;
    a.base = base;
    a.nports = (int)h->ports.size();
    a.port_off = h->dPortOff;
    a.port_slots = h->dPortSlots;
    a.port_pol = h->dPortPol;
    a.port_nb = h->dPortNb;
    a.nprobes = (int)h->probeCells.size();
    a.probe_slot = h->dProbeSlot;
    a.probe_scale = h->storage == TLM_STORE_F64 ? (R)tlmh::probe_scale_f64(h->g.dl)
                                                : (R)tlmh::probe_scale_f32(h->g.dl);
    a.eta0 = (R)tlmh::eta0_f32();
    a.vrec = h->dVrec;
    a.irec = h->dIrec;
    a.prec = h->dPrec;
    a.nfreq = h->dDft ? (int)h->dftFreqs.size() : 0;
    a.wdt = h->dWdt;
    a.dft = h->dDft;
    a.epart = h->dEpart;
    a.nblocks = h->nblocks;
    a.n_e = nE;
    a.e_first = eFirst;
    a.ehist = h->dEhist;
    a.elatest = h->dElatest;
    tlmk::windowEpilogue<R><<<1, 512, 0, h->stream>>>(a);
    return h->cuda(cudaGetLastError(), "windowEpilogue launch");
}

// Enqueue n steps in windows of h->window; optionally stop early.
tlm_status enqueueSteps(tlm_solver *h, int nsteps, bool honourStop, bool *stopped)
{
    if (stopped) *stopped = false;
    TLM_TRY(prepare(h));
    int remaining = nsteps;
    while (remaining > 0)
    {
        if (honourStop && h->stopFlag.load())
        {
            if (stopped) *stopped = true;
            break;
        }
        const int w = std::min(remaining, h->window);
        const long long base = h->curStep;
        TLM_TRY(ensureRecords(h, base + w));
        const long long eFirst = (base + 15) / 16 * 16;
        const int nE = eFirst < base + w ? (int)((base + w - 1 - eFirst) / 16 + 1) : 0;
        for (int i = 0; i < w; ++i)
        {
            const int n = (int)(base + i);
            switch (h->storage)
            {
            case TLM_STORE_F64: TLM_TRY(launchStep<double>(h, n, i, eFirst)); break;
            case TLM_STORE_BF16: TLM_TRY(launchStep<__nv_bfloat16>(h, n, i, eFirst)); break;
            case TLM_STORE_F16: TLM_TRY(launchStep<__half>(h, n, i, eFirst)); break;
            case TLM_STORE_BFP16: TLM_TRY(launchStep<tlmk::Bfp4>(h, n, i, eFirst)); break;
            default: TLM_TRY(launchStep<float>(h, n, i, eFirst)); break;
            }
        }
        if (h->storage == TLM_STORE_F64)
            TLM_TRY(launchEpilogue<double>(h, base, w, eFirst, nE));
        else
            TLM_TRY(launchEpilogue<float>(h, base, w, eFirst, nE));
        h->curStep += w;
        ++h->recVersion;
        remaining -= w;
        if (honourStop)
        {
            // keep at most one window in flight so that a stop request or a
            // progress poll sees the device's actual position
            TLM_CU(h, cudaStreamSynchronize(h->stream));
            h->doneStep.store(h->curStep);
            double e = 0.0;
            TLM_CU(h, cudaMemcpy(&e, h->dElatest, sizeof(double), cudaMemcpyDeviceToHost));
            h->energy.store((float)e);
        }
    }
    return TLM_OK;
}

tlm_status syncState(tlm_solver *h)
{
    TLM_CU(h, cudaStreamSynchronize(h->stream));
    if (h->dFault)
    {
        unsigned f = 0;
        TLM_CU(h, cudaMemcpy(&f, h->dFault, sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (f & tlmk::kStageTimeout) return h->fail(TLM_ECUDA, "a staged tile's bulk copies never arrived");
        if (f) return h->fail(TLM_ECUDA, "bounds check tripped, code mask " + std::to_string(f));
    }
    h->doneStep.store(h->curStep);
    if (h->dElatest)
    {
        double e = 0.0;
        TLM_CU(h, cudaMemcpy(&e, h->dElatest, sizeof(double), cudaMemcpyDeviceToHost));
        h->energy.store((float)e);
    }
    return TLM_OK;
}

tlm_status checkHandle(tlm_solver *h)
{
    if (!h)
    {
        g_threadError = "null handle";
        return TLM_EINVAL;
    }
    return TLM_OK;
}

tlm_status checkReady(tlm_solver *h)
{
    TLM_TRY(checkHandle(h));
    if (!h->configured) return h->fail(TLM_ESTATE, "tlm_setup has not been called");
    if (busy(h)) return h->fail(TLM_EBUSY, "the handle is running");
    return TLM_OK;
}

tlm_status checkAddable(tlm_solver *h)
{
    TLM_TRY(checkReady(h));
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch");
    if (h->curStep > 0)
        return h->fail(TLM_ESTATE, "sources and monitors must be added before the first step");
    h->prepared = false;
    return TLM_OK;
}

// Per-step source values on the device (the batched kernel reads them there
// instead of taking them as a launch argument): sourceValue for [0, steps).
tlm_status uploadSourceTable(tlm_solver *h, long long steps)
{
    const size_t rb = realBytes(h->storage);
    if (h->dSv && h->svCount >= steps) return TLM_OK;
    devFree(h, h->dSv);
    h->svCount = 0;
    TLM_TRY(devAlloc(h, &h->dSv, (size_t)std::max<long long>(steps, 1) * rb));
    std::vector<double> v64((size_t)std::max<long long>(steps, 1), 0.0);
    for (long long n = 0; n < steps; ++n) v64[(size_t)n] = sourceValue(h, (int)n);
    if (h->storage == TLM_STORE_F64)
    {
        TLM_CU(h, cudaMemcpyAsync(h->dSv, v64.data(), v64.size() * 8, cudaMemcpyHostToDevice, h->stream));
        TLM_CU(h, cudaStreamSynchronize(h->stream));
    }
    else
    {
        std::vector<float> v32(v64.size());
        // in storage units (the step kernels' sv)
        const float inv = 1.0f / h->scale;
        for (size_t t = 0; t < v64.size(); ++t) v32[t] = (float)v64[t] * inv;
        TLM_CU(h, cudaMemcpyAsync(h->dSv, v32.data(), v32.size() * 4, cudaMemcpyHostToDevice, h->stream));
        TLM_CU(h, cudaStreamSynchronize(h->stream));
    }
    h->svCount = steps;
    return TLM_OK;
}

// Steps per launch window: the per-window sample and energy-partial buffers
// are resized; records and DFT accumulators are kept.
tlm_status setWindow(tlm_solver *h, int window)
{
    TLM_TRY(prepare(h));
    if (window == h->window) return TLM_OK;
    const size_t rb = realBytes(h->storage);
    devFree(h, h->dSamples);
    devFree(h, h->dEpart);
    h->window = window;
    TLM_TRY(devAlloc(h, &h->dSamples, (size_t)h->window * std::max(h->nsamp, 1) * 6 * rb));
    TLM_TRY(devAlloc(h, &h->dEpart, (size_t)(h->window / 16 + 1) * h->nblocks * sizeof(double)));
    return TLM_OK;
}

// Back to step 0 with zero fields (the state after setup), keeping the
// sources, monitors and device allocations.
tlm_status rewind(tlm_solver *h)
{
    const size_t sb = storageBytes(h->storage), rb = realBytes(h->storage);
    TLM_CU(h, cudaStreamSynchronize(h->stream));
    TLM_CU(h, cudaMemsetAsync(h->dPulses[0], 0, 12 * (size_t)h->P * sb, h->stream));
    TLM_CU(h, cudaMemsetAsync(h->dPulses[1], 0, 12 * (size_t)h->P * sb, h->stream));
    if (h->dStub) TLM_CU(h, cudaMemsetAsync(h->dStub, 0, 3 * (size_t)h->P * rb, h->stream));
    if (h->dDft)
        TLM_CU(h, cudaMemsetAsync(h->dDft, 0,
                                  h->ports.size() * h->dftFreqs.size() * 4 * sizeof(double), h->stream));
    TLM_CU(h, cudaMemsetAsync(h->dElatest, 0, sizeof(double), h->stream));
    TLM_TRY(rewindSurface(h));
    TLM_CU(h, cudaStreamSynchronize(h->stream));
    h->curStep = 0;
    ++h->recVersion;
    h->curBuf = 0;
    h->stateIncident = false;
    h->doneStep.store(0);
    h->energy.store(0.0f);
    h->finished.store(false);
    return TLM_OK;
}

// Switch the step-kernel tile shape of a handle that is at step 0.
tlm_status reshape(tlm_solver *h, int variant)
{
    if (h->curStep != 0) return h->fail(TLM_ESTATE, "the tile shape can only change at step 0");
    if (variant < 0 || variant >= shapeCount(h->storage)) return h->fail(TLM_EINVAL, "no such variant");
    if (variant == h->variant && h->prepared) return TLM_OK;
    const long long cap = h->recCap;
    const long long nquads = (long long)(h->px / shapeOf(h->storage, variant).V) * h->ny * h->nz;
    if (nquads >= (1LL << 31)) return h->fail(TLM_EINVAL, "grid too large for this tile shape");
    h->variant = variant;
    h->V = shapeOf(h->storage, variant).V;
    h->nq = h->px / h->V;
    h->nquads = nquads;
    h->nblocks = (int)((h->nquads + kBlock - 1) / kBlock);
    h->prepared = false;
    TLM_TRY(prepare(h));
    if (cap > 0) TLM_TRY(ensureRecords(h, cap));
    return TLM_OK;
}

cudaMemPool_t devicePool(int device)
{
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)pools.size() <= device) pools.resize(device + 1, nullptr);
    if (!pools[device])
    {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess)
        {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;  // keep freed blocks for reuse
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        // no opportunistic reuse: with it, every allocation weighs the freed
        // blocks of other streams one by one, and once a few thousand are
        // cached (256 handles set up and freed) setting up a handle's 25
        // buffers took 9 ms instead of 0.07 ms (measured on B200). Blocks
        // freed on other streams are still reused, through an event
        // dependency on their free.
        int opportunistic = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &opportunistic);
        pools[device] = pool;
    }
    return pools[device];
}

static size_t poolSpare(int device)
{
    cudaMemPool_t pool = devicePool(device);
    uint64_t reserved = 0, used = 0;
    if (pool)
    {
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    }
    return (size_t)(reserved > used ? reserved - used : 0);
}

bool poolCovers(int device, size_t bytes) { return poolSpare(device) >= bytes; }

size_t poolAvailable(int device)
{
    const size_t spare = poolSpare(device);
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return freeB + spare;
}

int gridBlocksFor(long long n)
{
    long long b = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

template <class S, class O> static tlm_status pulsesToHost(tlm_solver *h, O *out, size_t cap)
{
    using R = typename tlmk::Traits<S>::R;
    const size_t need = (size_t)h->ncell * 12;
    if (cap < need) return h->fail(TLM_EINVAL, "output holds " + std::to_string(cap) +
                                                   " values, the state has " + std::to_string(need));
    O *d = nullptr;
    TLM_TRY(tmpAlloc(h, &d, need * sizeof(O)));
    const S *cur = static_cast<const S *>(h->dPulses[h->curBuf]);
    if (h->stateIncident)  // state written by tlm_set_pulses: already incident
        tlmk::planesToAos<S, O><<<gridBlocksFor(h->ncell), 256, 0, h->stream>>>(
            cur, h->P, h->nx, h->ny, h->nz, h->px, (R)h->scale, d, nearArgs(h, h->curBuf));
    else
        tlmk::incidentToAos<S, O><<<gridBlocksFor(h->ncell), 256, 0, h->stream>>>(
            cur, h->dMat, h->P, h->nx, h->ny, h->nz, h->px, (R)h->cfg.boundary_rho, (R)h->scale, d,
            nearArgs(h, h->curBuf));
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, need * sizeof(O), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFreeAsync(d, h->stream);
    return h->cuda(e, "incident state export");
}

template <class O> static tlm_status getPulsesImpl(tlm_solver *h, O *out, size_t cap)
{
    TLM_TRY(checkReady(h));
    if (!out) return h->fail(TLM_EINVAL, "null output");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    switch (h->storage)
    {
    case TLM_STORE_F64: return pulsesToHost<double, O>(h, out, cap);
    case TLM_STORE_BF16: return pulsesToHost<__nv_bfloat16, O>(h, out, cap);
    case TLM_STORE_F16: return pulsesToHost<__half, O>(h, out, cap);
    case TLM_STORE_BFP16: return pulsesToHost<tlmk::Bfp4, O>(h, out, cap);
    default: return pulsesToHost<float, O>(h, out, cap);
    }
}

template <class S> static tlm_status setPulsesT(tlm_solver *h, const float *in)
{
    using R = typename tlmk::Traits<S>::R;
    const size_t need = (size_t)h->ncell * 12;
    float *d = nullptr;
    TLM_TRY(tmpAlloc(h, &d, need * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(d, in, need * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
    {
        // the box's residuals go beside the buffer the next step reads
        tlmk::NearBox nb = nearArgs(h, h->curBuf);
        nb.lo_out = const_cast<float *>(nb.lo_in);
        tlmk::aosToIncident<S, float><<<gridBlocksFor(h->P), 256, 0, h->stream>>>(
            d, h->dMat, h->P, h->nx, h->ny, h->nz, h->px, (R)(1.0f / h->scale),
            static_cast<S *>(h->dPulses[h->curBuf]), nb);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFreeAsync(d, h->stream);
    TLM_CU(h, e);
    h->stateIncident = true;
    return TLM_OK;
}

} // namespace tlmi

using namespace tlmi;

// ======================================================================
extern "C" {

const char *tlm_version(void) { return kVersion; }

void tlm_config_default(tlm_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->f0 = 1e9f;
    c->waveform = TLM_WAVE_CW_RAMPED;
    c->total_steps = 2000;
    c->settle_steps = 600;
    c->boundary_rho = 0.0f;
    c->huy_offset = 0;
    c->use_gpu = 1;
    c->record_every = 0;
    c->storage = TLM_STORE_F32;
    c->pulse_scale = 0.0f;
    c->steps_per_launch = 0;
    c->kernel_variant = 0;
    c->rounding = 0;
    c->general_tiles = 0;
    c->no_staging = 0;
    c->stage_wait_us = 0;
    c->near_field = 0;
    c->surface_monitors = 0;
}

int tlm_kernel_variants(int storage) { return shapeCount(storage); }

tlm_status tlm_kernel_variant_info(int storage, int variant, int *nodes_per_thread,
                                   int *min_blocks_per_sm)
{
    if (variant < 0 || variant >= shapeCount(storage))
    {
        g_threadError = "no such kernel variant";
        return TLM_EINVAL;
    }
    const Shape sh = shapeOf(storage, variant);
    if (nodes_per_thread) *nodes_per_thread = sh.V;
    if (min_blocks_per_sm) *min_blocks_per_sm = sh.minb;
    return TLM_OK;
}

tlm_status tlm_create(tlm_handle *out, int device)
{
    if (!out)
    {
        g_threadError = "null output pointer";
        return TLM_EINVAL;
    }
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        g_threadError = std::string("no CUDA device: ") +
                        (e != cudaSuccess ? cudaGetErrorString(e) : "device count is 0");
        return TLM_ENODEV;
    }
    if (device < 0 || device >= count)
    {
        g_threadError = "device index out of range";
        return TLM_EINVAL;
    }
    int major = 0, minor = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device) != cudaSuccess ||
        major < 10)
    {
        cudaGetLastError();
        g_threadError = "the kernels are built for sm_100a; device " + std::to_string(device) +
                        " is sm_" + std::to_string(major) + std::to_string(minor);
        return TLM_ENODEV;
    }
    tlm_solver *h = new tlm_solver();
    h->device = device;
    DeviceGuard dg(device);
    h->pool = devicePool(device);
    if (!h->pool)
    {
        g_threadError = "could not create the device memory pool";
        delete h;
        return TLM_ECUDA;
    }
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess)
    {
        g_threadError = std::string("cudaStreamCreate: ") + cudaGetErrorString(e);
        delete h;
        return TLM_ECUDA;
    }
    e = cudaMallocFromPoolAsync((void **)&h->dElatest, sizeof(double), h->pool, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->dElatest, 0, sizeof(double), h->stream);
    // error flags of the kernels: bounds checks (checked build), staged-tile
    // waits that ran out (every build)
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&h->dFault, sizeof(unsigned), h->pool, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->dFault, 0, sizeof(unsigned), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess)
    {
        g_threadError = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        cudaStreamDestroy(h->stream);
        delete h;
        return TLM_ENOMEM;
    }
    *out = h;
    return TLM_OK;
}

tlm_status tlm_destroy(tlm_handle h)
{
    if (!h) return TLM_OK;
    if (busy(h)) return h->fail(TLM_EBUSY, "cannot destroy a running handle");
    if (h->batch) return h->fail(TLM_EBUSY, "detach the handle from its batch first");
    DeviceGuard dg(h->device);
    cudaStreamSynchronize(h->stream);
    freeAll(h);
    if (h->dElatest) cudaFreeAsync(h->dElatest, h->stream);
    if (h->dFault) cudaFreeAsync(h->dFault, h->stream);
    for (cudaEvent_t ev : h->evs) cudaEventDestroy(ev);
    if (h->side)
    {
        cudaStreamSynchronize(h->side);
        cudaEventDestroy(h->evFork);
        cudaEventDestroy(h->evJoin);
        cudaStreamDestroy(h->side);
    }
    if (h->halo)
    {
        cudaStreamSynchronize(h->halo);
        cudaEventDestroy(h->evBoundary);
        cudaEventDestroy(h->evHalo);
        cudaStreamDestroy(h->halo);
    }
    cudaStreamDestroy(h->stream);
    delete h;
    return TLM_OK;
}

const char *tlm_last_error(tlm_handle h)
{
    if (!h) return g_threadError.c_str();
    return h->err.c_str();
}

tlm_status tlm_setup(tlm_handle h, const tlm_grid *grid, const uint8_t *mat, size_t n_cells,
                     const tlm_matprops *table, int n_table, const tlm_config *cfg)
{
    TLM_TRY(checkHandle(h));
    if (busy(h)) return h->fail(TLM_EBUSY, "the handle is running");
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch");
    if (!grid || !mat || !cfg) return h->fail(TLM_EINVAL, "null grid, material map or config");
    if (grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0)
        return h->fail(TLM_EINVAL, "grid dimensions must be positive");
    if (!(grid->dl > 0.0f) || !std::isfinite(grid->dl))
        return h->fail(TLM_EINVAL, "cell size dl must be positive and finite");
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    if ((long long)n_cells != n)
        return h->fail(TLM_EINVAL, "material map has " + std::to_string(n_cells) +
                                       " cells, the grid has " + std::to_string(n));
    if (n_table < 0 || n_table > 254 || (n_table > 0 && !table))
        return h->fail(TLM_EINVAL, "material table must have 0..254 entries");
    if (cfg->storage < TLM_STORE_F32 || cfg->storage > TLM_STORE_BFP16)
        return h->fail(TLM_EINVAL, "unknown pulse storage mode");
    if (cfg->waveform < 0 || cfg->waveform > TLM_WAVE_TABLE)
        return h->fail(TLM_EINVAL, "unknown waveform");
    if (cfg->total_steps < 0) return h->fail(TLM_EINVAL, "total_steps must be >= 0");
    if (cfg->kernel_variant < 0 || cfg->kernel_variant >= shapeCount(cfg->storage))
        return h->fail(TLM_EINVAL, "kernel_variant out of range for this storage mode");
    if (cfg->rounding < 0 || cfg->rounding > 1) return h->fail(TLM_EINVAL, "rounding must be 0 or 1");
    if (cfg->general_tiles < 0 || cfg->general_tiles > 1)
        return h->fail(TLM_EINVAL, "general_tiles must be 0 or 1");
    if (cfg->no_staging < 0 || cfg->no_staging > 1) return h->fail(TLM_EINVAL, "no_staging must be 0 or 1");
    if (cfg->near_field < 0) return h->fail(TLM_EINVAL, "near_field must be >= 0");
    if (cfg->near_field > 0 && cfg->storage != TLM_STORE_F16 && cfg->storage != TLM_STORE_BF16)
        return h->fail(TLM_EINVAL, "near_field applies to FP16 and BF16 storage only");
    if (cfg->surface_monitors < 0 || cfg->surface_monitors > 1)
        return h->fail(TLM_EINVAL, "surface_monitors must be 0 or 1");
    if (cfg->record_every < 0 || cfg->huy_offset < 0)
        return h->fail(TLM_EINVAL, "record_every and huy_offset must be >= 0");
    if (!std::isfinite(cfg->boundary_rho)) return h->fail(TLM_EINVAL, "boundary_rho not finite");
    // the host copy of the map and its largest id in one vectorised pass
    // (tlm_host_math.cpp, built by g++; the same scan compiled here measured
    // 3.9 ms on 192^3); the largest id decides, and the first offending cell
    // is looked for only when there is one
    std::vector<uint8_t> hostMat((size_t)n);
    const uint8_t maxId = tlmh::copy_max_u8(mat, hostMat.data(), (size_t)n);
    const bool anyDiel = maxId >= TLM_MAT_DIEL0;
    if (anyDiel && maxId - TLM_MAT_DIEL0 >= n_table)
        for (long long c = 0; c < n; ++c)
            if (mat[c] >= TLM_MAT_DIEL0 && mat[c] - TLM_MAT_DIEL0 >= n_table)
                return h->fail(TLM_EINVAL, "material id " + std::to_string(mat[c]) + " at cell " +
                                               std::to_string(c) + " has no table entry");
    DeviceGuard dg(h->device);
    cudaStreamSynchronize(h->stream);
    freeAll(h);
    h->configured = false;

    h->g = *grid;
    h->cfg = *cfg;
    h->storage = cfg->storage;
    h->window = cfg->steps_per_launch > 0 ? std::min(cfg->steps_per_launch, 4096) : 64;
    h->nx = grid->nx;
    h->ny = grid->ny;
    h->nz = grid->nz;
    h->variant = cfg->kernel_variant;
    h->V = shapeOf(h->storage, h->variant).V;
    h->px = (h->nx + kPadX - 1) / kPadX * kPadX;
    h->nq = h->px / h->V;
    h->P = (long long)h->px * h->ny * h->nz;
    h->ncell = n;
    h->nquads = (long long)h->nq * h->ny * h->nz;
    const long long nb = (h->nquads + kBlock - 1) / kBlock;
    if (h->nquads >= (1LL << 31)) return h->fail(TLM_EINVAL, "grid too large");
    h->nblocks = (int)nb;
    h->anyDiel = anyDiel;
    h->mat.swap(hostMat);
    h->epsr.resize(n_table);
    h->sigma.resize(n_table);
    for (int t = 0; t < n_table; ++t)
    {
        h->epsr[t] = table[t].epsr;
        h->sigma[t] = table[t].sigma;
    }
    h->yhat32.assign(std::max(n_table, 1), 0.0f);
    h->ghat32.assign(std::max(n_table, 1), 0.0f);
    h->yhat64.assign(std::max(n_table, 1), 0.0);
    h->ghat64.assign(std::max(n_table, 1), 0.0);
    tlmh::tables_f32(h->epsr.data(), h->sigma.data(), n_table, grid->dl, h->yhat32.data(),
                     h->ghat32.data());
    tlmh::tables_f64(h->epsr.data(), h->sigma.data(), n_table, grid->dl, h->yhat64.data(),
                     h->ghat64.data());
    h->dt32 = tlmh::timestep_f32(grid->dl);
    h->dt64 = tlmh::timestep_f64(grid->dl);
    h->sources.clear();
    h->ports.clear();
    h->probeCells.clear();
    h->svTable.clear();
    h->dftFreqs.clear();
    h->curStep = 0;
    ++h->recVersion;
    h->curBuf = 0;
    h->stateIncident = false;
    h->doneStep.store(0);
    h->energy.store(0.0f);
    h->finished.store(false);
    h->stopFlag.store(false);
    h->evUsed = 0;
    h->scale = 1.0f;
    h->surf.planeAxis = -1;
    h->surf.planeIndex = 0;
    buildSurfaceLists(h);

    // HBM admission: refuse up front if the state would not fit.
    const size_t sb = storageBytes(h->storage), rb = realBytes(h->storage);
    const size_t need = 2 * 12 * (size_t)h->P * sb + (anyDiel ? 3 * (size_t)h->P * rb : 0) +
                        (size_t)h->P + (size_t)h->nblocks * 8 * 8;
    // (when the blocks the pool keeps cover the state, no device memory is
    // taken and the device query, a few hundred microseconds, is skipped)
    if (!poolCovers(h->device, need))
    {
        const size_t freeB = poolAvailable(h->device);
        if (need + (size_t)(256u << 20) > freeB)
            return h->fail(TLM_ENOMEM, "grid needs " + std::to_string(need >> 20) + " MiB of HBM, " +
                                           std::to_string(freeB >> 20) + " MiB free");
    }

    TLM_TRY(devAlloc(h, &h->dPulses[0], 12 * (size_t)h->P * sb));
    TLM_TRY(devAlloc(h, &h->dPulses[1], 12 * (size_t)h->P * sb));
    TLM_CU(h, cudaMemsetAsync(h->dPulses[0], 0, 12 * (size_t)h->P * sb, h->stream));
    TLM_CU(h, cudaMemsetAsync(h->dPulses[1], 0, 12 * (size_t)h->P * sb, h->stream));
    if (anyDiel)
    {
        TLM_TRY(devAlloc(h, &h->dStub, 3 * (size_t)h->P * rb));
        TLM_CU(h, cudaMemsetAsync(h->dStub, 0, 3 * (size_t)h->P * rb, h->stream));
    }
    // padded material map: padding columns are PEC (never updated, zero);
    // the caller's map goes up as it is and is padded on the device
    {
        uint8_t *raw = nullptr;
        TLM_TRY(devAlloc(h, &h->dMat, (size_t)h->P));
        TLM_TRY(tmpAlloc(h, &raw, (size_t)n));
        cudaError_t e = cudaMemcpyAsync(raw, mat, (size_t)n, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess)
        {
            const long long rows = (long long)h->ny * h->nz;
            tlmk::padMaterial<<<(int)std::min<long long>((h->P + 255) / 256, 148LL * 32), 256, 0, h->stream>>>(
                raw, h->nx, h->px, rows, h->dMat);
            e = cudaGetLastError();
        }
        cudaFreeAsync(raw, h->stream);
        TLM_CU(h, e);
    }
    TLM_TRY(devAlloc(h, &h->dYhat, h->yhat32.size() * rb));
    TLM_TRY(devAlloc(h, &h->dGhat, h->ghat32.size() * rb));
    if (h->storage == TLM_STORE_F64)
    {
        TLM_CU(h, cudaMemcpyAsync(h->dYhat, h->yhat64.data(), h->yhat64.size() * 8,
                                  cudaMemcpyHostToDevice, h->stream));
        TLM_CU(h, cudaMemcpyAsync(h->dGhat, h->ghat64.data(), h->ghat64.size() * 8,
                                  cudaMemcpyHostToDevice, h->stream));
    }
    else
    {
        TLM_CU(h, cudaMemcpyAsync(h->dYhat, h->yhat32.data(), h->yhat32.size() * 4,
                                  cudaMemcpyHostToDevice, h->stream));
        TLM_CU(h, cudaMemcpyAsync(h->dGhat, h->ghat32.data(), h->ghat32.size() * 4,
                                  cudaMemcpyHostToDevice, h->stream));
    }
    TLM_CU(h, cudaMemsetAsync(h->dElatest, 0, sizeof(double), h->stream));
    TLM_CU(h, cudaStreamSynchronize(h->stream));
    h->configured = true;
    return TLM_OK;
}

tlm_status tlm_add_port(tlm_handle h, const uint64_t *cells, int n_cells, int pol_axis, float amp,
                        int *out_idx)
{
    TLM_TRY(checkAddable(h));
    if (pol_axis < 0 || pol_axis > 2) return h->fail(TLM_EINVAL, "pol_axis must be 0, 1 or 2");
    if (n_cells < 0 || (n_cells > 0 && !cells)) return h->fail(TLM_EINVAL, "bad cell list");
    PortInfo p;
    p.pol = pol_axis;
    p.amp = amp;
    for (int t = 0; t < n_cells; ++t)
        if (cells[t] < (uint64_t)h->ncell && h->mat[cells[t]] == TLM_MAT_AIR) p.cells.push_back(cells[t]);
    if (!p.cells.empty())
    {
        const long long stride[3] = { 1, h->nx, (long long)h->nx * h->ny };
        const long long c = (long long)p.cells[p.cells.size() / 2];
        const long long s1 = stride[(pol_axis + 1) % 3], s2 = stride[(pol_axis + 2) % 3];
        const long long nb[4] = { c + s1, c - s1, c + s2, c - s2 };
        for (int t = 0; t < 4; ++t)
        {
            if (nb[t] < 0 || nb[t] >= h->ncell)
                return h->fail(TLM_EINVAL, "port current loop around cell " + std::to_string(c) +
                                               " leaves the grid");
            p.nb[t] = nb[t];
        }
    }
    h->ports.push_back(p);
    if (out_idx) *out_idx = (int)h->ports.size() - 1;
    return TLM_OK;
}

tlm_status tlm_add_plane_wave(tlm_handle h, int prop_axis, int plane_index, int pol_axis, float amp)
{
    TLM_TRY(checkAddable(h));
    if (prop_axis < 0 || prop_axis > 2 || pol_axis < 0 || pol_axis > 2)
        return h->fail(TLM_EINVAL, "axes must be 0, 1 or 2");
    for (int k = 0; k < h->nz; ++k)
        for (int j = 0; j < h->ny; ++j)
            for (int i = 0; i < h->nx; ++i)
            {
                const int co[3] = { i, j, k };
                if (co[prop_axis] != plane_index) continue;
                const uint64_t c = ((uint64_t)k * h->ny + j) * h->nx + i;
                if (h->mat[c] == TLM_MAT_AIR) h->sources.push_back({ c, pol_axis, amp });
            }
    return TLM_OK;
}

tlm_status tlm_add_source_cells(tlm_handle h, const uint64_t *cells, int n_cells, int pol_axis,
                                float amp)
{
    TLM_TRY(checkAddable(h));
    if (pol_axis < 0 || pol_axis > 2) return h->fail(TLM_EINVAL, "pol_axis must be 0, 1 or 2");
    if (n_cells < 0 || (n_cells > 0 && !cells)) return h->fail(TLM_EINVAL, "bad cell list");
    for (int t = 0; t < n_cells; ++t)
        if (cells[t] < (uint64_t)h->ncell && h->mat[cells[t]] == TLM_MAT_AIR)
            h->sources.push_back({ cells[t], pol_axis, amp });
    return TLM_OK;
}

tlm_status tlm_add_probe(tlm_handle h, float x, float y, float z, int *out_idx)
{
    TLM_TRY(checkAddable(h));
    int i, j, k;
    tlmh::cell_of(h->g.origin, h->g.dl, x, y, z, &i, &j, &k);
    if (i < 0 || j < 0 || k < 0 || i >= h->nx || j >= h->ny || k >= h->nz)
    {
        if (out_idx) *out_idx = -1;
        return TLM_OK;
    }
    h->probeCells.push_back(((uint64_t)k * h->ny + j) * h->nx + i);
    if (out_idx) *out_idx = (int)h->probeCells.size() - 1;
    return TLM_OK;
}

tlm_status tlm_add_probe_cell(tlm_handle h, int i, int j, int k, int *out_idx)
{
    TLM_TRY(checkAddable(h));
    if (i < 0 || j < 0 || k < 0 || i >= h->nx || j >= h->ny || k >= h->nz)
    {
        if (out_idx) *out_idx = -1;
        return TLM_OK;
    }
    h->probeCells.push_back(((uint64_t)k * h->ny + j) * h->nx + i);
    if (out_idx) *out_idx = (int)h->probeCells.size() - 1;
    return TLM_OK;
}

tlm_status tlm_set_source_table(tlm_handle h, const float *sv, int n_steps)
{
    TLM_TRY(checkReady(h));
    if (n_steps < 0 || (n_steps > 0 && !sv)) return h->fail(TLM_EINVAL, "bad source table");
    h->svTable.assign(sv, sv + n_steps);
    return TLM_OK;
}

tlm_status tlm_set_port_dft(tlm_handle h, const double *freqs, int n_freq)
{
    TLM_TRY(checkAddable(h));
    if (n_freq < 0 || n_freq > 4096 || (n_freq > 0 && !freqs))
        return h->fail(TLM_EINVAL, "bad DFT frequency list");
    h->dftFreqs.assign(freqs, freqs + n_freq);
    return TLM_OK;
}

} // extern "C"

tlm_status tlmi::chooseScale(tlm_solver *h)
{
    if (h->storage != TLM_STORE_F16 && h->storage != TLM_STORE_BF16)
    {
        h->scale = 1.0f;
        return TLM_OK;
    }
    if (h->cfg.pulse_scale > 0.0f)
    {
        h->scale = pow2Ceil(h->cfg.pulse_scale);
        return TLM_OK;
    }
    // Largest single injection 0.5*|amp|*max|sv| bounds the pulse peak; store
    // it near 2^10 so that FP16 keeps ~20 binades of headroom below it.
    float amax = 0.0f;
    for (const SourceInfo &s : h->sources) amax = std::max(amax, std::fabs(s.amp));
    for (const PortInfo &p : h->ports)
        if (!p.cells.empty()) amax = std::max(amax, std::fabs(p.amp) * (float)p.cells.size());
    float svmax = 1.0f;
    if (h->cfg.waveform == TLM_WAVE_TABLE)
    {
        svmax = 0.0f;
        for (float v : h->svTable) svmax = std::max(svmax, std::fabs(v));
    }
    const float peak = std::max(0.5f * amax * svmax, 1e-30f);
    h->scale = h->storage == TLM_STORE_F16 ? pow2Ceil(peak) / 1024.0f : 1.0f;
    return TLM_OK;
}

extern "C" {


tlm_status tlm_step_async(tlm_handle h, int n_steps)
{
    TLM_TRY(checkReady(h));
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch: step the batch");
    if (n_steps < 0) return h->fail(TLM_EINVAL, "n_steps must be >= 0");
    if (h->slabBegun || h->slabOpen)
        return h->fail(TLM_ESTATE, "slab steps are open: end them and call tlm_slab_flush first");
    DeviceGuard dg(h->device);
    if (h->curStep == 0 && !h->prepared) TLM_TRY(chooseScale(h));
    return enqueueSteps(h, n_steps, false, nullptr);
}

tlm_status tlm_sync(tlm_handle h)
{
    TLM_TRY(checkReady(h));
    DeviceGuard dg(h->device);
    return syncState(h);
}

tlm_status tlm_step(tlm_handle h, int n_steps)
{
    TLM_TRY(tlm_step_async(h, n_steps));
    DeviceGuard dg(h->device);
    return syncState(h);
}

tlm_status tlm_run(tlm_handle h)
{
    TLM_TRY(checkReady(h));
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch: step the batch");
    DeviceGuard dg(h->device);
    bool expected = false;
    if (!h->running.compare_exchange_strong(expected, true))
        return h->fail(TLM_EBUSY, "already running");
    h->finished.store(false);
    tlm_status st = TLM_OK;
    bool stopped = false;
    if (h->curStep == 0 && !h->prepared) st = chooseScale(h);
    const int todo = h->cfg.total_steps - h->curStep;
    if (st == TLM_OK && todo > 0) st = enqueueSteps(h, todo, true, &stopped);
    if (st == TLM_OK) st = syncState(h);
    h->finished.store(true);
    h->running.store(false);
    if (st == TLM_OK && stopped) return h->fail(TLM_ESTOPPED, "stopped at step " + std::to_string(h->curStep));
    return st;
}

tlm_status tlm_request_stop(tlm_handle h)
{
    if (!h) return TLM_EINVAL;
    h->stopFlag.store(true);
    return TLM_OK;
}
int tlm_current_step(tlm_handle h) { return h ? h->doneStep.load() : -1; }
float tlm_current_energy(tlm_handle h) { return h ? h->energy.load() : 0.0f; }
int tlm_is_running(tlm_handle h) { return h ? (int)h->running.load() : 0; }
int tlm_is_finished(tlm_handle h) { return h ? (int)h->finished.load() : 0; }
int tlm_total_steps(tlm_handle h) { return h ? h->cfg.total_steps : 0; }

tlm_status tlm_timestep(tlm_handle h, float *dt)
{
    TLM_TRY(checkHandle(h));
    if (!h->configured) return h->fail(TLM_ESTATE, "tlm_setup has not been called");
    if (dt) *dt = h->dt32;
    return TLM_OK;
}

tlm_status tlm_get_grid(tlm_handle h, tlm_grid *grid)
{
    TLM_TRY(checkHandle(h));
    if (!h->configured) return h->fail(TLM_ESTATE, "tlm_setup has not been called");
    if (!grid) return h->fail(TLM_EINVAL, "null output");
    *grid = h->g;
    return TLM_OK;
}

// ---- z-slabs ----------------------------------------------------------------
tlm_status tlm_set_slab(tlm_handle h, int ghost_lo, int ghost_hi)
{
    TLM_TRY(checkReady(h));
    if (h->curStep != 0 || h->prepared) return h->fail(TLM_ESTATE, "tlm_set_slab must come before the first step");
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch");
    if ((ghost_lo != 0 && ghost_lo != 1) || (ghost_hi != 0 && ghost_hi != 1))
        return h->fail(TLM_EINVAL, "ghost_lo and ghost_hi are 0 or 1");
    if (h->nz < ghost_lo + ghost_hi + 1) return h->fail(TLM_EINVAL, "a slab needs at least one plane of its own");
    if (surfaceActive(h) || h->cfg.surface_monitors || h->cfg.record_every > 0)
        return h->fail(TLM_EINVAL, "slabs do not run surface monitors, cut planes or frames");
    if ((h->storage == TLM_STORE_F16 || h->storage == TLM_STORE_BF16) && !(h->cfg.pulse_scale > 0.0f))
        return h->fail(TLM_EINVAL, "16-bit slabs need an explicit pulse_scale shared by every slab");
    if (h->cfg.near_field > 0)
        return h->fail(TLM_EINVAL, "slabs do not exchange near-field residuals (near_field must be 0)");
    h->ghostLo = ghost_lo;
    h->ghostHi = ghost_hi;
    return TLM_OK;
}

tlm_status tlm_halo_bytes(tlm_handle h, size_t *bytes)
{
    TLM_TRY(checkReady(h));
    if (!bytes) return h->fail(TLM_EINVAL, "null output");
    *bytes = 2 * (size_t)h->ny * h->px * tlmi::storageBytes(h->storage);
    return TLM_OK;
}

namespace {
// Byte offset of the pulse plane (slot s, z-plane k) in a state buffer: a
// z-plane of one slot is ny * px consecutive nodes of every storage type.
size_t haloOffset(const tlm_solver *h, int slot, int k)
{
    return ((size_t)slot * h->P + (size_t)k * h->ny * h->px) * tlmi::storageBytes(h->storage);
}

// Copy the halo between the messages and pulse buffer `buf` on `stream`.
tlm_status haloCopyOn(tlm_solver *h, bool pack, void *lo, void *hi, cudaStream_t stream, int buf)
{
    if ((lo != nullptr) != (h->ghostLo != 0) || (hi != nullptr) != (h->ghostHi != 0))
        return h->fail(TLM_EINVAL, "pass a buffer exactly for each side that has a ghost plane");
    if (!lo && !hi) return TLM_OK;  // a slab without neighbours
    char *state = static_cast<char *>(h->dPulses[buf]);
    const size_t half = (size_t)h->ny * h->px * tlmi::storageBytes(h->storage);
    const int first = h->ghostLo, last = h->nz - 1 - h->ghostHi;
    // slot = axis * 4 + side * 2 + pol: 8, 9 leave a node through its -z
    // face, 10, 11 through its +z face.
    struct Side { char *buf; int slot, plane; };
    const Side sides[2] = {
        { static_cast<char *>(lo), pack ? 8 : 10, pack ? first : 0 },
        { static_cast<char *>(hi), pack ? 10 : 8, pack ? last : h->nz - 1 },
    };
    for (const Side &sd : sides)
    {
        if (!sd.buf) continue;
        for (int t = 0; t < 2; ++t)
        {
            char *dev = state + haloOffset(h, sd.slot + t, sd.plane);
            char *msg = sd.buf + t * half;
            TLM_CU(h, cudaMemcpyAsync(pack ? msg : dev, pack ? dev : msg, half, cudaMemcpyDeviceToDevice, stream));
        }
    }
    return TLM_OK;
}

tlm_status haloCopy(tlm_solver *h, bool pack, void *lo, void *hi)
{
    TLM_TRY(checkReady(h));
    if (h->stateIncident) return h->fail(TLM_ESTATE, "the state is incident pulses (tlm_set_pulses): step first");
    DeviceGuard dg(h->device);
    return haloCopyOn(h, pack, lo, hi, h->stream, h->curBuf);
}

// Tile lists of the two-phase slab step: tiles that hold a node of an own
// plane next to a ghost plane (boundary), the other tiles with an own node
// (interior; FP32's staged tiles among them as packed entries), none of the
// tiles that lie in ghost planes alone (ghost planes are not stepped: the
// own planes read only the halo slots that tlm_slab_step_end writes).
tlm_status buildSlabLists(tlm_solver *h)
{
    if (h->slabLists) return TLM_OK;
    const long long T = (long long)kBlock * h->V, planeN = (long long)h->ny * h->px;
    const int lowB = h->ghostLo ? 1 : -1, highB = h->ghostHi ? h->nz - 2 : -1;
    auto ghost = [&](long long k) { return (h->ghostLo && k == 0) || (h->ghostHi && k == h->nz - 1); };
    const bool staged = h->storage == TLM_STORE_F32 && !h->cfg.no_staging && h->V == 2 &&
                        shapeOf(h->storage, h->variant).select;
    std::vector<int> B, I, St;
    for (int t = 0; t < h->nblocks; ++t)
    {
        const long long n0 = (long long)t * T, n1 = std::min(n0 + T, h->P) - 1;
        bool allGhost = true, boundary = false;
        for (long long k = n0 / planeN; k <= n1 / planeN; ++k)
        {
            allGhost = allGhost && ghost(k);
            boundary = boundary || k == lowB || k == highB;
        }
        if (allGhost) continue;
        const uint8_t f = h->tileFlagsHost[(size_t)t];
        if (boundary)
            B.push_back(t);
        else if (staged && !(f & (tlmk::kTileGeneral | tlmk::kTileEdge)))
            St.push_back(tlmk::packStagedEntry(t, f));
        else
            I.push_back(t);
    }
    auto upload = [&](int **d, const std::vector<int> &v) -> tlm_status {
        if (v.empty()) return TLM_OK;
        TLM_TRY(devAlloc(h, d, v.size() * sizeof(int)));
        return h->cuda(cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream),
                       "slab tile lists");
    };
    TLM_TRY(upload(&h->dSlabB, B));
    TLM_TRY(upload(&h->dSlabI, I));
    TLM_TRY(upload(&h->dSlabS, St));
    h->nSlabB = (int)B.size();
    h->nSlabI = (int)I.size();
    h->nSlabS = (int)St.size();
    if (h->nSlabS > 0)
    {
        int sms = 0;
        TLM_CU(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        TLM_TRY(stagedAttributes<float>(h));
        h->slabStagedGrid = std::min(h->nSlabS, 2 * sms);
    }
    // tiles of ghost planes alone never write their energy partials: zero
    TLM_CU(h, cudaMemsetAsync(h->dEpart, 0, (size_t)(h->window / 16 + 1) * h->nblocks * sizeof(double), h->stream));
    if (!h->halo)
    {
        TLM_CU(h, cudaStreamCreateWithFlags(&h->halo, cudaStreamNonBlocking));
        TLM_CU(h, cudaEventCreateWithFlags(&h->evBoundary, cudaEventDisableTiming));
        TLM_CU(h, cudaEventCreateWithFlags(&h->evHalo, cudaEventDisableTiming));
    }
    h->slabLists = true;
    return TLM_OK;
}

// One phase of a slab step: 0 the boundary tiles, 1 the interior tiles.
// (C++ linkage: this part of the file lies inside the C ABI's extern "C".)
extern "C++" {
template <class S> tlm_status slabLaunch(tlm_solver *h, int phase)
{
    const tlmk::StepArgs<S> a = stepArgs<S>(h, (int)(h->slabBase + h->slabPos), h->slabPos, h->slabEFirst);
    withShape<S>(h->variant, [&](auto V, auto MINB, auto SEL) {
        if (phase == 0)
        {
            if (h->nSlabB > 0)
                tlmk::stepKernelList<S, V(), MINB(), SEL()><<<h->nSlabB, kBlock, 0, h->stream>>>(a, h->dSlabB);
            return;
        }
        if constexpr (std::is_same<S, float>::value && V() == 2 && SEL())
        {
            if (h->nSlabS > 0 && h->sparseStaged)
                tlmk::stepKernelStaged<S, 2, tlmk::kStages, 2, true>
                    <<<h->slabStagedGrid, tlmk::kStagedThreads, tlmk::kStages * tlmk::Stage<S>::kBytes, h->stream>>>(
                        a, h->dSlabS, h->nSlabS);
            else if (h->nSlabS > 0)
                tlmk::stepKernelStaged<S, 2><<<h->slabStagedGrid, tlmk::kStagedThreads,
                                               tlmk::kStages * tlmk::Stage<S>::kBytes, h->stream>>>(a, h->dSlabS,
                                                                                                    h->nSlabS);
        }
        if (h->nSlabI > 0)
            tlmk::stepKernelList<S, V(), MINB(), SEL()><<<h->nSlabI, kBlock, 0, h->stream>>>(a, h->dSlabI);
    });
    return h->cuda(cudaGetLastError(), "slab step launch");
}
} // extern "C++"

tlm_status slabPhase(tlm_solver *h, int phase)
{
    switch (h->storage)
    {
    case TLM_STORE_F64: return slabLaunch<double>(h, phase);
    case TLM_STORE_BF16: return slabLaunch<__nv_bfloat16>(h, phase);
    case TLM_STORE_F16: return slabLaunch<__half>(h, phase);
    case TLM_STORE_BFP16: return slabLaunch<tlmk::Bfp4>(h, phase);
    default: return slabLaunch<float>(h, phase);
    }
}

// Close the open launch window: records, DFT and energy of its steps.
tlm_status slabCloseWindow(tlm_solver *h)
{
    if (!h->slabOpen) return TLM_OK;
    const long long base = h->slabBase, eFirst = h->slabEFirst;
    const int w = h->slabPos;
    const int nE = eFirst < base + w ? (int)((base + w - 1 - eFirst) / 16 + 1) : 0;
    if (w > 0)
    {
        if (h->storage == TLM_STORE_F64)
            TLM_TRY(launchEpilogue<double>(h, base, w, eFirst, nE));
        else
            TLM_TRY(launchEpilogue<float>(h, base, w, eFirst, nE));
    }
    h->curStep += w;
    ++h->recVersion;
    h->slabOpen = false;
    h->slabPos = 0;
    return TLM_OK;
}
} // namespace

tlm_status tlm_halo_pack(tlm_handle h, void *send_lo, void *send_hi) { return haloCopy(h, true, send_lo, send_hi); }

tlm_status tlm_halo_unpack(tlm_handle h, const void *recv_lo, const void *recv_hi)
{
    return haloCopy(h, false, const_cast<void *>(recv_lo), const_cast<void *>(recv_hi));
}

tlm_status tlm_slab_step_begin(tlm_handle h, void *send_lo, void *send_hi)
{
    TLM_TRY(checkReady(h));
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch");
    if (h->slabBegun) return h->fail(TLM_ESTATE, "end the begun slab step first (tlm_slab_step_end)");
    if (h->stateIncident) return h->fail(TLM_ESTATE, "the state is incident pulses (tlm_set_pulses): step first");
    if (surfaceActive(h)) return h->fail(TLM_EINVAL, "slab steps do not run surface monitors");
    if ((send_lo != nullptr) != (h->ghostLo != 0) || (send_hi != nullptr) != (h->ghostHi != 0))
        return h->fail(TLM_EINVAL, "pass a buffer exactly for each side that has a ghost plane");
    DeviceGuard dg(h->device);
    if (h->curStep == 0 && !h->prepared) TLM_TRY(chooseScale(h));
    TLM_TRY(prepare(h));
    TLM_TRY(buildSlabLists(h));
    if (!h->slabOpen)
    {
        h->slabBase = h->curStep;
        h->slabEFirst = (h->slabBase + 15) / 16 * 16;
        h->slabPos = 0;
        TLM_TRY(ensureRecords(h, h->slabBase + h->window));
        h->slabOpen = true;
    }
    // the boundary tiles, then their outgoing halo on the halo stream
    TLM_TRY(slabPhase(h, 0));
    TLM_CU(h, cudaEventRecord(h->evBoundary, h->stream));
    TLM_CU(h, cudaStreamWaitEvent(h->halo, h->evBoundary, 0));
    TLM_TRY(haloCopyOn(h, true, send_lo, send_hi, h->halo, h->curBuf ^ 1));
    h->slabBegun = true;
    return TLM_OK;
}

tlm_status tlm_slab_step_end(tlm_handle h, const void *recv_lo, const void *recv_hi)
{
    TLM_TRY(checkReady(h));
    if (!h->slabBegun) return h->fail(TLM_ESTATE, "no slab step has begun (tlm_slab_step_begin)");
    if ((recv_lo != nullptr) != (h->ghostLo != 0) || (recv_hi != nullptr) != (h->ghostHi != 0))
        return h->fail(TLM_EINVAL, "pass a buffer exactly for each side that has a ghost plane");
    DeviceGuard dg(h->device);
    // the received halo into the ghost planes, beside the interior tiles
    TLM_TRY(haloCopyOn(h, false, const_cast<void *>(recv_lo), const_cast<void *>(recv_hi), h->halo, h->curBuf ^ 1));
    TLM_CU(h, cudaEventRecord(h->evHalo, h->halo));
    TLM_TRY(slabPhase(h, 1));
    TLM_CU(h, cudaStreamWaitEvent(h->stream, h->evHalo, 0));  // the next step reads the ghost planes
    h->curBuf ^= 1;
    h->slabBegun = false;
    if (++h->slabPos == h->window) TLM_TRY(slabCloseWindow(h));
    return TLM_OK;
}

tlm_status tlm_slab_flush(tlm_handle h)
{
    TLM_TRY(checkReady(h));
    if (h->slabBegun) return h->fail(TLM_ESTATE, "end the begun slab step first (tlm_slab_step_end)");
    DeviceGuard dg(h->device);
    return slabCloseWindow(h);
}

tlm_status tlm_get_halo_stream(tlm_handle h, void **stream)
{
    TLM_TRY(checkReady(h));
    if (!stream) return h->fail(TLM_EINVAL, "null output");
    DeviceGuard dg(h->device);
    if (!h->halo)
    {
        TLM_CU(h, cudaStreamCreateWithFlags(&h->halo, cudaStreamNonBlocking));
        TLM_CU(h, cudaEventCreateWithFlags(&h->evBoundary, cudaEventDisableTiming));
        TLM_CU(h, cudaEventCreateWithFlags(&h->evHalo, cudaEventDisableTiming));
    }
    *stream = (void *)h->halo;
    return TLM_OK;
}

int tlm_probe_count(tlm_handle h) { return h ? (int)h->probeCells.size() : 0; }
int tlm_port_count(tlm_handle h) { return h ? (int)h->ports.size() : 0; }

// Bring the probe and port records of every step so far to the host (one
// synchronisation, three copies) unless the host copies are current.
static tlm_status hostRecords(tlm_solver *h)
{
    if (h->recHostVersion == h->recVersion && h->recHostSteps == h->curStep) return TLM_OK;
    TLM_TRY(syncState(h));
    const size_t steps = (size_t)std::max(h->curStep, 0);
    const size_t nr = h->probeCells.size(), np = h->ports.size();
    h->precHost.resize(steps * nr * 3);
    h->vrecHost.resize(steps * np);
    h->irecHost.resize(steps * np);
    if (!h->precHost.empty())
        TLM_CU(h, cudaMemcpy(h->precHost.data(), h->dPrec, h->precHost.size() * sizeof(double),
                             cudaMemcpyDeviceToHost));
    if (!h->vrecHost.empty())
    {
        TLM_CU(h, cudaMemcpy(h->vrecHost.data(), h->dVrec, h->vrecHost.size() * sizeof(double),
                             cudaMemcpyDeviceToHost));
        TLM_CU(h, cudaMemcpy(h->irecHost.data(), h->dIrec, h->irecHost.size() * sizeof(double),
                             cudaMemcpyDeviceToHost));
    }
    h->recHostVersion = h->recVersion;
    h->recHostSteps = h->curStep;
    return TLM_OK;
}

static tlm_status getProbeImpl(tlm_solver *h, int idx, double *ex, double *ey, double *ez, float *fx,
                               float *fy, float *fz, int cap, int *n_out)
{
    TLM_TRY(checkReady(h));
    if (idx < 0 || idx >= (int)h->probeCells.size()) return h->fail(TLM_EINVAL, "probe index out of range");
    DeviceGuard dg(h->device);
    TLM_TRY(hostRecords(h));
    const int nr = (int)h->probeCells.size();
    const int steps = h->curStep;
    const int n = std::min(steps, cap);
    if (n_out) *n_out = steps;
    if (n <= 0) return TLM_OK;
    const std::vector<double> &buf = h->precHost;
    for (int t = 0; t < n; ++t)
    {
        const double *d = &buf[((size_t)t * nr + idx) * 3];
        if (ex) ex[t] = d[0];
        if (ey) ey[t] = d[1];
        if (ez) ez[t] = d[2];
        if (fx) fx[t] = (float)d[0];
        if (fy) fy[t] = (float)d[1];
        if (fz) fz[t] = (float)d[2];
    }
    return TLM_OK;
}

tlm_status tlm_get_probe(tlm_handle h, int idx, float *ex, float *ey, float *ez, int cap, int *n_out)
{
    return getProbeImpl(h, idx, nullptr, nullptr, nullptr, ex, ey, ez, cap, n_out);
}
tlm_status tlm_get_probe_f64(tlm_handle h, int idx, double *ex, double *ey, double *ez, int cap,
                             int *n_out)
{
    return getProbeImpl(h, idx, ex, ey, ez, nullptr, nullptr, nullptr, cap, n_out);
}
tlm_status tlm_get_probe_cell(tlm_handle h, int idx, uint64_t *cell)
{
    TLM_TRY(checkHandle(h));
    if (idx < 0 || idx >= (int)h->probeCells.size()) return h->fail(TLM_EINVAL, "probe index out of range");
    if (cell) *cell = h->probeCells[idx];
    return TLM_OK;
}

static tlm_status getPortImpl(tlm_solver *h, int idx, double *v, double *i, float *fv, float *fi,
                              int cap, int *n_out)
{
    TLM_TRY(checkReady(h));
    if (idx < 0 || idx >= (int)h->ports.size()) return h->fail(TLM_EINVAL, "port index out of range");
    DeviceGuard dg(h->device);
    TLM_TRY(hostRecords(h));
    const int np = (int)h->ports.size();
    const int steps = h->curStep;
    const int n = std::min(steps, cap);
    if (n_out) *n_out = steps;
    if (n <= 0) return TLM_OK;
    const std::vector<double> &bv = h->vrecHost, &bi = h->irecHost;
    for (int t = 0; t < n; ++t)
    {
        const double a = bv[(size_t)t * np + idx], b = bi[(size_t)t * np + idx];
        if (v) v[t] = a;
        if (i) i[t] = b;
        if (fv) fv[t] = (float)a;
        if (fi) fi[t] = (float)b;
    }
    return TLM_OK;
}

tlm_status tlm_get_port(tlm_handle h, int idx, float *v, float *i, int cap, int *n_out)
{
    return getPortImpl(h, idx, nullptr, nullptr, v, i, cap, n_out);
}
tlm_status tlm_get_port_f64(tlm_handle h, int idx, double *v, double *i, int cap, int *n_out)
{
    return getPortImpl(h, idx, v, i, nullptr, nullptr, cap, n_out);
}
tlm_status tlm_get_port_cells(tlm_handle h, int idx, uint64_t *cells, int cap, int *n_out)
{
    TLM_TRY(checkHandle(h));
    if (idx < 0 || idx >= (int)h->ports.size()) return h->fail(TLM_EINVAL, "port index out of range");
    const auto &c = h->ports[idx].cells;
    if (n_out) *n_out = (int)c.size();
    for (int t = 0; cells && t < (int)c.size() && t < cap; ++t) cells[t] = c[t];
    return TLM_OK;
}

tlm_status tlm_get_port_dft(tlm_handle h, int idx, double *v_re, double *v_im, double *i_re,
                            double *i_im, int cap, int *n_out)
{
    TLM_TRY(checkReady(h));
    if (idx < 0 || idx >= (int)h->ports.size()) return h->fail(TLM_EINVAL, "port index out of range");
    const int nf = (int)h->dftFreqs.size();
    if (n_out) *n_out = nf;
    if (nf == 0) return TLM_OK;
    DeviceGuard dg(h->device);
    TLM_TRY(prepare(h));
    TLM_TRY(syncState(h));
    std::vector<double> buf((size_t)nf * 4);
    TLM_CU(h, cudaMemcpy(buf.data(), h->dDft + (size_t)idx * nf * 4, buf.size() * sizeof(double),
                         cudaMemcpyDeviceToHost));
    for (int f = 0; f < nf && f < cap; ++f)
    {
        if (v_re) v_re[f] = buf[f * 4 + 0];
        if (v_im) v_im[f] = buf[f * 4 + 1];
        if (i_re) i_re[f] = buf[f * 4 + 2];
        if (i_im) i_im[f] = buf[f * 4 + 3];
    }
    return TLM_OK;
}

tlm_status tlm_get_energy_history(tlm_handle h, int *steps, float *vals, double *vals64, int cap,
                                  int *n_out)
{
    TLM_TRY(checkReady(h));
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    const int ne = h->curStep > 0 ? (h->curStep - 1) / 16 + 1 : 0;
    if (n_out) *n_out = ne;
    const int n = std::min(ne, cap);
    if (n <= 0) return TLM_OK;
    std::vector<double> buf(n);
    TLM_CU(h, cudaMemcpy(buf.data(), h->dEhist, n * sizeof(double), cudaMemcpyDeviceToHost));
    for (int t = 0; t < n; ++t)
    {
        if (steps) steps[t] = 16 * t;
        if (vals) vals[t] = (float)buf[t];
        if (vals64) vals64[t] = buf[t];
    }
    return TLM_OK;
}

tlm_status tlm_get_pulses(tlm_handle h, float *out, size_t cap) { return getPulsesImpl(h, out, cap); }
tlm_status tlm_get_pulses_f64(tlm_handle h, double *out, size_t cap) { return getPulsesImpl(h, out, cap); }

tlm_status tlm_set_pulses(tlm_handle h, const float *in, size_t n)
{
    TLM_TRY(checkReady(h));
    if (h->batch) return h->fail(TLM_ESTATE, "the handle is attached to a batch");
    if (!in || n != (size_t)h->ncell * 12)
        return h->fail(TLM_EINVAL, "pulse array must hold 12 values per cell");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    // the state is stored with the scale the steps will decode it with, and
    // a near-field box needs its residual planes
    if (h->curStep == 0 && !h->prepared) TLM_TRY(chooseScale(h));
    if (h->cfg.near_field > 0) TLM_TRY(prepare(h));
    switch (h->storage)
    {
    case TLM_STORE_F64: return setPulsesT<double>(h, in);
    case TLM_STORE_BF16: return setPulsesT<__nv_bfloat16>(h, in);
    case TLM_STORE_F16: return setPulsesT<__half>(h, in);
    case TLM_STORE_BFP16: return setPulsesT<tlmk::Bfp4>(h, in);
    default: return setPulsesT<float>(h, in);
    }
}

tlm_status tlm_get_stubs(tlm_handle h, float *out, size_t cap)
{
    TLM_TRY(checkReady(h));
    if (!out) return h->fail(TLM_EINVAL, "null output");
    const size_t need = (size_t)h->ncell * 3;
    if (cap < need) return h->fail(TLM_EINVAL, "output too small for the stub state");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    if (!h->dStub)
    {
        std::fill(out, out + need, 0.0f);
        return TLM_OK;
    }
    float *d = nullptr;
    TLM_TRY(tmpAlloc(h, &d, need * sizeof(float)));
    if (h->storage == TLM_STORE_F64)
        tlmk::stubsToAos<double, float><<<gridBlocksFor(h->ncell), 256, 0, h->stream>>>(
            static_cast<const double *>(h->dStub), h->P, h->nx, h->ny, h->nz, h->px, d, 1.0);
    else
        tlmk::stubsToAos<float, float><<<gridBlocksFor(h->ncell), 256, 0, h->stream>>>(
            static_cast<const float *>(h->dStub), h->P, h->nx, h->ny, h->nz, h->px, d, h->scale);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, need * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFreeAsync(d, h->stream);
    return h->cuda(e, "stub export");
}

tlm_status tlm_get_materials(tlm_handle h, uint8_t *out, size_t cap)
{
    TLM_TRY(checkReady(h));
    if (!out || cap < (size_t)h->ncell) return h->fail(TLM_EINVAL, "output too small");
    DeviceGuard dg(h->device);
    TLM_TRY(syncState(h));
    std::vector<uint8_t> pm((size_t)h->P);
    TLM_CU(h, cudaMemcpy(pm.data(), h->dMat, pm.size(), cudaMemcpyDeviceToHost));
    for (long long r = 0; r < (long long)h->ny * h->nz; ++r)
        std::memcpy(out + (size_t)r * h->nx, &pm[(size_t)r * h->px], h->nx);
    return TLM_OK;
}

tlm_status tlm_get_tables(tlm_handle h, float *yhat, float *ghat, int cap, int *n_out)
{
    TLM_TRY(checkReady(h));
    const int n = (int)h->epsr.size();
    if (n_out) *n_out = n;
    DeviceGuard dg(h->device);
    if (h->storage == TLM_STORE_F64)
    {
        std::vector<double> y(std::max(n, 1)), gg(std::max(n, 1));
        TLM_CU(h, cudaMemcpy(y.data(), h->dYhat, y.size() * 8, cudaMemcpyDeviceToHost));
        TLM_CU(h, cudaMemcpy(gg.data(), h->dGhat, gg.size() * 8, cudaMemcpyDeviceToHost));
        for (int t = 0; t < n && t < cap; ++t)
        {
            if (yhat) yhat[t] = (float)y[t];
            if (ghat) ghat[t] = (float)gg[t];
        }
        return TLM_OK;
    }
    std::vector<float> y(std::max(n, 1)), gg(std::max(n, 1));
    TLM_CU(h, cudaMemcpy(y.data(), h->dYhat, y.size() * 4, cudaMemcpyDeviceToHost));
    TLM_CU(h, cudaMemcpy(gg.data(), h->dGhat, gg.size() * 4, cudaMemcpyDeviceToHost));
    for (int t = 0; t < n && t < cap; ++t)
    {
        if (yhat) yhat[t] = y[t];
        if (ghat) ghat[t] = gg[t];
    }
    return TLM_OK;
}

tlm_status tlm_waveform_value(int waveform, float f0, float dl, int n, float *out)
{
    if (!out || waveform < 0 || waveform > TLM_WAVE_GAUSSIAN_PULSE || !(dl > 0.0f))
    {
        g_threadError = "bad waveform arguments";
        return TLM_EINVAL;
    }
    *out = tlmh::waveform_f32(waveform, f0, tlmh::timestep_f32(dl), n);
    return TLM_OK;
}

static tlm_status unitarity(int device, float epsr, int stubs, float *err)
{
    if (!err)
    {
        g_threadError = "null output";
        return TLM_EINVAL;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    {
        cudaGetLastError();
        g_threadError = "no such CUDA device";
        return TLM_ENODEV;
    }
    DeviceGuard dg(device);
    float *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(float));
    if (e == cudaSuccess)
    {
        tlmk::unitarityKernel<<<1, 32>>>(epsr, stubs, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(err, d, sizeof(float), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess)
    {
        g_threadError = std::string("unitarity kernel: ") + cudaGetErrorString(e);
        return TLM_ECUDA;
    }
    return TLM_OK;
}

tlm_status tlm_scatter_unitarity_error(int device, float *err) { return unitarity(device, 1.0f, 0, err); }
tlm_status tlm_stub_unitarity_error(int device, float epsr, float *err)
{
    return unitarity(device, epsr, 1, err);
}

tlm_status tlm_get_stream(tlm_handle h, void **stream)
{
    TLM_TRY(checkHandle(h));
    if (stream) *stream = (void *)h->stream;
    return TLM_OK;
}

tlm_status tlm_device_bytes(tlm_handle h, size_t *bytes)
{
    TLM_TRY(checkHandle(h));
    if (bytes) *bytes = h->devBytes;
    return TLM_OK;
}

tlm_status tlm_set_kernel_timing(tlm_handle h, int enable)
{
    TLM_TRY(checkHandle(h));
    DeviceGuard dg(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->timing = enable != 0;
    h->evUsed = 0;
    return TLM_OK;
}

tlm_status tlm_near_field_box(tlm_handle h, int box[6])
{
    TLM_TRY(checkHandle(h));
    if (!box) return h->fail(TLM_EINVAL, "null output");
    const tlmk::NearBox &b = h->nearBox;
    const int v[6] = { b.x0, b.y0, b.z0, b.nx, b.ny, b.nz };
    for (int t = 0; t < 6; ++t) box[t] = b.bP > 0 ? v[t] : 0;
    return TLM_OK;
}

tlm_status tlm_step_launches(tlm_handle h, int *per_step)
{
    TLM_TRY(checkHandle(h));
    if (!per_step) return h->fail(TLM_EINVAL, "null output");
    TLM_TRY(prepare(h));
    *per_step = (h->nStaged > 0 ? (h->nListed > 0 ? 2 : 1) : 1) + (surfaceActive(h) ? 1 : 0);
    return TLM_OK;
}

tlm_status tlm_kernel_time(tlm_handle h, double *ms, long long *launches)
{
    TLM_TRY(checkHandle(h));
    DeviceGuard dg(h->device);
    TLM_CU(h, cudaStreamSynchronize(h->stream));
    double tot = 0.0;
    for (size_t t = 0; t + 1 < h->evUsed; t += 2)
    {
        float m = 0.0f;
        TLM_CU(h, cudaEventElapsedTime(&m, h->evs[t], h->evs[t + 1]));
        tot += m;
    }
    if (ms) *ms = tot;
    if (launches) *launches = (long long)(h->evUsed / 2);
    return TLM_OK;
}

} // extern "C"
