// tlm_step_kernel.cuh -- the fused SCN TLM time step (one launch per step).
//
// One thread owns V consecutive nodes along x (one aligned vector per plane).
// Per step it:
//   1. gathers the 12 incident pulses of its nodes from the reflected pulses
//      of the previous step (connect, TlmSolver.cpp:551-613): x-neighbours
//      come from the same vector or a lane shuffle, y/z neighbours from
//      aligned vector loads one row / one plane away;
//   2. adds the soft sources of its nodes (TlmSolver.cpp:487-505);
//   3. records monitor samples (node voltages and circulations) for probes
//      and ports (TlmSolver.cpp:677-713) and, every 16 steps, the block's
//      FP64 share of the link energy (TlmSolver.cpp:766-789);
//   4. scatters (air / stub-loaded, TlmSolver.cpp:59-113) and stores the
//      reflected pulses at its own, aligned position.
// DRAM traffic per node: 12 pulses read + 12 written + 1 material byte
// (+ 3 stub pulses read and written on dielectric nodes).
#pragma once

#include "tlm_device.cuh"

#include <climits>
#include <type_traits>

namespace tlmk {

template <class S> struct StepArgs
{
    using R = typename Traits<S>::R;
    const S *__restrict__ in;      // 12 planes, reflected pulses of step n-1
    S *__restrict__ out;           // 12 planes, reflected pulses of step n
    R *__restrict__ stub;          // 3 planes (nullptr without dielectrics)
    const uint8_t *__restrict__ mat;
    const R *__restrict__ yhat;
    const R *__restrict__ ghat;
    long long P;                   // plane stride (elements)
    long long nquads;              // number of V-node groups
    int nx, ny, nz, px, nq;        // nq = px / V
    FastDiv div_nq, div_ny;        // division by nq and by ny (nquads < 2^31)
    R rho;
    R scale, inv_scale;            // pulse = stored * scale (BF16/F16); the step works in
                                   // storage units: sv, stubs and residuals are in those
                                   // units, samples and energy partials are scaled back
    // sources and monitors
    const int *__restrict__ tile_begin;  // [gridDim.x + 1] ranges into spec
    const SpecEntry *__restrict__ spec;
    R sv;                          // source value of this step
    R *__restrict__ samples;       // [nsamp][6] of this step
    double *__restrict__ epart;    // [gridDim.x] energy partials (energy steps)
    long long e_lo, e_hi;          // nodes [e_lo, e_hi) count towards the energy (a slab's own planes)
    unsigned int *__restrict__ fault;  // bounds-check record (checked builds)
    unsigned int round_seed;       // per-step seed of stochastic rounding
    int stochastic;                // BF16/F16: round stochastically
    const uint8_t *__restrict__ tile_flags;  // per tile: kTileGeneral / kTileDiel (nullptr: all general)
    float neg_zero;                // -0.0f, supplied at run time (see mul2)
    unsigned long long stage_wait_ns;  // staged tiles: consumers' limit on a stage wait (0: first poll)
    NearBox near;                  // 16-bit storage: the near-field box (near.lo_in == nullptr: none)
};

// Per-tile flags, computed on the host from the material map and the source
// and monitor lists. A tile without kTileGeneral is an interior tile: every
// thread of it is live, neither its nodes nor their six neighbours are PEC,
// and it holds no source or monitor. kTileDiel: the tile has stub-loaded
// nodes.
// kTileEdge: the tile has a node on an outer y or z face (its stage is
// assembled from runs, see stageRuns).
// kTileNear: the tile has nodes in the near-field box (always with
// kTileGeneral: only the general body completes pulses with residuals).
// kTileStubSparse: at most a quarter of the tile's nodes are stub-loaded
// (with kTileDiel): a staged tile then leaves the three stub segments out of
// its stage and those nodes read their stubs from the stub planes.
enum : uint8_t { kTileGeneral = 1, kTileDiel = 2, kTileEdge = 4, kTileNear = 8, kTileStubSparse = 16 };
// the quarter of kTileStubSparse: stub-loaded nodes x this <= nodes of a tile
constexpr int kStubSparseDiv = 4;

#ifdef TLM_CHECKED
#define TLM_GUARD(idx, limit, code)                                                         \
    (((idx) >= 0 && (idx) < (limit)) ? true : (atomicOr(a.fault, (unsigned)(code)), false))
#else
#define TLM_GUARD(idx, limit, code) true
#endif

// Plane access by node index, for every storage type. Element storage
// (float, double, half, bfloat16) is read and written as aligned vectors of
// V nodes; block floating point (Bfp4) as one word per aligned 4-node group.
// kUnit: the value in storage units (decodeRaw), else scaled by `scale`.
template <class S, int V, bool kUnit = false>
__device__ __forceinline__ void loadVec(const S *__restrict__ base, long long node,
                                        typename Traits<S>::R (&dst)[V], typename Traits<S>::R scale)
{
    if constexpr (std::is_same<S, Bfp4>::value)
    {
        static_assert(V == 4, "block floating point groups hold 4 nodes");
        float v[4];
        bfpDecode(base[node >> 2], v);
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[c] = v[c];
    }
    else
    {
        const Pack<S, V> p = *reinterpret_cast<const Pack<S, V> *>(base + node);
#pragma unroll
        for (int c = 0; c < V; ++c)
        {
            if constexpr (kUnit)
                dst[c] = decodeRaw(p.v[c]);
            else
                dst[c] = decode(p.v[c], scale);
        }
    }
}

template <class S, bool kUnit = false>
__device__ __forceinline__ typename Traits<S>::R loadOne(const S *__restrict__ base, long long node,
                                                         typename Traits<S>::R scale)
{
    if constexpr (std::is_same<S, Bfp4>::value)
        return bfpDecodeOne(base[node >> 2], (int)(node & 3));
    else if constexpr (kUnit)
        return decodeRaw(base[node]);
    else
        return decode(base[node], scale);
}

// Store V nodes of plane slot `salt`; with stochastic rounding the random
// bits are a function of (node, slot, step seed).
template <class S, int V, bool kUnit = false>
__device__ __forceinline__ void storeVec(S *__restrict__ base, long long node,
                                         const typename Traits<S>::R (&src)[V],
                                         typename Traits<S>::R inv, bool stochastic, unsigned seed,
                                         int salt)
{
    if constexpr (kUnit) inv = typename Traits<S>::R(1);
    if constexpr (std::is_same<S, Bfp4>::value)
    {
        static_assert(V == 4, "block floating point groups hold 4 nodes");
        float v[4] = { src[0], src[1], src[2], src[3] };
        base[node >> 2] = bfpEncode(v, stochastic, (unsigned)(node * 12 + salt) ^ seed);
    }
    else
    {
        Pack<S, V> p;
        if (Traits<S>::kScaled && stochastic)
        {
#pragma unroll
            for (int c = 0; c < V; ++c)
                p.v[c] = encodeStochastic<S>(src[c], inv, mix32((unsigned)((node + c) * 12 + salt) ^ seed));
        }
        else if constexpr ((std::is_same<S, __half>::value || std::is_same<S, __nv_bfloat16>::value) && V % 2 == 0)
        {
            // two nodes per conversion instruction (cvt.rn.{f16,bf16}x2.f32),
            // rounding each exactly as encode<S> does
#pragma unroll
            for (int c = 0; c < V; c += 2)
            {
                const float lo = kUnit ? src[c] : src[c] * inv, hi = kUnit ? src[c + 1] : src[c + 1] * inv;
                if constexpr (std::is_same<S, __half>::value)
                    *reinterpret_cast<__half2 *>(&p.v[c]) = __floats2half2_rn(lo, hi);
                else
                    *reinterpret_cast<__nv_bfloat162 *>(&p.v[c]) = __floats2bfloat162_rn(lo, hi);
            }
        }
        else
        {
#pragma unroll
            for (int c = 0; c < V; ++c)
            {
                if constexpr (kUnit)
                    p.v[c] = encodeRaw<S>(src[c]);
                else
                    p.v[c] = encode<S>(src[c], inv);
            }
        }
        *reinterpret_cast<Pack<S, V> *>(base + node) = p;
    }
}

template <int V> __device__ __forceinline__ void loadMat(const uint8_t *__restrict__ m, long long idx,
                                                         uint8_t (&dst)[V])
{
    const Pack<uint8_t, V> p = *reinterpret_cast<const Pack<uint8_t, V> *>(m + idx);
#pragma unroll
    for (int c = 0; c < V; ++c) dst[c] = p.v[c];
}

template <int V> __device__ __forceinline__ unsigned pecMask(const uint8_t (&m)[V])
{
    unsigned r = 0;
#pragma unroll
    for (int c = 0; c < V; ++c) r |= (m[c] == kPec ? 1u : 0u) << c;
    return r;
}

// Shared-memory stage of one tile of kBlock x V nodes (storage S: FP32 with
// V = 2, FP16 or BF16 with V = 4), filled by bulk copies
// (stepKernelStaged): slots 0..3 at the tile's own nodes with 16 bytes of
// halo on each side (the x neighbours), then the eight y/z neighbour
// segments in the order of inc[4..11] (slot 6+t one row below, 4+t one row
// above, 10+t one plane below, 8+t one plane above), the three FP32 stub
// planes, and the material bytes. Offsets in bytes; every segment starts and
// ends on a 16-byte boundary.
template <class S, int V = 2> struct Stage
{
    static constexpr int kNodes = kBlock * V;
    static constexpr int kElem = (int)sizeof(S);
    static constexpr int kHalo = 16 / kElem;                // nodes of x halo on each side
    static constexpr int kSegX = kNodes + 2 * kHalo;        // elements of an x segment
    static constexpr int kOffYZ = 4 * kSegX * kElem;
    static constexpr int kOffStub = kOffYZ + 8 * kNodes * kElem;
    static constexpr int kOffMat = kOffStub + 3 * kNodes * 4;
    static constexpr int kBytes = kOffMat + kNodes;
    static_assert(kBytes % 16 == 0 && (kSegX * kElem) % 16 == 0 && kOffYZ % 16 == 0 && kOffStub % 16 == 0,
                  "bulk copies need 16-byte multiples");
};

constexpr int kStages = 3;
constexpr int kStagedThreads = kBlock + 32;
constexpr unsigned kStageTimeout = 1u << 31;
// A wait polls its mbarrier (test_wait, no suspension: a suspended thread
// measured slower to resume than a polling one) and gives up after about
// kStageWaitNs of the global timer, checked every 256 polls.
constexpr unsigned long long kStageWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned smemAddr(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbarTestWait(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}

__device__ __forceinline__ unsigned long long globalTimerNs()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbarWaitBounded(unsigned bar, unsigned parity,
                                                unsigned long long limitNs = kStageWaitNs)
{
    if (mbarTestWait(bar, parity)) return true;
    if (limitNs == 0) return false;
    const unsigned long long t0 = globalTimerNs();
    for (unsigned it = 1;; ++it)
    {
        if (mbarTestWait(bar, parity)) return true;
        if ((it & 255u) == 0 && globalTimerNs() - t0 > limitNs) return false;
    }
}

// Sparse-stub tiles (kTileStubSparse) skip staging their stubs in FP32 only:
// in the 16-bit staged kernel (4 nodes per thread, 96 registers) the second
// instantiation of the tile body spilled and the 384x384x256 dipole with the
// near-field box stepped in 0.392 ms against 0.347, so there every
// stub-loaded tile stages its stubs.
template <class S> constexpr bool kSparseStubs = std::is_same<S, float>::value;

// The producer's wait for a free stage: the same bounded wait, with a pause
// of about PAUSE_NS between polls, so that a producer waiting on its
// consumers does not take their issue slots with a tight polling loop.
template <unsigned PAUSE_NS>
__device__ __forceinline__ bool mbarWaitPaused(unsigned bar, unsigned parity,
                                               unsigned long long limitNs = kStageWaitNs)
{
    if constexpr (PAUSE_NS == 0)
        return mbarWaitBounded(bar, parity, limitNs);
    else
    {
        if (mbarTestWait(bar, parity)) return true;
        if (limitNs == 0) return false;
        const unsigned long long t0 = globalTimerNs();
        for (unsigned it = 1;; ++it)
        {
            __nanosleep(PAUSE_NS);
            if (mbarTestWait(bar, parity)) return true;
            if ((it & 15u) == 0 && globalTimerNs() - t0 > limitNs) return false;
        }
    }
}
// FP32 single grid: 512 ns (192^3 heterogeneous 127.9 -> 126.7 us per step;
// 32 polls before the first pause measured 128.0 us); the 16-bit and batch
// producers poll without a pause (with 512 ns the 384x384x256 dipole in
// FP16 stepped 5 % slower).
constexpr unsigned kProducerPauseNs = 512;

__device__ __forceinline__ void bulkCopy(unsigned dst, const void *src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :
                 : "r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Interior tile (see kTileGeneral): the gather needs no PEC handling, so
// every pulse load is issued before any material is read. On the outer faces
// the load of the neighbour's pulse becomes a load of the own pulse, scaled
// by rho afterwards (y/z faces: per thread; x faces, the first and last node
// of a row, and the row padding: fixed up per node). Pairs of nodes scatter
// with packed FP32x2 arithmetic. The results are bitwise those of the
// general tile body below. kStaged: the tile's inputs are already in the
// shared-memory stage `sm` (see Stage and stageRuns; V = 2), outer y/z faces
// included; the arithmetic is the same.
// kSparse (kStaged only): a kTileStubSparse tile, whose stage holds no
// stubs; its stub-loaded nodes load theirs from a.stub first thing (a
// separate instantiation, so the other tiles keep the code they had).
template <class S, int V, bool kStaged = false, bool kSparse = false, bool kZeroSkip = true>
__device__ __forceinline__ void stepTileInterior(const StepArgs<S> &a, int tile, double *red, bool diel,
                                                 const unsigned char *sm = nullptr, unsigned eBar = 0,
                                                 unsigned eParity = 0)
{
    using R = float;
    static_assert(V % 2 == 0, "interior tiles scatter node pairs");
    const int lane = threadIdx.x & 31;
    const unsigned q = (unsigned)tile * kBlock + threadIdx.x;  // every thread of the tile is live
    const unsigned rowu = fastDiv(q, a.div_nq);
    const int x0 = (int)(q - rowu * (unsigned)a.nq) * V;
    const unsigned ku = fastDiv(rowu, a.div_ny);
    const int j = (int)(rowu - ku * (unsigned)a.ny);
    const int k = (int)ku;
    const long long node0 = (long long)q * V;
    const long long P = a.P;
    const long long sy = a.px, sz = (long long)a.px * a.ny;
    const bool atYlo = j == 0, atYhi = j == a.ny - 1, atZlo = k == 0, atZhi = k == a.nz - 1;

    // ---- stub-loaded nodes of a sparse staged tile: their stubs come from
    // the stub planes, loaded first so that the loads overlap the rest ----
    static_assert(kStaged || !kSparse, "sparse-stub tiles are staged tiles");
    uint8_t mS[V];
    unsigned dielS = 0;
    R vsS[3][V];
    if constexpr (kSparse)
    {
#pragma unroll
        for (int c = 0; c < V; ++c) mS[c] = sm[Stage<S, V>::kOffMat + threadIdx.x * V + c];
#pragma unroll
        for (int c = 0; c < V; ++c) dielS |= ((mS[c] >= kDiel0) ? 1u : 0u) << c;
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
        {
#pragma unroll
            for (int c = 0; c < V; ++c) vsS[jj][c] = R(0);
        }
        if (dielS)
        {
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
            {
                const Pack<R, V> p = *reinterpret_cast<const Pack<R, V> *>(a.stub + jj * P + node0);
#pragma unroll
                for (int c = 0; c < V; ++c) vsS[jj][c] = p.v[c];
            }
        }
    }

    // ---- loads: own x-slots, then the y and z neighbours' opposite faces ----
    R ox[4][V];
    R inc[12][V];
    R prevX[2], nextX[2];
    if constexpr (kStaged)
    {
        static_assert((V == 2 || V == 4) && (std::is_same<S, float>::value || std::is_same<S, __half>::value ||
                                             std::is_same<S, __nv_bfloat16>::value),
                      "staged tiles hold 2 or 4 nodes per thread of FP32, FP16 or BF16");
        using L = Stage<S, V>;
        const S *X = reinterpret_cast<const S *>(sm);
        const S *YZ = reinterpret_cast<const S *>(sm + L::kOffYZ);
        const int l = threadIdx.x * V;
#pragma unroll
        for (int s = 0; s < 4; ++s) loadVec<S, V, true>(X + s * L::kSegX + L::kHalo, l, ox[s], a.scale);
#pragma unroll
        for (int g = 0; g < 8; ++g) loadVec<S, V, true>(YZ + g * L::kNodes, l, inc[4 + g], a.scale);
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
            prevX[t] = loadOne<S, true>(X + (2 + t) * L::kSegX + L::kHalo, l - 1, a.scale);
            nextX[t] = loadOne<S, true>(X + t * L::kSegX + L::kHalo, l + V, a.scale);
        }
        (void)lane;
    }
    else
    {
#pragma unroll
        for (int s = 0; s < 4; ++s) loadVec<S, V, true>(a.in, s * P + node0, ox[s], a.scale);
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
            // -y face: (y,+) of the row below; +y face: (y,-) of the row above;
            // on an outer face the own pulse of the face instead
            loadVec<S, V, true>(a.in, atYlo ? (4 + t) * P + node0 : (6 + t) * P + node0 - sy, inc[4 + t], a.scale);
            loadVec<S, V, true>(a.in, atYhi ? (6 + t) * P + node0 : (4 + t) * P + node0 + sy, inc[6 + t], a.scale);
            loadVec<S, V, true>(a.in, atZlo ? (8 + t) * P + node0 : (10 + t) * P + node0 - sz, inc[8 + t], a.scale);
            loadVec<S, V, true>(a.in, atZhi ? (10 + t) * P + node0 : (8 + t) * P + node0 + sz, inc[10 + t], a.scale);
        }
        // ---- x neighbours: own vector, adjacent lane, or (warp edge) a scalar load ----
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
            prevX[t] = __shfl_up_sync(0xffffffffu, ox[2 + t][V - 1], 1);
            nextX[t] = __shfl_down_sync(0xffffffffu, ox[t][0], 1);
        }
        if (lane == 0 && x0 > 0)
        {
#pragma unroll
            for (int t = 0; t < 2; ++t) prevX[t] = loadOne<S, true>(a.in, (2 + t) * P + node0 - 1, a.scale);
        }
        if (lane == 31 && x0 + V <= a.nx - 1)
        {
#pragma unroll
            for (int t = 0; t < 2; ++t) nextX[t] = loadOne<S, true>(a.in, t * P + node0 + V, a.scale);
        }
    }
#pragma unroll
    for (int t = 0; t < 2; ++t)
    {
#pragma unroll
        for (int c = 0; c < V; ++c)
        {
            inc[t][c] = (c > 0) ? ox[2 + t][c > 0 ? c - 1 : 0] : prevX[t];          // -x face
            inc[2 + t][c] = (c < V - 1) ? ox[t][c < V - 1 ? c + 1 : 0] : nextX[t];  // +x face
        }
    }
    // outer faces: rho times the own reflected pulse
    if (atYlo | atYhi | atZlo | atZhi)
    {
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
#pragma unroll
            for (int c = 0; c < V; ++c)
            {
                if (atYlo) inc[4 + t][c] = a.rho * inc[4 + t][c];
                if (atYhi) inc[6 + t][c] = a.rho * inc[6 + t][c];
                if (atZlo) inc[8 + t][c] = a.rho * inc[8 + t][c];
                if (atZhi) inc[10 + t][c] = a.rho * inc[10 + t][c];
            }
        }
    }
    if (x0 == 0)
    {
#pragma unroll
        for (int t = 0; t < 2; ++t) inc[t][0] = a.rho * ox[t][0];
    }
    const int cHi = a.nx - 1 - x0;  // the node at x = nx-1, if this thread holds it
    if (cHi < V)
    {
#pragma unroll
        for (int c = 0; c < V; ++c)
            if (c == cHi)
            {
#pragma unroll
                for (int t = 0; t < 2; ++t) inc[2 + t][c] = a.rho * ox[2 + t][c];
            }
    }
    const unsigned liveMask = cHi >= V - 1 ? (1u << V) - 1 : (cHi < 0 ? 0u : (1u << (cHi + 1)) - 1);

    // ---- energy: sum of squares of the incident link pulses, FP64 ----
    if (a.epart != nullptr)
    {
        double e = 0.0;
#pragma unroll
        for (int c = 0; c < V; ++c)
        {
            if (((liveMask >> c) & 1u) && node0 + c >= a.e_lo && node0 + c < a.e_hi)
            {
#pragma unroll
                for (int s = 0; s < 12; ++s) e += (double)inc[s][c] * (double)inc[s][c];
            }
        }
        if constexpr (kStaged)
        {
            // the same per-warp sums in the same order as blockSumDouble, but
            // gathered through the mbarrier eBar so that no warp waits for
            // the others (only thread 0 does, bounded)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
            if (lane == 0)
            {
                red[threadIdx.x >> 5] = e;
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(eBar) : "memory");
            }
            if (threadIdx.x == 0)
            {
                if (mbarWaitBounded(eBar, eParity))
                {
                    double tot = 0.0;
                    for (int w = 0; w < kBlock / 32; ++w) tot += red[w];
                    a.epart[tile] = tot * ((double)a.scale * (double)a.scale);
                }
                else if (a.fault)
                    atomicOr(a.fault, kStageTimeout);
            }
        }
        else
        {
            const double tot = blockSumDouble(e, red);
            if (threadIdx.x == 0) a.epart[tile] = tot * ((double)a.scale * (double)a.scale);
        }
    }

    // ---- scatter (pairs of nodes) and store ----
    uint8_t m[V];
    unsigned dielMask = 0;
    if constexpr (kSparse)
    {
#pragma unroll
        for (int c = 0; c < V; ++c) m[c] = mS[c];
        dielMask = dielS & liveMask;
    }
    else if (diel)
    {
        if constexpr (kStaged)
        {
#pragma unroll
            for (int c = 0; c < V; ++c) m[c] = sm[Stage<S, V>::kOffMat + threadIdx.x * V + c];
        }
        else
            loadMat<V>(a.mat, node0, m);
#pragma unroll
        for (int c = 0; c < V; ++c) dielMask |= ((m[c] >= kDiel0) ? 1u : 0u) << c;
        dielMask &= liveMask;
    }
    R vs[3][V];
#pragma unroll
    for (int jj = 0; jj < 3; ++jj)
    {
#pragma unroll
        for (int c = 0; c < V; ++c) vs[jj][c] = kSparse ? vsS[jj][c] : R(0);
    }
    if (!kSparse && dielMask)
    {
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
        {
            Pack<R, V> p;
            if constexpr (kStaged)
                p = *reinterpret_cast<const Pack<R, V> *>(reinterpret_cast<const float *>(sm + Stage<S, V>::kOffStub) +
                                                          jj * Stage<S, V>::kNodes + threadIdx.x * V);
            else
                p = *reinterpret_cast<const Pack<R, V> *>(a.stub + jj * P + node0);
#pragma unroll
            for (int c = 0; c < V; ++c) vs[jj][c] = p.v[c];
        }
    }
    R outv[12][V];
    const float2 z = splat2(a.neg_zero);
#pragma unroll
    for (int pr = 0; pr < V / 2; ++pr)
    {
        const int c0 = 2 * pr, c1 = 2 * pr + 1;
        const unsigned pm = (dielMask >> c0) & 3u;
        if (pm == 0u)
        {
            float2 in2[12], o2[12];
#pragma unroll
            for (int s = 0; s < 12; ++s) in2[s] = make_float2(inc[s][c0], inc[s][c1]);
            scatterAir2(in2, o2, z);
#pragma unroll
            for (int s = 0; s < 12; ++s)
            {
                outv[s][c0] = o2[s].x;
                outv[s][c1] = o2[s].y;
            }
        }
        else if (pm == 3u)
        {
            float2 in2[12], o2[12], v2[3];
#pragma unroll
            for (int s = 0; s < 12; ++s) in2[s] = make_float2(inc[s][c0], inc[s][c1]);
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) v2[jj] = make_float2(vs[jj][c0], vs[jj][c1]);
            const int id0 = m[c0] - kDiel0, id1 = m[c1] - kDiel0;
            scatterStub2<kZeroSkip>(in2, v2, make_float2(a.yhat[id0], a.yhat[id1]),
                                    make_float2(a.ghat[id0], a.ghat[id1]), o2, z);
#pragma unroll
            for (int s = 0; s < 12; ++s)
            {
                outv[s][c0] = o2[s].x;
                outv[s][c1] = o2[s].y;
            }
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
            {
                vs[jj][c0] = v2[jj].x;
                vs[jj][c1] = v2[jj].y;
            }
        }
        else
        {
            // one air and one stub-loaded node: scalar scatter of each
#pragma unroll
            for (int c = c0; c <= c1; ++c)
            {
                R in1[12], o1[12];
#pragma unroll
                for (int s = 0; s < 12; ++s) in1[s] = inc[s][c];
                if ((dielMask >> c) & 1u)
                {
                    const int id = m[c] - kDiel0;
                    R v3[3] = { vs[0][c], vs[1][c], vs[2][c] };
                    scatterStub(in1, v3, a.yhat[id], a.ghat[id], o1);
                    vs[0][c] = v3[0];
                    vs[1][c] = v3[1];
                    vs[2][c] = v3[2];
                }
                else
                    scatterAir(in1, o1);
#pragma unroll
                for (int s = 0; s < 12; ++s) outv[s][c] = o1[s];
            }
        }
    }
    if (liveMask != (1u << V) - 1)
    {
        // row padding (and nothing else) is not live: its pulses stay zero
#pragma unroll
        for (int c = 0; c < V; ++c)
            if (!((liveMask >> c) & 1u))
            {
#pragma unroll
                for (int s = 0; s < 12; ++s) outv[s][c] = R(0);
            }
    }
#pragma unroll
    for (int s = 0; s < 12; ++s)
        storeVec<S, V, true>(a.out, s * P + node0, outv[s], a.inv_scale, a.stochastic != 0, a.round_seed, s);
    if (dielMask)
    {
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
        {
            Pack<R, V> p;
#pragma unroll
            for (int c = 0; c < V; ++c) p.v[c] = vs[jj][c];
            *reinterpret_cast<Pack<R, V> *>(a.stub + jj * P + node0) = p;
        }
    }
}

// One tile of kBlock threads x V nodes: tile `tile` covers the V-node
// groups [tile*kBlock, (tile+1)*kBlock). `red` is kBlock/32 doubles of
// shared memory. kIncident: the input planes hold INCIDENT pulses (state
// written by tlm_set_pulses) instead of reflected ones; the gather is
// skipped.
template <class S, int V, bool kIncident, bool kSelect = true>
__device__ __forceinline__ void stepTile(const StepArgs<S> &a, int tile, double *red)
{
    using R = typename Traits<S>::R;
    if constexpr (!kIncident && std::is_same<R, float>::value && V % 2 == 0)
    {
        if (a.tile_flags != nullptr)
        {
            const uint8_t f = a.tile_flags[tile];
            if (!(f & kTileGeneral))
            {
                stepTileInterior<S, V>(a, tile, red, (f & kTileDiel) != 0);
                return;
            }
        }
    }

    const int lane = threadIdx.x & 31;
    const long long q = (long long)tile * kBlock + threadIdx.x;
    const bool live = q < a.nquads;
    const long long qq = live ? q : 0;
    const unsigned rowu = fastDiv((unsigned)qq, a.div_nq);
    const int xq = (int)((unsigned)qq - rowu * (unsigned)a.nq);
    const unsigned ku = fastDiv(rowu, a.div_ny);
    const int j = (int)(rowu - ku * (unsigned)a.ny);
    const int k = (int)ku;
    const int x0 = xq * V;
    const long long node0 = qq * V;
    const long long P = a.P;
    const long long sy = a.px, sz = (long long)a.px * a.ny;

    // near-field box (16-bit storage): residuals complete the decoded pulses
    // of box nodes, exactly (block-uniform: the tile's flag)
    constexpr bool kNearType = Traits<S>::kScaled;
    bool near = false;
    if constexpr (kNearType)
        near = a.near.lo_in != nullptr && a.tile_flags != nullptr && (a.tile_flags[tile] & kTileNear) != 0;
    // slot s of the V nodes x0.. of row (jj, kk)
    auto addLo = [&](R(&v)[V], int s, int jj, int kk) {
        if constexpr (kNearType)
        {
            if (near && live)
            {
#pragma unroll
                for (int c = 0; c < V; ++c)
                {
                    const long long b = a.near.at(x0 + c, jj, kk);
                    if (b >= 0) v[c] += a.near.lo_in[s * a.near.bP + b];
                }
            }
        }
    };
    // slot s of node (ii, jj, kk)
    auto addLo1 = [&](R &v, int s, int ii, int jj, int kk) {
        if constexpr (kNearType)
        {
            if (near && live)
            {
                const long long b = a.near.at(ii, jj, kk);
                if (b >= 0) v += a.near.lo_in[s * a.near.bP + b];
            }
        }
    };

    uint8_t m[V];
    if (live && TLM_GUARD(node0, P - V + 1, 1))
        loadMat<V>(a.mat, node0, m);
    else
    {
#pragma unroll
        for (int c = 0; c < V; ++c) m[c] = kPec;
    }

    R inc[12][V];
    unsigned nodeLive = 0;  // bit c: node x0+c is inside the grid and not PEC
#pragma unroll
    for (int c = 0; c < V; ++c)
        nodeLive |= ((live && x0 + c < a.nx && m[c] != kPec) ? 1u : 0u) << c;

    if (kIncident)
    {
#pragma unroll
        for (int s = 0; s < 12; ++s)
        {
            if (live && TLM_GUARD(s * P + node0, 12 * P - V + 1, 2))
                loadVec<S, V, true>(a.in, s * P + node0, inc[s], a.scale);
            else
            {
#pragma unroll
                for (int c = 0; c < V; ++c) inc[s][c] = R(0);
            }
            addLo(inc[s], s, j, k);
        }
    }
    else
    {
        // ---- neighbour materials (PEC masks per direction) ----
        uint8_t mn[V];
        unsigned pecYm = 0, pecYp = 0, pecZm = 0, pecZp = 0;
        if (live && j > 0 && TLM_GUARD(node0 - sy, P - V + 1, 3))
        {
            loadMat<V>(a.mat, node0 - sy, mn);
            pecYm = pecMask<V>(mn);
        }
        if (live && j < a.ny - 1 && TLM_GUARD(node0 + sy, P - V + 1, 3))
        {
            loadMat<V>(a.mat, node0 + sy, mn);
            pecYp = pecMask<V>(mn);
        }
        if (live && k > 0 && TLM_GUARD(node0 - sz, P - V + 1, 3))
        {
            loadMat<V>(a.mat, node0 - sz, mn);
            pecZm = pecMask<V>(mn);
        }
        if (live && k < a.nz - 1 && TLM_GUARD(node0 + sz, P - V + 1, 3))
        {
            loadMat<V>(a.mat, node0 + sz, mn);
            pecZp = pecMask<V>(mn);
        }
        const unsigned pecOwn = pecMask<V>(m);
        // x neighbours: inside the vector, else the adjacent lane's vector,
        // else (warp edge) one scalar load.
        unsigned prevPec = __shfl_up_sync(0xffffffffu, (pecOwn >> (V - 1)) & 1u, 1);
        unsigned nextPec = __shfl_down_sync(0xffffffffu, pecOwn & 1u, 1);
        const bool needPrev = live && x0 > 0;
        const bool needNext = live && x0 + V <= a.nx - 1;
        if (lane == 0 && needPrev && TLM_GUARD(node0 - 1, P, 4))
            prevPec = a.mat[node0 - 1] == kPec;
        if (lane == 31 && needNext && TLM_GUARD(node0 + V, P, 4))
            nextPec = a.mat[node0 + V] == kPec;
        const unsigned pecXm = ((pecOwn << 1) | (prevPec & 1u)) & ((1u << V) - 1);
        const unsigned pecXp = (pecOwn >> 1) | ((nextPec & 1u) << (V - 1));

        // ---- x axis: own vectors of slots 0..3 ----
        R ox[4][V];
#pragma unroll
        for (int s = 0; s < 4; ++s)
        {
            if (live && TLM_GUARD(s * P + node0, 12 * P - V + 1, 5))
                loadVec<S, V, true>(a.in, s * P + node0, ox[s], a.scale);
            else
            {
#pragma unroll
                for (int c = 0; c < V; ++c) ox[s][c] = R(0);
            }
            addLo(ox[s], s, j, k);  // before the lane shuffles below hand them on
        }
        R prevX[2], nextX[2];
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
            prevX[t] = __shfl_up_sync(0xffffffffu, ox[2 + t][V - 1], 1);
            nextX[t] = __shfl_down_sync(0xffffffffu, ox[t][0], 1);
        }
        if (lane == 0 && needPrev)
        {
#pragma unroll
            for (int t = 0; t < 2; ++t)
                if (TLM_GUARD((2 + t) * P + node0 - 1, 12 * P, 6))
                {
                    prevX[t] = loadOne<S, true>(a.in, (2 + t) * P + node0 - 1, a.scale);
                    addLo1(prevX[t], 2 + t, x0 - 1, j, k);
                }
        }
        if (lane == 31 && needNext)
        {
#pragma unroll
            for (int t = 0; t < 2; ++t)
                if (TLM_GUARD(t * P + node0 + V, 12 * P, 6))
                {
                    nextX[t] = loadOne<S, true>(a.in, t * P + node0 + V, a.scale);
                    addLo1(nextX[t], t, x0 + V, j, k);
                }
        }
#pragma unroll
        for (int c = 0; c < V; ++c)
        {
            const int x = x0 + c;
#pragma unroll
            for (int t = 0; t < 2; ++t)
            {
                // face -x: neighbour's +x reflected pulse (slot 2+t)
                R from = (c > 0) ? ox[2 + t][c > 0 ? c - 1 : 0] : prevX[t];
                R lo = (x == 0) ? a.rho * ox[t][c] : (((pecXm >> c) & 1u) ? -ox[t][c] : from);
                // face +x: neighbour's -x reflected pulse (slot t)
                R fromH = (c < V - 1) ? ox[t][c < V - 1 ? c + 1 : 0] : nextX[t];
                R hi = (x == a.nx - 1) ? a.rho * ox[2 + t][c]
                                       : (((pecXp >> c) & 1u) ? -ox[2 + t][c] : fromH);
                inc[t][c] = lo;
                inc[2 + t][c] = hi;
            }
        }

        // ---- y and z axes ----
        // face -a of node c reads slot (a,+,t) of the node one row/plane
        // below; face +a reads slot (a,-,t) one row/plane above. On the outer
        // face the own reflected pulse is loaded instead and scaled by rho;
        // next to a PEC node the own pulse is loaded as well and negated.
#pragma unroll
        for (int ax = 1; ax < 3; ++ax)
        {
            const long long st = ax == 1 ? sy : sz;
            const bool atLo = ax == 1 ? (j == 0) : (k == 0);
            const bool atHi = ax == 1 ? (j == a.ny - 1) : (k == a.nz - 1);
            const unsigned pm = ax == 1 ? pecYm : pecZm;
            const unsigned pp = ax == 1 ? pecYp : pecZp;
#pragma unroll
            for (int t = 0; t < 2; ++t)
            {
                const int sLo = ax * 4 + t;      // face -a
                const int sHi = ax * 4 + 2 + t;  // face +a
                R vLo[V], vHi[V];
                // -a face
                {
                    const long long idx = atLo ? sLo * P + node0 : sHi * P + node0 - st;
                    if (live && TLM_GUARD(idx, 12 * P - V + 1, 7))
                        loadVec<S, V, true>(a.in, idx, vLo, a.scale);
                    else
                    {
#pragma unroll
                        for (int c = 0; c < V; ++c) vLo[c] = R(0);
                    }
                    if (atLo)
                        addLo(vLo, sLo, j, k);
                    else
                        addLo(vLo, sHi, ax == 1 ? j - 1 : j, ax == 2 ? k - 1 : k);
                    if (atLo)
                    {
#pragma unroll
                        for (int c = 0; c < V; ++c) vLo[c] = a.rho * vLo[c];
                    }
                    else if (pm & nodeLive)
                    {
                        R own[V];
                        if (TLM_GUARD(sLo * P + node0, 12 * P - V + 1, 8))
                            loadVec<S, V, true>(a.in, sLo * P + node0, own, a.scale);
                        addLo(own, sLo, j, k);
#pragma unroll
                        for (int c = 0; c < V; ++c)
                            if ((pm >> c) & 1u) vLo[c] = -own[c];
                    }
                }
                // +a face
                {
                    const long long idx = atHi ? sHi * P + node0 : sLo * P + node0 + st;
                    if (live && TLM_GUARD(idx, 12 * P - V + 1, 9))
                        loadVec<S, V, true>(a.in, idx, vHi, a.scale);
                    else
                    {
#pragma unroll
                        for (int c = 0; c < V; ++c) vHi[c] = R(0);
                    }
                    if (atHi)
                        addLo(vHi, sHi, j, k);
                    else
                        addLo(vHi, sLo, ax == 1 ? j + 1 : j, ax == 2 ? k + 1 : k);
                    if (atHi)
                    {
#pragma unroll
                        for (int c = 0; c < V; ++c) vHi[c] = a.rho * vHi[c];
                    }
                    else if (pp & nodeLive)
                    {
                        R own[V];
                        if (TLM_GUARD(sHi * P + node0, 12 * P - V + 1, 10))
                            loadVec<S, V, true>(a.in, sHi * P + node0, own, a.scale);
                        addLo(own, sHi, j, k);
#pragma unroll
                        for (int c = 0; c < V; ++c)
                            if ((pp >> c) & 1u) vHi[c] = -own[c];
                    }
                }
#pragma unroll
                for (int c = 0; c < V; ++c)
                {
                    inc[sLo][c] = vLo[c];
                    inc[sHi][c] = vHi[c];
                }
            }
        }
    }

    // ---- sources and monitor samples (rare: only blocks that hold one) ----
    if (a.tile_begin != nullptr)
    {
        const int b0 = a.tile_begin[tile], b1 = a.tile_begin[tile + 1];
        if (b0 < b1 && live)
        {
            int lo = b0, hi = b1;
            while (lo < hi)
            {
                const int mid = (lo + hi) >> 1;
                if (a.spec[mid].node < node0) lo = mid + 1; else hi = mid;
            }
            for (int e = lo; e < b1; ++e)
            {
                const SpecEntry se = a.spec[e];
                if (se.node >= node0 + V) break;
                const int c = (int)(se.node - node0);
                if (se.kind == kInject)
                {
                    // q = (0.5*amp)*sv onto the 4 links carrying E_pol
                    const R qv = (R(0.5) * R(se.amp)) * a.sv;
                    const int pol = se.arg;
#pragma unroll
                    for (int s = 0; s < 12; ++s)
                    {
                        if ((s >> 2) != pol && fieldOfSlot(s) == pol)
                        {
#pragma unroll
                            for (int cc = 0; cc < V; ++cc)
                                if (cc == c) inc[s][cc] = inc[s][cc] + qv;
                        }
                    }
                }
                else
                {
                    // A PEC node's pulses are identically zero in the
                    // reference (never scattered, never connected), so its
                    // samples are zero; the gathered values are discarded.
                    const bool on = (nodeLive >> c) & 1u;
                    R v[12];
#pragma unroll
                    for (int s = 0; s < 12; ++s)
                    {
                        v[s] = inc[s][0];
#pragma unroll
                        for (int cc = 1; cc < V; ++cc)
                            if (cc == c) v[s] = inc[s][cc];
                        v[s] = on ? v[s] : R(0);
                    }
                    R *dst = a.samples + (long long)se.arg * 6;
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) dst[jj] = nodeVoltage(v, jj) * a.scale;
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) dst[3 + kk] = circulation(v, kk) * a.scale;
                }
            }
        }
    }

    // ---- energy: sum of squares of the incident link pulses, FP64 ----
    if (a.epart != nullptr)
    {
        double e = 0.0;
#pragma unroll
        for (int c = 0; c < V; ++c)
        {
            if (((nodeLive >> c) & 1u) && node0 + c >= a.e_lo && node0 + c < a.e_hi)
            {
#pragma unroll
                for (int s = 0; s < 12; ++s) e += (double)inc[s][c] * (double)inc[s][c];
            }
        }
        const double tot = blockSumDouble(e, red);
        if (threadIdx.x == 0) a.epart[tile] = tot * ((double)a.scale * (double)a.scale);
    }

    // ---- scatter and store ----
    R outv[12][V];
    R vs[3][V];
#pragma unroll
    for (int jj = 0; jj < 3; ++jj)
    {
#pragma unroll
        for (int c = 0; c < V; ++c) vs[jj][c] = R(0);
    }
    const bool anyDiel = a.stub != nullptr && live;
    unsigned dielMask = 0;
#pragma unroll
    for (int c = 0; c < V; ++c) dielMask |= ((m[c] >= kDiel0) ? 1u : 0u) << c;
    dielMask &= nodeLive;
    // Warp-uniform choice of scatter: all-air warps take the air scatter;
    // a warp holding any dielectric node takes one branch-free path in
    // which air nodes still use the air formula (selected, not diverged).
    const bool warpDiel = kSelect ? __any_sync(0xffffffffu, anyDiel && dielMask != 0) : false;
    if (anyDiel && dielMask)
    {
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
        {
            if (TLM_GUARD(jj * P + node0, 3 * P - V + 1, 11))
            {
                const Pack<R, V> p = *reinterpret_cast<const Pack<R, V> *>(a.stub + jj * P + node0);
#pragma unroll
                for (int c = 0; c < V; ++c) vs[jj][c] = p.v[c];
            }
        }
    }
    const bool allOn = nodeLive == ((1u << V) - 1);
#pragma unroll
    for (int c = 0; c < V; ++c)
    {
        R in1[12], o1[12];
#pragma unroll
        for (int s = 0; s < 12; ++s) in1[s] = inc[s][c];
        if (!kSelect && ((dielMask >> c) & 1u))
        {
            // per-node branch: stub formula only where the node is dielectric
            const int id = m[c] - kDiel0;
            R v3[3] = { vs[0][c], vs[1][c], vs[2][c] };
            scatterStub(in1, v3, a.yhat[id], a.ghat[id], o1);
            vs[0][c] = v3[0];
            vs[1][c] = v3[1];
            vs[2][c] = v3[2];
        }
        else if (kSelect && warpDiel)
        {
            const bool isD = (dielMask >> c) & 1u;
            const int id = isD ? m[c] - kDiel0 : 0;
            const R yh = isD ? a.yhat[id] : R(0);
            const R gh = isD ? a.ghat[id] : R(0);
            R v3[3] = { vs[0][c], vs[1][c], vs[2][c] };
            scatterSelect(in1, v3, yh, gh, isD, o1);
            vs[0][c] = v3[0];
            vs[1][c] = v3[1];
            vs[2][c] = v3[2];
        }
        else
            scatterAir(in1, o1);
        const bool on = (nodeLive >> c) & 1u;
#pragma unroll
        for (int s = 0; s < 12; ++s) outv[s][c] = (allOn || on) ? o1[s] : R(0);
    }
    if (live)
    {
#pragma unroll
        for (int s = 0; s < 12; ++s)
        {
            if (TLM_GUARD(s * P + node0, 12 * P - V + 1, 12))
            {
                // box nodes round to nearest: their residual completes that value
                storeVec<S, V, true>(a.out, s * P + node0, outv[s], a.inv_scale, a.stochastic != 0 && !near,
                               a.round_seed, s);
            }
        }
        if constexpr (kNearType)
        {
            if (near)
            {
#pragma unroll
                for (int c = 0; c < V; ++c)
                {
                    const long long b = a.near.at(x0 + c, j, k);
                    if (b < 0) continue;
#pragma unroll
                    for (int s = 0; s < 12; ++s)
                        a.near.lo_out[s * a.near.bP + b] =
                            outv[s][c] - decodeRaw(encodeRaw<S>(outv[s][c]));
                }
            }
        }
        if (anyDiel && dielMask)
        {
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
            {
                if (TLM_GUARD(jj * P + node0, 3 * P - V + 1, 13))
                {
                    Pack<R, V> p;
#pragma unroll
                    for (int c = 0; c < V; ++c) p.v[c] = vs[jj][c];
                    *reinterpret_cast<Pack<R, V> *>(a.stub + jj * P + node0) = p;
                }
            }
        }
    }
}

// Default tile shape of each storage type (Traits<S>::V nodes per thread,
// Traits<S>::kMinBlocks resident blocks per SM).
template <class S, bool kIncident>
__global__ void __launch_bounds__(kBlock, Traits<S>::kMinBlocks) stepKernel(const StepArgs<S> a)
{
    __shared__ double red[kBlock / 32];
    stepTile<S, Traits<S>::V, kIncident, Traits<S>::kSelect>(a, blockIdx.x, red);
}

// Other tile shapes, chosen by tlm_config.kernel_variant or the autotuner:
// V nodes per thread, register budget for at least MINB blocks per SM.
template <class S, int V, int MINB, bool kIncident, bool kSelect>
__global__ void __launch_bounds__(kBlock, MINB) stepKernelShaped(const StepArgs<S> a)
{
    __shared__ double red[kBlock / 32];
    stepTile<S, V, kIncident, kSelect>(a, blockIdx.x, red);
}

// Step kernel over a list of tiles (the tiles that the staged kernel below
// does not take), one tile per block.
template <class S, int V, int MINB, bool kSelect>
__global__ void __launch_bounds__(kBlock, MINB) stepKernelList(const StepArgs<S> a, const int *__restrict__ tiles)
{
    __shared__ double red[kBlock / 32];
    stepTile<S, V, false, kSelect>(a, tiles[blockIdx.x], red);
}

// ---- staged interior tiles (FP32, FP16, BF16) ------------------------------
// Interior tiles without a node on an outer y or z face, each staged in shared
// memory by bulk copies (the tensor-memory-access engine) before the interior
// body runs on it. A block of kBlock consumer threads and one producer warp
// owns every gridDim.x-th tile of the list and keeps kStages tiles in
// flight: the producer refills a stage as soon as every consumer warp has
// released it (mbarrier `empty`), the consumers start a tile as soon as its
// bytes are in (mbarrier `full`), and the energy sum of a tile gathers the
// warps' shares through a third mbarrier (`ered`) that only thread 0 waits
// on, so no warp waits for another. Every wait is bounded: one that runs out
// sets kStageTimeout in *a.fault and ends its thread; the producer first lets
// the copies it issued land (again bounded), and the host reports the error.
// Where the bulk copies of a staged tile read from: the input planes, stubs
// and material map of one grid and the extents its segment runs need.
template <class S> struct StageSrc
{
    const S *in;
    const float *stub;   // nullptr without dielectrics
    const uint8_t *mat;
    long long P;
    int px, ny, nz;
    FastDiv div_nq, div_ny;
};

template <class S> __device__ __forceinline__ StageSrc<S> stageSrcOf(const StepArgs<S> &a)
{
    StageSrc<S> r;
    r.in = a.in;
    r.stub = a.stub;
    r.mat = a.mat;
    r.P = a.P;
    r.px = a.px;
    r.ny = a.ny;
    r.nz = a.nz;
    r.div_nq = a.div_nq;
    r.div_ny = a.div_ny;
    return r;
}

// A staged tile list entry: the tile index in bits 0-23 (a grid has fewer
// than 2^23 tiles, since its V-node groups number below 2^31) and the tile's
// flags in bits 24-31, so that the producer needs no second load per tile.
constexpr int kEntryTileBits = 24;
__host__ __device__ __forceinline__ int packStagedEntry(int tile, unsigned flags)
{
    return (int)((unsigned)tile | (flags << kEntryTileBits));
}
__host__ __device__ __forceinline__ int entryTile(int e) { return e & ((1 << kEntryTileBits) - 1); }
__host__ __device__ __forceinline__ unsigned entryFlags(int e) { return (unsigned)e >> kEntryTileBits; }

// The pieces of stage segment g (inc[4 + g]) for the tile at node0, as
// (tile offset, nodes, source element) runs: a node on the segment's outer
// face takes its own pulse of that face (the body scales it by rho), every
// other node its neighbour's opposite pulse; runs that continue each other
// in both places are merged, so a tile away from the outer faces has one run
// per segment. Rows (y) and planes (z) hold multiples of 8 nodes, so every
// run starts and ends on a 16-byte boundary.
template <class S, int V, class F>
__device__ __forceinline__ void stageRuns(const StageSrc<S> &a, long long node0, int g, F &&emit)
{
    const bool zAxis = g >= 4, hi = ((g >> 1) & 1) != 0;
    const int t = g & 1;
    const long long P = a.P, sy = a.px, sz = (long long)a.px * a.ny;
    const int faceSlot = (zAxis ? 8 : 4) + (hi ? 2 : 0) + t;
    const int nbSlot = (zAxis ? 8 : 4) + (hi ? 0 : 2) + t;
    const long long shift = zAxis ? (hi ? sz : -sz) : (hi ? sy : -sy);
    const long long end = node0 + Stage<S, V>::kNodes;
    // row and plane of the first node (two multiply-high divisions), then
    // rows (y) or planes (z) one after the other
    const unsigned row0 = fastDiv((unsigned)(node0 / V), a.div_nq);
    const unsigned k0 = fastDiv(row0, a.div_ny);
    long long row = row0;
    int j = (int)(row0 - k0 * (unsigned)a.ny), k = (int)k0;
    long long rOff = -1, rLen = 0, rSrc = 0;
    for (long long n = node0; n < end;)
    {
        long long pieceEnd;
        bool face;
        if (zAxis)
        {
            pieceEnd = min((long long)(k + 1) * sz, end);
            face = hi ? (k == a.nz - 1) : (k == 0);
            ++k;
        }
        else
        {
            pieceEnd = min((row + 1) * sy, end);
            face = hi ? (j == a.ny - 1) : (j == 0);
            ++row;
            if (++j == a.ny) j = 0;
        }
        const long long src = face ? faceSlot * P + n : nbSlot * P + n + shift;
        if (rOff >= 0 && src == rSrc + rLen)
            rLen += pieceEnd - n;
        else
        {
            if (rOff >= 0) emit((int)rOff, (int)rLen, rSrc);
            rOff = n - node0;
            rLen = pieceEnd - n;
            rSrc = src;
        }
        n = pieceEnd;
    }
    emit((int)rOff, (int)rLen, rSrc);
}

// Issue the copies of `tile` (tile flags `flags`) into the stage at `st`,
// called by all 32 lanes of the producer warp. Lane 0 announces the byte
// count; away from the outer faces it also issues the tile's 14 to 17 copies
// itself (measured faster than spreading them), while on a tile with
// outer-face nodes lanes 0-3 copy the x segments, lanes 4-11 assemble one y/z
// segment each from its runs, lanes 12-14 copy the stubs and lane 15 the
// material. SPARSE: the consumers run sparse-stub tiles (kTileStubSparse)
// without staged stubs.
template <int V = 2, bool SPARSE = true, class S>
__device__ __forceinline__ void stageTile(const StageSrc<S> &a, int tile, unsigned flags, unsigned st, unsigned bar,
                                          int lane)
{
    using L = Stage<S, V>;
    constexpr unsigned E = L::kElem;
    constexpr int kNodes = L::kNodes;
    const long long node0 = (long long)tile * kNodes;
    const long long P = a.P;
    // stubs staged for stub-loaded tiles, unless only a few of their nodes are
    const bool diel = (flags & kTileDiel) != 0 && !(kSparseStubs<S> && SPARSE && (flags & kTileStubSparse) != 0) &&
                      a.stub != nullptr;
    // x segments: the tile and L::kHalo nodes on each side, clipped to the planes
    const long long x0 = max(node0 - L::kHalo, 0LL), x1 = min(node0 + kNodes + L::kHalo, P);
    const unsigned segX = L::kSegX * E, xOff = (unsigned)(x0 - (node0 - L::kHalo)) * E;
    const unsigned xBytes = (unsigned)(x1 - x0) * E, seg = kNodes * E, stubSeg = kNodes * 4;
    const bool edge = (flags & kTileEdge) != 0;
    if (lane == 0)
    {
        const unsigned bytes = 4 * xBytes + 8 * seg + (diel ? 3 * stubSeg : 0) + kNodes;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" : : "r"(bar), "r"(bytes) : "memory");
        if (!edge)
        {
            const long long sy = a.px, sz = (long long)a.px * a.ny;
            const unsigned yz = st + L::kOffYZ;
#pragma unroll
            for (int s = 0; s < 4; ++s) bulkCopy(st + s * segX + xOff, a.in + s * P + x0, xBytes, bar);
#pragma unroll
            for (int t = 0; t < 2; ++t)
            {
                bulkCopy(yz + (0 + t) * seg, a.in + (6 + t) * P + node0 - sy, seg, bar);
                bulkCopy(yz + (2 + t) * seg, a.in + (4 + t) * P + node0 + sy, seg, bar);
                bulkCopy(yz + (4 + t) * seg, a.in + (10 + t) * P + node0 - sz, seg, bar);
                bulkCopy(yz + (6 + t) * seg, a.in + (8 + t) * P + node0 + sz, seg, bar);
            }
            if (diel)
            {
#pragma unroll
                for (int jj = 0; jj < 3; ++jj)
                    bulkCopy(st + L::kOffStub + jj * stubSeg, a.stub + jj * P + node0, stubSeg, bar);
            }
            bulkCopy(st + L::kOffMat, a.mat + node0, kNodes, bar);
        }
    }
    if (!edge) return;
    __syncwarp();
    if (lane < 4)
        bulkCopy(st + lane * segX + xOff, a.in + lane * P + x0, xBytes, bar);
    else if (lane < 12)
    {
        const int g = lane - 4;
        const unsigned dst = st + L::kOffYZ + g * seg;
        stageRuns<S, V>(a, node0, g, [&](int off, int len, long long src) {
            bulkCopy(dst + (unsigned)off * E, a.in + src, (unsigned)len * E, bar);
        });
    }
    else if (lane < 15)
    {
        if (diel) bulkCopy(st + L::kOffStub + (lane - 12) * stubSeg, a.stub + (lane - 12) * P + node0, stubSeg, bar);
    }
    else if (lane == 15)
        bulkCopy(st + L::kOffMat, a.mat + node0, kNodes, bar);
}

// The producer's view of a staged tile list: lane l holds entries it0 + l
// and it0 + 32 + l of the block's share (every gridDim.x-th entry), so the
// entries of the next 32 tiles are loaded 32 tiles before they are needed.
template <class T> struct EntryWindow
{
    T a, b;
    int it0;
    const T *list;
    int mine;
    T zero;

    __device__ __forceinline__ T fetch(int it) const
    {
        return it < mine ? list[blockIdx.x + (long long)it * gridDim.x] : zero;
    }
    __device__ __forceinline__ void init(const T *l, int m, int lane, T z)
    {
        list = l;
        mine = m;
        zero = z;
        it0 = 0;
        a = fetch(lane);
        b = fetch(32 + lane);
    }
    // advance so that `it` lies in the first half (call with it = it0 + 32)
    __device__ __forceinline__ void slide(int lane)
    {
        it0 += 32;
        a = b;
        b = fetch(it0 + 32 + lane);
    }
};

// SPARSE: the grid has sparse-stub tiles (FP32): their instantiation of the
// tile body is compiled in only then, so that other grids keep the kernel
// they had (with it, a grid without dielectrics stepped 1 % slower).
template <class S, int V, int STAGES = kStages, int MINB = 2, bool SPARSE = false>
__global__ void __launch_bounds__(kStagedThreads, MINB)
    stepKernelStaged(const StepArgs<S> a, const int *__restrict__ tiles, int ntiles)
{
    constexpr int kBytes = Stage<S, V>::kBytes;
    static_assert(V == 2 || V == 4, "a stage holds kBlock x 2 or kBlock x 4 nodes");
    extern __shared__ __align__(128) unsigned char stage[];
    __shared__ double red[STAGES][kBlock / 32];
    __shared__ __align__(8) unsigned long long full[STAGES], empty[STAGES], ered[STAGES];
    const int mine = ntiles > (int)blockIdx.x ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    const unsigned st0 = smemAddr(stage), full0 = smemAddr(full), empty0 = smemAddr(empty), ered0 = smemAddr(ered);
    if (threadIdx.x == 0)
    {
        for (int s = 0; s < STAGES; ++s)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(full0 + 8 * s) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(empty0 + 8 * s), "n"(kBlock / 32) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(ered0 + 8 * s), "n"(kBlock / 32) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory");
    }
    __syncthreads();
    if (threadIdx.x >= kBlock)
    {
        // producer warp: the list entries (tile and flags) of the next 32 to
        // 64 tiles are held in the lanes' registers
        const int lane = threadIdx.x - kBlock;
        const StageSrc<S> src = stageSrcOf(a);
        EntryWindow<int> win;
        win.init(tiles, mine, lane, 0);
        int issued = 0;
        for (int i = 0; i < mine; ++i)
        {
            const int s = i % STAGES;
            if (i == win.it0 + 32) win.slide(lane);
            const int e = __shfl_sync(0xffffffffu, win.a, i - win.it0);
            bool ok = true;
            if (i >= STAGES && lane == 0)
                ok = mbarWaitPaused<std::is_same<S, float>::value ? kProducerPauseNs : 0>(
                    empty0 + 8 * s, (unsigned)(i / STAGES - 1) & 1u, a.stage_wait_ns);
            if (!__shfl_sync(0xffffffffu, ok, 0))
            {
                if (lane == 0 && a.fault) atomicOr(a.fault, kStageTimeout);
                break;
            }
            stageTile<V, SPARSE>(src, entryTile(e), entryFlags(e), st0 + s * kBytes, full0 + 8 * s, lane);
            issued = i + 1;
        }
        // the copies of the last STAGES tiles may still be landing: stay
        // until they are in, so that the block's shared memory outlives them
        if (lane == 0)
            for (int i = issued > STAGES ? issued - STAGES : 0; i < issued; ++i)
                mbarWaitBounded(full0 + 8 * (i % STAGES), (unsigned)(i / STAGES) & 1u);
        return;
    }
    for (int i = 0; i < mine; ++i)
    {
        const int s = i % STAGES;
        if (!mbarWaitBounded(full0 + 8 * s, (unsigned)(i / STAGES) & 1u, a.stage_wait_ns))
        {
            if (a.fault) atomicOr(a.fault, kStageTimeout);
            return;
        }
        // The tile comes from the list and its dielectric flag from the flag
        // array, a dependent load, although the producer has both: on the
        // 192^3 heterogeneous grid this measured 0.1273 ms per step against
        // 0.1405 with the flag taken from the entry and 0.1438 with both read
        // from a copy the producer left in shared memory.
        const int e = tiles[blockIdx.x + i * gridDim.x];
        const int tile = entryTile(e);
        const uint8_t tf = a.tile_flags[tile];
        bool done = false;
        if constexpr (kSparseStubs<S> && SPARSE)
        {
            if (tf & kTileStubSparse)
            {
                stepTileInterior<S, V, true, true>(a, tile, red[s], true, stage + s * kBytes, ered0 + 8 * s,
                                                   (unsigned)(i / STAGES) & 1u);
                done = true;
            }
        }
        if (!done)
            stepTileInterior<S, V, true>(a, tile, red[s], (tf & kTileDiel) != 0, stage + s * kBytes,
                                          ered0 + 8 * s, (unsigned)(i / STAGES) & 1u);
        __syncwarp();
        if ((threadIdx.x & 31) == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(empty0 + 8 * s) : "memory");
    }
}

} // namespace tlmk
