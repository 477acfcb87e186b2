// tlm_batch_kernels.cuh -- many TLM grids of different sizes advanced by one
// launch per step.
//
// Every member grid keeps its own planes, monitors and records (it is an
// ordinary solver handle). A tile table lists (member, tile) pairs, one tile
// = kBlock threads x V nodes of one member, exactly the tiles the single-grid
// kernel would launch as blocks. The step kernel runs a fixed grid of
// resident blocks, each walking a contiguous chunk of the tile table; the
// member table and the tile count live in device memory, so a CUDA graph of
// W steps captured once
// stays valid while members join and leave between windows. Each member
// advances from its own current step `base + i` and stops at its own
// `total`. The per-tile arithmetic is stepTile, the same code as the
// single-grid kernel, so a member's results are bitwise those it gets alone.
#pragma once

#include <cstddef>

#include "tlm_aux_kernels.cuh"
#include "tlm_step_kernel.cuh"

namespace tlmk {

// One member grid of a batch group. The first 128 bytes (the head, up to
// nblocks) hold everything the staged batch kernel reads, so that its
// producer warp loads a member with one coalesced 128-byte load (one 32-bit
// word per lane); records start on 128-byte boundaries.
template <class S> struct alignas(128) MemberDesc
{
    using R = typename Traits<S>::R;
    // ---- head ----
    S *buf[2];               // ping-pong planes: step n reads buf[n & 1]
    R *stub;
    const uint8_t *mat;
    const R *yhat;
    const R *ghat;
    double *epart;           // [window/16 + 1][nblocks]
    long long P;
    long long base;          // absolute step at the start of the current window
    long long total;         // the member stops before this step
    int nx, ny, nz, px, nq;
    FastDiv div_nq, div_ny;
    R rho;
    int nblocks;
    // ---- the rest ----
    long long nquads;
    R scale, inv_scale;
    const int *tile_begin;
    const SpecEntry *spec;
    const uint8_t *tile_flags;
    float neg_zero;          // -0.0f (see mul2)
    const R *sv;             // source value per absolute step, [total]
    R *samples;              // [window][nsamp][6]
    int nsamp;
    int stochastic;
    NearBox near;            // near-field box (lo_in/lo_out: the residuals beside buf[0] / buf[1])
    EpilogueArgs<R> epi;     // monitor outputs (window fields filled per window)
};

// 32-bit word indices of the head fields of an FP32 member.
struct HeadWords
{
    using D = MemberDesc<float>;
    static constexpr int kBuf = offsetof(D, buf) / 4, kStub = offsetof(D, stub) / 4, kMat = offsetof(D, mat) / 4,
                         kYhat = offsetof(D, yhat) / 4, kGhat = offsetof(D, ghat) / 4,
                         kEpart = offsetof(D, epart) / 4, kP = offsetof(D, P) / 4, kBase = offsetof(D, base) / 4,
                         kTotal = offsetof(D, total) / 4, kNx = offsetof(D, nx) / 4, kNy = offsetof(D, ny) / 4,
                         kNz = offsetof(D, nz) / 4, kPx = offsetof(D, px) / 4, kNq = offsetof(D, nq) / 4,
                         kDivNq = offsetof(D, div_nq) / 4, kDivNy = offsetof(D, div_ny) / 4,
                         kRho = offsetof(D, rho) / 4, kNblocks = offsetof(D, nblocks) / 4;
    static_assert(offsetof(D, nblocks) + 4 <= 128, "the head of an FP32 member fits 128 bytes");
    static_assert(sizeof(D) % 128 == 0, "member records start on 128-byte boundaries");
};

template <class S, int V, int MINB, bool SEL>
__global__ void __launch_bounds__(kBlock, MINB)
    batchStepKernel(MemberDesc<S> *__restrict__ members, const int2 *__restrict__ tiles,
                    const int *__restrict__ ntiles, int i, unsigned *fault)
{
    __shared__ double red[kBlock / 32];
    __shared__ StepArgs<S> sa;
    __shared__ int skip;
    // Each block walks a contiguous chunk of the tile table: consecutive
    // tiles mostly belong to the same member (its arguments are rebuilt only
    // when the member changes) and are spatial neighbours (shared rows and
    // planes stay in L2).
    const int nt = *ntiles;
    const int chunk = (nt + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * chunk;
    const int t1 = min(t0 + chunk, nt);
    int current = -1;
    for (int t = t0; t < t1; ++t)
    {
        const int2 tl = tiles[t];
        if (tl.x != current)
        {
            __syncthreads();  // every thread is done with the previous member's arguments
            if (threadIdx.x == 0)
            {
                const MemberDesc<S> &d = members[tl.x];
                const long long n = d.base + i;
                skip = n >= d.total;
                if (!skip)
                {
                    const long long eFirst = (d.base + 15) / 16 * 16;
                    sa.in = d.buf[n & 1];
                    sa.out = d.buf[(n + 1) & 1];
                    sa.stub = d.stub;
                    sa.mat = d.mat;
                    sa.yhat = d.yhat;
                    sa.ghat = d.ghat;
                    sa.P = d.P;
                    sa.nquads = d.nquads;
                    sa.nx = d.nx;
                    sa.ny = d.ny;
                    sa.nz = d.nz;
                    sa.px = d.px;
                    sa.nq = d.nq;
                    sa.div_nq = d.div_nq;
                    sa.div_ny = d.div_ny;
                    sa.rho = d.rho;
                    sa.scale = d.scale;
                    sa.inv_scale = d.inv_scale;
                    sa.tile_begin = d.tile_begin;
                    sa.spec = d.spec;
                    sa.tile_flags = d.tile_flags;
                    sa.neg_zero = d.neg_zero;
                    sa.sv = d.sv[n];
                    sa.samples = d.samples + (long long)i * d.nsamp * 6;
                    sa.epart = (n % 16 == 0) ? d.epart + ((n - eFirst) / 16) * d.nblocks : nullptr;
                    sa.e_lo = 0;
                    sa.e_hi = LLONG_MAX;
                    sa.fault = fault;
                    sa.round_seed = mix32((unsigned)n * 0x9E3779B9u + 0x7f4a7c15u);
                    sa.stochastic = d.stochastic;
                    sa.stage_wait_ns = kStageWaitNs;
                    sa.near = d.near;
                    if (n & 1)
                    {
                        sa.near.lo_in = d.near.lo_out;
                        sa.near.lo_out = const_cast<float *>(d.near.lo_in);
                    }
                }
            }
            __syncthreads();
            current = tl.x;
        }
        if (!skip)
        {
            stepTile<S, V, false, SEL>(sa, tl.y, red);
            // energy steps reduce through `red`: finish before the next tile reuses it
            if (sa.epart != nullptr) __syncthreads();
        }
    }
}

// Staged tiles of an FP32 batch group (2 nodes per thread): the single-grid
// staged kernel's pipeline over the (member, packed tile entry) pairs of
// every member's staged tiles. The producer warp holds the entries of the
// next 32 to 64 tiles; per tile its lanes load the member's 128-byte head as
// eight 16-byte vectors (L1-resident: a few hundred members) before waiting
// for the stage, take the fields they need from registers (warp shuffles
// share the pipe with the consumers' shared-memory loads and measured about
// 280 cycles each under load), and lane 0 writes the head, the step's output
// planes and energy partials and the tile's entry into the stage's header
// (or marks the stage empty when the member is past its last step), which
// the consumers read back as 16-byte vectors. Energy steps differ between
// members, so each consumer counts its own uses of every stage's energy
// barrier (the same sequence in every thread).
struct __align__(16) BatchStageHdr
{
    uint4 head[8];      // the member's head words (HeadWords)
    float *out;         // output planes of this tile's step
    double *epart;      // energy partials of this step (nullptr: not an energy step)
    int tile;           // -1: an empty stage
    unsigned flags;
    unsigned pad_[2];
};

// Word i (a compile-time index) of a head held as eight 16-byte vectors.
template <int I> __device__ __forceinline__ unsigned headWord(const uint4 (&h)[8])
{
    static_assert(I >= 0 && I < 32, "head word index");
    const uint4 v = h[I / 4];
    return (I % 4 == 0) ? v.x : (I % 4 == 1) ? v.y : (I % 4 == 2) ? v.z : v.w;
}
template <int I> __device__ __forceinline__ unsigned long long headU64(const uint4 (&h)[8])
{
    return (unsigned long long)headWord<I>(h) | ((unsigned long long)headWord<I + 1>(h) << 32);
}

template <int STAGES = kStages, int MINB = 2>
__global__ void __launch_bounds__(kStagedThreads, MINB)
    batchStepKernelStaged(const MemberDesc<float> *__restrict__ members, const int2 *__restrict__ tiles,
                          const int *__restrict__ ntiles, int i, unsigned *fault, float negZero)
{
    using H = HeadWords;
    constexpr int kData = Stage<float>::kBytes;
    extern __shared__ __align__(128) unsigned char stage[];
    __shared__ double red[STAGES][kBlock / 32];
    __shared__ __align__(8) unsigned long long full[STAGES], empty[STAGES], ered[STAGES];
    __shared__ __align__(16) BatchStageHdr hdr[STAGES];
    const int nt = *ntiles;
    const int mine = nt > (int)blockIdx.x ? (nt - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
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
        const int lane = threadIdx.x - kBlock;
        EntryWindow<int2> win;
        win.init(tiles, mine, lane, make_int2(0, 0));
        int issued = 0;
        for (int it = 0; it < mine; ++it)
        {
            const int s = it % STAGES;
            if (it == win.it0 + 32) win.slide(lane);
            const int2 ent = make_int2(__shfl_sync(0xffffffffu, win.a.x, it - win.it0),
                                       __shfl_sync(0xffffffffu, win.a.y, it - win.it0));
            const int e = ent.y;
            uint4 h[8];
            const uint4 *hp = reinterpret_cast<const uint4 *>(members + ent.x);
#pragma unroll
            for (int q = 0; q < 8; ++q) h[q] = __ldg(hp + q);
            bool ok = true;
            if (it >= STAGES && lane == 0)
                ok = mbarWaitPaused<0>(empty0 + 8 * s, (unsigned)(it / STAGES - 1) & 1u);
            if (!__shfl_sync(0xffffffffu, ok, 0))
            {
                if (lane == 0 && fault) atomicOr(fault, kStageTimeout);
                break;
            }
            const long long n = (long long)headU64<H::kBase>(h) + i;
            const bool live = n < (long long)headU64<H::kTotal>(h);
            float *const buf0 = reinterpret_cast<float *>(headU64<H::kBuf>(h));
            float *const buf1 = reinterpret_cast<float *>(headU64<H::kBuf + 2>(h));
            const unsigned bar = full0 + 8 * s;
            if (lane == 0)
            {
                BatchStageHdr &hd = hdr[s];
#pragma unroll
                for (int q = 0; q < 8; ++q) hd.head[q] = h[q];
                const long long base = n - i;
                const long long eFirst = (base + 15) / 16 * 16;
                double *const ep = reinterpret_cast<double *>(headU64<H::kEpart>(h));
                hd.out = (n & 1) ? buf0 : buf1;
                hd.epart = (n % 16 == 0) ? ep + ((n - eFirst) / 16) * (int)headWord<H::kNblocks>(h) : nullptr;
                hd.tile = live ? entryTile(e) : -1;
                hd.flags = entryFlags(e);
                if (!live) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(bar) : "memory");
            }
            if (live)
            {
                StageSrc<float> src;
                src.in = (n & 1) ? buf1 : buf0;
                src.stub = reinterpret_cast<const float *>(headU64<H::kStub>(h));
                src.mat = reinterpret_cast<const uint8_t *>(headU64<H::kMat>(h));
                src.P = (long long)headU64<H::kP>(h);
                src.px = (int)headWord<H::kPx>(h);
                src.ny = (int)headWord<H::kNy>(h);
                src.nz = (int)headWord<H::kNz>(h);
                src.div_nq.mul = headWord<H::kDivNq>(h);
                src.div_nq.shift = (int)headWord<H::kDivNq + 1>(h);
                src.div_ny.mul = headWord<H::kDivNy>(h);
                src.div_ny.shift = (int)headWord<H::kDivNy + 1>(h);
                stageTile(src, entryTile(e), entryFlags(e), st0 + s * kData, bar, lane);
            }
            issued = it + 1;
        }
        if (lane == 0)
            for (int it = issued > STAGES ? issued - STAGES : 0; it < issued; ++it)
                mbarWaitBounded(full0 + 8 * (it % STAGES), (unsigned)(it / STAGES) & 1u);
        return;
    }
    unsigned eBits = 0;
    for (int it = 0; it < mine; ++it)
    {
        const int s = it % STAGES;
        if (!mbarWaitBounded(full0 + 8 * s, (unsigned)(it / STAGES) & 1u))
        {
            if (fault) atomicOr(fault, kStageTimeout);
            return;
        }
        const BatchStageHdr &hd = hdr[s];
        const uint4 tail0 = *reinterpret_cast<const uint4 *>(&hd.out);   // out, epart
        const uint4 tail1 = *reinterpret_cast<const uint4 *>(&hd.tile);  // tile, flags
        const int tile = (int)tail1.x;
        if (tile >= 0)
        {
            uint4 h[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) h[q] = hd.head[q];
            StepArgs<float> a;
            a.in = nullptr;  // the staged body reads its inputs from the stage
            a.out = reinterpret_cast<float *>((unsigned long long)tail0.x | ((unsigned long long)tail0.y << 32));
            a.stub = reinterpret_cast<float *>(headU64<H::kStub>(h));
            a.mat = nullptr;
            a.yhat = reinterpret_cast<const float *>(headU64<H::kYhat>(h));
            a.ghat = reinterpret_cast<const float *>(headU64<H::kGhat>(h));
            a.P = (long long)headU64<H::kP>(h);
            a.nquads = 0;
            a.nx = (int)headWord<H::kNx>(h);
            a.ny = (int)headWord<H::kNy>(h);
            a.nz = (int)headWord<H::kNz>(h);
            a.px = (int)headWord<H::kPx>(h);
            a.nq = (int)headWord<H::kNq>(h);
            a.div_nq.mul = headWord<H::kDivNq>(h);
            a.div_nq.shift = (int)headWord<H::kDivNq + 1>(h);
            a.div_ny.mul = headWord<H::kDivNy>(h);
            a.div_ny.shift = (int)headWord<H::kDivNy + 1>(h);
            a.rho = __uint_as_float(headWord<H::kRho>(h));
            a.scale = 1.0f;
            a.inv_scale = 1.0f;
            a.tile_begin = nullptr;
            a.spec = nullptr;
            a.sv = 0.0f;
            a.samples = nullptr;
            a.epart = reinterpret_cast<double *>((unsigned long long)tail0.z | ((unsigned long long)tail0.w << 32));
            a.e_lo = 0;
            a.e_hi = LLONG_MAX;
            a.fault = fault;
            a.round_seed = 0;
            a.stochastic = 0;
            a.tile_flags = nullptr;
            a.neg_zero = negZero;
            a.stage_wait_ns = kStageWaitNs;
            a.near = NearBox{};
            const unsigned ep = (eBits >> s) & 1u;
            if (a.epart != nullptr) eBits ^= 1u << s;
            if (tail1.y & kTileStubSparse)
                stepTileInterior<float, 2, true, true, false>(a, tile, red[s], true, stage + s * kData, ered0 + 8 * s,
                                                              ep);
            else
                stepTileInterior<float, 2, true, false, false>(a, tile, red[s], (tail1.y & kTileDiel) != 0,
                                                               stage + s * kData, ered0 + 8 * s, ep);
        }
        __syncwarp();
        if ((threadIdx.x & 31) == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(empty0 + 8 * s) : "memory");
    }
}

// One block of 512 threads per member: the window's records, DFT and energy
// (the same body and block size as the single-grid epilogue, so even the
// FP64 energy sums round identically), then the member's base moves to the
// next window. Blocks past *nmembers return at once.
template <class S>
__global__ void __launch_bounds__(512)
    batchEpilogue(MemberDesc<S> *__restrict__ members, const int *__restrict__ nmembers, int w)
{
    using R = typename Traits<S>::R;
    __shared__ double red[16];
    __shared__ EpilogueArgs<R> ea;
    __shared__ int weff;
    const int m = blockIdx.x;
    if (m >= *nmembers) return;
    MemberDesc<S> &d = members[m];
    if (threadIdx.x == 0)
    {
        const long long base = d.base;
        const long long rem = d.total - base;
        weff = (int)(rem < (long long)w ? (rem > 0 ? rem : 0) : w);
        ea = d.epi;
        ea.base = base;
        ea.w = weff;
        const long long eFirst = (base + 15) / 16 * 16;
        ea.e_first = eFirst;
        ea.n_e = eFirst < base + weff ? (int)((base + weff - 1 - eFirst) / 16 + 1) : 0;
    }
    __syncthreads();
    if (weff > 0) epilogueBody(ea, red);
    __syncthreads();
    if (threadIdx.x == 0 && weff > 0) d.base = ea.base + weff;
}

} // namespace tlmk
