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

#include "tlm_aux_kernels.cuh"
#include "tlm_step_kernel.cuh"

namespace tlmk {

template <class S> struct MemberDesc
{
    using R = typename Traits<S>::R;
    S *buf[2];               // ping-pong planes: step n reads buf[n & 1]
    R *stub;
    const uint8_t *mat;
    const R *yhat;
    const R *ghat;
    long long P, nquads;
    int nx, ny, nz, px, nq;
    FastDiv div_nq, div_ny;
    R rho, scale, inv_scale;
    const int *tile_begin;
    const SpecEntry *spec;
    const uint8_t *tile_flags;
    float neg_zero;          // -0.0f (see mul2)
    const R *sv;             // source value per absolute step, [total]
    R *samples;              // [window][nsamp][6]
    int nsamp;
    double *epart;           // [window/16 + 1][nblocks]
    int nblocks;
    int stochastic;
    long long base;          // absolute step at the start of the current window
    long long total;         // the member stops before this step
    EpilogueArgs<R> epi;     // monitor outputs (window fields filled per window)
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
// staged kernel's pipeline over the (member, tile) pairs of every member's
// staged tiles. The producer lane builds the tile's member arguments for
// this step into the stage next to the pulses (so the consumers read them
// from shared memory), or marks the stage empty when the member is past its
// last step. Energy steps differ between members, so each consumer counts
// its own uses of every stage's energy barrier (the same sequence in every
// thread).
template <int STAGES = kStages, int MINB = 2>
__global__ void __launch_bounds__(kStagedThreads, MINB)
    batchStepKernelStaged(MemberDesc<float> *__restrict__ members, const int2 *__restrict__ tiles,
                          const int *__restrict__ ntiles, int i, unsigned *fault)
{
    constexpr int kData = Stage<float>::kBytes;
    constexpr int kSlot = kData + (int)((sizeof(StepArgs<float>) + 15) / 16 * 16);
    extern __shared__ __align__(128) unsigned char stage[];
    __shared__ double red[STAGES][kBlock / 32];
    __shared__ __align__(8) unsigned long long full[STAGES], empty[STAGES], ered[STAGES];
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
        // producer warp: lane 0 writes the member arguments, then every lane
        // issues its share of the copies
        const int lane = threadIdx.x - kBlock;
        int issued = 0;
        for (int it = 0; it < mine; ++it)
        {
            const int s = it % STAGES;
            bool ok = true;
            if (it >= STAGES && lane == 0) ok = mbarWaitBounded(empty0 + 8 * s, (unsigned)(it / STAGES - 1) & 1u);
            if (!__shfl_sync(0xffffffffu, ok, 0))
            {
                if (lane == 0 && fault) atomicOr(fault, kStageTimeout);
                break;
            }
            const int2 tl = tiles[blockIdx.x + it * gridDim.x];
            const MemberDesc<float> &d = members[tl.x];
            StepArgs<float> *sa = reinterpret_cast<StepArgs<float> *>(stage + s * kSlot + kData);
            const long long n = d.base + i;
            const unsigned bar = full0 + 8 * s;
            if (n >= d.total)
            {
                if (lane == 0)
                {
                    sa->nquads = -1;  // the member has finished: an empty stage
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(bar) : "memory");
                }
            }
            else
            {
                if (lane == 0)
                {
                    StepArgs<float> a;
                    const long long eFirst = (d.base + 15) / 16 * 16;
                    a.in = d.buf[n & 1];
                    a.out = d.buf[(n + 1) & 1];
                    a.stub = d.stub;
                    a.mat = d.mat;
                    a.yhat = d.yhat;
                    a.ghat = d.ghat;
                    a.P = d.P;
                    a.nquads = d.nquads;
                    a.nx = d.nx;
                    a.ny = d.ny;
                    a.nz = d.nz;
                    a.px = d.px;
                    a.nq = d.nq;
                    a.div_nq = d.div_nq;
                    a.div_ny = d.div_ny;
                    a.rho = d.rho;
                    a.scale = d.scale;
                    a.inv_scale = d.inv_scale;
                    a.tile_begin = d.tile_begin;
                    a.spec = d.spec;
                    a.tile_flags = d.tile_flags;
                    a.neg_zero = d.neg_zero;
                    a.sv = d.sv[n];
                    a.samples = d.samples + (long long)i * d.nsamp * 6;
                    a.epart = (n % 16 == 0) ? d.epart + ((n - eFirst) / 16) * d.nblocks : nullptr;
                    a.e_lo = 0;
                    a.e_hi = LLONG_MAX;
                    a.fault = fault;
                    a.round_seed = mix32((unsigned)n * 0x9E3779B9u + 0x7f4a7c15u);
                    a.stochastic = d.stochastic;
                    *sa = a;
                }
                __syncwarp();
                stageTile(*sa, tl.y, st0 + s * kSlot, bar, lane);
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
        const StepArgs<float> &a = *reinterpret_cast<const StepArgs<float> *>(stage + s * kSlot + kData);
        if (a.nquads >= 0)
        {
            const int tile = tiles[blockIdx.x + it * gridDim.x].y;
            const unsigned ep = (eBits >> s) & 1u;
            if (a.epart != nullptr) eBits ^= 1u << s;
            stepTileInterior<float, 2, true>(a, tile, red[s], (a.tile_flags[tile] & kTileDiel) != 0,
                                             stage + s * kSlot, ered0 + 8 * s, ep);
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
