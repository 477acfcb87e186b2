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
