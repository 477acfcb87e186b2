// tlm_device.cuh -- device-side building blocks of the SCN TLM step.
//
// Layout in HBM (structure of arrays): the 12 link pulses of a node live in
// 12 separate planes, plane `slot` holding that slot for every node in the
// padded order node = (k*ny + j)*px + i, px = nx rounded up to kPadX. The
// slot numbering is the reference's portOf (TlmSolver.cpp:19-29):
// slot = axis*4 + side*2 + pol, side 0 = -face, pol = index of the E axis in
// the link axis's transverse pair {x:(y,z), y:(x,z), z:(x,y)}.
//
// The state kept between steps is the REFLECTED pulses of the last scatter
// (before connect). Connect is folded into the next step as a gather: the
// pulse incident on face (a, s) of node c is the neighbour's reflected pulse
// on its opposite face, -(own reflected) if the neighbour is PEC, and
// rho*(own reflected) on the outer boundary. This is the reference's
// in-place swap/negate/scale of TlmSolver::connect (TlmSolver.cpp:551-613)
// written as a pure function, so each step reads every plane once and
// writes every plane once at aligned addresses.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tlmk {

constexpr int kBlock = 256;  // threads per block of the step kernel
constexpr int kPadX = 8;     // row pitch multiple (every vector width divides it)

enum : uint8_t { kAir = 0, kPec = 1, kDiel0 = 2 };

// Storage type S -> arithmetic type R, default nodes per thread V (one
// aligned vector load per plane) and resident blocks per SM the default
// kernel is compiled for, whether the default kernel scatters with the
// warp-uniform select (else a per-node branch) -- the fastest choices
// measured on B200 -- and whether stored values carry a per-grid scale.
template <class S> struct Traits;
template <> struct Traits<float>
{
    using R = float;
    static constexpr int V = 4;
    static constexpr int kMinBlocks = 3;
    static constexpr bool kSelect = false;
    static constexpr bool kScaled = false;
};
template <> struct Traits<double>
{
    using R = double;
    static constexpr int V = 1;
    static constexpr int kMinBlocks = 4;
    static constexpr bool kSelect = true;
    static constexpr bool kScaled = false;
};
template <> struct Traits<__half>
{
    using R = float;
    static constexpr int V = 4;
    static constexpr int kMinBlocks = 3;
    static constexpr bool kSelect = false;
    static constexpr bool kScaled = true;
};
template <> struct Traits<__nv_bfloat16>
{
    using R = float;
    static constexpr int V = 4;
    static constexpr int kMinBlocks = 3;
    static constexpr bool kSelect = false;
    static constexpr bool kScaled = true;
};

// 32-bit integer mixer (the MurmurHash3 finaliser): counter-based random
// bits for stochastic rounding, a pure function of (node, slot, step).
__host__ __device__ __forceinline__ unsigned mix32(unsigned h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// Block floating point, 16 bits per pulse: one 64-bit word holds an aligned
// group of 4 consecutive x-nodes of one plane -- four 14-bit two's-complement
// mantissas (bits 0-13, 14-27, 28-41, 42-55) and the group's biased binary
// exponent (bits 56-63). Value = mantissa * 2^(E - 13), E = exponent - 127,
// chosen so the group's largest magnitude uses the full 13 bits. Exponent 0
// encodes an all-zero group.
struct Bfp4
{
    unsigned long long w;
};
template <> struct Traits<Bfp4>
{
    using R = float;
    static constexpr int V = 4;
    static constexpr int kMinBlocks = 3;
    static constexpr bool kSelect = false;
    static constexpr bool kScaled = false;
};

template <class S, int V> struct alignas(sizeof(S) * V) Pack
{
    S v[V];
};

__device__ __forceinline__ float bfpUnit(int biasedExp)
{
    // 2^(E - 13) for E = biasedExp - 127 (exponents below 2^-112 are flushed
    // to zero by the encoder, so the result is a normal float)
    return __int_as_float((biasedExp - 13) << 23);
}

__device__ __forceinline__ void bfpDecode(unsigned long long w, float (&v)[4])
{
    const int e = (int)(w >> 56);
    const float unit = e ? bfpUnit(e) : 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        const long long m = ((long long)(w << (50 - 14 * c))) >> 50;  // sign-extend 14 bits
        v[c] = (float)(int)m * unit;
    }
}

__device__ __forceinline__ float bfpDecodeOne(unsigned long long w, int c)
{
    const int e = (int)(w >> 56);
    const long long m = ((long long)(w << (50 - 14 * c))) >> 50;
    return e ? (float)(int)m * bfpUnit(e) : 0.0f;
}

// Encode 4 values; `r` (when stochastic) supplies random bits for unbiased
// rounding of each mantissa.
__device__ __forceinline__ unsigned long long bfpEncode(const float (&v)[4], bool stochastic,
                                                        unsigned r)
{
    float M = 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c) M = fmaxf(M, fabsf(v[c]));
    if (!(M > 0x1p-112f) || !(M < 0x1p126f)) return 0ull;  // zero, tiny, or not finite
    int e = (int)((__float_as_uint(M) >> 23) & 0xff) + 1;       // biased E with M < 2^E
    unsigned long long w = 0;
#pragma unroll 1
    for (int attempt = 0; attempt < 2; ++attempt)
    {
        const float q = __int_as_float((127 + 127 + 13 - e) << 23);  // 2^(13 - E)
        int m[4];
        int big = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
            const float x = v[c] * q;  // exact power-of-two scaling
            if (stochastic)
            {
                const float u = (float)(mix32(r + (unsigned)c) >> 8) * (1.0f / 16777216.0f);  // [0, 1)
                m[c] = __float2int_rd(x + u);
            }
            else
                m[c] = __float2int_rn(x);
            big = max(big, abs(m[c]));
        }
        if (big > 8191 && attempt == 0)
        {
            ++e;  // rounding reached 2^13: use the next binade
            continue;
        }
        w = (unsigned long long)e << 56;
#pragma unroll
        for (int c = 0; c < 4; ++c) w |= ((unsigned long long)(m[c] & 0x3fff)) << (14 * c);
        break;
    }
    return w;
}

__device__ __forceinline__ float decode(float s, float) { return s; }
__device__ __forceinline__ double decode(double s, double) { return s; }
__device__ __forceinline__ float decode(__half s, float scale) { return __half2float(s) * scale; }
__device__ __forceinline__ float decode(__nv_bfloat16 s, float scale)
{
    return __bfloat162float(s) * scale;
}
template <class S> __device__ __forceinline__ S encode(float v, float inv);
template <> __device__ __forceinline__ float encode<float>(float v, float) { return v; }
template <> __device__ __forceinline__ __half encode<__half>(float v, float inv)
{
    return __float2half_rn(v * inv);
}
template <> __device__ __forceinline__ __nv_bfloat16 encode<__nv_bfloat16>(float v, float inv)
{
    return __float2bfloat16_rn(v * inv);
}
template <class S> __device__ __forceinline__ S encode(double v, double);
template <> __device__ __forceinline__ double encode<double>(double v, double) { return v; }

// Stochastic rounding to the storage type: round the magnitude up with
// probability equal to the fraction of the gap it covers, so the rounding
// error has zero mean. r supplies 32 random bits.
template <class S> __device__ __forceinline__ S encodeStochastic(float v, float inv, unsigned r);
template <> __device__ __forceinline__ float encodeStochastic<float>(float v, float, unsigned)
{
    return v;
}
template <> __device__ __forceinline__ __nv_bfloat16 encodeStochastic<__nv_bfloat16>(float v, float inv,
                                                                                     unsigned r)
{
    // bfloat16 keeps the upper 16 bits of the float: adding 16 random bits to
    // the discarded half before truncating rounds the magnitude up with the
    // right probability (a carry moves into the next binade correctly).
    unsigned u = __float_as_uint(v * inv);
    if ((u & 0x7f800000u) != 0x7f800000u) u += (r >> 16);
    return __ushort_as_bfloat16((unsigned short)(u >> 16));
}
template <> __device__ __forceinline__ __half encodeStochastic<__half>(float v, float inv, unsigned r)
{
    const float x = v * inv;
    const __half lo = __float2half_rz(x);  // toward zero
    const float xl = __half2float(lo);
    if (xl == x) return lo;
    const __half hi = __ushort_as_half((unsigned short)(__half_as_ushort(lo) + 1));  // away from zero
    const float xh = __half2float(hi);
    const float frac = (x - xl) / (xh - xl);                 // in (0, 1)
    const float u = (float)(r >> 8) * (1.0f / 16777216.0f);  // uniform in [0, 1)
    return (u < frac) ? hi : lo;
}
template <> __device__ __forceinline__ double encodeStochastic<double>(float v, float, unsigned)
{
    return v;
}

// Slot helpers (compile-time after unrolling).
__host__ __device__ constexpr int firstTransverse(int axis) { return axis == 0 ? 1 : 0; }
__host__ __device__ constexpr int secondTransverse(int axis) { return axis == 2 ? 1 : 2; }
__host__ __device__ constexpr int slotOf(int axis, int side, int field)
{
    return axis * 4 + side * 2 + (field == firstTransverse(axis) ? 0 : 1);
}
__host__ __device__ constexpr int fieldOfSlot(int s)
{
    return (s & 1) ? secondTransverse(s >> 2) : firstTransverse(s >> 2);
}

// Node voltage V_j (TlmSolver.cpp:46-52) and link circulation ZI_k
// (TlmSolver.cpp:33-42), with the reference's left-to-right summation so the
// float results are bitwise the reference's.
template <class R> __device__ __forceinline__ R nodeVoltage(const R (&v)[12], int j)
{
    const int a = (j == 0) ? 1 : 0;
    const int b = (j == 2) ? 1 : 2;
    return R(0.5) * (((v[slotOf(a, 0, j)] + v[slotOf(a, 1, j)]) + v[slotOf(b, 0, j)]) +
                     v[slotOf(b, 1, j)]);
}
template <class R> __device__ __forceinline__ R circulation(const R (&v)[12], int k)
{
    const int p = (k + 1) % 3, q = (k + 2) % 3;
    return R(0.5) * (((v[slotOf(p, 0, q)] - v[slotOf(p, 1, q)]) - v[slotOf(q, 0, p)]) +
                     v[slotOf(q, 1, p)]);
}

// Link reflections from the node quantities (TlmSolver.cpp:59-76):
// out[i,s,j] = (V_j +/- ZI_k) - in[i,1-s,j]; + when (j follows i cyclically)
// == (s is the + face). Adding -ZI equals subtracting ZI in IEEE arithmetic,
// so this rounds exactly like the reference's V_j + sg*ZI_k, sg = +/-1.
template <class R>
__device__ __forceinline__ void reflectLinks(const R (&in)[12], const R (&Vn)[3], const R (&ZI)[3],
                                             R (&out)[12])
{
#pragma unroll
    for (int s = 0; s < 12; ++s)
    {
        const int i = s >> 2, side = (s >> 1) & 1;
        const int j = fieldOfSlot(s);
        const int k = 3 - i - j;
        const bool plus = ((j == (i + 1) % 3) == (side == 1));
        const R base = plus ? (Vn[j] + ZI[k]) : (Vn[j] - ZI[k]);
        out[s] = base - in[s ^ 2];  // s ^ 2 = same axis and field, other face
    }
}

// Air node scatter (TlmSolver.cpp:59-76).
template <class R> __device__ __forceinline__ void scatterAir(const R (&in)[12], R (&out)[12])
{
    R Vn[3], ZI[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) Vn[j] = nodeVoltage(in, j);
#pragma unroll
    for (int k = 0; k < 3; ++k) ZI[k] = circulation(in, k);
    reflectLinks(in, Vn, ZI, out);
}

// Stub-loaded node with loss (TlmSolver.cpp:86-113):
// V_j = (2 (sum4 + yh*vs_j)) / ((4 + yh) + gh); stubs reflect V_j - vs_j.
// The library is compiled with --fmad=false, so yh*vs_j is rounded before
// the add exactly as in the reference.
template <class R>
__device__ __forceinline__ void scatterStub(const R (&in)[12], R (&vs)[3], R yh, R gh, R (&out)[12])
{
    R Vn[3], ZI[3];
    const R den = (R(4) + yh) + gh;
#pragma unroll
    for (int j = 0; j < 3; ++j)
    {
        const int a = (j == 0) ? 1 : 0;
        const int b = (j == 2) ? 1 : 2;
        const R sum4 = ((in[slotOf(a, 0, j)] + in[slotOf(a, 1, j)]) + in[slotOf(b, 0, j)]) +
                       in[slotOf(b, 1, j)];
        Vn[j] = (R(2) * (sum4 + yh * vs[j])) / den;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) ZI[k] = circulation(in, k);
    reflectLinks(in, Vn, ZI, out);
#pragma unroll
    for (int j = 0; j < 3; ++j) vs[j] = Vn[j] - vs[j];
}

// Scatter of a node that may be air or stub-loaded, without a branch: the
// node voltage is selected between the air formula (TlmSolver.cpp:46-52)
// and the stub formula (TlmSolver.cpp:86-98), so each node gets exactly the
// value its own formula rounds to; stubs are updated only when `diel`.
template <class R>
__device__ __forceinline__ void scatterSelect(const R (&in)[12], R (&vs)[3], R yh, R gh, bool diel,
                                              R (&out)[12])
{
    R Vn[3], ZI[3];
    const R den = (R(4) + yh) + gh;
#pragma unroll
    for (int j = 0; j < 3; ++j)
    {
        const int a = (j == 0) ? 1 : 0;
        const int b = (j == 2) ? 1 : 2;
        const R sum4 = ((in[slotOf(a, 0, j)] + in[slotOf(a, 1, j)]) + in[slotOf(b, 0, j)]) +
                       in[slotOf(b, 1, j)];
        const R vStub = (R(2) * (sum4 + yh * vs[j])) / den;
        Vn[j] = diel ? vStub : R(0.5) * sum4;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) ZI[k] = circulation(in, k);
    reflectLinks(in, Vn, ZI, out);
#pragma unroll
    for (int j = 0; j < 3; ++j) vs[j] = diel ? Vn[j] - vs[j] : vs[j];
}

// A source or monitor attached to one node. Entries are sorted by node
// (stable: per node, the reference's injection order, then the sample).
struct SpecEntry
{
    long long node;  // padded node index
    int kind;        // kInject / kSample
    int arg;         // kInject: E axis; kSample: sample slot
    float amp;
    int pad_;
};
enum { kInject = 0, kSample = 1 };

// Warp + block sum of doubles in a fixed order (deterministic).
__device__ __forceinline__ double blockSumDouble(double v, double *smem)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
    {
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 0; w < nw; ++w) s += smem[w];
    }
    return s;
}

} // namespace tlmk
