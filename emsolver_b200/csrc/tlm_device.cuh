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
    static constexpr int V = 2;
    static constexpr int kMinBlocks = 4;
    static constexpr bool kSelect = true;
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
    static constexpr bool kSelect = true;
    static constexpr bool kScaled = true;
};
template <> struct Traits<__nv_bfloat16>
{
    using R = float;
    static constexpr int V = 4;
    static constexpr int kMinBlocks = 3;
    static constexpr bool kSelect = true;
    static constexpr bool kScaled = true;
};

// Division of n < 2^31 by a divisor d >= 1 that is fixed for a launch,
// through a multiply-high (Granlund and Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994): with shift = ceil(log2 d) and
// mul = floor(2^32 (2^shift - d) / d) + 1, n / d = (umulhi(n, mul) + n) >> shift
// (the sum stays below 2^32 because n < 2^31).
struct FastDiv
{
    unsigned mul;
    int shift;
};

inline FastDiv makeFastDiv(unsigned d)
{
    int l = 0;
    while (l < 32 && (1ull << l) < d) ++l;
    FastDiv f;
    f.mul = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    f.shift = l;
    return f;
}

__device__ __forceinline__ unsigned fastDiv(unsigned n, FastDiv f) { return (__umulhi(n, f.mul) + n) >> f.shift; }

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
// group of 4 consecutive x-nodes of one plane. Each pulse keeps a 14-bit
// offset-binary mantissa u (value m = u - 8192, |m| <= 8191); the group shares
// an 8-bit exponent e: pulse = m * 2^(e - 140). Layout, as two 32-bit halves:
//   lo = u0 | u1 << 14 | (e & 15) << 28,   hi = u2 | u3 << 14 | (e >> 4) << 28.
// e = 0 encodes an all-zero group (a zero-filled buffer decodes to zeros).
// The encoder picks e so that the group's largest magnitude uses 13 bits.
// Conversions between the integer mantissas and floats go through the
// float-bits identity bits(2^23 + 2^22 + k) = 0x4B400000 + k (0 <= k < 2^22),
// so neither direction needs an int<->float conversion instruction, and both
// are exact: m * 2^(e-140) is a float, and x * 2^(153-e) is an exact scaling.
struct __align__(8) Bfp4
{
    unsigned lo, hi;
};
template <> struct Traits<Bfp4>
{
    using R = float;
    static constexpr int V = 4;
    static constexpr int kMinBlocks = 3;
    static constexpr bool kSelect = true;
    static constexpr bool kScaled = false;
};

template <class S, int V> struct alignas(sizeof(S) * V) Pack
{
    S v[V];
};

constexpr unsigned kBfpMagic = 0x4B400000u;  // bits of 2^23 + 2^22
constexpr float kBfpBias = 12591104.0f;      // 2^23 + 2^22 + 8192: float of (magic | u) minus m

__device__ __forceinline__ int bfpExp(const Bfp4 &w) { return (int)((w.lo >> 28) | ((w.hi >> 24) & 0xf0u)); }

// 2^(e - 140), or 0 for e = 0 (the encoder never writes 1 <= e <= 15)
__device__ __forceinline__ float bfpUnit(int e) { return __int_as_float(max((e - 13) << 23, 0)); }

__device__ __forceinline__ float bfpValue(unsigned field, float unit, float bias)
{
    // (2^23 + 2^22 + u) * unit - (2^23 + 2^22 + 8192) * unit, one rounding of
    // an exactly representable result
    return __fmaf_rn(__uint_as_float((field & 0x3fffu) | kBfpMagic), unit, bias);
}

__device__ __forceinline__ void bfpDecode(const Bfp4 &w, float (&v)[4])
{
    const float unit = bfpUnit(bfpExp(w));
    const float bias = __fmul_rn(-kBfpBias, unit);
    v[0] = bfpValue(w.lo, unit, bias);
    v[1] = bfpValue(w.lo >> 14, unit, bias);
    v[2] = bfpValue(w.hi, unit, bias);
    v[3] = bfpValue(w.hi >> 14, unit, bias);
}

__device__ __forceinline__ float bfpDecodeOne(const Bfp4 &w, int c)
{
    const float unit = bfpUnit(bfpExp(w));
    const unsigned half = (c & 2) ? w.hi : w.lo;
    return bfpValue((c & 1) ? half >> 14 : half, unit, __fmul_rn(-kBfpBias, unit));
}

// Encode 4 values (round to nearest even, or stochastically with the random
// bits `r`). Groups whose largest magnitude is below 2^-112 (or not finite,
// or above 2^125) are stored as zero.
__device__ __forceinline__ Bfp4 bfpEncode(const float (&v)[4], bool stochastic, unsigned r)
{
    const float M = fmaxf(fmaxf(fabsf(v[0]), fabsf(v[1])), fmaxf(fabsf(v[2]), fabsf(v[3])));
    // exponent of M * (1 + 2^-12): M * 2^(153 - e) <= 8190 + 2^-11, so neither
    // rounding mode can carry a mantissa past 8191
    const float Madj = __fmaf_rn(M, 0x1p-12f, M);
    const int e = (__float_as_int(Madj) >> 23) + 1;           // Madj < 2^(e - 127)
    const float q = __int_as_float((267 - e) << 23);           // 2^(13 - (e - 127))
    unsigned u[4];
    if (stochastic)
    {
        const unsigned h0 = mix32(r), h1 = mix32(r ^ 0x5bd1e995u);
        const unsigned bits[4] = { h0 << 7, h0 >> 9, h1 << 7, h1 >> 9 };
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
            // y = x*q + d, d uniform in [1, 2) (16 random bits); floor(y - 1)
            // through a round-down add into the magic range
            const float d = __uint_as_float(0x3f800000u | (bits[c] & 0x7fff80u));
            const float y = __fmaf_rn(v[c], q, d);
            u[c] = __float_as_uint(__fadd_rd(y, kBfpBias - 1.0f));
        }
    }
    else
    {
#pragma unroll
        for (int c = 0; c < 4; ++c) u[c] = __float_as_uint(__fmaf_rn(v[c], q, kBfpBias));
    }
    Bfp4 w;
    w.lo = (u[0] & 0x3fffu) | ((u[1] & 0x3fffu) << 14) | ((unsigned)e << 28);
    w.hi = (u[2] & 0x3fffu) | ((u[3] & 0x3fffu) << 14) | (((unsigned)e >> 4) << 28);
    const bool keep = (M > 0x1p-112f) && (Madj < 0x1p125f);
    w.lo = keep ? w.lo : 0u;
    w.hi = keep ? w.hi : 0u;
    return w;
}

__device__ __forceinline__ float decode(float s, float) { return s; }
__device__ __forceinline__ double decode(double s, double) { return s; }
__device__ __forceinline__ float decode(__half s, float scale) { return __half2float(s) * scale; }
__device__ __forceinline__ float decode(__nv_bfloat16 s, float scale)
{
    return __bfloat162float(s) * scale;
}
// Stored value <-> pulse in storage units (no per-grid scale): the step
// kernels work in storage units, since the scale is a power of two and the
// step is linear, which only differs from the scaled pulse by that exact
// factor.
__device__ __forceinline__ float decodeRaw(float s) { return s; }
__device__ __forceinline__ double decodeRaw(double s) { return s; }
__device__ __forceinline__ float decodeRaw(__half s) { return __half2float(s); }
__device__ __forceinline__ float decodeRaw(__nv_bfloat16 s) { return __bfloat162float(s); }
template <class S> __device__ __forceinline__ S encodeRaw(float v);
template <> __device__ __forceinline__ float encodeRaw<float>(float v) { return v; }
template <> __device__ __forceinline__ __half encodeRaw<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 encodeRaw<__nv_bfloat16>(float v)
{
    return __float2bfloat16_rn(v);
}
template <class S> __device__ __forceinline__ S encodeRaw(double v);
template <> __device__ __forceinline__ double encodeRaw<double>(double v) { return v; }

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

// num / den for the stub denominator den = 4 + yh + gh: a zero numerator
// gives the zero itself (its sign kept: den > 0, which also sends a NaN
// denominator to the division), which is the IEEE quotient, without the
// division -- whose slower path zero numerators took: while a wave fills
// the grid most stub nodes divide zeros, and those steps of the 192^3
// heterogeneous grid ran 4-5 % slower than later ones.
template <class R> __device__ __forceinline__ R stubDiv(R num, R den)
{
    return (num == R(0) && den > R(0)) ? num : num / den;
}
template <> __device__ __forceinline__ float stubDiv<float>(float num, float den)
{
    return (num == 0.0f && den > 0.0f) ? num : __fdiv_rn(num, den);
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
        Vn[j] = stubDiv(R(2) * (sum4 + yh * vs[j]), den);
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
        const R vStub = stubDiv(R(2) * (sum4 + yh * vs[j]), den);
        Vn[j] = diel ? vStub : R(0.5) * sum4;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) ZI[k] = circulation(in, k);
    reflectLinks(in, Vn, ZI, out);
#pragma unroll
    for (int j = 0; j < 3; ++j) vs[j] = diel ? Vn[j] - vs[j] : vs[j];
}

// ---- two nodes at once: packed FP32x2 arithmetic ----
// Each lane is rounded exactly like the scalar operation. The code generator
// fuses a packed multiply into a following packed add even when fused
// multiply-add is disabled, which would round a*b + c once instead of twice.
// Products are therefore formed as fma(a, b, z) with z = -0.0 supplied at run
// time (a kernel argument the compiler cannot see through): fma(a, b, -0) is
// the correctly rounded product (signed zeros included) and an FMA cannot be
// fused again, so the packed scatter below is bitwise the scalar one.
#define TLM_F32X2_OP(name, op)                                                                   \
    __device__ __forceinline__ float2 name(float2 a, float2 b)                                   \
    {                                                                                            \
        float2 r;                                                                                \
        asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t" \
            op " pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"                                       \
            : "=f"(r.x), "=f"(r.y)                                                               \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                           \
        return r;                                                                                \
    }
TLM_F32X2_OP(add2, "add.rn.f32x2")
TLM_F32X2_OP(sub2, "sub.rn.f32x2")
#undef TLM_F32X2_OP

// a * b, correctly rounded per lane; z must be (-0.0, -0.0) from run time
__device__ __forceinline__ float2 mul2(float2 a, float2 b, float2 z)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pz, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mov.b64 pz, {%6, %7};\n\tfma.rn.f32x2 pd, pa, pb, pz;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(z.x), "f"(z.y));
    return r;
}
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }

__device__ __forceinline__ float2 nodeVoltage2(const float2 (&v)[12], int j, float2 z)
{
    const int a = (j == 0) ? 1 : 0;
    const int b = (j == 2) ? 1 : 2;
    return mul2(splat2(0.5f),
                add2(add2(add2(v[slotOf(a, 0, j)], v[slotOf(a, 1, j)]), v[slotOf(b, 0, j)]), v[slotOf(b, 1, j)]),
                z);
}
__device__ __forceinline__ float2 circulation2(const float2 (&v)[12], int k, float2 z)
{
    const int p = (k + 1) % 3, q = (k + 2) % 3;
    return mul2(splat2(0.5f),
                add2(sub2(sub2(v[slotOf(p, 0, q)], v[slotOf(p, 1, q)]), v[slotOf(q, 0, p)]), v[slotOf(q, 1, p)]),
                z);
}
__device__ __forceinline__ void reflectLinks2(const float2 (&in)[12], const float2 (&Vn)[3],
                                              const float2 (&ZI)[3], float2 (&out)[12])
{
#pragma unroll
    for (int s = 0; s < 12; ++s)
    {
        const int i = s >> 2, side = (s >> 1) & 1;
        const int j = fieldOfSlot(s);
        const int k = 3 - i - j;
        const bool plus = ((j == (i + 1) % 3) == (side == 1));
        const float2 base = plus ? add2(Vn[j], ZI[k]) : sub2(Vn[j], ZI[k]);
        out[s] = sub2(base, in[s ^ 2]);
    }
}
// scatterAir for a pair of air nodes
__device__ __forceinline__ void scatterAir2(const float2 (&in)[12], float2 (&out)[12], float2 z)
{
    float2 Vn[3], ZI[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) Vn[j] = nodeVoltage2(in, j, z);
#pragma unroll
    for (int k = 0; k < 3; ++k) ZI[k] = circulation2(in, k, z);
    reflectLinks2(in, Vn, ZI, out);
}
// scatterStub for a pair of stub-loaded nodes (the divides stay scalar).
// kZeroSkip: zero numerators skip the division (stubDiv); the batched
// dipoles, whose numerators are rarely zero, measured 1.2 % slower with it.
template <bool kZeroSkip = true>
__device__ __forceinline__ void scatterStub2(const float2 (&in)[12], float2 (&vs)[3], float2 yh, float2 gh,
                                             float2 (&out)[12], float2 z)
{
    float2 Vn[3], ZI[3];
    const float2 den = add2(add2(splat2(4.0f), yh), gh);
#pragma unroll
    for (int j = 0; j < 3; ++j)
    {
        const int a = (j == 0) ? 1 : 0;
        const int b = (j == 2) ? 1 : 2;
        const float2 sum4 =
            add2(add2(add2(in[slotOf(a, 0, j)], in[slotOf(a, 1, j)]), in[slotOf(b, 0, j)]), in[slotOf(b, 1, j)]);
        const float2 num = mul2(splat2(2.0f), add2(sum4, mul2(yh, vs[j], z)), z);
        if constexpr (kZeroSkip)
            Vn[j] = make_float2(stubDiv(num.x, den.x), stubDiv(num.y, den.y));
        else
            Vn[j] = make_float2(__fdiv_rn(num.x, den.x), __fdiv_rn(num.y, den.y));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) ZI[k] = circulation2(in, k, z);
    reflectLinks2(in, Vn, ZI, out);
#pragma unroll
    for (int j = 0; j < 3; ++j) vs[j] = sub2(Vn[j], vs[j]);
}

// A source or monitor attached to one node. Entries are sorted by node
// (stable: per node, the reference's injection order, then the sample).
// The near-field box of 16-bit storage (tlm_config.near_field): every node
// inside it keeps, beside its stored 16-bit pulses, their FP32 residuals, so
// that decode(stored) + residual is exactly the FP32 pulse. Box nodes read
// their neighbours' pulses completed by the residuals (zero outside the box)
// and so step as FP32 storage would; nodes outside read the 16-bit values.
struct NearBox
{
    const float *lo_in;  // 12 residual planes of the input state, bP nodes each (nullptr: no box)
    float *lo_out;       // the same for the output state
    int x0, y0, z0;      // box origin (node coordinates)
    int nx, ny, nz;      // box extent
    long long bP;        // nx * ny * nz
    // residual index of node (i, j, k), -1 outside the box
    __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        const unsigned bi = (unsigned)(i - x0), bj = (unsigned)(j - y0), bk = (unsigned)(k - z0);
        return (bi < (unsigned)nx && bj < (unsigned)ny && bk < (unsigned)nz)
                   ? ((long long)bk * ny + bj) * nx + bi
                   : -1;
    }
};

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
