// common.cuh -- device helpers shared by the FP64 plain and FP32 batched paths:
// complex arithmetic on float2/double2 (and float4 = a pair of complex values
// for the two components of one cell), Philox4x32-10 and Box-Muller.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "twiddle_fp32.h"

#define BEC_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------- complex
BEC_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
BEC_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
BEC_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
BEC_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
BEC_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
BEC_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
BEC_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
BEC_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
BEC_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
BEC_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// float4 holds (a.re, a.im, b.re, b.im): both components of one cell.
BEC_HD float4 pmul(float4 v, float2 w)
{
    return make_float4(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x,
                       v.z * w.x - v.w * w.y, v.z * w.y + v.w * w.x);
}
BEC_HD float4 padd(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
BEC_HD float4 psub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
BEC_HD float4 pscale(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }

// Twiddle multiply used by the FFT stages, overloaded on the element type.
BEC_HD double2 tmul(double2 v, double2 w) { return cmul(v, w); }
BEC_HD float2 tmul(float2 v, float2 w) { return cmul(v, w); }
BEC_HD float4 tmul(float4 v, float2 w) { return pmul(v, w); }
BEC_HD double2 vadd(double2 a, double2 b) { return cadd(a, b); }
BEC_HD float2 vadd(float2 a, float2 b) { return cadd(a, b); }
BEC_HD float4 vadd(float4 a, float4 b) { return padd(a, b); }
BEC_HD double2 vsub(double2 a, double2 b) { return csub(a, b); }
BEC_HD float2 vsub(float2 a, float2 b) { return csub(a, b); }
BEC_HD float4 vsub(float4 a, float4 b) { return psub(a, b); }

// ---------------------------------------------------------------- Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror and Shaw (SC'11):
// ten rounds of two 32x32->64 multiplies with Weyl-sequence key bumps.
struct u32x4 { uint32_t x, y, z, w; };

BEC_HD u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
        uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return u32x4{c0, c1, c2, c3};
}

// hi and lo words of the 64-bit product a * b (one 32 x 32 -> 64 multiply)
__device__ __forceinline__ void mul_wide(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo)
{
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// The round keys of one key (k0, k1): (k0 + r W0, k1 + r W1) for rounds r < 10. A thread that draws many
// times under one key computes them once, before its loop, and the rounds only XOR them in (measured on
// the 32 x 32 plane pass: 0.85 % less time than bumping the key inside every draw, the same bits).
struct PhiloxKeys { uint32_t k0[10], k1[10]; };

__device__ __forceinline__ PhiloxKeys philox_keys(uint32_t k0, uint32_t k1)
{
    PhiloxKeys K;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        K.k0[r] = k0 + (uint32_t)r * 0x9E3779B9u;
        K.k1[r] = k1 + (uint32_t)r * 0xBB67AE85u;
    }
    return K;
}

// Two Philox4x32-10 draws under one key, their rounds interleaved: the two multiply chains are
// independent, so each hides the other's latency.
struct u32x4x2 { u32x4 a, b; };

__device__ __forceinline__ u32x4x2 philox4x32_10_x2(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                    uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3,
                                                    const PhiloxKeys &K)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t la0, ha0, la1, ha1, lb0, hb0, lb1, hb1;
        mul_wide(0xD2511F53u, a0, ha0, la0);
        mul_wide(0xCD9E8D57u, a2, ha1, la1);
        mul_wide(0xD2511F53u, b0, hb0, lb0);
        mul_wide(0xCD9E8D57u, b2, hb1, lb1);
        a0 = ha1 ^ a1 ^ K.k0[r]; a2 = ha0 ^ a3 ^ K.k1[r]; a1 = la1; a3 = la0;
        b0 = hb1 ^ b1 ^ K.k0[r]; b2 = hb0 ^ b3 ^ K.k1[r]; b1 = lb1; b3 = lb0;
    }
    return u32x4x2{u32x4{a0, a1, a2, a3}, u32x4{b0, b1, b2, b3}};
}

// Four draws under one key, their rounds interleaved (four independent multiply chains).
struct u32x4x4 { u32x4 a, b, c, d; };

__device__ __forceinline__ u32x4x4 philox4x32_10_x4(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                    const PhiloxKeys &K)
{
    // counters (c0 + i, c1, c2, c3), i < 4
    uint32_t a0 = c0, a1 = c1, a2 = c2, a3 = c3;
    uint32_t b0 = c0 + 1u, b1 = c1, b2 = c2, b3 = c3;
    uint32_t e0 = c0 + 2u, e1 = c1, e2 = c2, e3 = c3;
    uint32_t d0 = c0 + 3u, d1 = c1, d2 = c2, d3 = c3;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t la0, ha0, la1, ha1, lb0, hb0, lb1, hb1, le0, he0, le1, he1, ld0, hd0, ld1, hd1;
        mul_wide(0xD2511F53u, a0, ha0, la0);
        mul_wide(0xCD9E8D57u, a2, ha1, la1);
        mul_wide(0xD2511F53u, b0, hb0, lb0);
        mul_wide(0xCD9E8D57u, b2, hb1, lb1);
        mul_wide(0xD2511F53u, e0, he0, le0);
        mul_wide(0xCD9E8D57u, e2, he1, le1);
        mul_wide(0xD2511F53u, d0, hd0, ld0);
        mul_wide(0xCD9E8D57u, d2, hd1, ld1);
        a0 = ha1 ^ a1 ^ K.k0[r]; a2 = ha0 ^ a3 ^ K.k1[r]; a1 = la1; a3 = la0;
        b0 = hb1 ^ b1 ^ K.k0[r]; b2 = hb0 ^ b3 ^ K.k1[r]; b1 = lb1; b3 = lb0;
        e0 = he1 ^ e1 ^ K.k0[r]; e2 = he0 ^ e3 ^ K.k1[r]; e1 = le1; e3 = le0;
        d0 = hd1 ^ d1 ^ K.k0[r]; d2 = hd0 ^ d3 ^ K.k1[r]; d1 = ld1; d3 = ld0;
    }
    return u32x4x4{u32x4{a0, a1, a2, a3}, u32x4{b0, b1, b2, b3}, u32x4{e0, e1, e2, e3}, u32x4{d0, d1, d2, d3}};
}

// Stream tags of the counter's fourth word.
enum { RNG_TAG_INIT = 0, RNG_TAG_LOSS = 1 };

// The loss noise of one cell and step takes one Philox4x32-10 draw: its 128 bits are cut
// into six 21-bit fields, read as three Box-Muller pairs (u1 = (f + 1/2) / 2^21 in (0, 1),
// u2 = f / 2^21), i.e. six normals truncated beyond 5.5 standard deviations (tail mass 4e-8).
__host__ __device__ __forceinline__ void loss_fields(u32x4 w, uint32_t f[6])
{
    f[0] = w.x & 0x1FFFFFu;
    f[1] = (w.x >> 21) | ((w.y & 0x3FFu) << 11);
    f[2] = (w.y >> 10) & 0x1FFFFFu;
    f[3] = (w.y >> 31) | ((w.z & 0xFFFFFu) << 1);
    f[4] = (w.z >> 20) | ((w.w & 0x1FFu) << 12);
    f[5] = (w.w >> 9) & 0x1FFFFFu;
}

__device__ __forceinline__ void box_muller21(uint32_t f1, uint32_t f2, double &n1, double &n2)
{
    const double r = sqrt(-2.0 * log(((double)f1 + 0.5) * 0x1p-21));
    double s, c;
    sincospi(2.0 * ((double)f2 * 0x1p-21), &s, &c);
    n1 = r * c;
    n2 = r * s;
}

__device__ __forceinline__ void box_muller21(uint32_t f1, uint32_t f2, float &n1, float &n2)
{
    const float r = sqrtf(-2.0f * logf(((float)f1 + 0.5f) * 0x1p-21f));
    float s, c;
    sincospif(2.0f * ((float)f2 * 0x1p-21f), &s, &c);
    n1 = r * c;
    n2 = r * s;
}

// The six loss-noise normals of (seed, trajectory, step, cell).
template <typename R>
__device__ __forceinline__ void loss_normals6(uint64_t seed, uint32_t traj, uint32_t step, uint32_t cell, R out[6])
{
    uint32_t f[6];
    loss_fields(philox4x32_10(cell, step, traj, RNG_TAG_LOSS, (uint32_t)seed, (uint32_t)(seed >> 32)), f);
    box_muller21(f[0], f[1], out[0], out[1]);
    box_muller21(f[2], f[3], out[2], out[3]);
    box_muller21(f[4], f[5], out[4], out[5]);
}

// Box-Muller from two 32-bit words. u1 = (x1 + 1) / 2^32 in (0, 1],
// u2 = x2 / 2^32; -ln(u1) is taken through log1p near u1 = 1 so both tails
// keep full relative precision.
__device__ __forceinline__ void box_muller(uint32_t x1, uint32_t x2, double &n1, double &n2)
{
    double nl = (x1 < 0x80000000u) ? -log(((double)x1 + 1.0) * 0x1p-32)
                                   : -log1p(-((double)(0xFFFFFFFFu - x1)) * 0x1p-32);
    double r = sqrt(2.0 * nl);
    double s, c;
    sincospi(2.0 * ((double)x2 * 0x1p-32), &s, &c);
    n1 = r * c;
    n2 = r * s;
}

__device__ __forceinline__ void box_muller(uint32_t x1, uint32_t x2, float &n1, float &n2)
{
    float nl = (x1 < 0x80000000u) ? -logf(((float)x1 + 1.0f) * 0x1p-32f)
                                  : -log1pf(-((float)(0xFFFFFFFFu - x1)) * 0x1p-32f);
    float r = sqrtf(2.0f * nl);
    float s, c;
    sincospif(2.0f * ((float)x2 * 0x1p-32f), &s, &c);
    n1 = r * c;
    n2 = r * s;
}

// Four standard normals for (seed, trajectory, step, cell, tag).
template <typename R>
__device__ __forceinline__ void normals4(uint64_t seed, uint32_t traj, uint32_t step, uint32_t cell,
                                         uint32_t tag, R out[4])
{
    u32x4 r = philox4x32_10(cell, step, traj, tag, (uint32_t)seed, (uint32_t)(seed >> 32));
    box_muller(r.x, r.y, out[0], out[1]);
    box_muller(r.z, r.w, out[2], out[3]);
}

// ---------------------------------------------------------------- misc
__host__ __device__ __forceinline__ int brev_bits(int v, int bits)
{
#ifdef __CUDA_ARCH__
    return bits ? (int)(__brev((unsigned)v) >> (32 - bits)) : 0;
#else
    int r = 0;
    for (int b = 0; b < bits; ++b) if (v & (1 << b)) r |= 1 << (bits - 1 - b);
    return r;
#endif
}

// k value of lattice index i (getK, wigner_kernel.cu:15-21)
template <typename R>
__host__ __device__ __forceinline__ R getk(int i, R dk, int n) { return (2 * i > n) ? dk * (R)(i - n) : dk * (R)i; }

// signed index of lattice index i along an axis of n points (k = dk * kidx(i, n), getK)
__host__ __device__ __forceinline__ int kidx(int i, int n) { return (2 * i > n) ? i - n : i; }

// e^{+2 pi i turns}, turns = frac (c_x ix^2 + c_y iy^2 + c_z iz^2) formed in FP64 (GroupParamsF::kin_*):
// the kinetic phase e^{+i k^2/2 dt frac} (wigner_kernel.cu:137-151) reduced to [-1/2, 1/2] turn
// exactly, evaluated in FP64 and rounded to the FP32 pair of modulus closest to 1 (twiddle_fp32.h)
__device__ __forceinline__ float2 kin_phase(double turns)
{
    const double r = turns - rint(turns);
    double s, c;
    sincospi(2.0 * r, &s, &c);
    const fftreg::Twid t = fftreg::unit_cs(c, s);
    return make_float2(t.a, t.b);
}

// Neumaier-compensated accumulator.
struct KSum {
    double s, c;
    __host__ __device__ KSum() : s(0.0), c(0.0) {}
    __host__ __device__ void add(double v)
    {
        double t = s + v;
        if (fabs(s) >= fabs(v)) c += (s - t) + v; else c += (v - t) + s;
        s = t;
    }
    __host__ __device__ double value() const { return s + c; }
};
