// fft_reg.cuh -- register-resident DFTs of compile-time size.
//
// A thread holds a whole line (N <= 32 elements) in registers; the DFT is a
// fully unrolled radix-2 Cooley-Tukey recursion whose twiddles are
// compile-time constants, so trivial twiddles (1, -i, +i) cost nothing and
// the rest become FMA immediates of six-FMA butterflies (bfly_w). Elements are float2 (one complex value) or
// float4 (the two components a, b of one cell, transformed together).
//
// Twiddle values come from cos_2pi / sin_2pi below: exact octant reduction on the
// integer angle 2 pi k / n, then Taylor series on [0, pi/2) in double
// precision (error ~1e-16), evaluated by the compiler.
#pragma once

#include <utility>

#include "common.cuh"
#include "twiddle_fp32.h"

namespace fftreg {

constexpr double kPi = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double taylor_sin(double x)
{
    double t = x, s = x;
    for (int i = 1; i < 24; ++i) {
        t *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
        s += t;
    }
    return s;
}

__host__ __device__ constexpr double taylor_cos(double x)
{
    double t = 1.0, s = 1.0;
    for (int i = 1; i < 24; ++i) {
        t *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
        s += t;
    }
    return s;
}

// cos(2 pi k / n) and sin(2 pi k / n) for integer k, n > 0
__host__ __device__ constexpr double cos_2pi(long k, long n)
{
    k %= n;
    if (k < 0) k += n;
    const long q = (4 * k) / n, r = 4 * k - q * n;
    const double a = (kPi / 2.0) * (double)r / (double)n;
    const double sa = taylor_sin(a), ca = taylor_cos(a);
    return q == 0 ? ca : q == 1 ? -sa : q == 2 ? -ca : sa;
}

__host__ __device__ constexpr double sin_2pi(long k, long n)
{
    k %= n;
    if (k < 0) k += n;
    const long q = (4 * k) / n, r = 4 * k - q * n;
    const double a = (kPi / 2.0) * (double)r / (double)n;
    const double sa = taylor_sin(a), ca = taylor_cos(a);
    return q == 0 ? sa : q == 1 ? ca : q == 2 ? -sa : -ca;
}

// ---- element operations ----------------------------------------------------
__device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float4 add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 sub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }

// v * (c + i s)
// Complex products with the fused multiply-adds written out, so that a float2 and a float4 caller round
// every component the same way (left to the compiler, the contraction of a*b - c*d can differ between them).
__device__ __forceinline__ float2 cmulc(float2 v, float c, float s)
{
    return make_float2(fmaf(v.x, c, -(v.y * s)), fmaf(v.x, s, v.y * c));
}
__device__ __forceinline__ float4 cmulc(float4 v, float c, float s)
{
    const float2 a = cmulc(make_float2(v.x, v.y), c, s), b = cmulc(make_float2(v.z, v.w), c, s);
    return make_float4(a.x, a.y, b.x, b.y);
}
// v * (-i)
__device__ __forceinline__ float2 mul_negi(float2 v) { return make_float2(v.y, -v.x); }
__device__ __forceinline__ float4 mul_negi(float4 v) { return make_float4(v.y, -v.x, v.w, -v.z); }
// v * (+i)
__device__ __forceinline__ float2 mul_posi(float2 v) { return make_float2(-v.y, v.x); }
__device__ __forceinline__ float4 mul_posi(float4 v) { return make_float4(-v.y, v.x, -v.w, v.z); }

// v * w with w a runtime complex (float2)
__device__ __forceinline__ float2 cmulw(float2 v, float2 w) { return cmulc(v, w.x, w.y); }
__device__ __forceinline__ float4 cmulw(float4 v, float2 w) { return cmulc(v, w.x, w.y); }
// m0 a + m1 b, every rounding fixed
__device__ __forceinline__ float2 cmix(float2 m0, float2 a, float2 m1, float2 b)
{
    return make_float2(fmaf(m0.x, a.x, fmaf(-m0.y, a.y, fmaf(m1.x, b.x, -(m1.y * b.y)))),
                       fmaf(m0.x, a.y, fmaf(m0.y, a.x, fmaf(m1.x, b.y, m1.y * b.x))));
}

// ---- butterfly with a constant twiddle -------------------------------------------
// x0 = e + w o, x1 = e - w o for the compile-time twiddle w = c + i s, in six FMAs per complex value
// (Linzer and Feig, "Implementation of efficient FFT algorithms on fused multiply-add architectures",
// IEEE Trans. Signal Processing 41, 1993): the larger of |c|, |s| is factored out, so with r = s / c
// (or c / s) of magnitude <= 1, w o = c (o.re - r o.im, o.im + r o.re) (or s (r o.re - o.im, o.re + r o.im)),
// and both outputs are one FMA each from e.
__device__ __forceinline__ void bfly_c(float2 &x0, float2 &x1, float2 e, float2 o, float f, float r)
{
    const float ur = fmaf(-r, o.y, o.x), ui = fmaf(r, o.x, o.y);
    x0 = make_float2(fmaf(f, ur, e.x), fmaf(f, ui, e.y));
    x1 = make_float2(fmaf(-f, ur, e.x), fmaf(-f, ui, e.y));
}
__device__ __forceinline__ void bfly_s(float2 &x0, float2 &x1, float2 e, float2 o, float f, float r)
{
    const float ur = fmaf(r, o.x, -o.y), ui = fmaf(r, o.y, o.x);
    x0 = make_float2(fmaf(f, ur, e.x), fmaf(f, ui, e.y));
    x1 = make_float2(fmaf(-f, ur, e.x), fmaf(-f, ui, e.y));
}

// the butterfly of twiddle w = e^{-+2 pi i K / N} (sign - forward, + when INV)
// UNIT: the factors of modulus closest to 1 (twiddle_fp32.h; the real-time passes, where a modulus error
// drains the norm at every step), else the nearest FP32 factors (the imaginary-time passes, which
// renormalise at every step and gain nothing from the modulus)
template <int K, int N, bool INV, bool UNIT = true>
__device__ __forceinline__ void bfly_w(float2 &x0, float2 &x1, float2 e, float2 o)
{
    constexpr double c = cos_2pi(K, N), s = INV ? sin_2pi(K, N) : -sin_2pi(K, N);
    if constexpr ((c < 0 ? -c : c) >= (s < 0 ? -s : s)) {
        constexpr Twid t = UNIT ? unit_fr(c, s / c) : Twid{(float)c, (float)(s / c)};
        bfly_c(x0, x1, e, o, t.a, t.b);
    } else {
        constexpr Twid t = UNIT ? unit_fr(s, c / s) : Twid{(float)s, (float)(c / s)};
        bfly_s(x0, x1, e, o, t.a, t.b);
    }
}
template <int K, int N, bool INV, bool UNIT = true>
__device__ __forceinline__ void bfly_w(float4 &x0, float4 &x1, float4 e, float4 o)
{
    float2 a0, a1, b0, b1;
    bfly_w<K, N, INV, UNIT>(a0, a1, make_float2(e.x, e.y), make_float2(o.x, o.y));
    bfly_w<K, N, INV, UNIT>(b0, b1, make_float2(e.z, e.w), make_float2(o.z, o.w));
    x0 = make_float4(a0.x, a0.y, b0.x, b0.y);
    x1 = make_float4(a1.x, a1.y, b1.x, b1.y);
}

// ---- DFT ---------------------------------------------------------------------
// x[k] <- sum_n x[n] exp(-+2 pi i n k / N) (sign - forward, + when INV), unnormalised; UNIT as bfly_w.
template <int N, bool INV, bool UNIT = true, typename T>
__device__ __forceinline__ void dft(T *x);

template <int N, bool INV, bool UNIT, int K, typename T>
__device__ __forceinline__ void combine_one(T *x, const T *e, const T *o)
{
    if constexpr (K == 0 || 4 * K == N) {
        const T t = K == 0 ? o[K] : INV ? mul_posi(o[K]) : mul_negi(o[K]);
        x[K] = add(e[K], t);
        x[K + N / 2] = sub(e[K], t);
    } else {
        bfly_w<K, N, INV, UNIT>(x[K], x[K + N / 2], e[K], o[K]);
    }
}

template <int N, bool INV, bool UNIT, typename T, int... K>
__device__ __forceinline__ void combine_all(T *x, const T *e, const T *o, std::integer_sequence<int, K...>)
{
    (combine_one<N, INV, UNIT, K>(x, e, o), ...);
}

template <int N, bool INV, bool UNIT, typename T>
__device__ __forceinline__ void dft(T *x)
{
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        const T a = x[0], b = x[1];
        x[0] = add(a, b);
        x[1] = sub(a, b);
    } else {
        T e[N / 2], o[N / 2];
#pragma unroll
        for (int k = 0; k < N / 2; ++k) {
            e[k] = x[2 * k];
            o[k] = x[2 * k + 1];
        }
        dft<N / 2, INV, UNIT>(e);
        dft<N / 2, INV, UNIT>(o);
        combine_all<N, INV, UNIT>(x, e, o, std::make_integer_sequence<int, N / 2>{});
    }
}

} // namespace fftreg
