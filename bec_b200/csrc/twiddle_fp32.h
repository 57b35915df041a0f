// twiddle_fp32.h -- FP32 rotation factors whose modulus is as close to 1 as FP32 allows.
//
// Rounding cos and sin (or the factors f, r of the six-FMA butterfly) to FP32 independently leaves |w| a
// few 1e-8 off 1, and for the handful of constants of the register FFTs the error has one sign (every
// one of them lands inside the unit circle): applied to every element at every step it drains the norm
// coherently, about 2e-7 of the population per split step. The factors are therefore the FP32 values,
// within two units in the last place of the rounded ones, whose modulus is closest to 1. A unit-modulus
// twiddle keeps each butterfly unitary, and the inverse transform, built from the conjugate twiddles,
// still undoes the forward one exactly; the angle moves by at most a few 1e-8. The same holds for the
// kinetic phase factors, which multiply the most populated modes by the same value at every step.
// Host and device, constexpr (compile-time twiddles) or at run time (tables).
#pragma once

#include <cuda_runtime.h>

namespace fftreg {

// spacing of FP32 values at |x| (x a normal FP32 value, not 0)
__host__ __device__ constexpr double fulp(double x)
{
    double a = x < 0 ? -x : x, e = 1.0;
    while (e > a) e *= 0.5;
    while (2.0 * e <= a) e *= 2.0;
    return e * 0x1p-23;
}

__host__ __device__ constexpr double sqrt_newton(double x)
{
    double r = x > 1.0 ? x : 1.0;
    for (int i = 0; i < 64; ++i) r = 0.5 * (r + x / r);
    return r;
}

struct Twid {
    float a, b;
};

// w = f (1 + i r) (or f (r + i)) with |r| <= 1: r within 2 ulp of RN(r0), then f = RN(1 / sqrt(1 + r^2)) with
// the sign of f0, keeping the pair whose f^2 (1 + r^2) is closest to 1. Symmetric in the signs of f0 and r0,
// so a transform and its inverse (r -> -r) take exactly conjugate twiddles.
__host__ __device__ constexpr Twid unit_fr(double f0, double r0)
{
    const double ar = r0 < 0 ? -r0 : r0;
    const double rr = (double)(float)ar;
    double best_e = 1.0, best_f = 0.0, best_r = 0.0;
    for (int j = 0; j <= 4; ++j) {
        const int k = j == 0 ? 0 : (j % 2 ? (j + 1) / 2 : -(j / 2));       // 0, 1, -1, 2, -2
        const double r = rr + k * fulp(rr);
        const double f = (double)(float)(1.0 / sqrt_newton(1.0 + r * r));
        double e = f * f * (1.0 + r * r) - 1.0;
        e = e < 0 ? -e : e;
        if (e < best_e) { best_e = e; best_f = f; best_r = r; }
    }
    return Twid{(float)(f0 < 0 ? -best_f : best_f), (float)(r0 < 0 ? -best_r : best_r)};
}

// w = c + i s: the FP32 pair within 2 ulp of (RN(c0), RN(s0)) whose c^2 + s^2 is closest to 1 (ties: the
// nearer pair). Symmetric in the signs of c0 and s0.
__host__ __device__ constexpr Twid unit_cs(double c0, double s0)
{
    const double ac = c0 < 0 ? -c0 : c0, as = s0 < 0 ? -s0 : s0;
    if (ac == 0.0 || as == 0.0) return Twid{(float)c0, (float)s0};
    const double cr = (double)(float)ac, sr = (double)(float)as;
    const double uc = fulp(cr), us = fulp(sr);
    double best_e = 1.0, best_c = cr, best_s = sr;
    int best_d = 100;
    for (int i = -2; i <= 2; ++i)
        for (int j = -2; j <= 2; ++j) {
            const double c = cr + i * uc, s = sr + j * us;
            double e = c * c + s * s - 1.0;
            e = e < 0 ? -e : e;
            const int d = (i < 0 ? -i : i) + (j < 0 ? -j : j);
            if (e < best_e || (e == best_e && d < best_d)) { best_e = e; best_c = c; best_s = s; best_d = d; }
        }
    return Twid{(float)(c0 < 0 ? -best_c : best_c), (float)(s0 < 0 ? -best_s : best_s)};
}

} // namespace fftreg
