// physics.cuh -- the per-cell real-space step of the FP32 path, shared by the
// plane-pass kernels.
//
// propagateXSpaceTwoComponent (programs/bec_wigner_3d.cuda/wigner_kernel.cu:184-229):
// itmax midpoint iterations of the exponential integrator
//   pa = -(l111 na^2 + l12 nb)/2 + i (V + g11 na + g12 nb)
//   pb = -(l22 nb + l12 na)/2  + i (V + g22 nb + g12 na - detuning)
//   d  = exp(p dt/2),  psi = psi0 d  (x itmax),  out = psi d
// (the reference's sign: evolution by e^{+i H dt}, wigner_kernel.cu:206-215),
// followed by the Wigner loss-noise increment at the start of the substep:
//   a += 3 sqrt(l111/6) conj(a0)^2 dW1 + sqrt(l12/2) conj(b0) dW2
//   b +=   sqrt(l12/2)  conj(a0)   dW2 + sqrt(l22)   conj(b0) dW3,
// dW complex normal with <|dW|^2> = dt / dV; the six normals of a cell and step
// come from one Philox4x32-10 draw keyed by the ensemble seed with counter
// (cell, step, trajectory, 1) (loss_normals6, common.cuh).
#pragma once

#include "common.cuh"
#include "engine.h"

// One Box-Muller pair of loss_normals6 scaled by amp, with the SFU log2/rsqrt/sin/cos:
// r = amp sqrt(-2 ln u1), u1 = (f1 + 1/2) / 2^21 in (0, 1) so -2 ln u1 > 0 and the square root
// is taken as y rsqrt(y); (n1, n2) = r (cos, sin)(2 pi f2 / 2^21).
__device__ __forceinline__ float2 box_muller21_scaled(uint32_t f1, uint32_t f2, float amp)
{
    const float y = -1.38629436112f * __log2f(fmaf((float)f1, 0x1p-21f, 0x1p-22f));
    const float r = amp * (y * rsqrtf(y));
    float s, c;
    __sincosf((float)f2 * (6.28318530717958648f * 0x1p-21f), &s, &c);
    return make_float2(r * c, r * s);
}

// Phase and decay factors of the nonlinear substep. On the bench workloads |t| = |Im p| dt/2 stays below
// 0.38 and |Re p| dt/2 below 1e-6, so every cell takes the polynomial branch:
//   cos t, sin t: Taylor in u = t^2, Horner form, for |t| <= 0.5; sin to t^7 (truncation <= 0.5^9/9! = 5.4e-9),
//     cos to t^8 (<= 0.5^10/10! = 2.7e-10), both below half an FP32 ulp of the result;
//   exp x: Taylor to x^3 for |x| <= 1/64 (truncation <= (1/64)^4/4! = 2.5e-9).
// Arguments outside those ranges take sincosf / expf; one branch covers all four arguments of a cell.
__device__ __forceinline__ float2 cis_taylor(float t)
{
    const float u = t * t;
    const float s = fmaf(t * u, fmaf(u, fmaf(u, -1.f / 5040.f, 1.f / 120.f), -1.f / 6.f), t);
    const float c = fmaf(u, fmaf(u, fmaf(u, fmaf(u, 1.f / 40320.f, -1.f / 720.f), 1.f / 24.f), -0.5f), 1.f);
    return make_float2(c, s);
}

__device__ __forceinline__ float exp_taylor(float x) { return fmaf(x, fmaf(x, fmaf(x, 1.f / 6.f, 0.5f), 1.f), 1.f); }

// One cell: v = (a, b) at the start of the substep, V the trap potential.
__device__ __forceinline__ float4 nonlinear_cell(float4 v, float V, const GroupParamsF &P)
{
    const float2 a0 = make_float2(v.x, v.y), b0 = make_float2(v.z, v.w);
    const float hdt = P.dt * 0.5f;
    float2 xa = a0, xb = b0, da = make_float2(0.f, 0.f), db = make_float2(0.f, 0.f);
    for (int it = 0; it < P.itmax; ++it) {
        const float na = xa.x * xa.x + xa.y * xa.y;
        const float nb = xb.x * xb.x + xb.y * xb.y;
        const float ra = -(P.l111 * na * na + P.l12 * nb) * 0.5f * hdt;
        const float ta = (V + P.g11 * na + P.g12 * nb) * hdt;
        const float rb = -(P.l22 * nb + P.l12 * na) * 0.5f * hdt;
        const float tb = (V + P.g22 * nb + P.g12 * na - P.detuning) * hdt;
        float2 ea, eb;
        float ma, mb;
        if (fmaxf(fabsf(ta), fabsf(tb)) <= 0.5f && fmaxf(fabsf(ra), fabsf(rb)) <= 0.015625f) {
            ea = cis_taylor(ta);
            eb = cis_taylor(tb);
            ma = exp_taylor(ra);
            mb = exp_taylor(rb);
        } else {
            sincosf(ta, &ea.y, &ea.x);
            sincosf(tb, &eb.y, &eb.x);
            ma = expf(ra);
            mb = expf(rb);
        }
        da = make_float2(ma * ea.x, ma * ea.y);
        db = make_float2(mb * eb.x, mb * eb.y);
        xa = cmul(a0, da);
        xb = cmul(b0, db);
    }
    const float2 ao = cmul(xa, da), bo = cmul(xb, db);
    return make_float4(ao.x, ao.y, bo.x, bo.y);
}

// Loss-noise amplitudes of a trajectory: noise_amp x (c1, c2, c3), computed once per thread.
struct LossAmps { float w1, w2, w3; };
__device__ __forceinline__ LossAmps loss_amps(const GroupParamsF &P)
{
    return LossAmps{P.noise_amp * P.c1, P.noise_amp * P.c2, P.noise_amp * P.c3};
}

// The increment of loss_noise_cell from a given Philox output.
__device__ __forceinline__ float4 loss_noise_apply(float4 out, float4 v0, const LossAmps &A, u32x4 w)
{
    uint32_t f[6];
    loss_fields(w, f);
    const float2 w1 = box_muller21_scaled(f[0], f[1], A.w1);
    const float2 w2 = box_muller21_scaled(f[2], f[3], A.w2);
    const float2 w3 = box_muller21_scaled(f[4], f[5], A.w3);
    const float2 ca = make_float2(v0.x, -v0.y), cb = make_float2(v0.z, -v0.w);
    const float2 da = cadd(cmul(cmul(ca, ca), w1), cmul(cb, w2));
    const float2 db = cadd(cmul(ca, w2), cmul(cb, w3));
    return make_float4(out.x + da.x, out.y + da.y, out.z + db.x, out.w + db.y);
}

// loss_noise_cell for two cells of the same trajectory and step (interleaved Philox draws).
__device__ __forceinline__ void loss_noise_cell2(float4 &out0, float4 v0, float4 &out1, float4 v1, const LossAmps &A,
                                                 uint32_t k0, uint32_t k1, uint32_t traj, uint32_t step,
                                                 uint32_t cell0, uint32_t cell1)
{
    const u32x4x2 w = philox4x32_10_x2(cell0, step, traj, RNG_TAG_LOSS, cell1, step, traj, RNG_TAG_LOSS, k0, k1);
    out0 = loss_noise_apply(out0, v0, A, w.a);
    out1 = loss_noise_apply(out1, v1, A, w.b);
}

// Adds the loss-noise increment evaluated at v0 to out: the six normals of one Philox4x32-10 draw
// (loss_fields) as three complex Wiener increments w1, w2, w3 already scaled by their amplitudes.
__device__ __forceinline__ float4 loss_noise_cell(float4 out, float4 v0, const LossAmps &A, uint32_t k0,
                                                  uint32_t k1, uint32_t traj, uint32_t step, uint32_t cell)
{
    return loss_noise_apply(out, v0, A, philox4x32_10(cell, step, traj, RNG_TAG_LOSS, k0, k1));
}
