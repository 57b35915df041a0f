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

// loss_normals6 with the SFU log/sin/cos
__device__ __forceinline__ void box_muller21_fast(uint32_t f1, uint32_t f2, float &n1, float &n2)
{
    const float r = sqrtf(-2.0f * __logf(fmaf((float)f1, 0x1p-21f, 0x1p-22f)));
    float s, c;
    __sincosf(6.28318530717958648f * ((float)f2 * 0x1p-21f), &s, &c);
    n1 = r * c;
    n2 = r * s;
}

__device__ __forceinline__ void loss_normals6_fast(uint32_t k0, uint32_t k1, uint32_t traj, uint32_t step,
                                                   uint32_t cell, float out[6])
{
    uint32_t f[6];
    loss_fields(philox4x32_10(cell, step, traj, RNG_TAG_LOSS, k0, k1), f);
    box_muller21_fast(f[0], f[1], out[0], out[1]);
    box_muller21_fast(f[2], f[3], out[2], out[3]);
    box_muller21_fast(f[4], f[5], out[4], out[5]);
}

// (cos t, sin t): Taylor series in t^2 for |t| <= 0.5 (truncation < 1.2e-11, below
// FP32 rounding), sincosf beyond.
__device__ __forceinline__ float2 cis_small(float t)
{
    if (fabsf(t) <= 0.5f) {
        const float u = t * t;
        const float s = t * (1.f - u * (1.f / 6.f) * (1.f - u * (1.f / 20.f) * (1.f - u * (1.f / 42.f) *
                                                                                    (1.f - u * (1.f / 72.f)))));
        const float c = 1.f - u * 0.5f * (1.f - u * (1.f / 12.f) * (1.f - u * (1.f / 30.f) *
                                                                   (1.f - u * (1.f / 56.f) * (1.f - u * (1.f / 90.f)))));
        return make_float2(c, s);
    }
    float s, c;
    sincosf(t, &s, &c);
    return make_float2(c, s);
}

// exp(x): Taylor series for |x| <= 1/64 (truncation < 1e-11), expf beyond.
__device__ __forceinline__ float exp_small(float x)
{
    if (fabsf(x) <= 0.015625f)
        return 1.f + x * (1.f + x * 0.5f * (1.f + x * (1.f / 3.f) * (1.f + x * 0.25f * (1.f + x * 0.2f))));
    return expf(x);
}

// One cell: v = (a, b) at the start of the substep, V the trap potential.
__device__ __forceinline__ float4 nonlinear_cell(float4 v, float V, const GroupParamsF &P)
{
    const float2 a0 = make_float2(v.x, v.y), b0 = make_float2(v.z, v.w);
    const float hdt = P.dt * 0.5f;
    float2 xa = a0, xb = b0, da = make_float2(0.f, 0.f), db = make_float2(0.f, 0.f);
    for (int it = 0; it < P.itmax; ++it) {
        const float na = xa.x * xa.x + xa.y * xa.y;
        const float nb = xb.x * xb.x + xb.y * xb.y;
        const float pa_re = -(P.l111 * na * na + P.l12 * nb) * 0.5f;
        const float pa_im = V + P.g11 * na + P.g12 * nb;
        const float pb_re = -(P.l22 * nb + P.l12 * na) * 0.5f;
        const float pb_im = V + P.g22 * nb + P.g12 * na - P.detuning;
        const float2 ea = cis_small(pa_im * hdt), eb = cis_small(pb_im * hdt);
        const float ma = exp_small(pa_re * hdt), mb = exp_small(pb_re * hdt);
        da = make_float2(ma * ea.x, ma * ea.y);
        db = make_float2(mb * eb.x, mb * eb.y);
        xa = cmul(a0, da);
        xb = cmul(b0, db);
    }
    const float2 ao = cmul(xa, da), bo = cmul(xb, db);
    return make_float4(ao.x, ao.y, bo.x, bo.y);
}

// Adds the loss-noise increment evaluated at v0 to out.
__device__ __forceinline__ float4 loss_noise_cell(float4 out, float4 v0, const GroupParamsF &P, uint32_t traj,
                                                  uint32_t step, uint32_t cell)
{
    float r[6];
    loss_normals6_fast(P.seed_lo, P.seed_hi, traj, step, cell, r);
    const float s = P.noise_amp;
    const float2 w1 = make_float2(s * r[0], s * r[1]);
    const float2 w2 = make_float2(s * r[2], s * r[3]);
    const float2 w3 = make_float2(s * r[4], s * r[5]);
    const float2 ca = make_float2(v0.x, -v0.y), cb = make_float2(v0.z, -v0.w);
    const float2 da = cadd(cmul(cscale(cmul(ca, ca), P.c1), w1), cmul(cscale(cb, P.c2), w2));
    const float2 db = cadd(cmul(cscale(ca, P.c2), w2), cmul(cscale(cb, P.c3), w3));
    return make_float4(out.x + da.x, out.y + da.y, out.z + db.x, out.w + db.y);
}
