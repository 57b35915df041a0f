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

// Per-thread constants of a trajectory's cell step, computed once per thread from its GroupParamsF:
// the nonlinear coefficients scaled by dt/2 and the squared loss-noise amplitudes.
struct CellConsts {
    float hdt;                      // dt / 2
    float hg11, hg12, hg22, hdet;   // g_ij dt/2, detuning dt/2
    float hl111, hl12, hl22;        // -l dt/4 (the drift -(l111 na^2 + l12 nb)/2 times dt/2)
    float n1, n2, n3;               // -2 ln 2 (noise_amp c_i)^2
    int itmax;
};

__device__ __forceinline__ CellConsts cell_consts(const GroupParamsF &P)
{
    CellConsts K;
    K.hdt = 0.5f * P.dt;
    K.hg11 = P.g11 * K.hdt;
    K.hg12 = P.g12 * K.hdt;
    K.hg22 = P.g22 * K.hdt;
    K.hdet = P.detuning * K.hdt;
    K.hl111 = -0.5f * K.hdt * P.l111;
    K.hl12 = -0.5f * K.hdt * P.l12;
    K.hl22 = -0.5f * K.hdt * P.l22;
    const float a1 = P.noise_amp * P.c1, a2 = P.noise_amp * P.c2, a3 = P.noise_amp * P.c3;
    K.n1 = -1.38629436112f * a1 * a1;
    K.n2 = -1.38629436112f * a2 * a2;
    K.n3 = -1.38629436112f * a3 * a3;
    K.itmax = P.itmax;
    return K;
}

// One Box-Muller pair of loss_normals6 scaled by an amplitude amp, with the SFU log2/sqrt/sin/cos:
// r = amp sqrt(-2 ln u1) = sqrt(n log2 u1) for n = -2 ln 2 amp^2, u1 = (f1 + 1/2) / 2^21 in (0, 1);
// (n1, n2) = r (cos, sin)(2 pi f2 / 2^21). log2 u1 < 0 for every u1 here: its largest value,
// log2(1 - 2^-22) = -3.4e-7, is twice the SFU log2's absolute error bound on [0.5, 2].
__device__ __forceinline__ float2 box_muller21_scaled(uint32_t f1, uint32_t f2, float n)
{
    const float y = n * __log2f(fmaf((float)f1, 0x1p-21f, 0x1p-22f));
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
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

// |v|^2 and complex products with every fused multiply-add written out, so that every kernel that inlines the
// cell step rounds it the same way (the contraction of a*b + c*d left to the compiler can differ between them)
__device__ __forceinline__ float nrm2(float2 v) { return fmaf(v.x, v.x, v.y * v.y); }
__device__ __forceinline__ float2 cmulx(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}

// The substep's factors da, db from the midpoint estimate (xa, xb).
__device__ __forceinline__ void nonlinear_factors(float2 xa, float2 xb, float hV, float hVd, const CellConsts &K,
                                                  float2 &da, float2 &db)
{
    const float na = nrm2(xa);
    const float nb = nrm2(xb);
    const float ra = fmaf(K.hl111 * na, na, K.hl12 * nb);
    const float rb = fmaf(K.hl22, nb, K.hl12 * na);
    const float ta = fmaf(K.hg11, na, fmaf(K.hg12, nb, hV));
    const float tb = fmaf(K.hg22, nb, fmaf(K.hg12, na, hVd));
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
}

// One cell: v = (a, b) at the start of the substep, V the trap potential.
__device__ __forceinline__ float4 nonlinear_cell(float4 v, float V, const CellConsts &K)
{
    const float2 a0 = make_float2(v.x, v.y), b0 = make_float2(v.z, v.w);
    const float hV = __fmul_rn(V, K.hdt), hVd = __fsub_rn(hV, K.hdet);   // never contracted
    float2 da, db;
    if (K.itmax == 1) {
        // one midpoint iteration (every workload here): the factors of the start values, applied twice
        nonlinear_factors(a0, b0, hV, hVd, K, da, db);
        const float2 ao = cmulx(cmulx(a0, da), da), bo = cmulx(cmulx(b0, db), db);
        return make_float4(ao.x, ao.y, bo.x, bo.y);
    }
    float2 xa = a0, xb = b0;
    da = db = make_float2(0.f, 0.f);
    for (int it = 0; it < K.itmax; ++it) {
        nonlinear_factors(xa, xb, hV, hVd, K, da, db);
        xa = cmulx(a0, da);
        xb = cmulx(b0, db);
    }
    const float2 ao = cmulx(xa, da), bo = cmulx(xb, db);
    return make_float4(ao.x, ao.y, bo.x, bo.y);
}

// The loss-noise increment of one cell from its Philox output, accumulated into out as FMA chains:
//   a += conj(a0)^2 w1 + conj(b0) w2,  b += conj(a0) w2 + conj(b0) w3.
__device__ __forceinline__ float4 loss_noise_apply(float4 out, float4 v0, const CellConsts &K, u32x4 w)
{
    uint32_t f[6];
    loss_fields(w, f);
    const float2 w1 = box_muller21_scaled(f[0], f[1], K.n1);
    const float2 w2 = box_muller21_scaled(f[2], f[3], K.n2);
    const float2 w3 = box_muller21_scaled(f[4], f[5], K.n3);
    const float ax = v0.x, ay = v0.y, bx = v0.z, by = v0.w;
    const float qx = fmaf(ax, ax, -ay * ay), qy = -2.f * ax * ay;       // conj(a0)^2
    return make_float4(fmaf(qx, w1.x, fmaf(-qy, w1.y, fmaf(bx, w2.x, fmaf(by, w2.y, out.x)))),
                       fmaf(qx, w1.y, fmaf(qy, w1.x, fmaf(bx, w2.y, fmaf(-by, w2.x, out.y)))),
                       fmaf(ax, w2.x, fmaf(ay, w2.y, fmaf(bx, w3.x, fmaf(by, w3.y, out.z)))),
                       fmaf(ax, w2.y, fmaf(-ay, w2.x, fmaf(bx, w3.y, fmaf(-by, w3.x, out.w)))));
}

// Adds the loss-noise increments of two cells of the same trajectory and step, evaluated at v0 and v1, to
// out0 and out1: per cell the six normals of one Philox4x32-10 draw (loss_fields) as three complex Wiener
// increments already scaled by their amplitudes. The two draws' rounds interleave; keys: the round keys of
// the ensemble seed (philox_keys).
__device__ __forceinline__ void loss_noise_cell2(float4 &out0, float4 v0, float4 &out1, float4 v1, const CellConsts &K,
                                                 const PhiloxKeys &keys, uint32_t traj, uint32_t step,
                                                 uint32_t cell0, uint32_t cell1)
{
    const u32x4x2 w = philox4x32_10_x2(cell0, step, traj, RNG_TAG_LOSS, cell1, step, traj, RNG_TAG_LOSS, keys);
    out0 = loss_noise_apply(out0, v0, K, w.a);
    out1 = loss_noise_apply(out1, v1, K, w.b);
}


// The loss-noise increments of four consecutive cells cell0 .. cell0 + 3 of the same trajectory and step:
// one interleaved group of four Philox4x32-10 draws.
__device__ __forceinline__ void loss_noise_cell4(float4 out[4], const float4 v0[4], const CellConsts &K,
                                                 const PhiloxKeys &keys, uint32_t traj, uint32_t step, uint32_t cell0)
{
    const u32x4x4 w = philox4x32_10_x4(cell0, step, traj, RNG_TAG_LOSS, keys);
    out[0] = loss_noise_apply(out[0], v0[0], K, w.a);
    out[1] = loss_noise_apply(out[1], v0[1], K, w.b);
    out[2] = loss_noise_apply(out[2], v0[2], K, w.c);
    out[3] = loss_noise_apply(out[3], v0[3], K, w.d);
}
