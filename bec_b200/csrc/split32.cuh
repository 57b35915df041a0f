// split32.cuh -- a 32-point line transform shared by lane L of two warps (h = warp), 16 elements each.
//
// Used by the 32 x 32 plane passes, where a line held by one lane would take twice the registers and
// cap the warps per SM. Forward transforms are split by decimation in time: x[2j + h] in, a local
// 16-point DFT, one exchange of 8 values through shared memory, X[k] out in the block layout
// kblk(s, h) (h = 0: k = 0..7, 16..23; h = 1: k = 8..15, 24..31). Inverse transforms use decimation in
// frequency with the conjugate twiddles: block layout in, x[2m + h] out, which is the layout the next
// forward step expects. (Written as conj(FFT(conj v)) instead, the sign flips cost the real-time plane
// pass a 52-byte register spill and 4 % of its time.) tix() is the XOR swizzle of a 32 x 32 shared tile.
// Elements are float4 (the two components of a cell, real-time passes) or float2 (one component,
// imaginary-time passes).
#pragma once

#include <utility>

#include "fft_reg.cuh"

namespace split32 {

__device__ __forceinline__ int kblk(int s, int h) { return s < 8 ? s + 8 * h : s + 8 + 8 * h; }
__device__ __forceinline__ int tix(int row, int col) { return row * 32 + (col ^ (row & 7)); }

// v * e^{-2 pi i K / 32} (v * e^{+2 pi i K / 32} when INV)
template <int K, bool INV = false, typename T>
__device__ __forceinline__ T w32(T v)
{
    if constexpr (K == 0) {
        return v;
    } else if constexpr (K == 8) {
        return INV ? fftreg::mul_posi(v) : fftreg::mul_negi(v);
    } else {
        constexpr fftreg::Twid t =
            fftreg::unit_cs(fftreg::cos_2pi(K, 32), INV ? fftreg::sin_2pi(K, 32) : -fftreg::sin_2pi(K, 32));
        return fftreg::cmulc(v, t.a, t.b);
    }
}

// decimation in time, after the local DFT16: H = 0 keeps Y0[I] and receives Y1[I] -> X[I], X[16 + I];
// H = 1 keeps Y1[8 + I] and receives Y0[8 + I] -> X[8 + I], X[24 + I]
template <int H, int I, typename T>
__device__ __forceinline__ void dit_send_one(const T *v, T *xo) { xo[I * 32] = H == 0 ? v[8 + I] : v[I]; }
template <int H, int I, typename T>
__device__ __forceinline__ void dit_recv_one(T *v, const T *xi)
{
    const T r = xi[I * 32];
    const T e = H == 0 ? v[I] : r;
    const T o = H == 0 ? r : v[8 + I];
    constexpr int K = H == 0 ? I : 8 + I;
    if constexpr (K == 0 || K == 8) {
        const T t = w32<K>(o);
        v[I] = fftreg::add(e, t);
        v[8 + I] = fftreg::sub(e, t);
    } else {
        fftreg::bfly_w<K, 32, false>(v[I], v[8 + I], e, o);
    }
}
// decimation in frequency, before the local DFT16: n = I (H = 0) or 8 + I (H = 1),
// a[n] = x[n] + x[n + 16], b[n] = (x[n] - x[n + 16]) W^n; H = 0 gathers a[0..15], H = 1 b[0..15]
template <int H, int I, typename T>
__device__ __forceinline__ void dif_send_one(T *v, T *xo)
{
    const T a = fftreg::add(v[I], v[8 + I]);
    const T b = w32<H == 0 ? I : 8 + I, true>(fftreg::sub(v[I], v[8 + I]));
    if constexpr (H == 0) {
        v[I] = a;
        xo[I * 32] = b;
    } else {
        v[8 + I] = b;
        xo[I * 32] = a;
    }
}
template <int H, int I, typename T>
__device__ __forceinline__ void dif_recv_one(T *v, const T *xi)
{
    if constexpr (H == 0) v[8 + I] = xi[I * 32];
    else v[I] = xi[I * 32];
}

template <int H, typename T, int... I>
__device__ __forceinline__ void dit_send(const T *v, T *xo, std::integer_sequence<int, I...>) { (dit_send_one<H, I>(v, xo), ...); }
template <int H, typename T, int... I>
__device__ __forceinline__ void dit_recv(T *v, const T *xi, std::integer_sequence<int, I...>) { (dit_recv_one<H, I>(v, xi), ...); }
template <int H, typename T, int... I>
__device__ __forceinline__ void dif_send(T *v, T *xo, std::integer_sequence<int, I...>) { (dif_send_one<H, I>(v, xo), ...); }
template <int H, typename T, int... I>
__device__ __forceinline__ void dif_recv(T *v, const T *xi, std::integer_sequence<int, I...>) { (dif_recv_one<H, I>(v, xi), ...); }

using Seq8 = std::make_integer_sequence<int, 8>;

// forward: v[j] = x[2j + h] -> v[s] = X[kblk(s, h)]; xb: the plane's exchange slots [2][8][32];
// bar(): the barrier of the plane's two warps
template <typename T, typename Bar>
__device__ __forceinline__ void fwd_line(T *v, T *xb, int h, int lane, Bar bar)
{
    fftreg::dft<16, false>(v);
    T *xo = xb + h * 256 + lane;
    const T *xi = xb + (1 - h) * 256 + lane;
    if (h == 0) dit_send<0>(v, xo, Seq8{});
    else dit_send<1>(v, xo, Seq8{});
    bar();
    if (h == 0) dit_recv<0>(v, xi, Seq8{});
    else dit_recv<1>(v, xi, Seq8{});
}

// inverse (unnormalised): v[s] = x[kblk(s, h)] -> v[m] = y[2m + h]
template <typename T, typename Bar>
__device__ __forceinline__ void inv_line(T *v, T *xb, int h, int lane, Bar bar)
{
    T *xo = xb + h * 256 + lane;
    const T *xi = xb + (1 - h) * 256 + lane;
    if (h == 0) dif_send<0>(v, xo, Seq8{});
    else dif_send<1>(v, xo, Seq8{});
    bar();
    if (h == 0) dif_recv<0>(v, xi, Seq8{});
    else dif_recv<1>(v, xi, Seq8{});
    fftreg::dft<16, true>(v);
}

} // namespace split32
