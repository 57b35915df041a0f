// step_bodies.cuh -- the register-resident plane and pencil passes of the FP32 path as device bodies.
//
// One split step of the reference (propagate, programs/bec_wigner_3d.cuda/wigner.cu:178-199) is
// regrouped into a pencil pass (IFFT_z -> kinetic phase [-> pulse] -> FFT_z) and a plane pass
// (FFT_xy -> nonlinear + losses + loss noise -> IFFT_xy) over the stored representation (k-space
// along x and y, x-space along z; see batched_fp32.cu). Every line of the 3D transform lives in one
// thread's registers (or, for 32-point lines, in one lane of each of two warps); shared memory only
// transposes.
//
// The bodies run on a "virtual block" (VBlock): a contiguous group of a CTA's threads with its own
// index and barrier. The standalone kernels (fused_passes.cu) give each body a whole CTA; the fused
// step kernel (step_kernel.cu) runs several virtual blocks of one item side by side in a 256-thread
// CTA, each synchronising on its own named barrier.
//
// plane pass (square planes N x N, N = 8, 16): one warp per 32/N planes. Lane c loads column c of its
//   plane from HBM (each load instruction of the warp reads consecutive 16-byte cells), transforms it
//   along y, writes it to an XOR-swizzled shared tile, reads back row c, transforms along x, applies
//   the nonlinear / loss / loss-noise step to its N cells, and returns the same way. Both components of
//   a cell are one float4.
// plane pass, 32 x 32 planes: two warps per plane, a 32-point line shared by lane L of each warp
//   (split32.cuh).
// pencil pass (nz = 64, 128, 256 = 16 G): 16 adjacent pencils of a trajectory per virtual block of
//   nz threads. A four-step decomposition nz = 16 x G: each thread holds 16 elements (z = j + G m)
//   and does a 16-point DFT, twiddles, and after one shared-memory transpose a G-point DFT across j;
//   the kinetic phase e^{i k^2/2 dt} (wigner_kernel.cu:137-151) is applied in full k-space as the
//   product of a per-pencil (kx, ky) factor and a per-kz factor; the forward transform retraces the
//   same steps.
//
// Shared tiles are swizzled on the 16-byte unit index (col ^ (row & 7)) so that both the row-wise
// and the column-wise access of a quarter warp touch eight different bank groups.
//
// The plane bodies read the state with ld.global.cg (L2 only): inside the fused step kernel another
// SM's pencil item wrote those lines during the same launch, and L1 is not coherent across SMs.
#pragma once

#include "engine.h"
#include "fft_reg.cuh"
#include "physics.cuh"
#include "split32.cuh"

namespace stepk {

using fftreg::dft;

// A group of nthr consecutive threads of a CTA acting as one block.
struct VBlock {
    int tid;     // thread index within the group
    int bid;     // block index the body works on
    int bar;     // barrier: 0 = the whole CTA (__syncthreads), else a named barrier of nthr threads
    int nthr;
    __device__ __forceinline__ void sync() const
    {
        if (bar == 0) __syncthreads();
        else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nthr) : "memory");
    }
};

// ---------------------------------------------------------------- plane pass, N = 8, 16
// 4 warps (128 threads); tile: 4 warps x (32 / N) planes x N^2 float4
// SMEM: `state` is a trajectory held in shared memory and `tile` is the same memory (the transposes run in
// place): plain loads instead of L2-only ones, and the warp's loads all done before its first store.
template <int N, bool SMEM = false>
__device__ __forceinline__ void plane_body(const VBlock &vb, float4 *__restrict__ state, int nz, int cells,
                                           const GroupParamsF *__restrict__ gp, const int *__restrict__ tgroup,
                                           const int *__restrict__ tlocal, uint32_t step, float4 *tile)
{
    constexpr int W = 32 / N;          // planes per warp
    constexpr int PLANE = N * N;
    const int warp = vb.tid >> 5, lane = vb.tid & 31;
    const int wp = lane / N, c = lane % N;
    const int plane_id = (vb.bid * 4 + warp) * W + wp;
    const int traj = plane_id / nz, z = plane_id - traj * nz;
    float4 *__restrict__ g = state + (size_t)traj * cells + (size_t)z * PLANE;
    float4 *s = tile + (warp * W + wp) * PLANE;

    const GroupParamsF P = gp[tgroup[traj]];

    float4 v[N];
#pragma unroll
    for (int y = 0; y < N; ++y) v[y] = SMEM ? g[y * N + c] : __ldcg(g + y * N + c);
    if (SMEM) __syncwarp();

    // Four transforms share one loop body (the kernel is otherwise bound by
    // instruction fetch): pass 0 forward along y, pass 1 forward along x,
    // passes 2 and 3 inverse along x and y (the inverse DFT body, no sign flips).
#pragma unroll 1
    for (int pass = 0; pass < 4; ++pass) {
        if (pass >= 2) dft<N, true>(v);
        else dft<N, false>(v);
        if (pass == 0) {
            // column c -> row c
#pragma unroll
            for (int y = 0; y < N; ++y) s[y * N + (c ^ (y & 7))] = v[y];
            __syncwarp();
#pragma unroll
            for (int x = 0; x < N; ++x) v[x] = s[c * N + (x ^ (c & 7))];
        } else if (pass == 1) {
            // lane c owns row y = c: the cells go through the physics one at a time
            // from its own shared row (a rolled loop keeps the kernel small)
#pragma unroll
            for (int x = 0; x < N; ++x) s[c * N + (x ^ (c & 7))] = v[x];
            // coordinates and trap potential with every fused multiply-add written out (same bits in every kernel)
            const float Y = fmaf(P.dy, (float)c, -P.ymax);
            const float Z = fmaf(P.dz, (float)z, -P.zmax);
            const float base = fmaf(Y, Y, (Z * Z) * P.inv_lambda2);
            const uint32_t tl = (uint32_t)tlocal[traj];
            const CellConsts K = cell_consts(P);
            const uint32_t cell0 = (uint32_t)(z * PLANE + c * N);
            const PhiloxKeys keys = philox_keys(P.seed_lo, P.seed_hi);
            // cells in fours: the four Philox draws interleave (loss_noise_cell4)
#pragma unroll 1
            for (int x = 0; x < N; x += 4) {
                float4 v0[4], o[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float X = fmaf(P.dx, (float)(x + q), -P.xmax);
                    v0[q] = s[c * N + ((x + q) ^ (c & 7))];
                    o[q] = nonlinear_cell(v0[q], 0.5f * fmaf(X, X, base), K);
                }
                if (P.noise) loss_noise_cell4(o, v0, K, keys, tl, step, cell0 + x);
#pragma unroll
                for (int q = 0; q < 4; ++q) s[c * N + ((x + q) ^ (c & 7))] = o[q];
            }
#pragma unroll
            for (int x = 0; x < N; ++x) v[x] = s[c * N + (x ^ (c & 7))];
        } else if (pass == 2) {
            // row c -> column c
#pragma unroll
            for (int x = 0; x < N; ++x) s[c * N + (x ^ (c & 7))] = v[x];
            __syncwarp();
#pragma unroll
            for (int y = 0; y < N; ++y) v[y] = s[y * N + (c ^ (y & 7))];
        }
    }
    if (SMEM) __syncwarp();
#pragma unroll
    for (int y = 0; y < N; ++y) g[y * N + c] = v[y];
}

// ---------------------------------------------------------------- plane pass, 32 x 32, two warps a plane
// 64 threads; every 32-point line is shared by lane L of warp 0 and lane L of warp 1, 16 elements
// each, half the registers of a one-lane line, so more warps fit on an SM. tile: 1024 float4 (the
// plane, swizzled like plane_body's), xb: 512 float4 (the line exchange slots).
__device__ __forceinline__ void plane32_body(const VBlock &vb, float4 *__restrict__ state, int nz, int cells,
                                             const GroupParamsF *__restrict__ gp, const int *__restrict__ tgroup,
                                             const int *__restrict__ tlocal, uint32_t step, float4 *tile, float4 *xb)
{
    using namespace split32;
    const int h = vb.tid >> 5, lane = vb.tid & 31;
    const int plane_id = vb.bid;
    const int traj = plane_id / nz, z = plane_id - traj * nz;
    float4 *__restrict__ g = state + (size_t)traj * cells + (size_t)z * 1024;
    const GroupParamsF P = gp[tgroup[traj]];
    auto bar = [&vb]() { vb.sync(); };

    float4 v[16];
    // forward along y (lane = column), then along x (lane = row); shared code body
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = __ldcg(g + (2 * j + h) * 32 + lane);
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = tile[tix(lane, 2 * j + h)];
        }
        fwd_line(v, xb, h, lane, bar);
        if (pass == 0) {
#pragma unroll
            for (int s = 0; s < 16; ++s) tile[tix(kblk(s, h), lane)] = v[s];
            vb.sync();
        }
    }
    // x-space: lane owns row y = lane, cells x = kblk(s, h); the physics runs as a rolled loop
    // over those cells in the tile
    {
        const int r = lane;
#pragma unroll
        for (int s = 0; s < 16; ++s) tile[tix(r, kblk(s, h))] = v[s];
        const float Y = fmaf(P.dy, (float)r, -P.ymax);
        const float Z = fmaf(P.dz, (float)z, -P.zmax);
        const float base = fmaf(Y, Y, (Z * Z) * P.inv_lambda2);
        const uint32_t tl = (uint32_t)tlocal[traj];
        const CellConsts K = cell_consts(P);
        const uint32_t cell0 = (uint32_t)(z * 1024 + r * 32);
        const PhiloxKeys keys = philox_keys(P.seed_lo, P.seed_hi);
        // cells in pairs (x, x + 1; kblk keeps pairs of even s adjacent): the two Philox draws interleave.
        // (Fours measured slower here: the larger loop body misses in the instruction cache.)
#pragma unroll 1
        for (int s = 0; s < 16; s += 2) {
            const int x = kblk(s, h);
            const float X0 = fmaf(P.dx, (float)x, -P.xmax), X1 = fmaf(P.dx, (float)(x + 1), -P.xmax);
            float4 *s0 = tile + tix(r, x), *s1 = tile + tix(r, x + 1);
            const float4 v0 = *s0, v1 = *s1;
            float4 o0 = nonlinear_cell(v0, 0.5f * fmaf(X0, X0, base), K);
            float4 o1 = nonlinear_cell(v1, 0.5f * fmaf(X1, X1, base), K);
            if (P.noise)
                loss_noise_cell2(o0, v0, o1, v1, K, keys, tl, step, cell0 + x, cell0 + x + 1);
            *s0 = o0;
            *s1 = o1;
        }
#pragma unroll
        for (int s = 0; s < 16; ++s) v[s] = tile[tix(r, kblk(s, h))];
    }
    vb.sync();    // the partner's physics is done with the row, and its last exchange reads too
    // inverse along x (lane = row), then along y (lane = column); shared code body
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
#pragma unroll
            for (int s = 0; s < 16; ++s) v[s] = tile[tix(kblk(s, h), lane)];
        }
        inv_line(v, xb, h, lane, bar);
        if (pass == 0) {
#pragma unroll
            for (int m = 0; m < 16; ++m) tile[tix(lane, 2 * m + h)] = v[m];
            vb.sync();
        }
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) g[(2 * m + h) * 32 + lane] = v[m];
}

// ---------------------------------------------------------------- pencil pass
// 8-byte global -> shared copy that completes asynchronously (cp.async), and the wait for this thread's copies
__device__ __forceinline__ void copy_async8(float2 *dst_smem, const float2 *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct PencilArgs {
    float frac;          // kick in units of dt (0.5 + 0.5 for a full step)
    float scale;         // 1/cells times the output scale
    int has_m;
    float2 m[4];         // pulse matrix, row-major
};

// The four-step z transform of a tile of PEN adjacent pencils (nz = 16 G; PEN * G threads), in three
// stages separated by barriers of the tile's threads. buf holds PEN x NZ float4 (swizzled rows of 16).
//   inv1:  thread (p, j) = (t % PEN, t / PEN) holds z = j + G m, m < 16: inverse 16-point DFT over
//          m -> k1, twiddle W^{-j k1}, to buf
//   mid:   thread (q, p2) = (t % G, t / G) gathers k1 = q + G r (r < 16 / G) for all j: inverse G-point
//          DFT over j -> k2 (k = k1 + 16 k2), kinetic phase (and pulse), forward G-point DFT, twiddle;
//          mid_store writes it back after the caller's barrier
//   fwd3:  thread (p, j) gathers its k1 < 16 and finishes with the forward 16-point DFT over k1 -> m
// The buffer is a float4 pointer or an accessor (a functor mapping the buffer index to a float4 slot, e.g.
// into a tile of a state held in shared memory).
__device__ __forceinline__ float4 &zat(float4 *b, int i) { return b[i]; }
template <class F>
__device__ __forceinline__ float4 &zat(const F &f, int i) { return f(i); }

template <int NZ, int PEN>
struct ZTile {
    static constexpr int R = 16, G = NZ / 16;
    static_assert(NZ % 16 == 0 && G <= 16, "nz = 16 G with G <= 16");

    __device__ static __forceinline__ int bix(int p, int jj, int k1) { return (p * G + jj) * R + (k1 ^ (p & 7)); }

    template <class Buf>
    __device__ static __forceinline__ void inv1(float4 (&x)[R], Buf buf, const float2 *tw, int p, int j)
    {
        dft<R, true>(x);                                            // over m -> k1 (inverse)
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) {
            const float2 w = tw[j * k1];
            x[k1] = fftreg::cmulw(x[k1], make_float2(w.x, -w.y));   // W^{-j k1}
        }
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) zat(buf, bix(p, j, k1)) = x[k1];
    }

    // pxy: the pencil's (kx, ky) factor times the scale; kzp: the kz factors
    template <class Buf>
    __device__ static __forceinline__ void mid(float4 (&y)[R], Buf buf, const float2 *tw, const float2 *kzp,
                                               float2 pxy, const PencilArgs &pa, int q, int p2)
    {
#pragma unroll
        for (int r = 0; r < R / G; ++r)
#pragma unroll
            for (int jj = 0; jj < G; ++jj) y[r * G + jj] = zat(buf, bix(p2, jj, q + G * r));
#pragma unroll
        for (int r = 0; r < R / G; ++r) dft<G, true>(y + r * G);   // over j -> k2: k = k1 + 16 k2

        // the two unit-modulus factors are applied to the data one after the other: their product, the same
        // every step for a mode, would round the same way every step and drift the norm of the most
        // populated modes coherently
#pragma unroll
        for (int r = 0; r < R / G; ++r)
#pragma unroll
            for (int k2 = 0; k2 < G; ++k2) {
                const int k = q + G * r + R * k2;
                float4 v = fftreg::cmulw(fftreg::cmulw(y[r * G + k2], pxy), kzp[k]);
                if (pa.has_m) {
                    const float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
                    const float2 an = fftreg::cmix(pa.m[0], a, pa.m[1], b);
                    const float2 bn = fftreg::cmix(pa.m[2], a, pa.m[3], b);
                    v = make_float4(an.x, an.y, bn.x, bn.y);
                }
                y[r * G + k2] = v;
            }

#pragma unroll
        for (int r = 0; r < R / G; ++r) dft<G, false>(y + r * G); // over k2 -> j (forward)
#pragma unroll
        for (int r = 0; r < R / G; ++r)
#pragma unroll
            for (int jj = 1; jj < G; ++jj) y[r * G + jj] = fftreg::cmulw(y[r * G + jj], tw[(q + G * r) * jj]);
    }

    template <class Buf>
    __device__ static __forceinline__ void mid_store(const float4 (&y)[R], Buf buf, int q, int p2)
    {
#pragma unroll
        for (int r = 0; r < R / G; ++r)
#pragma unroll
            for (int jj = 0; jj < G; ++jj) zat(buf, bix(p2, jj, q + G * r)) = y[r * G + jj];
    }

    template <class Buf>
    __device__ static __forceinline__ void fwd3(float4 (&x)[R], Buf buf, int p, int j)
    {
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) x[k1] = zat(buf, bix(p, j, k1));
        dft<R, false>(x);
    }
};

// shared memory of one pencil body: 16 pencils x NZ float4, then W_NZ^e, the kz phase and the
// per-pencil (kx, ky) phase (float2 each)
template <int NZ>
__host__ __device__ constexpr size_t pencil_smem_bytes() { return sizeof(float4) * 16 * NZ + sizeof(float2) * (2 * NZ + 16); }

// OBS: the pass ends a step (no plane pass follows) and also writes, per z, the
// FP64 sums over the tile's 16 pencils of |a|^2, |b|^2 and conj(a) b of the
// z-transformed boundary state: obs[((traj * tiles + tile) * NZ + z) * 4 + k].
// NZ threads; dyn: pencil_smem_bytes<NZ>() of shared memory.
template <int NZ, bool OBS>
__device__ __forceinline__ void pencil_body(const VBlock &vb, float4 *__restrict__ state, int nx, int lx, int ny,
                                            int cells, int tiles, const GroupParamsF *__restrict__ gp,
                                            const int *__restrict__ tgroup, const float2 *__restrict__ tw_g,
                                            const PencilArgs &pa, double *__restrict__ obs, float inv_out_scale,
                                            const float2 *__restrict__ kin, float4 *dyn)
{
    using Z = ZTile<NZ, 16>;
    constexpr int R = 16, G = NZ / 16;
    (void)gp; (void)tgroup; (void)lx;
    float4 *buf = dyn;                                          // 16 pencils x NZ
    float2 *tw = reinterpret_cast<float2 *>(dyn + 16 * NZ);     // W_NZ^e, e < NZ
    float2 *kzp = tw + NZ;                                      // kz phase
    float2 *kxyp = kzp + NZ;                                    // (kx, ky) phase x scale, per pencil

    const int t = vb.tid;
    const int traj = vb.bid / tiles;
    const int pen0 = (vb.bid - traj * tiles) * 16;
    const int plane = nx * ny;

    // kinetic phase e^{+i k^2/2 dt frac} (wigner_kernel.cu:137-151) as the product of the per-kz and the
    // per-pencil factors, from the class's table for this kick fraction (fp32_kin_tables); kin == NULL
    // means frac == 0, no kick. Thread t fills entry t of the twiddle and kz tables (NZ threads).
    // The table entries go to shared memory by asynchronous copies, so the state loads below issue at once
    // and no register holds a table value in between.
    const float2 *kt = kin ? kin + (size_t)traj * (NZ + plane) : nullptr;
    copy_async8(tw + t, tw_g + t);
    if (kt) {
        copy_async8(kzp + t, kt + t);
        if (t < 16) copy_async8(kxyp + t, kt + NZ + pen0 + t);
    } else {
        kzp[t] = make_float2(1.f, 0.f);
        if (t < 16) kxyp[t] = make_float2(1.f, 0.f);
    }

    const int p = t & 15, j = t >> 4;
    float4 *__restrict__ g = state + (size_t)traj * cells + pen0 + p;
    float4 x[R];
#pragma unroll
    for (int m = 0; m < R; ++m) x[m] = g[(size_t)(j + G * m) * plane];
    copy_async_wait();
    if (t < 16) kxyp[t] = make_float2(pa.scale * kxyp[t].x, pa.scale * kxyp[t].y);
    vb.sync();                                                  // tables ready
    Z::inv1(x, buf, tw, p, j);
    vb.sync();

    const int q = t % G, p2 = t / G;
    float4 y[R];
    Z::mid(y, buf, tw, kzp, kxyp[p2], pa, q, p2);
    vb.sync();                                                  // stage-2 reads done
    Z::mid_store(y, buf, q, p2);
    vb.sync();

    Z::fwd3(x, buf, p, j);
    if constexpr (OBS) {
        // the output is out_scale * FFT_z(boundary state); undo the scale for the moments
        vb.sync();                                              // stage-3 reads of buf done
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const float4 v = x[m];
            const float ax = v.x * inv_out_scale, ay = v.y * inv_out_scale;
            const float bx = v.z * inv_out_scale, by = v.w * inv_out_scale;
            const int z = j + G * m;
            buf[p * NZ + (z ^ (p & 7))] = make_float4(ax * ax + ay * ay, bx * bx + by * by, ax * bx + ay * by,
                                                      ax * by - ay * bx);
        }
        vb.sync();
        const int tile = vb.bid - traj * tiles;
        for (int z = t; z < NZ; z += NZ) {
            KSum s0, s1, s2, s3;
#pragma unroll
            for (int q2 = 0; q2 < 16; ++q2) {
                const float4 u = buf[q2 * NZ + (z ^ (q2 & 7))];
                s0.add(u.x); s1.add(u.y); s2.add(u.z); s3.add(u.w);
            }
            double *o = obs + (((size_t)traj * tiles + tile) * NZ + z) * 4;
            o[0] = s0.value(); o[1] = s1.value(); o[2] = s2.value(); o[3] = s3.value();
        }
    }
#pragma unroll
    for (int m = 0; m < R; ++m) g[(size_t)(j + G * m) * plane] = x[m];
}

} // namespace stepk
