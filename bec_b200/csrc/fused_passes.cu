// fused_passes.cu -- register-resident plane and pencil passes of the FP32 path.
//
// Same two-pass regrouping of the reference's split step as batched_fp32.cu
// (propagate, programs/bec_wigner_3d.cuda/wigner.cu:178-199) and the same
// stored representation, but every line of the 3D transform lives in one
// thread's registers and shared memory is used only to transpose:
//
// plane pass (square planes N x N, N = 8, 16, 32): one warp per 32/N planes.
//   lane c loads column c of its plane straight from HBM (each load instruction
//   of the warp reads consecutive 16-byte cells), transforms it along y, writes
//   it to an XOR-swizzled shared tile, reads back row c, transforms along x,
//   applies the nonlinear / loss / loss-noise step to its N cells, and returns
//   the same way. Both components of a cell are one float4.
//
// pencil pass (nz = 64, 128, 256 = 16 G): one CTA per 16 adjacent pencils of a
//   trajectory, 16 G threads. A four-step decomposition nz = 16 x G: each
//   thread holds 16 elements (z = j + G m) and does a 16-point DFT, twiddles,
//   and after one shared-memory transpose a G-point DFT across j; the kinetic
//   phase e^{i k^2/2 dt} (wigner_kernel.cu:137-151) is applied in full k-space
//   as the product of a per-pencil (kx, ky) factor and a per-kz factor; the
//   forward transform retraces the same steps.
//
// Shared tiles are swizzled on the 16-byte unit index (col ^ (row & 7)) so
// that both the row-wise and the column-wise access of a quarter warp touch
// eight different bank groups.
#include "engine.h"
#include "fft_reg.cuh"
#include "physics.cuh"
#include "split32.cuh"

namespace {

using fftreg::dft;

// ---------------------------------------------------------------- plane pass
template <int N>
__global__ void __launch_bounds__(128, 4) k_plane(float4 *__restrict__ state, int nz, int cells,
                                               const GroupParamsF *__restrict__ gp, const int *__restrict__ tgroup,
                                               const int *__restrict__ tlocal, const uint32_t *__restrict__ stepp)
{
    constexpr int W = 32 / N;          // planes per warp
    const uint32_t step = *stepp;      // Philox step index (device scalar, see fp32_put_step)
    constexpr int PLANE = N * N;
    extern __shared__ float4 tile[];   // 4 warps x W planes x PLANE
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wp = lane / N, c = lane % N;
    const int plane_id = (blockIdx.x * 4 + warp) * W + wp;
    const int traj = plane_id / nz, z = plane_id - traj * nz;
    float4 *__restrict__ g = state + (size_t)traj * cells + (size_t)z * PLANE;
    float4 *s = tile + (warp * W + wp) * PLANE;

    const GroupParamsF P = gp[tgroup[traj]];

    float4 v[N];
#pragma unroll
    for (int y = 0; y < N; ++y) v[y] = g[y * N + c];

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
            const float Y = -P.ymax + P.dy * (float)c;
            const float Z = -P.zmax + P.dz * (float)z;
            const float base = Y * Y + Z * Z * P.inv_lambda2;
            const uint32_t tl = (uint32_t)tlocal[traj];
            const CellConsts K = cell_consts(P);
            const uint32_t cell0 = (uint32_t)(z * PLANE + c * N);
            // cells in pairs: the two Philox draws interleave (loss_noise_cell2)
#pragma unroll 1
            for (int x = 0; x < N; x += 2) {
                const float X0 = -P.xmax + P.dx * (float)x, X1 = -P.xmax + P.dx * (float)(x + 1);
                float4 *s0 = s + c * N + (x ^ (c & 7)), *s1 = s + c * N + ((x + 1) ^ (c & 7));
                const float4 v0 = *s0, v1 = *s1;
                float4 o0 = nonlinear_cell(v0, 0.5f * (X0 * X0 + base), K);
                float4 o1 = nonlinear_cell(v1, 0.5f * (X1 * X1 + base), K);
                if (P.noise)
                    loss_noise_cell2(o0, v0, o1, v1, K, P.seed_lo, P.seed_hi, tl, step, cell0 + x, cell0 + x + 1);
                *s0 = o0;
                *s1 = o1;
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
#pragma unroll
    for (int y = 0; y < N; ++y) g[y * N + c] = v[y];
}

// ---------------------------------------------------------------- plane pass, 32 x 32, two warps a plane
// k_plane's step for N = 32 with the line transforms of split32.cuh: every 32-point line is shared by
// lane L of warp 0 and lane L of warp 1 of the plane's CTA, 16 elements each, half the registers of a
// one-lane line, so more warps fit on an SM. The 32 x 32 float4 tile is swizzled like k_plane's.

template <int MINB>
__global__ void __launch_bounds__(64, MINB) k_plane32s(float4 *__restrict__ state, int nz, int cells,
                                                      const GroupParamsF *__restrict__ gp,
                                                      const int *__restrict__ tgroup, const int *__restrict__ tlocal,
                                                      const uint32_t *__restrict__ stepp)
{
    using namespace split32;
    const uint32_t step = *stepp;
    __shared__ float4 tile[1024];
    __shared__ float4 xb[512];
    const int h = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int plane_id = blockIdx.x;
    const int traj = plane_id / nz, z = plane_id - traj * nz;
    float4 *__restrict__ g = state + (size_t)traj * cells + (size_t)z * 1024;
    const GroupParamsF P = gp[tgroup[traj]];

    float4 v[16];
    // forward along y (lane = column), then along x (lane = row); shared code body
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = g[(2 * j + h) * 32 + lane];
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = tile[tix(lane, 2 * j + h)];
        }
        fwd_line(v, xb, h, lane);
        if (pass == 0) {
#pragma unroll
            for (int s = 0; s < 16; ++s) tile[tix(kblk(s, h), lane)] = v[s];
            __syncthreads();
        }
    }
    // x-space: lane owns row y = lane, cells x = kblk(s, h); the physics runs as a rolled loop
    // over those cells in the tile
    {
        const int r = lane;
#pragma unroll
        for (int s = 0; s < 16; ++s) tile[tix(r, kblk(s, h))] = v[s];
        const float Y = -P.ymax + P.dy * (float)r;
        const float Z = -P.zmax + P.dz * (float)z;
        const float base = Y * Y + Z * Z * P.inv_lambda2;
        const uint32_t tl = (uint32_t)tlocal[traj];
        const CellConsts K = cell_consts(P);
        const uint32_t cell0 = (uint32_t)(z * 1024 + r * 32);
        // cells in pairs (x, x + 1; kblk keeps pairs of even s adjacent): the two Philox draws interleave
#pragma unroll 1
        for (int s = 0; s < 16; s += 2) {
            const int x = kblk(s, h);
            const float X0 = -P.xmax + P.dx * (float)x, X1 = -P.xmax + P.dx * (float)(x + 1);
            float4 *s0 = tile + tix(r, x), *s1 = tile + tix(r, x + 1);
            const float4 v0 = *s0, v1 = *s1;
            float4 o0 = nonlinear_cell(v0, 0.5f * (X0 * X0 + base), K);
            float4 o1 = nonlinear_cell(v1, 0.5f * (X1 * X1 + base), K);
            if (P.noise)
                loss_noise_cell2(o0, v0, o1, v1, K, P.seed_lo, P.seed_hi, tl, step, cell0 + x, cell0 + x + 1);
            *s0 = o0;
            *s1 = o1;
        }
#pragma unroll
        for (int s = 0; s < 16; ++s) v[s] = tile[tix(r, kblk(s, h))];
    }
    __syncthreads();    // the partner's physics is done with the row, and its last exchange reads too
    // inverse along x (lane = row), then along y (lane = column); shared code body
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
#pragma unroll
            for (int s = 0; s < 16; ++s) v[s] = tile[tix(kblk(s, h), lane)];
        }
        inv_line(v, xb, h, lane);
        if (pass == 0) {
#pragma unroll
            for (int m = 0; m < 16; ++m) tile[tix(lane, 2 * m + h)] = v[m];
            __syncthreads();
        }
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) g[(2 * m + h) * 32 + lane] = v[m];
}

// ---------------------------------------------------------------- pencil pass
struct PencilArgs {
    float frac;          // kick in units of dt (0.5 + 0.5 for a full step)
    float scale;         // 1/cells times the output scale
    int has_m;
    float2 m[4];         // pulse matrix, row-major
};

// OBS: the pass ends a step (no plane pass follows) and also writes, per z, the
// FP64 sums over the tile's 16 pencils of |a|^2, |b|^2 and conj(a) b of the
// z-transformed boundary state: obs[((traj * tiles + tile) * NZ + z) * 4 + k].
template <int NZ, bool OBS>
__global__ void __launch_bounds__(NZ) k_pencil(float4 *__restrict__ state, int nx, int lx, int ny, int cells,
                                               int tiles, const GroupParamsF *__restrict__ gp,
                                               const int *__restrict__ tgroup, const float2 *__restrict__ tw_g,
                                               PencilArgs pa, double *__restrict__ obs, float inv_out_scale)
{
    constexpr int R = 16, G = NZ / 16;
    extern __shared__ float4 dyn[];
    float4 *buf = dyn;                                          // 16 pencils x NZ
    float2 *tw = reinterpret_cast<float2 *>(dyn + 16 * NZ);     // W_NZ^e, e < NZ
    float2 *kzp = tw + NZ;                                      // kz phase
    float2 *kxyp = kzp + NZ;                                    // (kx, ky) phase x scale, per pencil

    const int t = threadIdx.x;
    const int traj = blockIdx.x / tiles;
    const int pen0 = (blockIdx.x - traj * tiles) * 16;
    const GroupParamsF P = gp[tgroup[traj]];
    const int plane = nx * ny;

    for (int i = t; i < NZ; i += blockDim.x) {
        tw[i] = tw_g[i];
        const float kz = getk<float>(i, P.dkz, NZ);
        float s, c;
        sincosf(0.5f * kz * kz * P.dt * pa.frac, &s, &c);      // e^{+i k^2/2 dt frac}
        kzp[i] = make_float2(c, s);
    }
    if (t < 16) {
        const int pen = pen0 + t;
        const int x = pen & (nx - 1), y = pen >> lx;
        const float kx = getk<float>(x, P.dkx, nx);
        const float ky = (ny > 1) ? getk<float>(y, P.dky, ny) : 0.0f;
        float s, c;
        sincosf(0.5f * (kx * kx + ky * ky) * P.dt * pa.frac, &s, &c);
        kxyp[t] = make_float2(pa.scale * c, pa.scale * s);
    }

    // stage 1: thread (p, j) holds z = j + G m, m < 16
    const int p = t & 15, j = t >> 4;
    float4 *__restrict__ g = state + (size_t)traj * cells + pen0 + p;
    float4 x[R];
#pragma unroll
    for (int m = 0; m < R; ++m) x[m] = g[(size_t)(j + G * m) * plane];
    __syncthreads();                                            // tables ready
    dft<R, true>(x);                                            // over m -> k1 (inverse)
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
        const float2 w = tw[j * k1];
        x[k1] = fftreg::cmulw(x[k1], make_float2(w.x, -w.y));   // W^{-j k1}
    }
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[(p * G + j) * R + (k1 ^ (p & 7))] = x[k1];
    __syncthreads();

    // stage 2: thread (q, p2) holds k1 = q + G r (r < 16/G) for all j, then all k2
    const int q = t % G, p2 = t / G;
    float4 y[R];
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int jj = 0; jj < G; ++jj) y[r * G + jj] = buf[(p2 * G + jj) * R + ((q + G * r) ^ (p2 & 7))];
#pragma unroll
    for (int r = 0; r < R / G; ++r) dft<G, true>(y + r * G);   // over j -> k2: k = k1 + 16 k2

    const float2 pxy = kxyp[p2];
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int k2 = 0; k2 < G; ++k2) {
            const int k = q + G * r + R * k2;
            float4 v = fftreg::cmulw(y[r * G + k2], cmul(pxy, kzp[k]));
            if (pa.has_m) {
                const float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
                const float2 an = cadd(cmul(pa.m[0], a), cmul(pa.m[1], b));
                const float2 bn = cadd(cmul(pa.m[2], a), cmul(pa.m[3], b));
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
    __syncthreads();                                            // stage-2 reads done
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int jj = 0; jj < G; ++jj) buf[(p2 * G + jj) * R + ((q + G * r) ^ (p2 & 7))] = y[r * G + jj];
    __syncthreads();

    // stage 3: thread (p, j) gathers k1 < 16 and finishes over k1 -> m
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) x[k1] = buf[(p * G + j) * R + (k1 ^ (p & 7))];
    dft<R, false>(x);
    if constexpr (OBS) {
        // the output is out_scale * FFT_z(boundary state); undo the scale for the moments
        __syncthreads();                                        // stage-3 reads of buf done
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const float4 v = x[m];
            const float ax = v.x * inv_out_scale, ay = v.y * inv_out_scale;
            const float bx = v.z * inv_out_scale, by = v.w * inv_out_scale;
            const int z = j + G * m;
            buf[p * NZ + (z ^ (p & 7))] = make_float4(ax * ax + ay * ay, bx * bx + by * by, ax * bx + ay * by,
                                                      ax * by - ay * bx);
        }
        __syncthreads();
        const int tile = blockIdx.x - traj * tiles;
        for (int z = t; z < NZ; z += blockDim.x) {
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

template <int NZ, bool OBS>
void launch_pencil(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const float2 *tw,
                   const PencilArgs &pa, double *obs, float inv_out_scale, cudaStream_t s)
{
    const int tiles = c.nx * c.ny / 16;
    const size_t smem = sizeof(float4) * 16 * NZ + sizeof(float2) * (2 * NZ + 16);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_pencil<NZ, OBS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_pencil<NZ, OBS><<<c.n_traj * tiles, NZ, smem, s>>>(state, c.nx, c.lx, c.ny, c.cells, tiles, gp, tgroup, tw,
                                                         pa, obs, inv_out_scale);
    g_launches++;
}

template <int N>
void launch_plane(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                  const uint32_t *step, cudaStream_t s)
{
    constexpr int W = 32 / N;
    const int planes = c.n_traj * c.nz;
    const size_t smem = sizeof(float4) * 4 * W * N * N;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_plane<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_plane<N><<<planes / (4 * W), 128, smem, s>>>(state, c.nz, c.cells, gp, tgroup, tlocal, step);
    g_launches++;
}

template <int MINB>
void launch_plane32s(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                     const uint32_t *step, cudaStream_t s)
{
    k_plane32s<MINB><<<c.n_traj * c.nz, 64, 0, s>>>(state, c.nz, c.cells, gp, tgroup, tlocal, step);
    g_launches++;
}

} // namespace

bool fp32_fast_plane_supported(const ClassGeom &c)
{
    if (c.nx != c.ny || (c.nx != 8 && c.nx != 16 && c.nx != 32)) return false;
    const int W = 32 / c.nx;
    return ((long long)c.n_traj * c.nz) % (4 * W) == 0;
}

bool fp32_fast_pencil_supported(const ClassGeom &c)
{
    return (c.nz == 64 || c.nz == 128 || c.nz == 256) && (c.nx * c.ny) % 16 == 0 && c.nx * c.ny >= 16;
}

void fp32_plane_fast(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                     const uint32_t *step, cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    switch (c.nx) {
    case 8: launch_plane<8>(state, c, gp, tgroup, tlocal, step, s); break;
    case 16: launch_plane<16>(state, c, gp, tgroup, tlocal, step, s); break;
    case 32: launch_plane32s<8>(state, c, gp, tgroup, tlocal, step, s); break;
    default: break;
    }
}

void fp32_pencil_fast(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup,
                      const float2 *tw_full, float frac, float scale, const float2 *m, double *obs,
                      float out_scale, cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    PencilArgs pa{};
    pa.frac = frac;
    pa.scale = scale;
    pa.has_m = m ? 1 : 0;
    if (m)
        for (int i = 0; i < 4; ++i) pa.m[i] = m[i];
    const float inv = 1.0f / out_scale;
    switch (c.nz) {
    case 64:
        if (obs) launch_pencil<64, true>(state, c, gp, tgroup, tw_full, pa, obs, inv, s);
        else launch_pencil<64, false>(state, c, gp, tgroup, tw_full, pa, nullptr, inv, s);
        break;
    case 128:
        if (obs) launch_pencil<128, true>(state, c, gp, tgroup, tw_full, pa, obs, inv, s);
        else launch_pencil<128, false>(state, c, gp, tgroup, tw_full, pa, nullptr, inv, s);
        break;
    case 256:
        if (obs) launch_pencil<256, true>(state, c, gp, tgroup, tw_full, pa, obs, inv, s);
        else launch_pencil<256, false>(state, c, gp, tgroup, tw_full, pa, nullptr, inv, s);
        break;
    default: break;
    }
}

int fp32_fast_pencil_tiles(const ClassGeom &c) { return c.nx * c.ny / 16; }
