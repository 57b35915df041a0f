// gs_passes.cu -- batched FP32 imaginary-time ground states.
//
// calculateSteadyState (programs/bec_wigner_3d.cuda/wigner.cu:84-175) for many
// ensembles at once: every step is K/2 -> FFT -> N(dt) -> IFFT -> K/2 ->
// renormalise to N (wigner_kernel.cu:128-134, :154-181), regrouped like the
// real-time path into a pencil pass (IFFT_z, kinetic factor, FFT_z) and a plane
// pass (FFT_xy, nonlinear factor, IFFT_xy) over single-component float2 states
// in the same stored representation (k-space along x and y, x-space along z).
//
// The norm after the second half-kick is measured in k-space by Parseval
// (N' = cells dV sum |psi_k|^2), accumulated per trajectory in FP64, and the
// factor sqrt(N / N') is applied by the next plane pass before the nonlinear
// step (scaling commutes with the linear kick and transforms). Norm buffers
// alternate between steps: the pencil pass of step n adds into buffer n % 2,
// the plane pass of step n + 1 reads it and clears the other one.
#include "engine.h"
#include "fft_reg.cuh"

namespace {

using fftreg::dft;

struct GsArgs {
    float frac1, frac2;       // kick fractions of dt_steady before / after the measurement
    float scale;              // 1/cells (makes the inverse z transform the normalised k-space state)
    float out_scale;          // nx*ny when the pass ends a step, else 1
    int measure;              // 1: accumulate sum |psi_k|^2 (and the kinetic sum) per trajectory
};


// ---------------------------------------------------------------- pencil pass
// nz = 256: bounded to 3 CTAs (24 warps) per SM, 80 registers with a 60-byte spill; measured 4 % faster
// over a batched ground-state loop than 2 CTAs at 99 registers
template <int NZ>
__global__ void __launch_bounds__(NZ, (NZ == 256 ? 3 : 1)) k_gs_pencil(float2 *__restrict__ state, int nx, int lx, int ny, int cells,
                                                  int tiles, const GroupParamsF *__restrict__ gp,
                                                  const GsParamsF *__restrict__ gs, const int *__restrict__ tgroup,
                                                  const float2 *__restrict__ tw_g, GsArgs a,
                                                  double *__restrict__ norm, double *__restrict__ ekin,
                                                  const int *__restrict__ active)
{
    constexpr int R = 16, G = NZ / 16;
    extern __shared__ float2 dyn2[];
    float2 *buf = dyn2;                          // 16 pencils x NZ
    float2 *tw = buf + 16 * NZ;                  // W_NZ^e
    float *kz2 = reinterpret_cast<float *>(tw + NZ);   // kz^2/2 per kz
    float *kxy2 = kz2 + NZ;                      // (kx^2 + ky^2)/2 per pencil
    float *ez1 = kxy2 + 16, *ez2 = ez1 + NZ;     // exp(-dt frac1,2 kz^2/2) per kz
    float *exy1 = ez2 + NZ, *exy2 = exy1 + 16;   // exp(-dt frac1,2 (kx^2 + ky^2)/2) x scale, out_scale
    __shared__ double red[2][NZ / 32];

    const int t = threadIdx.x;
    const int lt = blockIdx.x / tiles;                   // position in the launch's trajectory list
    const int traj = active ? active[lt] : lt;
    const int pen0 = (blockIdx.x - lt * tiles) * 16;
    const int gi = tgroup[traj];
    const GroupParamsF P = gp[gi];
    const float dts = gs[gi].dt_steady;
    const int plane = nx * ny;

    for (int i = t; i < NZ; i += blockDim.x) {
        tw[i] = tw_g[i];
        const float kz = getk<float>(i, P.dkz, NZ);
        kz2[i] = 0.5f * kz * kz;
        ez1[i] = expf(-dts * a.frac1 * kz2[i]);
        ez2[i] = expf(-dts * a.frac2 * kz2[i]);
    }
    if (t < 16) {
        const int pen = pen0 + t;
        const int x = pen & (nx - 1), y = pen >> lx;
        const float kx = getk<float>(x, P.dkx, nx);
        const float ky = (ny > 1) ? getk<float>(y, P.dky, ny) : 0.0f;
        kxy2[t] = 0.5f * (kx * kx + ky * ky);
        exy1[t] = expf(-dts * a.frac1 * kxy2[t]) * a.scale;
        exy2[t] = expf(-dts * a.frac2 * kxy2[t]) * a.out_scale;
    }

    const int p = t & 15, j = t >> 4;
    float2 *__restrict__ g = state + (size_t)traj * cells + pen0 + p;
    float2 x[R];
#pragma unroll
    for (int m = 0; m < R; ++m) x[m] = g[(size_t)(j + G * m) * plane];
    __syncthreads();
    dft<R, true, false>(x);
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
        const float2 w = tw[j * k1];
        x[k1] = fftreg::cmulw(x[k1], make_float2(w.x, -w.y));
    }
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[(p * G + j) * R + (k1 ^ (p & 15))] = x[k1];
    __syncthreads();

    const int q = t % G, p2 = t / G;
    float2 y[R];
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int jj = 0; jj < G; ++jj) y[r * G + jj] = buf[(p2 * G + jj) * R + ((q + G * r) ^ (p2 & 15))];
#pragma unroll
    for (int r = 0; r < R / G; ++r) dft<G, true, false>(y + r * G);

    // propagateKSpaceImaginaryTime (wigner_kernel.cu:128-134): exp(-dt_steady frac k^2/2), real, as the
    // product of its (kx, ky) and kz factors
    double n_acc = 0.0, e_acc = 0.0;
    const float kxy = kxy2[p2], fxy1 = exy1[p2], fxy2 = exy2[p2];
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int k2 = 0; k2 < G; ++k2) {
            const int k = q + G * r + R * k2;
            const float k2h = kxy + kz2[k];
            float2 v = y[r * G + k2];
            const float e1 = fxy1 * ez1[k];
            v = make_float2(v.x * e1, v.y * e1);
            if (a.measure) {
                const double nk = (double)v.x * v.x + (double)v.y * v.y;
                n_acc += nk;
                e_acc += nk * k2h;
            }
            const float e2 = fxy2 * ez2[k];
            y[r * G + k2] = make_float2(v.x * e2, v.y * e2);
        }
    if (a.measure) {
        for (int off = 16; off > 0; off >>= 1) {
            n_acc += __shfl_down_sync(0xffffffffu, n_acc, off);
            e_acc += __shfl_down_sync(0xffffffffu, e_acc, off);
        }
        if ((t & 31) == 0) { red[0][t >> 5] = n_acc; red[1][t >> 5] = e_acc; }
    }

#pragma unroll
    for (int r = 0; r < R / G; ++r) dft<G, false, false>(y + r * G);
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int jj = 1; jj < G; ++jj) y[r * G + jj] = fftreg::cmulw(y[r * G + jj], tw[(q + G * r) * jj]);
    __syncthreads();
    if (a.measure && t == 0) {
        double sn = 0.0, se = 0.0;
        for (int w = 0; w < NZ / 32; ++w) { sn += red[0][w]; se += red[1][w]; }
        atomicAdd(norm + traj, sn);
        if (ekin) atomicAdd(ekin + traj, se);
    }
#pragma unroll
    for (int r = 0; r < R / G; ++r)
#pragma unroll
        for (int jj = 0; jj < G; ++jj) buf[(p2 * G + jj) * R + ((q + G * r) ^ (p2 & 15))] = y[r * G + jj];
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) x[k1] = buf[(p * G + j) * R + (k1 ^ (p & 15))];
    dft<R, false, false>(x);
#pragma unroll
    for (int m = 0; m < R; ++m) g[(size_t)(j + G * m) * plane] = x[m];
}

// ---------------------------------------------------------------- plane passes
// MODE 0: step (FFT_xy -> renormalise -> nonlinear -> IFFT_xy)
// MODE 1: prep (x-space natural in -> IFFT_xy)
// MODE 2: measure / output (FFT_xy, renormalise, write x-space rows to out, x-space sums)
template <int N, int MODE>
__global__ void __launch_bounds__(128, 4) k_gs_plane(float2 *__restrict__ state, int nz, int cells,
                                                  const GroupParamsF *__restrict__ gp,
                                                  const GsParamsF *__restrict__ gs, const int *__restrict__ tgroup,
                                                  const double *__restrict__ norm_in, double *__restrict__ norm_clear,
                                                  float2 *__restrict__ out, double *__restrict__ xsums, float in_scale,
                                                  const int *__restrict__ active)
{
    constexpr int W = 32 / N;
    constexpr int PLANE = N * N;
    constexpr int SW = N >= 16 ? 15 : 7;
    extern __shared__ float2 tile2[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wp = lane / N, c = lane % N;
    const int plane_id = (blockIdx.x * 4 + warp) * W + wp;
    const int lt = plane_id / nz, z = plane_id - lt * nz;
    const int traj = active ? active[lt] : lt;
    float2 *__restrict__ g = state + (size_t)traj * cells + (size_t)z * PLANE;
    float2 *s = tile2 + (warp * W + wp) * PLANE;
    const int gi = tgroup[traj];
    const GroupParamsF P = gp[gi];
    const GsParamsF Q = gs[gi];

    float scale = in_scale;
    if (norm_in) scale *= sqrtf((float)(Q.N / (norm_in[traj] * Q.parseval)));
    if (norm_clear && z == 0 && c == 0) norm_clear[traj] = 0.0;

    float2 v[N];
#pragma unroll
    for (int y = 0; y < N; ++y) v[y] = (MODE == 1) ? g[c * N + y] : g[y * N + c];   // prep starts from rows
    const int p_begin = (MODE == 1) ? 2 : 0;
    const int p_end = (MODE == 2) ? 2 : 4;
#pragma unroll 1
    for (int pass = p_begin; pass < p_end; ++pass) {
        if (pass >= 2) dft<N, true, false>(v);
        else dft<N, false, false>(v);
        if (pass == 0) {
#pragma unroll
            for (int y = 0; y < N; ++y) s[y * N + (c ^ (y & SW))] = v[y];
            __syncwarp();
#pragma unroll
            for (int x = 0; x < N; ++x) v[x] = s[c * N + (x ^ (c & SW))];
        } else if (pass == 1 && MODE == 0) {
            // propagateXSpaceOneComponent (wigner_kernel.cu:154-181) on the renormalised row
#pragma unroll
            for (int x = 0; x < N; ++x) s[c * N + (x ^ (c & SW))] = v[x];
            // coordinates and potential with the fused multiply-adds written out; four cells per iteration, their
            // exponentials independent (one midpoint iteration, every workload here, runs without its loop)
            const float Y = fmaf(P.dy, (float)c, -P.ymax);
            const float Z = fmaf(P.dz, (float)z, -P.zmax);
            const float base = fmaf(Y, Y, (Z * Z) * P.inv_lambda2);
            const float hdt = 0.5f * Q.dt_steady;
#pragma unroll 1
            for (int x = 0; x < N; x += 4) {
                float2 o[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float X = fmaf(P.dx, (float)(x + k), -P.xmax);
                    const float V = 0.5f * fmaf(X, X, base);
                    const float2 w = s[c * N + ((x + k) ^ (c & SW))];
                    const float2 a0 = make_float2(w.x * scale, w.y * scale);
                    float2 xa = a0;
                    float da = 0.0f;
                    if (P.itmax == 1) {
                        da = expf(hdt * fmaf(-P.g11, fmaf(a0.x, a0.x, a0.y * a0.y), -V));
                        xa = make_float2(a0.x * da, a0.y * da);
                    } else {
                        for (int it = 0; it < P.itmax; ++it) {
                            da = expf(hdt * fmaf(-P.g11, fmaf(xa.x, xa.x, xa.y * xa.y), -V));
                            xa = make_float2(a0.x * da, a0.y * da);
                        }
                    }
                    o[k] = make_float2(xa.x * da, xa.y * da);
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) s[c * N + ((x + k) ^ (c & SW))] = o[k];
            }
#pragma unroll
            for (int x = 0; x < N; ++x) v[x] = s[c * N + (x ^ (c & SW))];
        } else if (pass == 2) {
#pragma unroll
            for (int x = 0; x < N; ++x) s[c * N + (x ^ (c & SW))] = v[x];
            __syncwarp();
#pragma unroll
            for (int y = 0; y < N; ++y) v[y] = s[y * N + (c ^ (y & SW))];
        }
    }
    if (MODE == 2) {
        // lane c holds row y = c of the x-space state
        const float Y = -P.ymax + P.dy * (float)c;
        const float Z = -P.zmax + P.dz * (float)z;
        const float base = Y * Y + Z * Z * P.inv_lambda2;
        // sums: n V, n^2, n and |u - previous output|^2 (the state's change since the last output)
        double sv = 0.0, s2 = 0.0, s1 = 0.0, sd = 0.0;
        float2 *o = out + (size_t)traj * cells + (size_t)z * PLANE + c * N;
#pragma unroll
        for (int x = 0; x < N; ++x) {
            const float2 u = make_float2(v[x].x * scale, v[x].y * scale);
            const float2 w = o[x];
            o[x] = u;
            const float X = -P.xmax + P.dx * (float)x;
            const double n = (double)u.x * u.x + (double)u.y * u.y;
            const float ex = u.x - w.x, ey = u.y - w.y;
            sv += n * (double)(0.5f * (X * X + base));
            s2 += n * n;
            s1 += n;
            sd += (double)(ex * ex + ey * ey);
        }
        if (xsums) {
            for (int off = N / 2; off > 0; off >>= 1) {
                sv += __shfl_down_sync(0xffffffffu, sv, off, N);
                s2 += __shfl_down_sync(0xffffffffu, s2, off, N);
                s1 += __shfl_down_sync(0xffffffffu, s1, off, N);
                sd += __shfl_down_sync(0xffffffffu, sd, off, N);
            }
            if (c == 0) {
                atomicAdd(xsums + 4 * traj + 0, sv);
                atomicAdd(xsums + 4 * traj + 1, s2);
                atomicAdd(xsums + 4 * traj + 2, s1);
                atomicAdd(xsums + 4 * traj + 3, sd);
            }
        }
    } else {
#pragma unroll
        for (int y = 0; y < N; ++y) g[y * N + c] = v[y];
    }
}

// x-space Thomas-Fermi start (fillWithTFGroundState, wigner_kernel.cu:116-125) or a copy of a warm start
__global__ void k_gs_init(float2 *state, int nx, int lx, int ny, int ly, int cells, int n_traj,
                          const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup, const float2 *warm)
{
    const size_t n = (size_t)cells * n_traj;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(idx / cells), i = (int)(idx - (size_t)t * cells);
        if (warm) { state[idx] = warm[idx]; continue; }
        const int gi = tgroup[t];
        const GroupParamsF P = gp[gi];
        const int x = i & (nx - 1), y = (i >> lx) & (ny - 1), z = i >> (lx + ly);
        const float X = -P.xmax + P.dx * (float)x;
        const float Y = (ny > 1) ? -P.ymax + P.dy * (float)y : 0.0f;
        const float Z = -P.zmax + P.dz * (float)z;
        const float e = gs[gi].mu - 0.5f * (X * X + Y * Y + Z * Z * P.inv_lambda2);
        state[idx] = make_float2(e > 0.0f ? sqrtf(e / P.g11) : 0.0f, 0.0f);
    }
}

template <int N, int MODE>
void launch_gs_plane(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs,
                     const int *tgroup, const double *norm_in, double *norm_clear, float2 *out, double *xsums,
                     float in_scale, const int *active, cudaStream_t s)
{
    constexpr int W = 32 / N;
    const size_t smem = sizeof(float2) * 4 * W * N * N;
    ensure_smem_limit((const void *)k_gs_plane<N, MODE>, (int)smem);
    k_gs_plane<N, MODE><<<c.n_traj * c.nz / (4 * W), 128, smem, s>>>(state, c.nz, c.cells, gp, gs, tgroup, norm_in,
                                                                      norm_clear, out, xsums, in_scale, active);
    g_launches++;
}

template <int NZ>
void launch_gs_pencil(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs,
                      const int *tgroup, const float2 *tw, const GsArgs &a, double *norm, double *ekin,
                      const int *active, cudaStream_t s)
{
    const int tiles = c.nx * c.ny / 16;
    const size_t smem = sizeof(float2) * (16 * NZ + NZ) + sizeof(float) * (3 * NZ + 3 * 16);
    ensure_smem_limit((const void *)k_gs_pencil<NZ>, (int)smem);
    k_gs_pencil<NZ><<<c.n_traj * tiles, NZ, smem, s>>>(state, c.nx, c.lx, c.ny, c.cells, tiles, gp, gs, tgroup, tw,
                                                       a, norm, ekin, active);
    g_launches++;
}

template <int MODE>
void dispatch_plane(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
                    const double *norm_in, double *norm_clear, float2 *out, double *xsums, float in_scale,
                    const int *active, cudaStream_t s)
{
    switch (c.nx) {
    case 8: launch_gs_plane<8, MODE>(state, c, gp, gs, tgroup, norm_in, norm_clear, out, xsums, in_scale, active, s); break;
    case 16: launch_gs_plane<16, MODE>(state, c, gp, gs, tgroup, norm_in, norm_clear, out, xsums, in_scale, active, s); break;
    case 32: launch_gs_plane<32, MODE>(state, c, gp, gs, tgroup, norm_in, norm_clear, out, xsums, in_scale, active, s); break;
    default: break;
    }
}

} // namespace

namespace {
__global__ void k_to_double(const float2 *in, double2 *out, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_double2(in[i].x, in[i].y);
}
} // namespace

void gs_to_double(const float2 *in, double2 *out, size_t n, cudaStream_t s)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    k_to_double<<<blocks, 256, 0, s>>>(in, out, n);
    g_launches++;
}

bool gs_batched_supported(const ClassGeom &c)
{
    return fp32_fast_plane_supported(c) && fp32_fast_pencil_supported(c);
}

void gs_init(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
             const float2 *warm, cudaStream_t s)
{
    size_t n = (size_t)c.cells * c.n_traj;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_gs_init<<<blocks, 256, 0, s>>>(state, c.nx, c.lx, c.ny, c.ly, c.cells, c.n_traj, gp, gs, tgroup, warm);
    g_launches++;
}

void gs_prep(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
             cudaStream_t s)
{
    dispatch_plane<1>(state, c, gp, gs, tgroup, nullptr, nullptr, nullptr, nullptr, 1.0f, nullptr, s);
}

void gs_plane_step(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
                   const double *norm_in, double *norm_clear, cudaStream_t s, const int *active)
{
    dispatch_plane<0>(state, c, gp, gs, tgroup, norm_in, norm_clear, nullptr, nullptr, 1.0f, active, s);
}

void gs_output(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
               const double *norm_in, float2 *out, double *xsums, float in_scale, cudaStream_t s, const int *active)
{
    dispatch_plane<2>(state, c, gp, gs, tgroup, norm_in, nullptr, out, xsums, in_scale, active, s);
}

void gs_pencil(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
               const float2 *tw_full, float frac1, float frac2, float scale, float out_scale, double *norm,
               double *ekin, cudaStream_t s, const int *active)
{
    GsArgs a{frac1, frac2, scale, out_scale, norm ? 1 : 0};
    switch (c.nz) {
    case 64: launch_gs_pencil<64>(state, c, gp, gs, tgroup, tw_full, a, norm, ekin, active, s); break;
    case 128: launch_gs_pencil<128>(state, c, gp, gs, tgroup, tw_full, a, norm, ekin, active, s); break;
    case 256: launch_gs_pencil<256>(state, c, gp, gs, tgroup, tw_full, a, norm, ekin, active, s); break;
    default: break;
    }
}
