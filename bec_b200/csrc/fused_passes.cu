// fused_passes.cu -- the register-resident plane and pencil passes of the FP32 path as standalone
// kernels, one launch per pass and grid class; the bodies are in step_bodies.cuh (each kernel gives its
// body the whole CTA). Same two-pass regrouping of the reference's split step as batched_fp32.cu
// (propagate, programs/bec_wigner_3d.cuda/wigner.cu:178-199) and the same stored representation.
// A steady step of the fast classes runs instead as one launch of the fused step kernel
// (step_kernel.cu); these kernels serve the steps that observe, and the launch-per-pass schedule.
#include <algorithm>

#include "engine.h"
#include "step_bodies.cuh"

namespace {

using stepk::PencilArgs;
using stepk::VBlock;

// ---------------------------------------------------------------- plane pass, N = 8, 16
// done != NULL: this launch also advances the Philox step index *stepp once every CTA has finished (every CTA
// read it at its start): the CTA that finishes last (the atomic counter reaches the grid size) resets the counter
// and increments the index, which the next step's kernels read. The one-thread increment launch is then not needed.
__device__ __forceinline__ void advance_step_if_last(uint32_t *stepp, int *done)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(done, 1) == (int)gridDim.x - 1) {
            *done = 0;
            atomicAdd(stepp, 1u);
        }
    }
}

template <int N, int MINB>
__global__ void __launch_bounds__(128, MINB) k_plane(float4 *__restrict__ state, int nz, int cells,
                                               const GroupParamsF *__restrict__ gp, const int *__restrict__ tgroup,
                                               const int *__restrict__ tlocal, uint32_t *stepp, int *done)
{
    extern __shared__ float4 tile[];   // 4 warps x W planes x N^2
    stepk::plane_body<N>(VBlock{(int)threadIdx.x, (int)blockIdx.x, 0, 128}, state, nz, cells, gp, tgroup, tlocal,
                         *stepp, tile);
    if (done) advance_step_if_last(stepp, done);
}

// ---------------------------------------------------------------- plane pass, 32 x 32, two warps a plane
template <int MINB>
__global__ void __launch_bounds__(64, MINB) k_plane32s(float4 *__restrict__ state, int nz, int cells,
                                                      const GroupParamsF *__restrict__ gp,
                                                      const int *__restrict__ tgroup, const int *__restrict__ tlocal,
                                                      uint32_t *stepp, int *done)
{
    __shared__ float4 tile[1024];
    __shared__ float4 xb[512];
    stepk::plane32_body(VBlock{(int)threadIdx.x, (int)blockIdx.x, 0, 64}, state, nz, cells, gp, tgroup, tlocal,
                        *stepp, tile, xb);
    if (done) advance_step_if_last(stepp, done);
}

// ---------------------------------------------------------------- pencil pass
template <int NZ, bool OBS>
__global__ void __launch_bounds__(NZ) k_pencil(float4 *__restrict__ state, int nx, int lx, int ny, int cells,
                                               int tiles, const GroupParamsF *__restrict__ gp,
                                               const int *__restrict__ tgroup, const float2 *__restrict__ tw_g,
                                               PencilArgs pa, double *__restrict__ obs, float inv_out_scale,
                                               const float2 *__restrict__ kin)
{
    extern __shared__ float4 dyn[];
    stepk::pencil_body<NZ, OBS>(VBlock{(int)threadIdx.x, (int)blockIdx.x, 0, NZ}, state, nx, lx, ny, cells, tiles,
                                gp, tgroup, tw_g, pa, obs, inv_out_scale, kin, dyn);
}

__global__ void k_kin_tables(float2 *__restrict__ tab, const GroupParamsF *__restrict__ gp,
                             const int *__restrict__ tgroup, int nx, int ny, int nz, int lx, int n_traj, float frac)
{
    const int per = nz + nx * ny;
    const size_t n = (size_t)n_traj * per;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(idx / per), i = (int)(idx - (size_t)t * per);
        const GroupParamsF &P = gp[tgroup[t]];
        double turns;
        if (i < nz) {
            const int iz = kidx(i, nz);
            turns = P.kin_z * (double)(iz * iz);
        } else {
            const int pen = i - nz;
            const int ix = kidx(pen & (nx - 1), nx), iy = ny > 1 ? kidx(pen >> lx, ny) : 0;
            turns = P.kin_x * (double)(ix * ix) + P.kin_y * (double)(iy * iy);
        }
        tab[idx] = kin_phase(turns * (double)frac);
    }
}

template <int NZ, bool OBS>
void launch_pencil(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const float2 *tw,
                   const PencilArgs &pa, double *obs, float inv_out_scale, const float2 *kin, cudaStream_t s)
{
    const int tiles = c.nx * c.ny / 16;
    const size_t smem = stepk::pencil_smem_bytes<NZ>();
    ensure_smem_limit((const void *)k_pencil<NZ, OBS>, (int)smem);
    k_pencil<NZ, OBS><<<c.n_traj * tiles, NZ, smem, s>>>(state, c.nx, c.lx, c.ny, c.cells, tiles, gp, tgroup, tw,
                                                         pa, obs, inv_out_scale, kin);
    g_launches++;
}

template <int N, int MINB>
void launch_plane(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                  uint32_t *step, int *done, cudaStream_t s)
{
    constexpr int W = 32 / N;
    const int planes = c.n_traj * c.nz;
    const size_t smem = sizeof(float4) * 4 * W * N * N;
    ensure_smem_limit((const void *)k_plane<N, MINB>, (int)smem);
    k_plane<N, MINB><<<planes / (4 * W), 128, smem, s>>>(state, c.nz, c.cells, gp, tgroup, tlocal, step, done);
    g_launches++;
}

template <int MINB>
void launch_plane32s(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                     uint32_t *step, int *done, cudaStream_t s)
{
    k_plane32s<MINB><<<c.n_traj * c.nz, 64, 0, s>>>(state, c.nz, c.cells, gp, tgroup, tlocal, step, done);
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

int fp32_plane_fast_ctas(const ClassGeom &c)
{
    return c.nx == 32 ? c.n_traj * c.nz : c.n_traj * c.nz / (4 * (32 / c.nx));
}

void fp32_plane_fast(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                     uint32_t *step, int occupancy, int *inc_done, cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    // occupancy 0: 16 warps per SM (8x8 / 16x16: 4 CTAs of 128 threads; 32x32: 8 CTAs of 64), no register spill;
    // occupancy 1: 20 warps per SM (5 and 10 CTAs), 96 registers with a small spill
    switch (c.nx) {
    case 8:
        if (occupancy) launch_plane<8, 5>(state, c, gp, tgroup, tlocal, step, inc_done, s);
        else launch_plane<8, 4>(state, c, gp, tgroup, tlocal, step, inc_done, s);
        break;
    case 16:
        if (occupancy) launch_plane<16, 5>(state, c, gp, tgroup, tlocal, step, inc_done, s);
        else launch_plane<16, 4>(state, c, gp, tgroup, tlocal, step, inc_done, s);
        break;
    case 32:
        if (occupancy) launch_plane32s<10>(state, c, gp, tgroup, tlocal, step, inc_done, s);
        else launch_plane32s<8>(state, c, gp, tgroup, tlocal, step, inc_done, s);
        break;
    default: break;
    }
}

void fp32_kin_tables(float2 *tab, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, float frac,
                     cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    const size_t n = (size_t)c.n_traj * (c.nz + c.nx * c.ny);
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_kin_tables<<<blocks, 256, 0, s>>>(tab, gp, tgroup, c.nx, c.ny, c.nz, c.lx, c.n_traj, frac);
    g_launches++;
}

void fp32_pencil_fast(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup,
                      const float2 *tw_full, float frac, float scale, const float2 *m, double *obs,
                      float out_scale, const float2 *kin, cudaStream_t s)
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
        if (obs) launch_pencil<64, true>(state, c, gp, tgroup, tw_full, pa, obs, inv, kin, s);
        else launch_pencil<64, false>(state, c, gp, tgroup, tw_full, pa, nullptr, inv, kin, s);
        break;
    case 128:
        if (obs) launch_pencil<128, true>(state, c, gp, tgroup, tw_full, pa, obs, inv, kin, s);
        else launch_pencil<128, false>(state, c, gp, tgroup, tw_full, pa, nullptr, inv, kin, s);
        break;
    case 256:
        if (obs) launch_pencil<256, true>(state, c, gp, tgroup, tw_full, pa, obs, inv, kin, s);
        else launch_pencil<256, false>(state, c, gp, tgroup, tw_full, pa, nullptr, inv, kin, s);
        break;
    default: break;
    }
}

int fp32_fast_pencil_tiles(const ClassGeom &c) { return c.nx * c.ny / 16; }
