// onchip_step.cu -- a whole split step of an 8x8x64 trajectory with its state held in shared memory: one
// HBM round trip per step (32 B per cell) where the two-pass schedule makes two (64 B).
//
// One CTA of 128 threads per trajectory (64 KiB of state, three CTAs per SM). The step is the two passes of
// the register path (propagate, programs/bec_wigner_3d.cuda/wigner.cu:178-199, regrouped): the pencil pass
// (IFFT_z -> kinetic phase -> FFT_z, ZTile stages, two 64-thread groups of 16 pencils, the tile transposed in
// place in the resident state) and the plane pass (FFT_xy -> nonlinear + losses + loss noise -> IFFT_xy,
// plane_body with its transposes in place), with the same arithmetic, so the step computes the same bits as
// the two launches. Steady steps only (full kick, no pulse, no observation); the others take the two-pass
// route.
#include "engine.h"
#include "step_bodies.cuh"

namespace {

using stepk::PencilArgs;
using stepk::VBlock;
using stepk::ZTile;

constexpr int NZ = 64, PLANE = 64, CELLS = NZ * PLANE, kThreads = 128;
constexpr size_t kSmem = sizeof(float4) * CELLS + sizeof(float2) * (NZ + NZ + PLANE);

// ZTile's buffer over 16 pencils of the resident state: buffer index e -> row z = e / 16, pencil p0 + e % 16
struct PencilRegion {
    float4 *st;
    int p0;
    __device__ __forceinline__ float4 &operator()(int e) const { return st[(e >> 4) * PLANE + p0 + (e & 15)]; }
};

__device__ __forceinline__ void group_sync(int grp)
{
    asm volatile("bar.sync %0, 64;" ::"r"(1 + grp) : "memory");
}

__device__ __forceinline__ void copy_async16(void *dst_smem, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// done != NULL: the last CTA also advances the Philox step index (every CTA read it at its start)
__global__ void __launch_bounds__(kThreads, 3) k_onchip_8x8x64(float4 *__restrict__ state,
                                                             const GroupParamsF *__restrict__ gp,
                                                             const int *__restrict__ tgroup,
                                                             const int *__restrict__ tlocal,
                                                             const float2 *__restrict__ tw_g,
                                                             const float2 *__restrict__ kin, float scale,
                                                             uint32_t *stepp, int *done)
{
    extern __shared__ float4 st[];
    float2 *tw = reinterpret_cast<float2 *>(st + CELLS);
    float2 *kzp = tw + NZ;
    float2 *kxyp = kzp + NZ;
    const int t = threadIdx.x, traj = blockIdx.x;
    float4 *__restrict__ g = state + (size_t)traj * CELLS;
    const uint32_t step = *stepp;

    // W_64^e, this trajectory's kz and (kx, ky) kinetic factors (full kick), and the state, by asynchronous copies
    const float2 *kt = kin + (size_t)traj * (NZ + PLANE);
    if (t < NZ) {
        stepk::copy_async8(tw + t, tw_g + t);
        stepk::copy_async8(kzp + t, kt + t);
    } else {
        stepk::copy_async8(kxyp + (t - NZ), kt + NZ + (t - NZ));
    }
    for (int i = t; i < CELLS; i += kThreads) copy_async16(st + i, g + i);
    stepk::copy_async_wait();
    __syncthreads();

    // pencil pass: 4 tiles of 16 pencils, two 64-thread groups, two rounds
    using Z = ZTile<NZ, 16>;
    const int grp = t >> 6, u = t & 63;
    const int p = u & 15, j = u >> 4;            // stages 1 and 3 (G = 4)
    const int q = u & 3, p2 = u >> 2;            // stage 2
    PencilArgs pa{};
    pa.frac = 1.0f;
    pa.scale = scale;
    pa.has_m = 0;
#pragma unroll 1
    for (int round = 0; round < 2; ++round) {
        const int p0 = 16 * (2 * round + grp);
        const PencilRegion R{st, p0};
        float4 x[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = st[(j + 4 * m) * PLANE + p0 + p];
        group_sync(grp);                         // the tile is read before it is overwritten
        Z::inv1(x, R, tw, p, j);
        group_sync(grp);
        float4 y[16];
        const float2 kp = kxyp[p0 + p2];
        Z::mid(y, R, tw, kzp, make_float2(pa.scale * kp.x, pa.scale * kp.y), pa, q, p2);
        group_sync(grp);                         // stage-2 reads done
        Z::mid_store(y, R, q, p2);
        group_sync(grp);
        Z::fwd3(x, R, p, j);
        group_sync(grp);                         // stage-3 reads done
#pragma unroll
        for (int m = 0; m < 16; ++m) st[(j + 4 * m) * PLANE + p0 + p] = x[m];
    }
    __syncthreads();

    // plane pass: 64 planes, each warp 4 planes per round, four rounds; the trajectory's entries of the
    // group and stream tables are passed as element 0
#pragma unroll 1
    for (int round = 0; round < 4; ++round) {
        const VBlock vb{t, round, 0, kThreads};
        stepk::plane_body<8, true>(vb, st, NZ, CELLS, gp, tgroup + traj, tlocal + traj, step,
                                   st + round * 16 * PLANE);
    }
    __syncthreads();
    for (int i = t; i < CELLS; i += kThreads) g[i] = st[i];

    if (done) {
        __syncthreads();
        if (t == 0) {
            __threadfence();
            if (atomicAdd(done, 1) == (int)gridDim.x - 1) {
                *done = 0;
                atomicAdd(stepp, 1u);
            }
        }
    }
}

} // namespace

bool fp32_onchip_supported(const ClassGeom &c) { return c.nx == 8 && c.ny == 8 && c.nz == 64 && c.n_traj > 0; }

void fp32_onchip_step(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                      const float2 *tw_full, const float2 *kin_full, uint32_t *d_step, int *inc_done, cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    ensure_smem_limit((const void *)k_onchip_8x8x64, (int)kSmem);
    k_onchip_8x8x64<<<c.n_traj, kThreads, kSmem, s>>>(state, gp, tgroup, tlocal, tw_full, kin_full,
                                                       1.0f / (float)c.cells, d_step, inc_done);
    g_launches++;
}
