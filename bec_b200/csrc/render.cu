// render.cu -- headless density projections and their colour map.
//
// The reference draws, after its second pi/2 pulse (halfPiRotate with alpha = 0,
// wigner_kernel.cu:344-360) and the Wigner subtraction (density, :283-286), the
// density of each component summed over the ensemble and projected on the xy
// plane (sum over z) and the zy plane (sum over x) (wigner.cu:384-410), then
// maps level / max through a blue-white-yellow-red ramp of 3 x 255 colours with
// linear filtering into an OpenGL buffer (spectre.cu:34-46, :63-99;
// drawState, wigner.cu:413-430). Here the same arithmetic writes RGBA floats
// into device memory for the caller; no graphics API is involved.
#include "engine.h"

namespace {

// (a', b') = ((a - i b)/sqrt2, (-i a + b)/sqrt2); densities minus sub, accumulated
__global__ void k_project(const float4 *x, int nx, int lx, int ny, int ly, int nz, float in_scale, float sub,
                          float *xy_a, float *xy_b, float *zy_a, float *zy_b)
{
    const int cells = nx * ny * nz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) {
        const float4 v = x[i];
        const float ar = v.x * in_scale, ai = v.y * in_scale, br = v.z * in_scale, bi = v.w * in_scale;
        // a - i b = (ar + bi) + i (ai - br); -i a + b = (ai + br) + i (bi - ar); |.|^2 / 2 from the 1/sqrt2
        const float pa = ((ar + bi) * (ar + bi) + (ai - br) * (ai - br)) * 0.5f - sub;
        const float pb = ((ai + br) * (ai + br) + (bi - ar) * (bi - ar)) * 0.5f - sub;
        const int xx = i & (nx - 1), yy = (i >> lx) & (ny - 1), zz = i >> (lx + ly);
        atomicAdd(xy_a + yy * nx + xx, pa);
        atomicAdd(xy_b + yy * nx + xx, pb);
        atomicAdd(zy_a + yy * nz + zz, pa);
        atomicAdd(zy_b + yy * nz + zz, pb);
    }
}

// blueToRedSpectre (spectre.cu:34-46) as a continuous ramp sampled like a linearly
// filtered, clamped, normalised 1D texture of 765 texels
__device__ float3 ramp_texel(int idx)
{
    if (idx < 0) return make_float3(0.f, 0.f, 0.f);
    float r, g, b;
    if (idx <= 255) { r = (float)idx; g = (float)idx; b = 255.f; }
    else if (idx <= 510) { r = 255.f; g = 255.f; b = (float)(510 - idx); }
    else if (idx <= 765) { r = 255.f; g = (float)(765 - idx); b = 0.f; }
    else { r = 255.f; g = 0.f; b = 0.f; }
    return make_float3(r / 256.f, g / 256.f, b / 256.f);
}

__global__ void k_colour(const float *level, int n, float inv_max, float4 *rgba)
{
    const int texels = 765;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float u = level[i] * inv_max;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        const float p = u * texels - 0.5f;
        int i0 = (int)floorf(p);
        const float f = p - (float)i0;
        int i1 = i0 + 1;
        i0 = max(0, min(i0, texels - 1));
        i1 = max(0, min(i1, texels - 1));
        const float3 c0 = ramp_texel(i0), c1 = ramp_texel(i1);
        rgba[i] = make_float4(c0.x + f * (c1.x - c0.x), c0.y + f * (c1.y - c0.y), c0.z + f * (c1.z - c0.z), 1.0f);
    }
}

} // namespace

void render_project(const float4 *x, const ClassGeom &c, float in_scale, float sub, float *xy_a, float *xy_b,
                    float *zy_a, float *zy_b, cudaStream_t s)
{
    int blocks = (c.cells + 255) / 256;
    if (blocks > 2048) blocks = 2048;
    k_project<<<blocks, 256, 0, s>>>(x, c.nx, c.lx, c.ny, c.ly, c.nz, in_scale, sub, xy_a, xy_b, zy_a, zy_b);
    g_launches++;
}

void render_colour(const float *level, int n, float max_level, float4 *rgba, cudaStream_t s)
{
    int blocks = (n + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    k_colour<<<blocks, 256, 0, s>>>(level, n, 1.0f / max_level, rgba);
    g_launches++;
}
