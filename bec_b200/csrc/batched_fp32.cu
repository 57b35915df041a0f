// batched_fp32.cu -- the batched FP32 split-step path.
//
// One split step of the reference (propagate, programs/bec_wigner_3d.cuda/
// wigner.cu:178-199: K/2 -> FFT -> N(dt) -> IFFT -> 1/cells -> K/2) is
// regrouped into two fused passes over the state of every trajectory:
//
//   z pass (pencils along z):  IFFT_z -> 1/cells -> K (the previous step's
//                              second half-kick merged with this step's first)
//                              [-> pulse] [-> observe] -> FFT_z
//   plane pass (x-y planes):   FFT_xy -> nonlinear + losses + loss noise
//                              -> IFFT_xy
//
// The stored representation between passes is "k-space along x and y,
// x-space along z", in two scalings: a plane pass reads ifft_xy(psi_x)
// (normalised), so that FFT_xy returns psi_x exactly, and writes
// IFFT_xy(psi_x) (unnormalised, nx*ny times larger), which the next z pass
// turns into ifftn(psi_x) with its 1/cells. A z pass that ends a step (no
// plane pass follows) multiplies by nx*ny on the way out so the state is
// again in the form a z pass reads. Both components of a cell travel together as one float4
// (a.re, a.im, b.re, b.im), so every load and store is a 16-byte vector and
// the nonlinear step sees both components in registers. The FFTs run in
// shared memory (fft_smem.cuh); each pass reads and writes the state once.
#include "engine.h"
#include "fft_smem.cuh"
#include "reduce.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kTileElems = 2048;   // float4 elements per CTA tile (32 KiB)

inline int planes_per_cta(const ClassGeom &c)
{
    int ppc = kTileElems / (c.nx * c.ny);
    if (ppc < 1) ppc = 1;
    if (ppc > c.nz) ppc = c.nz;
    return ppc;
}

inline void ztile(const ClassGeom &c, int &tx, int &ty)
{
    tx = c.nx < 16 ? c.nx : 16;
    ty = kTileElems / (tx * c.nz);
    if (ty < 1) ty = 1;
    if (ty > c.ny) ty = c.ny;
}

// ---------------------------------------------------------------- init
// initializeEnsembles (wigner_kernel.cu:295-317): x-space a = gs + Va eta_a / sqrt(dV),
// b = Vb eta_b / sqrt(dV), eta = (n0 + i n1) / 2 from Philox or injected.
__global__ void k_init(float4 *state, int cells, int ne, GroupParamsF gp, const double2 *gs, const float2 *noise)
{
    const size_t n = (size_t)cells * ne;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(idx / cells);
        const int i = (int)(idx - (size_t)t * cells);
        float2 ea, eb;
        if (noise) {
            ea = noise[((size_t)t * 2 + 0) * cells + i];
            eb = noise[((size_t)t * 2 + 1) * cells + i];
        } else {
            float r[4];
            const uint64_t seed = ((uint64_t)gp.seed_hi << 32) | gp.seed_lo;
            normals4<float>(seed, (uint32_t)t, 0u, (uint32_t)i, RNG_TAG_INIT, r);
            ea = make_float2(0.5f * r[0], 0.5f * r[1]);
            eb = make_float2(0.5f * r[2], 0.5f * r[3]);
        }
        const double2 g = gs[i];
        state[idx] = make_float4((float)g.x + gp.init_a * ea.x, (float)g.y + gp.init_a * ea.y,
                                 gp.init_b * eb.x, gp.init_b * eb.y);
    }
}

// ground-state value i of a complex128 (double2), complex64 (float2) or real FP32 (float) array, as float2
__device__ __forceinline__ float2 gs_value(const double2 *p, int i) { return make_float2((float)p[i].x, (float)p[i].y); }
__device__ __forceinline__ float2 gs_value(const float2 *p, int i) { return p[i]; }
__device__ __forceinline__ float2 gs_value(const float *p, int i) { return make_float2(p[i], 0.f); }

// The same initial state as k_init for a run of trajectories of one grid class that may belong to many
// ensembles: trajectory t of the run takes its ensemble's parameters gp[tgroup[t]], its ground state
// gs_ptrs[tgroup[t]] (complex128, complex64 or real FP32 values, by T), and its Philox stream tlocal[t].
template <typename T>
__global__ void k_init_batched(float4 *state, int cells, int n_traj, const int *__restrict__ tgroup,
                               const int *__restrict__ tlocal, const GroupParamsF *__restrict__ gp,
                               const void *const *__restrict__ gs_ptrs)
{
    const size_t n = (size_t)cells * n_traj;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(idx / cells);
        const int i = (int)(idx - (size_t)t * cells);
        const int grp = tgroup[t];
        const GroupParamsF &P = gp[grp];
        float r[4];
        const uint64_t seed = ((uint64_t)P.seed_hi << 32) | P.seed_lo;
        normals4<float>(seed, (uint32_t)tlocal[t], 0u, (uint32_t)i, RNG_TAG_INIT, r);
        const float2 ea = make_float2(0.5f * r[0], 0.5f * r[1]);
        const float2 eb = make_float2(0.5f * r[2], 0.5f * r[3]);
        const float2 g = gs_value(static_cast<const T *>(gs_ptrs[grp]), i);
        state[idx] = make_float4(g.x + P.init_a * ea.x, g.y + P.init_a * ea.y, P.init_b * eb.x, P.init_b * eb.y);
    }
}

// ---------------------------------------------------------------- plane pass
// mode 0: full step (load bit-reversed, FFT_xy, nonlinear, IFFT_xy, store bit-reversed)
// mode 1: prep (x-space natural in -> IFFT_xy -> stored representation)
// mode 2: unprep (stored representation -> FFT_xy -> x-space natural out)
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_ppass(float4 *state, ClassGeom c, int ppc, const GroupParamsF *gp,
                                                   const int *tgroup, const int *tlocal, const float2 *tw_x,
                                                   const float2 *tw_y, const uint32_t *stepp)
{
    extern __shared__ float4 sm4[];
    const uint32_t step = stepp ? *stepp : 0u;   // Philox step index (device scalar, see fp32_put_step)
    const int plane = c.nx * c.ny;
    const int chunk = ppc * plane;
    float4 *buf = sm4;
    float2 *twx = reinterpret_cast<float2 *>(sm4 + chunk);
    float2 *twy = twx + (c.nx / 2 > 0 ? c.nx / 2 : 1);
    load_twiddles(twx, tw_x, c.nx / 2);
    load_twiddles(twy, tw_y, c.ny / 2);

    const int chunks_per_traj = c.nz / ppc;
    const int traj = blockIdx.x / chunks_per_traj;
    const int z0 = (blockIdx.x - traj * chunks_per_traj) * ppc;
    float4 *g = state + (size_t)traj * c.cells + (size_t)z0 * plane;

    const bool brev_in = (MODE == 0 || MODE == 2);
    for (int idx = threadIdx.x; idx < chunk; idx += blockDim.x) {
        const int x = idx & (c.nx - 1);
        const int y = (idx >> c.lx) & (c.ny - 1);
        const int p = idx >> (c.lx + c.ly);
        const int dst = brev_in ? (p * plane + brev_bits(y, c.ly) * c.nx + brev_bits(x, c.lx)) : idx;
        buf[dst] = g[idx];
    }
    __syncthreads();

    const LineMap mx{c.lx, ppc * c.ny, 1, c.nx, ppc * c.ny, 0, 0};
    const LineMap my{c.ly, ppc * c.nx, c.nx, 1, c.nx, plane, 1};

    if (MODE == 0 || MODE == 2) {
        fft_dit(buf, mx, twx, false);
        fft_dit(buf, my, twy, false);
    }
    if (MODE == 0) {
        const int gi = tgroup[traj];
        const GroupParamsF P = gp[gi];
        const uint32_t tl = (uint32_t)tlocal[traj];
        const uint64_t seed = ((uint64_t)P.seed_hi << 32) | P.seed_lo;
        const float hdt = P.dt * 0.5f;
        for (int idx = threadIdx.x; idx < chunk; idx += blockDim.x) {
            const int x = idx & (c.nx - 1);
            const int y = (idx >> c.lx) & (c.ny - 1);
            const int p = idx >> (c.lx + c.ly);
            const float X = -P.xmax + P.dx * (float)x;
            const float Y = (c.ny > 1) ? -P.ymax + P.dy * (float)y : 0.0f;
            const float Z = -P.zmax + P.dz * (float)(z0 + p);
            const float V = (X * X + Y * Y + Z * Z * P.inv_lambda2) * 0.5f;
            const float4 v0 = buf[idx];
            float2 a0 = make_float2(v0.x, v0.y), b0 = make_float2(v0.z, v0.w);
            float2 xa = a0, xb = b0, da = make_float2(0.f, 0.f), db = make_float2(0.f, 0.f);
            for (int it = 0; it < P.itmax; ++it) {
                const float na = xa.x * xa.x + xa.y * xa.y;
                const float nb = xb.x * xb.x + xb.y * xb.y;
                // propagateXSpaceTwoComponent (wigner_kernel.cu:203-223), reference sign
                const float pa_re = -(P.l111 * na * na + P.l12 * nb) * 0.5f;
                const float pa_im = V + P.g11 * na + P.g12 * nb;
                const float pb_re = -(P.l22 * nb + P.l12 * na) * 0.5f;
                const float pb_im = V + P.g22 * nb + P.g12 * na - P.detuning;
                float sa, ca, sb, cb;
                sincosf(pa_im * hdt, &sa, &ca);
                sincosf(pb_im * hdt, &sb, &cb);
                const float ma = expf(pa_re * hdt), mb = expf(pb_re * hdt);
                da = make_float2(ma * ca, ma * sa);
                db = make_float2(mb * cb, mb * sb);
                xa = cmul(a0, da);
                xb = cmul(b0, db);
            }
            float2 ao = cmul(xa, da), bo = cmul(xb, db);
            if (P.noise) {
                const uint32_t cell = (uint32_t)((z0 + p) * plane + y * c.nx + x);
                float r[6];
                loss_normals6<float>(seed, tl, step, cell, r);
                const float s = P.noise_amp;
                const float2 w1 = make_float2(s * r[0], s * r[1]);
                const float2 w2 = make_float2(s * r[2], s * r[3]);
                const float2 w3 = make_float2(s * r[4], s * r[5]);
                const float2 ca2 = cconj(a0), cb2 = cconj(b0);
                ao = cadd(ao, cadd(cmul(cscale(cmul(ca2, ca2), P.c1), w1), cmul(cscale(cb2, P.c2), w2)));
                bo = cadd(bo, cadd(cmul(cscale(ca2, P.c2), w2), cmul(cscale(cb2, P.c3), w3)));
            }
            buf[idx] = make_float4(ao.x, ao.y, bo.x, bo.y);
        }
        __syncthreads();
    }
    if (MODE == 0 || MODE == 1) {
        fft_dif(buf, my, twy, true);
        fft_dif(buf, mx, twx, true);
    }

    const bool brev_out = (MODE == 0 || MODE == 1);
    for (int idx = threadIdx.x; idx < chunk; idx += blockDim.x) {
        const int x = idx & (c.nx - 1);
        const int y = (idx >> c.lx) & (c.ny - 1);
        const int p = idx >> (c.lx + c.ly);
        const int src = brev_out ? (p * plane + brev_bits(y, c.ly) * c.nx + brev_bits(x, c.lx)) : idx;
        g[idx] = buf[src];
    }
}

// ---------------------------------------------------------------- z pass
// (a, b) <- M (a, b) with M row-major (m11, m12, m21, m22): a Rabi pulse
// (report.tex rotation matrix; applyHalfPiPulse / applyPiPulse,
// wigner_kernel.cu:320-341). It acts identically on every cell, so it
// commutes with the transforms and the kinetic phase.
__device__ __forceinline__ float4 apply_m(const float2 *m, float4 v)
{
    const float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
    const float2 an = cadd(cmul(m[0], a), cmul(m[1], b));
    const float2 bn = cadd(cmul(m[2], a), cmul(m[3], b));
    return make_float4(an.x, an.y, bn.x, bn.y);
}

__global__ void __launch_bounds__(kThreads) k_zpass(float4 *state, ClassGeom c, int tx, int ty,
                                                   const GroupParamsF *gp, const int *tgroup,
                                                   const float2 *tw_z, ZPassArgs za, double *obs_partial)
{
    extern __shared__ float4 sm4[];
    const int npen = tx * ty;
    const int n = c.nz;
    float4 *buf = sm4;
    float2 *twz = reinterpret_cast<float2 *>(sm4 + npen * n);
    load_twiddles(twz, tw_z, n / 2);

    const int tiles_x = c.nx / tx, tiles_y = c.ny / ty;
    const int tiles = tiles_x * tiles_y;
    const int traj = blockIdx.x / tiles;
    const int tile = blockIdx.x - traj * tiles;
    const int x0 = (tile % tiles_x) * tx, y0 = (tile / tiles_x) * ty;
    const int plane = c.nx * c.ny;
    float4 *g = state + (size_t)traj * c.cells;

    for (int idx = threadIdx.x; idx < npen * n; idx += blockDim.x) {
        const int xl = idx % tx;
        const int r = idx / tx;
        const int yl = r % ty;
        const int z = r / ty;
        buf[(yl * tx + xl) * n + brev_bits(z, c.lz)] = g[(size_t)z * plane + (y0 + yl) * c.nx + x0 + xl];
    }
    __syncthreads();

    const LineMap mz{c.lz, npen, 1, n, npen, 0, 0};
    fft_dit(buf, mz, twz, true);     // IFFT_z: now full k-space (unnormalised)

    const GroupParamsF P = gp[tgroup[traj]];
    const float kick_first = za.observe ? za.pre : (za.pre + za.post);
    for (int idx = threadIdx.x; idx < npen * n; idx += blockDim.x) {
        const int pen = idx / n, z = idx - pen * n;
        const int xl = pen % tx, yl = pen / tx;
        const int ix = kidx(x0 + xl, c.nx), iy = c.ny > 1 ? kidx(y0 + yl, c.ny) : 0, iz = kidx(z, n);
        const double k2h = P.kin_x * (double)(ix * ix) + P.kin_y * (double)(iy * iy) + P.kin_z * (double)(iz * iz);
        float4 v = pscale(buf[idx], za.observe ? za.scale : za.scale * za.out_scale);
        if (kick_first != 0.0f)
            v = pmul(v, kin_phase(k2h * (double)kick_first));   // e^{+i k^2/2 dt}, wigner_kernel.cu:143-144
        if (za.has_m1) v = apply_m(za.m1, v);
        if (!za.observe && za.has_m2) v = apply_m(za.m2, v);
        buf[idx] = v;
    }
    __syncthreads();

    if (za.observe) {
        // per-z moments: transform the boundary state along z, sum over the tile's pencils
        fft_dif(buf, mz, twz, false);
        const int tiles_total = tiles;
        for (int z = threadIdx.x; z < n; z += blockDim.x) {
            const int pos = brev_bits(z, c.lz);
            KSum s0, s1, s2, s3;
            for (int pen = 0; pen < npen; ++pen) {
                const float4 v = buf[pen * n + pos];
                s0.add((double)v.x * v.x + (double)v.y * v.y);
                s1.add((double)v.z * v.z + (double)v.w * v.w);
                s2.add((double)v.x * v.z + (double)v.y * v.w);
                s3.add((double)v.x * v.w - (double)v.y * v.z);
            }
            double *o = obs_partial + (((size_t)traj * tiles_total + tile) * n + z) * 4;
            o[0] = s0.value(); o[1] = s1.value(); o[2] = s2.value(); o[3] = s3.value();
        }
        __syncthreads();
        fft_dit(buf, mz, twz, true);   // back to k-space (times nz)
        const float inv_n = za.out_scale / (float)n;
        for (int idx = threadIdx.x; idx < npen * n; idx += blockDim.x) {
            const int pen = idx / n, z = idx - pen * n;
            const int xl = pen % tx, yl = pen / tx;
            float4 v = pscale(buf[idx], inv_n);
            if (za.has_m2) v = apply_m(za.m2, v);
            if (za.post != 0.0f) {
                const int ix = kidx(x0 + xl, c.nx), iy = c.ny > 1 ? kidx(y0 + yl, c.ny) : 0, iz = kidx(z, n);
                const double k2h =
                    P.kin_x * (double)(ix * ix) + P.kin_y * (double)(iy * iy) + P.kin_z * (double)(iz * iz);
                v = pmul(v, kin_phase(k2h * (double)za.post));
            }
            buf[idx] = v;
        }
        __syncthreads();
    }

    fft_dif(buf, mz, twz, false);    // FFT_z back to the stored representation (bit-reversed slots)

    for (int idx = threadIdx.x; idx < npen * n; idx += blockDim.x) {
        const int xl = idx % tx;
        const int r = idx / tx;
        const int yl = r % ty;
        const int z = r / ty;
        g[(size_t)z * plane + (y0 + yl) * c.nx + x0 + xl] = buf[(yl * tx + xl) * n + brev_bits(z, c.lz)];
    }
}

// obs_partial[traj][tile][z][4] -> traj_axial[traj][z][4] (scaled), traj_tot[traj][4]
__global__ void k_obs_reduce(const double *part, int tiles, int nz, const double *traj_scale, double *axial,
                             double *tot)
{
    const int traj = blockIdx.x;
    const double sc = traj_scale ? traj_scale[traj] : 1.0;
    KVec<4> acc;
    for (int z = threadIdx.x; z < nz; z += blockDim.x) {
        KSum s[4];
        for (int t = 0; t < tiles; ++t) {
            const double *p = part + (((size_t)traj * tiles + t) * nz + z) * 4;
            for (int k = 0; k < 4; ++k) s[k].add(p[k]);
        }
        for (int k = 0; k < 4; ++k) {
            const double v = s[k].value() * sc;
            if (axial) axial[((size_t)traj * nz + z) * 4 + k] = v;
            acc.v[k].add(v);
        }
    }
    KVec<4> r = block_reduce<4>(acc);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) tot[(size_t)traj * 4 + k] = r.v[k].value();
}

// FP64 sums of |a|^2, |b|^2 and Re, Im of conj(a) b over the stored state of a class, times `scale`: block
// `idx` sums range idx % blocks (of `blocks` equal ranges) of trajectory idx / blocks and writes
// part[idx * 4 + k], the [traj][tile][z = 0][4] layout of k_obs_reduce with `blocks` tiles.
__global__ void k_state_sums(const float4 *__restrict__ state, int cells, int blocks, double scale,
                             double *__restrict__ part)
{
    const int traj = blockIdx.x / blocks, b = blockIdx.x - traj * blocks;
    const int chunk = (cells + blocks - 1) / blocks;
    const int i0 = b * chunk, i1 = min(cells, i0 + chunk);
    const float4 *p = state + (size_t)traj * cells;
    // plain FP64 sums over a thread's few dozen cells (rounding ~1e-15 relative), compensated across threads
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const float4 u = p[i];
        const double ax = u.x, ay = u.y, bx = u.z, by = u.w;
        s0 = fma(ax, ax, fma(ay, ay, s0));
        s1 = fma(bx, bx, fma(by, by, s1));
        s2 = fma(ax, bx, fma(ay, by, s2));
        s3 = fma(ax, by, fma(-ay, bx, s3));
    }
    KVec<4> acc;
    acc.v[0].add(s0);
    acc.v[1].add(s1);
    acc.v[2].add(s2);
    acc.v[3].add(s3);
    KVec<4> r = block_reduce<4>(acc);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) part[(size_t)blockIdx.x * 4 + k] = r.v[k].value() * scale;
}

__global__ void k_group_reduce(const double *traj_tot, const int *first, const int *count, double *out)
{
    const int gidx = blockIdx.x;
    KVec<4> acc;
    for (int t = threadIdx.x; t < count[gidx]; t += blockDim.x)
        for (int k = 0; k < 4; ++k) acc.v[k].add(traj_tot[((size_t)first[gidx] + t) * 4 + k]);
    KVec<4> r = block_reduce<4>(acc);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) out[(size_t)gidx * 4 + k] = r.v[k].value();
}

size_t ppass_smem(const ClassGeom &c, int ppc)
{
    return sizeof(float4) * (size_t)ppc * c.nx * c.ny + sizeof(float2) * (size_t)((c.nx / 2 > 0 ? c.nx / 2 : 1) + (c.ny / 2 > 0 ? c.ny / 2 : 1));
}

template <int MODE>
void launch_ppass(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                  const float2 *tw_x, const float2 *tw_y, const uint32_t *step, cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    const int ppc = planes_per_cta(c);
    const int blocks = c.n_traj * (c.nz / ppc);
    const size_t smem = ppass_smem(c, ppc);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_ppass<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_ppass<MODE><<<blocks, kThreads, smem, s>>>(state, c, ppc, gp, tgroup, tlocal, tw_x, tw_y, step);
    g_launches++;
}

} // namespace

void fp32_init_group(float4 *state, int cells, int ne, const GroupParamsF &gp, const double2 *gs,
                     const float2 *noise, cudaStream_t s)
{
    size_t n = (size_t)cells * ne;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_init<<<blocks, 256, 0, s>>>(state, cells, ne, gp, gs, noise);
    g_launches++;
}

void fp32_init_batched(float4 *state, int cells, int n_traj, const int *tgroup, const int *tlocal,
                       const GroupParamsF *gp, const void *const *gs_ptrs, int host_type, cudaStream_t s)
{
    size_t n = (size_t)cells * n_traj;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (host_type == BEC_HOST_R32)
        k_init_batched<float><<<blocks, 256, 0, s>>>(state, cells, n_traj, tgroup, tlocal, gp, gs_ptrs);
    else if (host_type == BEC_HOST_C64)
        k_init_batched<float2><<<blocks, 256, 0, s>>>(state, cells, n_traj, tgroup, tlocal, gp, gs_ptrs);
    else
        k_init_batched<double2><<<blocks, 256, 0, s>>>(state, cells, n_traj, tgroup, tlocal, gp, gs_ptrs);
    g_launches++;
}

void fp32_prep(float4 *state, const ClassGeom &c, const float2 *tw_x, const float2 *tw_y, cudaStream_t s)
{
    launch_ppass<1>(state, c, nullptr, nullptr, nullptr, tw_x, tw_y, nullptr, s);
}

void fp32_unprep(float4 *state, const ClassGeom &c, const float2 *tw_x, const float2 *tw_y, cudaStream_t s)
{
    launch_ppass<2>(state, c, nullptr, nullptr, nullptr, tw_x, tw_y, nullptr, s);
}

void fp32_ppass(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                const float2 *tw_x, const float2 *tw_y, const uint32_t *d_step, cudaStream_t s)
{
    launch_ppass<0>(state, c, gp, tgroup, tlocal, tw_x, tw_y, d_step, s);
}

namespace {
__global__ void k_put_step(uint32_t *d, uint32_t v) { *d = v; }
__global__ void k_inc_step(uint32_t *d) { *d += 1u; }
} // namespace

void fp32_put_step(uint32_t *d_step, uint32_t v, cudaStream_t s)
{
    k_put_step<<<1, 1, 0, s>>>(d_step, v);
    g_launches++;
}

void fp32_inc_step(uint32_t *d_step, cudaStream_t s)
{
    k_inc_step<<<1, 1, 0, s>>>(d_step);
    g_launches++;
}

int fp32_zpass_tiles(const ClassGeom &c)
{
    int tx, ty;
    ztile(c, tx, ty);
    return (c.nx / tx) * (c.ny / ty);
}

void fp32_zpass(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const float2 *tw_z,
                const ZPassArgs &z, double *obs_partial, cudaStream_t s)
{
    if (c.n_traj <= 0) return;
    int tx, ty;
    ztile(c, tx, ty);
    const int tiles = (c.nx / tx) * (c.ny / ty);
    const int blocks = c.n_traj * tiles;
    const size_t smem = sizeof(float4) * (size_t)tx * ty * c.nz + sizeof(float2) * (size_t)(c.nz / 2);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_zpass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_zpass<<<blocks, kThreads, smem, s>>>(state, c, tx, ty, gp, tgroup, tw_z, z, obs_partial);
    g_launches++;
}

void obs_reduce(const double *obs_partial, int n_traj, int tiles, int nz, const double *traj_scale,
                double *traj_axial, double *traj_tot, cudaStream_t s)
{
    if (n_traj <= 0) return;
    k_obs_reduce<<<n_traj, 256, 0, s>>>(obs_partial, tiles, nz, traj_scale, traj_axial, traj_tot);
    g_launches++;
}

void fp32_state_sums(const float4 *state, int cells, int n_traj, int blocks, double scale, double *part,
                     cudaStream_t s)
{
    if (n_traj <= 0) return;
    k_state_sums<<<n_traj * blocks, 256, 0, s>>>(state, cells, blocks, scale, part);
    g_launches++;
}

void group_reduce(const double *traj_tot, const int *group_first, const int *group_count, int n_groups,
                  double *out, cudaStream_t s)
{
    if (n_groups <= 0) return;
    k_group_reduce<<<n_groups, 256, 0, s>>>(traj_tot, group_first, group_count, out);
    g_launches++;
}
