// plain_fp64.cu -- the plain per-trajectory FP64 path.
//
// Structured like the reference's propagate() (programs/bec_wigner_3d.cuda/
// wigner.cu:178-199): one kernel per operation, one trajectory at a time,
// separate passes for the k-space kick, each FFT axis, the nonlinear step and
// the 1/cells scaling. It is the FP64 parity path (matches the CPU oracle to
// ~1e-12 relative) and the baseline that the batched FP32 path is measured
// against. FFT axes use this library's shared-memory radix-2 stages
// (fft_smem.cuh) in place of cuFFT + transposes (batchfft.cu:130-180).
#include <mutex>
#include <set>
#include <utility>

#include "engine.h"
#include "fft_smem.cuh"
#include "reduce.cuh"

thread_local long long g_launches = 0;

cudaError_t ensure_smem_limit(const void *kernel, int bytes)
{
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (done.count({kernel, dev})) return cudaSuccess;
    if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    done.insert({kernel, dev});
    return cudaSuccess;
}

namespace {

__device__ __forceinline__ void cell_xyz(int i, const GeomD &g, int &x, int &y, int &z)
{
    x = i & (g.nx - 1);
    y = (i >> g.lx) & (g.ny - 1);
    z = i >> (g.lx + g.ly);
}

// (kx^2 + ky^2 + kz^2) / 2 of cell i (initWaveVectors, wigner_kernel.cu:25-41)
__device__ __forceinline__ double k2half(int i, const GeomD &g)
{
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    double kx = getk<double>(x, g.dkx, g.nx);
    double ky = (g.ny > 1) ? getk<double>(y, g.dky, g.ny) : 0.0;
    double kz = getk<double>(z, g.dkz, g.nz);
    return (kx * kx + ky * ky + kz * kz) / 2.0;
}

// potential (wigner_kernel.cu:99-113)
__device__ __forceinline__ double potential(int i, const GeomD &g)
{
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    double xx = -g.xmax + g.dx * x;
    double yy = (g.ny > 1) ? -g.ymax + g.dy * y : 0.0;
    double zz = -g.zmax + g.dz * z;
    return (xx * xx + yy * yy + zz * zz / (g.lambda * g.lambda)) / 2.0;
}

__device__ __forceinline__ double2 cexp_d(double re, double im)
{
    double m = exp(re), s, c;
    sincos(im, &s, &c);
    return make_double2(m * c, m * s);
}

// propagateKSpaceRealTime (wigner_kernel.cu:137-151), optionally preceded by
// multiplyPair's 1/cells (wigner_kernel.cu:269-274)
__global__ void k_kick(double2 *a, double2 *b, GeomD g, double scale, int apply_scale)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    double ang = k2half(i, g) * g.dt_evo / 2.0;
    double s, c;
    sincos(ang, &s, &c);
    double2 w = make_double2(c, s);
    double2 va = a[i], vb = b[i];
    if (apply_scale) { va = cscale(va, scale); vb = cscale(vb, scale); }
    a[i] = cmul(va, w);
    b[i] = cmul(vb, w);
}

// One FFT axis over `lines` lines of n elements with element stride `stride`
// (line l starts at (l / stride) * stride * n + l % stride).
__global__ void k_fft_axis(double2 *data, int n, int logn, int stride, int lines, int lpc, const double2 *tw,
                           int inv)
{
    extern __shared__ double2 sm[];
    double2 *twd = sm + lpc * n;
    load_twiddles(twd, tw, n / 2);
    const int l0 = blockIdx.x * lpc;
    const int L = min(lpc, lines - l0);
    for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
        int ll, e;
        if (stride == 1) { ll = idx / n; e = idx - ll * n; }
        else { e = idx / L; ll = idx - e * L; }
        const int l = l0 + ll;
        const size_t base = (size_t)(l / stride) * stride * n + (l % stride);
        sm[ll * n + brev_bits(e, logn)] = data[base + (size_t)e * stride];
    }
    __syncthreads();
    LineMap m{logn, L, 1, n, L, 0, 0};
    fft_dit(sm, m, twd, inv != 0);
    for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
        int ll, e;
        if (stride == 1) { ll = idx / n; e = idx - ll * n; }
        else { e = idx / L; ll = idx - e * L; }
        const int l = l0 + ll;
        const size_t base = (size_t)(l / stride) * stride * n + (l % stride);
        data[base + (size_t)e * stride] = sm[ll * n + e];
    }
}

// propagateXSpaceTwoComponent (wigner_kernel.cu:184-229) plus the Wigner
// loss-noise increment evaluated at the start of the substep.
__global__ void k_nl(double2 *a, double2 *b, GeomD g, uint32_t traj, uint32_t step)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    const double V = potential(i, g);
    const double dt = g.dt_evo;
    double2 a0 = a[i], b0 = b[i], x = a0, y = b0;
    double2 da = make_double2(0, 0), db = make_double2(0, 0);
    for (int it = 0; it < g.itmax; ++it) {
        double na = x.x * x.x + x.y * x.y;
        double nb = y.x * y.x + y.y * y.y;
        double pa_re = -(g.l111 * na * na + g.l12 * nb) / 2.0;
        double pa_im = -(-V - g.g11 * na - g.g12 * nb);
        double pb_re = -(g.l22 * nb + g.l12 * na) / 2.0;
        double pb_im = -(-V - g.g22 * nb - g.g12 * na + g.detuning);
        da = cexp_d(pa_re * (dt / 2.0), pa_im * (dt / 2.0));
        db = cexp_d(pb_re * (dt / 2.0), pb_im * (dt / 2.0));
        x = cmul(a0, da);
        y = cmul(b0, db);
    }
    double2 ao = cmul(x, da), bo = cmul(y, db);
    if (g.noise) {
        double r[6];
        loss_normals6<double>(g.seed, traj, step, (uint32_t)i, r);
        const double ns = sqrt(dt / (2.0 * g.dV));
        const double c1 = sqrt(g.l111 / 6.0) * 3.0, c2 = sqrt(g.l12 / 2.0), c3 = sqrt(g.l22);
        double2 w1 = make_double2(ns * r[0], ns * r[1]);
        double2 w2 = make_double2(ns * r[2], ns * r[3]);
        double2 w3 = make_double2(ns * r[4], ns * r[5]);
        double2 ca = cconj(a0), cb = cconj(b0);
        ao = cadd(ao, cadd(cmul(cscale(cmul(ca, ca), c1), w1), cmul(cscale(cb, c2), w2)));
        bo = cadd(bo, cadd(cmul(cscale(ca, c2), w2), cmul(cscale(cb, c3), w3)));
    }
    a[i] = ao;
    b[i] = bo;
}

__global__ void k_scale(double2 *a, int n, double s)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = cscale(a[i], s);
}

__global__ void k_pulse(double2 *a, double2 *b, int n, double2 m11, double2 m12, double2 m21, double2 m22)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 u = a[i], v = b[i];
    a[i] = cadd(cmul(m11, u), cmul(m12, v));
    b[i] = cadd(cmul(m21, u), cmul(m22, v));
}

// initializeEnsembles (wigner_kernel.cu:295-317) for one trajectory, x-space.
__global__ void k_init(double2 *a, double2 *b, const double2 *gs, const double2 *na, const double2 *nb, GeomD g,
                       uint32_t traj)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    const double coeff = 1.0 / sqrt(g.dV);
    double2 ea, eb;
    if (na) {
        ea = na[i];
        eb = nb[i];
    } else {
        double r[4];
        normals4<double>(g.seed, traj, 0u, (uint32_t)i, RNG_TAG_INIT, r);
        ea = make_double2(0.5 * r[0], 0.5 * r[1]);
        eb = make_double2(0.5 * r[2], 0.5 * r[3]);
    }
    a[i] = cadd(gs[i], cscale(cscale(ea, g.Va), coeff));
    b[i] = cscale(cscale(eb, g.Vb), coeff);
}

// per-z sums of one x-space trajectory, one block per z plane
__global__ void k_axial(const double2 *a, const double2 *b, GeomD g, double *out)
{
    const int plane = g.nx * g.ny;
    const int z = blockIdx.x;
    KVec<4> acc;
    for (int i = threadIdx.x; i < plane; i += blockDim.x) {
        double2 u = a[(size_t)z * plane + i], v = b[(size_t)z * plane + i];
        acc.v[0].add(u.x * u.x + u.y * u.y);
        acc.v[1].add(v.x * v.x + v.y * v.y);
        acc.v[2].add(u.x * v.x + u.y * v.y);
        acc.v[3].add(u.x * v.y - u.y * v.x);
    }
    KVec<4> r = block_reduce<4>(acc);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) out[4 * z + k] += r.v[k].value() * g.dV;
    }
}

// fillWithTFGroundState (wigner_kernel.cu:116-125)
__global__ void k_gs_tf(double2 *a, GeomD g, double mu)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    double e = mu - potential(i, g);
    a[i] = (e > 0) ? make_double2(sqrt(e / g.g11), 0.0) : make_double2(0.0, 0.0);
}

// propagateKSpaceImaginaryTime (wigner_kernel.cu:128-134)
__global__ void k_gs_kick(double2 *a, GeomD g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    a[i] = cscale(a[i], exp(-g.dt_steady / 2.0 * k2half(i, g)));
}

// propagateXSpaceOneComponent (wigner_kernel.cu:154-181)
__global__ void k_gs_nl(double2 *a, GeomD g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    const double V = potential(i, g);
    double2 a0 = a[i], x = a0;
    double da = 0.0;
    for (int it = 0; it < g.itmax; ++it) {
        double n = x.x * x.x + x.y * x.y;
        da = exp(g.dt_steady / 2.0 * (-V - g.g11 * n));
        x = cscale(a0, da);
    }
    a[i] = cscale(x, da);
}

__global__ void k_renorm(double2 *a, int n, const double *sum, double N, double dV)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double sc = sqrt(N / (sum[0] * dV));
    a[i] = cscale(a[i], sc);
}

__global__ void k_mul_k2(const double2 *ak, double2 *hk, GeomD g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.cells) return;
    hk[i] = cscale(ak[i], k2half(i, g));
}

struct F_abs2 {
    const double2 *a;
    __device__ void operator()(int i, double *v) const { double2 u = a[i]; v[0] = u.x * u.x + u.y * u.y; }
};

struct F_xsums {
    const double2 *a;
    GeomD g;
    __device__ void operator()(int i, double *v) const
    {
        double2 u = a[i];
        double n = u.x * u.x + u.y * u.y;
        v[0] = n * potential(i, g);
        v[1] = n * n;
        v[2] = n;
    }
};

struct F_ksum {
    const double2 *a;
    GeomD g;
    __device__ void operator()(int i, double *v) const
    {
        double2 u = a[i];
        v[0] = (u.x * u.x + u.y * u.y) * k2half(i, g);
    }
};

// calculateNonlinearEnergyPart + combineNonlinearAndDifferential
// (wigner_kernel.cu:232-238, :250-258): n (V + g11 n / 2) + Re(psi_x[i] psi_k[i] k_i^2/2)
struct F_refE {
    const double2 *ax, *ak;
    GeomD g;
    __device__ void operator()(int i, double *v) const
    {
        double2 u = ax[i];
        double n = u.x * u.x + u.y * u.y;
        double r = n * (potential(i, g) + g.g11 * n / 2.0);
        double2 t = cmul(u, cscale(ak[i], k2half(i, g)));
        v[0] = r + t.x;
    }
};

struct F_resid {
    const double2 *ax, *hk;
    GeomD g;
    double mu;
    __device__ void operator()(int i, double *v) const
    {
        double2 u = ax[i];
        double n = u.x * u.x + u.y * u.y;
        double f = potential(i, g) + g.g11 * n - mu;
        double2 h = cadd(hk[i], cscale(u, f));
        v[0] = h.x * h.x + h.y * h.y;
    }
};

// |a - prev|^2 and |a|^2: the fixed-point residual of the imaginary-time map between checks
struct F_diff2 {
    const double2 *a, *prev;
    __device__ void operator()(int i, double *v) const
    {
        const double2 u = a[i], p = prev[i];
        const double dx = u.x - p.x, dy = u.y - p.y;
        v[0] = dx * dx + dy * dy;
        v[1] = u.x * u.x + u.y * u.y;
    }
};

inline int nblk(int n) { return (n + 255) / 256; }

} // namespace

void plain_kick(double2 *a, double2 *b, const GeomD &g, double scale, int apply_scale, cudaStream_t s)
{
    k_kick<<<nblk(g.cells), 256, 0, s>>>(a, b, g, scale, apply_scale);
    g_launches++;
}

static void fft_axis(double2 *data, int n, int logn, int stride, int lines, const double2 *tw, int inv,
                     cudaStream_t s)
{
    if (n == 1) return;
    int lpc = 2048 / n;
    if (lpc < 1) lpc = 1;
    if (lpc > lines) lpc = lines;
    const int blocks = (lines + lpc - 1) / lpc;
    const size_t smem = sizeof(double2) * ((size_t)lpc * n + n / 2);
    k_fft_axis<<<blocks, 256, smem, s>>>(data, n, logn, stride, lines, lpc, tw, inv);
    g_launches++;
}

void plain_fft3d(double2 *data, const GeomD &g, const double2 *tw_x, const double2 *tw_y, const double2 *tw_z,
                 int inv, cudaStream_t s)
{
    fft_axis(data, g.nx, g.lx, 1, g.ny * g.nz, tw_x, inv, s);
    fft_axis(data, g.ny, g.ly, g.nx, g.nx * g.nz, tw_y, inv, s);
    fft_axis(data, g.nz, g.lz, g.nx * g.ny, g.nx * g.ny, tw_z, inv, s);
}

void plain_nl(double2 *a, double2 *b, const GeomD &g, uint32_t traj, uint32_t step, cudaStream_t s)
{
    k_nl<<<nblk(g.cells), 256, 0, s>>>(a, b, g, traj, step);
    g_launches++;
}

void plain_scale(double2 *a, int n, double scale, cudaStream_t s)
{
    k_scale<<<nblk(n), 256, 0, s>>>(a, n, scale);
    g_launches++;
}

void plain_pulse(double2 *a, double2 *b, int n, double2 m11, double2 m12, double2 m21, double2 m22,
                 cudaStream_t s)
{
    k_pulse<<<nblk(n), 256, 0, s>>>(a, b, n, m11, m12, m21, m22);
    g_launches++;
}

void plain_init(double2 *a, double2 *b, const double2 *gs, const double2 *noise_a, const double2 *noise_b,
                const GeomD &g, uint32_t traj, cudaStream_t s)
{
    k_init<<<nblk(g.cells), 256, 0, s>>>(a, b, gs, noise_a, noise_b, g, traj);
    g_launches++;
}

void plain_axial_sums(const double2 *a, const double2 *b, const GeomD &g, double *out, cudaStream_t s)
{
    k_axial<<<g.nz, 256, 0, s>>>(a, b, g, out);
    g_launches++;
}

void plain_gs_tf(double2 *a, const GeomD &g, double mu, cudaStream_t s)
{
    k_gs_tf<<<nblk(g.cells), 256, 0, s>>>(a, g, mu);
    g_launches++;
}

void plain_gs_kick(double2 *a, const GeomD &g, cudaStream_t s)
{
    k_gs_kick<<<nblk(g.cells), 256, 0, s>>>(a, g);
    g_launches++;
}

void plain_gs_nl(double2 *a, const GeomD &g, cudaStream_t s)
{
    k_gs_nl<<<nblk(g.cells), 256, 0, s>>>(a, g);
    g_launches++;
}

void plain_norm(const double2 *a, int n, double *out, double *tmp, cudaStream_t s)
{
    reduce_sum<1>(F_abs2{a}, n, out, tmp, s);
    g_launches += 2;
}

void plain_renorm(double2 *a, int n, const double *sum, double N, double dV, cudaStream_t s)
{
    k_renorm<<<nblk(n), 256, 0, s>>>(a, n, sum, N, dV);
    g_launches++;
}

void plain_gs_xsums(const double2 *a, const GeomD &g, double *out, double *tmp, cudaStream_t s)
{
    reduce_sum<3>(F_xsums{a, g}, g.cells, out, tmp, s);
    g_launches += 2;
}

void plain_gs_ksum(const double2 *ak, const GeomD &g, double *out, double *tmp, cudaStream_t s)
{
    reduce_sum<1>(F_ksum{ak, g}, g.cells, out, tmp, s);
    g_launches += 2;
}

void plain_gs_ref_energy(const double2 *ax, const double2 *ak, const GeomD &g, double *out, double *tmp,
                         cudaStream_t s)
{
    reduce_sum<1>(F_refE{ax, ak, g}, g.cells, out, tmp, s);
    g_launches += 2;
}

void plain_gs_residual(const double2 *ax, const double2 *hk, const GeomD &g, double mu, double *out, double *tmp,
                       cudaStream_t s)
{
    reduce_sum<1>(F_resid{ax, hk, g, mu}, g.cells, out, tmp, s);
    g_launches += 2;
}

void plain_diff2(const double2 *a, const double2 *prev, int n, double *out, double *tmp, cudaStream_t s)
{
    reduce_sum<2>(F_diff2{a, prev}, n, out, tmp, s);
    g_launches += 2;
}

void plain_mul_k2(const double2 *ak, double2 *hk, const GeomD &g, cudaStream_t s)
{
    k_mul_k2<<<nblk(g.cells), 256, 0, s>>>(ak, hk, g);
    g_launches++;
}
