// warmstart.cu -- the 64-term correction over Thomas-Fermi used by the warm start.
//
// No counterpart in the reference. A ground state psi of an ensemble is written
// in Thomas-Fermi-scaled coordinates X = x/R, Y = y/R, Zs = z/(lambda R) with
// R = sqrt(2 mu_TF) (the grid spans +-1.2 in each of them for every parameter
// set, wigner.cpp:153-160), amplitude unit A = sqrt(mu_TF / g11):
//     psi / A = f_TF(u) + sum_{i<16, j<4} c_ij B_ij,   f_TF = sqrt(max(1 - u, 0)),
//     B_ij = exp(-((r - r_i) / w_i)^2) P_j(2 cos^2(theta) - 1),
// u = X^2 + Y^2 + Zs^2 = r^2, cos^2(theta) = Zs^2 / u, P_j the Legendre
// polynomials. Four broad radial bumps cover the interior (kinetic-energy
// correction) and twelve narrow ones the condensate edge, where the ground
// state departs most from Thomas-Fermi. The projection solves the normal
// equations of this basis on the grid; the synthesis evaluates the expansion.
//
// Because every parameter set shares the same scaled grid, a basis can also be
// learned: a caller installs up to 64 rows of cell values for one grid (in
// practice the proper orthogonal decomposition of scaled corrections of ground
// states the method computed), and the same projection and synthesis then read
// the rows instead of evaluating the analytic functions.
#include <cmath>
#include <vector>

#include "engine.h"

namespace {

constexpr int kMaxGridY = 65535;   // largest gridDim.y of a launch


constexpr int kRad = 16, kAng = 4, kBasis = kRad * kAng;

__device__ __constant__ float c_rc[kRad];   // radial centres
__device__ __constant__ float c_rw[kRad];   // radial widths

struct WsGeom {
    int nx, ny, nz, lx, ly, cells;
    float dxs, dys, dzs;        // grid steps in scaled units
};

__device__ __forceinline__ void basis_at(int i, const WsGeom &g, float *b, float &ftf)
{
    const int x = i & (g.nx - 1), y = (i >> g.lx) & (g.ny - 1), z = i >> (g.lx + g.ly);
    const float X = -1.2f + g.dxs * x;
    const float Y = (g.ny > 1) ? -1.2f + g.dys * y : 0.0f;
    const float Z = -1.2f + g.dzs * z;
    const float u = X * X + Y * Y + Z * Z;
    const float r = sqrtf(u);
    const float c2 = (u > 0.0f) ? Z * Z / u : 0.0f;
    const float q = 2.0f * c2 - 1.0f;
    const float p[kAng] = {1.0f, q, 0.5f * (3.0f * q * q - 1.0f), 0.5f * q * (5.0f * q * q - 3.0f)};
    ftf = sqrtf(fmaxf(1.0f - u, 0.0f));
#pragma unroll
    for (int a = 0; a < kRad; ++a) {
        const float d = (r - c_rc[a]) / c_rw[a];
        const float e = __expf(-d * d);
#pragma unroll
        for (int j = 0; j < kAng; ++j) b[a * kAng + j] = e * p[j];
    }
}

// Basis values at cell i: the analytic functions, or the rows of an installed table
// (rows >= nb read as zero).
template <bool TAB>
__device__ __forceinline__ void basis_any(int i, const WsGeom &g, const float *tab, int nb, float *b, float &ftf)
{
    if (!TAB) {
        basis_at(i, g, b, ftf);
        return;
    }
    const int x = i & (g.nx - 1), y = (i >> g.lx) & (g.ny - 1), z = i >> (g.lx + g.ly);
    const float X = -1.2f + g.dxs * x;
    const float Y = (g.ny > 1) ? -1.2f + g.dys * y : 0.0f;
    const float Z = -1.2f + g.dzs * z;
    ftf = sqrtf(fmaxf(1.0f - (X * X + Y * Y + Z * Z), 0.0f));
#pragma unroll
    for (int k = 0; k < kBasis; ++k) b[k] = (k < nb) ? tab[(size_t)k * g.cells + i] : 0.0f;
}

// rhs[t][k] = sum_cells B_k d_t,  d_t = |psi_t| / A_t - f_TF  (written to profile when not NULL)
template <bool TAB>
__global__ void k_ws_project(const float2 *psi, int n_traj, WsGeom g, const float *amp, const float *tab, int nb,
                             double *rhs, float *profile)
{
    const int t = blockIdx.y;
    __shared__ double acc[kBasis];
    for (int k = threadIdx.x; k < kBasis; k += blockDim.x) acc[k] = 0.0;
    __syncthreads();
    float loc[kBasis];
#pragma unroll
    for (int k = 0; k < kBasis; ++k) loc[k] = 0.0f;
    const float inv_a = 1.0f / amp[t];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.cells; i += gridDim.x * blockDim.x) {
        float b[kBasis], ftf;
        basis_any<TAB>(i, g, tab, nb, b, ftf);
        const float2 v = psi[(size_t)t * g.cells + i];
        const float d = sqrtf(v.x * v.x + v.y * v.y) * inv_a - ftf;
        if (profile) profile[(size_t)t * g.cells + i] = d;
#pragma unroll
        for (int k = 0; k < kBasis; ++k) loc[k] += b[k] * d;
    }
#pragma unroll
    for (int k = 0; k < kBasis; ++k) {
        float v = loc[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(&acc[k], (double)v);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kBasis; k += blockDim.x) atomicAdd(rhs + (size_t)t * kBasis + k, acc[k]);
}

// gram[k][l] = sum_cells B_k B_l: 256 threads, each owns 16 of the 64 x 64 entries; the basis
// rows of 32 cells at a time are staged in shared memory.
template <bool TAB>
__global__ void __launch_bounds__(256) k_ws_gram(WsGeom g, const float *tab, int nb, double *gram)
{
    __shared__ float rows[32][kBasis];
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
    const int t = threadIdx.x;
    const int k = t >> 2, l0 = (t & 3) * 16;   // row k, columns l0 .. l0 + 15
    for (int base = blockIdx.x * 32; base < g.cells; base += gridDim.x * 32) {
        if (t < 32) {
            float b[kBasis], ftf;
            const int i = base + t;
            if (i < g.cells) {
                basis_any<TAB>(i, g, tab, nb, b, ftf);
#pragma unroll
                for (int q = 0; q < kBasis; ++q) rows[t][q] = b[q];
            } else {
#pragma unroll
                for (int q = 0; q < kBasis; ++q) rows[t][q] = 0.0f;
            }
        }
        __syncthreads();
        float part[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) part[e] = 0.0f;
        for (int c = 0; c < 32; ++c) {
            const float bk = rows[c][k];
#pragma unroll
            for (int e = 0; e < 16; ++e) part[e] += bk * rows[c][l0 + e];
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) acc[e] += part[e];
        __syncthreads();
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) atomicAdd(gram + k * kBasis + l0 + e, acc[e]);
}

// psi_t = A_t max(f_TF + sum c_k B_k, 0) (real, x-space)
template <bool TAB>
__global__ void k_ws_synth(float2 *psi, int n_traj, WsGeom g, const float *amp, const float *coef, const float *tab,
                           int nb)
{
    const int t = blockIdx.y;
    __shared__ float c[kBasis];
    for (int k = threadIdx.x; k < kBasis; k += blockDim.x) c[k] = coef[(size_t)t * kBasis + k];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.cells; i += gridDim.x * blockDim.x) {
        float b[kBasis], ftf;
        basis_any<TAB>(i, g, tab, nb, b, ftf);
        float f = ftf;
#pragma unroll
        for (int k = 0; k < kBasis; ++k) f += c[k] * b[k];
        psi[(size_t)t * g.cells + i] = make_float2(amp[t] * fmaxf(f, 0.0f), 0.0f);
    }
}

bool g_consts_set = false;

cudaError_t set_consts(cudaStream_t s)
{
    if (g_consts_set) return cudaSuccess;
    float rc[kRad], rw[kRad];
    const float broad[4] = {0.0f, 0.3f, 0.55f, 0.75f};
    for (int a = 0; a < 4; ++a) { rc[a] = broad[a]; rw[a] = 0.22f; }
    for (int a = 4; a < kRad; ++a) { rc[a] = 0.80f + 0.045f * (a - 4); rw[a] = 0.06f; }
    // stream-ordered (the work that reads them runs on s, which does not wait for the legacy stream)
    cudaError_t e = cudaMemcpyToSymbolAsync(c_rc, rc, sizeof(rc), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(c_rw, rw, sizeof(rw), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) g_consts_set = true;
    return e;
}

WsGeom geom_dims(int nx, int ny, int nz)
{
    WsGeom g{};
    g.nx = nx; g.ny = ny; g.nz = nz;
    int lx = 0, ly = 0;
    while ((1 << lx) < nx) ++lx;
    while ((1 << ly) < ny) ++ly;
    g.lx = lx; g.ly = ly;
    g.cells = nx * ny * nz;
    g.dxs = 2.4f / (float)(nx - 1);
    g.dys = ny > 1 ? 2.4f / (float)(ny - 1) : 0.0f;
    g.dzs = 2.4f / (float)(nz - 1);
    return g;
}

// Cholesky factor (lower, in place) of the SPD matrix G (upper triangle given) with a small ridge
bool chol_factor(std::vector<double> &G, int n)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) G[i * n + j] = G[j * n + i];
    double ridge = 1e-10 * G[0];
    for (int i = 0; i < n; ++i) G[i * n + i] += ridge;
    for (int j = 0; j < n; ++j) {
        double s = G[j * n + j];
        for (int k = 0; k < j; ++k) s -= G[j * n + k] * G[j * n + k];
        if (s <= 0) return false;
        const double d = std::sqrt(s);
        G[j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double t = G[i * n + j];
            for (int k = 0; k < j; ++k) t -= G[i * n + k] * G[j * n + k];
            G[i * n + j] = t / d;
        }
    }
    return true;
}

void chol_solve(const std::vector<double> &L, const double *r, double *c, int n)
{
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) {
        double t = r[i];
        for (int k = 0; k < i; ++k) t -= L[i * n + k] * y[k];
        y[i] = t / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double t = y[i];
        for (int k = i + 1; k < n; ++k) t -= L[k * n + i] * c[k];
        c[i] = t / L[i * n + i];
    }
}

// Gram matrix of the analytic basis (tab == NULL) or of a table, on the device
cudaError_t gram_of(const WsGeom &g, const float *tab, int nb, std::vector<double> &out, cudaStream_t s)
{
    double *gram = nullptr;
    cudaError_t e = cudaMalloc(&gram, sizeof(double) * kBasis * kBasis);
    if (e) return e;
    cudaMemsetAsync(gram, 0, sizeof(double) * kBasis * kBasis, s);
    if (tab) k_ws_gram<true><<<148, 256, 0, s>>>(g, tab, nb, gram);
    else k_ws_gram<false><<<148, 256, 0, s>>>(g, nullptr, kBasis, gram);
    g_launches++;
    out.assign(kBasis * kBasis, 0.0);
    cudaMemcpyAsync(out.data(), gram, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    cudaFree(gram);
    if (e) return e;
    for (int k = nb; k < kBasis; ++k)       // unused rows: identity (their coefficients come out zero)
        for (int l = 0; l < kBasis; ++l) out[k * kBasis + l] = out[l * kBasis + k] = (k == l) ? 1.0 : 0.0;
    return cudaGetLastError();
}

} // namespace

int warmstart_basis_size() { return kBasis; }

// t.nx, t.ny, t.nz, t.nb set by the caller; host_basis holds nb rows of nx*ny*nz floats
cudaError_t warmstart_table_init(WsTable &t, const float *host_basis, cudaStream_t s)
{
    const WsGeom g = geom_dims(t.nx, t.ny, t.nz);
    const size_t bytes = sizeof(float) * (size_t)g.cells * t.nb;
    cudaError_t e = cudaMalloc(&t.d_basis, bytes);
    if (e) return e;
    if ((e = cudaMemcpyAsync(t.d_basis, host_basis, bytes, cudaMemcpyHostToDevice, s))) return e;
    std::vector<double> G;
    if ((e = gram_of(g, t.d_basis, t.nb, G, s))) return e;
    if (!chol_factor(G, kBasis)) return cudaErrorInvalidValue;   // rows not linearly independent
    t.gram = G;                                                    // kept factored
    return cudaSuccess;
}

// psi: n x cells x-space states (float2, device) of ensembles with derived parameters d[t];
// coef_out: n x 64 (host, may be NULL); profile_out: n x cells scaled corrections |psi|/A - f_TF
// (host, may be NULL)
cudaError_t warmstart_project(const float2 *psi, int n, const bec_derived *d, const WsTable *tab, double *coef_out,
                              float *profile_out, cudaStream_t s)
{
    if (n < 1 || n > kMaxGridY) return cudaErrorInvalidValue;   // n is the launch's grid y
    cudaError_t e = set_consts(s);
    if (e) return e;
    const WsGeom g = geom_dims(d[0].nvx, d[0].nvy, d[0].nvz);
    std::vector<float> amp(n);
    for (int t = 0; t < n; ++t) amp[t] = (float)std::sqrt(d[t].mu / d[t].g11);
    float *damp = nullptr, *dprof = nullptr;
    double *rhs = nullptr;
    if ((e = cudaMalloc(&damp, sizeof(float) * n))) return e;
    if ((e = cudaMalloc(&rhs, sizeof(double) * n * kBasis))) { cudaFree(damp); return e; }
    if (profile_out && (e = cudaMalloc(&dprof, sizeof(float) * (size_t)n * g.cells))) {
        cudaFree(damp); cudaFree(rhs);
        return e;
    }
    cudaMemcpyAsync(damp, amp.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(rhs, 0, sizeof(double) * n * kBasis, s);
    dim3 grid(64, n);
    if (tab) k_ws_project<true><<<grid, 256, 0, s>>>(psi, n, g, damp, tab->d_basis, tab->nb, rhs, dprof);
    else k_ws_project<false><<<grid, 256, 0, s>>>(psi, n, g, damp, nullptr, kBasis, rhs, dprof);
    g_launches++;
    if ((e = cudaGetLastError())) {           // nothing solved from a projection that did not run
        cudaStreamSynchronize(s);
        cudaFree(damp); cudaFree(rhs); cudaFree(dprof);
        return e;
    }
    std::vector<double> hr((size_t)n * kBasis);
    cudaMemcpyAsync(hr.data(), rhs, sizeof(double) * hr.size(), cudaMemcpyDeviceToHost, s);
    if (profile_out)
        cudaMemcpyAsync(profile_out, dprof, sizeof(float) * (size_t)n * g.cells, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    cudaFree(damp); cudaFree(rhs); cudaFree(dprof);
    if (e) return e;
    if (coef_out) {
        std::vector<double> L;
        if (tab) {
            L = tab->gram;
        } else {
            if ((e = gram_of(g, nullptr, kBasis, L, s))) return e;
            if (!chol_factor(L, kBasis)) return cudaErrorInvalidValue;
        }
        for (int t = 0; t < n; ++t) chol_solve(L, hr.data() + (size_t)t * kBasis, coef_out + (size_t)t * kBasis, kBasis);
    }
    return cudaGetLastError();
}

// coef: n x 64 (host); psi_out: n x cells float2 (device)
cudaError_t warmstart_synth(const double *coef, int n, const bec_derived *d, const WsTable *tab, float2 *psi_out,
                            cudaStream_t s)
{
    if (n < 1 || n > kMaxGridY) return cudaErrorInvalidValue;   // n is the launch's grid y
    cudaError_t e = set_consts(s);
    if (e) return e;
    const WsGeom g = geom_dims(d[0].nvx, d[0].nvy, d[0].nvz);
    std::vector<float> amp(n), c((size_t)n * kBasis);
    for (int t = 0; t < n; ++t) amp[t] = (float)std::sqrt(d[t].mu / d[t].g11);
    for (size_t k = 0; k < c.size(); ++k) c[k] = (float)coef[k];
    float *damp = nullptr, *dc = nullptr;
    if ((e = cudaMalloc(&damp, sizeof(float) * n))) return e;
    if ((e = cudaMalloc(&dc, sizeof(float) * c.size()))) { cudaFree(damp); return e; }
    cudaMemcpyAsync(damp, amp.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dc, c.data(), sizeof(float) * c.size(), cudaMemcpyHostToDevice, s);
    dim3 grid(64, n);
    if (tab) k_ws_synth<true><<<grid, 256, 0, s>>>(psi_out, n, g, damp, dc, tab->d_basis, tab->nb);
    else k_ws_synth<false><<<grid, 256, 0, s>>>(psi_out, n, g, damp, dc, nullptr, kBasis);
    g_launches++;
    const cudaError_t el = cudaGetLastError();
    e = cudaStreamSynchronize(s);
    cudaFree(damp); cudaFree(dc);
    return el ? el : e;
}
