// nn.cu -- the warm-start network: a small MLP trained and evaluated on the GPU.
//
// No counterpart in the reference. The network maps an ensemble's parameters
// to the coefficients of a correction to the Thomas-Fermi profile; its output
// only seeds the imaginary-time ground-state loop (bec_ground_state_batch),
// which alone decides convergence.
//
// Layers are Y = act(X W^T + b) (W is [out x in], row-major, as a linear layer),
// tanh on hidden layers, identity on the last. GEMMs run on the 5th-generation
// tensor cores (tcgen05.mma, BF16 operands from shared memory, FP32 accumulator in
// tensor memory) with split operands: every FP32 operand x is held as two BF16
// values, hi = bf16(x) and lo = bf16(x - hi), and a product is accumulated as
// hi*hi + hi*lo + lo*hi (three MMAs), about 16 significant bits per operand instead
// of 8. Single BF16 products limited the trained network (its loss stalled at the
// BF16 rounding level and its warm starts needed 1.6x the steps of the same
// network trained in FP32). Master weights, Adam moments, activations' pre-images
// and gradients are FP32.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "engine.h"

namespace {

// ---------------------------------------------------------------- GEMM on the 5th-generation tensor cores
// C[M x N] = A[M x K] * B[N x K]^T (+ bias[N]) with A = A_hi + A_lo, B = B_hi + B_lo (BF16 row-major, K contiguous);
// C FP32; M, N, K multiples of 64. One CTA of 128 threads per 128 x 64 tile of C. The FP32 accumulator lives in
// tensor memory (64 columns, lane i = row i of the tile). K runs in groups of up to four 64-wide stages: the threads
// copy every stage's four tiles (A and B, hi and lo) to shared memory at once (cp.async, 16 bytes each) in the
// K-major canonical layout without swizzle (8-row x 16-byte core matrices; the two 16-byte K chunks of one
// instruction 128 B apart, consecutive 8-row groups 1024 B apart), then one thread issues, per 16-wide K step, the
// three tcgen05.mma (M 128, N 64, K 16, BF16 in, FP32 accumulate) lo*hi, hi*lo, hi*hi, and tcgen05.commit arrives
// on an mbarrier when they are done; every wait is bounded. Rows of a last 64-row tile (M = 64 mod 128) are zero in
// A and not stored. The epilogue reads the accumulator with tcgen05.ld (warp w owns lanes 32w..32w+31), adds the
// bias and stores FP32 rows.
constexpr int GM = 128, GN = 64, GK = 64, GSTAGES = 4;
constexpr int kTileA = GM * GK * 2, kTileB = GN * GK * 2;     // 16 KiB, 8 KiB
constexpr int kStageBytes = 2 * (kTileA + kTileB);          // hi and lo of both: 48 KiB
constexpr int kGemmSmem = GSTAGES * kStageBytes + 64;       // + mbarrier and TMEM slot: 192 KiB, one CTA per SM
// instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(GN >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading byte offset >> 4 (16-29) = the K-chunk
// stride 128 B, stride byte offset >> 4 (32-45) = the 8-row group stride 1024 B, descriptor version 1 (46-47),
// no swizzle (61-63 = 0)
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, unsigned long long limit_ns)
{
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_test(bar, parity))
        if (now_ns() - t0 > limit_ns) return false;
    return true;
}

// a wait for a flag that nothing sets (fault injection): false after limit_ns
__device__ __noinline__ bool wait_flag(const int *flag, unsigned long long limit_ns)
{
    const unsigned long long t0 = now_ns();
    while (*(volatile const int *)flag == 0) {
        __nanosleep(1000);
        if (now_ns() - t0 > limit_ns) return false;
    }
    return true;
}

// one tcgen05.mma of the tile: D (+)= A B^T from the shared-memory descriptors; accumulate = 0 overwrites D
__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(accumulate)
                 : "memory");
}

__global__ void __launch_bounds__(128) k_gemm_tc(const __nv_bfloat16 *__restrict__ A, const __nv_bfloat16 *__restrict__ Alo,
                                                 const __nv_bfloat16 *__restrict__ B, const __nv_bfloat16 *__restrict__ Blo,
                                                 float *__restrict__ C, const float *__restrict__ bias, int M, int N,
                                                 int K, int *err, const int *never, int stall,
                                                 unsigned long long limit_ns)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    // stage g at g * kStageBytes: A_hi (128 rows x 64 K), B_hi (64 rows x 64 K), A_lo, B_lo
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + GSTAGES * kStageBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + GSTAGES * kStageBytes + 8);
    const int t = threadIdx.x, warp = t >> 5;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(saddr(tslot)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;

    uint32_t parity = 0;
    bool failed = false;
    for (int kg = 0; kg < K; kg += GSTAGES * GK) {
        const int stages = min(GSTAGES, (K - kg) / GK);
        // chunk c (16 bytes = 8 K values) of a tile sits at byte 16 c: 8-row group c / 64, K chunk (c / 8) % 8,
        // row c % 8; A rows past M are zero-filled (source size 0)
        for (int g = 0; g < stages; ++g) {
            const int k0 = kg + g * GK;
            unsigned char *As = sm + g * kStageBytes, *Bs = As + kTileA, *Als = Bs + kTileB, *Bls = Als + kTileA;
            for (int c = t; c < GM * 8; c += 128) {
                const int row = (c >> 6) * 8 + (c & 7), kc = (c >> 3) & 7;
                const bool in = m0 + row < M;
                const size_t off = (size_t)(in ? m0 + row : 0) * K + k0 + kc * 8;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(As + 16 * c)), "l"(A + off),
                             "r"(in ? 16 : 0)
                             : "memory");
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(Als + 16 * c)), "l"(Alo + off),
                             "r"(in ? 16 : 0)
                             : "memory");
            }
            for (int c = t; c < GN * 8; c += 128) {
                const int row = (c >> 6) * 8 + (c & 7), kc = (c >> 3) & 7;
                const size_t off = (size_t)(n0 + row) * K + k0 + kc * 8;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(Bs + 16 * c)), "l"(B + off)
                             : "memory");
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(Bls + 16 * c)), "l"(Blo + off)
                             : "memory");
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the tiles, visible to the tensor core
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int g = 0; g < stages; ++g) {
                const uint32_t as = saddr(sm + g * kStageBytes), bs = as + kTileA, als = bs + kTileB,
                               bls = als + kTileA;
#pragma unroll
                for (int kk = 0; kk < GK / 16; ++kk) {
                    const uint64_t ad = kmajor_desc(as + 256 * kk), bd = kmajor_desc(bs + 256 * kk);
                    const uint64_t ald = kmajor_desc(als + 256 * kk), bld = kmajor_desc(bls + 256 * kk);
                    // the small products first; only the very first MMA of the tile starts D afresh
                    mma_f16(tmem, ald, bd, (kg > 0 || g > 0 || kk > 0) ? 1u : 0u);
                    mma_f16(tmem, ad, bld, 1u);
                    mma_f16(tmem, ad, bd, 1u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(saddr(bar)) : "memory");
        }
        // the group's MMAs read the tiles: every thread waits for them before the next group overwrites them;
        // stall (fault injection): the first group also waits for a flag that nothing sets
        bool ok = mbar_wait_bounded(saddr(bar), parity, limit_ns);
        if (stall && kg == 0 && ok) ok = wait_flag(never, limit_ns);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        parity ^= 1u;
    }
    if (failed) {
        // a wait that ran out: report it, give the group's MMAs once more the limit, free the columns
        if (t == 0) atomicExch(err, 1);
        mbar_wait_bounded(saddr(bar), parity, limit_ns);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
        return;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + (t & 31);
#pragma unroll
    for (int cb = 0; cb < GN; cb += 16) {
        uint32_t r[16];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                     "%13, %14, %15}, [%16];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                       "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                       "=r"(r[15])
                     : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < M) {
            float4 *dst = reinterpret_cast<float4 *>(C + (size_t)row * N + n0 + cb);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 o = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                       __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
                if (bias) {
                    const float4 b = *reinterpret_cast<const float4 *>(bias + n0 + cb + 4 * q);
                    o.x += b.x; o.y += b.y; o.z += b.z; o.w += b.w;
                }
                dst[q] = o;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
}

// the split of an FP32 value into hi = bf16(v) and lo = bf16(v - hi)
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16(v);
    lo = __float2bfloat16(v - __bfloat162float(hi));
}

// y = tanh(z) (or z on the output layer), FP32, and its split (yhi, ylo) for the next GEMM
__global__ void k_act(const float *z, float *y, __nv_bfloat16 *yhi, __nv_bfloat16 *ylo, size_t n, int linear)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = linear ? z[i] : tanhf(z[i]);
        y[i] = v;
        split_bf16(v, yhi[i], ylo[i]);
    }
}

// dZ = dY * (1 - y^2) (tanh) or dY (linear)
__global__ void k_act_back(const float *dy, const float *y, float *dz, size_t n, int linear)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dz[i] = linear ? dy[i] : dy[i] * (1.0f - y[i] * y[i]);
}

// (hi, lo)[c][r] = split(in[r][c]) for an R x Cn FP32 matrix (also plain splits with transpose = 0)
__global__ void k_cast_t(const float *in, __nv_bfloat16 *hi, __nv_bfloat16 *lo, int R, int Cn, int transpose)
{
    const size_t n = (size_t)R * Cn;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / Cn), c = (int)(i - (size_t)r * Cn);
        const size_t o = transpose ? (size_t)c * R + r : i;
        split_bf16(in[i], hi[o], lo[o]);
    }
}

// db[c] = sum_r dz[r][c]
__global__ void k_colsum(const float *dz, float *db, int R, int Cn)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Cn) return;
    float s = 0.0f;
    for (int r = 0; r < R; ++r) s += dz[(size_t)r * Cn + c];
    db[c] = s;
}

// dY = 2 (y - t) / (B * out) over the first `valid` rows (padding rows get 0), out = the caller's output width
// (real_cols; the padding columns of y and t are zero); loss partials
__global__ void k_mse(const float *y, const float *tgt, float *dy, int rows, int valid, int cols, int real_cols,
                      float *loss)
{
    const size_t n = (size_t)rows * cols;
    float l = 0.0f;
    const float s = 2.0f / ((float)valid * real_cols);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols);
        const float d = (r < valid) ? y[i] - tgt[i] : 0.0f;
        dy[i] = s * d;
        l += d * d;
    }
    for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / ((float)valid * real_cols));
}

__global__ void k_adam(float *w, float *m, float *v, const float *g, size_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// gather rows idx[r] of src (n_src x cols) into dst (rows x cols), zero rows past `valid`
__global__ void k_gather(const float *src, const int *idx, float *dst, int rows, int valid, int cols)
{
    const size_t n = (size_t)rows * cols;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i - (size_t)r * cols);
        dst[i] = (r < valid) ? src[(size_t)idx[r] * cols + c] : 0.0f;
    }
}

inline int grid_for(size_t n) { size_t b = (n + 255) / 256; return (int)(b > 4096 ? 4096 : (b < 1 ? 1 : b)); }

} // namespace

struct bec_mlp {
    std::vector<int> w;              // widths (padded): w[0] = padded inputs
    std::vector<int> w_real;         // caller's widths
    int L = 0;                       // weight layers
    std::vector<size_t> woff, boff;  // offsets into the parameter vector
    size_t n_params = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // FP32 params, grads, Adam moments
    __nv_bfloat16 *pbf = nullptr, *plo = nullptr;   // the weights' split [out x in] (hi, lo)
    __nv_bfloat16 *wt = nullptr, *wtlo = nullptr;   // scratch for the split of W^T
    int cap = 0;                     // batch capacity of the activation buffers
    std::vector<float *> z, y;       // per layer: pre-activation, activation (FP32) [cap x w]
    std::vector<__nv_bfloat16 *> xbf, xlo;   // per layer the input's split [cap x w]
    float *dy = nullptr, *dz = nullptr, *loss = nullptr;
    __nv_bfloat16 *tA = nullptr, *tB = nullptr, *tAlo = nullptr, *tBlo = nullptr;   // split scratch operands
    int *idx = nullptr;
    int *d_err = nullptr;            // [0] set by a GEMM whose wait ran out, [1] a flag nothing sets
    float *xin = nullptr, *tgt = nullptr;
    long long adam_t = 0;
    cudaStream_t s = nullptr;
    std::string err;
    std::vector<void *> allocs;
};

namespace {

bec_status mlp_alloc(bec_mlp *m, void **p, size_t bytes)
{
    if (cudaMalloc(p, bytes ? bytes : 16) != cudaSuccess) { cudaGetLastError(); return BEC_ERR_OUT_OF_MEMORY; }
    m->allocs.push_back(*p);
    return BEC_OK;
}

int round_up(int v, int q) { return (v + q - 1) / q * q; }

bec_status mlp_reserve(bec_mlp *m, int batch)
{
    if (batch <= m->cap) return BEC_OK;
    const int cap = round_up(batch, 64);
    int maxw = 0;
    for (int v : m->w) maxw = std::max(maxw, v);
    m->z.assign(m->L + 1, nullptr);
    m->y.assign(m->L + 1, nullptr);
    m->xbf.assign(m->L + 1, nullptr);
    m->xlo.assign(m->L + 1, nullptr);
    bec_status st;
    for (int l = 0; l <= m->L; ++l) {
        if ((st = mlp_alloc(m, (void **)&m->z[l], sizeof(float) * cap * m->w[l]))) return st;
        if ((st = mlp_alloc(m, (void **)&m->y[l], sizeof(float) * cap * m->w[l]))) return st;
        if ((st = mlp_alloc(m, (void **)&m->xbf[l], sizeof(__nv_bfloat16) * cap * m->w[l]))) return st;
        if ((st = mlp_alloc(m, (void **)&m->xlo[l], sizeof(__nv_bfloat16) * cap * m->w[l]))) return st;
    }
    if ((st = mlp_alloc(m, (void **)&m->dy, sizeof(float) * cap * maxw))) return st;
    if ((st = mlp_alloc(m, (void **)&m->dz, sizeof(float) * cap * maxw))) return st;
    if ((st = mlp_alloc(m, (void **)&m->tA, sizeof(__nv_bfloat16) * cap * maxw))) return st;
    if ((st = mlp_alloc(m, (void **)&m->tB, sizeof(__nv_bfloat16) * cap * maxw))) return st;
    if ((st = mlp_alloc(m, (void **)&m->tAlo, sizeof(__nv_bfloat16) * cap * maxw))) return st;
    if ((st = mlp_alloc(m, (void **)&m->tBlo, sizeof(__nv_bfloat16) * cap * maxw))) return st;
    if ((st = mlp_alloc(m, (void **)&m->tgt, sizeof(float) * cap * m->w[m->L]))) return st;
    m->cap = cap;
    return BEC_OK;
}

// C[M x N] = A[M x K] B[N x K]^T (+ bias) on m's stream; A and B each as their split (hi, lo)
void gemm_bt(bec_mlp *m, const __nv_bfloat16 *A, const __nv_bfloat16 *Alo, const __nv_bfloat16 *B,
             const __nv_bfloat16 *Blo, float *C, const float *bias, int M, int N, int K)
{
    ensure_smem_limit((const void *)k_gemm_tc, kGemmSmem);
    // BEC_STEP_WAIT_LIMIT_MS bounds the device-side waits (2 s by default); BEC_GEMM_INJECT_STALL=1 makes the
    // first K group of every CTA also wait for a flag that nothing sets (the error path, without a fault)
    unsigned long long limit_ns = 2000000000ull;
    if (const char *v = std::getenv("BEC_STEP_WAIT_LIMIT_MS")) limit_ns = 1000000ull * std::strtoull(v, nullptr, 10);
    const char *inj = std::getenv("BEC_GEMM_INJECT_STALL");
    const int stall = inj && std::atoi(inj) ? 1 : 0;
    dim3 grid(N / GN, (M + GM - 1) / GM);
    k_gemm_tc<<<grid, 128, kGemmSmem, m->s>>>(A, Alo, B, Blo, C, bias, M, N, K, m->d_err, m->d_err + 1, stall,
                                             limit_ns);
    g_launches++;
}

// BEC_ERR_CUDA when a GEMM since the last check gave up a wait (synchronises the stream)
bec_status check_gemm(bec_mlp *m)
{
    int e = 0;
    if (cudaMemcpyAsync(&e, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, m->s) != cudaSuccess ||
        cudaStreamSynchronize(m->s) != cudaSuccess) {
        m->err = cudaGetErrorString(cudaGetLastError());
        return BEC_ERR_CUDA;
    }
    if (e) {
        cudaMemsetAsync(m->d_err, 0, sizeof(int), m->s);
        m->err = "MLP GEMM: a tensor-core wait gave up";
        return BEC_ERR_CUDA;
    }
    return BEC_OK;
}

// forward on the first `rows` (multiple of 64) rows of y[0] (FP32 inputs, padded)
void mlp_forward_dev(bec_mlp *m, int rows)
{
    cudaStream_t s = m->s;
    k_cast_t<<<grid_for((size_t)rows * m->w[0]), 256, 0, s>>>(m->y[0], m->xbf[0], m->xlo[0], rows, m->w[0], 0);
    for (int l = 0; l < m->L; ++l) {
        const int in = m->w[l], out = m->w[l + 1];
        gemm_bt(m, m->xbf[l], m->xlo[l], m->pbf + m->woff[l], m->plo + m->woff[l], m->z[l + 1], m->p + m->boff[l],
                rows, out, in);
        const int linear = (l == m->L - 1);
        k_act<<<grid_for((size_t)rows * out), 256, 0, s>>>(m->z[l + 1], m->y[l + 1], m->xbf[l + 1], m->xlo[l + 1],
                                                           (size_t)rows * out, linear);
        g_launches++;
    }
    g_launches++;
}

// gradients of the MSE loss into m->g, after mlp_forward_dev; targets in m->tgt
void mlp_backward_dev(bec_mlp *m, int rows, int valid)
{
    cudaStream_t s = m->s;
    const int outw = m->w[m->L];
    cudaMemsetAsync(m->loss, 0, sizeof(float), s);
    k_mse<<<grid_for((size_t)rows * outw), 256, 0, s>>>(m->y[m->L], m->tgt, m->dy, rows, valid, outw,
                                                        m->w_real[m->L], m->loss);
    g_launches++;
    for (int l = m->L - 1; l >= 0; --l) {
        const int in = m->w[l], out = m->w[l + 1];
        const int linear = (l == m->L - 1);
        k_act_back<<<grid_for((size_t)rows * out), 256, 0, s>>>(m->dy, m->y[l + 1], m->dz, (size_t)rows * out, linear);
        k_colsum<<<(out + 127) / 128, 128, 0, s>>>(m->dz, m->g + m->boff[l], rows, out);
        // dW [out x in] = dZ^T [out x rows] * (X^T [in x rows])^T
        k_cast_t<<<grid_for((size_t)rows * out), 256, 0, s>>>(m->dz, m->tA, m->tAlo, rows, out, 1);
        k_cast_t<<<grid_for((size_t)rows * in), 256, 0, s>>>(m->y[l], m->tB, m->tBlo, rows, in, 1);
        gemm_bt(m, m->tA, m->tAlo, m->tB, m->tBlo, m->g + m->woff[l], nullptr, out, in, rows);
        g_launches += 4;
        if (l > 0) {
            // dX [rows x in] = dZ [rows x out] * W [out x in] = dZ * (W^T [in x out])^T
            k_cast_t<<<grid_for((size_t)rows * out), 256, 0, s>>>(m->dz, m->tA, m->tAlo, rows, out, 0);
            k_cast_t<<<grid_for((size_t)out * in), 256, 0, s>>>(m->p + m->woff[l], m->wt, m->wtlo, out, in, 1);
            gemm_bt(m, m->tA, m->tAlo, m->wt, m->wtlo, m->dy, nullptr, rows, in, out);
            g_launches += 2;
        }
    }
}

void mlp_sync_bf16(bec_mlp *m)
{
    for (int l = 0; l < m->L; ++l) {
        k_cast_t<<<grid_for((size_t)m->w[l] * m->w[l + 1]), 256, 0, m->s>>>(m->p + m->woff[l], m->pbf + m->woff[l],
                                                                             m->plo + m->woff[l], m->w[l + 1], m->w[l],
                                                                             0);
        g_launches++;
    }
}

// host x (batch x real_in) -> device y[0] (rows x padded_in)
bec_status upload_inputs(bec_mlp *m, const float *x, int batch, int rows)
{
    std::vector<float> h((size_t)rows * m->w[0], 0.0f);
    for (int r = 0; r < batch; ++r)
        for (int c = 0; c < m->w_real[0]; ++c) h[(size_t)r * m->w[0] + c] = x[(size_t)r * m->w_real[0] + c];
    if (cudaMemcpyAsync(m->y[0], h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, m->s) != cudaSuccess)
        return BEC_ERR_CUDA;
    return cudaStreamSynchronize(m->s) == cudaSuccess ? BEC_OK : BEC_ERR_CUDA;
}

} // namespace

extern "C" {

bec_status bec_mlp_create(const int32_t *widths, int32_t n_layers, uint64_t seed, bec_mlp **out)
{
    if (!out) return BEC_ERR_INVALID_ARG;
    *out = nullptr;
    if (!widths || n_layers < 1 || n_layers > 16) return BEC_ERR_INVALID_ARG;
    for (int l = 0; l <= n_layers; ++l)
        if (widths[l] < 1 || widths[l] > 4096) return BEC_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return BEC_ERR_NO_DEVICE; }
    bec_mlp *m = new bec_mlp();
    m->L = n_layers;
    m->w_real.assign(widths, widths + n_layers + 1);
    m->w.resize(n_layers + 1);
    for (int l = 0; l <= n_layers; ++l) m->w[l] = round_up(widths[l], 64);   // GEMM tiles are 64 wide
    for (int l = 0; l < n_layers; ++l) {
        m->woff.push_back(m->n_params);
        m->n_params += (size_t)m->w[l] * m->w[l + 1];
        m->boff.push_back(m->n_params);
        m->n_params += (size_t)m->w[l + 1];
    }
    auto bail = [&](bec_status st) { bec_mlp_destroy(m); return st; };
    bec_status st;
    if (cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) != cudaSuccess) return bail(BEC_ERR_CUDA);
    if ((st = mlp_alloc(m, (void **)&m->p, sizeof(float) * m->n_params))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->g, sizeof(float) * m->n_params))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->m, sizeof(float) * m->n_params))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->v, sizeof(float) * m->n_params))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->pbf, sizeof(__nv_bfloat16) * m->n_params))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->plo, sizeof(__nv_bfloat16) * m->n_params))) return bail(st);
    int maxw = 0;
    for (int v : m->w) maxw = std::max(maxw, v);
    if ((st = mlp_alloc(m, (void **)&m->wt, sizeof(__nv_bfloat16) * maxw * maxw))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->wtlo, sizeof(__nv_bfloat16) * maxw * maxw))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->loss, sizeof(float)))) return bail(st);
    if ((st = mlp_alloc(m, (void **)&m->d_err, 2 * sizeof(int)))) return bail(st);
    if (cudaMemsetAsync(m->d_err, 0, 2 * sizeof(int), m->s) != cudaSuccess) return bail(BEC_ERR_CUDA);
    // Glorot-uniform weights on the real block, zero padding and biases
    std::vector<float> h(m->n_params, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < n_layers; ++l) {
        const float a = std::sqrt(6.0f / (float)(widths[l] + widths[l + 1]));
        std::uniform_real_distribution<float> U(-a, a);
        for (int o = 0; o < widths[l + 1]; ++o)
            for (int i = 0; i < widths[l]; ++i) h[m->woff[l] + (size_t)o * m->w[l] + i] = U(rng);
    }
    cudaMemcpyAsync(m->p, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, m->s);
    cudaMemsetAsync(m->m, 0, sizeof(float) * m->n_params, m->s);
    cudaMemsetAsync(m->v, 0, sizeof(float) * m->n_params, m->s);
    mlp_sync_bf16(m);
    if (cudaStreamSynchronize(m->s) != cudaSuccess) return bail(BEC_ERR_CUDA);
    *out = m;
    return BEC_OK;
}

void bec_mlp_destroy(bec_mlp *m)
{
    if (!m) return;
    if (m->s) cudaStreamSynchronize(m->s);
    for (void *p : m->allocs) cudaFree(p);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
}

int64_t bec_mlp_param_count(const bec_mlp *m)
{
    if (!m) return 0;
    int64_t n = 0;
    for (int l = 0; l < m->L; ++l) n += (int64_t)m->w_real[l] * m->w_real[l + 1] + m->w_real[l + 1];
    return n;
}

// host layout: for each layer W [out x in] row-major then b [out] (caller's widths)
bec_status bec_mlp_get_params(bec_mlp *m, float *params)
{
    if (!m || !params) return BEC_ERR_INVALID_ARG;
    std::vector<float> h(m->n_params);
    cudaMemcpyAsync(h.data(), m->p, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, m->s);
    if (cudaStreamSynchronize(m->s) != cudaSuccess) return BEC_ERR_CUDA;
    size_t k = 0;
    for (int l = 0; l < m->L; ++l) {
        for (int o = 0; o < m->w_real[l + 1]; ++o)
            for (int i = 0; i < m->w_real[l]; ++i) params[k++] = h[m->woff[l] + (size_t)o * m->w[l] + i];
        for (int o = 0; o < m->w_real[l + 1]; ++o) params[k++] = h[m->boff[l] + o];
    }
    return BEC_OK;
}

bec_status bec_mlp_set_params(bec_mlp *m, const float *params)
{
    if (!m || !params) return BEC_ERR_INVALID_ARG;
    std::vector<float> h(m->n_params, 0.0f);
    size_t k = 0;
    for (int l = 0; l < m->L; ++l) {
        for (int o = 0; o < m->w_real[l + 1]; ++o)
            for (int i = 0; i < m->w_real[l]; ++i) h[m->woff[l] + (size_t)o * m->w[l] + i] = params[k++];
        for (int o = 0; o < m->w_real[l + 1]; ++o) h[m->boff[l] + o] = params[k++];
    }
    if (cudaMemcpyAsync(m->p, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, m->s) != cudaSuccess) return BEC_ERR_CUDA;
    mlp_sync_bf16(m);
    return cudaStreamSynchronize(m->s) == cudaSuccess ? BEC_OK : BEC_ERR_CUDA;
}

bec_status bec_mlp_forward(bec_mlp *m, const float *x, int32_t batch, float *y)
{
    if (!m || !x || !y || batch < 1) return BEC_ERR_INVALID_ARG;
    const int rows = round_up(batch, 64);
    bec_status st;
    if ((st = mlp_reserve(m, rows))) return st;
    if ((st = upload_inputs(m, x, batch, rows))) return st;
    mlp_forward_dev(m, rows);
    const int ow = m->w[m->L];
    std::vector<float> h((size_t)rows * ow);
    if (cudaMemcpyAsync(h.data(), m->y[m->L], sizeof(float) * h.size(), cudaMemcpyDeviceToHost, m->s) != cudaSuccess)
        return BEC_ERR_CUDA;
    if ((st = check_gemm(m))) return st;
    for (int r = 0; r < batch; ++r)
        for (int c = 0; c < m->w_real[m->L]; ++c) y[(size_t)r * m->w_real[m->L] + c] = h[(size_t)r * ow + c];
    return BEC_OK;
}

// Loss and gradients of mean((y - target)^2) over the batch (host params layout).
bec_status bec_mlp_gradients(bec_mlp *m, const float *x, const float *target, int32_t batch, float *loss,
                             float *grads)
{
    if (!m || !x || !target || batch < 1) return BEC_ERR_INVALID_ARG;
    const int rows = round_up(batch, 64);
    bec_status st;
    if ((st = mlp_reserve(m, rows))) return st;
    if ((st = upload_inputs(m, x, batch, rows))) return st;
    const int ow = m->w[m->L];
    std::vector<float> t((size_t)rows * ow, 0.0f);
    for (int r = 0; r < batch; ++r)
        for (int c = 0; c < m->w_real[m->L]; ++c) t[(size_t)r * ow + c] = target[(size_t)r * m->w_real[m->L] + c];
    cudaMemcpyAsync(m->tgt, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice, m->s);
    mlp_forward_dev(m, rows);
    mlp_backward_dev(m, rows, batch);
    float l = 0.f;
    cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->s);
    std::vector<float> h(m->n_params);
    cudaMemcpyAsync(h.data(), m->g, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, m->s);
    if ((st = check_gemm(m))) return st;
    if (loss) *loss = l;
    if (grads) {
        size_t k = 0;
        for (int li = 0; li < m->L; ++li) {
            for (int o = 0; o < m->w_real[li + 1]; ++o)
                for (int i = 0; i < m->w_real[li]; ++i) grads[k++] = h[m->woff[li] + (size_t)o * m->w[li] + i];
            for (int o = 0; o < m->w_real[li + 1]; ++o) grads[k++] = h[m->boff[li] + o];
        }
    }
    return BEC_OK;
}

// Adam on minibatches drawn (seeded) from n samples; loss_history[s] = loss of step s. Every
// minibatch's indices are drawn up front and uploaded once, and the losses stay on the device
// until the end, so the step loop issues work without waiting on the GPU.
bec_status bec_mlp_train(bec_mlp *m, const float *x, const float *target, int32_t n, int32_t batch, int32_t steps,
                         float lr, int32_t schedule, uint64_t seed, float *loss_history)
{
    if (!m || !x || !target || n < 1 || batch < 1 || steps < 0) return BEC_ERR_INVALID_ARG;
    if (schedule != BEC_LR_CONSTANT && schedule != BEC_LR_COSINE) return BEC_ERR_INVALID_ARG;
    const int rows = round_up(batch, 64);
    bec_status st;
    if ((st = mlp_reserve(m, rows))) return st;
    const int in_r = m->w_real[0], out_r = m->w_real[m->L], inw = m->w[0], ow = m->w[m->L];
    float *dx = nullptr, *dt = nullptr, *dhist = nullptr;
    int *didx = nullptr;
    std::vector<void *> loc;
    auto lalloc = [&](void **p, size_t b) {
        cudaError_t e = cudaMalloc(p, b > 0 ? b : 16);
        if (e == cudaSuccess) loc.push_back(*p);
        return e;
    };
    struct F { std::vector<void *> &v; cudaStream_t s; ~F() { cudaStreamSynchronize(s); for (void *p : v) cudaFree(p); } } f{loc, m->s};
    if (lalloc((void **)&dx, sizeof(float) * (size_t)n * inw) || lalloc((void **)&dt, sizeof(float) * (size_t)n * ow) ||
        lalloc((void **)&didx, sizeof(int) * (size_t)rows * steps) || lalloc((void **)&dhist, sizeof(float) * steps))
        return BEC_ERR_OUT_OF_MEMORY;
    {
        std::vector<float> hx((size_t)n * inw, 0.0f), ht((size_t)n * ow, 0.0f);
        for (int r = 0; r < n; ++r) {
            for (int c = 0; c < in_r; ++c) hx[(size_t)r * inw + c] = x[(size_t)r * in_r + c];
            for (int c = 0; c < out_r; ++c) ht[(size_t)r * ow + c] = target[(size_t)r * out_r + c];
        }
        cudaMemcpyAsync(dx, hx.data(), sizeof(float) * hx.size(), cudaMemcpyHostToDevice, m->s);
        cudaMemcpyAsync(dt, ht.data(), sizeof(float) * ht.size(), cudaMemcpyHostToDevice, m->s);
    }
    // minibatches: consecutive slices of seeded shuffles of the n samples
    std::mt19937_64 rng(seed);
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    int pos = n;
    const int valid = std::min(batch, n);
    std::vector<int> hidx((size_t)rows * steps, 0);
    for (int s = 0; s < steps; ++s)
        for (int r = 0; r < valid; ++r) {
            if (pos >= n) { std::shuffle(order.begin(), order.end(), rng); pos = 0; }
            hidx[(size_t)s * rows + r] = order[pos++];
        }
    if (steps > 0) cudaMemcpyAsync(didx, hidx.data(), sizeof(int) * hidx.size(), cudaMemcpyHostToDevice, m->s);
    const double pi = 3.14159265358979323846;
    for (int s = 0; s < steps; ++s) {
        const int *bidx = didx + (size_t)s * rows;
        k_gather<<<grid_for((size_t)rows * inw), 256, 0, m->s>>>(dx, bidx, m->y[0], rows, valid, inw);
        k_gather<<<grid_for((size_t)rows * ow), 256, 0, m->s>>>(dt, bidx, m->tgt, rows, valid, ow);
        mlp_forward_dev(m, rows);
        mlp_backward_dev(m, rows, valid);
        ++m->adam_t;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - std::pow(b1, (float)m->adam_t), c2 = 1.0f - std::pow(b2, (float)m->adam_t);
        const float lr_s = schedule == BEC_LR_COSINE ? (float)(lr * 0.5 * (1.0 + std::cos(pi * s / steps))) : lr;
        k_adam<<<grid_for(m->n_params), 256, 0, m->s>>>(m->p, m->m, m->v, m->g, m->n_params, lr_s, b1, b2, 1e-8f, c1,
                                                        c2);
        mlp_sync_bf16(m);
        cudaMemcpyAsync(dhist + s, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, m->s);
        g_launches += 3;
    }
    std::vector<float> hist(steps, 0.0f);
    if (steps > 0) cudaMemcpyAsync(hist.data(), dhist, sizeof(float) * steps, cudaMemcpyDeviceToHost, m->s);
    if ((st = check_gemm(m))) return st;
    if (loss_history)
        for (int s = 0; s < steps; ++s) loss_history[s] = hist[s];
    return cudaGetLastError() == cudaSuccess ? BEC_OK : BEC_ERR_CUDA;
}

} // extern "C"
