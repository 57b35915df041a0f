// pencil_tma.cu -- the pencil pass of the FP32 path (IFFT_z -> kinetic phase [-> pulse] -> FFT_z of every
// pencil of a grid class; kinetic step of programs/bec_wigner_3d.cuda/wigner_kernel.cu:137-151 between the
// z transforms of batchfft.cu) as a persistent kernel whose tiles move by TMA.
//
// The register pencil kernel (fused_passes.cu) loads a tile, computes, stores, and leaves the overlap of
// memory and arithmetic to whichever other CTA of the SM happens to be loading; at two CTAs per SM both are
// often computing and HBM idles (about 0.75 of the copy bandwidth). Here each CTA walks a contiguous run of
// tiles with the next tile's load always in flight:
//
//   tile i in buffer b = i & 1:  wait full[b] -> registers -> barrier -> [thread 0: wait until the store of
//   tile i - 1 has read buffer b ^ 1, then TMA-load tile i + 1 into it] -> z transform through buffer b
//   (ZTile, the same stages and arithmetic as the register kernel) -> result to buffer b in the tile's
//   global layout -> TMA store.
//
// A tile is PEN = 2048 / nz adjacent pencils (32 KiB: 8 x 256, 16 x 128, 32 x 64) of one trajectory, a box
// of {4 PEN floats, nz rows} of the class's state seen as a 2D tensor {4 nx ny floats, nz n_traj rows}.
// 128 threads, two tile buffers, three CTAs per SM: three loads and up to three stores in flight per SM.
// Each TMA load feeds only the CTA that issues it, and a tile's source is this GPU's own memory.
//
// Every wait is bounded: a load that has not landed after the limit (BEC_STEP_WAIT_LIMIT_MS, 2 s by
// default) sets the error flag, waits once more (bounded) for that load, drains its own stores and ends
// the CTA; the host reads the flag after the pass (bec_status BEC_ERR_CUDA). BEC_PENCIL_INJECT_STALL=1 makes
// the first tile of every CTA also wait for a flag that nothing sets, which exercises that path without
// any fault.
#include <cuda.h>
#include <cstdlib>

#include "engine.h"
#include "step_bodies.cuh"

namespace {

using stepk::PencilArgs;
using stepk::ZTile;

constexpr int kThreads = 128;
constexpr int kTileBytes = 32768;

template <int NZ>
constexpr size_t tma_smem_bytes()
{
    // two tiles, W_NZ^e and the kz factors (NZ float2 each), the pencil factors (PEN float2), two mbarriers,
    // the abort flag
    return 2 * (size_t)kTileBytes + sizeof(float2) * (2 * NZ + 2048 / NZ) + 2 * sizeof(uint64_t) + 16;
}

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(saddr(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

// true once the phase with this parity has completed; false after limit_ns without it
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, unsigned long long limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_try_wait(bar, parity))
        if (now_ns() - t0 > limit_ns) return false;
    return true;
}

// a wait for a flag that nothing sets (fault injection): returns false after limit_ns
__device__ __noinline__ bool wait_never(const int *flag, unsigned long long limit_ns)
{
    const unsigned long long t0 = now_ns();
    while (*(volatile const int *)flag == 0) {
        __nanosleep(1000);
        if (now_ns() - t0 > limit_ns) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(saddr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int x, int y, const void *src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

struct TmaArgs {
    int plane;                   // nx ny: pencils per trajectory
    int tiles_per_traj;          // plane / PEN
    int n_tiles;                 // n_traj tiles_per_traj
    const float2 *tw;            // W_NZ^e, e < NZ
    const float2 *kin;           // per trajectory: NZ kz factors, then plane pencil factors; null: no kick
    PencilArgs pa;
    int *err;                    // set to 1 when a wait gave up
    const int *never;            // a zero flag (fault injection)
    int stall;
    unsigned long long wait_limit_ns;
};

template <int NZ>
__global__ void __launch_bounds__(kThreads, 3) k_pencil_tma(const __grid_constant__ CUtensorMap map, TmaArgs A)
{
    constexpr int PEN = 2048 / NZ, G = NZ / 16, R = 16;
    static_assert(PEN * G == kThreads && PEN * NZ * 16 == kTileBytes, "tile shape");
    using Z = ZTile<NZ, PEN>;
    extern __shared__ __align__(1024) unsigned char smem[];
    float4 *bufs = reinterpret_cast<float4 *>(smem);
    float2 *tw = reinterpret_cast<float2 *>(smem + 2 * kTileBytes);
    float2 *kzp = tw + NZ;
    float2 *kxyp = kzp + NZ;
    uint64_t *full = reinterpret_cast<uint64_t *>(kxyp + PEN);
    int *abort_flag = reinterpret_cast<int *>(full + 2);

    const int t = threadIdx.x;
    const int first = (int)((long long)A.n_tiles * blockIdx.x / gridDim.x);
    const int last = (int)((long long)A.n_tiles * (blockIdx.x + 1) / gridDim.x);
    if (first >= last) return;

    if (t == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    for (int e = t; e < NZ; e += kThreads) tw[e] = A.tw[e];
    __syncthreads();
    if (t == 0) {
        const int traj = first / A.tiles_per_traj;
        mbar_expect_tx(&full[0], kTileBytes);
        tma_load_2d(bufs, &map, 4 * PEN * (first - traj * A.tiles_per_traj), traj * NZ, &full[0]);
    }
    if (!A.kin) {
        for (int e = t; e < NZ; e += kThreads) kzp[e] = make_float2(1.f, 0.f);
        if (t < PEN) kxyp[t] = make_float2(1.f, 0.f);
    }

    const int p = t % PEN, j = t / PEN;      // stages 1 and 3
    const int q = t % G, p2 = t / G;         // stage 2
    int cur_traj = -1;
    for (int i = first; i < last; ++i) {
        const int b = (i - first) & 1;
        const uint32_t parity = (uint32_t)((i - first) >> 1) & 1u;
        float4 *B = bufs + b * (kTileBytes / 16);
        const int traj = i / A.tiles_per_traj;
        const int pen0 = (i - traj * A.tiles_per_traj) * PEN;
        // this tile's kinetic factors: the kz table when the trajectory changes, the pencils' every tile
        // (the previous tile's last reads of both were before its final barriers)
        if (A.kin) {
            const float2 *kt = A.kin + (size_t)traj * (NZ + A.plane);
            if (traj != cur_traj)
                for (int e = t; e < NZ; e += kThreads) stepk::copy_async8(kzp + e, kt + e);
            if (t < PEN) stepk::copy_async8(kxyp + t, kt + NZ + pen0 + t);
        }
        cur_traj = traj;

        bool ok = mbar_wait_bounded(&full[b], parity, A.wait_limit_ns);
        if (A.stall && i == first && ok) ok = wait_never(A.never, A.wait_limit_ns);
        float4 x[R];
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = B[(j + G * m) * PEN + p];
        if (!ok) *abort_flag = 1;
        __syncthreads();                                   // buffer b read; abort decided
        if (*abort_flag) {
            if (t == 0) {
                atomicExch(A.err, 1);
                mbar_wait_bounded(&full[b], parity, A.wait_limit_ns);   // this tile's load, still in flight?
                bulk_wait0();
            }
            stepk::copy_async_wait();
            return;
        }
        if (t == 0 && i + 1 < last) {
            const int tn = (i + 1) / A.tiles_per_traj;
            bulk_wait_read0();                             // tile i - 1's store has read buffer b ^ 1
            mbar_expect_tx(&full[b ^ 1], kTileBytes);
            tma_load_2d(bufs + (b ^ 1) * (kTileBytes / 16), &map, 4 * PEN * (i + 1 - tn * A.tiles_per_traj), tn * NZ,
                        &full[b ^ 1]);
        }

        Z::inv1(x, B, tw, p, j);
        stepk::copy_async_wait();
        __syncthreads();
        float4 y[R];
        const float2 kp = kxyp[p2];
        Z::mid(y, B, tw, kzp, make_float2(A.pa.scale * kp.x, A.pa.scale * kp.y), A.pa, q, p2);
        __syncthreads();                                   // stage-2 reads done
        Z::mid_store(y, B, q, p2);
        __syncthreads();
        Z::fwd3(x, B, p, j);
        __syncthreads();                                   // stage-3 reads done
#pragma unroll
        for (int m = 0; m < R; ++m) B[(j + G * m) * PEN + p] = x[m];
        fence_proxy_async();                               // the generic writes, visible to the TMA store
        __syncthreads();
        if (t == 0) tma_store_2d(&map, 4 * pen0, traj * NZ, B);
    }
    if (t == 0) bulk_wait0();
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    // looked up once per process (a thread-safe static initialisation)
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
        return nullptr;
    }();
    return fn;
}

struct TmaEnv {
    int stall = 0;
    unsigned long long wait_limit_ns = 2000000000ull;
    TmaEnv()
    {
        if (const char *v = std::getenv("BEC_STEP_WAIT_LIMIT_MS")) wait_limit_ns = 1000000ull * std::strtoull(v, nullptr, 10);
        if (const char *v = std::getenv("BEC_PENCIL_INJECT_STALL")) stall = std::atoi(v) ? 1 : 0;
    }
};

template <int NZ>
cudaError_t launch_tma(float4 *state, const ClassGeom &c, const TmaArgs &A0, cudaStream_t s)
{
    constexpr int PEN = 2048 / NZ;
    const int plane = c.nx * c.ny;
    if (plane % PEN) return cudaErrorInvalidValue;
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    CUtensorMap map;
    const cuuint64_t dims[2] = {(cuuint64_t)4 * plane, (cuuint64_t)c.nz * c.n_traj};
    const cuuint64_t strides[1] = {(cuuint64_t)plane * sizeof(float4)};
    const cuuint32_t box[2] = {4 * PEN, NZ};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, state, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    constexpr size_t smem = tma_smem_bytes<NZ>();
    cudaError_t e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = ensure_smem_limit((const void *)k_pencil_tma<NZ>, (int)smem))) return e;
    if ((e = cudaGetDevice(&dev))) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pencil_tma<NZ>, kThreads, smem))) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid_max = sms * per_sm;
    TmaArgs A = A0;
    A.plane = plane;
    A.tiles_per_traj = plane / PEN;
    A.n_tiles = c.n_traj * A.tiles_per_traj;
    const int grid = A.n_tiles < grid_max ? A.n_tiles : grid_max;
    k_pencil_tma<NZ><<<grid, kThreads, smem, s>>>(map, A);
    g_launches++;
    return cudaGetLastError();
}

} // namespace

bool fp32_pencil_tma_supported(const ClassGeom &c)
{
    return (c.nz == 64 || c.nz == 128 || c.nz == 256) && (c.nx * c.ny) % (2048 / c.nz) == 0 && encode_fn() != nullptr;
}

cudaError_t fp32_pencil_tma(float4 *state, const ClassGeom &c, const float2 *tw_full, float frac, float scale,
                            const float2 *m, const float2 *kin, int *d_err, const int *d_never, cudaStream_t s)
{
    if (c.n_traj <= 0) return cudaSuccess;
    const TmaEnv env;   // read at every launch: a test may change it between contexts of one process
    TmaArgs A{};
    A.tw = tw_full;
    A.kin = kin;
    A.pa.frac = frac;
    A.pa.scale = scale;
    A.pa.has_m = m ? 1 : 0;
    if (m)
        for (int i = 0; i < 4; ++i) A.pa.m[i] = m[i];
    A.err = d_err;
    A.never = d_never;
    A.stall = env.stall;
    A.wait_limit_ns = env.wait_limit_ns;
    switch (c.nz) {
    case 64: return launch_tma<64>(state, c, A, s);
    case 128: return launch_tma<128>(state, c, A, s);
    case 256: return launch_tma<256>(state, c, A, s);
    default: return cudaErrorInvalidValue;
    }
}
