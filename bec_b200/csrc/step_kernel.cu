// step_kernel.cu -- one split step of every trajectory of the register-path grid classes in one
// persistent launch.
//
// The reference launches eight kernels per step for one ensemble (propagate,
// programs/bec_wigner_3d.cuda/wigner.cu:178-199: kick, 2 x 3D FFT, nonlinear step, 2 x 3D IFFT,
// scale, kick, each FFT itself 3 cuFFT passes and 4 transposes, batchfft.cu:158-180). Here a step is
// two passes per trajectory (step_bodies.cuh) and both passes of every class are items of one work
// list walked by a persistent grid:
//
//   pencil item  the pencil pass of a group of tiles of one trajectory (IFFT_z, kinetic phase, pulse,
//                FFT_z);
//   plane item   the plane pass of a group of planes of one trajectory (FFT_xy, nonlinear + losses +
//                loss noise, IFFT_xy); it waits until every pencil item of its trajectory is done
//                (a per-trajectory counter, released with a gpu-scope fence, acquired by one thread
//                of the waiting CTA).
//
// The list is longest-first (the classes by cells per trajectory, the largest first) and
// interleaved: a trajectory's plane items follow its pencil items at a distance of `lead` items.
// CTAs take items in list order with one atomic ticket each, so a waiting plane item only waits for
// items that running CTAs took before it, and no wait can depend on a CTA that has not started. (A CTA
// takes its next ticket once its current item is past its wait; the current item then completes, so a
// ticket held that way is always started.) The
// interleave lets memory-bound pencil items run beside issue-bound plane items, and a trajectory's
// plane items read what its pencil items wrote while it is still in L2. The last CTA to finish resets
// the counters and advances the Philox step index, so every launch is identical and a captured CUDA
// graph replays it.
//
// A two-phase plan runs the same list as two launches (all pencil items, then all plane items) with
// no waits. The plan (interleave distance or two phases) is chosen per context by timing the
// candidates on its first steady steps (plan_autotune); every plan computes the same bits.
//
// Every wait is bounded: after 2 s of polling (BEC_STEP_WAIT_LIMIT_MS) the item records an error flag
// and proceeds, the host reads the flag after the step (BEC_ERR_CUDA), and no launch can hang the device.
// BEC_STEP_INJECT_STALL=1 makes every plane item wait for one pencil item more than exists, so that a
// test can run the timeout path and check the reported status.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "step_bodies.cuh"

namespace {

using stepk::PencilArgs;
using stepk::VBlock;

constexpr int kThreads = 256;
constexpr int kPlane32PerItem = 4;                              // 64-thread virtual blocks
constexpr size_t kSmemPlane32 = sizeof(float4) * 1536;          // tile + exchange slots of one plane
constexpr size_t kSmemBytes = kSmemPlane32 * kPlane32PerItem;   // 96 KiB: the largest item's need

enum { ITEM_PENCIL = 0, ITEM_PLANE = 1 };

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int load_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <int NZ>
__device__ __forceinline__ void run_pencil(const StepClassDev &c, const GroupParamsF *gp, int traj, int sub,
                                           const PencilArgs &pa, float4 *smem)
{
    constexpr int VB = kThreads / NZ;       // tiles of 16 pencils per item
    const int v = threadIdx.x / NZ;
    PencilArgs p = pa;
    p.scale = 1.0f / (float)c.cells;        // exact: cells is a power of two
    const VBlock vb{(int)threadIdx.x % NZ, traj * c.tiles + sub * VB + v, VB == 1 ? 0 : 1 + v, NZ};
    float4 *dyn = smem + v * (stepk::pencil_smem_bytes<NZ>() / sizeof(float4));
    const float2 *kin = pa.frac == 1.0f ? c.kin[1] : pa.frac == 0.5f ? c.kin[0] : nullptr;
    stepk::pencil_body<NZ, false>(vb, c.state, c.nx, c.lx, c.ny, c.cells, c.tiles, gp, c.tgroup, c.tw, p, nullptr,
                                  1.0f, kin, dyn);
}

template <int N>
__device__ __forceinline__ void run_plane(const StepClassDev &c, const GroupParamsF *gp, int traj, int sub,
                                          uint32_t step, float4 *smem)
{
    constexpr int W = 32 / N;
    const int v = threadIdx.x / 128;        // two 128-thread virtual blocks of 4 warps
    const int planes_per_vb = 4 * W;
    const int bid = (traj * c.nz) / planes_per_vb + sub * 2 + v;
    const VBlock vb{(int)threadIdx.x % 128, bid, 0, 128};   // warp-synchronous: no block barrier used
    stepk::plane_body<N>(vb, c.state, c.nz, c.cells, gp, c.tgroup, c.tlocal, step, smem + v * 4 * W * N * N);
}

__device__ __forceinline__ void run_plane32(const StepClassDev &c, const GroupParamsF *gp, int traj, int sub,
                                            uint32_t step, float4 *smem)
{
    const int v = threadIdx.x / 64;
    const VBlock vb{(int)threadIdx.x % 64, traj * c.nz + sub * kPlane32PerItem + v, 1 + v, 64};
    float4 *tile = smem + v * 1536;
    stepk::plane32_body(vb, c.state, c.nz, c.cells, gp, c.tgroup, c.tlocal, step, tile, tile + 1024);
}

__global__ void __launch_bounds__(kThreads, 2) k_step(StepLaunch L, PencilArgs pa)
{
    extern __shared__ float4 smem[];
    __shared__ int4 s_item;
    __shared__ int s_last;
    const uint32_t step = *L.d_step;
    // thread 0 holds the ticket of the CTA's next item, taken while the current one runs, so the
    // atomic's round trip stays off the item-to-item path
    int next = 0;
    if (threadIdx.x == 0) next = atomicAdd(L.queue, 1);
    for (;;) {
        if (threadIdx.x == 0) {
            const int k = next;
            int4 it = make_int4(-1, 0, 0, 0);
            if (k < L.n_items) {
                it = L.items[k];
                if (L.wait && (it.x & 0xF) == ITEM_PLANE) {
                    const int need = L.cls[it.x >> 4].pencil_items + L.stall;
                    const int *cnt = L.done + it.w;
                    if (load_acquire(cnt) < need) {
                        const unsigned long long t0 = global_ns();
                        while (load_acquire(cnt) < need) {
                            __nanosleep(64);
                            if (global_ns() - t0 > L.wait_limit_ns) {
                                atomicExch(L.err, 1);
                                break;
                            }
                        }
                    }
                }
            }
            s_item = it;
            if (it.x >= 0) next = atomicAdd(L.queue, 1);
        }
        __syncthreads();
        const int4 it = s_item;
        if (it.x < 0) break;
        const StepClassDev &c = L.cls[it.x >> 4];
        if ((it.x & 0xF) == ITEM_PENCIL) {
            switch (c.nz) {
            case 64: run_pencil<64>(c, L.gp, it.y, it.z, pa, smem); break;
            case 128: run_pencil<128>(c, L.gp, it.y, it.z, pa, smem); break;
            default: run_pencil<256>(c, L.gp, it.y, it.z, pa, smem); break;
            }
            __syncthreads();                        // every thread's stores are issued
            if (threadIdx.x == 0) {
                __threadfence();                    // release them at gpu scope, then count the item
                atomicAdd(L.done + it.w, 1);
            }
        } else {
            switch (c.nx) {
            case 8: run_plane<8>(c, L.gp, it.y, it.z, step, smem); break;
            case 16: run_plane<16>(c, L.gp, it.y, it.z, step, smem); break;
            default: run_plane32(c, L.gp, it.y, it.z, step, smem); break;
            }
            __syncthreads();                        // shared memory free for the next item
        }
    }
    // the last CTA out resets the list for the next launch and advances the Philox step
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(L.finished, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        for (int i = threadIdx.x; i < L.n_counters; i += blockDim.x) L.done[i] = 0;
        if (threadIdx.x == 0) {
            *L.queue = 0;
            *L.finished = 0;
            if (L.inc_step) *L.d_step = step + 1u;
        }
    }
}

// ---------------------------------------------------------------- plans
struct PlanKey {
    std::vector<int> shape;     // (nx, ny, nz, n_traj) per fused class, then the SM count
    bool operator<(const PlanKey &o) const { return shape < o.shape; }
};

std::mutex g_plan_mutex;
std::map<PlanKey, int> g_plan_cache;   // chosen candidate per class mix and SM count

PlanKey plan_key(const std::vector<ClassGeom> &geoms)
{
    PlanKey k;
    for (const ClassGeom &g : geoms) k.shape.insert(k.shape.end(), {g.nx, g.ny, g.nz, g.n_traj});
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k.shape.push_back(sms);
    return k;
}

int plane_items_per_traj(const ClassGeom &g)
{
    if (g.nx == 32) return g.nz / kPlane32PerItem;
    return g.nz / (2 * 4 * (32 / g.nx));
}

int pencil_items_per_traj(const ClassGeom &g) { return (g.nx * g.ny / 16) / (kThreads / g.nz); }

} // namespace

// ---------------------------------------------------------------- host interface
bool step_class_supported(const ClassGeom &c)
{
    if (c.nx != c.ny || (c.nx != 8 && c.nx != 16 && c.nx != 32)) return false;
    if (c.nz != 64 && c.nz != 128 && c.nz != 256) return false;
    const int planes_per_item = c.nx == 32 ? kPlane32PerItem : 2 * 4 * (32 / c.nx);
    if (c.nz % planes_per_item) return false;
    const int tiles = c.nx * c.ny / 16;
    return tiles % (kThreads / c.nz) == 0;
}

const char *step_plan_name(int candidate)
{
    static const char *names[] = {"two-phase", "interleave 0.5 wave", "interleave 1 wave", "interleave 2 waves",
                                  "interleave 4 waves"};
    return candidate >= 0 && candidate < kStepCandidates ? names[candidate] : "per-pass launches";
}

cudaError_t step_plan_build(StepPlan &P, const std::vector<ClassGeom> &geoms, const std::vector<StepClassDev> &cls,
                            const std::vector<int> &traj_offset, int candidate, cudaStream_t s)
{
    P.candidate = candidate;
    if (const char *v = std::getenv("BEC_STEP_WAIT_LIMIT_MS")) P.wait_limit_ns = 1000000ull * std::strtoull(v, nullptr, 10);
    if (const char *v = std::getenv("BEC_STEP_INJECT_STALL")) P.stall = std::atoi(v) ? 1 : 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev))) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
    if ((e = cudaFuncSetAttribute(k_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes))) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step, kThreads, kSmemBytes))) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    P.grid = sms * per_sm;
    // classes longest-first
    std::vector<int> order(geoms.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return geoms[a].cells > geoms[b].cells; });
    std::vector<int4> pen, pla, mixed;
    // lead distance of the interleaved candidates, in waves of the grid
    static const double waves[kStepCandidates] = {0.0, 0.5, 1.0, 2.0, 4.0};
    const long long lead = (long long)(waves[candidate] * P.grid);
    struct Pending { int cls, traj, gtraj; long long ready_at; };
    std::vector<Pending> fifo;
    size_t head = 0;
    auto emit_planes = [&](const Pending &p) {
        const int n = plane_items_per_traj(geoms[p.cls]);
        for (int k = 0; k < n; ++k) {
            const int4 it = make_int4(ITEM_PLANE | (p.cls << 4), p.traj, k, p.gtraj);
            pla.push_back(it);
            mixed.push_back(it);
        }
    };
    for (int ci : order) {
        const ClassGeom &g = geoms[ci];
        const int np = pencil_items_per_traj(g);
        for (int t = 0; t < g.n_traj; ++t) {
            const int gt = traj_offset[ci] + t;
            for (int k = 0; k < np; ++k) {
                const int4 it = make_int4(ITEM_PENCIL | (ci << 4), t, k, gt);
                pen.push_back(it);
                mixed.push_back(it);
            }
            fifo.push_back(Pending{ci, t, gt, (long long)mixed.size() + lead});
            while (head < fifo.size() && fifo[head].ready_at <= (long long)mixed.size()) emit_planes(fifo[head++]);
        }
    }
    while (head < fifo.size()) emit_planes(fifo[head++]);
    P.two_phase = candidate == 0;
    P.n_pencil = (int)pen.size();
    P.n_plane = (int)pla.size();
    P.n_items = (int)mixed.size();
    int n_counters = 0;
    for (size_t i = 0; i < geoms.size(); ++i) n_counters = std::max(n_counters, traj_offset[i] + geoms[i].n_traj);
    P.n_counters = n_counters;
    std::vector<int4> all;
    if (P.two_phase) {
        all = pen;
        all.insert(all.end(), pla.begin(), pla.end());
    } else {
        all = mixed;
    }
    auto alloc = [&](void **p, size_t b) { return cudaMalloc(p, b > 0 ? b : 16); };
    if (!P.d_items && (e = alloc((void **)&P.d_items, sizeof(int4) * all.size()))) return e;
    if (!P.d_cls && (e = alloc((void **)&P.d_cls, sizeof(StepClassDev) * cls.size()))) return e;
    if (!P.d_counters && (e = alloc((void **)&P.d_counters, sizeof(int) * (4 + (size_t)n_counters)))) return e;
    if ((e = cudaMemcpyAsync(P.d_items, all.data(), sizeof(int4) * all.size(), cudaMemcpyHostToDevice, s))) return e;
    std::vector<StepClassDev> c2 = cls;
    for (size_t i = 0; i < c2.size(); ++i) c2[i].pencil_items = pencil_items_per_traj(geoms[i]);
    if ((e = cudaMemcpyAsync(P.d_cls, c2.data(), sizeof(StepClassDev) * c2.size(), cudaMemcpyHostToDevice, s))) return e;
    if ((e = cudaMemsetAsync(P.d_counters, 0, sizeof(int) * (4 + (size_t)n_counters), s))) return e;
    P.ready = true;
    return cudaSuccess;
}

void step_plan_free(StepPlan &P)
{
    cudaFree(P.d_items);
    cudaFree(P.d_cls);
    cudaFree(P.d_counters);
    P = StepPlan{};
}

void step_launch(const StepPlan &P, const GroupParamsF *gp, uint32_t *d_step, float frac, const float2 *m,
                 cudaStream_t s)
{
    PencilArgs pa{};
    pa.frac = frac;
    pa.scale = 0.0f;      // per class: 1 / cells (StepClassDev)
    pa.has_m = m ? 1 : 0;
    if (m)
        for (int i = 0; i < 4; ++i) pa.m[i] = m[i];
    StepLaunch L{};
    L.cls = P.d_cls;
    L.gp = gp;
    L.queue = P.d_counters;
    L.finished = P.d_counters + 1;
    L.err = P.d_counters + 2;
    L.done = P.d_counters + 4;
    L.n_counters = P.n_counters;
    L.d_step = d_step;
    L.stall = P.stall;
    L.wait_limit_ns = P.wait_limit_ns;
    if (P.two_phase) {
        L.items = P.d_items;
        L.n_items = P.n_pencil;
        L.wait = 0;
        L.inc_step = 0;
        k_step<<<P.grid, kThreads, kSmemBytes, s>>>(L, pa);
        g_launches++;
        L.items = P.d_items + P.n_pencil;
        L.n_items = P.n_plane;
        L.inc_step = 1;
        k_step<<<P.grid, kThreads, kSmemBytes, s>>>(L, pa);
        g_launches++;
    } else {
        L.items = P.d_items;
        L.n_items = P.n_items;
        L.wait = 1;
        L.inc_step = 1;
        k_step<<<P.grid, kThreads, kSmemBytes, s>>>(L, pa);
        g_launches++;
    }
}

cudaError_t step_read_error(const StepPlan &P, int *err, cudaStream_t s)
{
    *err = 0;
    if (!P.ready) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(err, P.d_counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    if (*err) e = cudaMemsetAsync(P.d_counters + 2, 0, sizeof(int), s);   // reported once
    return e;
}

bool step_plan_cached(const std::vector<ClassGeom> &geoms, int *candidate)
{
    PlanKey k = plan_key(geoms);
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    auto it = g_plan_cache.find(k);
    if (it == g_plan_cache.end()) return false;
    *candidate = it->second;
    return true;
}

void step_plan_remember(const std::vector<ClassGeom> &geoms, int candidate)
{
    PlanKey k = plan_key(geoms);
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    g_plan_cache[k] = candidate;
}
