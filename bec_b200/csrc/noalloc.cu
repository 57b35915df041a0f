// noalloc.cu -- moments of device-resident states without any device allocation.
//
// The library's other entry points allocate their device memory inside the
// context (bec_create, bec_ground_state). Some callers cannot allow that: a
// host framework that owns all device memory through its own pool and forbids
// third-party cudaMalloc/cudaFree (both synchronise the whole device and can
// fail in the middle of a long run), or a real-time loop that must never block
// on an allocation. For them bec_moments_device_noalloc computes the FP64
// moments of states that already sit in the caller's device memory, writing
// the result to caller-provided device memory, with the reduction's partial
// sums in a fixed array that is part of the library image.
//
// The scratch array below is a file-scope __device__ symbol: every GPU that
// loads this library holds its 64 KiB until the process exits. In host code
// its name is only a host-side stand-in, not a device address, so every call
// looks up its device address in the current context with cudaGetSymbolAddress
// (a host-side lookup that allocates nothing) and passes it to the kernels. A
// fresh lookup per call stays right after a device reset, which may load the
// module at another address, and under a non-primary context.
#include "engine.h"
#include "reduce.cuh"

namespace {

constexpr int kNoallocMaxBlocks = 1024;                 // partial sums kept per call
constexpr int kNoallocSums = 4;                         // |a|^2, |b|^2, Re and Im of conj(a) b

// Partial (sum, carry) pairs of the first reduction stage: 1024 blocks x 4 sums x 2 doubles = 64 KiB.
static __device__ __align__(256) double g_noalloc_partials[kNoallocMaxBlocks * kNoallocSums * 2];

// psi: [traj][a|b][cell] interleaved complex doubles (x-space)
struct F_moments {
    const double2 *psi;
    int cells;
    __device__ void operator()(int i, double *v) const
    {
        const int t = i / cells, c = i - t * cells;
        const double2 a = psi[(size_t)(2 * t) * cells + c];
        const double2 b = psi[(size_t)(2 * t + 1) * cells + c];
        v[0] = a.x * a.x + a.y * a.y;
        v[1] = b.x * b.x + b.y * b.y;
        v[2] = a.x * b.x + a.y * b.y;
        v[3] = a.x * b.y - a.y * b.x;
    }
};

// Second stage of the two-stage reduction, scaling the folded sums by dV.
__global__ void k_noalloc_finish(const double *part, int nparts, double dV, double *out)
{
    KVec<kNoallocSums> acc;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < kNoallocSums; ++k)
            ksum_merge(acc.v[k], part[(b * kNoallocSums + k) * 2], part[(b * kNoallocSums + k) * 2 + 1]);
    }
    KVec<kNoallocSums> r = block_reduce<kNoallocSums>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < kNoallocSums; ++k) out[k] = r.v[k].value() * dV;
    }
}

// Device address of the scratch array in the current context.
cudaError_t partials_on_current_device(double **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return e;
    *out = static_cast<double *>(p);
    return cudaSuccess;
}

} // namespace

extern "C" bec_status bec_moments_device_noalloc(const double *d_psi, int32_t cells, int32_t ne, double dV,
                                                 double *d_out, void *stream)
{
    if (!d_psi || !d_out || cells < 1 || ne < 1 || !(dV > 0.0)) return BEC_ERR_INVALID_ARG;
    // the flat cell index of the reduction is a 32-bit int
    if ((long long)cells * ne > (long long)BEC_NOALLOC_MAX_ELEMENTS) return BEC_ERR_INVALID_ARG;
    double *part = nullptr;
    if (partials_on_current_device(&part) != cudaSuccess) {
        cudaGetLastError();
        return BEC_ERR_CUDA;
    }
    const int n = cells * ne;
    int blocks = (n + 255) / 256;
    if (blocks > kNoallocMaxBlocks) blocks = kNoallocMaxBlocks;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    reduce_stage1<kNoallocSums, F_moments><<<blocks, 256, 0, s>>>(
        F_moments{reinterpret_cast<const double2 *>(d_psi), cells}, n, part);
    k_noalloc_finish<<<1, 256, 0, s>>>(part, blocks, dV, d_out);
    if (cudaGetLastError() != cudaSuccess) return BEC_ERR_CUDA;
    return BEC_OK;
}
