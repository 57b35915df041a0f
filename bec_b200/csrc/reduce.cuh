// reduce.cuh -- FP64 Neumaier-compensated block and grid reductions.
//
// Replaces the reference's FP32 tree reduction (reduce.cuh:27-154 of
// bec_wigner_3d.cuda), whose last-warp section relies on implicit warp
// synchrony and which copies every scalar to the host. Here each thread keeps
// a compensated (sum, carry) pair, warps combine with shuffles, and results
// stay in device memory.
#pragma once

#include "common.cuh"

template <int K>
struct KVec {
    KSum v[K];
};

__device__ __forceinline__ void ksum_merge(KSum &a, double s, double c)
{
    a.add(s);
    a.c += c;
}

// Reduces K compensated sums across the block; the result is valid in thread 0.
// Requires blockDim.x to be a multiple of 32 and at most 1024.
template <int K>
__device__ KVec<K> block_reduce(KVec<K> x)
{
    __shared__ double ss[K][32], cc[K][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            double s2 = __shfl_down_sync(0xffffffffu, x.v[k].s, off);
            double c2 = __shfl_down_sync(0xffffffffu, x.v[k].c, off);
            ksum_merge(x.v[k], s2, c2);
        }
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) { ss[k][warp] = x.v[k].s; cc[k][warp] = x.v[k].c; }
    }
    __syncthreads();
    KVec<K> r;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (lane < nw) { r.v[k].s = ss[k][lane]; r.v[k].c = cc[k][lane]; }
            for (int off = 16; off > 0; off >>= 1) {
                double s2 = __shfl_down_sync(0xffffffffu, r.v[k].s, off);
                double c2 = __shfl_down_sync(0xffffffffu, r.v[k].c, off);
                ksum_merge(r.v[k], s2, c2);
            }
        }
    }
    return r;
}

// Stage 1: every block reduces a grid-stride range of f(i), i < n, and writes
// (sum, carry) pairs to part[block][K][2]. Stage 2 (one block) folds them.
template <int K, typename F>
__global__ void reduce_stage1(F f, int n, double *part)
{
    KVec<K> acc;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v[K];
        f(i, v);
#pragma unroll
        for (int k = 0; k < K; ++k) acc.v[k].add(v[k]);
    }
    KVec<K> r = block_reduce<K>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            part[(blockIdx.x * K + k) * 2 + 0] = r.v[k].s;
            part[(blockIdx.x * K + k) * 2 + 1] = r.v[k].c;
        }
    }
}

template <int K>
__global__ void reduce_stage2(const double *part, int nparts, double *out)
{
    KVec<K> acc;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) ksum_merge(acc.v[k], part[(b * K + k) * 2], part[(b * K + k) * 2 + 1]);
    }
    KVec<K> r = block_reduce<K>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = r.v[k].value();
    }
}

// Two-stage reduction into out[0..K). tmp must hold 2*K*1024 doubles.
template <int K, typename F>
void reduce_sum(F f, int n, double *out, double *tmp, cudaStream_t s)
{
    int blocks = (n + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    if (blocks < 1) blocks = 1;
    reduce_stage1<K, F><<<blocks, 256, 0, s>>>(f, n, tmp);
    reduce_stage2<K><<<1, 256, 0, s>>>(tmp, blocks, out);
}
