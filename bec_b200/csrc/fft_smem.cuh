// fft_smem.cuh -- in-place radix-2 FFT stages over lines held in shared memory.
//
// A "line" is n = 2^logn elements at base(line) + e * es, with
//   base(line) = (line % n_in) * ls_in + (line / n_in) * ls_out,
// so rows, columns and pencils of a tile are all expressible. Every thread
// of the block takes part; stages are separated by __syncthreads().
//
//  fft_dit: bit-reversed input  -> natural output (Cooley-Tukey, decimation in time)
//  fft_dif: natural input       -> bit-reversed output (Gentleman-Sande)
// Pairing DIT for k->x with DIF for x->k needs no permutation pass: tiles are
// loaded into bit-reversed slots, transformed, processed in natural order,
// transformed back and stored from bit-reversed slots.
//
// tw holds n/2 twiddles W_n^k = exp(-2 pi i k / n); inv conjugates them
// (the unnormalised inverse transform, cuFFT's CUFFT_INVERSE convention).
#pragma once

#include "common.cuh"

struct LineMap {
    int logn;     // log2 of the line length
    int nlines;   // number of lines
    int es;       // element stride
    int ls_in;    // stride between consecutive lines within a group of n_in
    int n_in;     // lines per group
    int ls_out;   // stride between groups
    int line_fast;// 1: consecutive threads take consecutive lines (use when es != 1)
};

__device__ __forceinline__ int line_base(const LineMap &m, int line)
{
    return (line % m.n_in) * m.ls_in + (line / m.n_in) * m.ls_out;
}

template <typename V, typename W>
__device__ void fft_dit(V *buf, const LineMap m, const W *tw, bool inv)
{
    const int logn = m.logn;
    if (logn == 0) return;
    const int hn = 1 << (logn - 1);
    const int total = m.nlines * hn;
    for (int s = 0; s < logn; ++s) {
        const int half = 1 << s;
        const int tws = hn >> s;
        for (int w = threadIdx.x; w < total; w += blockDim.x) {
            int line, j;
            if (m.line_fast) { line = w % m.nlines; j = w / m.nlines; }
            else { j = w & (hn - 1); line = w >> (logn - 1); }
            const int pos = j & (half - 1);
            const int i0 = ((j >> s) << (s + 1)) + pos;
            const int base = line_base(m, line);
            V *p0 = buf + base + i0 * m.es;
            V *p1 = p0 + half * m.es;
            W t = tw[pos * tws];
            if (inv) t.y = -t.y;
            V u = *p0;
            V v = tmul(*p1, t);
            *p0 = vadd(u, v);
            *p1 = vsub(u, v);
        }
        __syncthreads();
    }
}

template <typename V, typename W>
__device__ void fft_dif(V *buf, const LineMap m, const W *tw, bool inv)
{
    const int logn = m.logn;
    if (logn == 0) return;
    const int hn = 1 << (logn - 1);
    const int total = m.nlines * hn;
    for (int s = logn - 1; s >= 0; --s) {
        const int half = 1 << s;
        const int tws = hn >> s;
        for (int w = threadIdx.x; w < total; w += blockDim.x) {
            int line, j;
            if (m.line_fast) { line = w % m.nlines; j = w / m.nlines; }
            else { j = w & (hn - 1); line = w >> (logn - 1); }
            const int pos = j & (half - 1);
            const int i0 = ((j >> s) << (s + 1)) + pos;
            const int base = line_base(m, line);
            V *p0 = buf + base + i0 * m.es;
            V *p1 = p0 + half * m.es;
            W t = tw[pos * tws];
            if (inv) t.y = -t.y;
            V u = *p0;
            V v = *p1;
            *p0 = vadd(u, v);
            *p1 = tmul(vsub(u, v), t);
        }
        __syncthreads();
    }
}

// Copies n/2 twiddles from global memory into shared memory.
template <typename W>
__device__ __forceinline__ void load_twiddles(W *dst, const W *src, int half_n)
{
    for (int i = threadIdx.x; i < half_n; i += blockDim.x) dst[i] = src[i];
}
