// hist.cu -- 256-bin byte histogram for sm_100a.
//
// Replaces cu_histgram + mergeHistogram (encoder/src/encoder.cu:33-116).
// Design: one pass, one launch, no scratch.  Each CTA keeps 32 lane-private
// copies of the 256 counters (h[bin*32 + lane]); lane L only touches bank L,
// so the shared-memory atomics of a warp never conflict, whatever the byte
// distribution (the reference's per-warp histograms serialise on skewed data).
// Input is read as 16-byte streaming loads (virtual 16-byte-aligned chunks;
// the ragged head/tail chunks are counted byte by byte).  At the end each CTA
// folds its 32 copies and adds them to the 256 global bins with one atomic
// per bin.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "launch_cache.h"

namespace hgap {

constexpr int kHistThreads = 512;
constexpr int kHistUnroll = 4;

// Byte b counts at h[b * 32 + lane], byte offset (b << 7) | (lane << 2): one
// shift and one and-or (lane4 = lane << 2) per byte, then the shared atomic.
__device__ __forceinline__ void hist_add(uint32_t* h, uint32_t off) {
    atomicAdd(reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(h) + off), 1u);
}

__device__ __forceinline__ void hist_word(uint32_t* h, uint32_t lane4, uint32_t w) {
    hist_add(h, ((w << 7) & 0x7f80u) | lane4);
    hist_add(h, ((w >> 1) & 0x7f80u) | lane4);
    hist_add(h, ((w >> 9) & 0x7f80u) | lane4);
    hist_add(h, ((w >> 17) & 0x7f80u) | lane4);
}

__device__ __forceinline__ void hist_chunk(uint32_t* h, uint32_t lane4, const uint4 v) {
    hist_word(h, lane4, v.x);
    hist_word(h, lane4, v.y);
    hist_word(h, lane4, v.z);
    hist_word(h, lane4, v.w);
}

__global__ void __launch_bounds__(kHistThreads, 4)
    hist_kernel(const uint8_t* __restrict__ in_al, uint64_t lo, uint64_t hi,
                uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256 * 32];
    for (int i = threadIdx.x; i < 256 * 32; i += kHistThreads) h[i] = 0;
    __syncthreads();
    const uint32_t lane4 = (threadIdx.x & 31) << 2;

    const uint64_t first_full = (lo + 15) >> 4;  // chunks wholly inside [lo, hi)
    const uint64_t end_full = hi >> 4;
    const uint64_t stride = (uint64_t)gridDim.x * kHistThreads;
    uint64_t c = first_full + (uint64_t)blockIdx.x * kHistThreads + threadIdx.x;
    for (; c + (kHistUnroll - 1) * stride < end_full; c += kHistUnroll * stride) {
        uint4 v[kHistUnroll];
#pragma unroll
        for (int u = 0; u < kHistUnroll; ++u) v[u] = ld_stream_v4(in_al + ((c + u * stride) << 4));
#pragma unroll
        for (int u = 0; u < kHistUnroll; ++u) hist_chunk(h, lane4, v[u]);
    }
    for (; c < end_full; c += stride) hist_chunk(h, lane4, ld_stream_v4(in_al + (c << 4)));

    // ragged head chunk (0, when lo > 0) and tail chunk (hi >> 4, when hi & 15)
    if (blockIdx.x == 0 && threadIdx.x < 2) {
        uint64_t q = threadIdx.x == 0 ? 0 : (hi >> 4);
        const bool is_edge = threadIdx.x == 0 ? (lo != 0) : ((hi & 15) != 0 && (q != 0 || lo == 0));
        if (is_edge && (q << 4) < hi) {
            const uint4 v = ld_stream_v4(in_al + (q << 4));
            const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
            for (uint64_t b = q << 4; b < (q << 4) + 16; ++b) {
                if (b < lo || b >= hi) continue;
                const uint32_t byte = (wv[(b & 15) >> 2] >> (8 * (b & 3))) & 0xffu;
                hist_add(h, (byte << 7) | lane4);
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += kHistThreads) {
        uint32_t s = 0;
#pragma unroll 8
        for (int j = 0; j < 32; ++j) s += h[b * 32 + ((j + b) & 31)];
        if (s) atomicAdd(hist + b, s);
    }
}

// Histogram pass of the encoder: the same lane-replicated counters, over the
// regions of one or many jobs.  After each region the CTA folds its 32 copies
// and stores the difference to the previous fold as that region's histogram,
// so the encoder can compute every region's bit count without reading its
// bytes again.  A job's histogram is the sum of its regions'.  One job (equal
// regions): each CTA takes a contiguous run of regions and adds the job's sum
// with one atomic per bin at the end.  Many jobs (a.counter set): regions of
// very different sizes (a 4 KiB buffer is one region, a 4 MiB one sixteen of
// 256 KiB), so equal-count runs would leave some CTAs several times the bytes
// of others; each CTA claims its next region from the counter while it
// counts the current one, and adds every region's histogram to its job's.
__global__ void __launch_bounds__(kHistThreads, 4) hist_st_kernel(const __grid_constant__ HistStArgs a) {
    __shared__ uint32_t h[256 * 32];
    for (int i = threadIdx.x; i < 256 * 32; i += kHistThreads) h[i] = 0;
    __syncthreads();
    const uint32_t tid = threadIdx.x;
    const uint32_t lane4 = (tid & 31) << 2;
    uint32_t prev = 0, acc = 0;  // running fold of bin `tid` (tid < 256); the job's sum so far
    const uint64_t nitems = a.nitems_dev ? *a.nitems_dev : a.nitems;
    const bool claims = a.counter != nullptr;
    __shared__ uint32_t s_first, s_next;
    uint64_t it0 = 0, it1 = 0;
    if (claims) {
        if (tid == 0) s_first = atomicAdd(a.counter, 1u);
        __syncthreads();
        it0 = s_first;
        it1 = nitems;
    } else {
        const uint64_t per = (nitems + gridDim.x - 1) / gridDim.x;
        it0 = (uint64_t)blockIdx.x * per;
        it1 = it0 + per < nitems ? it0 + per : nitems;
    }
    uint32_t job = 0;
    for (uint64_t it = it0; it < it1;) {
        if (claims && tid == 0) s_next = atomicAdd(a.counter, 1u);  // the next region, claimed early
        if (a.jobs && (claims || it == it0 || it >= a.item0s[job + 1])) job = find_job(a.item0s, a.count, it);
        const EncJob& J = a.jobs ? a.jobs[job] : a.single;
        const uint64_t v0 = (it - J.item0) * (uint64_t)J.st_bytes;
        const uint64_t v1 = (v0 + J.st_bytes < J.hi) ? v0 + J.st_bytes : J.hi;
        const uint64_t lo_v = v0 > J.lo ? v0 : J.lo;
        const uint8_t* in = J.in_aligned;
        const uint64_t c0 = (lo_v + 15) >> 4, c1 = v1 >> 4;  // chunks wholly inside
        uint64_t c = c0 + tid;
        for (; c + (kHistUnroll - 1) * kHistThreads < c1; c += kHistUnroll * kHistThreads) {
            uint4 v[kHistUnroll];
#pragma unroll
            for (int u = 0; u < kHistUnroll; ++u) v[u] = ld_stream_v4(in + ((c + u * kHistThreads) << 4));
#pragma unroll
            for (int u = 0; u < kHistUnroll; ++u) hist_chunk(h, lane4, v[u]);
        }
        for (; c < c1; c += kHistThreads) hist_chunk(h, lane4, ld_stream_v4(in + (c << 4)));
        // ragged head chunk (a job's first region only) and tail chunk (its last only)
        uint64_t q = ~0ull;
        if (tid == 0 && (lo_v & 15)) q = lo_v >> 4;
        if (tid == 1 && (v1 & 15) && (v1 >> 4) >= c0) q = v1 >> 4;
        if (q != ~0ull) {
            const uint4 v = ld_stream_v4(in + (q << 4));
            const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
            for (uint64_t b = q << 4; b < (q << 4) + 16; ++b) {
                if (b < lo_v || b >= v1) continue;
                hist_add(h, (((wv[(b & 15) >> 2] >> (8 * (b & 3))) & 0xffu) << 7) | lane4);
            }
        }
        __syncthreads();
        const uint64_t next = claims ? (uint64_t)s_next : it + 1;  // read before the second barrier
        const bool leave = claims || it + 1 == it1 || it + 1 == J.item0 + J.nst;
        if (tid < 256) {
            uint32_t s = 0;
#pragma unroll 8
            for (int j = 0; j < 32; ++j) s += h[tid * 32 + ((j + tid) & 31)];
            const uint32_t d = s - prev;
            a.st_hist[it * 256 + tid] = d;
            prev = s;
            acc += d;
            if (leave) {
                if (acc) atomicAdd(a.hist + 256 * (uint64_t)job + tid, acc);
                acc = 0;
            }
        }
        __syncthreads();
        it = next;
    }
    if (a.tag && blockIdx.x == 0 && tid == 0) {
        a.tag[0] = a.single.hi - a.single.lo;
        a.tag[1] = reinterpret_cast<uint64_t>(a.single.in_aligned) + a.single.lo;
    }
}

// `hist` must be zeroed by the caller ([count][256]).
int launch_hist_st(const HistStArgs& a, int ctas_per_sm, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    static LaunchCache cache;
    const LaunchFacts f = cache.get(reinterpret_cast<const void*>(hist_st_kernel), kHistThreads, 0);
    if (f.err != cudaSuccess) return f.err;
    const int sms = f.sms, per_sm = f.per_sm;
    const int k = (ctas_per_sm > 0 && ctas_per_sm < per_sm) ? ctas_per_sm : per_sm;
    const uint64_t cap = (uint64_t)sms * k;
    const unsigned grid = (unsigned)(a.nitems_dev ? cap : (a.nitems < cap ? (a.nitems ? a.nitems : 1) : cap));
    hist_st_kernel<<<grid, kHistThreads, 0, st>>>(a);
    return cudaGetLastError();
}

int launch_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_hist, 0, 256 * sizeof(uint32_t), st);
    if (e != cudaSuccess || n == 0) return e;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(d_in);
    const uint64_t lo = addr & 15;
    const uint8_t* al = reinterpret_cast<const uint8_t*>(addr - lo);
    static LaunchCache cache;
    const LaunchFacts f = cache.get(reinterpret_cast<const void*>(hist_kernel), kHistThreads, 0);
    if (f.err != cudaSuccess) return f.err;
    const int sms = f.sms, per_sm = f.per_sm;
    const uint64_t chunks = (lo + n + 15) >> 4;
    uint64_t want = (chunks + (uint64_t)kHistThreads * kHistUnroll - 1) / ((uint64_t)kHistThreads * kHistUnroll);
    const uint64_t cap = (uint64_t)sms * per_sm;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
    hist_kernel<<<grid, kHistThreads, 0, st>>>(al, lo, lo + n, d_hist);
    return cudaGetLastError();
}

}  // namespace hgap
