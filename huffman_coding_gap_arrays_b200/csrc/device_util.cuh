// device_util.cuh -- small sm_100a building blocks shared by the kernels:
// streaming loads, relaxed GPU-scope flag traffic, bounded waits and the
// warp-wide decoupled look-back.
#pragma once

#include <cstdint>

#include "hgap_internal.h"

namespace hgap {

constexpr unsigned kFull = 0xffffffffu;
// A wait gives up after this long (ns of %globaltimer) and flags kDevTimeout.
constexpr uint64_t kWaitLimitNs = 500ull * 1000 * 1000;

__device__ __forceinline__ uint4 ld_stream_v4(const void* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until *p != 0 and returns it.  Bounded: once `limit_ns` of
// %globaltimer have passed it flags kDevTimeout and returns `fallback`, so the
// caller finishes its tile and the kernel exits; once a timeout is flagged,
// every other wait gives up at once.  Other errors (a corrupt stream, a
// missing codeword, ...) never stop a tile from publishing, so they do not end
// a wait: a timeout is flagged only when a wait really expired, and in a batch
// the healthy buffers still decode around a corrupt one.
__device__ __forceinline__ uint64_t wait_nonzero(const uint64_t* p, uint32_t* status, uint64_t fallback,
                                                 uint64_t limit_ns) {
    uint64_t v = ld_relaxed_u64(p);
    if (v != 0) return v;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t it = 1;; ++it) {
        v = ld_relaxed_u64(p);
        if (v != 0) return v;
        if ((it & 31) == 0) {
            if (ld_relaxed_u32(status) & kDevTimeout) return fallback;
            if (global_timer_ns() - t0 > limit_ns) {
                atomicOr(status, kDevTimeout);
                return fallback;
            }
            __nanosleep(64);
        }
    }
}

// ------------------------------------------- bulk copies into shared memory --
// One-dimensional bulk copy (the TMA engine, no tensor map) from global to
// this CTA's shared memory, completing on an mbarrier with a byte count.
// Both addresses 16-byte aligned, size a multiple of 16; the copy lands in this
// CTA alone.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Per-thread asynchronous 16-byte copies from global to this CTA's shared
// memory (no registers held): a thread waits for its own copies with
// cp_async_wait_all, and a CTA barrier after that shows them to the others.
// Both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst_smem)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes initialised mbarriers visible to the async proxy (bulk copies)
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders this thread's earlier generic-proxy shared accesses (made visible to
// it by a CTA barrier) before a following bulk copy into the same bytes
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst_smem)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `bar` with the given parity to complete.  Bounded:
// after kWaitLimitNs it flags kDevTimeout and returns false; with `bail`, it
// also gives up as soon as a timeout is already flagged (the kernel's output
// is void then, and it only has to finish).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* status, bool bail) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_timer_ns() - t0 > kWaitLimitNs || (bail && (ld_relaxed_u32(status) & kDevTimeout))) {
            atomicOr(status, kDevTimeout);
            return false;
        }
    }
}

// The wait limit of a launch's look-back waits (the test hook may shorten it).
__device__ __forceinline__ uint64_t wait_limit(const LookbackHook& h) {
    return h.wait_ns ? h.wait_ns : kWaitLimitNs;
}

// The job owning global work item `it`: the largest j with item0s[j] <= it
// (item0s ascends, item0s[count] is the total; empty jobs are skipped).
__device__ __forceinline__ uint32_t find_job(const uint64_t* item0s, uint32_t count, uint64_t it) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (item0s[mid] <= it) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
    return v;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, uint32_t lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, v, d);
        if (lane >= (uint32_t)d) v += t;
    }
    return v;
}

// Single-pass decoupled look-back (the reference's scheme,
// encoder/src/encoder.cu:222-263, decoder/src/decoder.cu:601-638) run by one
// full warp, with a window of 32*K predecessors per round trip: lane
// l holds tiles top-K*l ... top-K*l-K+1 (nearest first, window position
// K*l + j).  The inclusive-prefix frontier advances at most one window per L2
// round trip, so the window must exceed the tiles started per round trip.
// Only the records between the tile and the nearest inclusive prefix matter:
// the window is loaded without blocking, and the warp waits only while an
// unpublished record lies in front of the nearest inclusive prefix (on that
// one record, bounded), then reloads.
// Publishing the aggregate and resolving the prefix are separate steps, so a
// CTA can publish a tile's aggregate, decode its next tile, and resolve the
// first tile afterwards, when its predecessors have long been published.
// `first`: the tile starts its own scan (tile 0, or a batched job's first
// tile); it publishes its inclusive prefix at once and resolves to 0, so no
// look-back ever crosses into another job's tiles.
__device__ __forceinline__ void lookback_publish(uint64_t* rec, uint64_t tile, uint64_t agg, bool first) {
    st_relaxed_u64(rec + tile, (first ? kFlagP : kFlagA) | (agg & kValueMask));
}

// `limit_ns` bounds each wait; `publish` = false keeps the inclusive prefix
// unpublished (the bounded-wait test hook only: LookbackHook).
template <int K>
__device__ __forceinline__ uint64_t lookback_resolve(uint64_t* rec, uint64_t tile, uint64_t agg, bool first,
                                                     uint32_t* status, uint32_t lane, uint64_t limit_ns,
                                                     bool publish = true) {
    if (first) return 0;
    uint64_t excl = 0;
    int64_t top = (int64_t)tile - 1;
    for (;;) {
        uint64_t v[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int64_t i = top - (int64_t)(K * lane + j);
            v[j] = i >= 0 ? ld_relaxed_u64(rec + i) : kFlagP;
        }
        int first_p = K, first_z = K;  // nearest inclusive prefix / unpublished record of this lane
#pragma unroll
        for (int j = K - 1; j >= 0; --j) {
            if (v[j] & kFlagP) first_p = j;
            if (v[j] == 0) first_z = j;
        }
        const uint32_t pmask = __ballot_sync(kFull, first_p < K);
        const uint32_t zmask = __ballot_sync(kFull, first_z < K);
        const int lp = pmask ? __ffs(pmask) - 1 : 32;
        const int lz = zmask ? __ffs(zmask) - 1 : 32;
        const int gp = lp < 32 ? K * lp + __shfl_sync(kFull, first_p, lp) : 32 * K;
        const int gz = lz < 32 ? K * lz + __shfl_sync(kFull, first_z, lz) : 32 * K;
        if (gz < gp) {  // an unpublished record in front of the nearest inclusive prefix
            if ((int)lane == lz) {
                const int64_t i = top - (int64_t)gz;
                wait_nonzero(rec + i, status, kFlagP, limit_ns);
            }
            __syncwarp();
            if (ld_relaxed_u32(status) & kDevTimeout) return excl;  // gave up: the status says so
            continue;  // reload the same window
        }
        uint64_t sum = 0;
#pragma unroll
        for (int j = 0; j < K; ++j)
            if ((int)(K * lane + j) <= gp) sum += v[j] & kValueMask;
        excl += warp_sum_u64(sum);
        if (gp < 32 * K) break;
        top -= 32 * K;
    }
    if (lane == 0 && publish) st_relaxed_u64(rec + tile, kFlagP | ((excl + agg) & kValueMask));
    return excl;
}

}  // namespace hgap
