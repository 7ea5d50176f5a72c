// decode.cu -- segment-parallel Huffman decoder driven by the gap array, sm_100a.
//
// Replaces gpu_dec_l1_l2 (decoder/src/decoder.cu:454-730).  Same unit of
// parallelism -- a 128-bit segment that starts at its gap offset -- but each
// segment is decoded ONCE (the reference decodes it twice: a counting pass,
// then a writing pass, decoder.cu:529-569,672-725):
//   1. a persistent CTA of 256 threads takes the next tile of 512 segments
//      (256 for books with 1-2 bit codes); every thread takes its segments'
//      words straight from global memory into registers a tile ahead (one
//      16-byte load per segment, the next segment's first word from the
//      neighbouring lane) and decodes them one after the other (interleaving
//      two chains measured slower: the loop is issue-bound) through a
//      two-level table (level 1 in shared memory, the rarely used level 2 read
//      from global memory), one 32-bit phase per word, so the loop tests only
//      the phase end; each segment's symbols are parked in its own shared row
//      sized for the book's shortest code (a segment holds at most
//      ceil(128 / shortest length) symbols);
//   2. block scan of the symbol counts (both halves of the tile packed in one
//      warp scan) + one bounded decoupled look-back
//      with a 64-tile window gives the tile's output offset;
//   3. the rows are compacted (whole words where the destination is aligned)
//      into a shared image of the tile's output and written one tile later,
//      once its offset is known, with 16-byte coalesced stores (byte stores
//      only on the two ragged edges), clipped at exactly n bytes (the
//      reference writes past n, decoder.cu:529).
// Checks: every segment must end exactly where the next gap entry says the
// next segment starts, every codeword must exist, and the stream must yield at
// least n symbols; failures set kDevCorrupt / kDevSize, never trap.
#include <cuda_runtime.h>

#include "dec_entry.cuh"
#include "device_util.cuh"
#include "launch_cache.h"

namespace hgap {

constexpr int kDecThreads = 256;
// Segments per tile: dec_tile_segs(R) by default, 256 or 512 by the launch shape
// (dec_tile_segs_for, hgap_internal.h).
// Look-back window = 32 * kDecLookK tiles per round trip.  Small is best:
// the resolve runs between two barriers, and a narrow window costs fewer
// loads per lane (measured 256 / 128 / 64 / 32 records: 0.731 / 0.679 /
// 0.674 / 0.683 ms for 256 MiB of the mixed stream).
constexpr int kDecLookK = 2;

// R: stage rows of 4 symbols per segment (at most 4R symbols per segment);
// SEGS: segments per tile, 256 (one per thread) or 512 (two per thread).
template <int R, int SEGS>
struct DecCfg {
    static constexpr int kMaxSym = 4 * R;
    static constexpr int kSegs = SEGS;
    static constexpr int kPer = kSegs / kDecThreads;   // segments per thread
    static constexpr int kWarps = kDecThreads / 32;
    static constexpr int kT1 = 1 << kDecPrefix;        // u32 level-1 entries
    static constexpr int kGapStage = kSegs / 8 + 4;     // gap words of the tile (+1 before)
    // stage row of one segment: its symbols (a multi entry's tail store may put two
    // bytes past the count: 4 spare bytes there), an odd number of words so that
    // the 32 rows a warp writes start in 32 different banks
    static constexpr int kRowWords = ((kMaxSym + (dec_multi(R, true) ? 4 : 0) + 3) / 4) | 1;
    static constexpr int kRow = 4 * kRowWords;
    static constexpr int kStageBytes = kSegs * kRow + 16;
    static constexpr int kCompactBytes = kSegs * kMaxSym + 64;
    // the level-2 table stays in global memory (or the kernel parameter): codes longer
    // than the 11-bit prefix are rare, and its shared memory buys CTAs per SM; so do
    // the multi entries' first-code lengths (read only where a multi entry would run
    // past the segment: 2 KiB less takes the 32-row decoder from 2 to 3 CTAs per SM)
    static constexpr size_t kSmem = (size_t)(kT1 + kGapStage) * 4 + kStageBytes + kCompactBytes;
    // CTAs per SM the shared memory allows (227 KiB usable, ~1.5 KiB static and
    // reserved per CTA), at most 5 for 256-segment tiles (48 registers a thread, no
    // spills) and 4 for 512-segment ones (64 registers: two segments' words in flight)
    static constexpr int kBySmem = (int)((227u * 1024u) / (kSmem + 1536u));
    static constexpr int kCap = SEGS == 256 ? 5 : 4;
    static constexpr int kMinBlocks = kBySmem >= kCap ? kCap : (kBySmem < 1 ? 1 : kBySmem);
    static_assert(kT1 % 4 == 0 && kGapStage % 4 == 0 && kStageBytes % 16 == 0, "16-byte aligned areas");
};

// One codeword from the 32-bit window x at the current position: level-1
// lookup, level 2 for the rare longer codes.  Returns the widened entry.
__device__ __forceinline__ uint32_t lookup(const uint32_t* t1, const uint16_t* __restrict__ t2, uint32_t x) {
    uint32_t e = t1[x >> (32 - kDecPrefix)];
    if (e & 0x80000000u) {
        const uint32_t wd = (e >> 16) & 7u;
        e = widen_entry(t2[(e & 0xffffu) + ((x << kDecPrefix) >> (32 - wd))]);
    }
    return e;
}

// Length of the first code of a multi entry's prefix: from the widened table's
// byte array in global memory (batched path) or derived from the u16 level-1
// table in the kernel parameter (single path).
struct FirstLen {
    const uint8_t* g;
    const uint16_t* t1src;
    __device__ __forceinline__ uint32_t operator()(uint32_t x) const {
        const uint32_t i = x >> (32 - kDecPrefix);
        return g ? (uint32_t)__ldg(g + i) : (uint32_t)first_len(t1src, i);
    }
};

// The words of one segment in registers: its own four and the next segment's
// first (a code that starts in the segment may end up to 15 bits into it).
struct SegWords {
    uint32_t w0, w1, w2, w3, w4;
};

// Decodes the codes that start in one 128-bit segment (not the stream's last
// one), from bit `pos` (its gap offset), as four phases of 32 bits: phase k
// decodes the codes starting in word k, from the window of words k and k+1,
// so the loop tests only `pos < 32` -- no word refill, no end test.  Codes of
// a pair / multi entry all start inside the segment in phases 0-2 (they fit
// the 11-bit window and phase 2 ends 32 bits before the segment does); in
// phase 3 that holds while pos <= 21, and the last bits take only the codes
// that start before bit 32 of the phase.  Returns the end bit of the last
// code relative to phase 3 (32 + the next gap entry for a valid stream; larger
// after an invalid code) and advances `out` past the symbols.
template <bool COMPLETE, bool PAIRS, bool MULTI>
__device__ __forceinline__ uint32_t decode_segment(const uint32_t* t1, const uint16_t* __restrict__ t2,
                                                   const FirstLen& fl, const SegWords& w, uint32_t pos,
                                                   uint8_t*& out) {
    constexpr uint32_t kBad = 1u << 16;  // position after an invalid code: every loop ends
    auto run_fast = [&](uint32_t cw, uint32_t nw, uint32_t stop) {
        while (pos < stop) {
            const uint32_t e = lookup(t1, t2, __funnelshift_l(nw, cw, pos));
            if (!COMPLETE && (e & 0x40000000u)) {
                pos = kBad;
                break;
            }
            if (MULTI) {
                out[0] = (uint8_t)e;
                out[1] = (uint8_t)(e >> 8);
                out[2] = (uint8_t)(e >> 16);
                out += 1 + ((e >> 29) & 3u);
                pos += (e >> 24) & 31u;
            } else if (PAIRS) {
                out[0] = (uint8_t)e;
                out[1] = (uint8_t)(e >> 8);  // a single entry's second byte: overwritten or past the count
                out += 1 + ((e >> 16) & 1u);
                pos += e >> 24;
            } else {
                *out++ = (uint8_t)e;
                pos += e >> 24;
            }
        }
    };
    run_fast(w.w0, w.w1, 32);
    pos -= 32;
    run_fast(w.w1, w.w2, 32);
    pos -= 32;
    run_fast(w.w2, w.w3, 32);
    pos -= 32;
    if (!PAIRS) {
        run_fast(w.w3, w.w4, 32);
        return pos;
    }
    run_fast(w.w3, w.w4, 32 - kDecPrefix + 1);
    while (pos < 32) {  // the last bits: only the codes that start before bit 32
        const uint32_t x = __funnelshift_l(w.w4, w.w3, pos);
        const uint32_t e = lookup(t1, t2, x);
        if (!COMPLETE && (e & 0x40000000u)) {
            pos = kBad;
            break;
        }
        if (MULTI) {
            const uint32_t tot = (e >> 24) & 31u, more = (e >> 29) & 3u;
            out[0] = (uint8_t)e;
            out[1] = (uint8_t)(e >> 8);
            out[2] = (uint8_t)(e >> 16);
            if (pos + tot <= 32) {  // every code of the entry ends, so starts, inside
                out += 1 + more;
                pos += tot;
            } else {
                out += 1;
                pos += more ? fl(x) : tot;
            }
        } else {
            const uint32_t tot = e >> 24;
            const bool pair = (e & 0x10000u) != 0;
            const uint32_t l1 = pair ? ((e >> 17) & 15u) : tot;
            const bool two = pair && pos + l1 < 32;
            out[0] = (uint8_t)e;
            if (two) out[1] = (uint8_t)(e >> 8);
            out += two ? 2 : 1;
            pos += two ? tot : l1;
        }
    }
    return pos;
}

// The stream's last segment: its codes end at bit `end` (<= 128) and zero
// padding follows, which may not decode.  One code per step (the first code of
// any pair or multi entry), the words picked by index.
template <bool COMPLETE, bool PAIRS, bool MULTI>
__device__ __forceinline__ uint32_t decode_last_segment(const uint32_t* t1, const uint16_t* __restrict__ t2,
                                                        const FirstLen& fl, const SegWords& w, uint32_t pos,
                                                        uint32_t end, uint8_t* out) {
    auto word = [&](uint32_t i) { return i == 0 ? w.w0 : i == 1 ? w.w1 : i == 2 ? w.w2 : i == 3 ? w.w3 : w.w4; };
    uint32_t cnt = 0;
    while (pos < end) {
        const uint32_t wi = pos >> 5;
        const uint32_t x = __funnelshift_l(word(wi + 1), word(wi), pos);
        const uint32_t e = lookup(t1, t2, x);
        if (!COMPLETE && (e & 0x40000000u)) break;  // the padding after the final codeword
        uint32_t len;
        if (MULTI) {
            len = ((e >> 29) & 3u) ? fl(x) : ((e >> 24) & 31u);
        } else if (PAIRS) {
            len = (e & 0x10000u) ? ((e >> 17) & 15u) : (e >> 24);
        } else {
            len = e >> 24;
        }
        out[cnt++] = (uint8_t)e;
        pos += len;
    }
    return cnt;
}

// A claimed tile and its job, in shared memory.
struct DecSlot {
    DecJob job;
    uint64_t item;    // tile id in the launch's numbering (>= nitems: none)
    uint64_t local;   // tile index within its job
    uint32_t job_id;
    uint32_t pad;
};

// COMPLETE: the book's Kraft sum is 1 (every package-merge book with two or
// more symbols), so no table entry is invalid and the decode loop skips that test.
// PAIRS: level-1 entries carry two symbols where both codes fit in the window
// (worth it for short-code books; for long codes the extra selects only cost);
// with a complete book, up to three (multi entries, widen_multi).
template <int R, int SEGS, bool COMPLETE, bool PAIRS>
__global__ void __launch_bounds__(kDecThreads, DecCfg<R, SEGS>::kMinBlocks)
    decode_kernel(const __grid_constant__ DecArgs a, const __grid_constant__ DecTable tab) {
    using C = DecCfg<R, SEGS>;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* t1 = smem;
    uint32_t* sg = smem + C::kT1;                         // gap words: sg[j] = gaps[s0/8 - 1 + j]
    uint8_t* stage = reinterpret_cast<uint8_t*>(sg + C::kGapStage);
    uint8_t* compact = stage + C::kStageBytes;
    __shared__ uint32_t warp_tot[C::kWarps];
    __shared__ DecSlot slot[3];  // ring: the tile being decoded, the next one, the previous one
    __shared__ uint64_t s_O;
    __shared__ uint64_t s_nitems;
    __shared__ uint32_t s_lut_job;

    constexpr bool MULTI = PAIRS && dec_multi(R, COMPLETE);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // single path: the u16 tables widened here, once per CTA
    auto load_tables = [&](const DecTable& t) {
        for (int i = tid; i < C::kT1; i += kDecThreads) {
            if (MULTI) {
                t1[i] = widen_multi(t.t1, i);
            } else {
                t1[i] = PAIRS ? widen_pair(t.t1, i) : widen_entry(t.t1[i]);
            }
        }
    };
    // batched path (always PAIRS): the buffer's tables come widened, copied in 16-byte groups
    auto copy_tables = [&](const DecTableW& t) {
        const uint4* s1 = reinterpret_cast<const uint4*>(t.t1);
        for (int i = tid; i < C::kT1 / 4; i += kDecThreads) reinterpret_cast<uint4*>(t1)[i] = s1[i];
    };
    // the same for the next tile of another job, as soon as this tile's decode is
    // done (nothing reads `t1` again before the next tile): asynchronous copies,
    // so their L2 round trip overlaps the look-back, write-out and compaction
    auto copy_tables_async = [&](const DecTableW& t) {
        const uint4* s1 = reinterpret_cast<const uint4*>(t.t1);
        for (int i = tid; i < C::kT1 / 4; i += kDecThreads) cp_async16(reinterpret_cast<uint4*>(t1) + i, s1 + i);
        cp_async_commit();
    };
    // thread 0: the tile `item` and its job into slot s
    auto fill_slot = [&](int s, uint64_t item) {
        DecSlot& d = slot[s];
        d.item = item;
        if (item < s_nitems) {
            const uint32_t j = a.jobs ? a.job_of[item] : 0u;
            d.job = a.jobs ? a.jobs[j] : a.single;
            d.local = a.jobs ? item - a.item0s[j] : item;
            d.job_id = j;
        }
    };

    // A tile's words go straight from global memory into registers, a tile
    // ahead: segment col's four words (one 16-byte load where the stream is
    // 16-byte aligned) and, for lane 31, the first word of the next segment
    // (the other lanes take it from their neighbour with a shuffle).  Its gap
    // words are staged in shared memory.
    uint4 pre_q[C::kPer];
    uint32_t pre_w4[C::kPer];
    uint32_t pre_gap = 0;
    auto prefetch = [&](const DecSlot& ps) {
        const bool ok = ps.item < s_nitems;
        const uint64_t s0p = ps.local * C::kSegs;
        const uint64_t words = ok ? ps.job.words : 0;
        const uint32_t* const bits = ps.job.bits;
        const bool al16 = (reinterpret_cast<uintptr_t>(bits) & 15) == 0;
#pragma unroll
        for (int k = 0; k < C::kPer; ++k) {
            const uint64_t w = 4 * (s0p + tid + k * kDecThreads);  // the segment's first word
            if (al16 && w + 4 <= words) {
                pre_q[k] = ld_stream_v4(bits + w);
            } else {
                pre_q[k].x = w < words ? ld_stream_u32(bits + w) : 0u;
                pre_q[k].y = w + 1 < words ? ld_stream_u32(bits + w + 1) : 0u;
                pre_q[k].z = w + 2 < words ? ld_stream_u32(bits + w + 2) : 0u;
                pre_q[k].w = w + 3 < words ? ld_stream_u32(bits + w + 3) : 0u;
            }
            pre_w4[k] = (lane == 31 && w + 4 < words) ? ld_stream_u32(bits + w + 4) : 0u;
        }
        // sg[j] = gaps[pg0 - 1 + j]: j = 0 exists unless the tile is its job's first
        const uint64_t pg0 = ps.local * (C::kSegs / 8);
        const uint64_t grem = ok && ps.job.gap_words + 1 > pg0 ? ps.job.gap_words + 1 - pg0 : 0;
        const uint32_t gavail = grem < (uint64_t)C::kGapStage ? (uint32_t)grem : (uint32_t)C::kGapStage;
        pre_gap = (tid < gavail && (tid > 0 || pg0 > 0)) ? __ldg(ps.job.gaps + pg0 - 1 + tid) : 0u;
    };

    if (!a.jobs) load_tables(tab);
    if (tid == 0) {
        s_nitems = a.nitems_dev ? *a.nitems_dev : a.nitems;
        fill_slot(0, atomicAdd(a.counter, 1u));
        s_lut_job = a.jobs ? ~0u : 0u;
    }
    __syncthreads();
    if (a.jobs && slot[0].item < s_nitems) copy_tables(a.tables[slot[0].job_id]);
    prefetch(slot[0]);
    if (tid < (uint32_t)C::kGapStage) sg[tid] = pre_gap;
    int ti = 0;        // slot of the tile decoded in this iteration
    int prev_s = -1;   // slot of the tile decoded one iteration earlier: its symbols wait in
                       // `compact` (at tile-local offsets) until its output offset is resolved
    uint32_t prev_ct = 0;

    for (;;) {
        __syncthreads();  // (1) gap words of the tile staged, its tables loaded; `compact` holds prev
        const DecSlot& T = slot[ti];
        const bool have = T.item < s_nitems;
        if (!have && prev_s < 0) break;
        if (tid == 0 && have) s_lut_job = T.job_id;
        const int ns = ti == 2 ? 0 : ti + 1;  // slot of the next tile
        uint32_t claim = 0;
        if (tid == 0 && have) claim = atomicAdd(a.counter, 1u);  // its latency hides behind the decode
        const uint64_t s0 = T.local * C::kSegs;  // first segment of the tile within its job
        const uint16_t* const t2 = a.jobs ? a.tables[T.job_id].t2 : tab.t2;  // level 2, not staged
        const FirstLen fl{a.jobs ? a.tables[T.job_id].l1 : nullptr, tab.t1};
        // tile-local, 32-bit from here on: segments [0, nseg) of the tile; the stream's last
        // segment (if in this tile) ends at bit end_last instead of at its 128-bit boundary
        const uint64_t seg_rem = have ? T.job.segments - s0 : 0;
        const uint32_t nseg = seg_rem < (uint64_t)C::kSegs ? (uint32_t)seg_rem : (uint32_t)C::kSegs;
        const bool last_tile = seg_rem <= (uint64_t)C::kSegs;
        // (every entry point checks segments == ceil(words / 4))
        const uint64_t bits_rem = last_tile && have ? T.job.words * 32 - 128 * s0 : 0;
        const uint32_t end_last = bits_rem < 128ull * nseg ? (uint32_t)bits_rem : 128 * nseg;
        const uint32_t first_gap = s0 ? ~0u : 0u;  // the job's first segment starts at bit 0
        // gap entry of tile segment u - 8 (u >= 7: u = 7 is the segment before the tile)
        auto gap_at = [&](uint32_t u) -> uint32_t { return (sg[u >> 3] >> (4 * (u & 7))) & 0xfu; };

        // ---- 1. decode segments tid (and tid + 256), one after the other -------
        uint32_t n[C::kPer];
#pragma unroll
        for (int k = 0; k < C::kPer; ++k) {
            SegWords w;
            w.w0 = pre_q[k].x;
            w.w1 = pre_q[k].y;
            w.w2 = pre_q[k].z;
            w.w3 = pre_q[k].w;
            const uint32_t up = __shfl_down_sync(kFull, pre_q[k].x, 1);
            w.w4 = lane == 31 ? pre_w4[k] : up;
            const uint32_t col = tid + k * kDecThreads;
            uint32_t cnt = 0;
            if (have && col < nseg) {
                const uint32_t pos = gap_at(col + 7) & (col ? ~0u : first_gap);
                uint8_t* const row = stage + col * C::kRow;
                if (last_tile && col + 1 == nseg) {
                    cnt = decode_last_segment<COMPLETE, PAIRS, MULTI>(t1, t2, fl, w, pos,
                                                                      end_last - 128 * col, row);
                } else {
                    uint8_t* out = row;
                    const uint32_t e = decode_segment<COMPLETE, PAIRS, MULTI>(t1, t2, fl, w, pos, out);
                    cnt = (uint32_t)(out - row);
                    if (e != 32 + gap_at(col + 8)) atomicOr(a.status, kDevCorrupt);
                }
            }
            n[k] = cnt;
        }

        // ---- 2. scan of the counts: both halves of the tile at once, packed in
        //         16-bit fields (a warp's 32 segments hold < 2^13 symbols)
        uint32_t packed = 0;
#pragma unroll
        for (int k = 0; k < C::kPer; ++k) packed |= n[k] << (16 * k);
        const uint32_t incl = warp_incl_scan(packed, lane);
        if (lane == 31) warp_tot[warp] = incl;
        if (tid == 0) {
            if (have) fill_slot(ns, claim);
            else slot[ns].item = ~0ull;
        }
        __syncthreads();  // (2) decode done; next tile known
        const DecSlot& N = slot[ns];
        const bool have_next = N.item < s_nitems;
        const bool reload = a.jobs && have_next && N.job_id != s_lut_job;
        if (reload) copy_tables_async(a.tables[N.job_id]);
        const uint32_t wt = warp_incl_scan(lane < (uint32_t)C::kWarps ? warp_tot[lane] : 0u, lane);
        const uint32_t totals = __shfl_sync(kFull, wt, C::kWarps - 1);
        const uint32_t before = warp ? __shfl_sync(kFull, wt, warp - 1) : 0u;
        const uint32_t total0 = totals & 0xffffu;
        const uint32_t Ct = total0 + (totals >> 16);
        const uint32_t ex = before + incl - packed;  // exclusive prefix, both fields
        uint32_t excl[C::kPer];
        excl[0] = ex & 0xffffu;
        if (C::kPer > 1) excl[C::kPer - 1] = total0 + (ex >> 16);
        if (tid == 0 && have && T.job.item0 + T.local + 1 != a.hook.hold_plus1)
            lookback_publish(a.lookback, T.job.item0 + T.local, Ct, T.local == 0);
        if (have_next) prefetch(N);  // in flight while prev is resolved and written
        if (prev_s >= 0 && warp == 0) {
            const DecSlot& Pv = slot[prev_s];
            const uint64_t rec = Pv.job.item0 + Pv.local;
            const uint64_t O = lookback_resolve<kDecLookK>(a.lookback, rec, prev_ct, Pv.local == 0, a.status, lane,
                                                           wait_limit(a.hook), rec + 1 != a.hook.hold_plus1);
            if (lane == 0) s_O = O;
        }
        __syncthreads();  // (3) prev's output offset known

        // ---- 3. write out prev: 16-byte output chunk q takes compact bytes
        //         [16q - base, 16q - base + 16), i.e. parts of two aligned groups
        if (prev_s >= 0) {
            const DecSlot& Pv = slot[prev_s];
            const uint64_t O = s_O;
            const uint32_t Cp = prev_ct;
            const uint64_t nout = Pv.job.n;
            if (tid == 0 && Pv.local + 1 == Pv.job.ntiles && O + Cp < nout) atomicOr(a.status, kDevSize);
            if (O < nout) {
                const uint64_t vstart = Pv.job.out_lo + O;
                const uint32_t base = (uint32_t)(vstart & 15);  // compact byte 0 sits at chunk offset base
                // tile-local byte positions from here on: [base, vend) of chunks 0..nq-1
                const uint32_t vend = base + (O + Cp < nout ? Cp : (uint32_t)(nout - O));
                const uint32_t nq = (vend + 15) >> 4;
                uint8_t* const out0 = Pv.job.out_aligned + (vstart & ~15ull);  // 16-byte aligned
                const uint32_t sh = 8 * (base & 3), sel = base >> 2;
                auto comb = [sh](uint32_t lo, uint32_t hi) { return sh ? __funnelshift_r(lo, hi, 32 - sh) : hi; };
                for (uint32_t lq = tid; lq < nq; lq += kDecThreads) {
                    // aligned group lq holds chunk lq's bytes [base, 16) and chunk lq+1's
                    // [0, base); group lq - 1 (for lq = 0 the stage's slack: bytes below
                    // base, never stored) the rest
                    const uint4 g = *reinterpret_cast<const uint4*>(compact + 16 * lq);
                    const uint4 p = *reinterpret_cast<const uint4*>(compact + 16 * lq - 16);
                    // output byte b = byte 16 - base + b of the 32-byte pair (p, g): output word i
                    // joins words k and k+1 of (p.x..p.w, g.x..g.w), k = 3 - base/4 + i
                    uint32_t o[4];
                    switch (sel) {  // uniform over the tile
                        case 0: o[0] = comb(p.w, g.x); o[1] = comb(g.x, g.y); o[2] = comb(g.y, g.z); o[3] = comb(g.z, g.w); break;
                        case 1: o[0] = comb(p.z, p.w); o[1] = comb(p.w, g.x); o[2] = comb(g.x, g.y); o[3] = comb(g.y, g.z); break;
                        case 2: o[0] = comb(p.y, p.z); o[1] = comb(p.z, p.w); o[2] = comb(p.w, g.x); o[3] = comb(g.x, g.y); break;
                        default: o[0] = comb(p.x, p.y); o[1] = comb(p.y, p.z); o[2] = comb(p.z, p.w); o[3] = comb(p.w, g.x); break;
                    }
                    const uint32_t c0 = 16 * lq;
                    if (c0 >= base && c0 + 16 <= vend) {
                        *reinterpret_cast<uint4*>(out0 + c0) = make_uint4(o[0], o[1], o[2], o[3]);
                    } else {  // the two ragged chunks
#pragma unroll
                        for (uint32_t b = 0; b < 16; ++b) {
                            const uint32_t vb = c0 + b;
                            if (vb >= base && vb < vend) out0[vb] = (uint8_t)(o[b >> 2] >> (8 * (b & 3)));
                        }
                    }
                }
            }
        }
        __syncthreads();  // (4) `compact` free again

        // ---- 4. compact this tile at tile-local offsets (alignment applied on write-out)
        if (have) {
#pragma unroll
            for (int k = 0; k < C::kPer; ++k) {
                // bytes up to the next word boundary of `compact` one by one, then whole
                // words (two source words funnel-shifted), then the last bytes
                const uint8_t* src = stage + (tid + k * kDecThreads) * C::kRow;
                const uint32_t d = excl[k], m = n[k];
                uint32_t h = (4u - (d & 3u)) & 3u;
                if (h > m) h = m;
                if (h > 0) compact[d] = src[0];
                if (h > 1) compact[d + 1] = src[1];
                if (h > 2) compact[d + 2] = src[2];
                const uint32_t nwords = (m - h) >> 2;
                const uint32_t* sw32 = reinterpret_cast<const uint32_t*>(src);
                uint32_t* dw = reinterpret_cast<uint32_t*>(compact + d + h);
                const uint32_t sh = 8 * h;
                uint32_t lo = sw32[0];
                for (uint32_t j = 0; j < nwords; ++j) {
                    const uint32_t hi = sw32[j + 1];
                    dw[j] = __funnelshift_r(lo, hi, sh);
                    lo = hi;
                }
                const uint32_t t = h + 4 * nwords, tl = m - t;  // 0..3 last bytes
                if (tl > 0) compact[d + t] = src[t];
                if (tl > 1) compact[d + t + 1] = src[t + 1];
                if (tl > 2) compact[d + t + 2] = src[t + 2];
            }
        }
        if (have_next) {  // sg is no longer read for this tile
            if (reload) cp_async_wait_all();
            if (tid < (uint32_t)C::kGapStage) sg[tid] = pre_gap;
        }
        prev_s = have ? ti : -1;
        prev_ct = Ct;
        ti = ns;
    }
}

uint64_t decode_tiles(uint64_t segments, uint32_t min_len, uint32_t tile_segs) {
    const uint64_t segs = dec_tile_segs_for(dec_stage_rows(min_len ? min_len : 1), tile_segs);
    return (segments + segs - 1) / segs;
}

template <int R, int SEGS, bool COMPLETE, bool PAIRS>
static int launch_decode_r(const DecArgs& a, const DecTable& t, int ctas_per_sm, cudaStream_t st) {
    using C = DecCfg<R, SEGS>;
    auto kern = decode_kernel<R, SEGS, COMPLETE, PAIRS>;
    static LaunchCache cache;  // one per kernel instantiation
    const LaunchFacts f = cache.get(reinterpret_cast<const void*>(kern), kDecThreads, C::kSmem);
    if (f.err != cudaSuccess) return f.err;
    const int sms = f.sms, per_sm = f.per_sm;
    const int k = (ctas_per_sm > 0 && ctas_per_sm < per_sm) ? ctas_per_sm : per_sm;
    const uint64_t cap = (uint64_t)sms * k;
    const unsigned grid = (unsigned)(a.nitems_dev ? cap : (a.nitems < cap ? (a.nitems ? a.nitems : 1) : cap));
    kern<<<grid, kDecThreads, C::kSmem, st>>>(a, t);
    return cudaGetLastError();
}

template <int R, bool COMPLETE, bool PAIRS>
static int launch_decode_s(const DecArgs& a, const DecTable& t, int k, uint32_t tile_segs, cudaStream_t st) {
    if (dec_tile_segs_for(R, tile_segs) == 512) return launch_decode_r<R, (R >= 32 ? 256 : 512), COMPLETE, PAIRS>(a, t, k, st);
    return launch_decode_r<R, 256, COMPLETE, PAIRS>(a, t, k, st);
}

template <bool COMPLETE, bool PAIRS>
static int launch_decode_c(const DecArgs& a, const DecTable& t, uint32_t min_len, int k, uint32_t tile_segs,
                           cudaStream_t st) {
    switch (dec_stage_rows(min_len)) {
        case 8: return launch_decode_s<8, COMPLETE, PAIRS>(a, t, k, tile_segs, st);
        case 11: return launch_decode_s<11, COMPLETE, PAIRS>(a, t, k, tile_segs, st);
        case 16: return launch_decode_s<16, COMPLETE, PAIRS>(a, t, k, tile_segs, st);
        default: return launch_decode_s<32, COMPLETE, PAIRS>(a, t, k, tile_segs, st);
    }
}

int launch_decode(const DecArgs& a, const DecTable& t, uint32_t min_len, bool complete, bool pairs,
                  int ctas_per_sm, uint32_t tile_segs, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (min_len == 0) min_len = 1;
    if (pairs)
        return complete ? launch_decode_c<true, true>(a, t, min_len, ctas_per_sm, tile_segs, st)
                        : launch_decode_c<false, true>(a, t, min_len, ctas_per_sm, tile_segs, st);
    return complete ? launch_decode_c<true, false>(a, t, min_len, ctas_per_sm, tile_segs, st)
                    : launch_decode_c<false, false>(a, t, min_len, ctas_per_sm, tile_segs, st);
}

}  // namespace hgap
