// batch.cu -- the batched path (include/hgap.h, "batched path") and the
// device-side codebook entry points.  No counterpart in the reference.
//
// Compress, all on the stream, nothing back to the host:
//   1. benc_setup   one CTA: each buffer's alignment, region size and region
//                   count; an exclusive scan numbers the regions globally;
//   2. hist_st      per-region histograms and per-buffer histograms;
//   3. book         one warp per buffer: length-limited canonical codebook,
//                   encoder table, sizes (book.cuh);
//   4. benc_place   one CTA: scans of the stream sizes place every bitstream
//                   (16-byte aligned) and gap array in the two arenas;
//   5. encode       the single-buffer encoder kernel over all regions, the
//                   CTA reloading its code tables when the buffer changes.
// Decompress:
//   1. bdec_table   one CTA per buffer: checks the book, builds its decoder
//                   table in shared memory, writes it in the widened form the
//                   decode kernel keeps in shared memory (DecTableW), and puts
//                   the buffer in one of 8 classes (decoder stage size by the
//                   shortest code x complete book or not), and writes its
//                   decode job (stream, output, tile count);
//   2. bdec_setup   one CTA: look-back record numbering over all tiles, and
//                   per class the numbering of the class's tiles;
//   3. bdec_map     tile -> buffer map of each class;
//   4. decode       one persistent launch per class (all 8, or those the
//                   caller names in dec_class_mask), the single-buffer
//                   decoder kernel over the class's tiles.
// Every launch has a fixed grid and reads its work counts from device memory,
// so the sequence can be captured once and replayed.
#include <cuda_runtime.h>

#include <cstring>

#include "book.cuh"
#include "dec_entry.cuh"
#include "launch_cache.h"

namespace hgap {
namespace {

// Books (warps) per CTA of the book kernels: 14 KiB of scratch a book, so two a
// CTA put 14 books on an SM (seven CTAs), where four a CTA fitted 12 (three).
constexpr int kBookWarps = 2;
constexpr size_t kBookSmem = kBookWarps * sizeof(BookScratch);
constexpr int kScanThreads = 1024;
constexpr uint32_t kClasses = 8;
constexpr uint32_t kNoClass = 0xffu;

// ----------------------------------------------------------- block scans ---
// Exclusive scan of one u64 per thread over a 1024-thread CTA; returns the
// exclusive prefix and the block total.
__device__ __forceinline__ uint64_t block_excl_scan_u64(uint64_t v, uint64_t* total, uint64_t* s_warp) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t t = __shfl_up_sync(kFull, x, d);
        if (lane >= (uint32_t)d) x += t;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = s_warp[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t t = __shfl_up_sync(kFull, w, d);
            if (lane >= (uint32_t)d) w += t;
        }
        s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const uint64_t before = warp ? s_warp[warp - 1] : 0;
    *total = s_warp[31];
    __syncthreads();  // s_warp free for the next call
    return before + x - v;
}

// The same for two values per thread at once (one set of barriers).
__device__ __forceinline__ void block_excl_scan2_u64(uint64_t& a, uint64_t& b, uint64_t* total_a, uint64_t* total_b,
                                                     uint64_t (*s_warp)[32]) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = a, y = b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t t = __shfl_up_sync(kFull, x, d);
        const uint64_t u = __shfl_up_sync(kFull, y, d);
        if (lane >= (uint32_t)d) {
            x += t;
            y += u;
        }
    }
    if (lane == 31) {
        s_warp[0][warp] = x;
        s_warp[1][warp] = y;
    }
    __syncthreads();
    if (warp < 2) {
        uint64_t w = s_warp[warp][lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t t = __shfl_up_sync(kFull, w, d);
            if (lane >= (uint32_t)d) w += t;
        }
        s_warp[warp][lane] = w;  // inclusive over warps
    }
    __syncthreads();
    a = (warp ? s_warp[0][warp - 1] : 0) + x - a;
    b = (warp ? s_warp[1][warp - 1] : 0) + y - b;
    *total_a = s_warp[0][31];
    *total_b = s_warp[1][31];
    __syncthreads();  // s_warp free for the next call
}

// --------------------------------------------------------------- compress ---

__global__ void __launch_bounds__(kScanThreads) benc_setup_kernel(uint32_t count, const uint8_t* const* inputs,
                                                                  const uint64_t* sizes,
                                                                  const uint8_t* region_chunks,
                                                                  uint32_t base_chunks, EncJob* jobs,
                                                                  uint64_t* item0s, uint64_t* nitems,
                                                                  uint64_t max_regions, uint32_t* status) {
    __shared__ uint64_t s_warp[32];
    uint64_t carry = 0;
    // each buffer's size, input pointer and region size, the next 1024 buffers' in flight
    uint64_t n_next = 0;
    const uint8_t* in_next = nullptr;
    uint32_t rc_next = base_chunks;
    auto load = [&](uint64_t j) {
        n_next = 0;
        in_next = nullptr;
        rc_next = base_chunks;
        if (j < count) {
            n_next = sizes[j];
            in_next = inputs[j];
            if (region_chunks) rc_next = region_chunks[j];
        }
    };
    load(threadIdx.x);
    for (uint64_t base = 0; base < count; base += kScanThreads) {
        const uint64_t j = base + threadIdx.x;
        const uint64_t n = n_next;
        const uint8_t* const in = in_next;
        uint32_t rc = rc_next;
        load(j + kScanThreads);
        uint64_t nst = 0, lo = 0;
        uint32_t st = 0;
        if (j < count) {
            lo = reinterpret_cast<uintptr_t>(in) & 15;
            if (rc < base_chunks) rc = base_chunks;
            if (rc > 32) rc = 32;
            st = rc * (uint32_t)kEncChunkBytes;
            nst = n ? (lo + n + st - 1) / st : 0;
        }
        uint64_t total = 0;
        const uint64_t excl = block_excl_scan_u64(nst, &total, s_warp);
        if (j < count) {
            EncJob J;
            memset(&J, 0, sizeof(J));
            J.in_aligned = in - lo;
            J.lo = lo;
            J.hi = lo + n;
            J.item0 = carry + excl;
            J.nst = nst;
            J.st_bytes = st;
            jobs[j] = J;
            item0s[j] = carry + excl;
        }
        carry += total;
    }
    if (threadIdx.x == 0) {
        item0s[count] = carry;
        // a workspace smaller than the query asked for: nothing is encoded
        if (carry > max_regions) atomicOr(status, kDevSize);
        *nitems = carry > max_regions ? 0 : carry;
    }
}

// One warp per book: codebook from the buffer's histogram.  Optional outputs:
// the public codebook, sizes, encoder table, batch entry.
__global__ void __launch_bounds__(32 * kBookWarps) book_kernel(uint32_t count, const uint32_t* hists,
                                                               hgap_codebook* books, hgap_sizes* sizes,
                                                               EncTable* enc, hgap_batch_entry* entries,
                                                               const uint64_t* in_sizes) {
    extern __shared__ __align__(16) unsigned char book_smem[];
    BookScratch& s = reinterpret_cast<BookScratch*>(book_smem)[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t j = blockIdx.x * kBookWarps + (threadIdx.x >> 5); j < count; j += gridDim.x * kBookWarps) {
        const uint32_t* h = hists + 256 * (uint64_t)j;
        const uint32_t n = warp_code_lengths(h, s, lane);
        warp_assign_codes(s, n, lane);
        uint64_t part = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t b = lane + 32 * k;
            part += (uint64_t)h[b] * s.blen[b];
        }
        const uint64_t bits = warp_sum_u64(part);
        const uint64_t words = (bits + 31) / 32, segs = (bits + 127) / 128;
        if (books) warp_write_book(s, n, books + j, lane);
        if (enc) warp_write_enc_table(s, n, enc + j, lane);
        if (sizes && lane == 0) {
            sizes[j].bits = bits;
            sizes[j].words = words;
            sizes[j].segments = segs;
            sizes[j].gap_words = (segs + 7) / 8;
        }
        if (entries) {
            hgap_batch_entry& e = entries[j];
            for (uint32_t c = lane; c < n; c += 32) {
                e.symbols[c].symbol = s.sym[c];
                e.symbols[c].length = s.clen[c];
            }
            if (lane == 0) {
                e.n = in_sizes ? in_sizes[j] : 0;
                e.bits = bits;
                e.words = words;
                e.segments = segs;
                e.gap_words = (segs + 7) / 8;
                e.symbol_count = n;
                e.status = 0;
            }
        }
        __syncwarp();
    }
}

// Places every stream in the arenas (bitstreams 16-byte aligned) and
// completes the encoder jobs.
__global__ void __launch_bounds__(kScanThreads) benc_place_kernel(uint32_t count, hgap_batch_entry* entries,
                                                                  EncJob* jobs, uint32_t* bits,
                                                                  uint64_t bits_cap, uint32_t* gaps,
                                                                  uint64_t gaps_cap, uint32_t* status) {
    __shared__ uint64_t s_warp[2][32];
    uint64_t cb = 0, cg = 0;
    // each stream's words, gap words and segments, the next 1024 streams' in flight
    uint64_t w_next = 0, g_next = 0, s_next = 0;
    auto load = [&](uint64_t j) {
        w_next = 0;
        g_next = 0;
        s_next = 0;
        if (j < count) {
            w_next = entries[j].words;
            g_next = entries[j].gap_words;
            s_next = entries[j].segments;
        }
    };
    load(threadIdx.x);
    for (uint64_t base = 0; base < count; base += kScanThreads) {
        const uint64_t j = base + threadIdx.x;
        const uint64_t words = w_next, gap_words = g_next, segments = s_next;
        load(j + kScanThreads);
        uint64_t ob = (words + 3) & ~3ull, og = gap_words, tb = 0, tg = 0;
        block_excl_scan2_u64(ob, og, &tb, &tg, s_warp);
        ob += cb;
        og += cg;
        if (j < count) {
            hgap_batch_entry& e = entries[j];
            EncJob& J = jobs[j];
            e.bits_offset = ob;
            e.gaps_offset = og;
            if (ob + words > bits_cap || og + gap_words > gaps_cap) {
                e.status = HGAP_ERR_SIZE;  // the arena is too small: this stream is not written
                atomicOr(status, kDevSize);
                J.bits = bits;
                J.words = 0;
                J.gaps = gaps;
                J.gap_words = 0;
            } else {
                J.bits = bits + ob;
                J.words = words;
                J.gaps = gaps + og;
                J.gap_words = gap_words;
            }
            J.segments = segments;
            J.bits_aligned16 = 1;
        }
        cb += tb;
        cg += tg;
    }
}

// ------------------------------------------------------------- decompress ---

// 8 classes: the decoder's stage size (from the shortest code) x complete book
__constant__ int kStageRows[4] = {8, 11, 16, 32};
__device__ __forceinline__ uint32_t class_of(uint32_t min_len, bool complete) {
    const uint32_t r = min_len >= 4 ? 0 : 4 - min_len;  // stage rows 8, 11, 16, 32
    return 2 * r + (complete ? 1 : 0);
}

constexpr int kTableThreads = 256;

// One CTA per buffer: checks the entry, builds its two-level decoder table in
// shared memory and writes the widened form the decode kernel copies per tile
// (DecTableW), then classifies the buffer and writes its decode job (all but
// its first look-back record, which bdec_setup numbers).  The table is the one
// warp_dec_table builds (book.cuh) -- every level-1 prefix, and every level-2
// suffix of a prefix whose codes are longer than kDecPrefix bits, takes the
// symbol whose left-aligned code is the largest not above it; the level-2
// groups sit in prefix order -- but every thread owns 8 consecutive prefixes
// and a block scan places the groups, and the widened entries and the level-2
// groups in use go out with coalesced stores, in one launch.  At 32 registers
// a thread (no spills) seven CTAs fit an SM, bound by shared memory, where 40
// registers allowed six.
__global__ void __launch_bounds__(kTableThreads, 8) bdec_table_kernel(uint32_t count, const hgap_batch_entry* entries,
                                                                   const uint32_t* bits, const uint32_t* gaps,
                                                                   uint8_t* const* outputs, uint32_t tile_segs,
                                                                   DecTableW* wtables, uint8_t* cls, DecJob* jobs,
                                                                   uint32_t* status) {
    constexpr uint32_t P = kDecPrefix, X = kMaxLen - kDecPrefix;  // 11, 5
    constexpr uint32_t kT1 = 1u << P, kPer = kT1 / kTableThreads;  // 8 prefixes a thread
    __shared__ BookScratch s;
    __shared__ __align__(16) uint16_t s1[kT1];
    __shared__ __align__(16) uint16_t s2[kDecT2Cap];
    __shared__ uint16_t s_end[kT1];  // level-2 offset after each prefix's group (0 for none)
    __shared__ uint32_t s_warp[kTableThreads / 32];
    __shared__ uint32_t s_kraft;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t j = blockIdx.x; j < count; j += gridDim.x) {
        const hgap_batch_entry& e = entries[j];
        const uint32_t n = e.symbol_count;
        bool bad = n > 256 || e.segments != (e.words + 3) / 4 || e.gap_words != (e.segments + 7) / 8 ||
                   (e.n != 0) != (e.words != 0) || (e.n != 0 && n == 0);
        if (warp == 0) {
            const uint32_t kraft = (!bad && n) ? warp_load_symbols(e.symbols, n, s, lane) : 0u;
            if (lane == 0) s_kraft = kraft;
        }
        __syncthreads();
        const uint32_t kraft = s_kraft;
        if (n && kraft == ~0u) bad = true;
        uint32_t c = kNoClass;
        if (!bad && n) {  // uniform over the CTA
            // the largest symbol index i >= from with la[i] <= v (la[0] = 0, la ascends)
            auto advance = [&](uint32_t i, uint32_t v) {
                while (i + 1 < n && s.la[i + 1] <= v) ++i;
                return i;
            };
            auto search = [&](uint32_t v) {
                uint32_t lo = 0, hi = n;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (s.la[mid] <= v) lo = mid;
                    else hi = mid;
                }
                return lo;
            };
            auto entry = [&](uint32_t i, uint32_t v) -> uint16_t {
                const uint32_t L = s.clen[i];
                if (v < s.la[i] || v - s.la[i] >= (1u << (kMaxLen - L))) return kDecInvalid;
                return (uint16_t)(((L - 1) << 8) | s.sym[i]);
            };
            const uint32_t x0 = kPer * tid;
            // pass 1: the level-1 entries, and the widths of this thread's pointer prefixes
            uint32_t span = 0, pmask = 0;
            uint32_t i_first = search(x0 << X), i_last = i_first;
            const uint32_t i_start = i_first;
#pragma unroll
            for (uint32_t k = 0; k < kPer; ++k) {
                const uint32_t x = x0 + k;
                const uint32_t v = x << X;
                i_first = advance(i_first, v);
                i_last = advance(i_last > i_first ? i_last : i_first, v | ((1u << X) - 1));
                const uint32_t L = s.clen[i_last];
                if (L > P && (s.la[i_last] >> X) == x) {
                    span += 1u << (L - P);
                    pmask |= 1u << k;
                } else {
                    s1[x] = entry(i_first, v);
                }
            }
            // block scan of the spans: the level-2 offset of this thread's first group
            const uint32_t incl = warp_incl_scan(span, lane);
            if (lane == 31) s_warp[warp] = incl;
            __syncthreads();
            const uint32_t wt = warp_incl_scan(lane < kTableThreads / 32 ? s_warp[lane] : 0u, lane);
            const uint32_t total = __shfl_sync(kFull, wt, kTableThreads / 32 - 1);
            uint32_t off = (warp ? __shfl_sync(kFull, wt, warp - 1) : 0u) + incl - span;
            if (total <= (uint32_t)kDecT2Cap) {  // uniform; larger only for an incomplete book
                // pass 2: the pointer prefixes, and every prefix's level-2 end offset
                i_first = i_start;
                for (uint32_t k = 0; k < kPer; ++k) {
                    const uint32_t x = x0 + k;
                    const uint32_t v = x << X;
                    i_first = advance(i_first, v);
                    if (pmask >> k & 1u) {
                        i_last = advance(i_first, v | ((1u << X) - 1));
                        const uint32_t w = s.clen[i_last] - P;
                        s1[x] = (uint16_t)(0x8000u | (w << 12) | off);
                        off += 1u << w;
                    }
                    s_end[x] = (uint16_t)off;
                }
                __syncthreads();
                // the level-2 entries, spread over all threads (the pointer prefixes sit
                // together at the top of the code space, so per-prefix ownership would leave
                // a few threads with hundreds of entries): entry k belongs to the first prefix
                // whose end offset exceeds k
                const uint32_t used = (total + 7) & ~7u;  // whole 16-byte groups, the tail invalid
                for (uint32_t k = tid; k < used; k += kTableThreads) {
                    uint16_t e2 = kDecInvalid;
                    if (k < total) {
                        uint32_t lo = 0, hi = kT1 - 1;
                        while (lo < hi) {
                            const uint32_t mid = (lo + hi) >> 1;
                            if (s_end[mid] > k) hi = mid;
                            else lo = mid + 1;
                        }
                        const uint32_t e1 = s1[lo];  // a pointer entry: width and start of its group
                        const uint32_t w = (e1 >> 12) & 7u;
                        const uint32_t vy = (lo << X) | ((k - (e1 & 0xfffu)) << (X - w));
                        e2 = entry(search(vy), vy);
                    }
                    s2[k] = e2;
                }
                __syncthreads();
                c = class_of(s.clen[0], kraft == (1u << kMaxLen));
                const bool multi = dec_multi(kStageRows[c >> 1], (c & 1u) != 0);
                DecTableW& w = wtables[j];
                for (uint32_t i = tid; i < kT1; i += kTableThreads) {
                    w.t1[i] = multi ? widen_multi(s1, i) : widen_pair(s1, i);
                    w.l1[i] = first_len(s1, i);
                }
                for (uint32_t i = tid; i < used / 8; i += kTableThreads)
                    reinterpret_cast<uint4*>(w.t2)[i] = reinterpret_cast<const uint4*>(s2)[i];
            } else {
                bad = true;
            }
        }
        if (tid == 0) {
            if (bad) {
                atomicOr(status, kDevCorrupt);
                c = kNoClass;
            }
            cls[j] = (uint8_t)c;
            // the buffer's decode job (its first look-back record comes from bdec_setup)
            uint64_t nt = 0;
            if (c != kNoClass) {  // tiles of the class's decoder
                const uint64_t segs = dec_tile_segs_for(dec_stage_rows(c / 2 == 0 ? 4 : 4 - c / 2), tile_segs);
                nt = (e.segments + segs - 1) / segs;
            }
            DecJob J;
            memset(&J, 0, sizeof(J));
            J.bits = bits + e.bits_offset;
            J.words = e.words;
            J.gaps = gaps + e.gaps_offset;
            J.gap_words = e.gap_words;
            J.segments = e.segments;
            uint8_t* out = outputs[j];
            J.out_lo = reinterpret_cast<uintptr_t>(out) & 15;
            J.out_aligned = out - J.out_lo;
            J.n = e.n;
            J.ntiles = nt;
            jobs[j] = J;
        }
        __syncthreads();  // s, s1, s2 are reused for the next buffer
    }
}

// One CTA: the look-back record numbering over all buffers' tiles, and per
// class the numbering of the class's tiles (the jobs come from bdec_table).
// Per 1024 buffers: nine warp scans of the tile counts (all tiles, and one per
// class with the other classes' buffers counting 0) need no barrier; nine
// warps then scan the 32 warp totals of one sum each, between two barriers,
// and every buffer writes its record and, for its own class only, its first
// class tile (the only entry the map and the decoder read).  The next 1024
// buffers' loads are in flight meanwhile.
__global__ void __launch_bounds__(kScanThreads) bdec_setup_kernel(uint32_t count, const uint8_t* cls, DecJob* jobs,
                                                                  uint64_t* item0s, uint64_t* class_nitems,
                                                                  uint64_t tiles_cap, uint32_t class_mask,
                                                                  uint32_t* status) {
    constexpr uint32_t kSums = kClasses + 1;  // the classes, then all tiles
    constexpr uint32_t kWarps = kScanThreads / 32;
    __shared__ uint64_t s_tot[2][kSums][kWarps];  // by chunk parity: warp totals, then warp offsets
    __shared__ uint64_t s_carry[kSums];           // the sums over the earlier chunks
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < kSums) s_carry[threadIdx.x] = 0;
    uint32_t c_next = kNoClass;
    uint64_t nt_next = 0;
    if (threadIdx.x < count) {
        c_next = cls[threadIdx.x];
        nt_next = jobs[threadIdx.x].ntiles;  // 0 for a buffer in no class
    }
    uint32_t par = 0;
    for (uint64_t base = 0; base < count; base += kScanThreads, par ^= 1u) {
        const uint64_t j = base + threadIdx.x;
        const uint32_t c = c_next;
        const uint64_t nt = nt_next;
        const uint64_t jn = j + kScanThreads;
        c_next = kNoClass;
        nt_next = 0;
        if (jn < count) {
            c_next = cls[jn];
            nt_next = jobs[jn].ntiles;
        }
        uint64_t x_all = nt, x_own = 0;
        for (uint32_t k = 0; k < kSums; ++k) {
            uint64_t x = k == kClasses ? nt : (c == k ? nt : 0);
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t t = __shfl_up_sync(kFull, x, d);
                if (lane >= (uint32_t)d) x += t;
            }
            if (lane == 31) s_tot[par][k][warp] = x;
            if (k == kClasses) x_all = x;
            else if (c == k) x_own = x;
        }
        __syncthreads();
        if (warp < kSums) {
            const uint64_t v = s_tot[par][warp][lane];
            uint64_t x = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t t = __shfl_up_sync(kFull, x, d);
                if (lane >= (uint32_t)d) x += t;
            }
            const uint64_t carry = s_carry[warp];
            __syncwarp();
            s_tot[par][warp][lane] = carry + x - v;
            if (lane == 31) s_carry[warp] = carry + x;
        }
        __syncthreads();
        if (j < count) {
            jobs[j].item0 = s_tot[par][kClasses][warp] + x_all - nt;
            if (c < kClasses) item0s[(uint64_t)c * (count + 1) + j] = s_tot[par][c][warp] + x_own - nt;
        }
    }
    // (the last chunk's second barrier orders every s_carry update before these reads)
    const uint64_t all = s_carry[kClasses];
    // a workspace smaller than the query asked for: nothing is decoded
    const bool fits = all <= tiles_cap;
    if (threadIdx.x == 0 && !fits) atomicOr(status, kDevSize);
    if (threadIdx.x < kClasses) {
        const uint64_t tk = s_carry[threadIdx.x];
        item0s[(uint64_t)threadIdx.x * (count + 1) + count] = tk;
        class_nitems[threadIdx.x] = fits ? tk : 0;
        // a class the caller left out of the launch holds buffers: they stay undecoded
        if (class_mask && tk && !(class_mask >> threadIdx.x & 1u)) atomicOr(status, kDevPlan);
    }
}

// tile -> job map of each class: job_of[k * cap + item] = job
__global__ void bdec_map_kernel(uint32_t count, const DecJob* jobs, const uint8_t* cls, const uint64_t* item0s,
                                uint32_t* job_of, uint64_t cap) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); j < count;
         j += gridDim.x * (blockDim.x >> 5)) {
        const uint32_t c = cls[j];
        if (c == kNoClass) continue;
        const uint64_t i0 = item0s[(uint64_t)c * (count + 1) + j];
        const uint64_t nt = jobs[j].ntiles;
        for (uint64_t t = lane; t < nt; t += 32)
            if (i0 + t < cap) job_of[(uint64_t)c * cap + i0 + t] = j;
    }
}

// One warp per book: the decoder table of a public codebook.
__global__ void __launch_bounds__(32 * kBookWarps) dec_table_kernel(uint32_t count, const hgap_codebook* books,
                                                                    uint16_t* tables, uint32_t* status) {
    extern __shared__ __align__(16) unsigned char book_smem[];
    BookScratch& s = reinterpret_cast<BookScratch*>(book_smem)[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t j = blockIdx.x * kBookWarps + (threadIdx.x >> 5); j < count; j += gridDim.x * kBookWarps) {
        const uint32_t n = books[j].symbol_count;
        DecTable* t = reinterpret_cast<DecTable*>(tables + (uint64_t)j * (HGAP_DEC_T1_ENTRIES + HGAP_DEC_T2_ENTRIES));
        bool ok = n >= 1 && n <= 256;
        if (ok) {
            const uint32_t kraft = warp_load_symbols(books[j].symbols, n, s, lane);
            ok = kraft != ~0u && warp_dec_table(s, n, t, lane);
        }
        if (!ok && lane == 0 && status) atomicOr(status + j, 1u);
        __syncwarp();
    }
}

// --------------------------------------------------------- host helpers ---

template <class K>
cudaError_t set_book_smem(K kern) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBookSmem);
}

// One warp per book (or buffer), every CTA launched at once: the block
// scheduler starts each as a slot frees.
unsigned book_grid(uint32_t count) {
    const uint64_t want = (count + kBookWarps - 1) / kBookWarps;
    const uint64_t cap = 1u << 24;
    return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

// One CTA per buffer: the block scheduler hands a buffer to whichever SM frees
// a slot first, where a grid of a fixed multiple of the SMs that looped over
// the buffers started its last CTAs only after the first ones' loops ended.
unsigned table_grid(uint32_t count) {
    constexpr uint32_t kMax = 1u << 24;
    return count < kMax ? (count ? count : 1) : kMax;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

uint32_t base_chunks(const hgap_batch_config* cfg) {
    uint32_t rc = cfg && cfg->region_chunks ? cfg->region_chunks : 8;
    return rc > 32 ? 32 : rc;
}

// Compress workspace: [header 1024: status @0, counter @4, nitems @64]
// [jobs] [item0s] [tables] [hists] then the per-region arrays [st_rec | st_hist]
// for as many regions as the rest of the workspace holds.
constexpr size_t kEncPerRegion = 8 + 1024;

struct EncLayout {
    size_t jobs, item0s, tables, hists, st_rec, st_hist, fixed;
    uint64_t max_regions;
};

EncLayout enc_layout(uint32_t count, size_t workspace_bytes) {
    EncLayout L;
    size_t off = 1024;
    L.jobs = off;
    off = align256(off + sizeof(EncJob) * (size_t)count);
    L.item0s = off;
    off = align256(off + 8 * ((size_t)count + 1));
    L.tables = off;
    off = align256(off + sizeof(EncTable) * (size_t)count);
    L.hists = off;
    off = align256(off + 1024 * (size_t)count);
    L.fixed = off;
    L.max_regions = workspace_bytes > off + 256 ? (workspace_bytes - off - 256) / kEncPerRegion : 0;
    L.st_rec = off;
    L.st_hist = align256(off + 8 * (size_t)L.max_regions);
    return L;
}

uint64_t worst_regions(uint32_t count, const uint64_t* sizes, const hgap_batch_config* cfg) {
    const uint64_t st = (uint64_t)base_chunks(cfg) * kEncChunkBytes;
    uint64_t r = 0;
    for (uint32_t j = 0; j < count; ++j) r += sizes[j] ? (sizes[j] + 15 + st - 1) / st : 0;
    return r;
}

// Decompress workspace: [header 1024: status @0, counters[8] @64, class nitems[8] @128]
// [jobs] [widened tables] [classes] [item0s 8 x (count+1)] then the per-tile arrays
// [records | job_of 8 x cap] for as many tiles as the rest holds.
constexpr size_t kDecPerTile = 8 + 4 * kClasses;

struct DecLayout {
    size_t jobs, wtables, cls, item0s, records, job_of, fixed;
    uint64_t tiles_cap;
};

DecLayout dec_layout(uint32_t count, size_t workspace_bytes) {
    DecLayout L;
    size_t off = 1024;
    L.jobs = off;
    off = align256(off + sizeof(DecJob) * (size_t)count);
    L.wtables = off;
    off = align256(off + sizeof(DecTableW) * (size_t)count);
    L.cls = off;
    off = align256(off + (size_t)count);
    L.item0s = off;
    off = align256(off + 8 * (size_t)kClasses * ((size_t)count + 1));
    L.fixed = off;
    L.tiles_cap = workspace_bytes > off + 256 ? (workspace_bytes - off - 256) / kDecPerTile : 0;
    L.records = off;
    L.job_of = align256(off + 8 * (size_t)L.tiles_cap);
    return L;
}

uint64_t worst_tiles(uint32_t count, const uint64_t* sizes) {
    // a stream has at most ceil(n / 8) segments (16-bit codes): ceil(n / 2048) tiles of 256
    uint64_t cap = 0;
    for (uint32_t j = 0; j < count; ++j) cap += (sizes[j] + 2047) / 2048;
    return cap;
}

inline hgap_status cuda_status(int e) { return e == 0 ? HGAP_OK : HGAP_ERR_CUDA; }

}  // namespace
}  // namespace hgap

using namespace hgap;

extern "C" {

hgap_status hgap_codebook_build_device(uint32_t count, const uint32_t* d_hists, hgap_codebook* d_books,
                                       hgap_sizes* d_sizes, hgap_stream_t stream) {
    if (count == 0) return HGAP_OK;
    if (!d_hists || !d_books) return HGAP_ERR_INVALID_ARG;
    if (set_book_smem(book_kernel) != cudaSuccess) return HGAP_ERR_CUDA;
    book_kernel<<<book_grid(count), 32 * kBookWarps, kBookSmem, reinterpret_cast<cudaStream_t>(stream)>>>(
        count, d_hists, d_books, d_sizes, nullptr, nullptr, nullptr);
    return cuda_status(cudaGetLastError());
}

hgap_status hgap_decode_table_build_device(uint32_t count, const hgap_codebook* d_books, uint16_t* d_tables,
                                           uint32_t* d_status, hgap_stream_t stream) {
    if (count == 0) return HGAP_OK;
    if (!d_books || !d_tables) return HGAP_ERR_INVALID_ARG;
    if (set_book_smem(dec_table_kernel) != cudaSuccess) return HGAP_ERR_CUDA;
    dec_table_kernel<<<book_grid(count), 32 * kBookWarps, kBookSmem, reinterpret_cast<cudaStream_t>(stream)>>>(
        count, d_books, d_tables, d_status);
    return cuda_status(cudaGetLastError());
}

size_t hgap_batch_compress_workspace_bytes(uint32_t count, const uint64_t* sizes, const hgap_batch_config* cfg) {
    if (count && !sizes) return 0;
    const EncLayout L = enc_layout(count, 0);
    return L.fixed + 256 + kEncPerRegion * (size_t)worst_regions(count, sizes, cfg) + 256;
}

size_t hgap_batch_decompress_workspace_bytes(uint32_t count, const uint64_t* sizes) {
    if (count && !sizes) return 0;
    const DecLayout L = dec_layout(count, 0);
    return L.fixed + 256 + kDecPerTile * (size_t)worst_tiles(count, sizes) + 256;
}

uint64_t hgap_batch_bits_capacity(uint32_t count, const uint64_t* sizes) {
    uint64_t w = 0;  // at most 16 bits per byte, each stream rounded up to 4 words
    for (uint32_t j = 0; j < count; ++j) w += ((sizes[j] * 16 + 31) / 32 + 3) & ~3ull;
    return w;
}

uint64_t hgap_batch_gaps_capacity(uint32_t count, const uint64_t* sizes) {
    uint64_t g = 0;
    for (uint32_t j = 0; j < count; ++j) g += ((sizes[j] * 16 + 127) / 128 + 7) / 8;
    return g;
}

hgap_status hgap_batch_compress(uint32_t count, const uint8_t* const* d_inputs, const uint64_t* d_sizes,
                                const uint8_t* d_region_chunks, uint32_t* d_bits, uint64_t bits_capacity,
                                uint32_t* d_gaps, uint64_t gaps_capacity, hgap_batch_entry* d_entries,
                                void* d_workspace, size_t workspace_bytes, const hgap_batch_config* cfg,
                                hgap_stream_t stream) {
    if (count == 0) return HGAP_OK;
    if (!d_inputs || !d_sizes || !d_bits || !d_gaps || !d_entries || !d_workspace) return HGAP_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 255) || (reinterpret_cast<uintptr_t>(d_bits) & 15) ||
        (reinterpret_cast<uintptr_t>(d_gaps) & 3))
        return HGAP_ERR_INVALID_ARG;
    const hgap_batch_config dflt = {0, 0, 0, 0, 0, 0};
    if (!cfg) cfg = &dflt;
    const EncLayout L = enc_layout(count, workspace_bytes);
    if (L.max_regions == 0) return HGAP_ERR_WORKSPACE;
    uint8_t* ws = static_cast<uint8_t*>(d_workspace);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* status = reinterpret_cast<uint32_t*>(ws);
    uint64_t* nitems = reinterpret_cast<uint64_t*>(ws + 64);
    EncJob* jobs = reinterpret_cast<EncJob*>(ws + L.jobs);
    uint64_t* item0s = reinterpret_cast<uint64_t*>(ws + L.item0s);
    EncTable* tables = reinterpret_cast<EncTable*>(ws + L.tables);
    uint32_t* hists = reinterpret_cast<uint32_t*>(ws + L.hists);
    uint64_t* st_rec = reinterpret_cast<uint64_t*>(ws + L.st_rec);
    uint32_t* st_hist = reinterpret_cast<uint32_t*>(ws + L.st_hist);

    if (cudaMemsetAsync(ws, 0, 1024, st) != cudaSuccess) return HGAP_ERR_CUDA;
    if (cudaMemsetAsync(hists, 0, 1024 * (size_t)count, st) != cudaSuccess) return HGAP_ERR_CUDA;
    benc_setup_kernel<<<1, kScanThreads, 0, st>>>(count, d_inputs, d_sizes, d_region_chunks, base_chunks(cfg), jobs,
                                                  item0s, nitems, L.max_regions, status);
    if (cudaGetLastError() != cudaSuccess) return HGAP_ERR_CUDA;
    if (cudaMemsetAsync(st_rec, 0, 8 * (size_t)L.max_regions, st) != cudaSuccess) return HGAP_ERR_CUDA;

    HistStArgs h;
    std::memset(&h, 0, sizeof(h));
    h.jobs = jobs;
    h.item0s = item0s;
    h.count = count;
    h.nitems_dev = nitems;
    h.hist = hists;
    h.st_hist = st_hist;
    h.counter = status + 2;  // in the zeroed header, beside the encoder's region counter
    if (launch_hist_st(h, (int)cfg->hist_ctas_per_sm, stream) != 0) return HGAP_ERR_CUDA;

    if (set_book_smem(book_kernel) != cudaSuccess) return HGAP_ERR_CUDA;
    book_kernel<<<book_grid(count), 32 * kBookWarps, kBookSmem, st>>>(count, hists, nullptr, nullptr, tables,
                                                                      d_entries, d_sizes);
    if (cudaGetLastError() != cudaSuccess) return HGAP_ERR_CUDA;
    benc_place_kernel<<<1, kScanThreads, 0, st>>>(count, d_entries, jobs, d_bits, bits_capacity, d_gaps,
                                                  gaps_capacity, status);
    if (cudaGetLastError() != cudaSuccess) return HGAP_ERR_CUDA;

    EncArgs a;
    std::memset(&a, 0, sizeof(a));
    a.jobs = jobs;
    a.item0s = item0s;
    a.tables = tables;
    a.count = count;
    a.nitems_dev = nitems;
    a.st_rec = st_rec;
    a.st_hist = st_hist;
    a.counter = status + 1;
    a.status = status;
    EncTable unused;
    std::memset(&unused, 0, sizeof(unused));
    return cuda_status(launch_encode(a, unused, (int)cfg->enc_ctas_per_sm, stream));
}

hgap_status hgap_batch_decompress(uint32_t count, const hgap_batch_entry* d_entries, const uint32_t* d_bits,
                                  const uint32_t* d_gaps, uint8_t* const* d_outputs, void* d_workspace,
                                  size_t workspace_bytes, const hgap_batch_config* cfg, hgap_stream_t stream) {
    if (count == 0) return HGAP_OK;
    if (!d_entries || !d_bits || !d_gaps || !d_outputs || !d_workspace) return HGAP_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(d_workspace) & 255) return HGAP_ERR_INVALID_ARG;
    const hgap_batch_config dflt = {0, 0, 0, 0, 0, 0};
    if (!cfg) cfg = &dflt;
    const DecLayout L = dec_layout(count, workspace_bytes);
    if (L.tiles_cap == 0) return HGAP_ERR_WORKSPACE;
    uint8_t* ws = static_cast<uint8_t*>(d_workspace);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* status = reinterpret_cast<uint32_t*>(ws);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + 64);
    uint64_t* class_nitems = reinterpret_cast<uint64_t*>(ws + 128);
    DecJob* jobs = reinterpret_cast<DecJob*>(ws + L.jobs);
    DecTableW* wtables = reinterpret_cast<DecTableW*>(ws + L.wtables);
    uint8_t* cls = ws + L.cls;
    uint64_t* item0s = reinterpret_cast<uint64_t*>(ws + L.item0s);
    uint64_t* records = reinterpret_cast<uint64_t*>(ws + L.records);
    uint32_t* job_of = reinterpret_cast<uint32_t*>(ws + L.job_of);

    if (cudaMemsetAsync(ws, 0, 1024, st) != cudaSuccess) return HGAP_ERR_CUDA;
    bdec_table_kernel<<<table_grid(count), kTableThreads, 0, st>>>(count, d_entries, d_bits, d_gaps, d_outputs,
                                                                   cfg->dec_tile_segs, wtables, cls, jobs, status);
    if (cudaGetLastError() != cudaSuccess) return HGAP_ERR_CUDA;
    bdec_setup_kernel<<<1, kScanThreads, 0, st>>>(count, cls, jobs, item0s, class_nitems, L.tiles_cap,
                                                  cfg->dec_class_mask, status);
    if (cudaGetLastError() != cudaSuccess) return HGAP_ERR_CUDA;
    bdec_map_kernel<<<book_grid(count), 32 * kBookWarps, 0, st>>>(count, jobs, cls, item0s, job_of, L.tiles_cap);
    if (cudaGetLastError() != cudaSuccess) return HGAP_ERR_CUDA;
    if (cudaMemsetAsync(records, 0, 8 * (size_t)L.tiles_cap, st) != cudaSuccess) return HGAP_ERR_CUDA;

    DecTable unused;
    std::memset(&unused, 0, sizeof(unused));
    static const uint32_t kMinLen[4] = {4, 3, 2, 1};  // a representative shortest code per stage size
    for (uint32_t c = 0; c < kClasses; ++c) {
        if (cfg->dec_class_mask && !(cfg->dec_class_mask >> c & 1u)) continue;
        DecArgs a;
        std::memset(&a, 0, sizeof(a));
        a.jobs = jobs;
        a.job_of = job_of + (uint64_t)c * L.tiles_cap;
        a.item0s = item0s + (uint64_t)c * (count + 1);
        a.tables = wtables;
        a.count = count;
        a.nitems_dev = class_nitems + c;
        a.lookback = records;
        a.counter = counters + c;
        a.status = status;
        // batched streams are compressible ones on the whole: always two symbols per lookup where they fit
        if (launch_decode(a, unused, kMinLen[c / 2], (c & 1) != 0, true, (int)cfg->dec_ctas_per_sm,
                          cfg->dec_tile_segs, stream) != 0)
            return HGAP_ERR_CUDA;
    }
    return HGAP_OK;
}

uint32_t hgap_batch_decoder_class(const hgap_symlen* symbols, uint32_t count) {
    if (!symbols || count == 0) return kNoClass;
    uint32_t min_len = kMaxLen;
    uint64_t kraft = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t L = symbols[i].length;
        if (L >= 1 && L <= (uint32_t)kMaxLen) {
            min_len = L < min_len ? L : min_len;
            kraft += 1ull << (kMaxLen - L);
        }
    }
    const uint32_t r = min_len >= 4 ? 0 : 4 - min_len;
    return 2 * r + (kraft == (1ull << kMaxLen) ? 1u : 0u);
}

hgap_status hgap_batch_status(const void* d_workspace, hgap_stream_t stream) {
    return hgap_workspace_status(d_workspace, stream);
}

}  // extern "C"
