// encode.cu -- fused Huffman encoder with gap-array emission, sm_100a.
//
// Replaces cuencoder + cu_get_gaparray (encoder/src/encoder.cu:142-379) and
// produces the same bitstream and gap array bit for bit.
//
// Work unit: a region (super-tile) of st_chunks x 8 KiB input bytes of one
// job, taken by global id by persistent CTAs of 512 threads; the single-buffer
// entry points run one job, the batched ones thousands, each with its own
// codebook (the CTA reloads its code tables when the job changes).  Its bit count is one dot product of
// its histogram (recorded by hist_st_kernel in the same pass that builds the
// global histogram) with the code lengths, so a single bounded look-back over
// super-tiles gives its first output bit G; no per-chunk look-back and no
// waiting on neighbours afterwards.  A CTA claims its next super-tile one
// ahead and publishes that one's bit count at once, so no look-back ever
// waits on a claimed super-tile, and the input stream never drains between
// super-tiles.
//
// Input: chunks are staged in a ring of kRing shared-memory buffers by 1-D
// bulk copies (TMA engine, completion on an mbarrier), issued by one thread
// kRing chunks ahead of the one being encoded: 48 KiB per SM in flight, which
// a one-load-per-thread register prefetch cannot reach.
//
// Per chunk:
//   * lookups in a 32-way lane-replicated codeword table ([byte][lane]: each
//     lane reads its own bank, never a conflict);
//   * one block scan of per-thread bit counts (warp scan + 16 warp totals);
//   * packing two codes at a time (<= 32 bits) into a shared image of the
//     output words, indexed from the segment-aligned word below the chunk's
//     first bit, so the image's 16-byte groups are the output's 16-byte
//     groups; every completed word is OR-ed in with a shared atomic (the
//     image is clear when a chunk starts, so for a word no neighbour shares
//     the OR is a store, and one path without a first-word flag measured 7 %
//     faster than plain stores plus an atomic for the shared word);
//   * a gap entry falls out of word completion: the code completing global
//     word w with w % 4 == 3 ends segment w/4 and its spill into the next
//     word is that segment's entry (encoder/src/encoder.cu:307-312); each
//     segment has exactly one such code, so entries are plain byte stores;
//   * complete words go out with 16-byte coalesced stores, and each group of
//     the image is cleared right after it is read; the partial last word and
//     gap word are carried to the next chunk.  Two barriers per chunk.
// The super-tile's first partial word and gap word also hold bits of the
// previous super-tile; one warp rebuilds those by re-encoding at most 1023
// bits backwards from G (the predecessor's last bytes), so neighbouring
// super-tiles never wait on each other.  The output needs no pre-zeroing (the
// reference memsets it, encoder.cu:412-414) and no global atomics.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "launch_cache.h"

namespace hgap {

constexpr int kEncThreads = 512;
constexpr int kEncBpt = 16;
constexpr int kEncWarps = kEncThreads / 32;
static_assert(kEncThreads * kEncBpt == kEncChunkBytes, "chunk = threads x bytes per thread");
constexpr int kRing = 3;                                  // input chunks staged ahead
constexpr int kImgWords = kEncChunkBytes * 16 / 32 + 16;  // <= 16 bits per byte, + carry/alignment
constexpr int kLutWords = 256 * 32;
// two lane-replicated tables (left-aligned codes, lengths), the input ring,
// the output image and one spill byte per image word
constexpr size_t kEncSmem =
    (size_t)2 * kLutWords * 4 + (size_t)kRing * kEncChunkBytes + (size_t)kImgWords * 4 + kImgWords;

struct EncShared {
    uint64_t mbar[kRing];       // one per ring buffer: its bulk copy landed
    EncJob job[2];              // slots: the current region's job and the next claimed one's
    uint64_t item[2];           // their global region ids (>= nitems: none)
    uint64_t agg[2];            // their bit counts
    uint32_t job_id[2];
    uint64_t G;                 // first output bit of the current region
    uint32_t warp_tot[kEncWarps];
    uint32_t carry;             // partial output word carried into the next chunk
    uint32_t gcarry[2];         // partial gap word carried, by chunk parity
    uint64_t nitems;            // regions of the launch
    uint32_t lut_job;           // job whose code tables are in the LUTs
    uint32_t abort;
    uint32_t p_issued;          // producer: copies issued so far (chunk sequence number)
    uint32_t p_chunk;           // producer: chunk index of the next copy within its region
    int p_which;                // producer: next copy from the current region (0) or the next one (1)
};

// Length and left-aligned code of `byte` from a job's table in global memory.
__device__ __forceinline__ void code_of(const EncTable* t, uint32_t byte, uint32_t& c, uint32_t& len) {
    const uint32_t e = t->e[byte];
    len = (e >> 16) & 31u;
    c = len ? (e & 0xffffu) << (32 - len) : 0u;
}

// Warp 0: claims a region into `slot`, copies its job there and publishes
// its bit count at once, so that no later region's look-back waits on it.
__device__ __forceinline__ void claim_region(const EncArgs& a, const uint32_t* lutl, EncShared& sh, int slot,
                                             uint32_t lane) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(a.counter, 1u);
    const uint64_t item = __shfl_sync(kFull, c, 0);
    uint32_t job = 0;
    uint64_t agg = 0;
    __syncwarp();  // every lane is done reading the slot
    if (item < sh.nitems) {
        if (a.jobs) job = find_job(a.item0s, a.count, item);
        const EncJob* src = a.jobs ? a.jobs + job : &a.single;
        static_assert(sizeof(EncJob) % 8 == 0 && sizeof(EncJob) <= 256, "job copied as u64 lanes");
        if (lane < sizeof(EncJob) / 8)
            reinterpret_cast<uint64_t*>(&sh.job[slot])[lane] = reinterpret_cast<const uint64_t*>(src)[lane];
        uint64_t part = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t b = lane + 32 * j;
            const uint32_t len = a.jobs ? ((a.tables[job].e[b] >> 16) & 31u) : (lutl[b << 5] & 31u);
            part += (uint64_t)a.st_hist[item * 256 + b] * len;
        }
        agg = warp_sum_u64(part);
        if (lane == 0 && item + 1 != a.hook.hold_plus1) lookback_publish(a.st_rec, item, agg, item == src->item0);
    }
    if (lane == 0) {
        sh.item[slot] = item;
        sh.agg[slot] = agg;
        sh.job_id[slot] = job;
    }
    __syncwarp();
}

__device__ __forceinline__ uint32_t st_chunks(const EncJob& J, uint64_t st) {
    const uint64_t v0 = st * (uint64_t)J.st_bytes;
    const uint64_t v1 = (v0 + J.st_bytes < J.hi) ? v0 + J.st_bytes : J.hi;
    return (uint32_t)((v1 - v0 + kEncChunkBytes - 1) / kEncChunkBytes);
}

// The bulk-copy producer: thread 0 at region boundaries, the last warp's first
// thread after each chunk's second barrier (never both at once; barriers order
// them).  Copies go out in the order the CTA encodes chunks: the rest of the
// current region, then the claimed next one; at most kRing beyond the last
// chunk whose buffer is free again.  Its state lives in shared memory (one
// thread touches it at a time), sparing every thread the registers.
__device__ __forceinline__ void produce(const EncArgs& a, uint8_t* ring, EncShared& sh, uint32_t freed, int cur_slot) {
    uint32_t issued = sh.p_issued, pc = sh.p_chunk;
    int which = sh.p_which;
    while (issued < freed + kRing) {
        const int slot = cur_slot ^ which;
        const uint64_t item = sh.item[slot];
        if (item >= sh.nitems) break;
        const EncJob& J = sh.job[slot];
        const uint64_t st = item - J.item0;
        if (pc >= st_chunks(J, st)) {
            if (which == 0) {
                which = 1;
                pc = 0;
                continue;
            }
            break;  // wait for the next claim
        }
        const uint64_t v = st * (uint64_t)J.st_bytes + (uint64_t)pc * kEncChunkBytes;
        const uint64_t rem = ((J.hi + 15) & ~15ull) - v;  // through the end of the last 16-byte group
        const uint32_t bytes = rem >= (uint64_t)kEncChunkBytes ? (uint32_t)kEncChunkBytes : (uint32_t)rem;
        const uint32_t s = issued % kRing;
        bulk_load(ring + (size_t)s * kEncChunkBytes, J.in_aligned + v, bytes, &sh.mbar[s]);
        ++issued;
        ++pc;
    }
    sh.p_issued = issued;
    sh.p_chunk = pc;
    sh.p_which = which;
}

__global__ void __launch_bounds__(kEncThreads, 2)
    encode_kernel(const __grid_constant__ EncArgs a, const __grid_constant__ EncTable tab) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* lutc = smem;                // [byte][lane]: code << (32 - len)
    uint32_t* lutl = smem + kLutWords;    // [byte][lane]: len (0x200 if absent)
    uint8_t* ring = reinterpret_cast<uint8_t*>(smem + 2 * kLutWords);  // kRing input chunks
    uint32_t* img = reinterpret_cast<uint32_t*>(ring + (size_t)kRing * kEncChunkBytes);
    uint8_t* spills = reinterpret_cast<uint8_t*>(img + kImgWords);     // per image word
    __shared__ EncShared sh;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto load_luts = [&](const EncTable& t) {
        for (int i = tid; i < kLutWords; i += kEncThreads) {
            const uint32_t e = t.e[i >> 5];
            const uint32_t l = (e >> 16) & 31u;
            lutc[i] = l ? (e & 0xffffu) << (32 - l) : 0u;
            lutl[i] = (e == kEncAbsent) ? 0x200u : l;
        }
    };
    if (!a.jobs) load_luts(tab);
    for (int i = tid; i < kImgWords; i += kEncThreads) img[i] = 0;
    if (tid == 0) {
        // single path: the histograms in the workspace must come from this very input
        sh.abort = a.tag && (a.tag[0] != a.single.hi - a.single.lo ||
                             a.tag[1] != reinterpret_cast<uint64_t>(a.single.in_aligned) + a.single.lo);
        if (sh.abort) atomicOr(a.status, kDevPlan);
        sh.lut_job = a.jobs ? ~0u : 0u;
        sh.nitems = a.nitems_dev ? *a.nitems_dev : a.nitems;
        sh.p_issued = 0;
        sh.p_chunk = 0;
        sh.p_which = 0;
        for (int s = 0; s < kRing; ++s) mbar_init(&sh.mbar[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (sh.abort) return;

    int cur_slot = 0;   // slot of the current region; the next one is in cur_slot ^ 1
    uint32_t cons = 0;  // chunks consumed so far (the ring's sequence number)
    if (warp == 0) {
        claim_region(a, lutl, sh, 0, lane);
        if (sh.item[0] < sh.nitems) claim_region(a, lutl, sh, 1, lane);
        else if (lane == 0) sh.item[1] = ~0ull;
        if (lane == 0) produce(a, ring, sh, 0, 0);
    }
    __syncthreads();

    for (;;) {
        const uint64_t item = sh.item[cur_slot];
        if (item >= sh.nitems) break;
        const EncJob& J = sh.job[cur_slot];
        const uint32_t jid = sh.job_id[cur_slot];
        const uint64_t st = item - J.item0;  // region within the job

        // ---- warp 0: G of the current region, bits before G ---------------------
        if (warp == 0) {
            const uint64_t G =
                J.bit0 + lookback_resolve<4>(a.st_rec, item, sh.agg[cur_slot], st == 0, a.status, lane,
                                             wait_limit(a.hook), item + 1 != a.hook.hold_plus1);
            uint32_t head = 0, gcarry = 0;
            const uint32_t r = (uint32_t)(G & 31);
            const uint32_t nibs = (uint32_t)((G >> 7) & 7);
            if (G > 0 && (r != 0 || nibs != 0)) {
                // walk the previous region's codes backwards from G
                const uint64_t wstart = G - r;
                const uint64_t gs = (G >> 10) << 10;
                // codes starting at or below `stop` can no longer reach the head
                // word (bits >= wstart) nor cross a boundary >= gs + 128
                uint64_t stop = r ? wstart : ~0ull;
                if (nibs && gs + 127 < stop) stop = gs + 127;
                uint64_t end = G;
                const uint64_t vfirst = st * (uint64_t)J.st_bytes;  // first byte of this region
                // 32 bytes a step, one per lane, going backwards; the bytes of kWalkAhead
                // steps are loaded at once (one memory round trip, not one per step)
                constexpr int kWalkAhead = 4;
                for (uint64_t base0 = 0;; base0 += 32 * kWalkAhead) {
                    uint32_t pre[kWalkAhead];
#pragma unroll
                    for (int k = 0; k < kWalkAhead; ++k) {
                        const uint64_t base = base0 + 32 * k;
                        const uint64_t v = vfirst - 1 - base - lane;  // may wrap below lo: no byte
                        pre[k] = (vfirst >= base + lane + 1 && v >= J.lo) ? (uint32_t)__ldg(J.in_aligned + v) : 0x100u;
                    }
                    bool done = false;  // warp-uniform
#pragma unroll
                    for (int k = 0; k < kWalkAhead; ++k) {
                        if (done) break;
                        uint32_t c = 0, len = 0;
                        if (pre[k] < 0x100u) {
                            const uint32_t byte = pre[k];
                            if (a.jobs) {
                                code_of(a.tables + jid, byte, c, len);
                            } else {
                                c = lutc[(byte << 5) | lane];
                                len = lutl[(byte << 5) | lane] & 31u;
                            }
                        }
                        const uint32_t incl = warp_incl_scan(len, lane);
                        const uint64_t ce = end - (incl - len);  // this code's end bit
                        const uint64_t cs = ce - len;            // and start bit
                        if (len) {
                            if (r && ce > wstart)  // the code's right-aligned value, placed to end at ce
                                head |= (uint32_t)(((uint64_t)(c >> (32 - len))) << (wstart + 32 - ce));
                            const uint64_t b = (ce >> 7) << 7;   // last segment boundary <= end
                            if (nibs && b > cs && b >= gs + 128)
                                gcarry |= (uint32_t)(ce - b) << (4 * (uint32_t)(((b >> 7) - 1) & 7));
                        }
                        const uint32_t total = __shfl_sync(kFull, incl, 31);
                        const uint64_t smin = end - total;  // start of the step's last code
                        end = smin;
                        if (smin <= stop || total == 0) done = true;
                    }
                    if (done) break;
                }
                head = __reduce_or_sync(kFull, head);
                gcarry = __reduce_or_sync(kFull, gcarry);
            }
            if (lane == 0) {
                sh.G = G;
                sh.carry = head;  // 0 unless G % 32 != 0
                sh.gcarry[cons & 1] = gcarry;
            }
        }
        // batched: the job's code tables into the LUTs (the previous region is done with them)
        if (a.jobs && jid != sh.lut_job) load_luts(a.tables[jid]);
        __syncthreads();
        if (tid == 0) sh.lut_job = jid;
        uint64_t P = sh.G;

        // ---- stream the chunks --------------------------------------------------
        const uint32_t nchunks = st_chunks(J, st);
        uint64_t v0 = st * (uint64_t)J.st_bytes + (uint64_t)tid * kEncBpt;  // this thread's first byte
        bool overflow = false;
        for (uint32_t c = 0; c < nchunks; ++c, ++cons, v0 += kEncChunkBytes) {
            const uint32_t stage = cons % kRing;
            mbar_wait(&sh.mbar[stage], (cons / kRing) & 1, a.status, true);
            const uint4 q = *reinterpret_cast<const uint4*>(ring + (size_t)stage * kEncChunkBytes + tid * 16);

            // lookups: left-aligned code and length per byte, bit count per thread
            const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
            uint32_t cc[kEncBpt], ll[kEncBpt];
            uint32_t nbits = 0;
            if (v0 >= J.lo && v0 + kEncBpt <= J.hi) {
#pragma unroll
                for (int k = 0; k < kEncBpt; ++k) {
                    const uint32_t w = w4[k >> 2];
                    const int s8 = 8 * (k & 3);
                    const uint32_t idx = ((s8 >= 5 ? (w >> (s8 - 5)) : (w << 5)) & 0x1fe0u) | lane;
                    cc[k] = lutc[idx];
                    ll[k] = lutl[idx];
                    nbits += ll[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < kEncBpt; ++k) {
                    const uint32_t idx = (((w4[k >> 2] >> (8 * (k & 3))) & 0xffu) << 5) | lane;
                    const bool in = v0 + k >= J.lo && v0 + k < J.hi;
                    cc[k] = in ? lutc[idx] : 0u;
                    ll[k] = in ? lutl[idx] : 0u;
                    nbits += ll[k];
                }
            }
            if (nbits >= 0x200u) {  // an absent byte adds 0x200 to the (< 0x200) bit count
                atomicOr(a.status, kDevNoCode);
                nbits &= 0x1ffu;
#pragma unroll
                for (int k = 0; k < kEncBpt; ++k) ll[k] &= 31u;
            }
            const uint32_t incl = warp_incl_scan(nbits, lane);
            if (lane == 31) sh.warp_tot[warp] = incl;
            __syncthreads();  // (1) warp totals visible; this ring buffer read; previous chunk written out
            // the word carried in (previous chunk's tail, or the rebuilt head word)
            if (tid == 0 && sh.carry) atomicOr(img + ((P >> 5) & 3), sh.carry);
            uint32_t wt = lane < (uint32_t)kEncWarps ? sh.warp_tot[lane] : 0u;
            wt = warp_incl_scan(wt, lane);
            const uint32_t L = __shfl_sync(kFull, wt, kEncWarps - 1);
            const uint32_t excl = incl - nbits + (warp ? __shfl_sync(kFull, wt, warp - 1) : 0u);

            // pack two codes at a time (<= 32 bits): at most one word per pair
            const uint64_t sb = (P >> 5) & ~3ull;  // segment-aligned image base (global word)
            if (nbits) {
                const uint32_t p = (uint32_t)(P - 32 * sb) + excl;  // bit offset within the image
                uint32_t wi = p >> 5;
                uint32_t nb = p & 31;
                uint32_t cur_w = 0;
#pragma unroll
                for (int k = 0; k < kEncBpt; k += 2) {
                    const uint32_t l1 = ll[k];
                    const uint32_t c12 = cc[k] | (cc[k + 1] >> l1);
                    const uint32_t nbo = nb;
                    cur_w |= c12 >> nb;
                    const uint32_t spill = __funnelshift_r(0u, c12, nb);
                    nb += l1 + ll[k + 1];
                    if (nb >= 32) {
                        atomicOr(img + wi, cur_w);  // the image starts clear: OR is a store
                        // bits of the code crossing the word end that spill over
                        spills[wi] = (uint8_t)(nbo + l1 >= 32 ? nbo + l1 - 32 : nb - 32);
                        ++wi;
                        cur_w = spill;
                        nb -= 32;
                    }
                }
                if (nb) atomicOr(img + wi, cur_w);
            }
            __syncthreads();  // (2) image complete
            // the last warp, whose write-out share is the smallest, refills the ring
            // (this chunk's buffer was read before barrier (1))
            if (tid == kEncThreads - 32) {
                fence_proxy_async_smem();
                produce(a, ring, sh, cons + 1, cur_slot);
            }

            // write out complete words [P>>5, E>>5), clearing the image behind;
            // the group holding word E>>5 hands it on as the carry
            const uint64_t E = P + L;
            const uint32_t j0 = (uint32_t)((P >> 5) - sb);
            const uint32_t j1 = (uint32_t)((E >> 5) - sb);
            uint32_t* const bits = J.bits;
            const uint64_t words = J.words;
            for (uint32_t g = tid; g <= j1 / 4; g += kEncThreads) {
                const uint32_t j = 4 * g;
                const uint4 wv = *reinterpret_cast<const uint4*>(img + j);
                const uint64_t w = sb + j;
                if (J.bits_aligned16 && j >= j0 && j + 4 <= j1 && w + 4 <= words) {
                    *reinterpret_cast<uint4*>(bits + w) = wv;
                } else {
                    const uint32_t wa[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k) {
                        if (j + k < j0 || j + k >= j1) continue;
                        if (w + k < words) bits[w + k] = wa[k];
                        else overflow = true;
                    }
                    if (j1 - j < 4) {
                        const uint32_t t = j1 - j;
                        sh.carry = (E & 31) ? (t == 0 ? wa[0] : t == 1 ? wa[1] : t == 2 ? wa[2] : wa[3]) : 0u;
                    }
                }
                *reinterpret_cast<uint4*>(img + j) = make_uint4(0, 0, 0, 0);
            }
            // gap words [P>>10, kn>>3): one thread per segment k (slot t = k - kb8)
            // puts its nibble in place, the 8 lanes of a gap word OR them with
            // shuffles; the word of kn>>3 is partial (or empty) and carried
            const uint64_t kb = P >> 7, kn = E >> 7;  // segments ending in this chunk: [kb, kn)
            const uint64_t kb8 = kb & ~7ull;
            const uint32_t nk = (uint32_t)(8 * ((kn >> 3) - (kb8 >> 3) + 1));
            // highest warps first: the write-out above took the lowest ones
            for (uint32_t t0 = (kEncWarps - 1 - warp) * 32; t0 < nk; t0 += kEncThreads) {  // warp-uniform
                const uint32_t t = t0 + lane;
                const uint64_t k = kb8 + t;
                uint32_t v = 0;
                if (t < nk && k >= kb && k < kn)  // entry k = spill of global word 4k+3
                    v = (uint32_t)spills[(uint32_t)(4 * k + 3 - sb)] << (4 * (uint32_t)(k & 7));
                if (t == 0) v |= sh.gcarry[cons & 1];  // nibbles carried into word kb8 >> 3
                v |= __shfl_xor_sync(kFull, v, 1);
                v |= __shfl_xor_sync(kFull, v, 2);
                v |= __shfl_xor_sync(kFull, v, 4);
                if (t < nk && (t & 7) == 0) {
                    const uint64_t g = k >> 3;
                    if (g < (kn >> 3)) {
                        if (g < J.gap_words) J.gaps[g] = v;
                        else overflow = true;
                    } else {
                        sh.gcarry[(cons + 1) & 1] = v;
                    }
                }
            }
            P = E;
        }
        if (overflow) atomicOr(a.status, kDevSize);
        __syncthreads();  // carries visible; the image is clear again

        // ---- end of the region --------------------------------------------------
        if (tid == 0) {
            if (P - sh.G != sh.agg[cur_slot]) atomicOr(a.status, kDevPlan);  // histograms were not this input's
            if (sh.item[cur_slot] - J.item0 + 1 == J.nst) {
                if ((P & 31) && (P >> 5) < J.words) J.bits[P >> 5] = sh.carry;
                const uint64_t gwe = (P >> 7) >> 3;
                if (gwe < J.gap_words) J.gaps[gwe] = sh.gcarry[cons & 1];
                if ((P + 31) / 32 != J.words || (P + 127) / 128 != J.segments) atomicOr(a.status, kDevSize);
            }
        }
        if (warp == 0) {
            // the next region becomes current; claim the one after it into the freed slot
            const int old = cur_slot;
            if (sh.item[old ^ 1] < sh.nitems) claim_region(a, lutl, sh, old, lane);
            else if (lane == 0) sh.item[old] = ~0ull;
            if (lane == 0) {
                // the producer's cursor follows its region into the current slot
                if (sh.p_which == 1) sh.p_which = 0;
                else sh.p_chunk = 0;
                produce(a, ring, sh, cons, old ^ 1);
            }
        }
        cur_slot ^= 1;
    }

    // every copy issued has been consumed, unless a wait gave up: never leave
    // the CTA with a copy still in flight into its shared memory
    if (tid == 0) {
        const uint32_t issued = sh.p_issued;
        const uint32_t first = issued > (uint32_t)kRing ? issued - kRing : 0u;
        for (uint32_t i = first; i < issued; ++i)
            mbar_wait(&sh.mbar[i % kRing], (i / kRing) & 1, a.status, false);
    }
}

// ------------------------------------------------------------- launchers ---

int launch_encode(const EncArgs& a, const EncTable& t, int ctas_per_sm, void* stream) {
    static LaunchCache cache;
    const LaunchFacts f = cache.get(reinterpret_cast<const void*>(encode_kernel), kEncThreads, kEncSmem);
    if (f.err != cudaSuccess) return f.err;
    const int sms = f.sms, per_sm = f.per_sm;
    const int k = (ctas_per_sm > 0 && ctas_per_sm < per_sm) ? ctas_per_sm : per_sm;
    const uint64_t cap = (uint64_t)sms * k;
    const unsigned grid = (unsigned)(a.nitems_dev ? cap : (a.nitems < cap ? (a.nitems ? a.nitems : 1) : cap));
    encode_kernel<<<grid, kEncThreads, kEncSmem, static_cast<cudaStream_t>(stream)>>>(a, t);
    return cudaGetLastError();
}

}  // namespace hgap
