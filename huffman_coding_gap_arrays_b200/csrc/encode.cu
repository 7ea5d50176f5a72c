// encode.cu -- fused Huffman encoder with gap-array emission, sm_100a.
//
// Replaces cuencoder + cu_get_gaparray (encoder/src/encoder.cu:142-379) and
// produces the same bitstream and gap array bit for bit.
//
// Work unit: a super-tile of st_chunks x 8 KiB input bytes, taken by dynamic
// id by persistent CTAs of 512 threads.  Its bit count is one dot product of
// its histogram (recorded by hist_st_kernel in the same pass that builds the
// global histogram) with the code lengths, so a single bounded look-back over
// super-tiles gives its first output bit G right away; no per-chunk look-back
// and no waiting on neighbours afterwards.  The CTA then streams its chunks in
// order, carrying the running bit offset:
//   * 16-byte load per thread (next chunk prefetched while this one packs);
//   * lookups in a 32-way lane-replicated codeword table ([byte][lane]: each
//     lane reads its own bank, never a conflict);
//   * one block scan of per-thread bit counts (warp scan + 16 warp totals);
//   * packing with a 64-bit accumulator into a shared image of the output
//     words, indexed from the segment-aligned word below the chunk's first
//     bit, so the image's 16-byte groups are the output's 16-byte groups;
//     word emission is predicated (no divergent branch); the one word a
//     thread shares with each neighbour is OR-ed in with a shared atomic;
//   * a gap entry falls out of word completion: the code completing global
//     word w with w % 4 == 3 ends segment w/4 and its spill into the next
//     word is that segment's entry (encoder/src/encoder.cu:307-312); each
//     segment has exactly one such code, so entries are plain byte stores;
//   * complete words go out with 16-byte coalesced stores; the partial last
//     word and gap word are carried to the next chunk (double-buffered image,
//     two barriers per chunk).
// The super-tile's first partial word and gap word also hold bits of the
// previous super-tile; one warp rebuilds those by re-encoding at most 1023
// bits backwards from G (the predecessor's last bytes), so neighbouring
// super-tiles never wait on each other.  The output needs no pre-zeroing (the
// reference memsets it, encoder.cu:412-414) and no global atomics.
#include <cuda_runtime.h>

#include "device_util.cuh"

namespace hgap {

constexpr int kEncThreads = 512;
constexpr int kEncBpt = 16;
constexpr int kEncWarps = kEncThreads / 32;
static_assert(kEncThreads * kEncBpt == kEncChunkBytes, "chunk = threads x bytes per thread");
constexpr int kStgWords = kEncChunkBytes * 16 / 32 + 16;    // <= 16 bits per byte, + carry/alignment
constexpr int kGapWords = kEncChunkBytes * 16 / 1024 + 8;
constexpr int kLutWords = 256 * 32;
// two lane-replicated tables (left-aligned codes, lengths), two output images,
// two gap-word carries, one spill byte per image word
constexpr size_t kEncSmem = (size_t)(2 * kLutWords + 2 * kStgWords + 2 * kGapWords) * 4 + kStgWords;

struct EncShared {
    uint32_t warp_tot[kEncWarps];
    uint64_t red[kEncWarps];
    uint64_t st;
    uint64_t G;
    uint32_t abort;
};

__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v, EncShared& sh, uint32_t lane,
                                                  uint32_t warp) {
    v = warp_sum_u64(v);
    if (lane == 0) sh.red[warp] = v;
    __syncthreads();
    uint64_t t = 0;
#pragma unroll
    for (int i = 0; i < kEncWarps; ++i) t += sh.red[i];
    return t;
}

__global__ void __launch_bounds__(kEncThreads, 2)
    encode_kernel(const EncArgs a, const __grid_constant__ EncTable tab) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* lutc = smem;                         // [byte][lane]: code << (32 - len)
    uint32_t* lutl = smem + kLutWords;             // [byte][lane]: len (0x200 if absent)
    uint32_t* stg0 = smem + 2 * kLutWords;         // two output images, ping-pong per chunk
    uint32_t* gst0 = stg0 + 2 * kStgWords;         // two gap-word carries
    uint8_t* spills = reinterpret_cast<uint8_t*>(gst0 + 2 * kGapWords);  // per image word
    __shared__ EncShared sh;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kLutWords; i += kEncThreads) {
        const uint32_t e = tab.e[i >> 5];
        const uint32_t l = (e >> 16) & 31u;
        lutc[i] = l ? (e & 0xffffu) << (32 - l) : 0u;
        lutl[i] = (e == kEncAbsent) ? 0x200u : l;
    }
    if (tid == 0) {
        // the histograms in the workspace must come from this very input
        sh.abort = (a.tag[0] != a.hi - a.lo ||
                    a.tag[1] != reinterpret_cast<uint64_t>(a.in_aligned) + a.lo);
        if (sh.abort) atomicOr(a.status, kDevPlan);
    }
    __syncthreads();
    if (sh.abort) return;
    const bool vec_ok = a.bits_aligned16 != 0;

    for (;;) {
        __syncthreads();  // the previous super-tile is finished, its tail words included
        for (int i = tid; i < 2 * (kStgWords + kGapWords); i += kEncThreads) stg0[i] = 0;
        if (tid == 0) sh.st = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint64_t st = sh.st;
        if (st >= a.nst) break;

        // ---- super-tile bit count, look-back, bits before G -----------------
        uint64_t part = 0;
        if (tid < 256) part = (uint64_t)a.st_hist[st * 256 + tid] * (lutl[tid << 5] & 31u);
        const uint64_t agg = block_sum_u64(part, sh, lane, warp);
        if (warp == 0) {
            const uint64_t G = lookback_warp(a.st_rec, st, agg, a.status, lane);
            if (lane == 0) sh.G = G;
            const uint32_t r = (uint32_t)(G & 31);
            const uint32_t nibs = (uint32_t)((G >> 7) & 7);
            if (G > 0 && (r != 0 || nibs != 0)) {
                // walk the previous super-tile's codes backwards from G
                const uint64_t wstart = G - r;
                const uint64_t gs = (G >> 10) << 10;
                // codes starting at or below `stop` can no longer reach the head word
                // (bits >= wstart) nor cross a boundary >= gs + 128
                uint64_t stop = r ? wstart : ~0ull;
                if (nibs && gs + 127 < stop) stop = gs + 127;
                uint32_t head = 0;
                uint64_t end = G;
                const uint64_t vfirst = st * (uint64_t)a.st_bytes;  // first byte of this super-tile
                for (uint64_t base = 0;; base += 32) {
                    const uint64_t v = vfirst - 1 - base - lane;    // may wrap below lo: no byte
                    uint32_t c = 0, len = 0;
                    if (vfirst >= base + lane + 1 && v >= a.lo) {
                        const uint32_t byte = __ldg(a.in_aligned + v);
                        c = lutc[(byte << 5) | lane];
                        len = lutl[(byte << 5) | lane] & 31u;
                    }
                    const uint32_t incl = warp_incl_scan(len, lane);
                    const uint64_t ce = end - (incl - len);          // this code's end bit
                    const uint64_t cs = ce - len;                    // and start bit
                    if (len) {
                        if (r && ce > wstart)  // the code's right-aligned value, placed to end at ce
                            head |= (uint32_t)(((uint64_t)(c >> (32 - len))) << (wstart + 32 - ce));
                        const uint64_t b = (ce >> 7) << 7;           // last segment boundary <= end
                        if (nibs && b > cs && b >= gs + 128) {
                            const uint64_t k = (b >> 7) - 1;
                            atomicOr(gst0, (uint32_t)(ce - b) << (4 * (uint32_t)(k & 7)));
                        }
                    }
                    const uint32_t total = __shfl_sync(kFull, incl, 31);
                    const uint64_t smin = end - total;               // start of the batch's last code
                    end = smin;
                    if (smin <= stop || total == 0) break;
                }
                head = __reduce_or_sync(kFull, head);
                if (lane == 0 && r) stg0[(G >> 5) & 3] = head;
            }
        }
        __syncthreads();
        uint64_t P = sh.G;
        uint64_t P_st = P;

        // ---- stream the chunks ---------------------------------------------
        const uint64_t v_st = st * (uint64_t)a.st_bytes;
        uint64_t v_end = v_st + a.st_bytes;
        if (v_end > a.hi) v_end = a.hi;
        const uint32_t nchunks = (uint32_t)((v_end - v_st + kEncChunkBytes - 1) / kEncChunkBytes);
        auto load = [&](uint32_t c) -> uint4 {
            const uint64_t v = v_st + (uint64_t)c * kEncChunkBytes + (uint64_t)tid * kEncBpt;
            uint4 q = make_uint4(0, 0, 0, 0);
            if (c < nchunks && v < a.hi && v + 16 > a.lo) q = ld_stream_v4(a.in_aligned + v);
            return q;
        };
        uint4 q_next = load(0);
        uint32_t prev_used = 0;  // image words touched by the previous chunk
        for (uint32_t c = 0; c < nchunks; ++c) {
            const uint4 q = q_next;
            q_next = load(c + 1);
            uint32_t* stg = stg0 + (c & 1) * kStgWords;
            uint32_t* stg_next = stg0 + ((c + 1) & 1) * kStgWords;
            uint32_t* gst = gst0 + (c & 1) * kGapWords;
            uint32_t* gst_next = gst0 + ((c + 1) & 1) * kGapWords;

            // lookups: left-aligned code and length per byte, bit count per thread
            const uint64_t v0 = v_st + (uint64_t)c * kEncChunkBytes + (uint64_t)tid * kEncBpt;
            const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
            uint32_t cc[kEncBpt], ll[kEncBpt];
            uint32_t nbits = 0;
            if (v0 >= a.lo && v0 + kEncBpt <= a.hi) {
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
                    const bool in = v0 + k >= a.lo && v0 + k < a.hi;
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
            __syncthreads();  // (1) warp totals visible; previous chunk fully written out
            // the previous chunk's image is free again: clear it for the next chunk
            for (uint32_t i = 4 * tid; i < prev_used; i += 4 * kEncThreads)
                *reinterpret_cast<uint4*>(stg_next + i) = make_uint4(0, 0, 0, 0);
            uint32_t wt = lane < (uint32_t)kEncWarps ? sh.warp_tot[lane] : 0u;
            wt = warp_incl_scan(wt, lane);
            const uint32_t L = __shfl_sync(kFull, wt, kEncWarps - 1);
            const uint32_t excl = incl - nbits + (warp ? __shfl_sync(kFull, wt, warp - 1) : 0u);

            // pack two codes per step (<= 32 bits), at most one word per step
            const uint64_t sb = (P >> 5) & ~3ull;  // segment-aligned image base (global word)
            if (nbits) {
                const uint32_t p = (uint32_t)(P - 32 * sb) + excl;  // bit offset within the image
                uint32_t wi = p >> 5;
                uint32_t nb = p & 31;
                bool first_shared = nb != 0;  // first word also holds the left neighbour's bits
                uint32_t cur = 0;
#pragma unroll
                for (int k = 0; k < kEncBpt; k += 2) {
                    const uint32_t l1 = ll[k];
                    const uint32_t c12 = cc[k] | (cc[k + 1] >> l1);
                    const uint32_t nbo = nb;
                    cur |= c12 >> nb;
                    const uint32_t spill = __funnelshift_r(0u, c12, nb);
                    nb += l1 + ll[k + 1];
                    if (nb >= 32) {
                        if (first_shared) atomicOr(stg + wi, cur);
                        else stg[wi] = cur;
                        first_shared = false;
                        // bits of the code crossing the word end that spill over
                        spills[wi] = (uint8_t)(nbo + l1 >= 32 ? nbo + l1 - 32 : nb - 32);
                        ++wi;
                        cur = spill;
                        nb -= 32;
                    }
                }
                if (nb) atomicOr(stg + wi, cur);
            }
            __syncthreads();  // (2) image complete

            // write out complete words [P>>5, E>>5) and gap words [P>>10, kn>>3)
            const uint64_t E = P + L;
            const uint32_t j0 = (uint32_t)((P >> 5) - sb);
            const uint32_t j1 = (uint32_t)((E >> 5) - sb);
            bool overflow = false;
            for (uint32_t g = tid; g < (j1 + 3) / 4; g += kEncThreads) {
                const uint32_t j = 4 * g;
                const uint64_t w = sb + j;
                if (vec_ok && j >= j0 && j + 4 <= j1 && w + 4 <= a.words) {
                    *reinterpret_cast<uint4*>(a.bits + w) = *reinterpret_cast<const uint4*>(stg + j);
                } else {
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k) {
                        if (j + k < j0 || j + k >= j1) continue;
                        if (w + k < a.words) a.bits[w + k] = stg[j + k];
                        else overflow = true;
                    }
                }
            }
            const uint64_t kb = P >> 7, kn = E >> 7;  // segments ending in this chunk: [kb, kn)
            const uint64_t gwb = P >> 10, gwe = kn >> 3;
            for (uint64_t g = gwb + tid; g <= gwe; g += kEncThreads) {
                uint32_t v = (g == gwb) ? gst[0] : 0u;
                const uint64_t k0 = (8 * g > kb) ? 8 * g : kb;
                const uint64_t k1 = (8 * g + 8 < kn) ? 8 * g + 8 : kn;
                for (uint64_t k = k0; k < k1; ++k)  // entry k = spill of global word 4k+3
                    v |= (uint32_t)spills[(uint32_t)(4 * k + 3 - sb)] << (4 * (uint32_t)(k & 7));
                if (g < gwe) {
                    if (g < a.gap_words) a.gaps[g] = v;
                    else overflow = true;
                } else {
                    gst_next[0] = v;  // partial gap word carried to the next chunk
                }
            }
            if (tid == 0) stg_next[(E >> 5) & 3] = stg[j1];  // partial word carried
            if (overflow) atomicOr(a.status, kDevSize);
            prev_used = j1 + 2;
            P = E;
        }
        __syncthreads();  // carries visible
        // ---- end of the super-tile ------------------------------------------
        if (tid == 0) {
            if (P - P_st != agg) atomicOr(a.status, kDevPlan);  // histograms were not this input's
            if (st + 1 == a.nst) {
                const uint32_t* stg = stg0 + (nchunks & 1) * kStgWords;
                const uint32_t* gst = gst0 + (nchunks & 1) * kGapWords;
                if ((P & 31) && (P >> 5) < a.words) a.bits[P >> 5] = stg[(P >> 5) & 3];
                const uint64_t gwe = (P >> 7) >> 3;
                if (gwe < a.gap_words) a.gaps[gwe] = gst[0];
                if ((P + 31) / 32 != a.words || (P + 127) / 128 != a.segments) atomicOr(a.status, kDevSize);
            }
        }
    }
}

// ------------------------------------------------------------- launchers ---

int launch_encode(const EncArgs& a, const EncTable& t, void* stream) {
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaFuncSetAttribute(encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kEncSmem);
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, encode_kernel, kEncThreads, kEncSmem);
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t cap = (uint64_t)sms * per_sm;
    const unsigned grid = (unsigned)(a.nst < cap ? a.nst : cap);
    encode_kernel<<<grid, kEncThreads, kEncSmem, static_cast<cudaStream_t>(stream)>>>(a, t);
    return cudaGetLastError();
}

}  // namespace hgap
