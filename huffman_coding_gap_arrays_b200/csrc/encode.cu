// encode.cu -- fused Huffman encoder with gap-array emission, sm_100a.
//
// Replaces cuencoder + cu_get_gaparray (encoder/src/encoder.cu:142-379) and
// produces the same bitstream and gap array bit for bit.
//
// One persistent kernel; each CTA repeatedly takes the next 8 KiB input tile
// (dynamic tile id, as the reference does, which is what makes the look-back
// deadlock-free) and for it:
//   1. streams the tile in with 16-byte loads and looks every byte up in a
//      32-way lane-replicated codeword table (entry [byte][lane]: each lane
//      reads its own bank, so lookups never conflict);
//   2. block-scans the per-thread bit counts and runs one bounded
//      decoupled look-back (device_util.cuh) for the tile's global bit offset G;
//   3. packs the codes into a shared-memory image of the output words at
//      their global alignment (plain stores, shared-memory atomicOr only for
//      the <= 2 words a thread shares with its neighbours).  A gap nibble
//      falls out of word completion: when the code completing global word w
//      ends segment w/4 (w % 4 == 3), the bits it spills into the next word
//      are that segment's gap entry (encoder/src/encoder.cu:307-312);
//   4. writes the words and gap words it completes with coalesced stores.
//      The one word (and gap word) a tile shares with its predecessor is
//      finished through a hand-off record: each tile publishes its trailing
//      partial word before waiting on its predecessor's, so the output needs
//      no pre-zeroing (the reference memsets it, encoder.cu:412-414) and no
//      global atomics.
// Every inter-tile wait is bounded and reports kDevTimeout instead of hanging.
#include <cuda_runtime.h>

#include "device_util.cuh"

namespace hgap {

template <int THREADS, int BPT>
struct EncCfg {
    static constexpr int kTile = THREADS * BPT;  // input bytes per tile
    static constexpr int kWarps = THREADS / 32;
    static constexpr int kStg = kTile / 2 + 8;   // output words: <= 16 bits per byte
    static constexpr int kGStg = kTile / 64 + 8; // gap words: 1024 bits per gap word
    static constexpr int kLut = 256 * 32;
    static constexpr size_t kSmem = (size_t)(kLut + kStg + kGStg) * 4;
};

constexpr int kEncThreads = 256;
constexpr int kEncBpt = 32;
using EncDefault = EncCfg<kEncThreads, kEncBpt>;
static_assert(EncDefault::kTile == kEncTileBytes, "tile size is part of the workspace contract");

template <int THREADS, int BPT>
__global__ void __launch_bounds__(THREADS, 4)
    encode_kernel(const EncArgs a, const __grid_constant__ EncTable tab) {
    using C = EncCfg<THREADS, BPT>;
    static_assert(BPT % 16 == 0, "16-byte loads");
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* lut = smem;
    uint32_t* stg = smem + C::kLut;
    uint32_t* gstg = stg + C::kStg;
    __shared__ uint32_t warp_tot[C::kWarps];
    __shared__ uint64_t s_tile;
    __shared__ uint64_t s_G;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < C::kLut; i += THREADS) lut[i] = tab.e[i >> 5];
    for (int i = tid; i < C::kStg + C::kGStg; i += THREADS) stg[i] = 0;

    for (;;) {
        if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= a.ntiles) break;

        // ---- 1. load + lookup -------------------------------------------
        const uint64_t v0 = tile * C::kTile + (uint64_t)tid * BPT;
        uint32_t cw[BPT];
        uint32_t nbits = 0;
        if (v0 >= a.lo && v0 + BPT <= a.hi) {
#pragma unroll
            for (int c = 0; c < BPT / 16; ++c) {
                const uint4 q = ld_stream_v4(a.in_aligned + v0 + 16 * c);
                const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const uint32_t w = w4[k >> 2];
                    const int sh = 8 * (k & 3);
                    const uint32_t idx = (sh >= 5 ? (w >> (sh - 5)) : (w << 5)) & 0x1fe0u;
                    const uint32_t e = lut[idx | lane];
                    cw[16 * c + k] = e;
                    nbits += e >> 16;
                }
            }
        } else {
#pragma unroll
            for (int c = 0; c < BPT / 16; ++c) {
                const uint64_t vc = v0 + 16 * c;
                uint4 q = make_uint4(0, 0, 0, 0);
                if (vc < a.hi && vc + 16 > a.lo) q = ld_stream_v4(a.in_aligned + vc);
                const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const uint64_t v = vc + k;
                    const uint32_t byte = (w4[k >> 2] >> (8 * (k & 3))) & 0xffu;
                    const uint32_t e = (v >= a.lo && v < a.hi) ? lut[(byte << 5) | lane] : 0u;
                    cw[16 * c + k] = e;
                    nbits += e >> 16;
                }
            }
        }
        if (nbits >= 0x8000u) {  // an absent byte adds 0x8000 (kEncAbsent >> 16)
            atomicOr(a.status, kDevNoCode);
            nbits &= 0x7fffu;
        }

        // ---- 2. block scan + look-back ------------------------------------
        const uint32_t incl = warp_incl_scan(nbits, lane);
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t v = lane < (uint32_t)C::kWarps ? warp_tot[lane] : 0u;
            v = warp_incl_scan(v, lane);
            if (lane < (uint32_t)C::kWarps) warp_tot[lane] = v;
            const uint32_t total = __shfl_sync(kFull, v, C::kWarps - 1);
            const uint64_t G = lookback_warp(a.lookback, tile, total, a.status, lane);
            if (lane == 0) s_G = G;
        }
        __syncthreads();
        const uint32_t L = warp_tot[C::kWarps - 1];
        const uint64_t G = s_G;
        const uint32_t excl = incl - nbits + (warp ? warp_tot[warp - 1] : 0u);

        // ---- 3. pack into the shared image of words [G/32, (G+L)/32] ------
        const uint64_t wb = G >> 5;    // first global word of the tile
        const uint64_t gwb = G >> 10;  // first global gap word of the tile
        if (nbits) {
            const uint64_t p = G + excl;
            uint32_t wi = (uint32_t)((p >> 5) - wb);
            uint32_t nb = (uint32_t)(p & 31);
            bool shared_first = nb != 0;
            uint64_t acc = 0;
#pragma unroll
            for (int j = 0; j < BPT; ++j) {
                const uint32_t e = cw[j];
                const uint32_t len = (e >> 16) & 31u;
                acc = (acc << len) | (e & 0xffffu);
                nb += len;
                if (nb >= 32) {
                    nb -= 32;
                    const uint32_t word = (uint32_t)(acc >> nb);
                    if (shared_first) {
                        atomicOr(stg + wi, word);
                        shared_first = false;
                    } else {
                        stg[wi] = word;
                    }
                    const uint64_t gw = wb + wi;
                    if ((gw & 3) == 3) {  // this code crosses/ends at segment boundary
                        const uint64_t k = gw >> 2;
                        atomicOr(gstg + (uint32_t)((k >> 3) - gwb), nb << (4 * (uint32_t)(k & 7)));
                    }
                    ++wi;
                }
            }
            if (nb) atomicOr(stg + wi, (uint32_t)(acc << (32 - nb)));
        }
        __syncthreads();

        // ---- 4. write out, hand-offs with the neighbouring tiles ----------
        const uint64_t E = G + L;
        const uint32_t nfull = (uint32_t)((E >> 5) - wb);    // words completed here
        const uint64_t kn = E >> 7;                          // next gap entry to produce
        const uint32_t gfull = (uint32_t)((kn >> 3) - gwb);  // gap words completed here
        const bool last = tile + 1 == a.ntiles;
        const bool head_pend = (G & 31) != 0;          // word wb holds predecessor bits
        const bool tail_pend = (E & 31) != 0;
        const bool ghead_pend = ((G >> 7) & 7) != 0;   // gap word gwb holds predecessor nibbles
        const bool gtail_pend = (kn & 7) != 0;
        const bool dep_b = head_pend && nfull == 0;   // tail word == head word
        const bool dep_g = ghead_pend && gfull == 0;
        if (tid == 0 && !last) {
            if (!dep_b) st_relaxed_u64(a.hand_bits + tile, kHandValid | (tail_pend ? stg[nfull] : 0u));
            if (!dep_g) st_relaxed_u64(a.hand_gap + tile, kHandValid | (gtail_pend ? gstg[gfull] : 0u));
        }
        bool overflow = false;
        for (uint32_t j = (head_pend ? 1u : 0u) + tid; j < nfull; j += THREADS) {
            const uint64_t w = wb + j;
            if (w < a.words) a.bits[w] = stg[j];
            else overflow = true;
        }
        for (uint32_t j = (ghead_pend ? 1u : 0u) + tid; j < gfull; j += THREADS) {
            const uint64_t g = gwb + j;
            if (g < a.gap_words) a.gaps[g] = gstg[j];
            else overflow = true;
        }
        if (tid == 0) {
            uint32_t hw = stg[0], hg = gstg[0];
            if (head_pend) hw |= (uint32_t)wait_nonzero(a.hand_bits + tile - 1, a.status, kHandValid);
            if (ghead_pend) hg |= (uint32_t)wait_nonzero(a.hand_gap + tile - 1, a.status, kHandValid);
            if (head_pend && nfull) {
                if (wb < a.words) a.bits[wb] = hw;
                else overflow = true;
            }
            if (ghead_pend && gfull) {
                if (gwb < a.gap_words) a.gaps[gwb] = hg;
                else overflow = true;
            }
            if (!last) {
                if (dep_b) st_relaxed_u64(a.hand_bits + tile, kHandValid | hw);
                if (dep_g) st_relaxed_u64(a.hand_gap + tile, kHandValid | (gtail_pend ? hg : 0u));
            } else {
                const uint64_t we = E >> 5, gwe = kn >> 3;
                if (tail_pend) {
                    if (we < a.words) a.bits[we] = nfull ? stg[nfull] : hw;
                    else overflow = true;
                }
                if (gwe < a.gap_words) a.gaps[gwe] = gfull ? gstg[gfull] : hg;
                if ((E + 31) / 32 != a.words || (E + 127) / 128 != a.segments) overflow = true;
            }
        }
        if (overflow) atomicOr(a.status, kDevSize);
        __syncthreads();
        for (uint32_t j = tid; j <= nfull + 1 && j < (uint32_t)C::kStg; j += THREADS) stg[j] = 0;
        for (uint32_t j = tid; j <= gfull + 1 && j < (uint32_t)C::kGStg; j += THREADS) gstg[j] = 0;
    }
}

uint64_t encode_tiles(uint64_t n) {
    return (n + 15 + EncDefault::kTile - 1) / EncDefault::kTile;
}

int launch_encode(const EncArgs& a, const EncTable& t, void* stream) {
    auto kern = encode_kernel<kEncThreads, kEncBpt>;
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)EncDefault::kSmem);
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEncThreads, EncDefault::kSmem);
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t cap = (uint64_t)sms * per_sm;
    const unsigned grid = (unsigned)(a.ntiles < cap ? a.ntiles : cap);
    kern<<<grid, kEncThreads, EncDefault::kSmem, static_cast<cudaStream_t>(stream)>>>(a, t);
    return cudaGetLastError();
}

}  // namespace hgap
