// decode.cu -- segment-parallel Huffman decoder driven by the gap array, sm_100a.
//
// Replaces gpu_dec_l1_l2 (decoder/src/decoder.cu:454-730).  Same unit of
// parallelism -- one thread per 128-bit segment, starting at the segment's
// gap offset -- but each segment is decoded ONCE (the reference decodes it
// twice: a counting pass, then a writing pass, decoder.cu:529-569,672-725):
//   1. a CTA stages its 128 segments' bitstream words in shared memory and
//      every thread decodes its segment through a shared-memory two-level
//      table (11-bit first level), parking the symbols in a private
//      column-major shared-memory area (conflict-free word stores);
//   2. block scan of the per-segment symbol counts + one bounded decoupled
//      look-back gives the tile's output offset;
//   3. the threads compact their symbols into a shared-memory image of the
//      output at its 16-byte alignment, and the CTA writes it with 16-byte
//      coalesced stores (byte stores only on the two ragged edges), clipped
//      at exactly n bytes (the reference writes past n, decoder.cu:529).
// Checks: every segment must end exactly where the next gap entry says the
// next segment starts, every codeword must exist, and the stream must yield
// at least n symbols; failures set kDevCorrupt / kDevSize, never trap.
#include <cuda_runtime.h>

#include "device_util.cuh"

namespace hgap {

template <int SEGS>
struct DecCfg {
    static constexpr int kWarps = SEGS / 32;
    static constexpr int kWords = 4 * SEGS + 8;         // staged bitstream words
    static constexpr int kStage = 33 * SEGS;            // <= 128 symbols per segment
    static constexpr int kCompact = (SEGS * 128 + 64) / 4;
    static constexpr int kTab = (int)(sizeof(DecTable) / 4);
    static constexpr size_t kSmem = (size_t)(kTab + kWords + kStage + kCompact) * 4;
};

constexpr int kDecSegs = 128;
using DecDefault = DecCfg<kDecSegs>;

__device__ __forceinline__ uint32_t gap_entry(const uint32_t* gaps, uint64_t k) {
    return (__ldg(gaps + (k >> 3)) >> (4 * (uint32_t)(k & 7))) & 0xfu;
}

template <int SEGS>
__global__ void __launch_bounds__(SEGS, 4)
    decode_kernel(const DecArgs a, const __grid_constant__ DecTable tab) {
    using C = DecCfg<SEGS>;
    extern __shared__ __align__(16) uint32_t smem[];
    const uint16_t* t1 = reinterpret_cast<const uint16_t*>(smem);
    const uint16_t* t2 = t1 + (1 << kDecPrefix);
    uint32_t* sw = smem + C::kTab;
    uint32_t* stage = sw + C::kWords;
    uint32_t* compact = stage + C::kStage;
    __shared__ uint32_t warp_tot[C::kWarps];
    __shared__ uint64_t s_tile;
    __shared__ uint64_t s_O;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&tab);
        for (int i = tid; i < C::kTab; i += SEGS) smem[i] = src[i];
        for (int i = tid; i < C::kCompact; i += SEGS) compact[i] = 0;
    }
    const uint64_t stream_bits = a.words * 32;

    for (;;) {
        if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= a.ntiles) break;
        const uint64_t s0 = tile * SEGS;
        for (int i = tid; i < C::kWords; i += SEGS) {
            const uint64_t w = 4 * s0 + i;
            sw[i] = w < a.words ? ld_stream_u32(a.bits + w) : 0u;
        }
        __syncthreads();

        // ---- 1. decode this thread's segment --------------------------------
        const uint64_t s = s0 + tid;
        uint32_t cnt = 0;
        if (s < a.segments) {
            const bool lastseg = s + 1 == a.segments;
            uint32_t pos = 128 * tid + (s ? gap_entry(a.gaps, s - 1) : 0u);
            uint32_t end = 128 * (tid + 1);
            if (lastseg && stream_bits - 128 * s0 < end) end = (uint32_t)(stream_bits - 128 * s0);
            uint32_t wi = pos >> 5;
            uint64_t win = ((((uint64_t)sw[wi]) << 32) | sw[wi + 1]) << (pos & 31);
            int avail = 64 - (int)(pos & 31);
            wi += 2;
            uint32_t packed = 0;
            bool bad = false;
            while (pos < end) {
                if (avail < 16) {
                    win |= (uint64_t)sw[wi++] << (32 - avail);
                    avail += 32;
                }
                const uint32_t x = (uint32_t)(win >> 48);
                uint32_t e = t1[x >> (16 - kDecPrefix)];
                if (e & 0x8000u) {
                    const uint32_t w = (e >> 12) & 7u;
                    e = t2[(e & 0xfffu) + ((x >> (16 - kDecPrefix - w)) & ((1u << w) - 1u))];
                }
                if (e & kDecInvalid) {
                    bad = !lastseg;  // zero padding after the final codeword may not decode
                    break;
                }
                const uint32_t len = ((e >> 8) & 15u) + 1u;
                win <<= len;
                avail -= (int)len;
                pos += len;
                packed |= (e & 0xffu) << (8 * (cnt & 3));
                ++cnt;
                if ((cnt & 3) == 0) {
                    stage[((cnt >> 2) - 1) * SEGS + tid] = packed;
                    packed = 0;
                }
            }
            if (cnt & 3) stage[(cnt >> 2) * SEGS + tid] = packed;
            if (!lastseg && !bad && pos != 128 * (tid + 1) + gap_entry(a.gaps, s)) bad = true;
            if (bad) atomicOr(a.status, kDevCorrupt);
        }

        // ---- 2. block scan of symbol counts + look-back ----------------------
        const uint32_t incl = warp_incl_scan(cnt, lane);
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t v = lane < (uint32_t)C::kWarps ? warp_tot[lane] : 0u;
            v = warp_incl_scan(v, lane);
            if (lane < (uint32_t)C::kWarps) warp_tot[lane] = v;
            const uint32_t total = __shfl_sync(kFull, v, C::kWarps - 1);
            const uint64_t O = lookback_warp(a.lookback, tile, total, a.status, lane);
            if (lane == 0) s_O = O;
        }
        __syncthreads();
        const uint32_t Ct = warp_tot[C::kWarps - 1];
        const uint64_t O = s_O;
        const uint32_t excl = incl - cnt + (warp ? warp_tot[warp - 1] : 0u);
        if (tid == 0 && tile + 1 == a.ntiles && O + Ct < a.n) atomicOr(a.status, kDevSize);

        // ---- 3. compact into the 16-byte-aligned output image, write out -----
        const uint64_t vstart = a.out_lo + O;  // virtual byte of the tile's first symbol
        const uint32_t base = (uint32_t)(vstart & 15);
        if (cnt) {
            const uint32_t d = base + excl;
            const uint32_t sh = 8 * (d & 3);
            const uint32_t dw = d >> 2;
            const uint32_t dend = d + cnt;
            const uint32_t nd = ((dend + 3) >> 2) - dw;
            const uint32_t nsrc = (cnt + 3) >> 2;
            uint32_t prev = 0;
            for (uint32_t m = 0; m < nd; ++m) {
                const uint32_t cur = m < nsrc ? stage[m * SEGS + tid] : 0u;
                const uint32_t v = sh ? ((cur << sh) | (prev >> (32 - sh))) : cur;
                prev = cur;
                const bool shared = (m == 0 && sh) || (m + 1 == nd && (dend & 3));
                if (shared) atomicOr(compact + dw + m, v);
                else compact[dw + m] = v;
            }
        }
        __syncthreads();
        if (O < a.n) {
            const uint64_t stop = (O + Ct < a.n ? O + Ct : a.n);
            const uint64_t vend = a.out_lo + stop;
            const uint64_t q0 = vstart >> 4;
            const uint64_t q1 = (vend + 15) >> 4;
            for (uint64_t q = q0 + tid; q < q1; q += SEGS) {
                const uint32_t lq = (uint32_t)(q - q0);
                const uint64_t c0 = q << 4;
                if (c0 >= vstart && c0 + 16 <= vend) {
                    const uint4 v = reinterpret_cast<const uint4*>(compact)[lq];
                    *reinterpret_cast<uint4*>(a.out_aligned + c0) = v;
                } else {
                    const uint8_t* cb = reinterpret_cast<const uint8_t*>(compact) + 16 * lq;
                    for (uint32_t b = 0; b < 16; ++b) {
                        const uint64_t vb = c0 + b;
                        if (vb >= vstart && vb < vend) a.out_aligned[vb] = cb[b];
                    }
                }
            }
        }
        __syncthreads();
        const uint32_t used = (base + Ct + 3) / 4 + 1;
        for (uint32_t i = tid; i < used && i < (uint32_t)C::kCompact; i += SEGS) compact[i] = 0;
    }
}

uint64_t decode_tiles(uint64_t segments) { return (segments + kDecSegs - 1) / kDecSegs; }

int launch_decode(const DecArgs& a, const DecTable& t, void* stream) {
    auto kern = decode_kernel<kDecSegs>;
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)DecDefault::kSmem);
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kDecSegs, DecDefault::kSmem);
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t cap = (uint64_t)sms * per_sm;
    const unsigned grid = (unsigned)(a.ntiles < cap ? a.ntiles : cap);
    kern<<<grid, kDecSegs, DecDefault::kSmem, static_cast<cudaStream_t>(stream)>>>(a, t);
    return cudaGetLastError();
}

}  // namespace hgap
