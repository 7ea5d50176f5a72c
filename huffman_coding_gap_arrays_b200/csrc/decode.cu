// decode.cu -- segment-parallel Huffman decoder driven by the gap array, sm_100a.
//
// Replaces gpu_dec_l1_l2 (decoder/src/decoder.cu:454-730).  Same unit of
// parallelism -- a 128-bit segment that starts at its gap offset -- but each
// segment is decoded ONCE (the reference decodes it twice: a counting pass,
// then a writing pass, decoder.cu:529-569,672-725):
//   1. a persistent CTA of 256 threads takes the next tile of 512 segments,
//      stages its bitstream words in shared memory (padded one word in eight
//      so the threads' windows, 4 words apart, fall in different banks) and
//      every thread decodes TWO segments interleaved (two independent
//      dependency chains) through a shared-memory two-level table, parking the
//      symbols in a column-major shared area sized for the book's shortest
//      code (a segment holds at most ceil(128 / shortest length) symbols);
//   2. block scan of the 512 symbol counts + one bounded decoupled look-back
//      with a 256-tile window gives the tile's output offset;
//   3. the symbols are compacted into a shared image of the output at its
//      16-byte alignment and written with 16-byte coalesced stores (byte
//      stores only on the two ragged edges), clipped at exactly n bytes (the
//      reference writes past n, decoder.cu:529).
// Checks: every segment must end exactly where the next gap entry says the
// next segment starts, every codeword must exist, and the stream must yield at
// least n symbols; failures set kDevCorrupt / kDevSize, never trap.
#include <cuda_runtime.h>

#include "device_util.cuh"

namespace hgap {

constexpr int kDecThreads = 256;
constexpr int kDecSegs = 512;   // segments per tile: two per thread
constexpr int kDecLookK = 8;    // look-back window = 32 * 8 tiles

template <int R>  // stage rows of 4 symbols per segment: at most 4R symbols per segment
struct DecCfg {
    static constexpr int kMaxSym = 4 * R;
    static constexpr int kWarps = kDecThreads / 32;
    static constexpr int kT1 = 1 << kDecPrefix;        // u32 level-1 entries
    static constexpr int kT2 = kDecT2Cap;              // u32 level-2 entries
    static constexpr int kWords = 4 * kDecSegs + 8;
    static constexpr int kWordsPad = (kWords + kWords / 8 + 8 + 3) & ~3;
    static constexpr int kStage = kDecSegs * R;        // words: bytes [row][segment]
    static constexpr int kCompact = (kDecSegs * kMaxSym + 64) / 4;
    static constexpr size_t kSmem = (size_t)(kT1 + kT2 + kWordsPad + kStage + kCompact) * 4;
    static_assert(kT1 % 4 == 0 && kT2 % 4 == 0 && kWordsPad % 4 == 0 && kStage % 4 == 0,
                  "16-byte aligned areas");
};

// Shared-memory table entry (u32): direct = len << 8 | symbol; pointer =
// bit 31 | extra width << 16 | level-2 offset; invalid = bit 30.
__device__ __forceinline__ uint32_t widen_entry(uint32_t e) {
    if (e & 0x8000u) return 0x80000000u | (((e >> 12) & 7u) << 16) | (e & 0xfffu);
    if (e & kDecInvalid) return 0x40000000u;
    return ((((e >> 8) & 15u) + 1u) << 8) | (e & 0xffu);
}

__device__ __forceinline__ uint32_t pidx(uint32_t w) { return w + (w >> 3); }

__device__ __forceinline__ uint32_t gap_entry(const uint32_t* gaps, uint64_t k) {
    return (__ldg(gaps + (k >> 3)) >> (4 * (uint32_t)(k & 7))) & 0xfu;
}

template <int R>
__global__ void __launch_bounds__(kDecThreads, 3)
    decode_kernel(const DecArgs a, const __grid_constant__ DecTable tab) {
    using C = DecCfg<R>;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* t1 = smem;
    uint32_t* t2 = t1 + C::kT1;
    uint32_t* sw = t2 + C::kT2;
    uint8_t* stage = reinterpret_cast<uint8_t*>(sw + C::kWordsPad);
    uint32_t* compact = sw + C::kWordsPad + C::kStage;
    __shared__ uint32_t warp_tot[C::kWarps];
    __shared__ uint64_t s_tile;
    __shared__ uint64_t s_O;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < C::kT1; i += kDecThreads) t1[i] = widen_entry(tab.t1[i]);
    for (int i = tid; i < C::kT2; i += kDecThreads) t2[i] = widen_entry(tab.t2[i]);
    for (int i = tid; i < C::kCompact; i += kDecThreads) compact[i] = 0;
    const uint64_t stream_bits = a.words * 32;

    for (;;) {
        if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= a.ntiles) break;
        const uint64_t s0 = tile * kDecSegs;
        for (uint32_t i = tid; i < (uint32_t)C::kWords; i += kDecThreads) {
            const uint64_t w = 4 * s0 + i;
            sw[pidx(i)] = w < a.words ? ld_stream_u32(a.bits + w) : 0u;
        }
        __syncthreads();

        // ---- 1. decode segments tid and tid + 256 ---------------------------
        uint32_t cnt[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t col = tid + k * kDecThreads;
            const uint64_t s = s0 + col;
            uint32_t n = 0;
            if (s < a.segments) {
                const bool last = s + 1 == a.segments;
                uint32_t pos = 128 * col + (s ? gap_entry(a.gaps, s - 1) : 0u);
                uint32_t end = 128 * col + 128;
                if (last && stream_bits - 128 * s0 < end) end = (uint32_t)(stream_bits - 128 * s0);
                bool bad = false;
                uint8_t* out = stage + col;
                while (pos < end) {
                    const uint32_t w = pos >> 5;
                    const uint32_t x = __funnelshift_l(sw[pidx(w + 1)], sw[pidx(w)], pos);
                    uint32_t e = t1[x >> (32 - kDecPrefix)];
                    if (e & 0x80000000u) {  // longer than the prefix: level 2
                        const uint32_t wd = (e >> 16) & 7u;
                        e = t2[(e & 0xffffu) + ((x << kDecPrefix) >> (32 - wd))];
                    }
                    if ((e & 0x40000000u) || n >= (uint32_t)C::kMaxSym) {
                        bad = !last;  // zero padding after the final codeword may not decode
                        break;
                    }
                    pos += (e >> 8) & 31u;
                    *out = (uint8_t)e;
                    out += kDecSegs;
                    ++n;
                }
                if (!last && !bad && pos != 128 * col + 128 + gap_entry(a.gaps, s)) bad = true;
                if (bad) atomicOr(a.status, kDevCorrupt);
            }
            cnt[k] = n;
        }

        // ---- 2. scan of the 512 counts (segments 0..255 are k = 0, 256..511 k = 1)
        const uint32_t i0 = warp_incl_scan(cnt[0], lane);
        const uint32_t i1 = warp_incl_scan(cnt[1], lane);
        if (lane == 31) warp_tot[warp] = i0 | (i1 << 16);  // a warp's 32 segments: < 2^13 symbols
        __syncthreads();
        uint32_t wt = lane < (uint32_t)C::kWarps ? warp_tot[lane] : 0u;
        uint32_t w0 = wt & 0xffffu, w1 = wt >> 16;
        w0 = warp_incl_scan(w0, lane);
        w1 = warp_incl_scan(w1, lane);
        const uint32_t total0 = __shfl_sync(kFull, w0, C::kWarps - 1);
        const uint32_t total1 = __shfl_sync(kFull, w1, C::kWarps - 1);
        const uint32_t before0 = warp ? __shfl_sync(kFull, w0, warp - 1) : 0u;
        const uint32_t before1 = warp ? __shfl_sync(kFull, w1, warp - 1) : 0u;
        const uint32_t Ct = total0 + total1;
        const uint32_t excl0 = before0 + i0 - cnt[0];
        const uint32_t excl1 = total0 + before1 + i1 - cnt[1];
        if (warp == 0) {
            const uint64_t O = lookback_warp_wide<kDecLookK>(a.lookback, tile, Ct, a.status, lane);
            if (lane == 0) s_O = O;
        }
        __syncthreads();
        const uint64_t O = s_O;
        if (tid == 0 && tile + 1 == a.ntiles && O + Ct < a.n) atomicOr(a.status, kDevSize);

        // ---- 3. compact into the 16-byte-aligned output image, write out -----
        const uint64_t vstart = a.out_lo + O;
        const uint32_t base = (uint32_t)(vstart & 15);
        uint8_t* cbytes = reinterpret_cast<uint8_t*>(compact);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint8_t* src = stage + tid + k * kDecThreads;
            uint8_t* dst = cbytes + base + (k ? excl1 : excl0);
            for (uint32_t j = 0; j < cnt[k]; ++j) dst[j] = src[j * kDecSegs];
        }
        __syncthreads();
        if (O < a.n) {
            const uint64_t stop = (O + Ct < a.n ? O + Ct : a.n);
            const uint64_t vend = a.out_lo + stop;
            const uint64_t q0 = vstart >> 4;
            const uint64_t q1 = (vend + 15) >> 4;
            for (uint64_t q = q0 + tid; q < q1; q += kDecThreads) {
                const uint32_t lq = (uint32_t)(q - q0);
                const uint64_t c0 = q << 4;
                if (c0 >= vstart && c0 + 16 <= vend) {
                    const uint4 v = reinterpret_cast<const uint4*>(compact)[lq];
                    *reinterpret_cast<uint4*>(a.out_aligned + c0) = v;
                } else {
                    const uint8_t* cb = cbytes + 16 * lq;
                    for (uint32_t b = 0; b < 16; ++b) {
                        const uint64_t vb = c0 + b;
                        if (vb >= vstart && vb < vend) a.out_aligned[vb] = cb[b];
                    }
                }
            }
        }
        __syncthreads();
    }
}

uint64_t decode_tiles(uint64_t segments) { return (segments + kDecSegs - 1) / kDecSegs; }

template <int R>
static int launch_decode_r(const DecArgs& a, const DecTable& t, cudaStream_t st) {
    using C = DecCfg<R>;
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaFuncSetAttribute(decode_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)C::kSmem);
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decode_kernel<R>, kDecThreads, C::kSmem);
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t cap = (uint64_t)sms * per_sm;
    const unsigned grid = (unsigned)(a.ntiles < cap ? a.ntiles : cap);
    decode_kernel<R><<<grid, kDecThreads, C::kSmem, st>>>(a, t);
    return cudaGetLastError();
}

// min_len: shortest code length of the book.  A segment holds at most
// ceil(128 / min_len) codeword starts; the stage is sized for that.
int launch_decode(const DecArgs& a, const DecTable& t, uint32_t min_len, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t max_sym = (128 + min_len - 1) / (min_len ? min_len : 1);
    if (max_sym <= 32) return launch_decode_r<8>(a, t, st);
    if (max_sym <= 44) return launch_decode_r<11>(a, t, st);
    if (max_sym <= 64) return launch_decode_r<16>(a, t, st);
    return launch_decode_r<32>(a, t, st);
}

}  // namespace hgap
