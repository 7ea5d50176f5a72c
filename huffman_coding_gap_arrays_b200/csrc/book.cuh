// book.cuh -- codebook construction on the device, one warp per book.
//
// Replaces the host round trip of store_symbols + qsort + boundary_PM +
// canonical code assignment (encoder/src/symbols.cpp:29-55,
// encoder/src/huff.cpp:17-21, encoder/src/package_merge.cpp:107-182) and the
// decoder's table build (decoder/src/get_table.cpp:48-139), so that batched
// and serving callers build thousands of books without leaving the GPU.  The
// results are identical to the host builder's (host.cpp): the same stable
// order by count, the same package-merge tie rule, the same canonical codes
// and the same two-level decoder table.
//
//   * sort: bitonic sort of (count << 8 | byte) keys, so equal counts keep
//     byte order (what the reference's qsort yields on glibc);
//   * package-merge, L = 16: level l merges the sorted leaves with the pairwise
//     packages of level l-1 (a package first on equal weight), keeping 2n-2
//     items; each level is one merge-path step -- every lane finds where its
//     16 outputs start by a binary search on its diagonal, then merges them;
//     a 16-bit mask per lane records which items are packages;
//   * lengths: walking down from level 16, the packages in a level's active
//     prefix make the next level's active prefix twice as long; a leaf's
//     length is the number of levels whose active prefix holds it;
//   * canonical codes: in container order (most frequent first) the code of
//     symbol i is the Kraft prefix sum before it, in units of 2^-16, shifted
//     down to its length -- the closed form of code = (code + 1) << (l' - l)
//     (encoder/src/package_merge.cpp:168-181);
//   * decoder table: every level-1 prefix, and every level-2 suffix of a
//     prefix whose codes are longer than kDecPrefix bits, looks up the
//     symbol whose left-aligned code is the largest not above it (canonical
//     codes ascend in container order); the lane walks its 64 prefixes in
//     order, so the search is a forward scan.
#pragma once

#include "device_util.cuh"

namespace hgap {

// The package-merge lanes read items 16 apart (weights) and about 8 apart
// (leaves): unpadded, a whole warp's 8-byte reads land in one bank pair (the
// capture of one-warp-per-book showed two thirds of its shared wavefronts were
// conflicts).  One pad slot per 16 weights and per 8 keys spreads them.
__device__ __forceinline__ uint32_t wpad(uint32_t i) { return i + (i >> 4); }
__device__ __forceinline__ uint32_t kpad(uint32_t i) { return i + (i >> 3); }

struct BookScratch {
    uint64_t w[2][512 + 32];      // weights of two consecutive package-merge levels (at wpad)
    uint64_t key[256 + 32];       // count << 8 | byte, ~0 for absent bytes; sorted in place (at kpad)
    uint16_t pk[kMaxLen + 1][32]; // bit b of pk[l][q]: item 16q+b of level l is a package
    uint16_t size[kMaxLen + 1];   // items kept at each level
    uint32_t la[256];             // container order: code << (16 - length)
    uint8_t len[256];             // ascending-count order: code lengths
    uint8_t sym[256];             // container order: bytes
    uint8_t clen[256];            // container order: lengths
    uint8_t blen[256];            // per byte: code length (0: absent)
};

__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, uint32_t lane, uint32_t* total) {
    const uint32_t incl = warp_incl_scan(v, lane);
    *total = __shfl_sync(kFull, incl, 31);
    return incl - v;
}

// Fills s.key (sorted) and s.len for the present bytes of `hist` and returns
// their number n.  Leaf r (ascending count, ties by byte) is s.key[kpad(r)].
__device__ inline uint32_t warp_code_lengths(const uint32_t* hist, BookScratch& s, uint32_t lane) {
    uint32_t n = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t b = lane + 32 * j;
        const uint32_t h = hist[b];
        s.key[kpad(b)] = h ? (((uint64_t)h << 8) | b) : ~0ull;
        n += __popc(__ballot_sync(kFull, h != 0));
    }
    __syncwarp();
    // bitonic sort, ascending; absent bytes (~0) sink to the end
    for (uint32_t k = 2; k <= 256; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (uint32_t t = lane; t < 128; t += 32) {
                const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const uint32_t p = i + j;
                const uint64_t x = s.key[kpad(i)], y = s.key[kpad(p)];
                if ((x > y) == ((i & k) == 0)) {
                    s.key[kpad(i)] = y;
                    s.key[kpad(p)] = x;
                }
            }
            __syncwarp();
        }
    }
    if (n == 1) {
        if (lane == 0) s.len[0] = 1;  // one symbol: a 1-bit code (the reference is undefined here)
        __syncwarp();
        return n;
    }
    if (n < 2) return n;

    const uint32_t keep = 2 * n - 2;
    for (uint32_t r = lane; r < 512; r += 32) s.w[0][wpad(r)] = r < n ? (s.key[kpad(r)] >> 8) : 0;
    s.pk[1][lane] = 0;
    if (lane == 0) s.size[1] = (uint16_t)n;
    __syncwarp();
    uint32_t prev_size = n;
    int cur = 0;
    for (int l = 2; l <= kMaxLen; ++l) {
        const uint64_t* below = s.w[cur];
        uint64_t* out = s.w[cur ^ 1];
        const uint32_t np = prev_size / 2;
        const uint32_t m = keep < n + np ? keep : n + np;
        const uint32_t d = 16 * lane;
        uint32_t mask = 0;
        if (d < m) {
            // leaves among the first d items: leaf i precedes package j iff w(leaf i) < w(package j)
            uint32_t lo = d > np ? d - np : 0, hi = d < n ? d : n;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                const uint32_t jj = d - mid - 1;
                if ((s.key[kpad(mid)] >> 8) < below[wpad(2 * jj)] + below[wpad(2 * jj + 1)]) lo = mid + 1;
                else hi = mid;
            }
            uint32_t i = lo, j = d - lo;
            const uint32_t e = d + 16 < m ? d + 16 : m;
            for (uint32_t pos = d; pos < e; ++pos) {
                const uint64_t pw = j < np ? below[wpad(2 * j)] + below[wpad(2 * j + 1)] : 0;
                if (j < np && (i >= n || pw <= (s.key[kpad(i)] >> 8))) {
                    out[wpad(pos)] = pw;
                    mask |= 1u << (pos - d);
                    ++j;
                } else {
                    out[wpad(pos)] = s.key[kpad(i)] >> 8;
                    ++i;
                }
            }
        }
        s.pk[l][lane] = (uint16_t)mask;
        if (lane == 0) s.size[l] = (uint16_t)m;
        prev_size = m;
        cur ^= 1;
        __syncwarp();
    }
    // walk down: leaves in each level's active prefix gain one bit
    uint32_t nleaf[kMaxLen + 1];
    uint32_t active = keep;
#pragma unroll
    for (int l = kMaxLen; l >= 1; --l) {
        const uint32_t a = active < s.size[l] ? active : s.size[l];
        const uint32_t q = a >> 4, rb = a & 15;
        uint32_t c = 0;
        if (lane < q) c = __popc(s.pk[l][lane]);
        else if (lane == q && rb) c = __popc(s.pk[l][lane] & ((1u << rb) - 1u));
        c = __reduce_add_sync(kFull, c);
        nleaf[l] = a - c;
        active = 2 * c;
    }
    for (uint32_t r = lane; r < n; r += 32) {
        uint32_t L = 0;
#pragma unroll
        for (int l = 1; l <= kMaxLen; ++l) L += nleaf[l] > r;
        s.len[r] = (uint8_t)L;
    }
    __syncwarp();
    return n;
}

// Container order from ascending order (symbol i = leaf n-1-i) and the
// canonical codes, into s.sym / s.clen / s.la, plus the per-byte lengths
// s.blen.  Returns the Kraft sum in units of 2^-16 (65536: a complete book).
__device__ inline uint32_t warp_assign_codes(BookScratch& s, uint32_t n, uint32_t lane) {
    for (uint32_t b = lane; b < 256; b += 32) s.blen[b] = 0;
    __syncwarp();
    uint32_t kr[8], tot = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const uint32_t c = 8 * lane + t;
        kr[t] = 0;
        if (c < n) {
            const uint32_t r = n - 1 - c;
            const uint32_t L = s.len[r];
            const uint32_t sym = (uint32_t)(s.key[kpad(r)] & 0xff);
            s.sym[c] = (uint8_t)sym;
            s.clen[c] = (uint8_t)L;
            s.blen[sym] = (uint8_t)L;
            kr[t] = 1u << (kMaxLen - L);
        }
        tot += kr[t];
    }
    uint32_t kraft = 0;
    uint32_t run = warp_excl_scan(tot, lane, &kraft);
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const uint32_t c = 8 * lane + t;
        if (c < n) s.la[c] = run;
        run += kr[t];
    }
    __syncwarp();
    return kraft;
}

// The book in the public layout (symbols in container order, per-byte table).
__device__ inline void warp_write_book(const BookScratch& s, uint32_t n, hgap_codebook* cb, uint32_t lane) {
    for (uint32_t b = lane; b < 256; b += 32) {
        cb->table[b].code = 0;
        cb->table[b].length = 0;
    }
    __syncwarp();
    for (uint32_t c = lane; c < n; c += 32) {
        const uint32_t L = s.clen[c], sym = s.sym[c];
        cb->symbols[c].symbol = (uint8_t)sym;
        cb->symbols[c].length = (uint8_t)L;
        cb->table[sym].code = s.la[c] >> (kMaxLen - L);
        cb->table[sym].length = L;
    }
    if (lane == 0) cb->symbol_count = n;
    __syncwarp();
}

// The encoder's per-byte table (code | length << 16, kEncAbsent if absent).
__device__ inline void warp_write_enc_table(const BookScratch& s, uint32_t n, EncTable* t, uint32_t lane) {
    for (uint32_t b = lane; b < 256; b += 32) t->e[b] = kEncAbsent;
    __syncwarp();
    for (uint32_t c = lane; c < n; c += 32) {
        const uint32_t L = s.clen[c];
        t->e[s.sym[c]] = (s.la[c] >> (kMaxLen - L)) | (L << 16);
    }
    __syncwarp();
}

// The same container-order arrays from a given symbol list (decoder side).
// Returns the Kraft sum, or ~0u if the list is not a valid canonical book
// (a length outside 1..16, a repeated byte, lengths not ascending, Kraft > 1).
__device__ inline uint32_t warp_load_symbols(const hgap_symlen* syms, uint32_t n, BookScratch& s, uint32_t lane) {
    uint32_t kr[8], tot = 0;
    bool bad = n > 256;
    if (lane < 8) s.key[lane] = 0;  // byte-seen bitmap: 256 bits in key[0..3]
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const uint32_t c = 8 * lane + t;
        kr[t] = 0;
        if (c < n && c < 256) {
            const uint32_t L = syms[c].length, sym = syms[c].symbol;
            s.sym[c] = (uint8_t)sym;
            s.clen[c] = (uint8_t)L;
            if (L < 1 || L > (uint32_t)kMaxLen) bad = true;
            else kr[t] = 1u << (kMaxLen - L);
            const unsigned long long bit = 1ull << (sym & 63);
            if (atomicOr(reinterpret_cast<unsigned long long*>(&s.key[sym >> 6]), bit) & bit) bad = true;
        }
        tot += kr[t];
    }
    __syncwarp();
    for (uint32_t c = lane; c + 1 < n && c + 1 < 256; c += 32)
        if (s.clen[c + 1] < s.clen[c]) bad = true;
    uint32_t kraft = 0;
    uint32_t run = warp_excl_scan(tot, lane, &kraft);
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const uint32_t c = 8 * lane + t;
        if (c < n && c < 256) s.la[c] = run;
        run += kr[t];
    }
    if (kraft > (1u << kMaxLen)) bad = true;
    bad = __any_sync(kFull, bad);
    __syncwarp();
    return bad ? ~0u : kraft;
}

// Decoder table (layout in hgap_internal.h) from the container-order arrays
// s.la / s.sym / s.clen of n >= 1 symbols.  Returns false if the level-2 part
// would exceed kDecT2Cap (only possible for an incomplete book).
__device__ inline bool warp_dec_table(const BookScratch& s, uint32_t n, DecTable* t, uint32_t lane) {
    constexpr uint32_t P = kDecPrefix, X = kMaxLen - kDecPrefix;  // 11, 5
    // symbol index of the largest left-aligned code <= v, starting from i
    auto advance = [&](uint32_t i, uint32_t v) {
        while (i + 1 < n && s.la[i + 1] <= v) ++i;
        return i;
    };
    auto entry = [&](uint32_t i, uint32_t v) -> uint16_t {
        const uint32_t L = s.clen[i];
        if (v < s.la[i] || v - s.la[i] >= (1u << (kMaxLen - L))) return kDecInvalid;
        return (uint16_t)(((L - 1) << 8) | s.sym[i]);
    };
    const uint32_t x0 = 64 * lane;
    // first pass: widths of this lane's pointer prefixes, for the level-2 offsets
    uint32_t i_last = 0, span = 0;
    for (uint32_t k = 0; k < 64; ++k) {
        const uint32_t x = x0 + k;
        i_last = advance(i_last, (x << X) | ((1u << X) - 1));
        const uint32_t L = s.clen[i_last];
        if (L > P && (s.la[i_last] >> X) == x) span += 1u << (L - P);
    }
    uint32_t total = 0;
    uint32_t off = warp_excl_scan(span, lane, &total);
    if (total > (uint32_t)kDecT2Cap) return false;
    for (uint32_t k = lane; k < (uint32_t)kDecT2Cap; k += 32) t->t2[k] = kDecInvalid;
    __syncwarp();  // cleared before any lane fills its level-2 groups
    uint32_t i_first = 0;
    i_last = 0;
    for (uint32_t k = 0; k < 64; ++k) {
        const uint32_t x = x0 + k;
        const uint32_t v = x << X;
        i_first = advance(i_first, v);
        i_last = advance(i_last, v | ((1u << X) - 1));
        const uint32_t L = s.clen[i_last];
        if (L > P && (s.la[i_last] >> X) == x) {
            const uint32_t w = L - P;
            t->t1[x] = (uint16_t)(0x8000u | (w << 12) | off);
            uint32_t i = i_first;
            for (uint32_t y = 0; y < (1u << w); ++y) {
                const uint32_t vy = v | (y << (X - w));
                i = advance(i, vy);
                t->t2[off + y] = entry(i, vy);
            }
            off += 1u << w;
        } else {
            t->t1[x] = entry(i_first, v);
        }
    }
    __syncwarp();
    return true;
}

}  // namespace hgap
