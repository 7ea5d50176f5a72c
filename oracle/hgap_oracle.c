/*
 * hgap_oracle.c -- CPU oracle for Huffman coding with gap arrays.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library (loaded by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by
 * the product).  It restates the reference algorithm in plain C; each
 * function names the reference file:line it follows.  Parity of this
 * restatement is pinned against the reference's own host sources compiled
 * into oracle/_ref and against golden containers written by the reference's
 * GPU encoder (tests/golden/).
 */
#include "hgap_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* histogram                                                                 */
/* ------------------------------------------------------------------------ */

/* encoder/src/symbols.cpp:18-27 (byte-wise count; the GPU version
 * encoder/src/encoder.cu:33-116 counts the same bytes of little-endian words). */
void orc_histogram(const uint8_t* in, uint64_t n, uint32_t hist[256]) {
    memset(hist, 0, 256 * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; ++i) hist[in[i]]++;
}

/* ------------------------------------------------------------------------ */
/* codebook                                                                  */
/* ------------------------------------------------------------------------ */

/* store_symbols (encoder/src/symbols.cpp:29-43) lists non-zero bins in byte
 * order; qsort with `compare` (encoder/src/huff.cpp:17-21) orders them by
 * ascending count.  glibc's qsort is a stable merge sort at this size, so
 * ties keep byte order: a stable insertion sort reproduces it. */
static int sort_symbols(const uint32_t hist[256], orc_symbol out[256]) {
    int count = 0;
    for (int b = 0; b < 256; ++b) {
        if (hist[b] == 0) continue;
        orc_symbol s;
        s.symbol = (uint8_t)b;
        s.length = 0;
        s.count = hist[b];
        int j = count++;
        while (j > 0 && out[j - 1].count > s.count) {
            out[j] = out[j - 1];
            --j;
        }
        out[j] = s;
    }
    return count;
}

/* Length-limited code lengths by package-merge, limit ORC_MAX_LEN.
 * The reference runs the lazy "boundary" form of the algorithm
 * (encoder/src/package_merge.cpp:12-80,107-166); this is the plain
 * list form, which selects the same items.  Tie rule, taken from
 * package_merge.cpp:37,52,136: a package goes before a leaf of equal weight.
 * Level 1 holds the leaves; level l > 1 merges the leaves with the pairs of
 * level l-1; the top level keeps its first 2n-2 items, and a leaf's length is
 * the number of levels whose active prefix contains it
 * (package_merge.cpp:152-159). */
static void package_merge(const orc_symbol* s, int n, uint8_t* lens) {
    const int keep = 2 * n - 2;
    uint64_t* w[ORC_MAX_LEN + 1];
    uint8_t* pkg[ORC_MAX_LEN + 1];
    int cnt[ORC_MAX_LEN + 1];
    for (int l = 1; l <= ORC_MAX_LEN; ++l) {
        w[l] = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(2 * n));
        pkg[l] = (uint8_t*)malloc((size_t)(2 * n));
    }
    for (int i = 0; i < n; ++i) {
        w[1][i] = s[i].count;
        pkg[1][i] = 0;
    }
    cnt[1] = n;
    for (int l = 2; l <= ORC_MAX_LEN; ++l) {
        const int np = cnt[l - 1] / 2;
        int li = 0, pi = 0, k = 0;
        while (k < keep && (li < n || pi < np)) {
            uint64_t pw = 0;
            if (pi < np) pw = w[l - 1][2 * pi] + w[l - 1][2 * pi + 1];
            if (pi < np && (li >= n || pw <= (uint64_t)s[li].count)) {
                w[l][k] = pw;
                pkg[l][k] = 1;
                ++pi;
            } else {
                w[l][k] = s[li].count;
                pkg[l][k] = 0;
                ++li;
            }
            ++k;
        }
        cnt[l] = k;
    }
    memset(lens, 0, (size_t)n);
    int active = keep;
    for (int l = ORC_MAX_LEN; l >= 1 && active > 0; --l) {
        int leaves = 0, packs = 0;
        for (int k = 0; k < active && k < cnt[l]; ++k) {
            if (pkg[l][k]) ++packs;
            else ++leaves;
        }
        for (int i = 0; i < leaves; ++i) lens[i]++;
        active = 2 * packs;
    }
    for (int l = 1; l <= ORC_MAX_LEN; ++l) {
        free(w[l]);
        free(pkg[l]);
    }
}

/* Canonical codes from the most frequent symbol down
 * (encoder/src/package_merge.cpp:168-181):
 * code_{next} = (code + 1) << (len_next - len). */
void orc_canonical_codes(const uint8_t* symbols, const uint8_t* lengths, int count,
                         uint32_t code[256], uint32_t len[256]) {
    memset(code, 0, 256 * sizeof(uint32_t));
    memset(len, 0, 256 * sizeof(uint32_t));
    uint32_t c = 0;
    for (int i = 0; i < count; ++i) {
        const uint32_t l = lengths[i];
        code[symbols[i]] = c;
        len[symbols[i]] = l;
        const uint32_t nl = (i + 1 < count) ? lengths[i + 1] : l;
        c = (c + 1) << (nl - l);
    }
}

int orc_codebook(const uint32_t hist[256], orc_symbol sorted[256], uint32_t code[256],
                 uint32_t len[256]) {
    const int n = sort_symbols(hist, sorted);
    memset(code, 0, 256 * sizeof(uint32_t));
    memset(len, 0, 256 * sizeof(uint32_t));
    if (n == 0) return 0;
    if (n == 1) {
        /* defined here (reference: undefined behaviour, package_merge.cpp:113-132) */
        sorted[0].length = 1;
        len[sorted[0].symbol] = 1;
        code[sorted[0].symbol] = 0;
        return 1;
    }
    uint8_t lens[256];
    package_merge(sorted, n, lens);
    for (int i = 0; i < n; ++i) sorted[i].length = lens[i];
    /* container order is the sorted array walked backwards (huff.cpp:114) */
    uint8_t syms_c[256], lens_c[256];
    for (int i = 0; i < n; ++i) {
        syms_c[i] = sorted[n - 1 - i].symbol;
        lens_c[i] = sorted[n - 1 - i].length;
    }
    orc_canonical_codes(syms_c, lens_c, n, code, len);
    return n;
}

orc_sizes orc_sizes_from_bits(uint64_t bits) {
    orc_sizes z;
    z.bits = bits;
    z.words = (bits + 31) / 32;
    z.segments = (bits + ORC_SEGMENT - 1) / ORC_SEGMENT;
    z.gap_words = (z.segments + ORC_GAPS_PER_WORD - 1) / ORC_GAPS_PER_WORD;
    return z;
}

/* get_outputfilesize (encoder/src/symbols.cpp:45-55), in 64-bit arithmetic. */
orc_sizes orc_sizes_for(const orc_symbol* sorted, int count) {
    uint64_t bits = 0;
    for (int i = 0; i < count; ++i) bits += (uint64_t)sorted[i].length * sorted[i].count;
    return orc_sizes_from_bits(bits);
}

/* ------------------------------------------------------------------------ */
/* encoder                                                                   */
/* ------------------------------------------------------------------------ */

/* Codes are packed MSB-first into u32 words, bit b of the stream at bit
 * (31 - b%32) of word b/32; the last word is zero-padded
 * (encoder/src/encoder.cu:314-347).  For the code that crosses or ends at
 * bit 128(k+1), gap[k] = end - 128(k+1) in [0,15]
 * (encoder/src/encoder.cu:307-312); gap[k] goes to nibble k%8 of gap word
 * k/8, low nibble first (encoder/src/encoder.cu:371-374). */
uint64_t orc_encode_chunk(const uint8_t* in, uint64_t n, const uint32_t code[256],
                          const uint32_t len[256], uint64_t first_bit, uint32_t* bits,
                          uint32_t* gaps) {
    uint64_t pos = first_bit;
    uint64_t word = first_bit / 32;
    uint64_t acc = 0;
    uint32_t nb = (uint32_t)(first_bit % 32);
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t l = len[in[i]];
        const uint32_t c = code[in[i]];
        acc = (acc << l) | c;
        nb += l;
        const uint64_t end = pos + l;
        if (end / ORC_SEGMENT != pos / ORC_SEGMENT) {
            const uint64_t k = end / ORC_SEGMENT - 1;
            gaps[k / 8] |= (uint32_t)(end % ORC_SEGMENT) << (4 * (k % 8));
        }
        pos = end;
        if (nb >= 32) {
            bits[word++] |= (uint32_t)(acc >> (nb - 32));
            nb -= 32;
        }
    }
    if (nb > 0) bits[word] |= (uint32_t)(acc << (32 - nb));
    return pos - first_bit;
}

int orc_encode(const uint8_t* in, uint64_t n, const uint32_t code[256], const uint32_t len[256],
               uint32_t* bits, uint64_t words, uint32_t* gaps, uint64_t gap_words,
               uint64_t* bits_out) {
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (len[in[i]] == 0) return -1; /* byte without a codeword */
        total += len[in[i]];
    }
    const orc_sizes z = orc_sizes_from_bits(total);
    if (z.words != words || z.gap_words != gap_words) return -2;
    memset(bits, 0, words * sizeof(uint32_t));
    memset(gaps, 0, gap_words * sizeof(uint32_t));
    orc_encode_chunk(in, n, code, len, 0, bits, gaps);
    if (bits_out) *bits_out = total;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* decoder                                                                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint32_t first[ORC_MAX_LEN + 2]; /* first canonical code of each length */
    uint32_t count[ORC_MAX_LEN + 2];
    uint32_t base[ORC_MAX_LEN + 2];  /* index of that code in the list */
    const uint8_t* symbols;
} canon_t;

static int canon_init(canon_t* t, const uint8_t* symbols, const uint8_t* lengths, int count) {
    memset(t, 0, sizeof(*t));
    t->symbols = symbols;
    for (int i = 0; i < count; ++i) {
        if (lengths[i] < 1 || lengths[i] > ORC_MAX_LEN) return -1;
        if (i > 0 && lengths[i] < lengths[i - 1]) return -1;
        t->count[lengths[i]]++;
    }
    uint32_t c = 0, idx = 0;
    for (int l = 1; l <= ORC_MAX_LEN; ++l) {
        t->first[l] = c;
        t->base[l] = idx;
        idx += t->count[l];
        c = (c + t->count[l]) << 1;
    }
    return 0;
}

static inline uint32_t get_bit(const uint32_t* bits, uint64_t words, uint64_t pos) {
    const uint64_t w = pos >> 5;
    if (w >= words) return 0;
    return (bits[w] >> (31 - (pos & 31))) & 1u;
}

/* One codeword at `pos`; returns its length, 0 if no codeword matches. */
static inline uint32_t decode_one(const canon_t* t, const uint32_t* bits, uint64_t words,
                                  uint64_t pos, uint8_t* sym) {
    uint32_t c = 0;
    for (uint32_t l = 1; l <= ORC_MAX_LEN; ++l) {
        c = (c << 1) | get_bit(bits, words, pos + l - 1);
        const uint32_t d = c - t->first[l];
        if (t->count[l] && d < t->count[l]) {
            *sym = t->symbols[t->base[l] + d];
            return l;
        }
    }
    return 0;
}

static inline uint32_t gap_of(const uint32_t* gaps, uint64_t k) {
    return (gaps[k / 8] >> (4 * (k % 8))) & 0xFu;
}

/* gpu_dec_l1_l2 (decoder/src/decoder.cu:501-569): segment s starts at bit
 * 128s + gap[s-1] (0 for s = 0) and decodes every codeword that starts
 * before 128(s+1).  Checked here: the last codeword of segment s ends at
 * 128(s+1) + gap[s]; the stream stops at exactly n symbols. */
int orc_decode(const uint32_t* bits, uint64_t words, const uint32_t* gaps, uint64_t segments,
               const uint8_t* symbols, const uint8_t* lengths, int count, uint8_t* out,
               uint64_t n) {
    canon_t t;
    if (n == 0) return (words == 0 && segments == 0) ? 0 : -1;
    if (count < 1 || canon_init(&t, symbols, lengths, count)) return -1;
    if (segments != (words + 3) / 4) return -2; /* a segment is exactly 4 words */
    uint64_t produced = 0;
    for (uint64_t s = 0; s < segments; ++s) {
        uint64_t pos = ORC_SEGMENT * s + (s ? gap_of(gaps, s - 1) : 0);
        const uint64_t end = ORC_SEGMENT * (s + 1);
        const int last = (s + 1 == segments);
        while (last ? (produced < n) : (pos < end)) {
            if (produced >= n) return -3;
            uint8_t sym;
            const uint32_t l = decode_one(&t, bits, words, pos, &sym);
            if (l == 0 || pos + l > words * 32) return -4;
            out[produced++] = sym;
            pos += l;
        }
        if (!last && pos != end + gap_of(gaps, s)) return -5;
    }
    return produced == n ? 0 : -6;
}

int64_t orc_decode_segments(const uint32_t* bits, uint64_t words, const uint32_t* gaps,
                            uint64_t segments, uint64_t s0, uint64_t s1,
                            const uint8_t* symbols, const uint8_t* lengths, int count,
                            uint8_t* out, uint64_t cap) {
    canon_t t;
    if (count < 1 || canon_init(&t, symbols, lengths, count)) return -1;
    uint64_t produced = 0;
    for (uint64_t s = s0; s < s1; ++s) {
        uint64_t pos = ORC_SEGMENT * s + (s ? gap_of(gaps, s - 1) : 0);
        uint64_t end = ORC_SEGMENT * (s + 1);
        const int last = (s + 1 == segments);
        if (last && end > words * 32) end = words * 32;
        while (pos < end) {
            uint8_t sym;
            const uint32_t l = decode_one(&t, bits, words, pos, &sym);
            if (l == 0 || pos + l > words * 32) {
                if (last) break; /* zero padding after the final codeword */
                return -4;
            }
            if (produced >= cap) return -3;
            out[produced++] = sym;
            pos += l;
        }
        if (!last && pos != ORC_SEGMENT * (s + 1) + gap_of(gaps, s)) return -5;
    }
    return (int64_t)produced;
}

/* ------------------------------------------------------------------------ */
/* reference two-level LUT                                                   */
/* ------------------------------------------------------------------------ */

/* get_table_info (decoder/src/get_table.cpp:3-46).  With reference_bug the
 * running code is advanced before it is used (get_table.cpp:20 vs :22-27),
 * as the reference does; without it the code of the current symbol is used
 * and the level-2 sizes follow the group widths get_twolevel_table lays out. */
uint32_t orc_ref_table_info(const uint8_t* symbols, const uint8_t* lengths, int count,
                            uint32_t prefix_bit, orc_table_info* info, int reference_bug) {
    (void)symbols;
    uint32_t code = 0, prev_prefix = 0, ptr = 0, l2 = 0, l1 = 0;
    const uint32_t mask = ~((~0u) << prefix_bit);
    if (reference_bug) {
        for (int i = 0; i < count; ++i) {
            const uint32_t cur = lengths[i];
            const uint32_t nxt = (i + 1 == count) ? cur : lengths[i + 1];
            code = (code + 1) << (nxt - cur);
            if (cur > prefix_bit) {
                const uint32_t sh = cur - prefix_bit;
                const uint32_t pc = (code >> sh) & mask;
                if (l1 == 0) l1 = code >> sh;
                if (prev_prefix != pc) {
                    l2 += 1u << sh;
                    ptr++;
                }
                prev_prefix = pc;
            }
        }
    } else {
        int i = 0;
        while (i < count) {
            const uint32_t cur = lengths[i];
            if (cur <= prefix_bit) {
                const uint32_t nxt = (i + 1 == count) ? cur : lengths[i + 1];
                code = (code + 1) << (nxt - cur);
                ++i;
                continue;
            }
            const uint32_t pc = code >> (cur - prefix_bit);
            if (l1 == 0) l1 = pc;
            uint32_t width = cur - prefix_bit;
            while (i < count && (code >> (lengths[i] - prefix_bit)) == pc) {
                const uint32_t li = lengths[i];
                width = li - prefix_bit;
                const uint32_t nxt = (i + 1 == count) ? li : lengths[i + 1];
                code = (code + 1) << (nxt - li);
                ++i;
            }
            l2 += 1u << width;
            ptr++;
        }
    }
    info->l1table_size = l1;
    info->l2table_size = l2;
    info->ptrtable_size = ptr;
    if (l1 == 0) {
        const uint32_t bit = lengths[count - 1];
        info->l1table_size = 1u << bit;
        return bit;
    }
    return prefix_bit;
}

size_t orc_ref_table_bytes(orc_table_info info) {
    return sizeof(uint32_t) * info.ptrtable_size + 256 + info.l1table_size + info.l2table_size;
}

/* get_twolevel_table (decoder/src/get_table.cpp:48-139).  Codes of length
 * <= prefix fill 2^(prefix-len) l1 slots; each run of longer codes sharing a
 * prefix gets an l2 table of width (longest length in the run - prefix) and
 * a ptr entry (width << 16 | l2 offset). */
uint32_t orc_ref_twolevel_table(void* blob, uint32_t prefix_bit, const uint8_t* symbols,
                                const uint8_t* lengths, int count, orc_table_info info) {
    uint32_t* ptr_table = (uint32_t*)blob;
    uint8_t* length_table = (uint8_t*)blob + info.ptrtable_size * sizeof(uint32_t);
    uint8_t* l1 = length_table + 256;
    uint8_t* l2 = l1 + info.l1table_size;
    uint32_t code = 0, boundary = 0, l2off = 0, groups = 0;
    int i = 0;
    while (i < count) {
        uint32_t cur = lengths[i];
        length_table[symbols[i]] = (uint8_t)cur;
        if (cur <= prefix_bit) {
            const uint32_t sh = prefix_bit - cur;
            for (uint32_t e = 0; e < (1u << sh); ++e) l1[(code << sh) + e] = symbols[i];
            const uint32_t nxt = (i == count - 1) ? cur : lengths[i + 1];
            code = (code + 1) << (nxt - cur);
            ++i;
            continue;
        }
        const uint32_t pc = code >> (cur - prefix_bit);
        if (boundary == 0) boundary = pc;
        /* the run of codes that share this prefix */
        int run = 0;
        uint32_t c = code, width = cur - prefix_bit;
        while (i + run < count && (c >> (lengths[i + run] - prefix_bit)) == pc) {
            const uint32_t li = lengths[i + run];
            width = li - prefix_bit;
            const uint32_t nxt = (i + run == count - 1) ? li : lengths[i + run + 1];
            c = (c + 1) << (nxt - li);
            ++run;
        }
        uint8_t* t = l2 + l2off;
        c = code;
        for (int k = 0; k < run; ++k) {
            const uint32_t li = lengths[i + k];
            length_table[symbols[i + k]] = (uint8_t)li;
            const uint32_t sfx = li - prefix_bit;
            const uint32_t at = (c & ~((~0u) << sfx)) << (width - sfx);
            for (uint32_t e = 0; e < (1u << (width - sfx)); ++e) t[at + e] = symbols[i + k];
            const uint32_t nxt = (i + k == count - 1) ? li : lengths[i + k + 1];
            c = (c + 1) << (nxt - li);
        }
        ptr_table[groups++] = (width << 16) | l2off;
        i += run;
        l2off += 1u << width;
        code = c;
    }
    return boundary;
}

/* ------------------------------------------------------------------------ */
/* container                                                                 */
/* ------------------------------------------------------------------------ */

/* Writer encoder/src/huff.cpp:111-125; reader decoder/src/huff.cpp:27-81.
 * Little-endian, unaligned: u64 symbol_count; symbol_count x {u8 symbol,
 * u8 length} (most frequent first); u32 n; u32 W; u32 S; u32 gap[ceil(S/8)];
 * u32 bits[W]. */
size_t orc_container_bytes(int count, uint64_t words, uint64_t gap_words) {
    return 8 + 2 * (size_t)count + 12 + 4 * (size_t)gap_words + 4 * (size_t)words;
}

size_t orc_container_write(uint8_t* dst, const uint8_t* symbols, const uint8_t* lengths, int count,
                           uint32_t n, uint32_t words, uint32_t segments, const uint32_t* gaps,
                           const uint32_t* bits) {
    uint8_t* p = dst;
    const uint64_t c64 = (uint64_t)count;
    memcpy(p, &c64, 8);
    p += 8;
    for (int i = 0; i < count; ++i) {
        *p++ = symbols[i];
        *p++ = lengths[i];
    }
    memcpy(p, &n, 4);
    memcpy(p + 4, &words, 4);
    memcpy(p + 8, &segments, 4);
    p += 12;
    const uint64_t gw = ((uint64_t)segments + 7) / 8;
    memcpy(p, gaps, 4 * gw);
    p += 4 * gw;
    memcpy(p, bits, 4 * (size_t)words);
    p += 4 * (size_t)words;
    return (size_t)(p - dst);
}

int orc_container_parse(const uint8_t* src, size_t size, int* count, const uint8_t** symlens,
                        uint32_t* n, uint32_t* words, uint32_t* segments, const uint8_t** gaps,
                        const uint8_t** bits) {
    if (size < 8) return -1;
    uint64_t c64;
    memcpy(&c64, src, 8);
    if (c64 > 256) return -2;
    size_t off = 8;
    if (size < off + 2 * c64 + 12) return -1;
    *count = (int)c64;
    *symlens = src + off;
    off += 2 * c64;
    memcpy(n, src + off, 4);
    memcpy(words, src + off + 4, 4);
    memcpy(segments, src + off + 8, 4);
    off += 12;
    const uint64_t gw = ((uint64_t)*segments + 7) / 8;
    if (size < off + 4 * gw + 4 * (uint64_t)*words) return -1;
    *gaps = src + off;
    *bits = src + off + 4 * gw;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* threaded CPU baseline (same format)                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    const uint8_t* in;
    uint64_t lo, hi;
    const uint32_t* code;
    const uint32_t* len;
    uint64_t first_bit;
    uint64_t nbits;
    uint32_t hist[256];
    uint32_t* bits;
    uint32_t* gaps;
} enc_job;

static void* job_hist(void* p) {
    enc_job* j = (enc_job*)p;
    memset(j->hist, 0, sizeof(j->hist));
    for (uint64_t i = j->lo; i < j->hi; ++i) j->hist[j->in[i]]++;
    return NULL;
}

static void* job_count(void* p) {
    enc_job* j = (enc_job*)p;
    uint64_t b = 0;
    for (uint64_t i = j->lo; i < j->hi; ++i) b += j->len[j->in[i]];
    j->nbits = b;
    return NULL;
}

/* Chunks write disjoint interior words; the word (and gap word) a chunk
 * shares with its neighbours is merged after the join. */
static void* job_pack(void* p) {
    enc_job* j = (enc_job*)p;
    if (j->hi <= j->lo) return NULL;
    orc_encode_chunk(j->in + j->lo, j->hi - j->lo, j->code, j->len, j->first_bit, j->bits,
                     j->gaps);
    return NULL;
}

static int clamp_threads(int threads) {
    if (threads < 1) return 1;
    if (threads > 256) return 256;
    return threads;
}

int orc_mt_histogram(const uint8_t* in, uint64_t n, uint32_t hist[256], int threads) {
    threads = clamp_threads(threads);
    enc_job* jobs = (enc_job*)calloc((size_t)threads, sizeof(enc_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        jobs[t].in = in;
        jobs[t].lo = n * (uint64_t)t / (uint64_t)threads;
        jobs[t].hi = n * (uint64_t)(t + 1) / (uint64_t)threads;
        pthread_create(&th[t], NULL, job_hist, &jobs[t]);
    }
    memset(hist, 0, 256 * sizeof(uint32_t));
    for (int t = 0; t < threads; ++t) {
        pthread_join(th[t], NULL);
        for (int b = 0; b < 256; ++b) hist[b] += jobs[t].hist[b];
    }
    free(jobs);
    free(th);
    return 0;
}

/* Parallel encode in the reference's own three steps (encoder/src/encoder.cu:
 * per-chunk bit counts, exclusive scan, pack at the scanned offset).  Each
 * chunk packs into zeroed output with OR, so words shared by two chunks
 * combine; chunks are processed in two phases (even, then odd) so no two
 * concurrently running chunks touch the same word. */
int orc_mt_encode(const uint8_t* in, uint64_t n, const uint32_t code[256], const uint32_t len[256],
                  uint32_t* bits, uint64_t words, uint32_t* gaps, uint64_t gap_words, int threads) {
    threads = clamp_threads(threads);
    /* every chunk must span more than one gap word (1024 bits) so that only
       neighbouring chunks share words; small inputs run as one chunk */
    if (n < (uint64_t)threads * 2 * 4096) threads = 1;
    const int chunks = threads == 1 ? 1 : 2 * threads;
    enc_job* jobs = (enc_job*)calloc((size_t)chunks, sizeof(enc_job));
    pthread_t* th = (pthread_t*)calloc((size_t)chunks, sizeof(pthread_t));
    for (int t = 0; t < chunks; ++t) {
        jobs[t].in = in;
        jobs[t].lo = n * (uint64_t)t / (uint64_t)chunks;
        jobs[t].hi = n * (uint64_t)(t + 1) / (uint64_t)chunks;
        jobs[t].code = code;
        jobs[t].len = len;
        jobs[t].bits = bits;
        jobs[t].gaps = gaps;
    }
    for (int t = 0; t < chunks; t += threads) {
        for (int u = t; u < t + threads && u < chunks; ++u)
            pthread_create(&th[u], NULL, job_count, &jobs[u]);
        for (int u = t; u < t + threads && u < chunks; ++u) pthread_join(th[u], NULL);
    }
    uint64_t acc = 0;
    for (int t = 0; t < chunks; ++t) {
        jobs[t].first_bit = acc;
        acc += jobs[t].nbits;
    }
    const orc_sizes z = orc_sizes_from_bits(acc);
    if (z.words != words || z.gap_words != gap_words) {
        free(jobs);
        free(th);
        return -2;
    }
    memset(bits, 0, words * sizeof(uint32_t));
    memset(gaps, 0, gap_words * sizeof(uint32_t));
    for (int phase = 0; phase < 2; ++phase) {
        for (int t = phase; t < chunks; t += 2) pthread_create(&th[t], NULL, job_pack, &jobs[t]);
        for (int t = phase; t < chunks; t += 2) pthread_join(th[t], NULL);
    }
    free(jobs);
    free(th);
    return 0;
}

typedef struct {
    const uint32_t* bits;
    uint64_t words;
    const uint32_t* gaps;
    uint64_t segments, s0, s1;
    const uint8_t* symbols;
    const uint8_t* lengths;
    int count;
    uint8_t* buf;
    uint64_t cap;
    int64_t produced;
} dec_job;

static void* job_decode(void* p) {
    dec_job* j = (dec_job*)p;
    j->cap = (j->s1 - j->s0) * 24 + 256;
    j->buf = (uint8_t*)malloc(j->cap);
    for (;;) {
        j->produced = orc_decode_segments(j->bits, j->words, j->gaps, j->segments, j->s0, j->s1,
                                          j->symbols, j->lengths, j->count, j->buf, j->cap);
        if (j->produced != -3) break;
        j->cap *= 2; /* more symbols than guessed: retry with a larger buffer */
        free(j->buf);
        j->buf = (uint8_t*)malloc(j->cap);
    }
    return NULL;
}

/* Parallel decode over segment ranges (the reference's unit of parallelism,
 * decoder/src/decoder.cu:501-507), concatenated in order and clipped at n. */
int orc_mt_decode(const uint32_t* bits, uint64_t words, const uint32_t* gaps, uint64_t segments,
                  const uint8_t* symbols, const uint8_t* lengths, int count, uint8_t* out,
                  uint64_t n, int threads) {
    threads = clamp_threads(threads);
    if (n == 0) return 0;
    dec_job* jobs = (dec_job*)calloc((size_t)threads, sizeof(dec_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        dec_job* j = &jobs[t];
        j->bits = bits;
        j->words = words;
        j->gaps = gaps;
        j->segments = segments;
        j->s0 = segments * (uint64_t)t / (uint64_t)threads;
        j->s1 = segments * (uint64_t)(t + 1) / (uint64_t)threads;
        j->symbols = symbols;
        j->lengths = lengths;
        j->count = count;
        pthread_create(&th[t], NULL, job_decode, j);
    }
    uint64_t at = 0;
    int rc = 0;
    for (int t = 0; t < threads; ++t) {
        pthread_join(th[t], NULL);
        if (jobs[t].produced < 0) rc = -1;
        if (rc == 0) {
            uint64_t k = (uint64_t)jobs[t].produced;
            if (at + k > n) k = n - at;
            memcpy(out + at, jobs[t].buf, k);
            at += k;
        }
        free(jobs[t].buf);
    }
    free(jobs);
    free(th);
    if (rc == 0 && at != n) rc = -6;
    return rc;
}
