// host.cpp -- host-side half of the path: codebook construction, the
// encoder/decoder tables the kernels take as launch parameters, and the
// container format.  Pure C++ (no CUDA calls).
#include <algorithm>
#include <cstring>
#include <vector>

#include "hgap_internal.h"

namespace {

struct Leaf {
    uint8_t symbol;
    uint32_t count;
};

// Length-limited (16-bit) code lengths by package-merge, with the
// reference's tie rule: a package precedes a leaf of equal weight
// (encoder/src/package_merge.cpp:37,52,136).  `leaves` ascend by count.
// Level 1 is the leaf list; level l merges the leaves with the pairwise
// packages of level l-1; the top level keeps 2n-2 items.  Walking down from
// the top, the leaves inside each level's active prefix gain one bit, and the
// packages in it make the next level's active prefix twice as long.
void package_merge(const std::vector<Leaf>& leaves, std::vector<uint8_t>& len) {
    const int n = (int)leaves.size();
    const int keep = 2 * n - 2;
    struct Item {
        uint64_t w;
        bool pkg;
    };
    std::vector<std::vector<Item>> lvl(hgap::kMaxLen + 1);
    lvl[1].reserve(n);
    for (const Leaf& l : leaves) lvl[1].push_back({l.count, false});
    for (int l = 2; l <= hgap::kMaxLen; ++l) {
        const std::vector<Item>& below = lvl[l - 1];
        std::vector<Item>& cur = lvl[l];
        cur.reserve(keep);
        const size_t npk = below.size() / 2;
        size_t li = 0, pi = 0;
        while ((int)cur.size() < keep && (li < (size_t)n || pi < npk)) {
            const bool have_pkg = pi < npk;
            const uint64_t pw = have_pkg ? below[2 * pi].w + below[2 * pi + 1].w : 0;
            if (have_pkg && (li >= (size_t)n || pw <= leaves[li].count)) {
                cur.push_back({pw, true});
                ++pi;
            } else {
                cur.push_back({leaves[li].count, false});
                ++li;
            }
        }
    }
    len.assign(n, 0);
    size_t active = keep;
    for (int l = hgap::kMaxLen; l >= 1 && active > 0; --l) {
        size_t nleaf = 0, npkg = 0;
        for (size_t k = 0; k < active && k < lvl[l].size(); ++k) (lvl[l][k].pkg ? npkg : nleaf)++;
        for (size_t i = 0; i < nleaf; ++i) len[i]++;
        active = 2 * npkg;
    }
}

// Canonical codes from a container-order list (encoder/src/package_merge.cpp:168-181).
hgap_status assign_codes(hgap_codebook* cb) {
    std::memset(cb->table, 0, sizeof(cb->table));
    uint64_t kraft = 0;  // in units of 2^-16
    uint32_t code = 0;
    bool seen[256] = {};
    for (uint32_t i = 0; i < cb->symbol_count; ++i) {
        const uint32_t l = cb->symbols[i].length;
        const uint8_t s = cb->symbols[i].symbol;
        if (l < 1 || l > (uint32_t)hgap::kMaxLen || seen[s]) return HGAP_ERR_CORRUPT;
        seen[s] = true;
        const uint32_t nl = i + 1 < cb->symbol_count ? cb->symbols[i + 1].length : l;
        if (nl < l) return HGAP_ERR_CORRUPT;
        kraft += 1ull << (hgap::kMaxLen - l);
        cb->table[s].code = code;
        cb->table[s].length = l;
        code = (code + 1) << (nl - l);
    }
    if (kraft > (1ull << hgap::kMaxLen)) return HGAP_ERR_CORRUPT;
    return HGAP_OK;
}

}  // namespace

namespace hgap {

void make_enc_table(const hgap_codebook& cb, EncTable* t) {
    for (int b = 0; b < 256; ++b) {
        const uint32_t l = cb.table[b].length;
        t->e[b] = l ? ((cb.table[b].code & 0xffffu) | (l << 16)) : kEncAbsent;
    }
}

// Level-1 / level-2 tables of the decoder (layout in hgap_internal.h).  The
// level-1 boundary is the first prefix of a long code taken from the code
// itself -- the value the reference's get_twolevel_table computes
// (decoder/src/get_table.cpp:93-95) -- not the next symbol's code that its
// get_table_info uses (get_table.cpp:20).  A complete book (Kraft sum 1, what
// package-merge builds) needs at most 2368 level-2 entries: a prefix whose
// longest code has w extra bits is split by at least w+1 codes, so 256 codes
// give at most 36 prefixes of 2^6 entries and a remainder.
hgap_status make_dec_table(const hgap_codebook& cb, DecTable* t) {
    constexpr int P = kDecPrefix;
    for (int i = 0; i < (1 << P); ++i) t->t1[i] = kDecInvalid;
    for (int i = 0; i < kDecT2Cap; ++i) t->t2[i] = kDecInvalid;
    const uint32_t n = cb.symbol_count;
    uint32_t i = 0, t2off = 0;
    while (i < n) {
        const uint8_t sym = cb.symbols[i].symbol;
        const uint32_t l = cb.symbols[i].length;
        const uint32_t code = cb.table[sym].code;
        if (l <= (uint32_t)P) {
            const uint16_t e = (uint16_t)(((l - 1) << 8) | sym);
            const uint32_t first = code << (P - l), cnt = 1u << (P - l);
            for (uint32_t k = 0; k < cnt; ++k) t->t1[first + k] = e;
            ++i;
            continue;
        }
        // run of longer codes sharing this prefix; lengths ascend, so the
        // last one sets the level-2 width
        const uint32_t prefix = code >> (l - P);
        uint32_t j = i, width = 0;
        while (j < n) {
            const uint32_t lj = cb.symbols[j].length;
            if ((cb.table[cb.symbols[j].symbol].code >> (lj - P)) != prefix) break;
            width = lj - P;
            ++j;
        }
        if (t2off + (1u << width) > (uint32_t)kDecT2Cap) return HGAP_ERR_UNSUPPORTED;
        t->t1[prefix] = (uint16_t)(0x8000u | (width << 12) | t2off);
        for (uint32_t k = i; k < j; ++k) {
            const uint8_t sk = cb.symbols[k].symbol;
            const uint32_t lk = cb.symbols[k].length;
            const uint32_t sfx = cb.table[sk].code & ((1u << (lk - P)) - 1u);
            const uint32_t first = sfx << (width - (lk - P)), cnt = 1u << (width - (lk - P));
            const uint16_t e = (uint16_t)(((lk - 1) << 8) | sk);
            for (uint32_t m = 0; m < cnt; ++m) t->t2[t2off + first + m] = e;
        }
        t2off += 1u << width;
        i = j;
    }
    return HGAP_OK;
}

double dec_pair_fraction(const DecTable& t) {
    constexpr uint32_t P = kDecPrefix, mask = (1u << P) - 1u;
    auto direct_len = [&](uint32_t x) -> uint32_t {  // 0 unless a valid direct entry
        const uint16_t e = t.t1[x];
        return (e & 0x8000u) || (e & kDecInvalid) ? 0u : ((e >> 8) & 15u) + 1u;
    };
    uint32_t pairs = 0;
    for (uint32_t x = 0; x <= mask; ++x) {
        const uint32_t l1 = direct_len(x);
        if (l1 == 0 || l1 >= P) continue;
        const uint32_t l2 = direct_len((x << l1) & mask);
        if (l2 && l1 + l2 <= P) ++pairs;
    }
    return pairs / double(mask + 1);
}

}  // namespace hgap

extern "C" {

const char* hgap_status_string(hgap_status s) {
    switch (s) {
        case HGAP_OK: return "ok";
        case HGAP_ERR_INVALID_ARG: return "invalid argument";
        case HGAP_ERR_CUDA: return "CUDA runtime error";
        case HGAP_ERR_TIMEOUT: return "device wait timed out";
        case HGAP_ERR_CORRUPT: return "corrupt stream, gap array or codebook";
        case HGAP_ERR_SIZE: return "size mismatch";
        case HGAP_ERR_WORKSPACE: return "workspace too small";
        case HGAP_ERR_NO_CODE: return "input byte without a codeword";
        case HGAP_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

hgap_sizes hgap_sizes_from_bits(uint64_t bits) {
    hgap_sizes z;
    z.bits = bits;
    z.words = (bits + 31) / 32;
    z.segments = (bits + HGAP_SEGMENT_BITS - 1) / HGAP_SEGMENT_BITS;
    z.gap_words = (z.segments + HGAP_GAPS_PER_WORD - 1) / HGAP_GAPS_PER_WORD;
    return z;
}

uint64_t hgap_encoded_bits(const hgap_codebook* cb, const uint32_t hist[256]) {
    uint64_t bits = 0;
    for (int b = 0; b < 256; ++b) bits += (uint64_t)cb->table[b].length * hist[b];
    return bits;
}

// store_symbols (encoder/src/symbols.cpp:29-43) + qsort(compare)
// (encoder/src/huff.cpp:17-21, stable on glibc for this size, so ties stay in
// byte order) + boundary_PM (encoder/src/package_merge.cpp:107-182).
hgap_status hgap_codebook_build(const uint32_t hist[256], hgap_codebook* cb, hgap_sizes* sizes) {
    if (!hist || !cb) return HGAP_ERR_INVALID_ARG;
    std::memset(cb, 0, sizeof(*cb));
    std::vector<Leaf> leaves;
    for (int b = 0; b < 256; ++b)
        if (hist[b]) leaves.push_back({(uint8_t)b, hist[b]});
    std::stable_sort(leaves.begin(), leaves.end(),
                     [](const Leaf& x, const Leaf& y) { return x.count < y.count; });
    const uint32_t n = (uint32_t)leaves.size();
    cb->symbol_count = n;
    std::vector<uint8_t> len;
    if (n == 1) {
        len.assign(1, 1);  // defined here; the reference is undefined (package_merge.cpp:113-132)
    } else if (n >= 2) {
        package_merge(leaves, len);
    }
    for (uint32_t i = 0; i < n; ++i) {  // container order: most frequent first (huff.cpp:114)
        cb->symbols[i].symbol = leaves[n - 1 - i].symbol;
        cb->symbols[i].length = len[n - 1 - i];
    }
    const hgap_status st = assign_codes(cb);
    if (st != HGAP_OK) return st;
    if (sizes) *sizes = hgap_sizes_from_bits(hgap_encoded_bits(cb, hist));
    return HGAP_OK;
}

hgap_status hgap_codebook_from_symbols(const hgap_symlen* symbols, uint32_t count,
                                       hgap_codebook* cb) {
    if (!cb || count > 256 || (count && !symbols)) return HGAP_ERR_INVALID_ARG;
    std::memset(cb, 0, sizeof(*cb));
    cb->symbol_count = count;
    for (uint32_t i = 0; i < count; ++i) cb->symbols[i] = symbols[i];
    return assign_codes(cb);
}

hgap_status hgap_decode_table_build(const hgap_codebook* cb, uint16_t* t1, uint16_t* t2) {
    if (!cb || !t1 || !t2) return HGAP_ERR_INVALID_ARG;
    hgap_codebook book;
    if (cb->symbol_count > 256) return HGAP_ERR_CORRUPT;
    hgap_status st = hgap_codebook_from_symbols(cb->symbols, cb->symbol_count, &book);
    if (st != HGAP_OK) return st;
    if (book.symbol_count == 0) return HGAP_ERR_CORRUPT;
    hgap::DecTable t;
    st = hgap::make_dec_table(book, &t);
    if (st != HGAP_OK) return st;
    std::memcpy(t1, t.t1, sizeof(t.t1));
    std::memcpy(t2, t.t2, sizeof(t.t2));
    return HGAP_OK;
}

size_t hgap_container_bytes(uint32_t symbol_count, uint64_t words, uint64_t segments) {
    return 8 + 2 * (size_t)symbol_count + 12 + 4 * (size_t)((segments + 7) / 8) + 4 * (size_t)words;
}

hgap_status hgap_container_write(void* dst, size_t capacity, const hgap_codebook* cb, uint64_t n,
                                 uint64_t words, uint64_t segments, const uint32_t* gaps,
                                 const uint32_t* bits, size_t* written) {
    if (!dst || !cb) return HGAP_ERR_INVALID_ARG;
    if (n > 0xffffffffull || words > 0xffffffffull || segments > 0xffffffffull)
        return HGAP_ERR_UNSUPPORTED;  // the header fields are u32 (encoder/src/huff.cpp:121-123)
    const size_t need = hgap_container_bytes(cb->symbol_count, words, segments);
    if (capacity < need) return HGAP_ERR_SIZE;
    uint8_t* p = static_cast<uint8_t*>(dst);
    const uint64_t c64 = cb->symbol_count;
    std::memcpy(p, &c64, 8);
    p += 8;
    for (uint32_t i = 0; i < cb->symbol_count; ++i) {
        *p++ = cb->symbols[i].symbol;
        *p++ = cb->symbols[i].length;
    }
    const uint32_t hdr[3] = {(uint32_t)n, (uint32_t)words, (uint32_t)segments};
    std::memcpy(p, hdr, 12);
    p += 12;
    const size_t gw = (size_t)((segments + 7) / 8);
    if (gw) std::memcpy(p, gaps, 4 * gw);
    p += 4 * gw;
    if (words) std::memcpy(p, bits, 4 * (size_t)words);
    p += 4 * (size_t)words;
    if (written) *written = (size_t)(p - static_cast<uint8_t*>(dst));
    return HGAP_OK;
}

hgap_status hgap_container_parse(const void* src, size_t size, hgap_codebook* cb, uint64_t* n,
                                 uint64_t* words, uint64_t* segments, const void** gaps,
                                 const void** bits) {
    if (!src || !cb || !n || !words || !segments) return HGAP_ERR_INVALID_ARG;
    const uint8_t* p = static_cast<const uint8_t*>(src);
    if (size < 8) return HGAP_ERR_CORRUPT;
    uint64_t c64;
    std::memcpy(&c64, p, 8);
    if (c64 > 256) return HGAP_ERR_CORRUPT;
    size_t off = 8;
    if (size < off + 2 * c64 + 12) return HGAP_ERR_CORRUPT;
    hgap_symlen syms[256];
    for (uint64_t i = 0; i < c64; ++i) {
        syms[i].symbol = p[off + 2 * i];
        syms[i].length = p[off + 2 * i + 1];
    }
    off += 2 * c64;
    uint32_t hdr[3];
    std::memcpy(hdr, p + off, 12);
    off += 12;
    const uint64_t gw = ((uint64_t)hdr[2] + 7) / 8;
    if (size < off + 4 * gw + 4 * (uint64_t)hdr[1]) return HGAP_ERR_CORRUPT;
    if (hdr[2] != (hdr[1] + 3) / 4) return HGAP_ERR_CORRUPT;  // a segment is 4 words
    if ((hdr[0] == 0) != (hdr[1] == 0) || (hdr[0] && c64 == 0)) return HGAP_ERR_CORRUPT;
    const hgap_status st = hgap_codebook_from_symbols(syms, (uint32_t)c64, cb);
    if (st != HGAP_OK) return st;
    *n = hdr[0];
    *words = hdr[1];
    *segments = hdr[2];
    if (gaps) *gaps = p + off;
    if (bits) *bits = p + off + 4 * gw;
    return HGAP_OK;
}

}  // extern "C"
