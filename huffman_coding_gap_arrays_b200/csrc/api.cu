// api.cu -- the extern "C" device entry points of libhgap.so (include/hgap.h).
// Validation, workspace carving and launches; no allocation anywhere.
#include <cuda_runtime.h>

#include <cstring>

#include "hgap_internal.h"

namespace {

using hgap::kWsHeader;

inline bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

inline hgap_status cuda_status(int e) { return e == 0 ? HGAP_OK : HGAP_ERR_CUDA; }

// Recomputes the canonical codes from the book's own symbol list, so a
// hand-edited table can never reach the decoder inconsistent.
hgap_status canonical_copy(const hgap_codebook* in, hgap_codebook* out) {
    if (in->symbol_count > 256) return HGAP_ERR_CORRUPT;
    return hgap_codebook_from_symbols(in->symbols, in->symbol_count, out);
}

}  // namespace

extern "C" {

hgap_status hgap_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, hgap_stream_t stream) {
    if (!d_hist || (n && !d_in)) return HGAP_ERR_INVALID_ARG;
    return cuda_status(hgap::launch_histogram(d_in, n, d_hist, stream));
}

size_t hgap_encode_workspace_bytes(uint64_t n) {
    const uint64_t nst = hgap::encode_super_tiles_cap(n);  // every input of up to n bytes, any alignment
    return hgap::kEncWsHeader + (size_t)nst * (sizeof(uint64_t) + 256 * sizeof(uint32_t));
}

}  // extern "C"

namespace {

// Carves the encoder workspace for input (d_in, n):
// [status][counter][..][tag @16][scratch hist @1024][st_rec @2048][st_hist].
hgap_status encode_layout(const void* d_in, uint64_t n, void* d_workspace, size_t workspace_bytes,
                          hgap::EncArgs* a, hgap::HistStArgs* h) {
    if (!d_in || !d_workspace || !aligned(d_workspace, 16)) return HGAP_ERR_INVALID_ARG;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(d_in);
    const uint64_t lo = addr & 15;
    const uint64_t st_bytes = hgap::encode_st_chunks(n) * hgap::kEncChunkBytes;
    const uint64_t nst = hgap::encode_super_tiles(lo + n, n);
    if (nst >= 0xffffffffull) return HGAP_ERR_UNSUPPORTED;
    const size_t need = hgap::kEncWsHeader + (size_t)nst * (sizeof(uint64_t) + 256 * sizeof(uint32_t));
    if (workspace_bytes < need) return HGAP_ERR_WORKSPACE;
    uint8_t* ws = static_cast<uint8_t*>(d_workspace);
    std::memset(a, 0, sizeof(*a));
    std::memset(h, 0, sizeof(*h));
    hgap::EncJob& J = a->single;
    J.in_aligned = reinterpret_cast<const uint8_t*>(addr - lo);
    J.lo = lo;
    J.hi = lo + n;
    J.item0 = 0;
    J.nst = nst;
    J.st_bytes = (uint32_t)st_bytes;
    a->count = 1;
    a->nitems = nst;
    a->status = reinterpret_cast<uint32_t*>(ws);
    a->counter = reinterpret_cast<uint32_t*>(ws) + 1;
    a->tag = reinterpret_cast<const uint64_t*>(ws + hgap::kEncWsTag);
    a->st_rec = reinterpret_cast<uint64_t*>(ws + hgap::kEncWsHeader);
    a->st_hist = reinterpret_cast<const uint32_t*>(a->st_rec + nst);
    h->single = J;
    h->count = 1;
    h->nitems = nst;
    h->hist = reinterpret_cast<uint32_t*>(ws + hgap::kEncWsScratchHist);
    h->st_hist = const_cast<uint32_t*>(a->st_hist);
    h->tag = reinterpret_cast<uint64_t*>(ws + hgap::kEncWsTag);
    return HGAP_OK;
}

hgap_status encode_outputs(const hgap_codebook* cb, uint32_t* d_bits, uint64_t words, uint32_t* d_gaps,
                           uint64_t segments, hgap::EncArgs* a) {
    if (!d_bits || !d_gaps || !aligned(d_bits, 4) || !aligned(d_gaps, 4)) return HGAP_ERR_INVALID_ARG;
    if (segments != (words + 3) / 4 || words == 0) return HGAP_ERR_SIZE;
    for (int b = 0; b < 256; ++b) {
        const uint32_t l = cb->table[b].length;
        if (l > (uint32_t)hgap::kMaxLen || (l && (cb->table[b].code >> l) != 0)) return HGAP_ERR_CORRUPT;
    }
    hgap::EncJob& J = a->single;
    J.bits = d_bits;
    J.words = words;
    J.gaps = d_gaps;
    J.segments = segments;
    J.gap_words = (segments + 7) / 8;
    J.bits_aligned16 = aligned(d_bits, 16) ? 1u : 0u;
    return HGAP_OK;
}

// Clears status + counter, and the super-tile look-back records.
hgap_status encode_clear(const hgap::EncArgs& a, bool tag_too, cudaStream_t st) {
    uint8_t* ws = reinterpret_cast<uint8_t*>(a.status);
    if (cudaMemsetAsync(ws, 0, tag_too ? hgap::kEncWsHeader : hgap::kEncWsTag, st) != cudaSuccess)
        return HGAP_ERR_CUDA;
    if (cudaMemsetAsync(a.st_rec, 0, sizeof(uint64_t) * a.nitems, st) != cudaSuccess) return HGAP_ERR_CUDA;
    return HGAP_OK;
}

}  // namespace

extern "C" {

hgap_status hgap_encode_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, void* d_workspace,
                                  size_t workspace_bytes, hgap_stream_t stream) {
    if (!d_hist) return HGAP_ERR_INVALID_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) return cudaMemsetAsync(d_hist, 0, 1024, st) == cudaSuccess ? HGAP_OK : HGAP_ERR_CUDA;
    hgap::EncArgs a;
    hgap::HistStArgs h;
    hgap_status s = encode_layout(d_in, n, d_workspace, workspace_bytes, &a, &h);
    if (s != HGAP_OK) return s;
    h.hist = d_hist;
    s = encode_clear(a, true, st);
    if (s != HGAP_OK) return s;
    if (cudaMemsetAsync(d_hist, 0, 256 * sizeof(uint32_t), st) != cudaSuccess) return HGAP_ERR_CUDA;
    return cuda_status(hgap::launch_hist_st(h, 0, stream));
}

hgap_status hgap_encode_prepared(const void* d_in, uint64_t n, const hgap_codebook* cb, uint32_t* d_bits,
                                 uint64_t words, uint32_t* d_gaps, uint64_t segments, void* d_workspace,
                                 size_t workspace_bytes, hgap_stream_t stream) {
    if (!cb) return HGAP_ERR_INVALID_ARG;
    if (n == 0) return (words == 0 && segments == 0) ? HGAP_OK : HGAP_ERR_SIZE;
    hgap::EncArgs a;
    hgap::HistStArgs h;
    hgap_status s = encode_layout(d_in, n, d_workspace, workspace_bytes, &a, &h);
    if (s == HGAP_OK) s = encode_outputs(cb, d_bits, words, d_gaps, segments, &a);
    if (s != HGAP_OK) return s;
    hgap::EncTable t;
    hgap::make_enc_table(*cb, &t);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    s = encode_clear(a, false, st);
    if (s != HGAP_OK) return s;
    return cuda_status(hgap::launch_encode(a, t, 0, stream));
}

hgap_status hgap_encode_part_prepared(const void* d_in, uint64_t n, const hgap_codebook* cb, uint64_t bit0,
                                      uint64_t part_bits, uint32_t* d_bits, uint64_t bits_word0,
                                      uint32_t* d_gaps, uint64_t gaps_word0, void* d_workspace,
                                      size_t workspace_bytes, hgap_stream_t stream) {
    if (!cb) return HGAP_ERR_INVALID_ARG;
    if (n == 0) return part_bits == 0 ? HGAP_OK : HGAP_ERR_SIZE;
    if ((bits_word0 & 3) || bits_word0 > (bit0 >> 5) || gaps_word0 > (bit0 >> 10)) return HGAP_ERR_INVALID_ARG;
    const uint64_t end = bit0 + part_bits;
    if (end < bit0) return HGAP_ERR_SIZE;
    hgap::EncArgs a;
    hgap::HistStArgs h;
    hgap_status s = encode_layout(d_in, n, d_workspace, workspace_bytes, &a, &h);
    // the stream's word and segment counts through the end of this part
    if (s == HGAP_OK) s = encode_outputs(cb, d_bits, (end + 31) / 32, d_gaps, (end + 127) / 128, &a);
    if (s != HGAP_OK) return s;
    // the windows hold stream words [bits_word0, ..) and gap words [gaps_word0, ..): the job
    // addresses stream word w at bits + w, never below bits_word0 (w >= bit0 / 32), and
    // bits_word0 % 4 == 0 keeps the 16-byte alignment of the window's vector stores
    hgap::EncJob& J = a.single;
    J.bits = reinterpret_cast<uint32_t*>(reinterpret_cast<uintptr_t>(d_bits) - 4 * bits_word0);
    J.gaps = reinterpret_cast<uint32_t*>(reinterpret_cast<uintptr_t>(d_gaps) - 4 * gaps_word0);
    J.bit0 = bit0;
    hgap::EncTable t;
    hgap::make_enc_table(*cb, &t);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    s = encode_clear(a, false, st);
    if (s != HGAP_OK) return s;
    return cuda_status(hgap::launch_encode(a, t, 0, stream));
}

}  // extern "C"

namespace {

hgap_status encode_impl(const void* d_in, uint64_t n, const hgap_codebook* cb, uint32_t* d_bits, uint64_t words,
                        uint32_t* d_gaps, uint64_t segments, void* d_workspace, size_t workspace_bytes,
                        hgap_stream_t stream, const hgap::LookbackHook& hook) {
    if (!cb) return HGAP_ERR_INVALID_ARG;
    if (n == 0) return (words == 0 && segments == 0) ? HGAP_OK : HGAP_ERR_SIZE;
    hgap::EncArgs a;
    hgap::HistStArgs h;
    hgap_status s = encode_layout(d_in, n, d_workspace, workspace_bytes, &a, &h);
    if (s == HGAP_OK) s = encode_outputs(cb, d_bits, words, d_gaps, segments, &a);
    if (s != HGAP_OK) return s;
    hgap::EncTable t;
    hgap::make_enc_table(*cb, &t);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    s = encode_clear(a, true, st);
    if (s != HGAP_OK) return s;
    // per-region histograms into the workspace (the scratch histogram was cleared with the header)
    int e = hgap::launch_hist_st(h, 0, stream);
    if (e != 0) return HGAP_ERR_CUDA;
    a.hook = hook;
    return cuda_status(hgap::launch_encode(a, t, 0, stream));
}

// The decoder table of the last symbol list this host thread decoded with: a
// stream is often decoded again with the same book (a served payload, a
// benchmark loop), and building the table is most of a call's host time.
struct DecBookCache {
    bool valid = false;
    uint32_t count = 0;
    hgap_symlen symbols[256];
    uint32_t min_len = 0;
    bool complete = false;
    bool pairs = false;
    hgap::DecTable table;
};

hgap_status decode_impl(const uint32_t* d_bits, uint64_t words, const uint32_t* d_gaps, uint64_t segments,
                        const hgap_codebook* cb, uint8_t* d_out, uint64_t n, void* d_workspace,
                        size_t workspace_bytes, hgap_stream_t stream, const hgap::LookbackHook& hook) {
    if (!cb) return HGAP_ERR_INVALID_ARG;
    if (n == 0) return (words == 0 && segments == 0) ? HGAP_OK : HGAP_ERR_SIZE;
    if (!d_bits || !d_gaps || !d_out || !d_workspace) return HGAP_ERR_INVALID_ARG;
    if (!aligned(d_bits, 4) || !aligned(d_gaps, 4) || !aligned(d_workspace, 8))
        return HGAP_ERR_INVALID_ARG;
    if (words == 0 || segments != (words + 3) / 4) return HGAP_ERR_SIZE;
    thread_local DecBookCache cache;
    const bool hit = cache.valid && cb->symbol_count == cache.count &&
                     std::memcmp(cb->symbols, cache.symbols, sizeof(hgap_symlen) * cache.count) == 0;
    hgap_codebook book;
    hgap_status s = HGAP_OK;
    uint32_t min_len = hgap::kMaxLen;
    bool complete = false;
    if (hit) {
        min_len = cache.min_len;
        complete = cache.complete;
    } else {
        s = canonical_copy(cb, &book);
        if (s != HGAP_OK) return s;
        if (book.symbol_count == 0) return HGAP_ERR_CORRUPT;
        uint64_t kraft = 0;  // units of 2^-16; a complete book (sum 1) has no invalid table entry
        for (uint32_t i = 0; i < book.symbol_count; ++i) {
            if (book.symbols[i].length < min_len) min_len = book.symbols[i].length;
            kraft += 1ull << (hgap::kMaxLen - book.symbols[i].length);
        }
        complete = kraft == (1ull << hgap::kMaxLen);
    }
    hgap::DecArgs a;
    std::memset(&a, 0, sizeof(a));
    hgap::DecJob& J = a.single;
    J.bits = d_bits;
    J.words = words;
    J.gaps = d_gaps;
    J.segments = segments;
    J.gap_words = (segments + 7) / 8;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(d_out);
    J.out_lo = addr & 15;
    J.out_aligned = reinterpret_cast<uint8_t*>(addr - J.out_lo);
    J.n = n;
    J.item0 = 0;
    J.ntiles = hgap::decode_tiles(segments, min_len);
    if (J.ntiles >= 0xffffffffull) return HGAP_ERR_UNSUPPORTED;
    a.count = 1;
    a.nitems = J.ntiles;
    const size_t need = kWsHeader + sizeof(uint64_t) * (size_t)J.ntiles;
    if (workspace_bytes < need) return HGAP_ERR_WORKSPACE;
    uint8_t* ws = static_cast<uint8_t*>(d_workspace);
    a.status = reinterpret_cast<uint32_t*>(ws);
    a.counter = reinterpret_cast<uint32_t*>(ws) + 1;
    a.lookback = reinterpret_cast<uint64_t*>(ws + kWsHeader);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // the workspace is cleared on the device while the host builds the table
    if (cudaMemsetAsync(ws, 0, need, st) != cudaSuccess) return HGAP_ERR_CUDA;
    if (!hit) {
        cache.valid = false;
        s = hgap::make_dec_table(book, &cache.table);
        if (s != HGAP_OK) return s;
        // two symbols per lookup pay off once about a third of the lookups yield two
        cache.pairs = hgap::dec_pair_fraction(cache.table) >= 0.3;
        cache.count = cb->symbol_count;
        std::memcpy(cache.symbols, cb->symbols, sizeof(hgap_symlen) * cache.count);
        cache.min_len = min_len;
        cache.complete = complete;
        cache.valid = true;
    }
    a.hook = hook;
    // the table travels as a kernel parameter: copied at launch, so the cache may change after
    return cuda_status(hgap::launch_decode(a, cache.table, min_len, complete, cache.pairs, 0, 0, stream));
}

hgap::LookbackHook hold_hook(uint64_t hold, uint64_t wait_limit_ns) {
    hgap::LookbackHook h;
    h.hold_plus1 = hold == ~0ull ? 0 : hold + 1;
    h.wait_ns = wait_limit_ns;
    return h;
}

}  // namespace

extern "C" {

hgap_status hgap_encode(const void* d_in, uint64_t n, const hgap_codebook* cb, uint32_t* d_bits,
                        uint64_t words, uint32_t* d_gaps, uint64_t segments, void* d_workspace,
                        size_t workspace_bytes, hgap_stream_t stream) {
    return encode_impl(d_in, n, cb, d_bits, words, d_gaps, segments, d_workspace, workspace_bytes, stream,
                       hgap::LookbackHook{0, 0});
}

hgap_status hgap_encode_hold(const void* d_in, uint64_t n, const hgap_codebook* cb, uint32_t* d_bits,
                             uint64_t words, uint32_t* d_gaps, uint64_t segments, void* d_workspace,
                             size_t workspace_bytes, hgap_stream_t stream, uint64_t hold, uint64_t wait_limit_ns) {
    return encode_impl(d_in, n, cb, d_bits, words, d_gaps, segments, d_workspace, workspace_bytes, stream,
                       hold_hook(hold, wait_limit_ns));
}

size_t hgap_decode_workspace_bytes(uint64_t segments) {
    return kWsHeader + sizeof(uint64_t) * (size_t)hgap::decode_tiles(segments, 1);  // worst case
}

hgap_status hgap_decode(const uint32_t* d_bits, uint64_t words, const uint32_t* d_gaps,
                        uint64_t segments, const hgap_codebook* cb, uint8_t* d_out, uint64_t n,
                        void* d_workspace, size_t workspace_bytes, hgap_stream_t stream) {
    return decode_impl(d_bits, words, d_gaps, segments, cb, d_out, n, d_workspace, workspace_bytes, stream,
                       hgap::LookbackHook{0, 0});
}

hgap_status hgap_decode_hold(const uint32_t* d_bits, uint64_t words, const uint32_t* d_gaps,
                             uint64_t segments, const hgap_codebook* cb, uint8_t* d_out, uint64_t n,
                             void* d_workspace, size_t workspace_bytes, hgap_stream_t stream, uint64_t hold,
                             uint64_t wait_limit_ns) {
    return decode_impl(d_bits, words, d_gaps, segments, cb, d_out, n, d_workspace, workspace_bytes, stream,
                       hold_hook(hold, wait_limit_ns));
}

hgap_status hgap_workspace_status(const void* d_workspace, hgap_stream_t stream) {
    if (!d_workspace) return HGAP_ERR_INVALID_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint32_t flags = 0;
    if (cudaMemcpyAsync(&flags, d_workspace, sizeof(flags), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return HGAP_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return HGAP_ERR_CUDA;
    return hgap_status_from_word(flags);
}

hgap_status hgap_status_from_word(uint32_t flags) {
    if (flags & hgap::kDevTimeout) return HGAP_ERR_TIMEOUT;
    if (flags & hgap::kDevNoCode) return HGAP_ERR_NO_CODE;
    if (flags & hgap::kDevCorrupt) return HGAP_ERR_CORRUPT;
    if (flags & hgap::kDevSize) return HGAP_ERR_SIZE;
    if (flags & hgap::kDevPlan) return HGAP_ERR_INVALID_ARG;
    return HGAP_OK;
}

}  // extern "C"
