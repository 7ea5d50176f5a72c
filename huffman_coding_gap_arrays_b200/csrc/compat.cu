// compat.cu -- the reference's own entry-point signatures, implemented on the
// hgap_* API, so the reference's bin/encoder and bin/decoder link against
// libhgap.so unchanged.  Like the reference these are host-synchronous and
// allocate per call; unlike it they never exit() -- errors print to stderr and
// come back as hgap_status.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "hgap_internal.h"

namespace {

hgap_status report(const char* where, hgap_status s) {
    if (s != HGAP_OK) std::fprintf(stderr, "hgap: %s: %s\n", where, hgap_status_string(s));
    return s;
}

// Reads a reference two-level table blob (decoder/src/get_table.cpp:48-139:
// [ptr u32 x ptrtable_size][length u8 x 256][l1 u8 x l1table_size][l2 u8 ...])
// back into the container-order symbol list.  Walks level 1 in code order
// while entries form valid runs of unseen symbols, then each level-2 table in
// pointer order; the result must hold exactly symbol_count distinct symbols
// and pass the canonical-book checks.  The l1table_size the reference passes
// may exceed the true boundary (its get_table_info advances the code before
// using it, get_table.cpp:20); the walk stops at the true boundary, where the
// first invalid run begins.
hgap_status book_from_ref_table(const uint8_t* blob, size_t blob_bytes, uint32_t prefix_bit,
                                uint32_t symbol_count, uint32_t l1size, uint32_t l2size,
                                uint32_t ptrsize, hgap_codebook* cb) {
    if (prefix_bit < 1 || prefix_bit > 16 || symbol_count < 1 || symbol_count > 256)
        return HGAP_ERR_CORRUPT;
    const size_t need = 4 * (size_t)ptrsize + 256 + (size_t)l1size + l2size;
    if (need > blob_bytes) return HGAP_ERR_CORRUPT;
    const uint32_t* ptr = reinterpret_cast<const uint32_t*>(blob);
    const uint8_t* lentab = blob + 4 * (size_t)ptrsize;
    const uint8_t* l1 = lentab + 256;
    const uint8_t* l2 = l1 + l1size;
    hgap_symlen list[256];
    bool seen[256] = {};
    uint32_t count = 0;
    uint32_t i = 0;
    while (count < symbol_count && i < l1size && i < (1u << prefix_bit)) {
        const uint8_t s = l1[i];
        const uint32_t len = lentab[s];
        if (len < 1 || len > prefix_bit || seen[s]) break;
        const uint32_t run = 1u << (prefix_bit - len);
        if (i + run > l1size) break;
        bool same = true;
        for (uint32_t k = 1; k < run && same; ++k) same = l1[i + k] == s;
        if (!same) break;
        seen[s] = true;
        list[count++] = {s, (uint8_t)len};
        i += run;
    }
    uint32_t off = 0;
    for (uint32_t g = 0; count < symbol_count && g < ptrsize; ++g) {
        const uint32_t w = ptr[g] >> 16, o = ptr[g] & 0xffffu;
        if (w < 1 || w + prefix_bit > 16 || o != off || (size_t)off + (1u << w) > l2size)
            return HGAP_ERR_CORRUPT;
        for (uint32_t j = 0; j < (1u << w);) {
            const uint8_t s = l2[o + j];
            const uint32_t len = lentab[s];
            if (len <= prefix_bit || len > prefix_bit + w || seen[s]) return HGAP_ERR_CORRUPT;
            const uint32_t run = 1u << (w - (len - prefix_bit));
            for (uint32_t k = 1; k < run; ++k)
                if (l2[o + j + k] != s) return HGAP_ERR_CORRUPT;
            seen[s] = true;
            list[count++] = {s, (uint8_t)len};
            j += run;
            if (count > symbol_count) return HGAP_ERR_CORRUPT;
        }
        off += 1u << w;
    }
    if (count != symbol_count) return HGAP_ERR_CORRUPT;
    return hgap_codebook_from_symbols(list, count, cb);
}

}  // namespace

extern "C" {

// encoder/src/encoder.cu:118-140.
void histgram(unsigned int* d_Histogram, unsigned int* d_Data, unsigned int byteCount) {
    report("histgram", hgap_histogram(d_Data, byteCount, d_Histogram, nullptr));
}

// encoder/src/encoder.cu:381-457.
hgap_status hgap_ref_encode(unsigned int* outputfile, unsigned int outputfilesize,
                            unsigned int* d_inputfile, unsigned int inputfilesize,
                            unsigned int gap_array_elements_num, const hgap_codeword* codetable) {
    if (!outputfile || !codetable || (inputfilesize && !d_inputfile))
        return report("encode", HGAP_ERR_INVALID_ARG);
    hgap_codebook cb;
    std::memset(&cb, 0, sizeof(cb));
    std::memcpy(cb.table, codetable, sizeof(cb.table));
    const uint64_t W = outputfilesize, S = gap_array_elements_num, G = (S + 7) / 8;
    uint32_t* d_out = nullptr;
    void* d_ws = nullptr;
    const size_t ws_bytes = hgap_encode_workspace_bytes(inputfilesize);
    hgap_status s = HGAP_OK;
    if (cudaMalloc(&d_out, 4 * (W + G) + 4) != cudaSuccess || cudaMalloc(&d_ws, ws_bytes) != cudaSuccess)
        s = HGAP_ERR_CUDA;
    if (s == HGAP_OK)
        s = hgap_encode(d_inputfile, inputfilesize, &cb, d_out, W, d_out + W, S, d_ws, ws_bytes, nullptr);
    if (s == HGAP_OK) s = hgap_workspace_status(d_ws, nullptr);
    if (s == HGAP_OK && W + G > 0 &&
        cudaMemcpy(outputfile, d_out, 4 * (W + G), cudaMemcpyDeviceToHost) != cudaSuccess)
        s = HGAP_ERR_CUDA;
    cudaFree(d_inputfile);  // the reference's encode() takes ownership (encoder.cu:451)
    cudaFree(d_out);
    cudaFree(d_ws);
    return report("encode", s);
}

// decoder/src/decoder.cu:732-815 without the timing loop.
hgap_status hgap_ref_decoder_l1_l2(unsigned int* input, int inputfilesize, unsigned int* output,
                                   int outputfilesize, int gap_elements_num, const void* dectable,
                                   int tablesize, unsigned int prefix_bit,
                                   unsigned int symbol_count, uint32_t l1table_size,
                                   uint32_t l2table_size, uint32_t ptrtable_size) {
    if (!input || !output || !dectable || inputfilesize < 0 || outputfilesize < 0 ||
        gap_elements_num < 0 || tablesize < 0)
        return report("decoder_l1_l2", HGAP_ERR_INVALID_ARG);
    hgap_codebook cb;
    hgap_status s = book_from_ref_table(static_cast<const uint8_t*>(dectable), (size_t)tablesize,
                                        prefix_bit, symbol_count, l1table_size, l2table_size,
                                        ptrtable_size, &cb);
    if (s != HGAP_OK) return report("decoder_l1_l2", s);
    const uint64_t W = (uint64_t)inputfilesize, S = (uint64_t)gap_elements_num, G = (S + 7) / 8;
    const uint64_t n = (uint64_t)outputfilesize;
    uint32_t* d_in = nullptr;
    uint8_t* d_out = nullptr;
    void* d_ws = nullptr;
    const size_t ws_bytes = hgap_decode_workspace_bytes(S);
    if (cudaMalloc(&d_in, 4 * (W + G) + 4) != cudaSuccess || cudaMalloc(&d_out, n + 16) != cudaSuccess ||
        cudaMalloc(&d_ws, ws_bytes) != cudaSuccess)
        s = HGAP_ERR_CUDA;
    if (s == HGAP_OK && cudaMemcpy(d_in, input, 4 * (W + G), cudaMemcpyHostToDevice) != cudaSuccess)
        s = HGAP_ERR_CUDA;
    if (s == HGAP_OK) s = hgap_decode(d_in + G, W, d_in, S, &cb, d_out, n, d_ws, ws_bytes, nullptr);
    if (s == HGAP_OK) s = hgap_workspace_status(d_ws, nullptr);
    if (s == HGAP_OK && n && cudaMemcpy(output, d_out, n, cudaMemcpyDeviceToHost) != cudaSuccess)
        s = HGAP_ERR_CUDA;
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_ws);
    return report("decoder_l1_l2", s);
}

}  // extern "C"
