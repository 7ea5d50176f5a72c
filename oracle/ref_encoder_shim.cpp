// ref_encoder_shim.cpp -- extern "C" entry points into the reference encoder.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own,
// unmodified encoder sources (read in place at build time by oracle/Makefile)
// into oracle/_ref/libref_encoder.so.  It lets the tests call the reference's
// codebook builder and, on a GPU host, the reference's own histogram and
// encode kernels, so that the CPU oracle and the CUDA library are pinned to
// what the reference really produces.
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

#include "constants.hpp"      // reference: encoder/include/constants.hpp
#include "encoder.cuh"        // reference: encode(), histgram()
#include "package_merge.hpp"  // reference: boundary_PM()
#include "symbols.hpp"        // reference: store_symbols(), get_outputfilesize()

// The comparator of encoder/src/huff.cpp:17-21 (compiled from that file with
// its main() renamed).
int compare(const void* p, const void* q);

extern "C" {

// Codebook exactly as encoder/src/huff.cpp:77-88 builds it: store_symbols,
// qsort(compare), boundary_PM, get_outputfilesize.  Outputs the list in
// container order (huff.cpp:114-119) and the per-byte codetable.  Returns the
// symbol count; for fewer than two symbols the reference is undefined and
// nothing is computed (returns the count, outputs untouched).
int hgapref_codebook(const uint32_t* hist, uint8_t* syms, uint8_t* lens, uint32_t* code,
                     uint32_t* len, uint64_t* total_bits) {
    unsigned int num[MAX_CODE_NUM];
    for (int i = 0; i < MAX_CODE_NUM; ++i) num[i] = hist[i];
    // one spare entry: add_node() reads symbols[symbol_count] (package_merge.cpp:37,52)
    struct Symbol symbols[MAX_CODE_NUM + 1];
    std::memset(symbols, 0, sizeof(symbols));
    const int count = store_symbols(num, symbols);
    if (count < 2) return count;
    qsort(symbols, count, sizeof(struct Symbol), compare);
    struct Codetable table[MAX_CODE_NUM];
    std::memset(table, 0, sizeof(table));
    boundary_PM(symbols, count, table);
    for (int i = 0; i < count; ++i) {
        syms[i] = symbols[count - 1 - i].symbol;
        lens[i] = symbols[count - 1 - i].length;
    }
    for (int b = 0; b < MAX_CODE_NUM; ++b) {
        code[b] = table[b].code;
        len[b] = table[b].length;
    }
    *total_bits = get_outputfilesize(symbols, count);
    return count;
}

// The reference GPU path of encoder/src/huff.cpp:60-99: upload, histgram(),
// encode().  The device input gets 8 KiB of zeroed slack beyond the data so
// that the idle threads of the last tile, which read their first word before
// checking the length (encoder/src/encoder.cu:183), stay inside the
// allocation.  encode() frees the device input itself (encoder.cu:451).
// `out` receives W bitstream words followed by ceil(S/8) gap words
// (huff.cpp:90-91).  Returns 0, or the CUDA error code.
int hgapref_gpu_encode(const uint8_t* in, uint32_t n, uint32_t* hist_out, const uint32_t* code,
                       const uint32_t* len, uint32_t out_words, uint32_t gap_elems,
                       uint32_t* out) {
    const size_t words = (n + 3) / 4 + 1 + 2048 + 4;
    unsigned int* d_in = nullptr;
    unsigned int* d_hist = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&d_in), words * 4) != cudaSuccess) return 1;
    if (cudaMalloc(reinterpret_cast<void**>(&d_hist), MAX_CODE_NUM * 4) != cudaSuccess) return 2;
    cudaMemset(d_in, 0, words * 4);
    cudaMemset(d_hist, 0, MAX_CODE_NUM * 4);
    cudaMemcpy(d_in, in, n, cudaMemcpyHostToDevice);
    histgram(d_hist, d_in, n);
    cudaMemcpy(hist_out, d_hist, MAX_CODE_NUM * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_hist);
    struct Codetable table[MAX_CODE_NUM];
    for (int b = 0; b < MAX_CODE_NUM; ++b) {
        table[b].code = code[b];
        table[b].length = len[b];
    }
    unsigned int* pinned = nullptr;
    const uint32_t gap_words = (gap_elems + 7) / 8;
    if (cudaMallocHost(reinterpret_cast<void**>(&pinned), (size_t)(out_words + gap_words) * 4 + 4) !=
        cudaSuccess)
        return 3;
    encode(pinned, out_words, d_in, n, gap_elems, table);
    std::memcpy(out, pinned, (size_t)(out_words + gap_words) * 4);
    cudaFreeHost(pinned);
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : static_cast<int>(e);
}

}  // extern "C"
