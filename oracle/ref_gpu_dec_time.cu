// ref_gpu_dec_time.cu -- the reference's own GPU decoder kernel, launched and
// timed.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY.  oracle/Makefile compiles this
// file with the reference's unmodified decoder/src/decoder.cu #included (read
// in place; nothing of it is copied here), together with its
// decoder/src/get_table.cpp, for sm_100a into oracle/_ref/libref_gpu_time.so.
// gpu_dec_l1_l2 (decoder/src/decoder.cu:454-730) is launched as
// decoder_l1_l2() does (:732-815: the same grid, block and table, the same
// memsets before it) minus its allocations, host copies and 200-fold loop.
//
// The reference decoder is run only where its own table is right: the caller
// gets -2 and nothing runs when get_table_info's level-1 boundary
// (decoder/src/get_table.cpp:20-27, taken from the next symbol's code)
// differs from the boundary get_twolevel_table derives (the LUT would send
// codes to the wrong level and index past the pointer table).  Its buffers
// follow its reads and writes past the stream (decoder.cu:529,560,716,763):
// the caller passes the gap array and bitstream back to back with >= 64
// spare bytes after them, and an output buffer of at least
// max(n + 512, 4 * (gap words + words)) + 4096 bytes.
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "decoder.cu"  // the reference: decoder/src/decoder.cu
#include "get_table.h"    // reference: decoder/include/get_table.h

extern "C" {

// d_input: ceil(S/8) gap words then W bitstream words (the container's order,
// decoder/src/huff.cpp:73-84).  syms/lens: the container-order symbol list.
// Per repetition r: ms[2r] the memsets decoder_l1_l2 issues before each
// launch (counter, output offsets, output), ms[2r+1] gpu_dec_l1_l2.
// Returns 0, -2 (the reference's level-1 boundary is wrong for this book: not
// run), or a CUDA error code.
int hgapref_gpu_decode_time(const uint32_t* d_input, uint32_t words, uint32_t n, uint32_t gap_elems,
                            const uint8_t* syms, const uint8_t* lens, int count, uint32_t* d_out,
                            size_t out_bytes, int reps, float* ms) {
    std::vector<struct Symbol> symbols(count > 0 ? count : 1);
    for (int i = 0; i < count; ++i) {
        symbols[i].symbol = syms[i];
        symbols[i].length = lens[i];
        symbols[i].num = 0;
    }
    struct TableInfo info;
    const unsigned int prefix_bit = get_table_info(symbols.data(), count, FIXED_PREFIX_BIT, info);
    const int table_size = (int)(sizeof(int) * info.ptrtable_size +
                                 (MAX_CODE_NUM + info.l1table_size + info.l2table_size));
    std::vector<unsigned char> table(table_size);
    const unsigned int boundary = get_twolevel_table(table.data(), prefix_bit, symbols.data(), count, info);
    if (boundary != info.l1table_size) return -2;
    const int gap_size = (gap_elems + GAP_FAC_NUM - 1) / GAP_FAC_NUM;
    const size_t memset_bytes = sizeof(int) * ((size_t)gap_size + words);  // as decoder.cu:763
    if (out_bytes < memset_bytes || out_bytes < (size_t)n + 512) return -3;
    void* d_table = nullptr;
    unsigned long long* d_pos = nullptr;
    int* d_counter = nullptr;
    if (cudaMalloc(&d_table, table_size) != cudaSuccess) return 1;
    if (cudaMalloc(reinterpret_cast<void**>(&d_pos), sizeof(unsigned long long) * ((size_t)gap_elems + 1)) !=
        cudaSuccess)
        return 1;
    if (cudaMalloc(reinterpret_cast<void**>(&d_counter), sizeof(int)) != cudaSuccess) return 1;
    cudaMemcpy(d_table, table.data(), table_size, cudaMemcpyHostToDevice);
    const int blocks = (gap_elems + NUM_THREADS - 1) / NUM_THREADS;
    cudaEvent_t e[3];
    for (auto& x : e) cudaEventCreate(&x);
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e[0], 0);
        cudaMemsetAsync(d_counter, 0, sizeof(int), 0);
        cudaMemsetAsync(d_pos, 0, sizeof(unsigned long long) * ((size_t)gap_elems + 1), 0);
        cudaMemsetAsync(d_out, 0, memset_bytes, 0);
        cudaEventRecord(e[1], 0);
        gpu_dec_l1_l2<<<blocks, NUM_THREADS, table_size>>>(
            (unsigned int*)d_input, (int)words, d_table, d_pos, (unsigned int*)d_input, (int)gap_elems, gap_size,
            d_out, (int)n, d_counter, table_size, prefix_bit, (unsigned int)count, info);
        cudaEventRecord(e[2], 0);
        cudaEventSynchronize(e[2]);
        cudaEventElapsedTime(&ms[2 * r + 0], e[0], e[1]);
        cudaEventElapsedTime(&ms[2 * r + 1], e[1], e[2]);
    }
    for (auto& x : e) cudaEventDestroy(x);
    cudaFree(d_table);
    cudaFree(d_pos);
    cudaFree(d_counter);
    const cudaError_t err = cudaDeviceSynchronize();
    return err == cudaSuccess ? 0 : static_cast<int>(err);
}

}  // extern "C"
