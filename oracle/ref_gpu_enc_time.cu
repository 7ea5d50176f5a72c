// ref_gpu_enc_time.cu -- the reference's own GPU histogram and encoder
// kernels, launched and timed one by one.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY.  oracle/Makefile compiles this
// file with the reference's unmodified encoder/src/encoder.cu #included (read
// in place; nothing of it is copied here) for sm_100a into
// oracle/_ref/libref_gpu_time.so.  It is the "plain reference on B200"
// measurement: cu_histgram + mergeHistogram (encoder/src/encoder.cu:33-116,
// launched as histgram() does, :118-140, minus its per-call cudaMalloc and
// cudaFree) and cuencoder + cu_get_gaparray (:142-379, launched as encode()
// does, :381-457, minus its allocations and host copies), every kernel and
// the memsets the reference needs before them bracketed by CUDA events on the
// legacy default stream, which is where the reference launches them.
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "encoder.cu"  // the reference: encoder/src/encoder.cu

namespace {

struct Events {
    cudaEvent_t e[6];
    Events() {
        for (auto& x : e) cudaEventCreate(&x);
    }
    ~Events() {
        for (auto& x : e) cudaEventDestroy(x);
    }
    float ms(int a, int b) const {
        float t = 0;
        cudaEventElapsedTime(&t, e[a], e[b]);
        return t;
    }
};

}  // namespace

extern "C" {

// The reference histogram kernels on `d_in` (n bytes; the buffer must hold
// ceil(n / 4) whole words), `reps` times.  d_hist receives the 256 counts.
// ms[2 * r + 0]: cu_histgram, ms[2 * r + 1]: mergeHistogram of repetition r.
// Returns 0 or a CUDA error code.
int hgapref_gpu_histogram_time(const void* d_in, uint32_t n, uint32_t* d_hist, int reps, float* ms) {
    unsigned int* partial = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&partial), sizeof(int) * HIST_BLOCK * HIST_SIZE) != cudaSuccess)
        return 1;
    const unsigned int data_count = (n + 3) / 4;
    Events ev;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(ev.e[0], 0);
        cu_histgram<<<HIST_BLOCK, HIST_THREADS>>>(partial, (unsigned int*)d_in, data_count, n);
        cudaEventRecord(ev.e[1], 0);
        mergeHistogram<<<HIST_SIZE, MERGE_THREADBLOCK_SIZE>>>(d_hist, partial, HIST_BLOCK);
        cudaEventRecord(ev.e[2], 0);
        cudaEventSynchronize(ev.e[2]);
        ms[2 * r + 0] = ev.ms(0, 1);
        ms[2 * r + 1] = ev.ms(1, 2);
    }
    cudaFree(partial);
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : static_cast<int>(e);
}

// The reference encoder kernels, `reps` times: d_in holds n input bytes plus
// at least 8 KiB of zeroed slack (cuencoder's idle threads of the last tile
// read their first word before testing the length, encoder.cu:183);
// code/len: the per-byte codetable; out_words = W, gap_elems = S (as
// encoder/src/huff.cpp:84-88 computes them).  d_bits (W words) and d_gaps
// (ceil(S/8) words) receive the stream.  Per repetition r:
// ms[3r]: the memsets encode() issues (output, look-back sums, gap entries,
// counter), ms[3r+1]: cuencoder, ms[3r+2]: cu_get_gaparray.
int hgapref_gpu_encode_time(const void* d_in, uint32_t n, const uint32_t* code, const uint32_t* len,
                            uint32_t out_words, uint32_t gap_elems, uint32_t* d_bits, uint32_t* d_gaps, int reps,
                            float* ms) {
    struct Codetable table[MAX_CODE_NUM];
    for (int b = 0; b < MAX_CODE_NUM; ++b) {
        table[b].code = code[b];
        table[b].length = len[b];
    }
    const unsigned int gap_size = (gap_elems + GAP_ELEMENTS_NUM - 1) / GAP_ELEMENTS_NUM;
    const unsigned int block_num = (n + THREAD_ELEMENT * THREAD_NUM - 1) / (THREAD_ELEMENT * THREAD_NUM);
    struct Codetable* d_table = nullptr;
    unsigned long long* d_sums = nullptr;
    unsigned int* d_gap_bytes = nullptr;
    unsigned int* d_counter = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&d_table), sizeof(table)) != cudaSuccess) return 1;
    if (cudaMalloc(reinterpret_cast<void**>(&d_sums), sizeof(unsigned long long) * (block_num + 1)) != cudaSuccess)
        return 1;
    if (cudaMalloc(reinterpret_cast<void**>(&d_gap_bytes), sizeof(unsigned int) * (gap_elems + 1)) != cudaSuccess)
        return 1;
    if (cudaMalloc(reinterpret_cast<void**>(&d_counter), sizeof(unsigned int)) != cudaSuccess) return 1;
    cudaMemcpy(d_table, table, sizeof(table), cudaMemcpyHostToDevice);
    const unsigned int gap_blocks = (gap_size + GAP_THREADS - 1) / GAP_THREADS;
    Events ev;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(ev.e[0], 0);
        cudaMemsetAsync(d_bits, 0, sizeof(int) * out_words, 0);
        cudaMemsetAsync(d_sums, 0, sizeof(unsigned long long) * block_num, 0);
        cudaMemsetAsync(d_gap_bytes, 0, sizeof(int) * gap_elems, 0);
        cudaMemsetAsync(d_counter, 0, sizeof(int), 0);
        cudaEventRecord(ev.e[1], 0);
        cuencoder<<<BLOCKNUM, THREAD_NUM>>>(d_bits, out_words, (unsigned int*)d_in, n, d_table, d_sums, d_gap_bytes,
                                            gap_elems, d_counter);
        cudaEventRecord(ev.e[2], 0);
        cu_get_gaparray<<<gap_blocks, GAP_THREADS>>>(d_gap_bytes, d_gaps, gap_elems, gap_size);
        cudaEventRecord(ev.e[3], 0);
        cudaEventSynchronize(ev.e[3]);
        ms[3 * r + 0] = ev.ms(0, 1);
        ms[3 * r + 1] = ev.ms(1, 2);
        ms[3 * r + 2] = ev.ms(2, 3);
    }
    cudaFree(d_table);
    cudaFree(d_sums);
    cudaFree(d_gap_bytes);
    cudaFree(d_counter);
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : static_cast<int>(e);
}

}  // extern "C"
