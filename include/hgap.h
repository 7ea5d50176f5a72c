/*
 * hgap.h -- C ABI of the B200 Huffman-with-gap-arrays library (libhgap.so).
 *
 * Drop-in for the hot path of daisuke-takafuji/Huffman_coding_Gap_arrays:
 * byte histogram -> length-limited canonical codebook -> bit-packing encoder
 * that emits the gap array -> segment-parallel decoder, in the reference's
 * compressed format.  Every entry point names the reference interface it
 * replaces.  Device entry points are stream-ordered, allocate nothing (the
 * caller passes a workspace sized by the *_workspace_bytes queries), never
 * exit the process, and return an hgap_status.
 *
 * Format (fixed by the reference, encoder/include/constants.hpp:4-12):
 *   - codewords of at most 16 bits, canonical, most frequent symbol first;
 *   - bitstream: u32 words, codes packed MSB first, last word zero-padded;
 *   - gap array: one 4-bit entry per 128-bit segment, eight per u32, low
 *     nibble first; entry k = bit offset of the first codeword that starts in
 *     segment k+1, relative to that segment's start (encoder/src/encoder.cu:307-312).
 *   - sizes: B code bits, W = ceil(B/32) words, S = ceil(B/128) segments,
 *     ceil(S/8) gap words (encoder/src/huff.cpp:84-88).
 */
#ifndef HGAP_H
#define HGAP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same type as cudaStream_t (struct CUstream_st*); 0 = the legacy default stream. */
typedef struct CUstream_st* hgap_stream_t;

typedef enum hgap_status {
    HGAP_OK = 0,
    HGAP_ERR_INVALID_ARG = 1,  /* bad pointer, size or alignment */
    HGAP_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    HGAP_ERR_TIMEOUT = 3,      /* a bounded inter-tile wait expired on the device */
    HGAP_ERR_CORRUPT = 4,      /* stream, gap array or codebook failed validation */
    HGAP_ERR_SIZE = 5,         /* sizes disagree (input vs. codebook vs. W/S) */
    HGAP_ERR_WORKSPACE = 6,    /* workspace too small */
    HGAP_ERR_NO_CODE = 7,      /* input byte without a codeword */
    HGAP_ERR_UNSUPPORTED = 8   /* valid request outside this build's limits */
} hgap_status;

#define HGAP_MAX_CODE_LEN 16
#define HGAP_SEGMENT_BITS 128
#define HGAP_GAPS_PER_WORD 8

/* Container entry, reference decoder/src/huff.cpp:45-52 ({u8 symbol, u8 length}). */
typedef struct hgap_symlen {
    uint8_t symbol;
    uint8_t length;
} hgap_symlen;

/* Reference struct Codetable (encoder/include/constants.hpp:40-43). */
typedef struct hgap_codeword {
    uint32_t code;
    uint32_t length; /* 0 = byte value absent from the book */
} hgap_codeword;

/* A codebook: the container-order symbol list (most frequent first, as the
 * reference writes it, encoder/src/huff.cpp:114-119) and the per-byte table. */
typedef struct hgap_codebook {
    uint32_t symbol_count;
    hgap_symlen symbols[256];
    hgap_codeword table[256];
} hgap_codebook;

typedef struct hgap_sizes {
    uint64_t bits;      /* B */
    uint64_t words;     /* W = ceil(B/32) */
    uint64_t segments;  /* S = ceil(B/128) */
    uint64_t gap_words; /* ceil(S/8) */
} hgap_sizes;

const char* hgap_status_string(hgap_status s);

/* ------------------------------------------------------------------ histogram
 * Replaces extern "C" histgram(unsigned *d_Histogram, unsigned *d_Data,
 * unsigned byteCount) (encoder/src/encoder.cu:118-140, decl
 * encoder/include/encoder.cuh:20-23).  d_in: any alignment; d_hist: 256 u32,
 * overwritten.  No scratch memory. */
hgap_status hgap_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, hgap_stream_t stream);

/* ------------------------------------------------------------------- codebook
 * Replaces store_symbols + qsort(compare) + boundary_PM + get_outputfilesize
 * (encoder/src/symbols.cpp:29-55, encoder/src/huff.cpp:17-21,77-88,
 * encoder/src/package_merge.cpp:107-182).  Byte-identical lengths, tie order
 * and codes.  One distinct symbol gets a 1-bit code (the reference is
 * undefined there); zero symbols give an empty book.  `sizes` may be NULL. */
hgap_status hgap_codebook_build(const uint32_t hist[256], hgap_codebook* cb, hgap_sizes* sizes);

/* Rebuilds the canonical codes from a container-order list (the decoder's
 * view, decoder/src/huff.cpp:140-152).  Rejects non-monotone lengths, lengths
 * outside 1..16 and over-full (Kraft sum > 1) books. */
hgap_status hgap_codebook_from_symbols(const hgap_symlen* symbols, uint32_t count,
                                       hgap_codebook* cb);

hgap_sizes hgap_sizes_from_bits(uint64_t bits);

/* B = sum(len[b] * hist[b]) in 64-bit arithmetic (get_outputfilesize,
 * encoder/src/symbols.cpp:45-55, whose u32 products overflow for huge counts). */
uint64_t hgap_encoded_bits(const hgap_codebook* cb, const uint32_t hist[256]);

/* --------------------------------------------------------------------- encode
 * Replaces void encode(unsigned* outputfile, unsigned outputfilesize,
 * unsigned* d_inputfile, unsigned inputfilesize, unsigned gap_elements,
 * Codetable* codetable) (encoder/src/encoder.cu:381-457, decl
 * encoder/include/encoder.cuh:12-18): device in, device out, no ownership
 * transfer, no pre-zeroing of the outputs.  `words` and `segments` are W and
 * S of the stream (hgap_sizes); d_bits gets W words, d_gaps ceil(S/8) words.
 * d_in: any alignment; d_bits/d_gaps: 4-byte aligned (16 for vector stores);
 * d_workspace: 16-byte aligned, hgap_encode_workspace_bytes(n) bytes.
 * Device-side errors are reported by hgap_workspace_status().
 *
 * The encoder cuts the input into super-tiles and needs each one's byte
 * histogram; the pipeline the reference runs (histgram, then encode,
 * encoder/src/huff.cpp:70-99) therefore maps to two calls that read the input
 * once each:
 *   hgap_encode_histogram  -- replaces histgram() in that pipeline: the global
 *                             histogram into d_hist AND the per-super-tile
 *                             histograms into the workspace;
 *   hgap_encode_prepared   -- the encoder proper, reusing them (same input,
 *                             same workspace; otherwise HGAP_ERR_INVALID_ARG
 *                             from hgap_workspace_status).
 * hgap_encode does both passes itself, for callers that only have the codebook. */
size_t hgap_encode_workspace_bytes(uint64_t n);
hgap_status hgap_encode_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, void* d_workspace,
                                  size_t workspace_bytes, hgap_stream_t stream);
hgap_status hgap_encode_prepared(const void* d_in, uint64_t n, const hgap_codebook* cb,
                                 uint32_t* d_bits, uint64_t words, uint32_t* d_gaps,
                                 uint64_t segments, void* d_workspace, size_t workspace_bytes,
                                 hgap_stream_t stream);
hgap_status hgap_encode(const void* d_in, uint64_t n, const hgap_codebook* cb, uint32_t* d_bits,
                        uint64_t words, uint32_t* d_gaps, uint64_t segments, void* d_workspace,
                        size_t workspace_bytes, hgap_stream_t stream);

/* One part of a stream split across devices (no counterpart in the reference):
 * each device encodes a contiguous byte range of one buffer.  The parts share
 * one codebook, built from the sum of the parts' histograms, and part p starts
 * at stream bit bit0 = the sum of the earlier parts' bit counts
 * (hgap_encoded_bits of each part's histogram: an exclusive scan of one 8-byte
 * value per device).  Call after hgap_encode_histogram on this part (same
 * input, same workspace).
 * d_bits is a window holding stream words [bits_word0, ceil((bit0 +
 * part_bits) / 32)), bits_word0 a multiple of 4 and <= bit0 / 32; d_gaps a
 * window holding gap words [gaps_word0, ceil(ceil((bit0 + part_bits) / 128) /
 * 8)), gaps_word0 <= bit0 / 1024.  Window words before bit0 / 32 (gap words
 * before bit0 / 1024) are not written.  The word holding bit0 and the one
 * holding the part's last bit carry only this part's bits (zeros elsewhere),
 * and the first and last gap words only this part's entries -- entry k
 * belongs to the part with bit0 < 128(k+1) <= bit0 + part_bits -- so the
 * whole stream is the OR of all parts' windows, word by word. */
hgap_status hgap_encode_part_prepared(const void* d_in, uint64_t n, const hgap_codebook* cb, uint64_t bit0,
                                      uint64_t part_bits, uint32_t* d_bits, uint64_t bits_word0,
                                      uint32_t* d_gaps, uint64_t gaps_word0, void* d_workspace,
                                      size_t workspace_bytes, hgap_stream_t stream);

/* --------------------------------------------------------------------- decode
 * Replaces void decoder_l1_l2(unsigned* input, int inputfilesize,
 * unsigned* output, int outputfilesize, int gap_elements, void* dectable,
 * int tablesize, unsigned prefix_bit, unsigned symbol_count, TableInfo)
 * (decoder/src/decoder.cu:732-815, decl decoder/include/decoder.cuh:4-15):
 * device in/out, gap array and bitstream as separate pointers, the two-level
 * table built internally from the codebook (with the correct level-1
 * boundary, see decoder/src/get_table.cpp:20 for the reference's).  Decodes
 * each 128-bit segment once, stops at exactly n symbols and checks every
 * segment's end against the next gap entry.  d_bits/d_gaps: 4-byte aligned;
 * d_out: any alignment. */
size_t hgap_decode_workspace_bytes(uint64_t segments);
hgap_status hgap_decode(const uint32_t* d_bits, uint64_t words, const uint32_t* d_gaps,
                        uint64_t segments, const hgap_codebook* cb, uint8_t* d_out, uint64_t n,
                        void* d_workspace, size_t workspace_bytes, hgap_stream_t stream);

/* Synchronizes `stream` and returns the device-side status of the last
 * hgap_encode / hgap_decode that used this workspace (HGAP_OK,
 * HGAP_ERR_TIMEOUT, HGAP_ERR_CORRUPT, HGAP_ERR_SIZE, HGAP_ERR_NO_CODE, or
 * HGAP_ERR_INVALID_ARG when hgap_encode_prepared got a workspace that was not
 * prepared by hgap_encode_histogram on the same input). */
hgap_status hgap_workspace_status(const void* d_workspace, hgap_stream_t stream);

/* The same status from the workspace's first 32-bit word, already copied to
 * the host by the caller (e.g. an asynchronous copy into pinned memory
 * ordered after the launch): no synchronization, no device access. */
hgap_status hgap_status_from_word(uint32_t word);

/* ------------------------------------------------------- bounded-wait hooks
 * No counterpart in the reference, whose look-back spins never give up
 * (encoder/src/encoder.cu:239-241, decoder/src/decoder.cu:615-632).  For
 * testing the bounded waits only: hgap_encode / hgap_decode, except that one
 * work item, `hold` (encoder: region, decoder: tile, numbered from 0 in stream
 * order), never publishes its look-back records, and every look-back wait
 * gives up after `wait_limit_ns` (0: the default of 0.5 s).  The items after
 * it wait for the withheld record until the limit, the kernel then finishes
 * with HGAP_ERR_TIMEOUT in the workspace status, and the output is void.
 * Every write stays inside the output buffers.  hold = UINT64_MAX withholds
 * nothing (the call is then hgap_encode / hgap_decode with that limit). */
hgap_status hgap_encode_hold(const void* d_in, uint64_t n, const hgap_codebook* cb, uint32_t* d_bits,
                             uint64_t words, uint32_t* d_gaps, uint64_t segments, void* d_workspace,
                             size_t workspace_bytes, hgap_stream_t stream, uint64_t hold,
                             uint64_t wait_limit_ns);
hgap_status hgap_decode_hold(const uint32_t* d_bits, uint64_t words, const uint32_t* d_gaps,
                             uint64_t segments, const hgap_codebook* cb, uint8_t* d_out, uint64_t n,
                             void* d_workspace, size_t workspace_bytes, hgap_stream_t stream, uint64_t hold,
                             uint64_t wait_limit_ns);

/* ------------------------------------------------- decode without allocation
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory at all (code inside a framework that owns every
 * device allocation through its own pool, plugins barred from allocating on
 * the hot path, language bindings that only pass the input and output
 * buffers).  Same arguments and results as hgap_decode minus the workspace:
 * the decoder's scratch is a fixed HGAP_NOALLOC_SCRATCH_BYTES array inside
 * libhgap.so, held by every GPU that loads the library until exit.  Streams
 * with hgap_decode_workspace_bytes(segments) > HGAP_NOALLOC_SCRATCH_BYTES are
 * rejected with HGAP_ERR_WORKSPACE before anything runs.  The call waits for
 * `stream` and returns the device-side status too.  The first call on each
 * device looks up the array's device address, which is kept for the life of
 * the process, so a cudaDeviceReset between calls (which unloads the
 * library's device code and may move the array) is not supported.  All calls share the one array: calls
 * that overlap on the GPU (other streams, other host threads) race and must
 * be serialized by the caller.  Allocates nothing. */
#define HGAP_NOALLOC_SCRATCH_BYTES (256u * 1024u)
hgap_status hgap_decode_noalloc(const uint32_t* d_bits, uint64_t words, const uint32_t* d_gaps,
                                uint64_t segments, const hgap_codebook* cb, uint8_t* d_out,
                                uint64_t n, hgap_stream_t stream);

/* ---------------------------------------------------- codebooks on the device
 * No counterpart in the reference (its device-side attempt,
 * decoder/src/decoder.cu:36-88, is unfinished): the host builder
 * hgap_codebook_build run on the GPU, one warp per book, with identical
 * results (stable order by count, package-merge with the same tie rule,
 * canonical codes).  d_hists: count x 256 counts; d_books: count codebooks;
 * d_sizes: count sizes (may be NULL).  Stream-ordered, allocates nothing. */
hgap_status hgap_codebook_build_device(uint32_t count, const uint32_t* d_hists, hgap_codebook* d_books,
                                       hgap_sizes* d_sizes, hgap_stream_t stream);

/* The decoder's two-level table (level 1: 2^11 u16 entries, level 2: 2560
 * u16 entries) from a codebook, on the host and on the device (one warp per
 * book).  Exposed so the two builders can be checked against each other. */
#define HGAP_DEC_T1_ENTRIES 2048
#define HGAP_DEC_T2_ENTRIES 2560
hgap_status hgap_decode_table_build(const hgap_codebook* cb, uint16_t* t1, uint16_t* t2);
hgap_status hgap_decode_table_build_device(uint32_t count, const hgap_codebook* d_books, uint16_t* d_tables,
                                           uint32_t* d_status, hgap_stream_t stream);

/* -------------------------------------------------------------- batched path
 * No counterpart in the reference.  Thousands of independent buffers, each
 * with its own codebook built on the device, compressed or decompressed by a
 * fixed sequence of persistent launches that never returns to the host (so
 * it can be captured in a CUDA graph).  Each buffer keeps the reference's
 * format: the bitstream and gap array of buffer i are exactly what
 * hgap_encode would write for it with the book hgap_codebook_build makes
 * from its histogram.
 *
 * Outputs of hgap_batch_compress: the bitstreams, packed into one bits arena
 * (each starting 16-byte aligned), the gap arrays packed into one gaps arena,
 * and one hgap_batch_entry per buffer in device memory with its sizes,
 * offsets and codebook (container order).  hgap_batch_decompress takes the
 * same arenas and entries back. */
typedef struct hgap_batch_entry {
    uint64_t n;            /* uncompressed bytes */
    uint64_t bits;         /* code bits */
    uint64_t words;        /* W */
    uint64_t segments;     /* S */
    uint64_t gap_words;    /* ceil(S / 8) */
    uint64_t bits_offset;  /* word offset of the bitstream in the bits arena */
    uint64_t gaps_offset;  /* word offset of the gap array in the gaps arena */
    uint32_t symbol_count;
    uint32_t status;       /* 0, or an hgap_status for this buffer (e.g. arena too small) */
    hgap_symlen symbols[256]; /* container order: most frequent first */
} hgap_batch_entry;

/* Launch shape; every choice leaves the output format unchanged. */
typedef struct hgap_batch_config {
    uint32_t region_chunks;    /* encoder region = region_chunks x 8 KiB (1..32; 0 = 8) */
    uint32_t hist_ctas_per_sm; /* persistent grids, CTAs per SM (0 = occupancy maximum) */
    uint32_t enc_ctas_per_sm;
    uint32_t dec_ctas_per_sm;
    uint32_t dec_tile_segs;    /* decoder tile, 256 or 512 segments (0 = by the book's shortest
                                  code: 512 from 3 bits up, 256 below); books with a 1-bit code
                                  always take 256 */
    uint32_t dec_class_mask;   /* decoder classes hgap_batch_decompress launches: bit k as
                                  hgap_batch_decoder_class numbers them; 0 = all 8.  For callers
                                  that know their books on the host: an empty class then costs
                                  no launch.  A buffer whose class is left out is not decoded
                                  and the call's status is HGAP_ERR_INVALID_ARG. */
} hgap_batch_config;

/* The decoder class of a buffer from its container-order symbol list (as in
 * hgap_batch_entry): 2 * s + c, where s = 0, 1, 2, 3 for a shortest code of
 * 4 bits or more, 3, 2 and 1 bits, and c = 1 for a complete book (Kraft sum
 * 1); 255 for an empty list.  The class picks the decoder's stage size. */
uint32_t hgap_batch_decoder_class(const hgap_symlen* symbols, uint32_t count);

/* Worst-case sizes from the uncompressed sizes (host array). */
size_t hgap_batch_compress_workspace_bytes(uint32_t count, const uint64_t* sizes,
                                           const hgap_batch_config* cfg);
size_t hgap_batch_decompress_workspace_bytes(uint32_t count, const uint64_t* sizes);
uint64_t hgap_batch_bits_capacity(uint32_t count, const uint64_t* sizes);  /* words */
uint64_t hgap_batch_gaps_capacity(uint32_t count, const uint64_t* sizes);  /* words */

/* d_inputs / d_sizes: device arrays of count input pointers and sizes.
 * d_region_chunks: optional device array of per-buffer region sizes (in 8 KiB
 * chunks, raised to cfg->region_chunks at least); NULL = cfg for all.
 * Workspace 16-byte aligned, from hgap_batch_compress_workspace_bytes with
 * the same sizes and cfg. */
hgap_status hgap_batch_compress(uint32_t count, const uint8_t* const* d_inputs, const uint64_t* d_sizes,
                                const uint8_t* d_region_chunks, uint32_t* d_bits, uint64_t bits_capacity,
                                uint32_t* d_gaps, uint64_t gaps_capacity, hgap_batch_entry* d_entries,
                                void* d_workspace, size_t workspace_bytes, const hgap_batch_config* cfg,
                                hgap_stream_t stream);
/* d_outputs: device array of count output pointers (entry i's n bytes each). */
hgap_status hgap_batch_decompress(uint32_t count, const hgap_batch_entry* d_entries, const uint32_t* d_bits,
                                  const uint32_t* d_gaps, uint8_t* const* d_outputs, void* d_workspace,
                                  size_t workspace_bytes, const hgap_batch_config* cfg, hgap_stream_t stream);
/* Waits for `stream`; the device status of the last batched call that used
 * this workspace, like hgap_workspace_status. */
hgap_status hgap_batch_status(const void* d_workspace, hgap_stream_t stream);

/* --------------------------------------------------------- learned launch tuner
 * No counterpart in the reference.  A small MLP (10 inputs -> 32 ReLU -> 32
 * ReLU -> 2 outputs, fp32) that predicts the log times of the batched
 * compress and decompress from a batch's features and a launch shape,
 * trained and run on the GPU by these kernels.  Parameters: one flat array of
 * HGAP_MLP_PARAMS floats, W1[32][10] b1[32] W2[32][32] b2[32] W3[2][32] b3[2].
 * d_x: n x 10 inputs, d_y / d_target: n x 2 (NaN targets are unmeasured and
 * carry no loss).  loss = scale * sum (y - t)^2 / 2; hgap_mlp_loss_grad
 * overwrites d_grad (HGAP_MLP_PARAMS floats) and *d_loss.  Adam with bias
 * correction for step >= 1, on the gradient plus weight_decay * params. */
#define HGAP_MLP_IN 10
#define HGAP_MLP_HIDDEN 32
#define HGAP_MLP_OUT 2
#define HGAP_MLP_PARAMS (HGAP_MLP_HIDDEN * HGAP_MLP_IN + HGAP_MLP_HIDDEN + HGAP_MLP_HIDDEN * HGAP_MLP_HIDDEN + \
                         HGAP_MLP_HIDDEN + HGAP_MLP_OUT * HGAP_MLP_HIDDEN + HGAP_MLP_OUT)
hgap_status hgap_mlp_forward(const float* d_params, const float* d_x, uint32_t n, float* d_y,
                             hgap_stream_t stream);
hgap_status hgap_mlp_loss_grad(const float* d_params, const float* d_x, const float* d_target, uint32_t n,
                               float scale, float* d_grad, float* d_loss, hgap_stream_t stream);
hgap_status hgap_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, uint32_t step,
                          float lr, float beta1, float beta2, float eps, float weight_decay,
                          hgap_stream_t stream);

/* ------------------------------------------------------------------ container
 * Writer encoder/src/huff.cpp:111-125, reader decoder/src/huff.cpp:27-81:
 * u64 symbol_count; symbol_count x {u8 symbol, u8 length}; u32 n; u32 W;
 * u32 S; u32 gap[ceil(S/8)]; u32 bits[W]; little-endian, unaligned. */
size_t hgap_container_bytes(uint32_t symbol_count, uint64_t words, uint64_t segments);
hgap_status hgap_container_write(void* dst, size_t capacity, const hgap_codebook* cb, uint64_t n,
                                 uint64_t words, uint64_t segments, const uint32_t* gaps,
                                 const uint32_t* bits, size_t* written);
/* Parses and validates a container held in host memory; `gaps`/`bits` point
 * into `src` (unaligned). */
hgap_status hgap_container_parse(const void* src, size_t size, hgap_codebook* cb, uint64_t* n,
                                 uint64_t* words, uint64_t* segments, const void** gaps,
                                 const void** bits);

/* ------------------------------------------------ reference-signature entries
 * Same arguments and semantics as the reference's own functions, host-side
 * and synchronous like them, so the reference's bin/encoder and bin/decoder
 * mains link against this library unchanged (see include/hgap_ref_compat.h
 * for the C++-linkage forwarders).  Errors print and return instead of
 * exit(). */

/* encoder/src/encoder.cu:118-140: d_Data holds ceil(byteCount/4) words. */
void histgram(unsigned int* d_Histogram, unsigned int* d_Data, unsigned int byteCount);

/* encoder/src/encoder.cu:381-457: writes outputfilesize bitstream words then
 * ceil(gap_array_elements_num/8) gap words into the (pinned) host buffer
 * outputfile, and frees d_inputfile like the reference (encoder.cu:451). */
hgap_status hgap_ref_encode(unsigned int* outputfile, unsigned int outputfilesize,
                            unsigned int* d_inputfile, unsigned int inputfilesize,
                            unsigned int gap_array_elements_num, const hgap_codeword* codetable);

/* decoder/src/decoder.cu:732-815 minus the 200-iteration timing loop: input =
 * host gap array followed by the bitstream (inputfilesize words), output =
 * host buffer of ceil(outputfilesize/4) words.  The reference LUT blob
 * (decoder/src/get_table.cpp:48-139 layout) is read back into a codebook;
 * the l1 boundary in tableinfo is ignored (the reference's can be wrong,
 * get_table.cpp:20) and recomputed. */
hgap_status hgap_ref_decoder_l1_l2(unsigned int* input, int inputfilesize, unsigned int* output,
                                   int outputfilesize, int gap_elements_num, const void* dectable,
                                   int tablesize, unsigned int prefix_bit,
                                   unsigned int symbol_count, uint32_t l1table_size,
                                   uint32_t l2table_size, uint32_t ptrtable_size);

#ifdef __cplusplus
}
#endif
#endif /* HGAP_H */
