/*
 * hgap_oracle.h -- CPU oracle for Huffman coding with gap arrays.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (daisuke-takafuji/Huffman_coding_Gap_arrays) used as the checker
 * for the CUDA library: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it.  The product path never calls it.
 *
 * Parity pin: the codebook and LUT halves are checked against the
 * reference's own host sources compiled unmodified into oracle/_ref
 * (tests/test_oracle_pin.py); the bitstream/gap-array half is checked against
 * golden containers produced by the reference's own GPU encoder
 * (tests/golden/, generated by tests/golden/make_golden.py).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef HGAP_ORACLE_H
#define HGAP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_LEN 16     /* MAX_CODEWORD_LENGTH, encoder/include/constants.hpp:5 */
#define ORC_SEGMENT 128    /* SEGMENTSIZE, encoder/include/constants.hpp:12 */
#define ORC_GAPS_PER_WORD 8 /* GAP_ELEMENTS_NUM, encoder/include/constants.hpp:10 */

/* One entry of the symbol list: reference struct Symbol
 * (encoder/include/constants.hpp:34-38). */
typedef struct {
    uint8_t symbol;
    uint8_t length;
    uint32_t count;
} orc_symbol;

/* Sizes of an encoded stream (encoder/src/huff.cpp:84-88). */
typedef struct {
    uint64_t bits;       /* B: total code bits */
    uint64_t words;      /* W = ceil(B/32): bitstream u32 words */
    uint64_t segments;   /* S = ceil(B/128): gap elements */
    uint64_t gap_words;  /* G = ceil(S/8): packed gap u32 words */
} orc_sizes;

/* Reference TableInfo (decoder/include/constants.hpp:53-57). */
typedef struct {
    uint32_t l1table_size;
    uint32_t l2table_size;
    uint32_t ptrtable_size;
} orc_table_info;

/* ---- histogram: encoder/src/symbols.cpp:18-27 (serial), encoder/src/encoder.cu:33-116 (GPU) */
void orc_histogram(const uint8_t* in, uint64_t n, uint32_t hist[256]);

/* ---- codebook: store_symbols (encoder/src/symbols.cpp:29-43), qsort(compare)
 * (encoder/src/huff.cpp:17-21,78-79), boundary_PM (encoder/src/package_merge.cpp:107-182).
 * Fills `sorted` (ascending by count, ties by symbol value) with lengths and
 * returns the number of distinct symbols.  code[]/len[] are indexed by byte
 * value (reference struct Codetable, encoder/include/constants.hpp:40-43).
 * Defined for every count: 0 symbols -> empty book; 1 symbol -> length 1,
 * code 0 (the reference is undefined there, package_merge.cpp:113-132). */
int orc_codebook(const uint32_t hist[256], orc_symbol sorted[256],
                 uint32_t code[256], uint32_t len[256]);

/* Canonical code assignment from a list in container order (most frequent
 * first), boundary_PM tail encoder/src/package_merge.cpp:168-181 and the
 * decoder's identical walk decoder/src/get_table.cpp:20,300. */
void orc_canonical_codes(const uint8_t* symbols, const uint8_t* lengths, int count,
                         uint32_t code[256], uint32_t len[256]);

/* get_outputfilesize (encoder/src/symbols.cpp:45-55) + huff.cpp:84-88. */
orc_sizes orc_sizes_for(const orc_symbol* sorted, int count);
orc_sizes orc_sizes_from_bits(uint64_t bits);

/* ---- encoder: bit order and padding of cuencoder (encoder/src/encoder.cu:279-347),
 * gap semantics (encoder/src/encoder.cu:307-312) and nibble packing of
 * cu_get_gaparray (encoder/src/encoder.cu:357-379).
 * Writes exactly sz.words bitstream words and sz.gap_words gap words. */
int orc_encode(const uint8_t* in, uint64_t n, const uint32_t code[256], const uint32_t len[256],
               uint32_t* bits, uint64_t words, uint32_t* gaps, uint64_t gap_words,
               uint64_t* bits_out);

/* Encode one chunk starting at an absolute bit position: the threaded CPU
 * baseline builds on it.  Writes words [first_bit/32, ceil(end/32)) of `bits`
 * by OR (caller zeroes), and ORs the gap nibbles the chunk's codes produce
 * into `gaps` (caller zeroes).  Returns the chunk's bit count. */
uint64_t orc_encode_chunk(const uint8_t* in, uint64_t n, const uint32_t code[256],
                          const uint32_t len[256], uint64_t first_bit,
                          uint32_t* bits, uint32_t* gaps);

/* ---- decoder: per-segment decode of gpu_dec_l1_l2 (decoder/src/decoder.cu:501-569,655-728),
 * restated with canonical (first-code, limit) decoding instead of the LUT,
 * with the shift-by-32 case made explicit and termination at n symbols.
 * Every segment is decoded from its own gap offset and checked against the
 * next segment's gap.  Returns 0 on success, a negative value on a corrupt
 * stream. */
int orc_decode(const uint32_t* bits, uint64_t words, const uint32_t* gaps, uint64_t segments,
               const uint8_t* symbols, const uint8_t* lengths, int count,
               uint8_t* out, uint64_t n);

/* Decode segments [s0, s1) into `out` (capacity cap); returns the number of
 * symbols produced (the last segment of the stream stops at end_bit), or a
 * negative value on a corrupt stream.  Used by the threaded CPU baseline. */
int64_t orc_decode_segments(const uint32_t* bits, uint64_t words, const uint32_t* gaps,
                            uint64_t segments, uint64_t s0, uint64_t s1,
                            const uint8_t* symbols, const uint8_t* lengths, int count,
                            uint8_t* out, uint64_t cap);

/* ---- reference two-level LUT (decoder/src/get_table.cpp).
 * orc_ref_table_info restates get_table_info (get_table.cpp:3-46) exactly,
 * including its off-by-one-code boundary when `reference_bug` != 0; with
 * reference_bug == 0 it returns the boundary get_twolevel_table computes
 * (get_table.cpp:93-95).  Returns the prefix width used. */
uint32_t orc_ref_table_info(const uint8_t* symbols, const uint8_t* lengths, int count,
                            uint32_t prefix_bit, orc_table_info* info, int reference_bug);
/* get_twolevel_table (get_table.cpp:48-139): blob layout
 * [ptr u32 x P][length u8 x 256][l1 u8 x L1][l2 u8 x L2].  Returns the boundary code. */
uint32_t orc_ref_twolevel_table(void* blob, uint32_t prefix_bit, const uint8_t* symbols,
                                const uint8_t* lengths, int count, orc_table_info info);
size_t orc_ref_table_bytes(orc_table_info info);

/* ---- container (writer encoder/src/huff.cpp:111-125, reader decoder/src/huff.cpp:27-81) */
size_t orc_container_bytes(int count, uint64_t words, uint64_t gap_words);
size_t orc_container_write(uint8_t* dst, const uint8_t* symbols, const uint8_t* lengths, int count,
                           uint32_t n, uint32_t words, uint32_t segments,
                           const uint32_t* gaps, const uint32_t* bits);
/* Parses the header; returns 0 and fills the outputs (pointers into src), or
 * a negative value if the buffer is truncated or inconsistent. */
int orc_container_parse(const uint8_t* src, size_t size, int* count, const uint8_t** symlens,
                        uint32_t* n, uint32_t* words, uint32_t* segments,
                        const uint8_t** gaps, const uint8_t** bits);

/* ---- threaded CPU baseline (same format; pthreads over chunks / segment ranges) */
int orc_mt_encode(const uint8_t* in, uint64_t n, const uint32_t code[256], const uint32_t len[256],
                  uint32_t* bits, uint64_t words, uint32_t* gaps, uint64_t gap_words, int threads);
int orc_mt_histogram(const uint8_t* in, uint64_t n, uint32_t hist[256], int threads);
int orc_mt_decode(const uint32_t* bits, uint64_t words, const uint32_t* gaps, uint64_t segments,
                  const uint8_t* symbols, const uint8_t* lengths, int count,
                  uint8_t* out, uint64_t n, int threads);

#ifdef __cplusplus
}
#endif
#endif
