/*
 * hgap_ref_compat.h -- C++-linkage forwarders with the reference's exact
 * encode() / decoder_l1_l2() signatures, for building the reference's own
 * mains (encoder/src/huff.cpp, decoder/src/huff.cpp) on libhgap.so.
 *
 * The reference declares these with C++ linkage (encoder/include/encoder.cuh:12-18,
 * decoder/include/decoder.cuh:4-15) and its own struct Codetable / struct
 * TableInfo (encoder/include/constants.hpp:40-43, decoder/include/constants.hpp:53-57).
 * Include this header AFTER the reference's constants.hpp in the one
 * translation unit that replaces encoder.cu / decoder.cu:
 *
 *     #include "constants.hpp"          // reference types
 *     #define HGAP_REF_ENCODER          // and/or HGAP_REF_DECODER
 *     #include "hgap_ref_compat.h"
 *
 * histgram() needs no forwarder: libhgap.so exports it with the reference's
 * extern "C" signature (encoder/src/encoder.cu:118).
 */
#ifndef HGAP_REF_COMPAT_H
#define HGAP_REF_COMPAT_H

#include "hgap.h"

#ifdef __cplusplus

#ifdef HGAP_REF_ENCODER
static_assert(sizeof(struct Codetable) == sizeof(hgap_codeword),
              "reference Codetable is {u32 code, u32 length}");
/* encoder/src/encoder.cu:381-388 */
void encode(unsigned int* outputfile, unsigned int outputfilesize, unsigned int* inputfile,
            unsigned int inputfilesize, unsigned int gap_array_elements_num,
            struct Codetable* codetable) {
    hgap_ref_encode(outputfile, outputfilesize, inputfile, inputfilesize, gap_array_elements_num,
                    reinterpret_cast<const hgap_codeword*>(codetable));
}
#endif

#ifdef HGAP_REF_DECODER
/* decoder/src/decoder.cu:732-743 */
void decoder_l1_l2(unsigned int* input, int inputfilesize, unsigned int* output, int outputfilesize,
                   int gap_element_num, void* dectable, int tablesize, unsigned int prefix_bit,
                   unsigned int symbol_count, struct TableInfo tableinfo) {
    hgap_ref_decoder_l1_l2(input, inputfilesize, output, outputfilesize, gap_element_num, dectable,
                           tablesize, prefix_bit, symbol_count, tableinfo.l1table_size,
                           tableinfo.l2table_size, tableinfo.ptrtable_size);
}
#endif

#endif /* __cplusplus */
#endif /* HGAP_REF_COMPAT_H */
