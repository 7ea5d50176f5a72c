// dropin_decoder.cpp -- replaces the reference's decoder/src/decoder.cu when
// the reference's own bin/decoder main (decoder/src/huff.cpp, unmodified) is
// linked against libhgap.so (recipe: oracle/Makefile, target `dropin`).
// Test infrastructure: it demonstrates the drop-in boundary end to end.
#include "constants.hpp"  // reference: struct TableInfo
#define HGAP_REF_DECODER
#include "hgap_ref_compat.h"
