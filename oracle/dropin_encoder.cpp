// dropin_encoder.cpp -- replaces the reference's encoder/src/encoder.cu when
// the reference's own bin/encoder main (encoder/src/huff.cpp, unmodified) is
// linked against libhgap.so (recipe: oracle/Makefile, target `dropin`).
// Test infrastructure: it demonstrates the drop-in boundary end to end.
#include "constants.hpp"  // reference: struct Codetable
#define HGAP_REF_ENCODER
#include "hgap_ref_compat.h"
