// ref_decoder_shim.cpp -- extern "C" entry points into the reference decoder's
// host-side LUT builder.
//
// TEST INFRASTRUCTURE ONLY.  Compiled with the reference's unmodified
// decoder/src/get_table.cpp (read in place by oracle/Makefile) into
// oracle/_ref/libref_decoder_host.so, so the tests can compare the oracle's
// restatement of the two-level table against the reference's own bytes.
#include <cstdint>
#include <cstring>

#include "constants.hpp"  // reference: decoder/include/constants.hpp
#include "get_table.h"    // reference: get_table_info(), get_twolevel_table()

extern "C" {

// decoder/src/huff.cpp:50-69 without the timing loop: get_table_info on the
// container-order list, then get_twolevel_table into `blob` (capacity
// `blob_cap`).  info_out receives {l1table_size, l2table_size, ptrtable_size}.
// Returns the prefix width, or -1 if the reference's own sizes exceed blob_cap
// (the table is then not built).
int hgapref_twolevel_table(const uint8_t* syms, const uint8_t* lens, int count, int prefix_bit,
                           uint32_t* info_out, uint8_t* blob, uint64_t blob_cap,
                           uint32_t* boundary_out) {
    struct Symbol symbols[MAX_CODE_NUM];
    std::memset(symbols, 0, sizeof(symbols));
    for (int i = 0; i < count; ++i) {
        symbols[i].symbol = syms[i];
        symbols[i].length = lens[i];
    }
    struct TableInfo info;
    const unsigned int prefix = get_table_info(symbols, count, prefix_bit, info);
    info_out[0] = info.l1table_size;
    info_out[1] = info.l2table_size;
    info_out[2] = info.ptrtable_size;
    const uint64_t size = sizeof(int) * (uint64_t)info.ptrtable_size +
                          (uint64_t)(MAX_CODE_NUM + info.l1table_size + info.l2table_size);
    if (size > blob_cap) return -1;
    std::memset(blob, 0, size);
    *boundary_out = get_twolevel_table(blob, prefix, symbols, count, info);
    return static_cast<int>(prefix);
}

}  // extern "C"
