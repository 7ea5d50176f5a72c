// dec_entry.cuh -- the decoder's level-1 entries in the u32 form the decode
// kernel keeps in shared memory, widened from the u16 table (DecTable).  Used
// by the decode kernel (single path: widened once per CTA) and by the batched
// path's per-buffer table build (bdec_table_kernel: widened once per buffer,
// copied per tile).
#pragma once

#include "hgap_internal.h"

namespace hgap {

// Table entry in shared memory (u32): direct = len << 24 | symbol;
// pointer = bit 31 | extra width << 16 | level-2 offset; invalid = bit 30;
// pair (level 1 only, see widen_pair) = two symbols with bit 16 set.
__device__ __forceinline__ uint32_t widen_entry(uint32_t e) {
    if (e & 0x8000u) return 0x80000000u | (((e >> 12) & 7u) << 16) | (e & 0xfffu);
    if (e & kDecInvalid) return 0x40000000u;
    return ((((e >> 8) & 15u) + 1u) << 24) | (e & 0xffu);
}

// Level-1 entry in shared memory for prefix x, from the u16 table: when the
// first code leaves room for a whole second code inside the same 11-bit
// window, both are returned at once (a pair entry: symbol 1 | symbol 2 << 8 |
// bit 16 | length 1 << 17 | total length << 24).  The second code is known
// from the bits after the first alone, because it ends inside the window.
__device__ __forceinline__ uint32_t widen_pair(const uint16_t* t1src, uint32_t x) {
    const uint32_t e = widen_entry(t1src[x]);
    if (e & 0xC0000000u) return e;  // pointer or invalid
    const uint32_t l1 = e >> 24;
    if (l1 >= (uint32_t)kDecPrefix) return e;
    const uint32_t e2 = widen_entry(t1src[(x << l1) & ((1u << kDecPrefix) - 1u)]);
    if (e2 & 0xC0000000u) return e;
    const uint32_t l2 = e2 >> 24;
    if (l1 + l2 > (uint32_t)kDecPrefix) return e;
    return (e & 0xffu) | ((e2 & 0xffu) << 8) | 0x10000u | (l1 << 17) | ((l1 + l2) << 24);
}

// Level-1 entry for a complete book (multi entry): up to three codes that
// fit the 11-bit window at once -- symbol 1 | symbol 2 << 8 | symbol 3 << 16 |
// total length << 24 | (count - 1) << 29; a pointer entry stays as is.  A
// level-2 result (length <= 16 in bits 24-28) reads as a one-symbol entry.
__device__ __forceinline__ uint32_t widen_multi(const uint16_t* t1src, uint32_t x) {
    constexpr uint32_t mask = (1u << kDecPrefix) - 1u;
    const uint32_t e = widen_entry(t1src[x]);
    if (e & 0xC0000000u) return e;
    const uint32_t l1 = e >> 24;
    if (l1 >= (uint32_t)kDecPrefix) return e;
    const uint32_t e2 = widen_entry(t1src[(x << l1) & mask]);
    if (e2 & 0xC0000000u) return e;
    const uint32_t l12 = l1 + (e2 >> 24);
    if (l12 > (uint32_t)kDecPrefix) return e;
    const uint32_t two = (e & 0xffu) | ((e2 & 0xffu) << 8) | (l12 << 24) | (1u << 29);
    if (l12 >= (uint32_t)kDecPrefix) return two;
    const uint32_t e3 = widen_entry(t1src[(x << l12) & mask]);
    if (e3 & 0xC0000000u) return two;
    const uint32_t l123 = l12 + (e3 >> 24);
    if (l123 > (uint32_t)kDecPrefix) return two;
    return (e & 0xffu) | ((e2 & 0xffu) << 8) | ((e3 & 0xffu) << 16) | (l123 << 24) | (2u << 29);
}

// Length of the first code at prefix x (0 where it is longer than the prefix).
__device__ __forceinline__ uint8_t first_len(const uint16_t* t1src, uint32_t x) {
    const uint32_t e = widen_entry(t1src[x]);
    return (uint8_t)(e & 0xC0000000u ? 0u : e >> 24);
}

}  // namespace hgap
