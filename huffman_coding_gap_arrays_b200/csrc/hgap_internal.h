// hgap_internal.h -- types shared by the host code and the sm_100a kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/hgap.h"

namespace hgap {

// ---------------------------------------------------------------- format ---
constexpr int kMaxLen = HGAP_MAX_CODE_LEN;  // encoder/include/constants.hpp:5
constexpr int kSegBits = HGAP_SEGMENT_BITS; // encoder/include/constants.hpp:12

// ------------------------------------------------------- device status bits -
// OR-ed into the workspace status word by the kernels; read back by
// hgap_workspace_status().  No kernel traps: every failure is a bit here.
enum : uint32_t {
    kDevTimeout = 1u,   // a bounded inter-tile wait gave up
    kDevCorrupt = 2u,   // decoder: invalid codeword / segment end != next gap
    kDevNoCode = 4u,    // encoder: an input byte has no codeword
    kDevSize = 8u,      // total bits / symbols disagree with W, S or n
};

// Look-back record: 2 flag bits over a 62-bit value (aggregate or inclusive
// prefix).  Zero = not yet published.
constexpr uint64_t kFlagA = 1ull << 62;
constexpr uint64_t kFlagP = 2ull << 62;
constexpr uint64_t kFlagMask = 3ull << 62;
constexpr uint64_t kValueMask = ~kFlagMask;
// Hand-off record: valid bit over a 32-bit payload.
constexpr uint64_t kHandValid = 1ull << 32;

// Workspace header (both kernels): status word, tile counter, padding.
constexpr size_t kWsHeader = 256;

// ---------------------------------------------------------------- encoder ---
// Per byte value: code in bits 0..15, length in bits 16..20; an absent byte
// is 0x80000000 (length field 0, and 0x8000 when summed as e >> 16 so that a
// thread's bit count reveals it without a per-byte test).
struct EncTable {
    uint32_t e[256];
};
constexpr uint32_t kEncAbsent = 0x80000000u;

constexpr int kEncTileBytes = 8192;  // input bytes per encoder tile

struct EncArgs {
    const uint8_t* in_aligned;  // input rounded down to 16 bytes
    uint64_t lo;                // virtual index of the first input byte (in & 15)
    uint64_t hi;                // lo + n
    uint32_t* bits;
    uint64_t words;
    uint32_t* gaps;
    uint64_t gap_words;
    uint64_t segments;
    uint64_t* lookback;  // [ntiles]
    uint64_t* hand_bits; // [ntiles] partial last bitstream word of each tile
    uint64_t* hand_gap;  // [ntiles] partial last gap word of each tile
    uint32_t* counter;
    uint32_t* status;
    uint64_t ntiles;
};

// ---------------------------------------------------------------- decoder ---
// Two-level table.  Level 1 is indexed by the next kDecPrefix bits:
//   direct entry : bit15=0, bit14 = invalid, bits 8..11 = length-1, bits 0..7 = symbol
//   pointer entry: bit15=1, bits 12..14 = extra width w, bits 0..11 = level-2 offset
// Level 2 holds direct entries, 2^w per level-1 prefix whose codes are longer.
constexpr int kDecPrefix = 11;
constexpr int kDecT2Cap = 2560;  // >= the largest complete 16-bit book (see host.cpp)
constexpr uint16_t kDecInvalid = 0x4000;
struct DecTable {
    uint16_t t1[1 << kDecPrefix];
    uint16_t t2[kDecT2Cap];
};

struct DecArgs {
    const uint32_t* bits;
    uint64_t words;
    const uint32_t* gaps;
    uint64_t segments;
    uint8_t* out_aligned;  // output rounded down to 16 bytes
    uint64_t out_lo;       // out & 15
    uint64_t n;
    uint64_t* lookback;
    uint32_t* counter;
    uint32_t* status;
    uint64_t ntiles;
};

// --------------------------------------------------------------- launchers --
// Implemented in the .cu files; return cudaError_t as int.
int launch_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, void* stream);
int launch_encode(const EncArgs& a, const EncTable& t, void* stream);
int launch_decode(const DecArgs& a, const DecTable& t, void* stream);
uint64_t encode_tiles(uint64_t n);          // tiles for an n-byte input (any alignment)
uint64_t decode_tiles(uint64_t segments);

// ------------------------------------------------------------- host helpers -
void make_enc_table(const hgap_codebook& cb, EncTable* t);
hgap_status make_dec_table(const hgap_codebook& cb, DecTable* t);

}  // namespace hgap
