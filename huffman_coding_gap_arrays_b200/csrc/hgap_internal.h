// hgap_internal.h -- types shared by the host code and the sm_100a kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/hgap.h"

#ifdef __CUDACC__
#define HGAP_HD __host__ __device__
#else
#define HGAP_HD
#endif

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
    kDevPlan = 16u,     // encoder: workspace histograms are not this input's
};

// Look-back record: 2 flag bits over a 62-bit value (aggregate or inclusive
// prefix).  Zero = not yet published.
constexpr uint64_t kFlagA = 1ull << 62;
constexpr uint64_t kFlagP = 2ull << 62;
constexpr uint64_t kFlagMask = 3ull << 62;
constexpr uint64_t kValueMask = ~kFlagMask;
// Hand-off record: valid bit over a 32-bit payload.
constexpr uint64_t kHandValid = 1ull << 32;

// Bounded-wait test hook, all zero in every product call: the work item
// (encoder region / decoder tile, in the launch's numbering) plus one whose
// look-back records are never published, and the limit of every look-back
// wait in ns (0: the default, kWaitLimitNs).
struct LookbackHook {
    uint64_t hold_plus1;
    uint64_t wait_ns;
};

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

// The encoder works on super-tiles: `st_chunks` chunks of kEncChunkBytes input
// bytes each.  The histogram pass that precedes it also records one 256-bin
// histogram per super-tile, so a super-tile's bit count -- and, after one
// look-back over super-tiles, its first output bit -- is known before any of
// its bytes are encoded.  st_chunks depends on n only (hgap_internal
// encode_st_chunks), so both passes and the workspace query agree.
constexpr int kEncChunkBytes = 8192;
constexpr int kEncMaxStChunks = 32;
// The super-tile size minimises the encoder's modelled makespan: persistent CTAs
// (2 per SM, 296 on a 148-SM B200) take equal super-tiles of c chunks in waves,
// each costing c chunks plus about one chunk's worth of fixed work (look-back,
// the head word rebuilt backwards, the ring crossing into the next super-tile).
// Measured on C1 (16 MiB, 2048 chunks): 1-chunk super-tiles (7 waves) 0.070 ms,
// 2 chunks 0.055, 4 chunks 0.047, 7 chunks (one wave) 0.041 ms.  The count is
// kept under encode_super_tiles_cap, so a workspace sized for n bytes serves
// every smaller input.
constexpr uint64_t kEncCtas = 296;
constexpr uint64_t kEncStOverhead = 1;  // chunks

// Encoder workspace: [status u32][counter u32][pad][tag: n u64, input u64] ...
// [scratch histogram u32 x 256 at 1024] [st_rec u64 x nst at 2048] [st_hist u32 x 256 x nst]
constexpr size_t kEncWsHeader = 2048;
constexpr size_t kEncWsTag = 16;
constexpr size_t kEncWsScratchHist = 1024;

inline uint64_t encode_chunks(uint64_t n) { return (n + 15 + kEncChunkBytes - 1) / kEncChunkBytes; }
// An upper bound of the super-tile count of every input of up to n bytes (at any
// alignment), non-decreasing in n: what a workspace for inputs of up to n bytes holds.
inline uint64_t encode_super_tiles_cap(uint64_t n) {
    const uint64_t ch = encode_chunks(n);
    const uint64_t a = ch < 2 * kEncCtas ? ch : 2 * kEncCtas;
    const uint64_t b = (ch + 15) / 16;
    return a > b ? a : b;
}
inline uint64_t encode_st_chunks(uint64_t n) {
    const uint64_t chunks = encode_chunks(n), cap = encode_super_tiles_cap(n);
    uint64_t best = kEncMaxStChunks, best_cost = ~0ull;
    for (uint64_t c = 1; c <= (uint64_t)kEncMaxStChunks; ++c) {
        const uint64_t tiles = (chunks + c - 1) / c;
        if (tiles > cap) continue;  // within the workspace bound (c = 32 always is)
        const uint64_t cost = (tiles + kEncCtas - 1) / kEncCtas * (c + kEncStOverhead);
        if (cost < best_cost) {  // ties keep the smaller super-tile (finer balance)
            best = c;
            best_cost = cost;
        }
    }
    return best;
}
inline uint64_t encode_super_tiles(uint64_t lo_plus_n, uint64_t n) {
    const uint64_t st = encode_st_chunks(n) * kEncChunkBytes;
    return (lo_plus_n + st - 1) / st;
}

// One buffer to encode.  The single-buffer entry points pass one job by value;
// the batched ones keep an array of them in the workspace.  Regions (units of
// st_bytes input bytes) are numbered globally over the jobs of a launch: job
// j owns regions [item0, item0 + nst).
// 16-byte aligned (and a multiple of 16 bytes): the one-CTA setup kernels write
// whole jobs with vector stores
struct alignas(16) EncJob {
    const uint8_t* in_aligned;  // input rounded down to 16 bytes
    uint64_t lo;                // virtual index of the first input byte (in & 15)
    uint64_t hi;                // lo + n
    uint32_t* bits;
    uint64_t words;
    uint32_t* gaps;
    uint64_t gap_words;
    uint64_t segments;
    uint64_t item0;             // global index of the job's first region
    uint64_t nst;               // its regions
    uint32_t st_bytes;          // region size in input bytes (a multiple of kEncChunkBytes)
    uint32_t bits_aligned16;    // bits is 16-byte aligned: vector stores allowed
    uint64_t bit0;              // stream bit of the job's first code: 0, unless the job is one
                                // part of a stream split across devices (bits / gaps then
                                // address stream word / gap word 0 of a window)
};
static_assert(sizeof(EncJob) == 96, "EncJob: six 16-byte groups");

struct EncArgs {
    EncJob single;              // the job, when jobs == nullptr
    const EncJob* jobs;         // batched: [count]
    const uint64_t* item0s;     // batched: [count + 1], item0 of each job and the total
    const EncTable* tables;     // batched: [count]
    uint32_t count;             // jobs (1 for the single-buffer path)
    uint64_t nitems;            // regions over all jobs
    const uint64_t* nitems_dev; // batched: the region count in device memory (overrides nitems)
    uint64_t* st_rec;           // [nitems] look-back records over regions
    const uint32_t* st_hist;    // [nitems][256] per-region histograms
    const uint64_t* tag;        // single path: {n, input address} written by the histogram pass
    uint32_t* counter;
    uint32_t* status;
    LookbackHook hook;
};

struct HistStArgs {
    EncJob single;
    const EncJob* jobs;
    const uint64_t* item0s;
    uint32_t count;
    uint64_t nitems;
    const uint64_t* nitems_dev; // batched: the region count in device memory (overrides nitems)
    uint32_t* hist;             // [count][256] histograms (zeroed before the launch)
    uint32_t* st_hist;          // [nitems][256]
    uint64_t* tag;              // single path: receives {n, input address}
    uint32_t* counter;          // batched: zeroed region counter (regions claimed one at a time)
};

// ---------------------------------------------------------------- decoder ---
// Two-level table.  Level 1 is indexed by the next kDecPrefix bits:
//   direct entry : bit15=0, bit14 = invalid, bits 8..11 = length-1, bits 0..7 = symbol
//   pointer entry: bit15=1, bits 12..14 = extra width w, bits 0..11 = level-2 offset
// Level 2 holds direct entries, 2^w per level-1 prefix whose codes are longer.
constexpr int kDecPrefix = 11;
// Decoder stage rows (of 4 symbols) for a book whose shortest code has
// min_len bits: a 128-bit segment holds at most ceil(128 / min_len) symbols.
HGAP_HD constexpr int dec_stage_rows(uint32_t min_len) {
    return min_len >= 4 ? 8 : min_len == 3 ? 11 : min_len == 2 ? 16 : 32;
}
// Segments per decoder tile for a stage of R rows: two per thread, or one
// per thread where the stage is large (R >= 16: it halves the stage and
// compact areas so that more CTAs share an SM; measured 31 % faster for
// R = 32, 3 % for R = 16, and 33 % slower for R = 11, where the per-tile
// work then dominates).
HGAP_HD constexpr int dec_tile_segs(int R) { return R >= 16 ? 256 : 512; }
// The same with a launch-shape override of 256 or 512 segments (0: the
// default).  32 stage rows keep 256: their 512-segment tile would leave one
// CTA per SM.
HGAP_HD constexpr int dec_tile_segs_for(int R, uint32_t override_segs) {
    return R >= 32 ? 256 : (override_segs == 256 || override_segs == 512) ? (int)override_segs : dec_tile_segs(R);
}
constexpr int kDecT2Cap = 2560;  // >= the largest complete 16-bit book (see host.cpp)
constexpr uint16_t kDecInvalid = 0x4000;
struct DecTable {
    uint16_t t1[1 << kDecPrefix];
    uint16_t t2[kDecT2Cap];
};

// Multi entries (up to three symbols per level-1 lookup) pay for their wider
// stores and tail test only where codes are very short: complete books whose
// stage has at least this many rows (32: a shortest code of 1 bit).  Measured
// per 256 MiB: 2.2 bits/byte 0.518 -> 0.484 ms; from 16 rows on, Zipf(1.2)
// (shortest code 2 bits) 0.699 -> 0.722 ms.
constexpr int kDecMultiMinRows = 32;
HGAP_HD constexpr bool dec_multi(int rows, bool complete) { return complete && rows >= kDecMultiMinRows; }

// The decode kernel's level-1 tables in their widened form (u32 entries: pair
// form, or multi form for a complete book, with the length of the first code
// per prefix), built once per buffer on the batched path so that a CTA moving
// to another buffer's tile copies them into shared memory with 16-byte loads
// instead of re-deriving every entry.  The level-2 table (its groups in use)
// is read from here directly.
struct DecTableW {
    uint32_t t1[1 << kDecPrefix];
    uint8_t l1[1 << kDecPrefix];
    uint16_t t2[kDecT2Cap];
};
static_assert(sizeof(DecTableW) % 16 == 0, "16-byte copies");

// One stream to decode (same single / batched scheme as EncJob).  Its tiles
// use look-back records [item0, item0 + ntiles).
struct alignas(16) DecJob {
    const uint32_t* bits;
    uint64_t words;
    const uint32_t* gaps;
    uint64_t gap_words;
    uint64_t segments;
    uint8_t* out_aligned;  // output rounded down to 16 bytes
    uint64_t out_lo;       // out & 15
    uint64_t n;
    uint64_t item0;        // first look-back record of the job
    uint64_t ntiles;
};
static_assert(sizeof(DecJob) == 80, "DecJob: five 16-byte groups");

struct DecArgs {
    DecJob single;              // the job, when jobs == nullptr
    const DecJob* jobs;         // batched: [count]
    const uint32_t* job_of;     // batched: [nitems] job of each tile of this launch
    const uint64_t* item0s;     // batched: [count] first tile of each job in this launch's numbering
    const DecTableW* tables;    // batched: [count]
    uint32_t count;
    uint64_t nitems;            // tiles in this launch
    const uint64_t* nitems_dev; // batched: the tile count in device memory (overrides nitems)
    uint64_t* lookback;
    uint32_t* counter;
    uint32_t* status;
    LookbackHook hook;
};

// --------------------------------------------------------------- launchers --
// Implemented in the .cu files; return cudaError_t as int.
int launch_histogram(const void* d_in, uint64_t n, uint32_t* d_hist, void* stream);
int launch_encode(const EncArgs& a, const EncTable& t, int ctas_per_sm, void* stream);
int launch_hist_st(const HistStArgs& a, int ctas_per_sm, void* stream);
int launch_decode(const DecArgs& a, const DecTable& t, uint32_t min_len, bool complete, bool pairs,
                  int ctas_per_sm, uint32_t tile_segs, void* stream);
// Fraction of level-1 entries that decode two symbols (the decoder's pair
// rate under the code's own distribution, where every 11-bit prefix is
// equally likely).
double dec_pair_fraction(const DecTable& t);
// Tiles of a stream for a book whose shortest code is min_len bits (the
// decoder's tile size depends on it, and on a tile-size override, 0: none);
// min_len = 1 with 256-segment tiles gives the most.
uint64_t decode_tiles(uint64_t segments, uint32_t min_len, uint32_t tile_segs = 0);

// ------------------------------------------------------------- host helpers -
void make_enc_table(const hgap_codebook& cb, EncTable* t);
hgap_status make_dec_table(const hgap_codebook& cb, DecTable* t);

}  // namespace hgap
