// noalloc.cu -- hgap_decode_noalloc: the decoder for callers that cannot
// allocate device memory.
//
// Some callers have no way to obtain scratch memory: code running inside a
// framework whose device memory is owned by its own pool (so a raw
// cudaMalloc is not allowed, and the caller holds no spare buffer to lend us),
// plugins loaded into a host process that forbids allocation on its hot path,
// or bindings in other languages that only hand over the input and output
// buffers.  For them the decoder's look-back scratch lives in a fixed array
// compiled into this library: every GPU that loads the library holds
// HGAP_NOALLOC_SCRATCH_BYTES for it until the process exits.
//
// The array's name is only a host-side stand-in in host code; its device
// address is fetched once per device with cudaGetSymbolAddress, with that
// device current, on the first call made on that device.  Make that first
// call before any stream capture.  All calls share the one array and it keeps
// the previous call's contents: the decoder clears the part that must start
// at zero on every call, and two calls that run at the same time on the GPU
// (different streams, or different host threads) race on it, so they must not
// overlap.
#include <cuda_runtime.h>

#include <mutex>

#include "hgap_internal.h"

namespace {

constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_decode_scratch[HGAP_NOALLOC_SCRATCH_BYTES];

std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_decode_scratch on the current device (set up once).
hgap_status scratch_for_current_device(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HGAP_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return HGAP_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_decode_scratch) != cudaSuccess || !p) return HGAP_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return HGAP_OK;
}

}  // namespace

extern "C" hgap_status hgap_decode_noalloc(const uint32_t* d_bits, uint64_t words,
                                           const uint32_t* d_gaps, uint64_t segments,
                                           const hgap_codebook* cb, uint8_t* d_out, uint64_t n,
                                           hgap_stream_t stream) {
    if (hgap_decode_workspace_bytes(segments) > HGAP_NOALLOC_SCRATCH_BYTES)
        return HGAP_ERR_WORKSPACE;  // stream too long for the built-in scratch
    void* scratch = nullptr;
    hgap_status s = scratch_for_current_device(&scratch);
    if (s != HGAP_OK) return s;
    s = hgap_decode(d_bits, words, d_gaps, segments, cb, d_out, n, scratch,
                    HGAP_NOALLOC_SCRATCH_BYTES, stream);
    if (s != HGAP_OK || n == 0) return s;
    return hgap_workspace_status(scratch, stream);
}
