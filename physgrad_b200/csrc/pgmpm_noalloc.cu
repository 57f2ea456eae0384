// pgmpm_noalloc.cu -- a stable radix sort that allocates no device memory.
//
// Who needs it: callers that are not allowed to call cudaMalloc at the
// moment they sort.  Examples are host frameworks that hand a plugin a fixed
// GPU memory budget and forbid allocations outside their own allocator, and
// frame-time-critical loops where cudaMalloc's implicit device-wide
// synchronisation is not acceptable.  pgmpm_radix_sort_pairs allocates its
// ping-pong buffers and histograms on every call; this variant uses a
// fixed-size scratch array that lives in the library's device image instead.
//
// The scratch array below is allocated once per GPU when the library's
// device code is loaded on that GPU and is held until the process exits
// (about 8.9 MB: one (key, value) ping-pong buffer of PGMPM_NOALLOC_MAX_PAIRS
// pairs plus the histogram words for that many pairs).  The caller's output
// arrays serve as the other ping-pong buffer.
//
// Host code cannot use the array's name as a device pointer (on the host it
// names a stand-in object), so its device address is looked up with
// cudaGetSymbolAddress: once per device, with that device current, on the
// first call made on that device.  That first call may load the module, so
// make it before starting any stream capture.
//
// The address found on the first call is kept for the life of the process.
// A cudaDeviceReset after that call reloads the module and would leave the
// kept address stale, so resetting a device that this entry point has used
// is not supported.
//
// Every call shares the one array and leaves its contents behind.  Nothing in
// it needs to start at zero: each pass writes all the histogram words it
// later reads, and the ping-pong buffer is fully written before it is read.
// Calls that can overlap on the GPU (different streams, or different host
// threads without ordering) race on the array and must be serialised by the
// caller.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/pgmpm.h"
#include "pgmpm_internal.h"

using namespace pgmpm;

namespace {

constexpr int64_t kMaxPairs = PGMPM_NOALLOC_MAX_PAIRS;
constexpr int64_t kHistWords = radix_scratch_words_for(kMaxPairs);
constexpr int64_t kScratchWords = 2 * kMaxPairs + kHistWords;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_dev_addr[kMaxDevices] = {};

thread_local std::string g_msg;

// Device address of the scratch array on the current device (looked up
// once per device).
cudaError_t scratch_on_current_device(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_dev_addr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_dev_addr[dev];
    return cudaSuccess;
}

// True when the byte ranges of two n-word arrays overlap (either may be null).
bool overlaps(const uint32_t* a, const uint32_t* b, int64_t n) {
    if (!a || !b) return false;
    const uintptr_t pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = (uintptr_t)n * sizeof(uint32_t);
    return pa < pb + len && pb < pa + len;
}

}  // namespace

// Defined in pgmpm_capi.cu: records the message returned by pgmpm_last_error().
int pgmpm_set_error(int code, const char* msg);

extern "C" int pgmpm_radix_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                              uint32_t* vals_out, int64_t n, int32_t key_bits, void* stream) {
    if (n < 0 || key_bits < 1 || key_bits > 32)
        return pgmpm_set_error(PGMPM_ERR_ARG, "pgmpm_radix_sort_pairs_noalloc: n must be >= 0, key_bits in [1, 32]");
    if (n > kMaxPairs) {
        char buf[200];
        std::snprintf(buf, sizeof(buf),
                      "pgmpm_radix_sort_pairs_noalloc: n = %lld exceeds the maximum of %lld pairs "
                      "(PGMPM_NOALLOC_MAX_PAIRS); use pgmpm_radix_sort_pairs",
                      (long long)n, (long long)kMaxPairs);
        return pgmpm_set_error(PGMPM_ERR_ARG, buf);
    }
    if (n == 0) return PGMPM_OK;
    if (!keys_in || !keys_out || !vals_out)
        return pgmpm_set_error(PGMPM_ERR_ARG, "pgmpm_radix_sort_pairs_noalloc: null pointer");
    // The first pass writes the caller's outputs (or the scratch) while it
    // still reads the inputs, so no output may overlap an input or the other
    // output.
    if (overlaps(keys_in, keys_out, n) || overlaps(keys_in, vals_out, n) || overlaps(vals_in, keys_out, n) ||
        overlaps(vals_in, vals_out, n) || overlaps(keys_out, vals_out, n))
        return pgmpm_set_error(PGMPM_ERR_ARG,
                               "pgmpm_radix_sort_pairs_noalloc: the output arrays must not overlap the input "
                               "arrays or each other");
    uint32_t* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) {
        g_msg = std::string("pgmpm_radix_sort_pairs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return pgmpm_set_error(PGMPM_ERR_CUDA, g_msg.c_str());
    }
    uint32_t* pk = scratch;              // ping-pong keys   [kMaxPairs]
    uint32_t* pv = scratch + kMaxPairs;  // ping-pong values [kMaxPairs]
    uint32_t* hist = scratch + 2 * kMaxPairs;
    // The last pass must write the caller's arrays: pass p targets buffer a
    // when p is even and b when p is odd.
    const int passes = radix_passes(key_bits);
    const bool out_is_a = ((passes - 1) & 1) == 0;
    uint32_t* ka = out_is_a ? keys_out : pk;
    uint32_t* va = out_is_a ? vals_out : pv;
    uint32_t* kb = out_is_a ? pk : keys_out;
    uint32_t* vb = out_is_a ? pv : vals_out;
    int which = 0;
    e = radix_sort_pairs(keys_in, vals_in, ka, va, kb, vb, hist, n, key_bits, &which,
                         reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        g_msg = std::string("pgmpm_radix_sort_pairs_noalloc: ") + cudaGetErrorString(e);
        return pgmpm_set_error(PGMPM_ERR_CUDA, g_msg.c_str());
    }
    return PGMPM_OK;
}
