// caelix_radix_sort_pairs_static: the radix sort for callers that cannot allocate device memory.
//
// Some hosts must not call cudaMalloc (or anything that may allocate) on the thread that records
// their GPU work: a render thread of an engine plugin that must not stall the frame it records on
// an allocation, or a host with a fixed device memory budget set at start-up. caelix_radix_sort_pairs keeps a
// scratch buffer that it grows with cudaMalloc on demand; this variant instead uses a scratch
// array compiled into the library (a file-scope __device__ array of a fixed size), so a call
// allocates nothing. The price: the array is reserved on every GPU that loads the library, from
// load to process exit, and the sort size is capped by it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/caelix_b200.h"
#include "abi_internal.h"
#include "radix_sort.cuh"

namespace {

// Largest count of pairs one call sorts.
constexpr uint32_t kStaticSortMaxPairs = 1u << 18;  // 262144
// Scratch layout (u32 words): ping-pong keys [max], ping-pong values [max], a status word block
// [64] that takes the failure bits of calls without a status word of their own (nothing reads it:
// such a call drops its device-side failures), then the onesweep words (histograms, tile counters,
// look-back tile states).
constexpr uint64_t kStaticStatusWords = 64;
constexpr uint64_t kStaticScratchWords =
    2ull * kStaticSortMaxPairs + kStaticStatusWords + cx::sort_scratch_words(kStaticSortMaxPairs);

// The scratch array: about 2.4 MB on every device that loads the library. In host code this name is
// only a stand-in for the device symbol; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) uint32_t g_sort_scratch[kStaticScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
uint32_t* g_address[kMaxDevices] = {};

// The device address of g_sort_scratch on the current device, looked up once per device with that
// device current.
CaelixResult scratch_address(uint32_t** out)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_radix_sort_pairs_static");
    if (device < 0 || device >= kMaxDevices) {
        cx::log(CAELIX_LOG_ERROR, "caelix_radix_sort_pairs_static: device %d above the supported %d", device,
                kMaxDevices);
        return CAELIX_ERROR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_address[device]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_radix_sort_pairs_static: cudaGetSymbolAddress");
        g_address[device] = static_cast<uint32_t*>(p);
    }
    *out = g_address[device];
    return CAELIX_OK;
}

}  // namespace

extern "C" {

CAELIX_API CaelixResult caelix_radix_sort_pairs_static(uint32_t* keys, uint32_t* values, uint32_t count,
                                                       uint32_t identity_values, uint32_t* status, uint64_t stream)
{
    if ((count > 0 && (!keys || !values)) || identity_values > 1) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (count > kStaticSortMaxPairs) {
        cx::log(CAELIX_LOG_ERROR, "caelix_radix_sort_pairs_static: %u pairs exceed the static scratch limit of %u",
                count, kStaticSortMaxPairs);
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    if (count == 0) return CAELIX_OK;
    uint32_t* base = nullptr;
    const CaelixResult r = scratch_address(&base);
    if (r != CAELIX_OK) return r;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* keys_b = base;
    uint32_t* values_b = base + kStaticSortMaxPairs;
    uint32_t* fallback_status = base + 2ull * kStaticSortMaxPairs;
    uint32_t* scratch = fallback_status + kStaticStatusWords;
    if (count > cx::kSmallSortKeys) {
        // The array keeps the previous call's contents: clear the words that must start at zero
        // (the histograms, tile counters and look-back states of this call's size). A sort of at
        // most kSmallSortKeys pairs runs in one CTA's shared memory and reads none of them.
        cudaError_t e = cudaMemsetAsync(scratch, 0, cx::sort_scratch_words(count) * 4, s);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_radix_sort_pairs_static");
        const uint32_t grid = std::min<uint32_t>((count + 2047) / 2048, cx::current_sm_count() * 4);
        cx::radix_histogram(keys, count, scratch, grid, s);
    }
    cx::onesweep_sort(keys, values, keys_b, values_b, count, identity_values != 0, scratch,
                      status ? status : fallback_status, s);
    return cx::cuda_result(cudaGetLastError(), "caelix_radix_sort_pairs_static");
}

}  // extern "C"
