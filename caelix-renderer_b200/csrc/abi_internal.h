// Internal declarations shared by the translation units behind the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <new>

#include "../../include/caelix_b200.h"

// Exceptions never cross the C ABI: the body of every entry point that may allocate on the host
// runs inside CAELIX_GUARD_BEGIN / CAELIX_GUARD_END.
#define CAELIX_GUARD_BEGIN try {
#define CAELIX_GUARD_END                                                \
    }                                                                   \
    catch (const std::bad_alloc&)                                       \
    {                                                                   \
        cx::log(CAELIX_LOG_ERROR, "%s: out of host memory", __func__);   \
        return CAELIX_ERROR_OUT_OF_MEMORY;                              \
    }                                                                   \
    catch (...)                                                         \
    {                                                                   \
        cx::log(CAELIX_LOG_ERROR, "%s: unexpected exception", __func__); \
        return CAELIX_ERROR_INVALID_ARGUMENT;                           \
    }

namespace cx {

void log(CaelixLogLevel level, const char* fmt, ...);
CaelixResult cuda_result(cudaError_t e, const char* what);
CaelixResult status_result(uint32_t status, const char* what);

// Device memory grown on demand (never shrunk); freed by release().
struct GrowBuffer
{
    void* ptr = nullptr;
    uint64_t bytes = 0;
    CaelixResult reserve(uint64_t want, const char* what);
    // reserve, growing by an extra eighth when it has to grow (buffers sized by a scene).
    CaelixResult reserve_grow(uint64_t want, const char* what) { return want <= bytes ? CAELIX_OK : reserve(want + want / 8, what); }
    void release();
};

}  // namespace cx

struct CaelixDevice
{
    int ordinal = 0;
    uint32_t sm_count = 148;
    cx::GrowBuffer sort_scratch;  // caelix_radix_sort_pairs
    uint32_t* status = nullptr;   // device word the asynchronous entry points OR their failures into
};
