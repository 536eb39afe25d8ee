// Host-side shared declarations: result codes, logging, thread-local last
// error (reference core/include/mrt/Common.hpp:11-42 and
// core/src/gpu/GpuContext.cpp:13-45), and CUDA error mapping.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>

#include "../../../include/mini_raytrace.h"

namespace mrt {

// Log levels as in the C ABI callback: 0 = debug .. 3 = error.
enum class LogLevel : int { Debug = 0, Info = 1, Warn = 2, Error = 3 };

void setLogCallback(mrtLogFn fn, void* user);
void log(LogLevel level, const std::string& msg);

const char* resultName(mrtResult r);
const std::string& lastError();
void setLastError(const std::string& msg);

// Records the failure (last error + error log) and returns `code`.
mrtResult fail(mrtResult code, const std::string& msg);

// Maps a CUDA error to an mrtResult: allocation failures to
// MRT_ERROR_OUT_OF_MEMORY, a missing kernel image to MRT_ERROR_SHADER_LOAD,
// errors that poison the CUDA context to MRT_ERROR_DEVICE_LOST, anything
// else to MRT_ERROR_UNKNOWN.
mrtResult fromCuda(cudaError_t e, const char* what);
bool isStickyCudaError(cudaError_t e);

// Allocation-failure injection for tests (mrtxInjectAllocationFailure):
// with a budget n >= 0, the next n device or pinned-host allocations
// succeed and every later one fails as out of memory, until the budget is
// set back to -1. allocationFailureInjected() is asked at each allocation.
void setAllocationFailureInjection(int64_t succeedFirst);
bool allocationFailureInjected();

// A named range on the host timeline for profilers (NVTX, header-only;
// without a tool attached a push or pop is one pointer test). The engine
// marks commits, render calls and readbacks, so that for example
// `ncu --nvtx --nvtx-include "mrt render/"` profiles only the kernels a
// render call launches.
class TraceRange {
public:
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace mrt

// Evaluate a CUDA call; on failure record it and return the mapped result
// from the enclosing function (which must return mrtResult).
#define MRT_CUDA(expr)                                                  \
    do {                                                                \
        const cudaError_t _e = (expr);                                  \
        if (_e != cudaSuccess) return ::mrt::fromCuda(_e, #expr);       \
    } while (0)

#define MRT_TRY(expr)                                                   \
    do {                                                                \
        const mrtResult _r = (expr);                                    \
        if (_r != MRT_SUCCESS) return _r;                               \
    } while (0)
