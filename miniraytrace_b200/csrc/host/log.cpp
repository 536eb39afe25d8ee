// Logging, last-error and result-name plumbing. Semantics follow the
// reference: one global callback guarded by a mutex, stderr "[mrt] ..." when
// none is set (GpuContext.cpp:13-25); a thread-local last-error string that
// is never NULL (GpuContext.cpp:27-32); result names (GpuContext.cpp:34-45).
#include <cstdio>
#include <mutex>

#include "common.h"

namespace mrt {

namespace {
std::mutex g_logMutex;
mrtLogFn g_logFn = nullptr;
void* g_logUser = nullptr;
thread_local std::string g_lastError;
}  // namespace

void setLogCallback(mrtLogFn fn, void* user) {
    std::lock_guard<std::mutex> lock(g_logMutex);
    g_logFn = fn;
    g_logUser = user;
}

void log(LogLevel level, const std::string& msg) {
    std::lock_guard<std::mutex> lock(g_logMutex);
    if (g_logFn) {
        g_logFn(static_cast<int>(level), msg.c_str(), g_logUser);
        return;
    }
    std::fprintf(stderr, "[mrt] %s\n", msg.c_str());
}

const std::string& lastError() { return g_lastError; }
void setLastError(const std::string& msg) { g_lastError = msg; }

const char* resultName(mrtResult r) {
    switch (r) {
        case MRT_SUCCESS: return "Success";
        case MRT_ERROR_VULKAN_INIT: return "ErrorVulkanInit";
        case MRT_ERROR_OUT_OF_MEMORY: return "ErrorOutOfMemory";
        case MRT_ERROR_INVALID_ARGUMENT: return "ErrorInvalidArgument";
        case MRT_ERROR_INVALID_HANDLE: return "ErrorInvalidHandle";
        case MRT_ERROR_SHADER_LOAD: return "ErrorShaderLoad";
        case MRT_ERROR_DEVICE_LOST: return "ErrorDeviceLost";
        default: return "ErrorUnknown";
    }
}

mrtResult fail(mrtResult code, const std::string& msg) {
    setLastError(msg);
    log(LogLevel::Error, msg);
    return code;
}

bool isStickyCudaError(cudaError_t e) {
    switch (e) {
        case cudaErrorIllegalAddress:
        case cudaErrorLaunchFailure:
        case cudaErrorIllegalInstruction:
        case cudaErrorMisalignedAddress:
        case cudaErrorInvalidAddressSpace:
        case cudaErrorInvalidPc:
        case cudaErrorHardwareStackError:
        case cudaErrorAssert:
        case cudaErrorLaunchTimeout:
        case cudaErrorECCUncorrectable:
        case cudaErrorContextIsDestroyed:
        case cudaErrorDevicesUnavailable:
            return true;
        default:
            return false;
    }
}

mrtResult fromCuda(cudaError_t e, const char* what) {
    const std::string msg = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
                            ") at " + what;
    if (e == cudaErrorMemoryAllocation) return fail(MRT_ERROR_OUT_OF_MEMORY, msg);
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidKernelImage)
        return fail(MRT_ERROR_SHADER_LOAD, msg);
    if (isStickyCudaError(e)) return fail(MRT_ERROR_DEVICE_LOST, msg);
    return fail(MRT_ERROR_UNKNOWN, msg);
}

}  // namespace mrt
