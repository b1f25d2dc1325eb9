// Error reporting, version and device probing of the C ABI.
#include <cuda_runtime.h>

#include <string>

#include "yrc_internal.hpp"

namespace yrc {
namespace {
thread_local std::string g_last_error;
}  // namespace

yrc_status Fail(yrc_status status, const std::string& message) {
    g_last_error = message;
    return status;
}

yrc_status Ok() {
    g_last_error.clear();
    return YRC_OK;
}

}  // namespace yrc

extern "C" {

const char* yrc_last_error(void) { return yrc::g_last_error.c_str(); }

const char* yrc_version(void) { return "0.1.0"; }

int yrc_device_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count > 0 ? 1 : 0;
}

}  // extern "C"
