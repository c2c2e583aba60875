// status.h — error reporting shared by the C-ABI translation units (internal).
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace bmfr {

// Records `msg` as the calling thread's last error and returns `status`.
int fail(int status, const std::string& msg);
// BMFR_E_CUDA with the runtime's error text.
int cuda_fail(cudaError_t e, const char* what);

}  // namespace bmfr
