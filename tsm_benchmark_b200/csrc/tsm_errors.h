// tsm_errors.h -- the per-thread message behind tsm_last_cuda_error(),
// shared by every translation unit of the library.
#pragma once

#include <string>

namespace tsm {

// The calling thread's last error message (defined in tsm_capi.cu).
std::string& last_error();

}  // namespace tsm
