// Shared helpers of the engine: error reporting and CUDA call checking.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "t3ns_b200.h"

namespace t3ns {

// Records the message of the last failure on this thread (t3ns_last_error).
int set_error(int code, const std::string &msg);

#define T3NS_CUDA_TRY(expr)                                                   \
        do {                                                                  \
                cudaError_t e_ = (expr);                                      \
                if (e_ != cudaSuccess)                                        \
                        return ::t3ns::set_error(T3NS_E_CUDA,                 \
                                std::string(#expr) + ": " +                   \
                                cudaGetErrorString(e_));                      \
        } while (0)

#define T3NS_TRY(expr)                                                        \
        do {                                                                  \
                int r_ = (expr);                                              \
                if (r_ != T3NS_OK) return r_;                                 \
        } while (0)

}  // namespace t3ns
