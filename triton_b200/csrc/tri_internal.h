// tri_internal.h -- host-side helpers shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "triton_b200.h"

namespace tri {

// Records the message of the last failure on this thread and returns code.
int set_error(int code, const char* fmt, ...);

#define TRI_CUDA_TRY(expr)                                                                        \
  do {                                                                                            \
    cudaError_t _e = (expr);                                                                      \
    if (_e != cudaSuccess) return ::tri::set_error(TRI_E_CUDA, "%s: %s (%s:%d)", #expr,           \
                                                   cudaGetErrorString(_e), __FILE__, __LINE__);   \
  } while (0)

#define TRI_CHECK_ARG(cond, ...)                                       \
  do {                                                                 \
    if (!(cond)) return ::tri::set_error(TRI_E_INVALID, __VA_ARGS__); \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace tri
