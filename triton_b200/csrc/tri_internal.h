// tri_internal.h -- host-side helpers shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

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

// Conflict-free waves: item k goes one wave after the latest earlier item
// that touches one of its cells, so items sharing a cell keep their index
// order and all others run in parallel.  'order' lists items wave by wave,
// wave w is order[wave_start[w] .. wave_start[w+1]).
void build_waves(const std::vector<std::vector<int64_t>>& touches, std::vector<int32_t>& order,
                 std::vector<int32_t>& wave_start);

// Cells one external-boundary item may read or write (compute_extbc_values,
// kernels.h:237-424): its own cell ii and the ghost next to it on every edge
// the cell lies on (that covers the ghost it writes and, at a corner, the
// second one).  Items on different cells never share a cell, so boundary
// rows and columns run as one wave; only a cell listed twice is ordered.
inline std::vector<int64_t> extbc_touches(int64_t ii, int rows, int cols) {
  const int64_t ix = ii / cols, iy = ii % cols;
  std::vector<int64_t> t{ii};
  if (iy == 1) t.push_back(ii - 1);
  if (iy == cols - 2) t.push_back(ii + 1);
  if (ix == 1) t.push_back(ii - cols);
  if (ix == rows - 2) t.push_back(ii + cols);
  return t;
}

}  // namespace tri
