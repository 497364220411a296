// Test infrastructure (oracle only): the reference includes this header but,
// without TRITON_REDUCE_1, uses nothing from it.
#pragma once
#include "Kokkos_Core.hpp"
