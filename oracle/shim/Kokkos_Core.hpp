// Test infrastructure (oracle only): a minimal host-only stand-in for the
// handful of Kokkos entry points the reference TRITON sources use, so that
// the unmodified reference `src/main.cpp` compiles into a CPU oracle.
//
// Written from the public Kokkos API names only.  Dispatch is a plain loop
// (OpenMP `parallel for` when compiled with -fopenmp); every kernel body in
// the reference is data-parallel per index, so the schedule does not change
// results.  The one reduction (`Kokkos::Min`) is order-independent.
//
// Used by: oracle/Makefile (reference build into oracle/_ref/).  Never linked
// into the product library.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_LAMBDA [=]
#define KOKKOS_RESTRICT __restrict__
#define KOKKOS_INLINE_FUNCTION inline

namespace Kokkos {

inline void initialize() {}
inline void initialize(int&, char**) {}
inline void finalize() {}
inline void fence() {}

inline void* kokkos_malloc(size_t bytes) { return std::malloc(bytes ? bytes : 1); }
inline void* kokkos_malloc(const std::string&, size_t bytes) { return kokkos_malloc(bytes); }
inline void kokkos_free(void* p) { std::free(p); }

struct HostSpace {};
struct LayoutRight {};
struct Unmanaged {};
template <class... Ts> struct MemoryTraits {};

struct DefaultExecutionSpace { using memory_space = HostSpace; };
struct DefaultHostExecutionSpace { using memory_space = HostSpace; };

// Unmanaged 1-D view over a raw pointer (the only form the reference builds).
template <class DataType, class... Props> class View;
template <class T, class... Props> class View<T*, Props...> {
 public:
  View(T* p, size_t n) : ptr_(p), n_(n) {}
  T* data() const { return ptr_; }
  size_t size() const { return n_; }
  size_t extent(int) const { return n_; }
  T& operator[](size_t i) const { return ptr_[i]; }
  T& operator()(size_t i) const { return ptr_[i]; }
 private:
  T* ptr_;
  size_t n_;
};

template <class A, class B> inline void deep_copy(const A& dst, const B& src) {
  if (dst.size() != src.size()) throw std::runtime_error("deep_copy: size mismatch");
  std::memmove(dst.data(), src.data(), dst.size() * sizeof(*dst.data()));
}

template <class F> inline void parallel_for(const std::string&, int n, const F& f) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int i = 0; i < n; ++i) f(i);
}

template <class T> struct Min {
  T& result;
  explicit Min(T& r) : result(r) {}
};

// Min reduction: each thread folds its indices with the caller's lambda,
// starting from the largest finite value, then the partials are folded with
// the same "a < b ? a : b" rule.  NaN inputs are never selected, as in a
// serial fold.
template <class F, class T>
inline void parallel_reduce(const std::string&, int n, const F& f, Min<T> red) {
  T acc = std::numeric_limits<T>::max();
#ifdef _OPENMP
  int nt = omp_get_max_threads();
  std::vector<T> part(nt, std::numeric_limits<T>::max());
#pragma omp parallel
  {
    int t = omp_get_thread_num();
    T local = std::numeric_limits<T>::max();
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) f(i, local);
    part[t] = local;
  }
  for (int t = 0; t < nt; ++t) acc = part[t] < acc ? part[t] : acc;
#else
  for (int i = 0; i < n; ++i) f(i, acc);
#endif
  red.result = acc;
}

}  // namespace Kokkos
