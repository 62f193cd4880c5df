// Minimal host-only stand-in for <Kokkos_Core.hpp>.
//
// TEST INFRASTRUCTURE ONLY.  It supplies just what the reference header
// src/cpp/ksim/zx_eval.hpp names (KOKKOS_INLINE_FUNCTION, a 1-D View with
// operator(), DefaultExecutionSpace::memory_space) so that header compiles
// unmodified with g++ into oracle/_ref.  Views here are non-owning pointers
// over host memory.
#pragma once
#include <cstddef>

#define KOKKOS_INLINE_FUNCTION inline

namespace Kokkos {
struct HostSpace {};
struct DefaultExecutionSpace { using memory_space = HostSpace; };

template <class DataType, class... Props> struct View;

template <class T, class... Props> struct View<T *, Props...> {
    T *ptr = nullptr;
    std::size_t n = 0;
    View() = default;
    View(T *p, std::size_t count) : ptr(p), n(count) {}
    T &operator()(std::size_t i) const { return ptr[i]; }
};
}  // namespace Kokkos
