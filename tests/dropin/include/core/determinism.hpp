// core/determinism.hpp -- include-path shim for compiling reference callers
// unchanged.  The reference fixes the reduction mode at build time
// (TDMD_DETERMINISTIC_REDUCE -> kDeterministicReduce); this library switches
// it at run time, so a caller built with the macro turns the library's
// ID-ordered mode on before main.  Test infrastructure only.
#pragma once
#include "tdmd_b200.hpp"

namespace tdmd {
#if defined(TDMD_DETERMINISTIC_REDUCE) && TDMD_DETERMINISTIC_REDUCE
inline constexpr bool kDeterministicReduce = true;
namespace detail {
inline const bool deterministic_reduce_on_load = [] {
  set_deterministic_reduce(true);
  return true;
}();
}  // namespace detail
#else
inline constexpr bool kDeterministicReduce = false;
#endif
}  // namespace tdmd
