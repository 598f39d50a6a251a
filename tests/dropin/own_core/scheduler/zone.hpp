// scheduler/zone.hpp -- include-path shim for compiling reference callers unchanged:
// the reference header maps onto the C++ layer of this library (its
// single-rank zone types).
#pragma once
#include "tdmd_b200.hpp"
