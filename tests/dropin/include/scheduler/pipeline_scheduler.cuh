// scheduler/pipeline_scheduler.cuh -- include-path shim for compiling reference callers
// unchanged: the reference header of this path maps onto the C++ layer of this library.
#pragma once
#include "tdmd_b200.hpp"
