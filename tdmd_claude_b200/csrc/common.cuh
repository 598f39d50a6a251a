// common.cuh -- shared host/device plumbing of the B200 TDMD library:
// status/error handling behind the C ABI, the device-side box, fixed-point
// position encoding, warp/block reductions and compensated FP32 sums.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "tdmd_b200.h"

namespace tdmd_b200 {

// Metal units, src/core/constants.hpp:15,28 (double in both precisions).
constexpr double kMvv2e = 1.0364269e-4;
constexpr double kBoltzmann = 8.617333262e-5;

// --------------------------------------------------------------------------
// Errors: every C entry point returns a tdmd_status and records a message.
// --------------------------------------------------------------------------
void set_error(int32_t code, const std::string& msg);
int32_t fail(int32_t code, const std::string& msg);

struct Error {
  int32_t code;
  std::string msg;
};

#define TDMD_CU(call)                                                                 \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      throw ::tdmd_b200::Error{e_ == cudaErrorMemoryAllocation ? TDMD_ERR_OUT_OF_MEMORY \
                                                               : TDMD_ERR_CUDA,       \
                               std::string(#call) + ": " + cudaGetErrorString(e_)};  \
    }                                                                                 \
  } while (0)

#define TDMD_REQUIRE(cond, msg)                                                   \
  do {                                                                            \
    if (!(cond)) throw ::tdmd_b200::Error{TDMD_ERR_INVALID_ARGUMENT, (msg)};      \
  } while (0)

#define TDMD_LAUNCH_CHECK() TDMD_CU(cudaGetLastError())

// Runs `body` and converts exceptions to a status code.
template <class F>
int32_t guarded(F&& body) {
  try {
    body();
    return TDMD_OK;
  } catch (const Error& e) {
    return fail(e.code, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(TDMD_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(TDMD_ERR_CUDA, e.what());
  }
}

// --------------------------------------------------------------------------
// Device box: orthorhombic, per-axis periodicity (Box, src/core/box.hpp:17),
// cell grid (CellList, src/domain/cell_list.cpp:21-23) and the fixed-point
// scales of the mixed path.
// --------------------------------------------------------------------------
struct DevBox {
  double lo[3];
  double L[3];
  double halfL[3];
  double cs[3];      // cell size L/nc
  double qlo[3];     // fixed-point origin (lo on periodic axes)
  double qinv[3];    // 2^32 / Lq  (fixed-point encode)
  float qscale[3];   // Lq / 2^32  (fixed-point decode, FP32)
  double qstep[3];   // Lq / 2^32  (fixed-point decode, FP64)
  int nc[3];
  int periodic[3];
};

DevBox make_devbox(const tdmd_box& b, double r_list);

// Cell of a position, CellList::cell_of (cell_list.hpp:60-72): double
// division (IEEE), truncation toward zero, clamp to the grid.
__device__ __forceinline__ int cell_coord(double x, double lo, double cs, int nc) {
  int c = __double2int_rz(__ddiv_rn(__dsub_rn(x, lo), cs));
  c = c >= nc ? nc - 1 : c;
  return c < 0 ? 0 : c;
}

__device__ __forceinline__ int wrap_cell(int c, int nc) {
  return c < 0 ? c + nc : (c >= nc ? c - nc : c);
}

// Minimum image on a delta, math.hpp:78-107 / device kernels' if-else form.
template <class T>
__device__ __forceinline__ T min_image1(T d, T L, T halfL, int periodic) {
  if (periodic) {
    if (d > halfL)
      d -= L;
    else if (d < -halfL)
      d += L;
  }
  return d;
}

// Fixed-point position: q = round((x - qlo)/Lq * 2^32) mod 2^32.  On a
// periodic axis Lq = L and qlo = lo: int32 differences wrap modulo 2^32,
// which IS the minimum image, at a resolution of L/2^32 (2.7e-8 A at
// L = 115.68 A).  On a non-periodic axis Lq = 4L centred on the box, so
// differences of atoms within 1.5 L of the box never wrap.
__device__ __forceinline__ int32_t encode_q(double x, double lo, double qinv) {
  const long long v = __double2ll_rn(__dmul_rn(__dsub_rn(x, lo), qinv));
  return static_cast<int32_t>(static_cast<uint32_t>(static_cast<unsigned long long>(v)));
}

// --------------------------------------------------------------------------
// Compensated FP32 accumulation (Knuth TwoSum, error-free): s + c holds the
// running sum with ~FP64-like accuracy for the per-atom force/density sums.
// __fadd_rn/__fsub_rn keep the compiler from contracting or reassociating.
// --------------------------------------------------------------------------
struct CSum {
  float s, c;
  __device__ __forceinline__ CSum() : s(0.f), c(0.f) {}
  __device__ __forceinline__ void add(float x) {
    const float t = __fadd_rn(s, x);
    const float z = __fsub_rn(t, s);
    const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, z)), __fsub_rn(x, z));
    s = t;
    c = __fadd_rn(c, e);
  }
  // Merge another compensated partial sum.
  __device__ __forceinline__ void merge(float os, float oc) {
    add(os);
    c = __fadd_rn(c, oc);
  }
  __device__ __forceinline__ float value() const { return __fadd_rn(s, c); }
};

// --------------------------------------------------------------------------
// Reductions.  Block results go to per-block partial arrays that a
// single-block kernel sums in block order: fixed order, bit-reproducible,
// no atomics.
// --------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sums NV doubles across the block; thread 0 gets the totals in v[].
// Requires blockDim.x to be a multiple of 32 and <= 1024; smem >= 32*NV.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[warp * NV + k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = lane < nwarps ? smem[lane * NV + k] : 0.0;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  }
}

// One read-only 32-byte record (32-byte aligned) in one 256-bit load.  The
// inline-asm loads here and in forces.cuh are volatile so that the compiler
// keeps them after grid_dependency_wait() (also a volatile asm): a load
// without a memory operand could otherwise be hoisted above the wait.
__device__ __forceinline__ double4 ld_d4(const double4* p) {
  double4 v;
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
      : "l"(p));
  return v;
}

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// Number of SMs of the current device (148 on B200), cached per process.
int sm_count();

// Stream from the C ABI's void*.
inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// --------------------------------------------------------------------------
// Programmatic dependent launch.  A kernel started by launch() may become
// resident while the kernel before it in the stream (or graph) drains: its
// blocks park in griddepcontrol.wait, which returns once every prerequisite
// grid has completed and its memory operations are visible.  So a kernel
// launched this way calls grid_dependency_wait() before its first global
// memory access, read or write; release_dependents() then lets the next
// launch be scheduled as this grid's blocks finish.  Both are no-ops in a
// kernel launched without the attribute (or after a copy or memset).
// --------------------------------------------------------------------------
__device__ __forceinline__ void grid_dependency_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void release_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// At the top of a kernel.  The next launch is released implicitly as this
// grid's blocks exit: releasing it at the top measured slower, the parked
// blocks of the next pass sharing the SMs with this pass's last wave.
__device__ __forceinline__ void dependent_launch_prologue() { grid_dependency_wait(); }

// Whether launch() sets the programmatic-serialization attribute (environment
// TDMD_PDL=0 turns it off; read once per process).
bool programmatic_launch();
// Turns the attribute off for this host thread's launches while set (a
// profiling capture: event nodes sit between its kernels).
void suppress_programmatic_launch(bool off);

template <class... P, class... A>
void launch(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
            A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  if (programmatic_launch()) {
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  TDMD_CU(cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...));
}

}  // namespace tdmd_b200
