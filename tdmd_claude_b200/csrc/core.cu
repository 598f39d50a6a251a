// core.cu -- error state, device box set-up and the fixed-order device scan.
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <string>

#include "buffers.cuh"
#include "common.cuh"

namespace tdmd_b200 {

namespace {
thread_local std::string g_last_error;
}

void set_error(int32_t code, const std::string& msg) {
  g_last_error = "tdmd_b200 error " + std::to_string(code) + ": " + msg;
}

int32_t fail(int32_t code, const std::string& msg) {
  set_error(code, msg);
  return code;
}

// SM count per device ordinal, cached; concurrent first calls from several
// host threads may both query the attribute, but they store the same value.
int sm_count() {
  constexpr int kMaxCachedDevices = 64;
  static std::atomic<int> cached[kMaxCachedDevices];
  int dev = 0;
  TDMD_CU(cudaGetDevice(&dev));
  if (dev >= 0 && dev < kMaxCachedDevices) {
    const int c = cached[dev].load(std::memory_order_relaxed);
    if (c > 0) return c;
  }
  int v = 0;
  TDMD_CU(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
  if (dev >= 0 && dev < kMaxCachedDevices) cached[dev].store(v, std::memory_order_relaxed);
  return v;
}

namespace {
thread_local bool t_pdl_suppressed = false;
}

bool programmatic_launch() {
  static const bool on = [] {
    const char* v = std::getenv("TDMD_PDL");
    return !(v && v[0] == '0');
  }();
  return on && !t_pdl_suppressed;
}

void suppress_programmatic_launch(bool off) { t_pdl_suppressed = off; }

DevBox make_devbox(const tdmd_box& b, double r_list) {
  DevBox d{};
  for (int a = 0; a < 3; ++a) {
    const double L = b.hi[a] - b.lo[a];
    TDMD_REQUIRE(L > 0.0, "box extent must be positive on every axis");
    d.lo[a] = b.lo[a];
    d.L[a] = L;
    d.halfL[a] = 0.5 * L;
    d.periodic[a] = b.periodic[a] ? 1 : 0;
    // nc = max(3, floor(L / r_list)), cell size L/nc -- cell_list.cpp:21-23.
    int n = 3;
    if (r_list > 0.0) {
      const double f = std::floor(L / r_list);
      n = f > 3.0 ? static_cast<int>(std::fmin(f, 1.0e6)) : 3;
    }
    d.nc[a] = n;
    d.cs[a] = L / n;
    const double Lq = d.periodic[a] ? L : 4.0 * L;
    d.qlo[a] = d.periodic[a] ? b.lo[a] : b.lo[a] - 1.5 * L;
    d.qinv[a] = 4294967296.0 / Lq;
    d.qscale[a] = static_cast<float>(Lq / 4294967296.0);
    d.qstep[a] = Lq / 4294967296.0;
  }
  return d;
}

// --------------------------------------------------------------------------
// Exclusive scan: per-block reduce -> single-block scan of block sums ->
// per-block scan with carry-in.  4096 items per block (1024 threads x 4).
// --------------------------------------------------------------------------
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr long long kScanSingleTiles = 16;  // 65536 items

// Block-wide exclusive scan of one int per thread; returns the block total.
__device__ int block_exclusive_scan(int v, int* smem, int* total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int w = lane < nw ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem[lane] = w;  // inclusive warp prefix
  }
  __syncthreads();
  const int warp_prefix = warp > 0 ? smem[warp - 1] : 0;
  *total = smem[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

__global__ void k_scan_reduce(const int* __restrict__ in, long long n, int* __restrict__ sums) {
  dependent_launch_prologue();
  __shared__ int smem[32];
  const long long base = static_cast<long long>(blockIdx.x) * kScanTile;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long long idx = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
    if (idx < n) s += in[idx];
  }
  int total;
  block_exclusive_scan(s, smem, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Scans `in` in place over tiles of kScanTile with a running carry (single
// block).  out may alias in.  *total gets the overall sum when non-null.
__global__ void k_scan_single(const int* __restrict__ in, int* __restrict__ out, long long n,
                              int* __restrict__ total_out) {
  dependent_launch_prologue();
  __shared__ int smem[32];
  int carry = 0;
  for (long long base = 0; base < n; base += kScanTile) {
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const long long idx = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
      v[k] = idx < n ? in[idx] : 0;
      s += v[k];
    }
    int tile_total;
    int pre = block_exclusive_scan(s, smem, &tile_total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const long long idx = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
      if (idx < n) out[idx] = pre;
      pre += v[k];
    }
    carry += tile_total;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

// One-pass single-block scan of up to kScanThreads * kScanWide items, all
// loads and stores coalesced: thread t holds items t + k * kScanThreads
// (k < kScanWide), i.e. column t of kScanWide rows; the kScanWide row scans
// run side by side (warp shuffles, then the warps' totals of each row, then
// the rows' totals), so item (k, t)'s prefix is rows_before(k) +
// warps_before(k, t) + lanes_before(k, t).  out may alias in.
constexpr int kScanWide = 16;
__global__ void __launch_bounds__(kScanThreads) k_scan_wide(const int* __restrict__ in,
                                                            int* __restrict__ out,
                                                            int* __restrict__ out2, int n,
                                                            int* __restrict__ total_out) {
  dependent_launch_prologue();
  __shared__ int wsum[kScanWide][kScanThreads / 32];  // row k: per-warp totals -> prefixes
  __shared__ int rsum[kScanWide + 1];                 // rows' exclusive prefixes, total
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  int v[kScanWide], incl[kScanWide];
#pragma unroll
  for (int k = 0; k < kScanWide; ++k) {
    const int i = k * kScanThreads + t;
    v[k] = i < n ? in[i] : 0;
    incl[k] = v[k];
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int k = 0; k < kScanWide; ++k) {
      const int y = __shfl_up_sync(0xffffffffu, incl[k], o);
      if (lane >= o) incl[k] += y;
    }
  }
  if (lane == 31) {
#pragma unroll
    for (int k = 0; k < kScanWide; ++k) wsum[k][warp] = incl[k];
  }
  __syncthreads();
  // warp k scans row k's warp totals (kScanThreads / 32 = 32 of them)
  if (warp < kScanWide) {
    const int x = wsum[warp][lane];
    int y = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    wsum[warp][lane] = y - x;  // exclusive
    if (lane == 31) rsum[warp] = y;
  }
  __syncthreads();
  if (t == 0) {
    int c = 0;
    for (int k = 0; k < kScanWide; ++k) {
      const int r = rsum[k];
      rsum[k] = c;
      c += r;
    }
    rsum[kScanWide] = c;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kScanWide; ++k) {
    const int i = k * kScanThreads + t;
    if (i < n) {
      const int e = rsum[k] + wsum[k][warp] + incl[k] - v[k];
      out[i] = e;
      if (out2) out2[i] = e;
    }
  }
  if (t == 0 && total_out) *total_out = rsum[kScanWide];
}

__global__ void k_scan_apply(const int* __restrict__ in, int* __restrict__ out, long long n,
                             const int* __restrict__ block_prefix) {
  dependent_launch_prologue();
  __shared__ int smem[32];
  const long long base = static_cast<long long>(blockIdx.x) * kScanTile;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long long idx = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
    v[k] = idx < n ? in[idx] : 0;
    s += v[k];
  }
  int tile_total;
  int pre = block_exclusive_scan(s, smem, &tile_total) + block_prefix[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long long idx = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
    if (idx < n) out[idx] = pre;
    pre += v[k];
  }
}

}  // namespace

int device_scan_launches(long long n) {
  if (n <= 0) return 0;
  return (n + kScanTile - 1) / kScanTile <= kScanSingleTiles ? 1 : 3;
}

void device_exclusive_scan(const int* in, int* out, long long n, int* total, DevArray<int>& tmp,
                           cudaStream_t stream, int* out2) {
  if (n <= 0) {
    if (total) TDMD_CU(cudaMemsetAsync(total, 0, sizeof(int), stream));
    return;
  }
  const long long nblocks = (n + kScanTile - 1) / kScanTile;
  if (n <= static_cast<long long>(kScanThreads) * kScanWide) {
    launch(k_scan_wide, 1, kScanThreads, 0, stream, in, out, out2, static_cast<int>(n), total);
    TDMD_LAUNCH_CHECK();
    return;
  }
  if (out2) {  // the tiled scans write one output; copy it after them
    device_exclusive_scan(in, out, n, total, tmp, stream, nullptr);
    TDMD_CU(cudaMemcpyAsync(out2, out, sizeof(int) * n, cudaMemcpyDeviceToDevice, stream));
    return;
  }
  // Up to kScanSingleTiles tiles one block walking the tiles beats three
  // launches; beyond that, reduce -> scan of block sums -> apply.
  if (nblocks <= kScanSingleTiles) {
    launch(k_scan_single, 1, kScanThreads, 0, stream, in, out, n, total);
    TDMD_LAUNCH_CHECK();
    return;
  }
  tmp.reserve(static_cast<size_t>(nblocks));
  launch(k_scan_reduce, static_cast<unsigned>(nblocks), kScanThreads, 0, stream, in, n, tmp.data());
  TDMD_LAUNCH_CHECK();
  launch(k_scan_single, 1, kScanThreads, 0, stream, tmp.data(), tmp.data(), nblocks, total);
  TDMD_LAUNCH_CHECK();
  launch(k_scan_apply, static_cast<unsigned>(nblocks), kScanThreads, 0, stream, in, out, n,
         tmp.data());
  TDMD_LAUNCH_CHECK();
}

}  // namespace tdmd_b200

extern "C" {

const char* tdmd_last_error(void) { return tdmd_b200::g_last_error.c_str(); }

int32_t tdmd_abi_version(void) { return TDMD_B200_ABI_VERSION; }

int32_t tdmd_copy(void* dst, const void* src, size_t bytes, void* stream) {
  return tdmd_b200::guarded([&] {
    if (bytes == 0) return;
    TDMD_REQUIRE(dst && src, "null pointer");
    cudaStream_t s = tdmd_b200::as_stream(stream);
    TDMD_CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
    TDMD_CU(cudaStreamSynchronize(s));
  });
}

void tdmd_fast_pipeline_config_default(tdmd_fast_pipeline_config* cfg) {
  if (!cfg) return;
  *cfg = tdmd_fast_pipeline_config{};
  cfg->dt = 0.001;
  cfg->r_skin = 1.0;
  cfg->rebuild_every = 10;
  cfg->precision = TDMD_FP64;
  cfg->use_graphs = 1;
  cfg->lanes_per_atom = 0;
  cfg->t_target = 0.0;
  cfg->t_period = 0.1;
  cfg->nhc_length = 3;
  cfg->adaptive_dt = 0;
  cfg->dt_min = 0.0001;
  cfg->dt_max = 0.002;
  cfg->c2 = 0.05;
  cfg->energy_every = 0;
  cfg->energy_log_capacity = 0;
}

}  // extern "C"
