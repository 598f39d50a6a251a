// nlist.cu -- cell-list binning and Verlet neighbor-list build (sm_100a).
//
// Reference path (tdmd_Claude): DeviceCellList::build
// (src/domain/device_cell_list.cu:59-150) and DeviceNeighborList::build
// (src/neighbors/device_neighbor_list.cu:158-278), with the CPU semantics of
// CellList::cell_of (src/domain/cell_list.hpp:60-72) and the ID-ordered cell
// scatter of the reference's deterministic mode (device_cell_list.cu:114-136).
//
// Design (B200):
//  * binning: one thread per atom, IEEE double division for the cell index
//    (bit-identical to the CPU cell_of), atomic histogram, fixed-order device
//    scan, atomic scatter and a per-cell sort that restores ID order -- so the
//    result is deterministic with no host round trip (the reference copies the
//    counts to the host and scans there).
//  * list build: one CTA per cell stages the 27-cell candidate tile in shared
//    memory as fixed-point records; warps sweep it 32 candidates at a time
//    with an FP32 filter and fall back to the reference's exact FP64
//    expression (round-to-nearest ops, no FMA contraction) only within 1e-5
//    of r_list^2, so the lists match the CPU reference bit for bit; a
//    ballot/popc compaction writes accepted neighbors in stencil order.
//    Candidates that cannot be within r_list of any center atom (FP32 r^2 to
//    the center atoms' bounding box above the band) are dropped while
//    staging, in order; the replica kernel keeps one such list per warp
//    slab of center atoms.  One pass: rows are padded to a fixed capacity and
//    an overflow flag replaces the reference's count pass + 8-byte D2H sync.
#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>

#include "buffers.cuh"
#include "common.cuh"
#include "replicas.cuh"

namespace tdmd_b200 {

namespace {

struct LoadAoS3 {
  const double* p;
  __device__ __forceinline__ double3 operator()(int i) const {
    const double* q = p + 3ll * i;
    return make_double3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
  }
};

struct LoadD4 {
  const double4* p;
  __device__ __forceinline__ double3 operator()(int i) const {
    const double4 a = ld_d4(p + i);
    return make_double3(a.x, a.y, a.z);
  }
};

template <class Load>
__global__ void k_bin_atoms(Load pos, int n, DevBox b, int* __restrict__ atom_cell,
                            int* __restrict__ cell_count) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double3 p = pos(i);
  const int ix = cell_coord(p.x, b.lo[0], b.cs[0], b.nc[0]);
  const int iy = cell_coord(p.y, b.lo[1], b.cs[1], b.nc[1]);
  const int iz = cell_coord(p.z, b.lo[2], b.cs[2], b.nc[2]);
  const int c = iz * b.nc[0] * b.nc[1] + iy * b.nc[0] + ix;
  atom_cell[i] = c;
  atomicAdd(&cell_count[c], 1);
}

__global__ void k_scatter_atoms(const int* __restrict__ atom_cell, int n,
                                int* __restrict__ cursor, int* __restrict__ cell_atoms) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = atomicAdd(&cursor[atom_cell[i]], 1);
  cell_atoms[slot] = i;
}

// Restores ID-ascending order inside each cell: one warp per cell, rank
// sort through shuffles for cells of up to 32 * kSortPerLane atoms (lane l
// holds entries l, l + 32, ...; an entry's rank is the number of smaller
// ids), lane-0 insertion sort beyond that.  key (nullable) gives each array
// index its ID when the arrays are held in another order than the caller's
// (the scheduler's cell-ordered layout); keys are unique.
constexpr int kSortPerLane = 4;
__global__ void k_sort_cells(const int* __restrict__ cell_start, const int* __restrict__ cell_count,
                             int ncells, int* __restrict__ cell_atoms,
                             const int* __restrict__ key) {
  dependent_launch_prologue();
  const long long gw = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= ncells) return;  // uniform per warp
  const int c = static_cast<int>(gw);
  int* a = cell_atoms + cell_start[c];
  const int m = cell_count[c];
  if (m <= 32) {
    const int v = lane < m ? a[lane] : INT_MAX;
    const int kv = lane < m ? (key ? __ldg(key + v) : v) : INT_MAX;
    int rank = 0;
#pragma unroll
    for (int k = 0; k < 32; ++k) rank += __shfl_sync(0xffffffffu, kv, k) < kv ? 1 : 0;
    if (lane < m) a[rank] = v;
    return;
  }
  if (m <= 32 * kSortPerLane) {
    int v[kSortPerLane], kv[kSortPerLane], rank[kSortPerLane];
#pragma unroll
    for (int r = 0; r < kSortPerLane; ++r) {
      const int e = lane + 32 * r;
      v[r] = e < m ? a[e] : INT_MAX;
      kv[r] = e < m ? (key ? __ldg(key + v[r]) : v[r]) : INT_MAX;
      rank[r] = 0;
    }
    // every read is in registers before the first write: the shuffles
    // below synchronise the warp
#pragma unroll
    for (int q = 0; q < kSortPerLane; ++q) {
      if (32 * q >= m) break;  // uniform
      for (int k = 0; k < 32; ++k) {
        const int o = __shfl_sync(0xffffffffu, kv[q], k);
#pragma unroll
        for (int r = 0; r < kSortPerLane; ++r) rank[r] += o < kv[r] ? 1 : 0;
      }
    }
#pragma unroll
    for (int r = 0; r < kSortPerLane; ++r)
      if (lane + 32 * r < m) a[rank[r]] = v[r];
    return;
  }
  if (lane == 0) {
    for (int k = 1; k < m; ++k) {
      const int v = a[k];
      const int kv = key ? __ldg(key + v) : v;
      int j = k - 1;
      while (j >= 0 && (key ? __ldg(key + a[j]) : a[j]) > kv) {
        a[j + 1] = a[j];
        --j;
      }
      a[j + 1] = v;
    }
  }
}

// --------------------------------------------------------------------------
// Row build, one CTA per cell.  The 27 stencil cells (dz, dy, dx in -1..1,
// wrapped) are concatenated in stencil order; their atoms (ID order within
// each cell) become candidate records {x, y, z, j}: FP32 coordinates
// relative to the center cell's lower corner, taken from the exact int32
// fixed-point difference (so the minimum image is already applied when the
// grid has at least 4 cells per periodic axis; WRAP re-applies it in FP32
// for 3-cell axes).  Records are staged in shared memory when they fit
// (kStageCap); otherwise each warp rebuilds them on the fly.  Each warp takes
// center-cell atoms in turn and sweeps the candidates 32 at a time:
//   * FP32 filter: a candidate whose r^2 lies outside the band
//     rl^2 (1 -+ eps) is decided by it.  Each coordinate carries at most
//     ~2^-23 of its magnitude (< 3 cells) in rounding, plus one fixed-point
//     unit L/2^32; eps = 3e-5 + 8 (L/2^32)/rl bounds the resulting r^2 error
//     several times over, so the decision equals the FP64 one;
//   * inside the band the reference expression decides: delta = r_j - r_i
//     in FP64, minimum image, (x*x + y*y) + z*z with round-to-nearest ops,
//     < rl^2.
// Accepted candidates are compacted with ballot/popc in candidate order, so
// every row is the reference's per-atom list, bit for bit.
//
// Cell pruning (staged, no FP32 re-wrap): a candidate whose FP32 r^2 to the
// bounding box of the center cell's own records exceeds the band's upper end
// is dropped while staging (order kept).  Rounding is monotone, so the sweep's
// r^2 to any center atom is at least that bound: every dropped candidate is
// one the filter would reject for every center atom, and the rows do not
// change.  About 30 % of a 27-cell neighborhood lies farther than r_list from
// the center cell.
// --------------------------------------------------------------------------
constexpr int kRowThreads = 128;
constexpr int kStageCap = 1536;  // staged candidate records (24 KiB)
constexpr int kSlabMax = 128;    // center atoms handled as warp slabs
constexpr int kIdxCap = 512;     // kept candidates per warp slab

// The reference's decision for one pair (NeighborList::build,
// neighbor_list.cpp:57-63): delta = r_j - r_i in FP64, minimum image,
// r^2 = (x*x + y*y) + z*z with round-to-nearest ops, r^2 < rl^2.  Not
// inlined: it runs for a handful of candidates per rebuild, and as a call
// it stays out of the filter loop's instruction stream.
// The box travels as scalars: a reference to it would make every thread
// copy the whole box into local memory at kernel start.
template <class Load>
__device__ __noinline__ bool exact_within(Load pos, int i, int j, double rl2, double Lx, double Ly,
                                          double Lz, double hx, double hy, double hz, int px,
                                          int py, int pz) {
  const double3 pi = pos(i), pj = pos(j);
  const double ex = min_image1(__dsub_rn(pj.x, pi.x), Lx, hx, px);
  const double ey = min_image1(__dsub_rn(pj.y, pi.y), Ly, hy, py);
  const double ez = min_image1(__dsub_rn(pj.z, pi.z), Lz, hz, pz);
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
  return r2 < rl2;
}

// Shared memory of one row-building CTA.
struct RowSmem {
  int s_start[27], s_pre[28];
  int s_max[kRowThreads / 32];
  int s_wcnt[kRowThreads / 32];  // kept candidates per warp (staging chunk)
  float s_bb[6];                 // center cell's bounding box: min xyz, max xyz
  int s_c0;                      // staged index of the center cell's first atom
};

// Shared memory of the warp-slab variant (4.3 KiB more per CTA).
struct SlabSmem {
  short s_order[kSlabMax];                          // center atoms by x
  unsigned short s_idx[kRowThreads / 32][kIdxCap];  // each warp's kept candidates
};

// FP32 r^2 in one fixed order of round-to-nearest ops; the filter and the
// pruning bound both use it (the bound relies on its monotonicity).
__device__ __forceinline__ float r2_rn(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// Rows of the atoms of cell c of box b's grid; cell_start / cell_count index
// that grid's cells, cell_atoms and the atom indices are global.
template <class Load, bool WRAP, bool WRITE, bool SLAB>
__device__ __forceinline__ void build_cell_rows(
    RowSmem& sm, float4* stage, int stage_cap, SlabSmem* ss, Load pos, const DevBox& b, int c,
    const int* __restrict__ cell_start,
    const int* __restrict__ cell_count, const int* __restrict__ cell_atoms, double rl2,
    float lo_f, float hi_f, int* __restrict__ nbr, const int* __restrict__ row_off, int cap,
    int* __restrict__ counts, int* __restrict__ status) {
  int* const s_start = sm.s_start;
  int* const s_pre = sm.s_pre;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ncx = b.nc[0], ncy = b.nc[1], ncz = b.nc[2];
  const int ncxy = ncx * ncy;
  const int iz = c / ncxy, iy = (c - iz * ncxy) / ncx, ix = c - iz * ncxy - iy * ncx;
  if (threadIdx.x < 32) {
    int cnt = 0, st = 0;
    if (lane < 27) {
      const int dz = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dx = lane % 3 - 1;
      const int nb_c = wrap_cell(iz + dz, ncz) * ncxy + wrap_cell(iy + dy, ncy) * ncx +
                       wrap_cell(ix + dx, ncx);
      st = cell_start[nb_c];
      cnt = cell_count[nb_c];
      s_start[lane] = st;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < 27) s_pre[lane + 1] = incl;
    if (lane == 0) s_pre[0] = 0;
  }
  __syncthreads();
  const int total = s_pre[27];
  // Staged records are padded to whole 32-candidate sweeps with sentinels
  // far outside any box (their r^2 overflows to +inf and fails both the
  // filter and the band), so the staged sweep needs no bounds select.
  const int padded = (total + 31) & ~31;
  const bool staged = padded <= stage_cap;
  // Lower corner of the center cell: fixed point (periodic axes) and FP64.
  const double cx = b.lo[0] + ix * b.cs[0], cy = b.lo[1] + iy * b.cs[1],
               cz = b.lo[2] + iz * b.cs[2];
  const int ox = encode_q(cx, b.qlo[0], b.qinv[0]);
  const int oy = encode_q(cy, b.qlo[1], b.qinv[1]);
  const int oz = encode_q(cz, b.qlo[2], b.qinv[2]);
  const float s0 = b.qscale[0], s1 = b.qscale[1], s2 = b.qscale[2];
  // One coordinate of a record.  Periodic axis: the exact int32 fixed-point
  // difference (its wrap is the minimum image).  Non-periodic axis: the FP64
  // difference rounded once to FP32 -- the fixed-point difference would wrap
  // for an atom more than 2L from the corner (the cell list clamps atoms
  // outside the box into its edge cells); a coordinate farther than four
  // cells from the corner (outside the filter's error analysis) becomes NaN,
  // which sends every pair of that record to the exact FP64 test.
  auto coord = [](double x, double c, double qlo, double qinv, int oq, float sc, int per,
                  double cs) -> float {
    if (per) return __fmul_rn(__int2float_rn(encode_q(x, qlo, qinv) - oq), sc);
    const float r = __double2float_rn(__dsub_rn(x, c));
    return fabsf(r) <= static_cast<float>(4.0 * cs) ? r : __int_as_float(0x7fc00000);
  };
  // Candidate record k (cell t with s_pre[t] <= k < s_pre[t+1]).
  auto record = [&](int k) -> float4 {
    int lo = 0, hi = 27;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s_pre[mid] <= k) lo = mid; else hi = mid;
    }
    const int j = __ldg(cell_atoms + s_start[lo] + (k - s_pre[lo]));
    const double3 p = pos(j);
    return make_float4(coord(p.x, cx, b.qlo[0], b.qinv[0], ox, s0, b.periodic[0], b.cs[0]),
                       coord(p.y, cy, b.qlo[1], b.qinv[1], oy, s1, b.periodic[1], b.cs[1]),
                       coord(p.z, cz, b.qlo[2], b.qinv[2], oz, s2, b.periodic[2], b.cs[2]),
                       __int_as_float(j));
  };
  const int c0 = s_pre[13], ncen = s_pre[14] - s_pre[13];  // center = slot 13
  const unsigned lt_mask = (1u << lane) - 1u;
  const float Lx = static_cast<float>(b.L[0]), Ly = static_cast<float>(b.L[1]),
              Lz = static_cast<float>(b.L[2]);
  const float hx = 0.5f * Lx, hy = 0.5f * Ly, hz = 0.5f * Lz;
  int wmax = 0;  // lane 0: this warp's longest row
  // The row of one center atom (record ci, candidate index self_k) over
  // candidates cand(0 .. nloop): padded sources carry sentinels up to whole
  // sweeps; otherwise lanes past the end read atom i itself (j == i,
  // rejected).
  auto row = [&](const float4 ci, int self_k, auto cand, int nloop, auto padded_tag) {
    constexpr bool kPadded = decltype(padded_tag)::value;
    const int i = __float_as_int(ci.w);
    const long long base = row_off ? static_cast<long long>(row_off[i])
                                   : static_cast<long long>(i) * cap;
    const int limit = row_off ? INT_MAX : cap;
    int cnt = 0;
    for (int k0 = 0; k0 < nloop; k0 += 32) {
      const int k = k0 + lane;
      const float4 cj = cand(kPadded ? k : (k < nloop ? k : self_k));
      const int j = __float_as_int(cj.w);
      float dx = __fsub_rn(cj.x, ci.x), dy = __fsub_rn(cj.y, ci.y), dz = __fsub_rn(cj.z, ci.z);
      if (WRAP) {
        dx = min_image1(dx, Lx, hx, b.periodic[0]);
        dy = min_image1(dy, Ly, hy, b.periodic[1]);
        dz = min_image1(dz, Lz, hz, b.periodic[2]);
      }
      const float r2f = r2_rn(dx, dy, dz);
      const bool other = j != i;
      unsigned m = __ballot_sync(0xffffffffu, other && r2f < lo_f);
      // Candidates inside the filter's band go to the exact FP64 test:
      // rare, so the warp enters that path only when some lane needs it.
      // (Written with negations so that a NaN r^2 -- a far record -- lands
      // in the band.)
      const bool band = other && !(r2f < lo_f) && !(r2f > hi_f);
      if (__any_sync(0xffffffffu, band)) {
        const bool ok = band && exact_within(pos, i, j, rl2, b.L[0], b.L[1], b.L[2],
                                             b.halfL[0], b.halfL[1], b.halfL[2],
                                             b.periodic[0], b.periodic[1], b.periodic[2]);
        m |= __ballot_sync(0xffffffffu, ok);
      }
      if (WRITE && ((m >> lane) & 1u)) {
        const int p = cnt + __popc(m & lt_mask);
        if (p < limit) nbr[base + p] = j;
      }
      cnt += __popc(m);
    }
    if (lane == 0) {
      counts[i] = cnt;
      wmax = cnt > wmax ? cnt : wmax;
    }
  };
  const float4 sentinel = make_float4(1e30f, 1e30f, 1e30f, __int_as_float(-1));
  if (SLAB && !WRAP && total < stage_cap && ncen <= kSlabMax) {
    // Warp slabs: all candidates staged once (one sentinel after them); the
    // center atoms ranked by x and cut into one contiguous slab per warp;
    // each warp keeps, in candidate order, the candidates within the band
    // of its slab's bounding box (an index list), and sweeps only those.
    for (int k = threadIdx.x; k < total; k += kRowThreads) stage[k] = record(k);
    if (threadIdx.x == 0) stage[total] = sentinel;
    __syncthreads();
    // (a far record's NaN x ranks as +inf, so the ranks stay a permutation)
    auto xkey = [](float x) { return x == x ? x : INFINITY; };
    for (int t = threadIdx.x; t < ncen; t += kRowThreads) {
      const float xt = xkey(stage[c0 + t].x);
      int rank = 0;
      for (int u = 0; u < ncen; ++u) {
        const float xu = xkey(stage[c0 + u].x);
        rank += (xu < xt || (xu == xt && u < t)) ? 1 : 0;
      }
      ss->s_order[rank] = static_cast<short>(t);
    }
    __syncthreads();
    constexpr int kWarps = kRowThreads / 32;
    const int rlo = warp * ncen / kWarps, rhi = (warp + 1) * ncen / kWarps;
    if (rlo < rhi) {
      float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
      bool far = false;
      for (int r = rlo + lane; r < rhi; r += 32) {
        const float4 q = stage[c0 + ss->s_order[r]];
        far = far || !(q.x == q.x && q.y == q.y && q.z == q.z);
        mn[0] = fminf(mn[0], q.x), mn[1] = fminf(mn[1], q.y), mn[2] = fminf(mn[2], q.z);
        mx[0] = fmaxf(mx[0], q.x), mx[1] = fmaxf(mx[1], q.y), mx[2] = fmaxf(mx[2], q.z);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
          mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
      }
      // a far center atom: no bounding box, every candidate is kept
      if (__any_sync(0xffffffffu, far)) {
#pragma unroll
        for (int d = 0; d < 3; ++d) mn[d] = -INFINITY, mx[d] = INFINITY;
      }
      unsigned short* const idx = ss->s_idx[warp];
      int cnt = 0;
      for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        bool keep = false;
        if (k < total) {
          const float4 q = stage[k];
          const float ex = fmaxf(0.f, fmaxf(__fsub_rn(mn[0], q.x), __fsub_rn(q.x, mx[0])));
          const float ey = fmaxf(0.f, fmaxf(__fsub_rn(mn[1], q.y), __fsub_rn(q.y, mx[1])));
          const float ez = fmaxf(0.f, fmaxf(__fsub_rn(mn[2], q.z), __fsub_rn(q.z, mx[2])));
          keep = !(r2_rn(ex, ey, ez) > hi_f);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        const int p = cnt + __popc(m & lt_mask);
        if (keep && p < kIdxCap) idx[p] = static_cast<unsigned short>(k);
        cnt += __popc(m);
      }
      const int npad = (cnt + 31) & ~31;
      const bool fits = npad <= kIdxCap;
      if (fits)
        for (int p = cnt + lane; p < npad; p += 32) idx[p] = static_cast<unsigned short>(total);
      __syncwarp();
      if (fits) {
        for (int r = rlo; r < rhi; ++r) {
          const int self = c0 + ss->s_order[r];
          row(stage[self], self, [&](int k) { return stage[idx[k]]; }, cnt, std::true_type{});
        }
      } else {  // more kept candidates than the index list holds: all of them
        for (int r = rlo; r < rhi; ++r) {
          const int self = c0 + ss->s_order[r];
          row(stage[self], self, [&](int k) { return stage[k]; }, total, std::false_type{});
        }
      }
    }
  } else {
    int kept = total;  // staged candidates (after pruning)
    if (staged) {
      if (WRAP) {
        for (int k = threadIdx.x; k < total; k += kRowThreads) stage[k] = record(k);
      } else {
        if (warp == 0) {
          float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
          bool far = false;
          for (int a = lane; a < ncen; a += 32) {
            const float4 r = record(c0 + a);
            far = far || !(r.x == r.x && r.y == r.y && r.z == r.z);
            mn[0] = fminf(mn[0], r.x), mn[1] = fminf(mn[1], r.y), mn[2] = fminf(mn[2], r.z);
            mx[0] = fmaxf(mx[0], r.x), mx[1] = fmaxf(mx[1], r.y), mx[2] = fmaxf(mx[2], r.z);
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
              mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
            }
          }
          // a far center atom: no bounding box, every candidate is kept
          if (__any_sync(0xffffffffu, far)) {
#pragma unroll
            for (int d = 0; d < 3; ++d) mn[d] = -INFINITY, mx[d] = INFINITY;
          }
          if (lane == 0) {
#pragma unroll
            for (int d = 0; d < 3; ++d) sm.s_bb[d] = mn[d], sm.s_bb[3 + d] = mx[d];
          }
        }
        __syncthreads();
        const float bx0 = sm.s_bb[0], by0 = sm.s_bb[1], bz0 = sm.s_bb[2];
        const float bx1 = sm.s_bb[3], by1 = sm.s_bb[4], bz1 = sm.s_bb[5];
        kept = 0;
        for (int k0 = 0; k0 < total; k0 += kRowThreads) {
          const int k = k0 + threadIdx.x;
          float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
          bool keep = false;
          if (k < total) {
            r = record(k);
            const float ex = fmaxf(0.f, fmaxf(__fsub_rn(bx0, r.x), __fsub_rn(r.x, bx1)));
            const float ey = fmaxf(0.f, fmaxf(__fsub_rn(by0, r.y), __fsub_rn(r.y, by1)));
            const float ez = fmaxf(0.f, fmaxf(__fsub_rn(bz0, r.z), __fsub_rn(r.z, bz1)));
            keep = (k >= c0 && k < c0 + ncen) || !(r2_rn(ex, ey, ez) > hi_f);
          }
          const unsigned m = __ballot_sync(0xffffffffu, keep);
          if (lane == 0) sm.s_wcnt[warp] = __popc(m);
          __syncthreads();
          int off = kept, tot = kept;
#pragma unroll
          for (int w = 0; w < kRowThreads / 32; ++w) {
            const int cw = sm.s_wcnt[w];
            off += w < warp ? cw : 0;
            tot += cw;
          }
          off += __popc(m & lt_mask);
          if (keep) stage[off] = r;
          if (k == c0 && ncen > 0) sm.s_c0 = off;
          kept = tot;
          __syncthreads();
        }
      }
      for (int k = kept + threadIdx.x; k < ((kept + 31) & ~31); k += kRowThreads)
        stage[k] = sentinel;
    }
    __syncthreads();
    // candidates swept and the center cell's first one
    const int ncand = kept;
    const int cbase = (staged && !WRAP && ncen > 0) ? sm.s_c0 : c0;
    // staged records (the hot path) or records rebuilt on the fly
    if (staged) {
      for (int a = warp; a < ncen; a += kRowThreads / 32)
        row(stage[cbase + a], cbase + a, [&](int k) { return stage[k]; }, ncand,
            std::true_type{});
    } else {
      for (int a = warp; a < ncen; a += kRowThreads / 32)
        row(record(cbase + a), cbase + a, record, ncand, std::false_type{});
    }
  }
  // Status: one atomic per CTA, and only when something needs reporting --
  // the maximum for a sizing (count-only) pass, the overflow flag when a
  // padded row is too short.
  if (status) {
    int* const s_max = sm.s_max;
    if (lane == 0) s_max[warp] = wmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      int m = 0;
      for (int w = 0; w < kRowThreads / 32; ++w) m = s_max[w] > m ? s_max[w] : m;
      const bool overflow = WRITE && !row_off && m > cap;
      if (overflow) atomicOr(&status[0], 1);
      if (overflow || !WRITE) atomicMax(&status[1], m);
    }
  }
}

template <class Load, bool WRAP, bool WRITE>
__global__ void __launch_bounds__(kRowThreads) k_build_cells(
    Load pos, DevBox b, const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const int* __restrict__ cell_atoms, double rl2, float lo_f, float hi_f, int* __restrict__ nbr,
    const int* __restrict__ row_off, int cap, int* __restrict__ counts,
    int* __restrict__ status, int stage_cap) {
  dependent_launch_prologue();
  // The stage is dynamic shared memory of stage_cap records (sized by the
  // launch from the mean cell occupancy, so that more CTAs fit on an SM).
  extern __shared__ float4 stage[];
  __shared__ RowSmem sm;
  build_cell_rows<Load, WRAP, WRITE, false>(sm, stage, stage_cap, nullptr, pos, b, blockIdx.x,
                                            cell_start, cell_count, cell_atoms, rl2, lo_f, hi_f,
                                            nbr, row_off, cap, counts, status);
}

// Batched replicas: one CTA per cell of any replica (cells of replica r are
// global cells [cell0, cell0 + ncells)); the replica's box, filter band and
// 3-cell-axis flag come from its descriptor.
template <bool WRITE>
__global__ void __launch_bounds__(kRowThreads) k_build_cells_batch(
    LoadD4 pos, const RepDesc* __restrict__ reps, const int* __restrict__ cell_rep,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const int* __restrict__ cell_atoms, double rl2, int* __restrict__ nbr, int cap,
    int* __restrict__ counts, int* __restrict__ status) {
  dependent_launch_prologue();
  __shared__ float4 stage[kStageCap];
  __shared__ RowSmem sm;
  __shared__ SlabSmem ss;
  __shared__ RepDesc d;
  const int gc = blockIdx.x;
  if (threadIdx.x == 0) d = reps[__ldg(cell_rep + gc)];
  __syncthreads();
  if (d.wrap)
    build_cell_rows<LoadD4, true, WRITE, true>(sm, stage, kStageCap, &ss, pos, d.box, gc - d.cell0,
                                               cell_start + d.cell0, cell_count + d.cell0,
                                               cell_atoms, rl2, d.lo_f, d.hi_f, nbr, nullptr,
                                               cap, counts, status);
  else
    build_cell_rows<LoadD4, false, WRITE, true>(sm, stage, kStageCap, &ss, pos, d.box,
                                                gc - d.cell0,
                                                cell_start + d.cell0, cell_count + d.cell0,
                                                cell_atoms, rl2, d.lo_f, d.hi_f, nbr, nullptr,
                                                cap, counts, status);
}

// Batched binning: the replica of atom i is rep[i]; its cell is the
// replica's first global cell plus the local index in the replica's grid.
__global__ void k_bin_atoms_batch(LoadD4 pos, const int* __restrict__ rep,
                                  const RepDesc* __restrict__ reps, int n,
                                  int* __restrict__ atom_cell, int* __restrict__ cell_count) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDesc* d = reps + __ldg(rep + i);
  const DevBox& b = d->box;
  const double3 p = pos(i);
  const int ix = cell_coord(p.x, b.lo[0], b.cs[0], b.nc[0]);
  const int iy = cell_coord(p.y, b.lo[1], b.cs[1], b.nc[1]);
  const int iz = cell_coord(p.z, b.lo[2], b.cs[2], b.nc[2]);
  const int c = d->cell0 + iz * b.nc[0] * b.nc[1] + iy * b.nc[0] + ix;
  atom_cell[i] = c;
  atomicAdd(&cell_count[c], 1);
}

}  // namespace

void build_cell_list(CellListDev& cl, const void* d_pos, PosLayout layout, long long n,
                     const DevBox& box, cudaStream_t stream, const int* key) {
  TDMD_REQUIRE(n >= 0 && n < INT_MAX, "atom count out of range");
  const long long ncells = 1ll * box.nc[0] * box.nc[1] * box.nc[2];
  TDMD_REQUIRE(ncells < INT_MAX / 2, "cell grid too large");
  cl.nc[0] = box.nc[0];
  cl.nc[1] = box.nc[1];
  cl.nc[2] = box.nc[2];
  cl.ncells = static_cast<int>(ncells);
  cl.natoms = n;
  cl.atom_cell.reserve(static_cast<size_t>(n));
  cl.cell_atoms.reserve(static_cast<size_t>(n));
  cl.cell_count.reserve(static_cast<size_t>(ncells));
  cl.cell_start.reserve(static_cast<size_t>(ncells));
  cl.cursor.reserve(static_cast<size_t>(ncells));
  if (n == 0) return;
  TDMD_CU(cudaMemsetAsync(cl.cell_count.data(), 0, sizeof(int) * ncells, stream));
  const int nb = ceil_div(n, 256);
  if (layout == PosLayout::AoS3)
    launch(k_bin_atoms<LoadAoS3>, nb, 256, 0, stream, LoadAoS3{static_cast<const double*>(d_pos)},
           static_cast<int>(n), box, cl.atom_cell.data(), cl.cell_count.data());
  else
    launch(k_bin_atoms<LoadD4>, nb, 256, 0, stream, LoadD4{static_cast<const double4*>(d_pos)},
           static_cast<int>(n), box, cl.atom_cell.data(), cl.cell_count.data());
  TDMD_LAUNCH_CHECK();
  // the scatter's cursors start as a copy of the cell starts
  device_exclusive_scan(cl.cell_count.data(), cl.cell_start.data(), ncells, nullptr, cl.scan_tmp,
                        stream, cl.cursor.data());
  launch(k_scatter_atoms, nb, 256, 0, stream, cl.atom_cell.data(), static_cast<int>(n),
         cl.cursor.data(), cl.cell_atoms.data());
  TDMD_LAUNCH_CHECK();
  launch(k_sort_cells, ceil_div(ncells * 32, 256), 256, 0, stream, cl.cell_start.data(),
         cl.cell_count.data(), static_cast<int>(ncells), cl.cell_atoms.data(), key);
  TDMD_LAUNCH_CHECK();
}

void row_filter_band(const DevBox& box, double r_list_sq, float* lo_f, float* hi_f, int* wrap) {
  // Band of the FP32 filter (see build_cell_rows).
  const double step = std::max(box.qstep[0], std::max(box.qstep[1], box.qstep[2]));
  const double rl = std::sqrt(r_list_sq);
  const double eps = 3e-5 + 8.0 * step / (rl > 0.0 ? rl : 1.0);
  *lo_f = static_cast<float>(r_list_sq * (1.0 - eps));
  *hi_f = static_cast<float>(r_list_sq * (1.0 + eps));
  // Relative coordinates are minimum-imaged by the int32 wrap when every
  // periodic axis has >= 4 cells (candidates then lie within 2 cells of the
  // corner, under L/2); 3-cell axes re-apply the minimum image in FP32.
  int w = 0;
  for (int a = 0; a < 3; ++a) w = w || (box.periodic[a] && box.nc[a] < 4);
  *wrap = w;
}

void build_cell_list_batch(CellListDev& cl, const double4* pos, const int* rep,
                           const RepDesc* reps, long long n, int ncells_total,
                           cudaStream_t stream) {
  TDMD_REQUIRE(n >= 0 && n < INT_MAX, "atom count out of range");
  cl.nc[0] = cl.nc[1] = cl.nc[2] = 0;
  cl.ncells = ncells_total;
  cl.natoms = n;
  cl.atom_cell.reserve(static_cast<size_t>(n));
  cl.cell_atoms.reserve(static_cast<size_t>(n));
  cl.cell_count.reserve(static_cast<size_t>(ncells_total));
  cl.cell_start.reserve(static_cast<size_t>(ncells_total));
  cl.cursor.reserve(static_cast<size_t>(ncells_total));
  if (n == 0) return;
  TDMD_CU(cudaMemsetAsync(cl.cell_count.data(), 0, sizeof(int) * ncells_total, stream));
  const int nb = ceil_div(n, 256);
  launch(k_bin_atoms_batch, nb, 256, 0, stream, LoadD4{pos}, rep, reps, static_cast<int>(n),
         cl.atom_cell.data(), cl.cell_count.data());
  TDMD_LAUNCH_CHECK();
  device_exclusive_scan(cl.cell_count.data(), cl.cell_start.data(), ncells_total, nullptr,
                        cl.scan_tmp, stream, cl.cursor.data());
  launch(k_scatter_atoms, nb, 256, 0, stream, cl.atom_cell.data(), static_cast<int>(n),
         cl.cursor.data(), cl.cell_atoms.data());
  TDMD_LAUNCH_CHECK();
  launch(k_sort_cells, ceil_div(1ll * ncells_total * 32, 256), 256, 0, stream, cl.cell_start.data(),
         cl.cell_count.data(), ncells_total, cl.cell_atoms.data(), nullptr);
  TDMD_LAUNCH_CHECK();
}

void build_neighbor_rows_batch(const CellListDev& cl, const double4* pos, const RepDesc* reps,
                               const int* cell_rep, double r_list_sq, int* nbr, int cap,
                               int* counts, int* status, cudaStream_t stream) {
  if (cl.natoms == 0 || cl.ncells == 0) return;
  if (nbr)
    launch(k_build_cells_batch<true>, cl.ncells, kRowThreads, 0, stream, LoadD4{pos}, reps,
           cell_rep, cl.cell_start.data(), cl.cell_count.data(), cl.cell_atoms.data(), r_list_sq,
           nbr, cap, counts, status);
  else
    launch(k_build_cells_batch<false>, cl.ncells, kRowThreads, 0, stream, LoadD4{pos}, reps,
           cell_rep, cl.cell_start.data(), cl.cell_count.data(), cl.cell_atoms.data(), r_list_sq,
           nullptr, cap, counts, status);
  TDMD_LAUNCH_CHECK();
}

// Staged records per row-building CTA from the largest cell occupancy seen
// (27 cells of it, plus a quarter for atoms that move in later): 768 to 1536
// records (12 to 24 KiB); unknown (<= 0): 1536.  Cells with more candidates
// build their rows from records made on the fly.
static int stage_capacity(int max_cell) {
  if (max_cell <= 0) return kStageCap;
  const int want = (static_cast<int>(std::ceil(27.0 * 1.25 * max_cell)) + 31) & ~31;
  return std::min(kStageCap, std::max(768, want));
}

namespace {
// Largest cell occupancy, one block.
__global__ void k_max_count(const int* __restrict__ count, int ncells, int* __restrict__ out) {
  dependent_launch_prologue();
  __shared__ int red[32];
  int m = 0;
  for (int c = threadIdx.x; c < ncells; c += blockDim.x) m = max(m, count[c]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = max(m, red[w]);
    *out = m;
  }
}
}  // namespace

void cell_count_max(const CellListDev& cl, int* d_out, cudaStream_t stream) {
  launch(k_max_count, 1, 1024, 0, stream, cl.cell_count.data(), cl.ncells, d_out);
  TDMD_LAUNCH_CHECK();
}

void build_neighbor_rows(const CellListDev& cl, const void* d_pos, PosLayout layout,
                         long long n, const DevBox& box, double r_list_sq, int* nbr,
                         const int* row_off, int cap, int* counts, int* status,
                         cudaStream_t stream, int max_cell) {
  if (n == 0) return;
  float lo_f = 0.f, hi_f = 0.f;
  int wrap = 0;
  row_filter_band(box, r_list_sq, &lo_f, &hi_f, &wrap);
  const int scap = stage_capacity(max_cell);
  const size_t smem = sizeof(float4) * static_cast<size_t>(scap);
  auto go = [&](auto load, auto wrap_tag) {
    constexpr bool W = decltype(wrap_tag)::value;
    if (nbr)
      launch(k_build_cells<decltype(load), W, true>, cl.ncells, kRowThreads, smem, stream, load,
             box, cl.cell_start.data(), cl.cell_count.data(), cl.cell_atoms.data(), r_list_sq, lo_f,
             hi_f, nbr, row_off, cap, counts, status, scap);
    else
      launch(k_build_cells<decltype(load), W, false>, cl.ncells, kRowThreads, smem, stream, load,
             box, cl.cell_start.data(), cl.cell_count.data(), cl.cell_atoms.data(), r_list_sq, lo_f,
             hi_f, nullptr, row_off, cap, counts, status, scap);
  };
  if (layout == PosLayout::AoS3) {
    const LoadAoS3 ld{static_cast<const double*>(d_pos)};
    if (wrap) go(ld, std::true_type{}); else go(ld, std::false_type{});
  } else {
    const LoadD4 ld{static_cast<const double4*>(d_pos)};
    if (wrap) go(ld, std::true_type{}); else go(ld, std::false_type{});
  }
  TDMD_LAUNCH_CHECK();
}

}  // namespace tdmd_b200

// ---------------------------------------------------------------------------
// C ABI: DeviceCellList / DeviceNeighborList on caller-owned positions.
// ---------------------------------------------------------------------------
using namespace tdmd_b200;

struct tdmd_cell_list {
  CellListDev cl;
};

struct tdmd_nlist {
  CellListDev cl;
  DevArray<int> counts;
  DevArray<int> offsets;
  DevArray<int> nbrs;
  DevArray<int> status;  // [0] overflow, [1] max count, [2] total
  int max_neighbors = 0;
  long long total = 0;
  long long natoms = 0;
};

extern "C" {

int32_t tdmd_cell_list_create(tdmd_cell_list** out) {
  return guarded([&] {
    TDMD_REQUIRE(out, "out is null");
    *out = new tdmd_cell_list();
  });
}

int32_t tdmd_cell_list_destroy(tdmd_cell_list* cl) {
  delete cl;
  return TDMD_OK;
}

int32_t tdmd_cell_list_build(tdmd_cell_list* cl, const double* d_positions, int64_t natoms,
                             const tdmd_box* box, double r_list, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(cl && box, "null handle or box");
    TDMD_REQUIRE(r_list > 0.0, "r_list must be positive");
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    TDMD_REQUIRE(natoms == 0 || d_positions, "positions are null");
    const DevBox b = make_devbox(*box, r_list);
    build_cell_list(cl->cl, d_positions, PosLayout::AoS3, natoms, b, as_stream(stream));
  });
}

int32_t tdmd_cell_list_get(const tdmd_cell_list* cl, const int32_t** cell_atoms,
                           const int32_t** cell_offsets, const int32_t** cell_counts,
                           const int32_t** atom_cells, int32_t nc[3]) {
  return guarded([&] {
    TDMD_REQUIRE(cl, "null handle");
    if (cell_atoms) *cell_atoms = cl->cl.cell_atoms.data();
    if (cell_offsets) *cell_offsets = cl->cl.cell_start.data();
    if (cell_counts) *cell_counts = cl->cl.cell_count.data();
    if (atom_cells) *atom_cells = cl->cl.atom_cell.data();
    if (nc) {
      nc[0] = cl->cl.nc[0];
      nc[1] = cl->cl.nc[1];
      nc[2] = cl->cl.nc[2];
    }
  });
}

int32_t tdmd_nlist_create(tdmd_nlist** out) {
  return guarded([&] {
    TDMD_REQUIRE(out, "out is null");
    *out = new tdmd_nlist();
  });
}

int32_t tdmd_nlist_destroy(tdmd_nlist* nl) {
  delete nl;
  return TDMD_OK;
}

// Two passes (count, device scan, fill) into dense CSR, like the reference;
// the one host round trip sizes the neighbor array, as in
// device_neighbor_list.cu:246-249.
int32_t tdmd_nlist_build(tdmd_nlist* nl, const double* d_positions, int64_t natoms,
                         const tdmd_box* box, double r_cut, double r_skin, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(nl && box, "null handle or box");
    TDMD_REQUIRE(r_cut > 0.0, "r_cut must be positive");
    TDMD_REQUIRE(r_skin >= 0.0, "r_skin must be non-negative");
    TDMD_REQUIRE(natoms >= 0 && natoms < INT_MAX, "natoms out of range");
    TDMD_REQUIRE(natoms == 0 || d_positions, "positions are null");
    nl->natoms = natoms;
    nl->total = 0;
    nl->max_neighbors = 0;
    if (natoms == 0) return;
    cudaStream_t s = as_stream(stream);
    const double r_list = r_cut + r_skin;
    const double rl2 = r_list * r_list;
    const DevBox b = make_devbox(*box, r_list);
    build_cell_list(nl->cl, d_positions, PosLayout::AoS3, natoms, b, s);
    nl->counts.reserve(static_cast<size_t>(natoms));
    nl->offsets.reserve(static_cast<size_t>(natoms));
    nl->status.reserve(4);
    TDMD_CU(cudaMemsetAsync(nl->status.data(), 0, 4 * sizeof(int), s));
    build_neighbor_rows(nl->cl, d_positions, PosLayout::AoS3, natoms, b, rl2, nullptr, nullptr,
                        0, nl->counts.data(), nl->status.data(), s);
    device_exclusive_scan(nl->counts.data(), nl->offsets.data(), natoms, nl->status.data() + 2,
                          nl->cl.scan_tmp, s);
    int h[4] = {0, 0, 0, 0};
    TDMD_CU(cudaMemcpyAsync(h, nl->status.data(), sizeof(h), cudaMemcpyDeviceToHost, s));
    TDMD_CU(cudaStreamSynchronize(s));
    nl->max_neighbors = h[1];
    nl->total = h[2];
    nl->nbrs.reserve(static_cast<size_t>(nl->total > 0 ? nl->total : 1));
    build_neighbor_rows(nl->cl, d_positions, PosLayout::AoS3, natoms, b, rl2, nl->nbrs.data(),
                        nl->offsets.data(), 0, nl->counts.data(), nullptr, s);
  });
}

int32_t tdmd_nlist_get(const tdmd_nlist* nl, const int32_t** d_neighbors,
                       const int32_t** d_offsets, const int32_t** d_counts,
                       int32_t* max_neighbors, int64_t* total_pairs) {
  return guarded([&] {
    TDMD_REQUIRE(nl, "null handle");
    if (d_neighbors) *d_neighbors = nl->nbrs.data();
    if (d_offsets) *d_offsets = nl->offsets.data();
    if (d_counts) *d_counts = nl->counts.data();
    if (max_neighbors) *max_neighbors = nl->max_neighbors;
    if (total_pairs) *total_pairs = nl->total;
  });
}

}  // extern "C"
