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
//  * list build: one warp per atom.  The 27-cell stencil is walked as 9 rows
//    of 3 x-adjacent cells; the lanes take 32 candidates at a time, test
//    r^2 < (rc+skin)^2 in FP64 with explicit round-to-nearest ops (no FMA
//    contraction, so r^2 matches the CPU reference bit for bit), and a
//    ballot/popc compaction writes accepted neighbors in stencil order.  One
//    pass: rows are padded to a fixed capacity and an overflow flag replaces
//    the reference's count pass + 8-byte D2H sync.
#include <climits>

#include "buffers.cuh"
#include "common.cuh"

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
    const double2* q = reinterpret_cast<const double2*>(p + i);
    const double2 a = __ldg(q);
    const double b = __ldg(reinterpret_cast<const double*>(q + 1));
    return make_double3(a.x, a.y, b);
  }
};

template <class Load>
__global__ void k_bin_atoms(Load pos, int n, DevBox b, int* __restrict__ atom_cell,
                            int* __restrict__ cell_count) {
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
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = atomicAdd(&cursor[atom_cell[i]], 1);
  cell_atoms[slot] = i;
}

// Restores ID-ascending order inside each cell (insertion sort; cells hold
// a few tens of atoms).  One thread per cell.
__global__ void k_sort_cells(const int* __restrict__ cell_start, const int* __restrict__ cell_count,
                             int ncells, int* __restrict__ cell_atoms) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int* a = cell_atoms + cell_start[c];
  const int m = cell_count[c];
  for (int k = 1; k < m; ++k) {
    const int v = a[k];
    int j = k - 1;
    while (j >= 0 && a[j] > v) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = v;
  }
}

// Warp per atom.  See the file comment for the scheme.
template <class Load>
__global__ void __launch_bounds__(256) k_build_rows(
    Load pos, int n, DevBox b, const int* __restrict__ atom_cell,
    const int* __restrict__ cell_start, const int* __restrict__ cell_count,
    const int* __restrict__ cell_atoms, double rl2, int* __restrict__ nbr,
    const int* __restrict__ row_off, int cap, int* __restrict__ counts,
    int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const long long gw = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (gw >= n) return;  // uniform per warp
  const int i = static_cast<int>(gw);
  const double3 pi = pos(i);
  const int ncx = b.nc[0], ncy = b.nc[1], ncz = b.nc[2];
  const int ncxy = ncx * ncy;
  const int ci = atom_cell[i];
  const int iz = ci / ncxy;
  const int iy = (ci - iz * ncxy) / ncx;
  const int ix = ci - iz * ncxy - iy * ncx;
  const long long base = row_off ? static_cast<long long>(row_off[i])
                                 : static_cast<long long>(i) * cap;
  const int limit = row_off ? INT_MAX : cap;
  const int xm = wrap_cell(ix - 1, ncx), xp = wrap_cell(ix + 1, ncx);
  const unsigned lt_mask = (1u << lane) - 1u;
  int cnt = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    const int cz = wrap_cell(iz + dz, ncz);
    for (int dy = -1; dy <= 1; ++dy) {
      const int row = cz * ncxy + wrap_cell(iy + dy, ncy) * ncx;
      const int c0 = row + xm, c1 = row + ix, c2 = row + xp;
      const int s0 = cell_start[c0], n0 = cell_count[c0];
      const int s1 = cell_start[c1], n1 = cell_count[c1];
      const int s2 = cell_start[c2], n2 = cell_count[c2];
      const int n01 = n0 + n1;
      const int T = n01 + n2;
      for (int k0 = 0; k0 < T; k0 += 32) {
        const int k = k0 + lane;
        bool pred = false;
        int j = -1;
        if (k < T) {
          const int slot = k < n0 ? s0 + k : (k < n01 ? s1 + (k - n0) : s2 + (k - n01));
          j = cell_atoms[slot];
          if (j != i) {
            const double3 pj = pos(j);
            // delta = r_j - r_i, minimum image, r^2 = (x*x + y*y) + z*z,
            // all round-to-nearest: NeighborList::build, neighbor_list.cpp:57-63.
            double dx = min_image1(__dsub_rn(pj.x, pi.x), b.L[0], b.halfL[0], b.periodic[0]);
            double dy2 = min_image1(__dsub_rn(pj.y, pi.y), b.L[1], b.halfL[1], b.periodic[1]);
            double dz2 = min_image1(__dsub_rn(pj.z, pi.z), b.L[2], b.halfL[2], b.periodic[2]);
            const double r2 =
                __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy2, dy2)), __dmul_rn(dz2, dz2));
            pred = r2 < rl2;
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, pred);
        if (pred && nbr) {
          const int p = cnt + __popc(m & lt_mask);
          if (p < limit) nbr[base + p] = j;
        }
        cnt += __popc(m);
      }
    }
  }
  if (lane == 0) {
    counts[i] = cnt;
    if (status) {
      if (!row_off && cnt > cap) atomicOr(&status[0], 1);
      atomicMax(&status[1], cnt);
    }
  }
}

}  // namespace

void build_cell_list(CellListDev& cl, const void* d_pos, PosLayout layout, long long n,
                     const DevBox& box, cudaStream_t stream) {
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
    k_bin_atoms<<<nb, 256, 0, stream>>>(LoadAoS3{static_cast<const double*>(d_pos)},
                                        static_cast<int>(n), box, cl.atom_cell.data(),
                                        cl.cell_count.data());
  else
    k_bin_atoms<<<nb, 256, 0, stream>>>(LoadD4{static_cast<const double4*>(d_pos)},
                                        static_cast<int>(n), box, cl.atom_cell.data(),
                                        cl.cell_count.data());
  TDMD_LAUNCH_CHECK();
  device_exclusive_scan(cl.cell_count.data(), cl.cell_start.data(), ncells, nullptr, cl.scan_tmp,
                        stream);
  TDMD_CU(cudaMemcpyAsync(cl.cursor.data(), cl.cell_start.data(), sizeof(int) * ncells,
                          cudaMemcpyDeviceToDevice, stream));
  k_scatter_atoms<<<nb, 256, 0, stream>>>(cl.atom_cell.data(), static_cast<int>(n),
                                          cl.cursor.data(), cl.cell_atoms.data());
  TDMD_LAUNCH_CHECK();
  k_sort_cells<<<ceil_div(ncells, 128), 128, 0, stream>>>(cl.cell_start.data(),
                                                          cl.cell_count.data(),
                                                          static_cast<int>(ncells),
                                                          cl.cell_atoms.data());
  TDMD_LAUNCH_CHECK();
}

void build_neighbor_rows(const CellListDev& cl, const void* d_pos, PosLayout layout,
                         long long n, const DevBox& box, double r_list_sq, int* nbr,
                         const int* row_off, int cap, int* counts, int* status,
                         cudaStream_t stream) {
  if (n == 0) return;
  const int threads = 256;
  const long long blocks = (n * 32 + threads - 1) / threads;
  TDMD_REQUIRE(blocks < INT_MAX, "too many atoms for the list build grid");
  if (layout == PosLayout::AoS3)
    k_build_rows<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(
        LoadAoS3{static_cast<const double*>(d_pos)}, static_cast<int>(n), box,
        cl.atom_cell.data(), cl.cell_start.data(), cl.cell_count.data(), cl.cell_atoms.data(),
        r_list_sq, nbr, row_off, cap, counts, status);
  else
    k_build_rows<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(
        LoadD4{static_cast<const double4*>(d_pos)}, static_cast<int>(n), box,
        cl.atom_cell.data(), cl.cell_start.data(), cl.cell_count.data(), cl.cell_atoms.data(),
        r_list_sq, nbr, row_off, cap, counts, status);
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
