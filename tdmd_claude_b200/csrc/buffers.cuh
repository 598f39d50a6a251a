// buffers.cuh -- owning device arrays and the cell/neighbor list data the
// kernels share.  The reference's DeviceBuffer<T> (src/core/device_buffer.cuh:
// 30-116) copies synchronously on the legacy stream; these arrays only
// allocate, and every copy or memset is issued by the caller on its stream.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <utility>

#include "common.cuh"

namespace tdmd_b200 {

template <class T>
class DevArray {
 public:
  DevArray() = default;
  explicit DevArray(size_t n) { reserve(n); }
  ~DevArray() { release(); }
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  DevArray(DevArray&& o) noexcept : p_(o.p_), cap_(o.cap_) {
    o.p_ = nullptr;
    o.cap_ = 0;
  }
  DevArray& operator=(DevArray&& o) noexcept {
    if (this != &o) {
      release();
      p_ = std::exchange(o.p_, nullptr);
      cap_ = std::exchange(o.cap_, 0);
    }
    return *this;
  }

  // Grow-only: keeps the allocation when it is already large enough.
  // Contents are NOT preserved on growth.
  void reserve(size_t n) {
    if (n <= cap_) return;
    release();
    void* p = nullptr;
    TDMD_CU(cudaMalloc(&p, (n > 0 ? n : 1) * sizeof(T)));
    p_ = static_cast<T*>(p);
    cap_ = n;
  }
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    cap_ = 0;
  }
  T* data() const { return p_; }
  size_t capacity() const { return cap_; }

 private:
  T* p_ = nullptr;
  size_t cap_ = 0;
};

// Device-resident cell list (counting sort of atoms into cells), produced by
// build_cell_list() in nlist.cu.
struct CellListDev {
  DevArray<int> atom_cell;   // [n]
  DevArray<int> cell_count;  // [ncells]
  DevArray<int> cell_start;  // [ncells] exclusive scan of cell_count
  DevArray<int> cursor;      // [ncells] scatter cursor
  DevArray<int> cell_atoms;  // [n] atoms sorted by cell, ID-ascending
  DevArray<int> scan_tmp;    // block sums of the device scan
  int nc[3] = {0, 0, 0};
  int ncells = 0;
  long long natoms = 0;
};

// Exclusive scan of in[0..n) into out[0..n) (and out2, when non-null);
// *total (device, nullable) gets the sum.  Fixed order.
void device_exclusive_scan(const int* in, int* out, long long n, int* total, DevArray<int>& tmp,
                           cudaStream_t stream, int* out2 = nullptr);
// Kernels one device_exclusive_scan of n items launches (1 or 3).
int device_scan_launches(long long n);

// Positions are read either as the reference's Vec3D AoS (double[3n]) or as
// the scheduler's double4 {x, y, z, type} records.
enum class PosLayout { AoS3, D4 };

// Builds the cell list of n atoms (positions on the device, laid out per
// `layout`) on `stream`.  Grid and cell size come from `box`.  Atoms within
// a cell are ordered by index, or by key[index] when key is given (arrays
// held in an internal order; key[i] = the caller's index of atom i).
void build_cell_list(CellListDev& cl, const void* d_pos, PosLayout layout, long long n,
                     const DevBox& box, cudaStream_t stream, const int* key = nullptr);

// Neighbor list build over a built cell list.
//   row_off == nullptr: padded rows, entry k of atom i at nbr[i*cap + k];
//                       status[0] |= 1 when some atom has more than cap.
//   row_off != nullptr: dense CSR rows at nbr[row_off[i] + k].
//   nbr == nullptr:     count only.
// counts[i] always gets the full count; status[1] = max count (atomicMax).
// max_cell: the largest cell occupancy seen (sizes the shared-memory stage;
// <= 0 = unknown, the full stage).
void build_neighbor_rows(const CellListDev& cl, const void* d_pos, PosLayout layout,
                         long long n, const DevBox& box, double r_list_sq, int* nbr,
                         const int* row_off, int cap, int* counts, int* status,
                         cudaStream_t stream, int max_cell = 0);

// *d_out = the largest cell occupancy of a built cell list (one launch).
void cell_count_max(const CellListDev& cl, int* d_out, cudaStream_t stream);

}  // namespace tdmd_b200
