// replicas.cuh -- descriptors of batched independent replicas (batch.cu)
// shared with the batched cell-list / neighbor-list kernels in nlist.cu.
#pragma once

#include "buffers.cuh"
#include "common.cuh"

namespace tdmd_b200 {

// One replica of a batch.  Its atoms are [atom0, atom0 + natoms) of the
// batch arrays, its cells [cell0, cell0 + ncells) of the batch cell list.
struct RepDesc {
  DevBox box;       // box, cell grid for r_list, fixed-point map
  int atom0, natoms;
  int cell0, ncells;
  float lo_f, hi_f;  // FP32 filter band of the list build
  int wrap;          // a periodic axis with 3 cells (FP32 minimum image)
  int pad;
};

// Per-replica fixed-point decode scales of the mixed force path.
struct RepScale {
  float s[3];
  int iso;       // one step on all three axes
  double s2[3];  // (Lq / 2^32)^2
  double pad2;
};

// Band [lo_f, hi_f] around r_list^2 outside which the list build's FP32
// filter decides (inside it the FP64 reference expression decides), and
// whether the grid needs the FP32 minimum image (a 3-cell periodic axis).
void row_filter_band(const DevBox& box, double r_list_sq, float* lo_f, float* hi_f, int* wrap);

// Cell list of all replicas at once (global cells; ID order within each).
void build_cell_list_batch(CellListDev& cl, const double4* pos, const int* rep,
                           const RepDesc* reps, long long n, int ncells_total,
                           cudaStream_t stream);

// Padded neighbor rows (entry k of atom i at nbr[i*cap + k]) of every
// replica; status[0] |= 1 on overflow, status[1] = max count.
void build_neighbor_rows_batch(const CellListDev& cl, const double4* pos, const RepDesc* reps,
                               const int* cell_rep, double r_list_sq, int* nbr, int cap,
                               int* counts, int* status, cudaStream_t stream);

}  // namespace tdmd_b200
