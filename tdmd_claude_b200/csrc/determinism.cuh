// determinism.cuh -- the ID-ordered energy mode of the free-function force
// calls (determinism.cu).
#pragma once

#include <cuda_runtime.h>

#include "buffers.cuh"
#include "eam_tables.cuh"
#include "tdmd_b200.h"

namespace tdmd_b200 {

// tdmd_set_deterministic_reduce's process-wide switch.
bool deterministic_reduce();

// One spline in the reference's device layout (DeviceSpline,
// src/potentials/device_eam.cuh:15-20): a|b|c|d blocks of n-1 entries at
// `offset` of one flat FP64 coefficient array.
struct RefSpline {
  double dr;
  double rmin;
  int n;
  int offset;
};

// All splines of an EAM in that layout: embedding per type, density per
// type, phi per pair, one flat array (DeviceEam::upload_tables,
// device_eam.cu:282-340).
struct RefEamTables {
  DevArray<double> coeff;
  DevArray<RefSpline> splines;  // [nt embedding | nt density | npairs phi]
  int ntypes = 0;
  double cutoff = 0.0;
  void upload(const tdmd_eam& e);
};

// FP64 forces (stored), and energy / virial ADDED in atom-ID order
// (nullable), from the reference's per-atom arithmetic; rows are dense CSR.
void morse_id_ordered(const double* pos, double* forces, const int* nbr, const int* off,
                      const int* cnt, int n, const tdmd_box& box, const tdmd_morse_params& p,
                      double* energy, double* virial, cudaStream_t s);
void eam_id_ordered(const RefEamTables& t, const double* pos, double* forces, const int* types,
                    const int* nbr, const int* off, const int* cnt, int n, const tdmd_box& box,
                    double* energy, double* virial, double* rho_out, double* fp_out,
                    cudaStream_t s);

}  // namespace tdmd_b200
