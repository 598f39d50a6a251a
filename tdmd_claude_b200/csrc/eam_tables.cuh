// eam_tables.cuh -- host-side EAM/alloy tables (the tdmd_eam handle) and
// their device copies.
//
// Mirrors EamAlloy (src/potentials/eam_alloy.hpp:47-93): per-type embedding
// F(rho) and density rho(r), per-pair phi(r) in the upper-triangle order
// phi_index(i,j) = i*nt - i*(i+1)/2 + j, phi stored as (r*phi)/r with
// phi(0) = 0, all as finite-difference cubic-Hermite splines
// (SplineTable::build_splines, eam_alloy.cpp:19-50).
#pragma once

#include <string>
#include <vector>

#include "buffers.cuh"
#include "forces.cuh"

struct tdmd_eam {
  int ntypes = 0;
  int nrho = 0;
  int nr = 0;
  double drho = 0.0;
  double dr = 0.0;
  double cutoff = 0.0;
  std::vector<std::string> elements;
  // setfl text kept for writing the tables back out: the 3 comment lines
  // and each element's header line (empty for tables built from arrays)
  std::vector<std::string> comments;
  std::vector<std::string> headers;
  std::vector<double> F;     // [ntypes][nrho] raw F(rho)
  std::vector<double> rho;   // [ntypes][nr]   raw rho(r)
  std::vector<double> rphi;  // [npairs][nr]   raw r*phi(r)
  // [npairs][nr] phi(r) itself, when the tables were given as phi samples
  // (empty otherwise: phi is then r*phi / r)
  std::vector<double> phi;
  // Packed a|b|c|d coefficients per spline, each block 4*(n-1) long.
  std::vector<double> Fc, rhoc, phic;
};

namespace tdmd_b200 {

// Builds the FD-Hermite coefficients (a|b|c|d blocks) of n knot values.
void build_spline(const double* values, int n, double dr, double* coef);

// Fills the coefficient arrays of an EAM whose raw tables are set.
void eam_build_coeffs(tdmd_eam& e);

// Device copy of one tdmd_eam: FP64 and FP32 r-spline rows plus the FP64
// embedding table.
struct EamDevTables {
  DevArray<double4> rtab64;  // force rows (b, 2c, 3d, a)
  DevArray<float4> rtab32;
  DevArray<double4> dtab64;  // density rows (a, b, c, d)
  DevArray<float4> dtab32;
  DevArray<double4> ftab;
  EamDev<double> d64{};
  EamDev<float> d32{};
  int ntypes = 0;
  double cutoff = 0.0;
  void upload(const tdmd_eam& e, cudaStream_t stream);
};

}  // namespace tdmd_b200
