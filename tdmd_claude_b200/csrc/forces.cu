// forces.cu -- EAM table set-up (setfl reader, spline coefficients, device
// upload), the fixed-order energy/virial reduction and the free-function
// force entry points of the C ABI (compute_morse_gpu, DeviceEam).
#include <cctype>
#include <climits>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "buffers.cuh"
#include "common.cuh"
#include "eam_tables.cuh"
#include "forces.cuh"
#include "determinism.cuh"
#include "launch.cuh"

namespace tdmd_b200 {

// --------------------------------------------------------------------------
// Splines: SplineTable::build_splines, src/potentials/eam_alloy.cpp:19-50
// (cubic Hermite with averaged finite-difference slopes, one-sided at the
// two ends).  Restated; the coefficient formulas must be the same for the
// tables to agree with the reference.
// --------------------------------------------------------------------------
void build_spline(const double* v, int n, double dr, double* coef) {
  if (n < 2) return;
  const int ns = n - 1;
  double* a = coef;
  double* b = coef + ns;
  double* c = coef + 2 * ns;
  double* d = coef + 3 * ns;
  for (int i = 0; i < ns; ++i) {
    const double right = (v[i + 1] - v[i]) / dr;
    const double left = i > 0 ? (v[i] - v[i - 1]) / dr : 0.0;
    const double next = i + 2 < n ? (v[i + 2] - v[i + 1]) / dr : right;
    double m0 = (left + right) * 0.5;
    double m1 = (right + next) * 0.5;
    if (i == 0) m0 = right;
    if (i == ns - 1) m1 = right;
    a[i] = v[i];
    b[i] = m0;
    c[i] = (3.0 * right - 2.0 * m0 - m1) / dr;
    d[i] = (m0 + m1 - 2.0 * right) / (dr * dr);
  }
}

void eam_build_coeffs(tdmd_eam& e) {
  const int nt = e.ntypes;
  const int npairs = nt * (nt + 1) / 2;
  e.Fc.assign(static_cast<size_t>(nt) * 4 * (e.nrho - 1), 0.0);
  e.rhoc.assign(static_cast<size_t>(nt) * 4 * (e.nr - 1), 0.0);
  e.phic.assign(static_cast<size_t>(npairs) * 4 * (e.nr - 1), 0.0);
  for (int t = 0; t < nt; ++t) {
    build_spline(e.F.data() + static_cast<size_t>(t) * e.nrho, e.nrho, e.drho,
                 e.Fc.data() + static_cast<size_t>(t) * 4 * (e.nrho - 1));
    build_spline(e.rho.data() + static_cast<size_t>(t) * e.nr, e.nr, e.dr,
                 e.rhoc.data() + static_cast<size_t>(t) * 4 * (e.nr - 1));
  }
  // phi = (r*phi)/r with phi(0) = 0, eam_alloy.cpp:176-188, unless the
  // tables came as phi samples.
  std::vector<double> phi(static_cast<size_t>(e.nr));
  for (int p = 0; p < npairs; ++p) {
    const size_t off = static_cast<size_t>(p) * e.nr;
    if (!e.phi.empty()) {
      std::copy(e.phi.begin() + static_cast<long>(off),
                e.phi.begin() + static_cast<long>(off + e.nr), phi.begin());
    } else {
      const double* rp = e.rphi.data() + off;
      phi[0] = 0.0;
      for (int k = 1; k < e.nr; ++k) phi[static_cast<size_t>(k)] = rp[k] / (k * e.dr);
    }
    build_spline(phi.data(), e.nr, e.dr, e.phic.data() + static_cast<size_t>(p) * 4 * (e.nr - 1));
  }
}

// --------------------------------------------------------------------------
// setfl reader, EamAlloy::read_setfl (eam_alloy.cpp:90-192): 3 comment
// lines; "ntypes el1 el2 ..."; "Nrho drho Nr dr cutoff"; per element a
// header line (atomic number, mass, lattice constant, lattice type -- not
// used) then Nrho F values and Nr rho values; then for each pair i <= j, Nr
// values of r*phi(r).  Values are whitespace separated, any number per line.
// --------------------------------------------------------------------------
namespace {

struct SetflReader {
  std::istream& in;
  std::string line;
  size_t pos = 0;  // position inside `line` (values may continue mid-line)
  bool have_line = false;

  bool next_line() {
    if (!std::getline(in, line)) return false;
    pos = 0;
    have_line = true;
    return true;
  }
  // Next whitespace-separated token, crossing lines.
  bool token(std::string& tok) {
    for (;;) {
      if (!have_line && !next_line()) return false;
      while (pos < line.size() && std::isspace(static_cast<unsigned char>(line[pos]))) ++pos;
      if (pos < line.size()) {
        const size_t start = pos;
        while (pos < line.size() && !std::isspace(static_cast<unsigned char>(line[pos]))) ++pos;
        tok = line.substr(start, pos - start);
        return true;
      }
      have_line = false;
    }
  }
  void values(int count, double* out, const char* what) {
    std::string tok;
    for (int k = 0; k < count; ++k) {
      if (!token(tok))
        throw Error{TDMD_ERR_PARSE, std::string("unexpected end of EAM file while reading ") + what};
      char* end = nullptr;
      out[k] = std::strtod(tok.c_str(), &end);
      if (end == tok.c_str() || *end != '\0')
        throw Error{TDMD_ERR_PARSE, std::string("bad number '") + tok + "' in " + what};
    }
  }
  // The element header: the rest of the current line if it holds anything,
  // else the next non-blank line.
  std::string header() {
    if (have_line) {
      while (pos < line.size() && std::isspace(static_cast<unsigned char>(line[pos]))) ++pos;
      if (pos < line.size()) {
        std::string h = line.substr(pos);
        have_line = false;
        return h;
      }
      have_line = false;
    }
    while (next_line()) {
      for (char ch : line)
        if (!std::isspace(static_cast<unsigned char>(ch))) {
          have_line = false;
          return line;
        }
    }
    throw Error{TDMD_ERR_PARSE, "premature end of EAM file (element header)"};
  }
};

}  // namespace

static void read_setfl(const std::string& path, tdmd_eam& e) {
  std::ifstream f(path);
  if (!f.is_open()) throw Error{TDMD_ERR_IO, "cannot open EAM file: " + path};
  std::string line;
  e.comments.clear();
  for (int k = 0; k < 3; ++k) {
    if (!std::getline(f, line)) throw Error{TDMD_ERR_PARSE, "premature end of EAM file"};
    if (!line.empty() && line.back() == '\r') line.pop_back();
    e.comments.push_back(line);
  }
  if (!std::getline(f, line)) throw Error{TDMD_ERR_PARSE, "premature end of EAM file"};
  {
    std::istringstream is(line);
    if (!(is >> e.ntypes) || e.ntypes < 1 || e.ntypes > 64)
      throw Error{TDMD_ERR_PARSE, "bad element count line: " + line};
    e.elements.resize(static_cast<size_t>(e.ntypes));
    for (auto& el : e.elements) is >> el;
  }
  if (!std::getline(f, line)) throw Error{TDMD_ERR_PARSE, "premature end of EAM file"};
  {
    std::istringstream is(line);
    if (!(is >> e.nrho >> e.drho >> e.nr >> e.dr >> e.cutoff))
      throw Error{TDMD_ERR_PARSE, "bad grid line: " + line};
  }
  if (e.nrho < 2 || e.nr < 2 || !(e.drho > 0) || !(e.dr > 0) || !(e.cutoff > 0))
    throw Error{TDMD_ERR_PARSE, "invalid grid sizes in EAM file"};
  const int nt = e.ntypes;
  const int npairs = nt * (nt + 1) / 2;
  e.F.assign(static_cast<size_t>(nt) * e.nrho, 0.0);
  e.rho.assign(static_cast<size_t>(nt) * e.nr, 0.0);
  e.rphi.assign(static_cast<size_t>(npairs) * e.nr, 0.0);
  SetflReader r{f};
  e.headers.assign(static_cast<size_t>(nt), std::string());
  for (int t = 0; t < nt; ++t) {
    std::string h = r.header();
    while (!h.empty() && (h.back() == '\r' || h.back() == ' ')) h.pop_back();
    e.headers[static_cast<size_t>(t)] = h;
    r.values(e.nrho, e.F.data() + static_cast<size_t>(t) * e.nrho, "F(rho)");
    r.values(e.nr, e.rho.data() + static_cast<size_t>(t) * e.nr, "rho(r)");
  }
  for (int p = 0; p < npairs; ++p)
    r.values(e.nr, e.rphi.data() + static_cast<size_t>(p) * e.nr, "r*phi(r)");
  eam_build_coeffs(e);
}

void EamDevTables::upload(const tdmd_eam& e, cudaStream_t stream) {
  const int nt = e.ntypes;
  const int npairs = nt * (nt + 1) / 2;
  const int S = nt + npairs;
  const int nsr = e.nr - 1;
  const int nsf = e.nrho - 1;
  // Density rows (a, b, c, d) of rho_t, stride nt.
  std::vector<double4> d64h(static_cast<size_t>(nsr) * nt);
  std::vector<float4> d32h(static_cast<size_t>(nsr) * nt);
  // Force rows (b, 2c, 3d, a) of every r-spline, stride S.
  std::vector<double4> r64(static_cast<size_t>(nsr) * S);
  std::vector<float4> r32(static_cast<size_t>(nsr) * S);
  auto f4 = [](const double4& v) {
    return make_float4(static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z),
                       static_cast<float>(v.w));
  };
  auto put = [&](int s, const double* coef) {
    for (int k = 0; k < nsr; ++k) {
      const double a = coef[k], b = coef[nsr + k], c = coef[2 * nsr + k], d = coef[3 * nsr + k];
      const double4 v = make_double4(b, 2.0 * c, 3.0 * d, a);
      r64[static_cast<size_t>(k) * S + s] = v;
      r32[static_cast<size_t>(k) * S + s] = f4(v);
      if (s < nt) {
        const double4 u = make_double4(a, b, c, d);
        d64h[static_cast<size_t>(k) * nt + s] = u;
        d32h[static_cast<size_t>(k) * nt + s] = f4(u);
      }
    }
  };
  for (int t = 0; t < nt; ++t) put(t, e.rhoc.data() + static_cast<size_t>(t) * 4 * nsr);
  for (int p = 0; p < npairs; ++p) put(nt + p, e.phic.data() + static_cast<size_t>(p) * 4 * nsr);
  std::vector<double4> f64(static_cast<size_t>(nsf) * nt);
  for (int t = 0; t < nt; ++t) {
    const double* c = e.Fc.data() + static_cast<size_t>(t) * 4 * nsf;
    for (int k = 0; k < nsf; ++k)
      f64[static_cast<size_t>(t) * nsf + k] =
          make_double4(c[k], c[nsf + k], c[2 * nsf + k], c[3 * nsf + k]);
  }
  rtab64.reserve(r64.size());
  rtab32.reserve(r32.size());
  dtab64.reserve(d64h.size());
  dtab32.reserve(d32h.size());
  ftab.reserve(f64.size());
  TDMD_CU(cudaMemcpyAsync(rtab64.data(), r64.data(), r64.size() * sizeof(double4),
                          cudaMemcpyHostToDevice, stream));
  TDMD_CU(cudaMemcpyAsync(rtab32.data(), r32.data(), r32.size() * sizeof(float4),
                          cudaMemcpyHostToDevice, stream));
  TDMD_CU(cudaMemcpyAsync(dtab64.data(), d64h.data(), d64h.size() * sizeof(double4),
                          cudaMemcpyHostToDevice, stream));
  TDMD_CU(cudaMemcpyAsync(dtab32.data(), d32h.data(), d32h.size() * sizeof(float4),
                          cudaMemcpyHostToDevice, stream));
  TDMD_CU(cudaMemcpyAsync(ftab.data(), f64.data(), f64.size() * sizeof(double4),
                          cudaMemcpyHostToDevice, stream));
  // The host vectors go out of scope: finish the copies first.
  TDMD_CU(cudaStreamSynchronize(stream));
  ntypes = nt;
  cutoff = e.cutoff;
  // type bits in the mixed gather records: ceil(log2(nt)) for 2..16 types
  int tbits = 0;
  if (nt > 1 && nt <= 16)
    while ((1 << tbits) < nt) ++tbits;
  d64 = EamDev<double>{dtab64.data(), rtab64.data(), ftab.data(), nt, S, e.nr, e.nrho, e.dr,
                       1.0 / e.dr, e.cutoff * e.cutoff, e.drho, e.dr, 0.0, 0};
  const float dr32 = static_cast<float>(e.dr);
  d32 = EamDev<float>{dtab32.data(), rtab32.data(), ftab.data(), nt, S, e.nr, e.nrho, dr32,
                      static_cast<float>(1.0 / e.dr), static_cast<float>(e.cutoff * e.cutoff),
                      e.drho, e.dr, static_cast<float>(e.dr - static_cast<double>(dr32)), tbits};
}

// --------------------------------------------------------------------------
// Fixed-order reduction of per-block energy/virial partials.
// --------------------------------------------------------------------------
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblk,
                                  double* __restrict__ energy, double* __restrict__ virial) {
  dependent_launch_prologue();
  __shared__ double red[32 * 7];
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const double* p = partials + static_cast<long long>(b) * kEvStride;
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] += p[k];
  }
  block_sum<7>(v, red);
  if (threadIdx.x == 0) {
    if (energy) energy[0] += v[0];
    if (virial) {
#pragma unroll
      for (int k = 0; k < 6; ++k) virial[k] += v[1 + k];
    }
  }
}

int force_blocks(long long n, int lpa) { return ceil_div(n * lpa, kForceThreads); }

int default_lpa(long long n) {
  // Enough groups to fill the GPU several times over; 8 lanes keep rows of
  // ~50-90 neighbors in a few coalesced sweeps.
  const long long want = 8ll * sm_count() * (2048 / 8);
  if (n * 8 >= want) return 8;
  if (n * 16 >= want) return 16;
  return 32;
}

}  // namespace tdmd_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace tdmd_b200;

struct tdmd_device_eam {
  EamDevTables tabs;
  DevArray<float> fp32;
  DevArray<double> fp64;
  // the reference's flat layout, for the ID-ordered energy mode
  RefEamTables ref;
};

namespace {

NbrView make_view(const int32_t* nbrs, const int32_t* offsets, const int32_t* counts) {
  return NbrView{nbrs, offsets, counts, 0};
}

// Scratch for per-block partials from the stream-ordered pool.
struct Partials {
  double* p = nullptr;
  cudaStream_t s;
  Partials(int nblk, cudaStream_t st) : s(st) {
    TDMD_CU(cudaMallocAsync(reinterpret_cast<void**>(&p),
                            sizeof(double) * kEvStride * (nblk > 0 ? nblk : 1), st));
  }
  ~Partials() {
    if (p) cudaFreeAsync(p, s);
  }
};

}  // namespace

extern "C" {

int32_t tdmd_eam_read_setfl(const char* path, tdmd_eam** out) {
  return guarded([&] {
    TDMD_REQUIRE(path && out, "null argument");
    auto* e = new tdmd_eam();
    try {
      read_setfl(path, *e);
    } catch (...) {
      delete e;
      throw;
    }
    *out = e;
  });
}

int32_t tdmd_eam_create(int32_t ntypes, int32_t nrho, double drho, int32_t nr, double dr,
                        double cutoff, const double* F, const double* rho, const double* rphi,
                        tdmd_eam** out) {
  return guarded([&] {
    TDMD_REQUIRE(out && F && rho && rphi, "null argument");
    TDMD_REQUIRE(ntypes >= 1 && ntypes <= 64, "ntypes out of range");
    TDMD_REQUIRE(nrho >= 2 && nr >= 2 && drho > 0 && dr > 0 && cutoff > 0, "bad grid");
    auto* e = new tdmd_eam();
    e->ntypes = ntypes;
    e->nrho = nrho;
    e->nr = nr;
    e->drho = drho;
    e->dr = dr;
    e->cutoff = cutoff;
    const int npairs = ntypes * (ntypes + 1) / 2;
    e->F.assign(F, F + static_cast<size_t>(ntypes) * nrho);
    e->rho.assign(rho, rho + static_cast<size_t>(ntypes) * nr);
    e->rphi.assign(rphi, rphi + static_cast<size_t>(npairs) * nr);
    e->elements.assign(static_cast<size_t>(ntypes), "X");
    eam_build_coeffs(*e);
    *out = e;
  });
}

int32_t tdmd_eam_create_sampled(int32_t ntypes, int32_t nrho, double drho, int32_t nr,
                                double dr, double cutoff, const double* F, const double* rho,
                                const double* phi, tdmd_eam** out) {
  return guarded([&] {
    TDMD_REQUIRE(out && F && rho && phi, "null argument");
    TDMD_REQUIRE(ntypes >= 1 && ntypes <= 64, "ntypes out of range");
    TDMD_REQUIRE(nrho >= 2 && nr >= 2 && drho > 0 && dr > 0 && cutoff > 0, "bad grid");
    auto* e = new tdmd_eam();
    e->ntypes = ntypes;
    e->nrho = nrho;
    e->nr = nr;
    e->drho = drho;
    e->dr = dr;
    e->cutoff = cutoff;
    const int npairs = ntypes * (ntypes + 1) / 2;
    const size_t np = static_cast<size_t>(npairs) * nr;
    e->F.assign(F, F + static_cast<size_t>(ntypes) * nrho);
    e->rho.assign(rho, rho + static_cast<size_t>(ntypes) * nr);
    e->phi.assign(phi, phi + np);
    // r*phi for writing the tables out as setfl
    e->rphi.resize(np);
    for (size_t i = 0; i < np; ++i) e->rphi[i] = phi[i] * (static_cast<double>(i % nr) * dr);
    e->elements.assign(static_cast<size_t>(ntypes), "X");
    eam_build_coeffs(*e);
    *out = e;
  });
}

int32_t tdmd_eam_destroy(tdmd_eam* eam) {
  delete eam;
  return TDMD_OK;
}

int32_t tdmd_eam_info(const tdmd_eam* e, int32_t* ntypes, int32_t* nrho, double* drho,
                      int32_t* nr, double* dr, double* cutoff) {
  return guarded([&] {
    TDMD_REQUIRE(e, "null handle");
    if (ntypes) *ntypes = e->ntypes;
    if (nrho) *nrho = e->nrho;
    if (drho) *drho = e->drho;
    if (nr) *nr = e->nr;
    if (dr) *dr = e->dr;
    if (cutoff) *cutoff = e->cutoff;
  });
}

int32_t tdmd_eam_coeffs(const tdmd_eam* e, int32_t kind, int32_t index, double* out) {
  return guarded([&] {
    TDMD_REQUIRE(e && out, "null argument");
    const int npairs = e->ntypes * (e->ntypes + 1) / 2;
    const int n = kind == 0 ? e->nrho : e->nr;
    const std::vector<double>& src = kind == 0 ? e->Fc : (kind == 1 ? e->rhoc : e->phic);
    const int limit = kind == 2 ? npairs : e->ntypes;
    TDMD_REQUIRE(kind >= 0 && kind <= 2 && index >= 0 && index < limit, "spline index");
    const size_t len = 4 * static_cast<size_t>(n - 1);
    std::copy(src.begin() + static_cast<long>(index * len),
              src.begin() + static_cast<long>((index + 1) * len), out);
  });
}

int32_t tdmd_morse_compute(const double* d_positions, void* d_forces, int32_t precision,
                           const int32_t* d_neighbors, const int32_t* d_offsets,
                           const int32_t* d_counts, int32_t natoms, const tdmd_box* box,
                           const tdmd_morse_params* params, double* d_energy, double* d_virial,
                           void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(box && params, "null box or params");
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_positions && d_forces && d_offsets && d_counts, "null device array");
    cudaStream_t s = as_stream(stream);
    const bool ev = d_energy || d_virial;
    if (ev && precision == TDMD_FP64 && deterministic_reduce()) {
      TDMD_REQUIRE(d_neighbors || natoms == 0, "null device array");
      morse_id_ordered(d_positions, static_cast<double*>(d_forces), d_neighbors, d_offsets,
                       d_counts, natoms, *box, *params, d_energy, d_virial, s);
      return;
    }
    const DevBox b = make_devbox(*box, 0.0);
    const NbrView nl = make_view(d_neighbors, d_offsets, d_counts);
    const int lpa = default_lpa(natoms);
    const int nblk = force_blocks(natoms, lpa);
    Partials part(ev ? nblk : 0, s);
    if (precision == TDMD_FP64) {
      GeoAoS64 g{d_positions, {b.L[0], b.L[1], b.L[2]}, {b.halfL[0], b.halfL[1], b.halfL[2]},
                 {b.periodic[0], b.periodic[1], b.periodic[2]}};
      MorseP<double> mp{params->d, params->alpha, params->r0, params->rc_sq, params->r0};
      launch_morse(g, nl, natoms, mp, static_cast<double*>(d_forces), ev, part.p, lpa, s);
    } else {
      TDMD_REQUIRE(precision == TDMD_MIXED, "unknown precision");
      const GeoAoS32 g = make_geo_aos32(d_positions, b);
      MorseP<float> mp{float(params->d), float(params->alpha), float(params->r0),
                       float(params->rc_sq), params->r0};
      launch_morse(g, nl, natoms, mp, static_cast<float*>(d_forces), ev, part.p, lpa, s);
    }
    if (ev) {
      launch(k_reduce_partials, 1, 256, 0, s, part.p, nblk, d_energy, d_virial);
      TDMD_LAUNCH_CHECK();
    }
  });
}

int32_t tdmd_morse_compute_zone(const double* d_positions, void* d_forces, int32_t precision,
                                const int32_t* d_neighbors, const int32_t* d_offsets,
                                const int32_t* d_counts, int32_t first_atom, int32_t atom_count,
                                const tdmd_box* box, const tdmd_morse_params* params,
                                double* d_energy, double* d_virial, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(box && params, "null box or params");
    TDMD_REQUIRE(first_atom >= 0 && atom_count >= 0, "first_atom and atom_count must be >= 0");
    if (atom_count == 0) return;
    TDMD_REQUIRE(d_positions && d_forces && d_offsets && d_counts, "null device array");
    cudaStream_t s = as_stream(stream);
    const bool ev = d_energy || d_virial;
    const DevBox b = make_devbox(*box, 0.0);
    // the range's rows: offsets and counts shifted, neighbor indices global
    const NbrView nl = make_view(d_neighbors, d_offsets + first_atom, d_counts + first_atom);
    const int lpa = default_lpa(atom_count);
    const int nblk = force_blocks(atom_count, lpa);
    Partials part(ev ? nblk : 0, s);
    if (precision == TDMD_FP64) {
      GeoAoS64 g{d_positions, {b.L[0], b.L[1], b.L[2]}, {b.halfL[0], b.halfL[1], b.halfL[2]},
                 {b.periodic[0], b.periodic[1], b.periodic[2]}};
      MorseP<double> mp{params->d, params->alpha, params->r0, params->rc_sq, params->r0};
      launch_morse_zone(g, first_atom, nl, atom_count, mp, static_cast<double*>(d_forces), ev,
                        part.p, lpa, s);
    } else {
      TDMD_REQUIRE(precision == TDMD_MIXED, "unknown precision");
      const GeoAoS32 g = make_geo_aos32(d_positions, b);
      MorseP<float> mp{float(params->d), float(params->alpha), float(params->r0),
                       float(params->rc_sq), params->r0};
      launch_morse_zone(g, first_atom, nl, atom_count, mp, static_cast<float*>(d_forces), ev,
                        part.p, lpa, s);
    }
    if (ev) {
      launch(k_reduce_partials, 1, 256, 0, s, part.p, nblk, d_energy, d_virial);
      TDMD_LAUNCH_CHECK();
    }
  });
}

int32_t tdmd_device_eam_create(const tdmd_eam* eam, tdmd_device_eam** out) {
  return guarded([&] {
    TDMD_REQUIRE(eam && out, "null argument");
    auto* de = new tdmd_device_eam();
    try {
      de->tabs.upload(*eam, nullptr);
      de->ref.upload(*eam);
    } catch (...) {
      delete de;
      throw;
    }
    *out = de;
  });
}

int32_t tdmd_device_eam_destroy(tdmd_device_eam* de) {
  delete de;
  return TDMD_OK;
}

int32_t tdmd_device_eam_compute(tdmd_device_eam* de, const double* d_positions, void* d_forces,
                                int32_t precision, const int32_t* d_types,
                                const int32_t* d_neighbors, const int32_t* d_offsets,
                                const int32_t* d_counts, int32_t natoms, const tdmd_box* box,
                                double* d_energy, double* d_virial, double* d_rho, double* d_fp,
                                void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(de && box, "null handle or box");
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_positions && d_forces && d_offsets && d_counts && d_types,
                 "null device array");
    cudaStream_t s = as_stream(stream);
    const bool ev = d_energy || d_virial;
    if (ev && precision == TDMD_FP64 && deterministic_reduce()) {
      eam_id_ordered(de->ref, d_positions, static_cast<double*>(d_forces), d_types, d_neighbors,
                     d_offsets, d_counts, natoms, *box, d_energy, d_virial, d_rho, d_fp, s);
      return;
    }
    const DevBox b = make_devbox(*box, 0.0);
    const NbrView nl = make_view(d_neighbors, d_offsets, d_counts);
    const int lpa = default_lpa(natoms);
    const int nblk = force_blocks(natoms, lpa);
    // Density records [0, nblk) and force records [nblk, 2*nblk).
    Partials part(ev ? 2 * nblk : 0, s);
    const int* types = de->tabs.ntypes > 1 ? d_types : nullptr;
    if (precision == TDMD_FP64) {
      de->fp64.reserve(static_cast<size_t>(natoms));
      GeoAoS64 g{d_positions, {b.L[0], b.L[1], b.L[2]}, {b.halfL[0], b.halfL[1], b.halfL[2]},
                 {b.periodic[0], b.periodic[1], b.periodic[2]}};
      launch_eam(g, nl, natoms, de->tabs.d64, types, de->fp64.data(), d_rho, d_fp,
                 static_cast<double*>(d_forces), ev, part.p, lpa, s);
    } else {
      TDMD_REQUIRE(precision == TDMD_MIXED, "unknown precision");
      de->fp32.reserve(static_cast<size_t>(natoms));
      const GeoAoS32 g = make_geo_aos32(d_positions, b);
      launch_eam(g, nl, natoms, de->tabs.d32, types, de->fp32.data(), d_rho, d_fp,
                 static_cast<float*>(d_forces), ev, part.p, lpa, s);
    }
    if (ev) {
      launch(k_reduce_partials, 1, 256, 0, s, part.p, 2 * nblk, d_energy, d_virial);
      TDMD_LAUNCH_CHECK();
    }
  });
}

}  // extern "C"
