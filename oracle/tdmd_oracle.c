/*
 * tdmd_oracle.c -- CPU restatement of TDMD's single-rank force + integration
 * path, used ONLY as test infrastructure (the checker).  Nothing in the
 * product library links, loads or calls this file; only tests/, the smoke
 * check in __graft_entry__.py and bench.py's CPU-baseline leg do.
 *
 * Every routine is a plain-C FP64 restatement of the reference algorithm and
 * cites the reference file:line it follows (paths relative to the
 * tdmd_Claude source tree).  Build: see oracle/Makefile
 * (gcc -O2 -ffp-contract=off, so no FMA contraction changes rounding).
 *
 * Parity pins (checked by tests/test_oracle.py):
 *   - two-atom analytic Morse and the run-0 LAMMPS force dumps of the
 *     reference's VerifyLab cases (golden fixtures under tests/golden/);
 *   - the reference CPU path itself, compiled from its sources into
 *     oracle/_ref/ (cell list, half list, Morse/EAM forces+energies,
 *     spline coefficients, NHC half-steps, VV trajectories).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MVV2E 1.0364269e-4      /* src/core/constants.hpp:28 */
#define ORC_KB 8.617333262e-5       /* src/core/constants.hpp:15 */

typedef struct {
  double lo[3];
  double hi[3];
  int32_t periodic[3];
} orc_box;

/* ------------------------------------------------------------------------ */
/* Periodic helpers: minimum_image / wrap_position, src/core/math.hpp:78-131 */
/* ------------------------------------------------------------------------ */
static void min_image(double d[3], const orc_box* b) {
  for (int a = 0; a < 3; ++a) {
    if (!b->periodic[a]) continue;
    const double bs = b->hi[a] - b->lo[a];
    if (d[a] > 0.5 * bs)
      d[a] -= bs;
    else if (d[a] < -0.5 * bs)
      d[a] += bs;
  }
}

static double len_sq(const double d[3]) { return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]; }

/* ------------------------------------------------------------------------ */
/* Cell list: CellList::build / cell_of / cell_index,                        */
/* src/domain/cell_list.cpp:13-58, src/domain/cell_list.hpp:47-72            */
/* ------------------------------------------------------------------------ */
void orc_cell_grid(const orc_box* b, double r_list, int32_t nc[3], double cs[3]) {
  for (int a = 0; a < 3; ++a) {
    const double L = b->hi[a] - b->lo[a];
    int32_t n = (int32_t)floor(L / r_list);
    nc[a] = n < 3 ? 3 : n;
    cs[a] = L / nc[a];
  }
}

static int32_t cell_of(const double* p, const orc_box* b, const int32_t nc[3], const double cs[3]) {
  int32_t ix = (int32_t)((p[0] - b->lo[0]) / cs[0]);
  int32_t iy = (int32_t)((p[1] - b->lo[1]) / cs[1]);
  int32_t iz = (int32_t)((p[2] - b->lo[2]) / cs[2]);
  if (ix >= nc[0]) ix = nc[0] - 1;
  if (iy >= nc[1]) iy = nc[1] - 1;
  if (iz >= nc[2]) iz = nc[2] - 1;
  if (ix < 0) ix = 0;
  if (iy < 0) iy = 0;
  if (iz < 0) iz = 0;
  return iz * nc[0] * nc[1] + iy * nc[0] + ix;
}

static int32_t cell_index(int32_t ix, int32_t iy, int32_t iz, const int32_t nc[3]) {
  if (ix < 0) ix += nc[0]; else if (ix >= nc[0]) ix -= nc[0];
  if (iy < 0) iy += nc[1]; else if (iy >= nc[1]) iy -= nc[1];
  if (iz < 0) iz += nc[2]; else if (iz >= nc[2]) iz -= nc[2];
  return iz * nc[0] * nc[1] + iy * nc[0] + ix;
}

/* Counting sort, atoms ID-ascending within a cell.  counts/offsets have
 * nc[0]*nc[1]*nc[2] entries, atoms and atom_cell have n entries. */
void orc_cell_list_build(const double* pos, int64_t n, const orc_box* b, double r_list,
                         int32_t nc[3], int32_t* counts, int32_t* offsets, int32_t* atoms,
                         int32_t* atom_cell) {
  double cs[3];
  orc_cell_grid(b, r_list, nc, cs);
  const int32_t ncell = nc[0] * nc[1] * nc[2];
  memset(counts, 0, sizeof(int32_t) * (size_t)ncell);
  for (int64_t i = 0; i < n; ++i) {
    const int32_t c = cell_of(pos + 3 * i, b, nc, cs);
    atom_cell[i] = c;
    ++counts[c];
  }
  offsets[0] = 0;
  for (int32_t c = 1; c < ncell; ++c) offsets[c] = offsets[c - 1] + counts[c - 1];
  int32_t* placed = (int32_t*)calloc((size_t)ncell, sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) {
    const int32_t c = atom_cell[i];
    atoms[offsets[c] + placed[c]++] = (int32_t)i;
  }
  free(placed);
}

/* ------------------------------------------------------------------------ */
/* Neighbor lists.                                                           */
/* half=1: NeighborList::build half list (j > i), neighbor_list.cpp:14-89.   */
/* half=0: full list in the order of DeviceNeighborList's build kernel with  */
/*   the ID-ordered cell scatter (device_neighbor_list.cu:26-139,            */
/*   device_cell_list.cu:114-136): stencil dz,dy,dx in -1..1, atoms of each  */
/*   cell ID-ascending, j != i, r^2 < (rc+skin)^2 on the FP64 min-image delta.*/
/* Output: counts[n], offsets[n] (dense exclusive scan), nbrs[<=cap].        */
/* Returns the total number of entries (write skipped past cap).             */
/* ------------------------------------------------------------------------ */
int64_t orc_neighbor_list(const double* pos, int64_t n, const orc_box* b, double r_cut,
                          double r_skin, int32_t half, int32_t* counts, int32_t* offsets,
                          int32_t* nbrs, int64_t cap) {
  const double r_list = r_cut + r_skin;
  const double r_list_sq = r_list * r_list;
  int32_t nc[3];
  double cs[3];
  orc_cell_grid(b, r_list, nc, cs);
  const int32_t ncell = nc[0] * nc[1] * nc[2];
  int32_t* ccount = (int32_t*)malloc(sizeof(int32_t) * (size_t)ncell);
  int32_t* coff = (int32_t*)malloc(sizeof(int32_t) * (size_t)ncell);
  int32_t* catoms = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  int32_t* acell = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  orc_cell_list_build(pos, n, b, r_list, nc, ccount, coff, catoms, acell);
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double* pi = pos + 3 * i;
    const int32_t ci = acell[i];
    const int32_t iz = ci / (nc[0] * nc[1]);
    const int32_t iy = (ci - iz * nc[0] * nc[1]) / nc[0];
    const int32_t ix = ci - iz * nc[0] * nc[1] - iy * nc[0];
    offsets[i] = (int32_t)total;
    int32_t cnt = 0;
    for (int32_t dz = -1; dz <= 1; ++dz)
      for (int32_t dy = -1; dy <= 1; ++dy)
        for (int32_t dx = -1; dx <= 1; ++dx) {
          const int32_t c = cell_index(ix + dx, iy + dy, iz + dz, nc);
          for (int32_t k = 0; k < ccount[c]; ++k) {
            const int32_t j = catoms[coff[c] + k];
            if (half ? (j <= (int32_t)i) : (j == (int32_t)i)) continue;
            double d[3] = {pos[3 * j] - pi[0], pos[3 * j + 1] - pi[1], pos[3 * j + 2] - pi[2]};
            min_image(d, b);
            if (len_sq(d) < r_list_sq) {
              if (total + cnt < cap) nbrs[total + cnt] = j;
              ++cnt;
            }
          }
        }
    counts[i] = cnt;
    total += cnt;
  }
  free(ccount);
  free(coff);
  free(catoms);
  free(acell);
  return total;
}

/* Skin check NeighborList::needs_rebuild, neighbor_list.cpp:91-100 (raw
 * displacement, no minimum image). */
int32_t orc_needs_rebuild(const double* pos, const double* pos_at_build, int64_t n, double r_skin) {
  const double half_skin_sq = 0.25 * r_skin * r_skin;
  for (int64_t i = 0; i < n; ++i) {
    double d[3] = {pos[3 * i] - pos_at_build[3 * i], pos[3 * i + 1] - pos_at_build[3 * i + 1],
                   pos[3 * i + 2] - pos_at_build[3 * i + 2]};
    if (len_sq(d) > half_skin_sq) return 1;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Morse: MorsePair::compute, src/potentials/morse.hpp:37-55;               */
/* compute_pair_forces (half list, Newton 3), force_compute.cpp:10-56.       */
/* Virial (no reference symbol): W_ab = sum over pairs of d_a * fpair * d_b  */
/* with d = r_i - r_j (LAMMPS pair-virial convention); order xx,yy,zz,xy,xz,yz.*/
/* ------------------------------------------------------------------------ */
static void morse_pair(double r2, double D, double alpha, double r0, double rc_sq, double* e,
                       double* fpair) {
  if (r2 >= rc_sq) {
    *e = 0.0;
    *fpair = 0.0;
    return;
  }
  const double r = sqrt(r2);
  const double dr = r - r0;
  const double ex = exp(-alpha * dr);
  const double ome = 1.0 - ex;
  *e = D * (ome * ome - 1.0);
  const double dudr = 2.0 * D * alpha * ome * ex;
  *fpair = -dudr / r;
}

double orc_morse_forces(const double* pos, int64_t n, const orc_box* b, double D, double alpha,
                        double r0, double rc, const int32_t* counts, const int32_t* offsets,
                        const int32_t* nbrs, double* forces, double* virial6) {
  const double rc_sq = rc * rc;
  double pe = 0.0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  memset(forces, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const double* pi = pos + 3 * i;
    for (int32_t k = 0; k < counts[i]; ++k) {
      const int32_t j = nbrs[offsets[i] + k];
      double d[3] = {pi[0] - pos[3 * j], pi[1] - pos[3 * j + 1], pi[2] - pos[3 * j + 2]};
      min_image(d, b);
      double e, fp;
      morse_pair(len_sq(d), D, alpha, r0, rc_sq, &e, &fp);
      pe += e;
      for (int a = 0; a < 3; ++a) {
        forces[3 * i + a] += fp * d[a];
        forces[3 * (int64_t)j + a] -= fp * d[a];
      }
      w[0] += d[0] * d[0] * fp;
      w[1] += d[1] * d[1] * fp;
      w[2] += d[2] * d[2] * fp;
      w[3] += d[0] * d[1] * fp;
      w[4] += d[0] * d[2] * fp;
      w[5] += d[1] * d[2] * fp;
    }
  }
  if (virial6) memcpy(virial6, w, sizeof(w));
  return pe;
}

/* ------------------------------------------------------------------------ */
/* Splines: SplineTable::build_splines / eval / eval_deriv,                  */
/* src/potentials/eam_alloy.cpp:19-72 (finite-difference cubic Hermite,      */
/* interval index clamped to [0, n-2]).  Coefficients packed a|b|c|d, each   */
/* n-1 long, into coef[4*(n-1)].                                             */
/* ------------------------------------------------------------------------ */
void orc_spline_build(const double* values, int32_t n, double dr, double* coef) {
  if (n < 2) return;
  const int32_t ns = n - 1;
  double* a = coef;
  double* bb = coef + ns;
  double* c = coef + 2 * ns;
  double* d = coef + 3 * ns;
  for (int32_t i = 0; i < ns; ++i) {
    a[i] = values[i];
    const double sl = (i > 0) ? (values[i] - values[i - 1]) / dr : 0.0;
    const double sr = (values[i + 1] - values[i]) / dr;
    const double sn = (i + 2 < n) ? (values[i + 2] - values[i + 1]) / dr : sr;
    double m0 = (sl + sr) * 0.5;
    double m1 = (sr + sn) * 0.5;
    if (i == 0) m0 = sr;
    if (i == n - 2) m1 = sr;
    bb[i] = m0;
    c[i] = (3.0 * sr - 2.0 * m0 - m1) / dr;
    d[i] = (m0 + m1 - 2.0 * sr) / (dr * dr);
  }
}

double orc_spline_eval(const double* coef, int32_t n, double dr, double rmin, double r) {
  if (n < 2) return 0.0;
  const int32_t ns = n - 1;
  const double x = (r - rmin) / dr;
  int32_t idx = (int32_t)x;
  if (idx < 0) idx = 0;
  if (idx >= n - 1) idx = n - 2;
  const double dx = r - (rmin + (double)idx * dr);
  return coef[idx] + dx * (coef[ns + idx] + dx * (coef[2 * ns + idx] + dx * coef[3 * ns + idx]));
}

double orc_spline_deriv(const double* coef, int32_t n, double dr, double rmin, double r) {
  if (n < 2) return 0.0;
  const int32_t ns = n - 1;
  const double x = (r - rmin) / dr;
  int32_t idx = (int32_t)x;
  if (idx < 0) idx = 0;
  if (idx >= n - 1) idx = n - 2;
  const double dx = r - (rmin + (double)idx * dr);
  return coef[ns + idx] + dx * (2.0 * coef[2 * ns + idx] + dx * 3.0 * coef[3 * ns + idx]);
}

/* ------------------------------------------------------------------------ */
/* EAM/alloy tables.  Layout mirrors EamAlloy (eam_alloy.hpp:75-92):         */
/* F[t] (nrho knots, drho), rho[t] (nr knots, dr), phi[p] (nr knots) with    */
/* p = phi_index(ti,tj) = ti*nt - ti*(ti+1)/2 + tj for ti <= tj.  phi values */
/* are r*phi(r)/r with phi[0] = 0 (eam_alloy.cpp:176-188).                   */
/* ------------------------------------------------------------------------ */
typedef struct {
  int32_t ntypes, nrho, nr;
  double drho, dr, cutoff;
  double* F_coef;   /* ntypes * 4*(nrho-1) */
  double* rho_coef; /* ntypes * 4*(nr-1)   */
  double* phi_coef; /* npairs * 4*(nr-1)   */
} orc_eam;

static int32_t phi_index(int32_t ti, int32_t tj, int32_t nt) {
  if (ti > tj) {
    int32_t t = ti;
    ti = tj;
    tj = t;
  }
  return ti * nt - ti * (ti + 1) / 2 + tj;
}

/* Build an orc_eam from raw setfl arrays: F_vals[ntypes*nrho],
 * rho_vals[ntypes*nr], rphi_vals[npairs*nr] (r*phi, setfl order). */
orc_eam* orc_eam_create(int32_t ntypes, int32_t nrho, double drho, int32_t nr, double dr,
                        double cutoff, const double* F_vals, const double* rho_vals,
                        const double* rphi_vals) {
  orc_eam* e = (orc_eam*)calloc(1, sizeof(orc_eam));
  const int32_t npairs = ntypes * (ntypes + 1) / 2;
  e->ntypes = ntypes;
  e->nrho = nrho;
  e->nr = nr;
  e->drho = drho;
  e->dr = dr;
  e->cutoff = cutoff;
  e->F_coef = (double*)calloc((size_t)ntypes * 4 * (size_t)(nrho - 1), sizeof(double));
  e->rho_coef = (double*)calloc((size_t)ntypes * 4 * (size_t)(nr - 1), sizeof(double));
  e->phi_coef = (double*)calloc((size_t)npairs * 4 * (size_t)(nr - 1), sizeof(double));
  for (int32_t t = 0; t < ntypes; ++t) {
    orc_spline_build(F_vals + (size_t)t * nrho, nrho, drho, e->F_coef + (size_t)t * 4 * (nrho - 1));
    orc_spline_build(rho_vals + (size_t)t * nr, nr, dr, e->rho_coef + (size_t)t * 4 * (nr - 1));
  }
  double* phi = (double*)malloc(sizeof(double) * (size_t)nr);
  for (int32_t p = 0; p < npairs; ++p) {
    const double* rp = rphi_vals + (size_t)p * nr;
    phi[0] = 0.0;
    for (int32_t k = 1; k < nr; ++k) phi[k] = rp[k] / ((double)k * dr);
    orc_spline_build(phi, nr, dr, e->phi_coef + (size_t)p * 4 * (nr - 1));
  }
  free(phi);
  return e;
}

void orc_eam_destroy(orc_eam* e) {
  if (!e) return;
  free(e->F_coef);
  free(e->rho_coef);
  free(e->phi_coef);
  free(e);
}

/* Copies one spline's packed coefficients out (kind 0=F,1=rho,2=phi). */
int32_t orc_eam_coeffs(const orc_eam* e, int32_t kind, int32_t idx, double* out) {
  const int32_t n = kind == 0 ? e->nrho : e->nr;
  const double* src = kind == 0 ? e->F_coef : (kind == 1 ? e->rho_coef : e->phi_coef);
  memcpy(out, src + (size_t)idx * 4 * (n - 1), sizeof(double) * 4 * (size_t)(n - 1));
  return 4 * (n - 1);
}

/* EamAlloy::compute_forces (3-pass on the half list), eam_alloy.cpp:196-295.
 * types are 1-based.  Optional outputs: rho[n], fp[n], virial6, and the
 * split of the energy into embedding / pair parts. */
double orc_eam_forces(const orc_eam* e, const double* pos, const int32_t* types, int64_t n,
                      const orc_box* b, const int32_t* counts, const int32_t* offsets,
                      const int32_t* nbrs, double* forces, double* rho_out, double* fp_out,
                      double* virial6, double* e_embed_out, double* e_pair_out) {
  const double rc_sq = e->cutoff * e->cutoff;
  const int32_t nt = e->ntypes;
  const int32_t nsr = 4 * (e->nr - 1);
  const int32_t nsf = 4 * (e->nrho - 1);
  double* rho = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  double* fp = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  double w[6] = {0, 0, 0, 0, 0, 0};
  memset(forces, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const double* pi = pos + 3 * i;
    const int32_t ti = types[i] - 1;
    for (int32_t k = 0; k < counts[i]; ++k) {
      const int32_t j = nbrs[offsets[i] + k];
      double d[3] = {pi[0] - pos[3 * j], pi[1] - pos[3 * j + 1], pi[2] - pos[3 * j + 2]};
      min_image(d, b);
      const double r2 = len_sq(d);
      if (r2 >= rc_sq) continue;
      const double r = sqrt(r2);
      const int32_t tj = types[j] - 1;
      rho[i] += orc_spline_eval(e->rho_coef + (size_t)tj * nsr, e->nr, e->dr, 0.0, r);
      rho[j] += orc_spline_eval(e->rho_coef + (size_t)ti * nsr, e->nr, e->dr, 0.0, r);
    }
  }
  double e_embed = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t ti = types[i] - 1;
    e_embed += orc_spline_eval(e->F_coef + (size_t)ti * nsf, e->nrho, e->drho, 0.0, rho[i]);
    fp[i] = orc_spline_deriv(e->F_coef + (size_t)ti * nsf, e->nrho, e->drho, 0.0, rho[i]);
  }
  double e_pair = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double* pi = pos + 3 * i;
    const int32_t ti = types[i] - 1;
    for (int32_t k = 0; k < counts[i]; ++k) {
      const int32_t j = nbrs[offsets[i] + k];
      double d[3] = {pi[0] - pos[3 * j], pi[1] - pos[3 * j + 1], pi[2] - pos[3 * j + 2]};
      min_image(d, b);
      const double r2 = len_sq(d);
      if (r2 >= rc_sq) continue;
      const double r = sqrt(r2);
      const int32_t tj = types[j] - 1;
      const double* phc = e->phi_coef + (size_t)phi_index(ti, tj, nt) * nsr;
      e_pair += orc_spline_eval(phc, e->nr, e->dr, 0.0, r);
      const double dphi = orc_spline_deriv(phc, e->nr, e->dr, 0.0, r);
      const double drj = orc_spline_deriv(e->rho_coef + (size_t)tj * nsr, e->nr, e->dr, 0.0, r);
      const double dri = orc_spline_deriv(e->rho_coef + (size_t)ti * nsr, e->nr, e->dr, 0.0, r);
      const double fpair = -(dphi + fp[i] * drj + fp[j] * dri) / r;
      for (int a = 0; a < 3; ++a) {
        forces[3 * i + a] += fpair * d[a];
        forces[3 * (int64_t)j + a] -= fpair * d[a];
      }
      w[0] += d[0] * d[0] * fpair;
      w[1] += d[1] * d[1] * fpair;
      w[2] += d[2] * d[2] * fpair;
      w[3] += d[0] * d[1] * fpair;
      w[4] += d[0] * d[2] * fpair;
      w[5] += d[1] * d[2] * fpair;
    }
  }
  if (rho_out) memcpy(rho_out, rho, sizeof(double) * (size_t)n);
  if (fp_out) memcpy(fp_out, fp, sizeof(double) * (size_t)n);
  if (virial6) memcpy(virial6, w, sizeof(w));
  if (e_embed_out) *e_embed_out = e_embed;
  if (e_pair_out) *e_pair_out = e_pair;
  free(rho);
  free(fp);
  return e_embed + e_pair;
}

/* ------------------------------------------------------------------------ */
/* Velocity Verlet.                                                          */
/* CPU: VelocityVerlet::half_kick / drift (floor wrap),                       */
/*   src/integrator/velocity_verlet.cpp:11-48.                                */
/* GPU: fused_kick_drift_kernel<kFullKick> and half_kick_kernel              */
/*   (single-image wrap), src/integrator/device_velocity_verlet.cu:14-130.    */
/* masses are indexed by the 1-based type directly (size ntypes+1).          */
/* ------------------------------------------------------------------------ */
void orc_half_kick(double* vel, const double* forces, const int32_t* types, const double* masses,
                   int64_t n, double dt) {
  const double half_dt = dt * 0.5;
  for (int64_t i = 0; i < n; ++i) {
    const double factor = half_dt / (masses[types[i]] * ORC_MVV2E);
    for (int a = 0; a < 3; ++a) vel[3 * i + a] += factor * forces[3 * i + a];
  }
}

void orc_drift(double* pos, const double* vel, int64_t n, double dt, const orc_box* b) {
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      double p = pos[3 * i + a] + dt * vel[3 * i + a];
      if (b->periodic[a]) {
        const double bs = b->hi[a] - b->lo[a];
        double rel = p - b->lo[a];
        rel -= floor(rel / bs) * bs;
        p = b->lo[a] + rel;
      }
      pos[3 * i + a] = p;
    }
}

/* full_kick != 0: kick with dt (OPT-FUSE-1c), else dt/2; then drift + single
 * image wrap. */
void orc_fused_kick_drift(double* vel, double* pos, const double* forces, const int32_t* types,
                          const double* masses, int64_t n, double dt, const orc_box* b,
                          int32_t full_kick) {
  const double kick_dt = full_kick ? dt : 0.5 * dt;
  for (int64_t i = 0; i < n; ++i) {
    const double factor = kick_dt / (masses[types[i]] * ORC_MVV2E);
    for (int a = 0; a < 3; ++a) {
      const double v = vel[3 * i + a] + factor * forces[3 * i + a];
      double p = pos[3 * i + a] + dt * v;
      if (b->periodic[a]) {
        const double bs = b->hi[a] - b->lo[a];
        if (p < b->lo[a])
          p += bs;
        else if (p >= b->lo[a] + bs)
          p -= bs;
      }
      vel[3 * i + a] = v;
      pos[3 * i + a] = p;
    }
  }
}

/* Kinetic energy, tdmd_main.cpp:97-108 / ke_reduce_kernel (FP64). */
double orc_kinetic_energy(const double* vel, const int32_t* types, const double* masses, int64_t n) {
  double ke = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double* v = vel + 3 * i;
    ke += 0.5 * masses[types[i]] * ORC_MVV2E * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  return ke;
}

/* device_compute_vmax, device_nose_hoover.cu:129-183: sqrt(max |v|^2). */
double orc_vmax(const double* vel, int64_t n) {
  double m = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double* v = vel + 3 * i;
    const double s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (s > m) m = s;
  }
  return sqrt(m);
}

/* ------------------------------------------------------------------------ */
/* Nose-Hoover chain: NoseHooverChain ctor + half_step,                      */
/* src/integrator/device_nose_hoover.cu:187-289.  state = [eta(M) eta_v(M)   */
/* eta_m(M)], M = chain length.                                              */
/* ------------------------------------------------------------------------ */
void orc_nhc_init(double* state, int32_t M, double t_target, double t_period, int32_t n_dof) {
  double* eta = state;
  double* eta_v = state + M;
  double* eta_m = state + 2 * M;
  const double kt = ORC_KB * t_target;
  const double tau2 = t_period * t_period;
  for (int32_t k = 0; k < M; ++k) {
    eta[k] = 0.0;
    eta_v[k] = 0.0;
    eta_m[k] = (k == 0) ? (double)n_dof * kt * tau2 : kt * tau2;
  }
}

double orc_nhc_half_step(double* state, int32_t M, double t_target, double t_period,
                         int32_t n_dof, double dt, double ke) {
  if (M == 0) return 1.0;
  double* eta = state;
  double* eta_v = state + M;
  double* eta_m = state + 2 * M;
  const double half_dt = 0.5 * dt;
  const double ke_target = 0.5 * (double)n_dof * ORC_KB * t_target;
  const double kt = ORC_KB * t_target;
  const double tau2 = t_period * t_period;
  eta_m[0] = (double)n_dof * kt * tau2;
  for (int32_t k = 1; k < M; ++k) eta_m[k] = kt * tau2;
  const int32_t last = M - 1;
  if (M > 1) {
    const double g = (eta_m[last - 1] * eta_v[last - 1] * eta_v[last - 1] - ORC_KB * t_target) /
                     eta_m[last];
    eta_v[last] += g * half_dt;
  }
  for (int32_t k = M - 2; k >= 1; --k) {
    const double ef = exp(-eta_v[k + 1] * half_dt / 4.0);
    eta_v[k] *= ef;
    const double g = (eta_m[k - 1] * eta_v[k - 1] * eta_v[k - 1] - ORC_KB * t_target) / eta_m[k];
    eta_v[k] += g * half_dt;
    eta_v[k] *= ef;
  }
  {
    const double ef = (M > 1) ? exp(-eta_v[1] * half_dt / 4.0) : 1.0;
    eta_v[0] *= ef;
    const double g0 = (2.0 * ke - 2.0 * ke_target) / eta_m[0];
    eta_v[0] += g0 * half_dt;
    eta_v[0] *= ef;
  }
  const double scale = exp(-eta_v[0] * half_dt);
  for (int32_t k = 0; k < M; ++k) eta[k] += eta_v[k] * half_dt;
  return scale;
}

/* ------------------------------------------------------------------------ */
/* MD driver restating FastPipelineScheduler::run_until, fast_pipeline_      */
/* scheduler.cu:87-233: initial list+forces, per step fused kick-drift (half */
/* on the first step of a window, full afterwards), rebuild every            */
/* rebuild_every steps (maybe_rebuild_nlist :225-232), force; one closing    */
/* half-kick per window.  Forces come from the CPU half-list path (the       */
/* reference's FP64 oracle).                                                 */
/*                                                                           */
/* With nhc_M > 0 the step follows PipelineScheduler's NVT order             */
/* (pipeline_scheduler.cu:246-276): KE -> half_step -> scale, plain VV step  */
/* (half kick, drift, rebuild?, force, half kick), KE -> half_step -> scale. */
/* adaptive != 0 sets dt = clamp(c2*rc/vmax, dt_min, dt_max) at each step    */
/* start (pipeline_scheduler.cu:235-244).                                     */
/*                                                                           */
/* windows[nwin] are the successive run_until targets.  pe_out/ke_out (if    */
/* non-null) get the PE and KE after every step (length = last target).     */
/* ------------------------------------------------------------------------ */
typedef struct {
  int32_t kind; /* 0 = Morse, 1 = EAM */
  double D, alpha, r0, rc;
  const orc_eam* eam;
} orc_potential;

static double compute_forces(const orc_potential* p, const double* pos, const int32_t* types,
                             int64_t n, const orc_box* b, const int32_t* counts,
                             const int32_t* offsets, const int32_t* nbrs, double* forces) {
  if (p->kind == 0)
    return orc_morse_forces(pos, n, b, p->D, p->alpha, p->r0, p->rc, counts, offsets, nbrs,
                            forces, NULL);
  return orc_eam_forces(p->eam, pos, types, n, b, counts, offsets, nbrs, forces, NULL, NULL, NULL,
                        NULL, NULL);
}

typedef struct {
  int32_t* counts;
  int32_t* offsets;
  int32_t* nbrs;
  int64_t cap;
} orc_list;

static void list_build(orc_list* L, const double* pos, int64_t n, const orc_box* b, double rc,
                       double skin) {
  for (;;) {
    int64_t tot = orc_neighbor_list(pos, n, b, rc, skin, 1, L->counts, L->offsets, L->nbrs, L->cap);
    if (tot <= L->cap) return;
    free(L->nbrs);
    L->cap = tot + tot / 4 + 16;
    L->nbrs = (int32_t*)malloc(sizeof(int32_t) * (size_t)L->cap);
  }
}

int32_t orc_md_run(const orc_potential* pot, double* pos, double* vel, double* forces,
                   const int32_t* types, const double* masses, int64_t n, const orc_box* b,
                   double dt, double skin, int32_t rebuild_every, const int32_t* windows,
                   int32_t nwin, int32_t nhc_M, double t_target, double t_period,
                   int32_t adaptive, double dt_min, double dt_max, double c2, double* pe_out,
                   double* ke_out, double* dt_out) {
  const double rc = pot->kind == 0 ? pot->rc : pot->eam->cutoff;
  orc_list L;
  L.counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  L.offsets = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  L.cap = 64 * (n > 0 ? n : 1);
  L.nbrs = (int32_t*)malloc(sizeof(int32_t) * (size_t)L.cap);
  double* nhc = NULL;
  const int32_t n_dof = 3 * (int32_t)n - 3;
  if (nhc_M > 0) {
    nhc = (double*)malloc(sizeof(double) * 3 * (size_t)nhc_M);
    orc_nhc_init(nhc, nhc_M, t_target, t_period, n_dof);
  }
  list_build(&L, pos, n, b, rc, skin);
  int32_t steps_since = 0;
  double pe = compute_forces(pot, pos, types, n, b, L.counts, L.offsets, L.nbrs, forces);
  int32_t step = 0;
  for (int32_t w = 0; w < nwin; ++w) {
    int32_t first = 1;
    const int32_t target = windows[w];
    if (step >= target) continue;
    while (step < target) {
      double cur_dt = dt;
      if (adaptive) {
        const double vmax = orc_vmax(vel, n);
        if (vmax > 0) {
          cur_dt = c2 * rc / vmax;
          if (cur_dt > dt_max) cur_dt = dt_max;
          if (cur_dt < dt_min) cur_dt = dt_min;
        }
      }
      if (nhc_M > 0 || adaptive) {
        if (nhc_M > 0) {
          const double ke = orc_kinetic_energy(vel, types, masses, n);
          const double s = orc_nhc_half_step(nhc, nhc_M, t_target, t_period, n_dof, cur_dt, ke);
          for (int64_t i = 0; i < 3 * n; ++i) vel[i] *= s;
        }
        orc_fused_kick_drift(vel, pos, forces, types, masses, n, cur_dt, b, 0);
      } else {
        orc_fused_kick_drift(vel, pos, forces, types, masses, n, cur_dt, b, first ? 0 : 1);
      }
      if (steps_since >= rebuild_every) {
        list_build(&L, pos, n, b, rc, skin);
        steps_since = 0;
      }
      pe = compute_forces(pot, pos, types, n, b, L.counts, L.offsets, L.nbrs, forces);
      if (nhc_M > 0 || adaptive) {
        orc_half_kick(vel, forces, types, masses, n, cur_dt);
        if (nhc_M > 0) {
          const double ke = orc_kinetic_energy(vel, types, masses, n);
          const double s = orc_nhc_half_step(nhc, nhc_M, t_target, t_period, n_dof, cur_dt, ke);
          for (int64_t i = 0; i < 3 * n; ++i) vel[i] *= s;
        }
      }
      ++step;
      ++steps_since;
      first = 0;
      if (dt_out) dt_out[step - 1] = cur_dt;
      if (pe_out) pe_out[step - 1] = pe;
      if (ke_out) {
        if (nhc_M > 0 || adaptive) {
          ke_out[step - 1] = orc_kinetic_energy(vel, types, masses, n);
        } else {
          /* velocities are half-advanced inside a window; report the KE at
           * integer time by applying the closing half kick to a copy. */
          double* vtmp = (double*)malloc(sizeof(double) * 3 * (size_t)n);
          memcpy(vtmp, vel, sizeof(double) * 3 * (size_t)n);
          orc_half_kick(vtmp, forces, types, masses, n, cur_dt);
          ke_out[step - 1] = orc_kinetic_energy(vtmp, types, masses, n);
          free(vtmp);
        }
      }
    }
    if (!(nhc_M > 0 || adaptive)) orc_half_kick(vel, forces, types, masses, n, dt);
  }
  free(L.counts);
  free(L.offsets);
  free(L.nbrs);
  free(nhc);
  return step;
}

/* ------------------------------------------------------------------------ */
/* Force matching (no reference counterpart: the reference computes no      */
/* gradients).  Loss over nsnap snapshots of n atoms each (same box):        */
/*   L = 1/(3 nsnap n) * sum_s sum_i |F_i(theta) - T_i|^2                    */
/* with F from the half-list Morse / EAM forces above (r_list = rc).         */
/* Gradient by the adjoint of the force expressions, in FP64:                */
/*   G_i = dL/dF_i = 2 (F_i - T_i) / (3 nsnap n),                            */
/*   q_ij = G_i . (r_i - r_j) / r_ij  (ordered pair).                        */
/* ------------------------------------------------------------------------ */
static void fm_list(const double* pos, int64_t n, const orc_box* b, double rc, int32_t* counts,
                    int32_t* offsets, int32_t** nbrs, int64_t* cap) {
  for (;;) {
    const int64_t tot = orc_neighbor_list(pos, n, b, rc, 0.0, 1, counts, offsets, *nbrs, *cap);
    if (tot <= *cap) return;
    free(*nbrs);
    *cap = tot + tot / 4 + 16;
    *nbrs = (int32_t*)malloc(sizeof(int32_t) * (size_t)*cap);
  }
}

/* Morse: fpair(r) = -2 D a (1 - e) e / r, e = exp(-a (r - r0)), F_i = sum
 * fpair d_ij, so dL/dtheta = sum over ordered pairs of q_ij r_ij dfpair/dtheta
 * with
 *   dfpair/dD  = fpair / D,
 *   dfpair/da  = -2 D [ (1 - e) e - a (1 - 2e)(r - r0) e ] / r,
 *   dfpair/dr0 = -2 D a^2 (1 - 2e) e / r.
 * grad3 = {dL/dD, dL/dalpha, dL/dr0}. */
double orc_morse_fm_loss_grad(int32_t nsnap, int64_t n, const double* pos, const orc_box* b,
                              double D, double alpha, double r0, double rc,
                              const double* target, double* grad3) {
  int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  int32_t* offsets = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  int64_t cap = 64 * (n > 0 ? n : 1);
  int32_t* nbrs = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
  double* f = (double*)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  double* G = (double*)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  const double c = 1.0 / (3.0 * (double)nsnap * (double)n);
  const double rc_sq = rc * rc;
  double loss = 0.0;
  double g[3] = {0.0, 0.0, 0.0};
  for (int32_t s = 0; s < nsnap; ++s) {
    const double* p = pos + (size_t)s * 3 * (size_t)n;
    const double* t = target + (size_t)s * 3 * (size_t)n;
    fm_list(p, n, b, rc, counts, offsets, &nbrs, &cap);
    orc_morse_forces(p, n, b, D, alpha, r0, rc, counts, offsets, nbrs, f, NULL);
    for (int64_t k = 0; k < 3 * n; ++k) {
      const double e = f[k] - t[k];
      loss += c * e * e;
      G[k] = 2.0 * c * e;
    }
    for (int64_t i = 0; i < n; ++i) {
      for (int32_t k = 0; k < counts[i]; ++k) {
        const int32_t j = nbrs[offsets[i] + k];
        double d[3] = {p[3 * i] - p[3 * j], p[3 * i + 1] - p[3 * j + 1], p[3 * i + 2] - p[3 * j + 2]};
        min_image(d, b);
        const double r2 = len_sq(d);
        if (r2 >= rc_sq) continue;
        const double r = sqrt(r2);
        const double ex = exp(-alpha * (r - r0));
        const double ome = 1.0 - ex;
        /* sum of both ordered pairs: (G_i - G_j) . d  (d = r_i - r_j) */
        const double gd = (G[3 * i] - G[3 * j]) * d[0] + (G[3 * i + 1] - G[3 * j + 1]) * d[1] +
                          (G[3 * i + 2] - G[3 * j + 2]) * d[2];
        const double fpair = -2.0 * D * alpha * ome * ex / r;
        g[0] += gd * fpair / D;
        g[1] += gd * (-2.0 * D * (ome * ex - alpha * (1.0 - 2.0 * ex) * (r - r0) * ex) / r);
        g[2] += gd * (-2.0 * D * alpha * alpha * (1.0 - 2.0 * ex) * ex / r);
      }
    }
  }
  if (grad3) memcpy(grad3, g, sizeof(g));
  free(counts);
  free(offsets);
  free(nbrs);
  free(f);
  free(G);
  return loss;
}

/* Interval index and offset of a spline argument (SplineTable::eval,
 * eam_alloy.cpp:53-62). */
static int32_t spl_idx(int32_t n, double dx_step, double x, double* dx) {
  int32_t idx = (int32_t)(x / dx_step);
  if (idx < 0) idx = 0;
  if (idx >= n - 1) idx = n - 2;
  *dx = x - (double)idx * dx_step;
  return idx;
}

/* Adds w * d(value)/d(a,b,c,d) or w * d(derivative)/d(a,b,c,d) of interval
 * idx into a packed a|b|c|d gradient of one spline (ns intervals). */
static void spl_add_value(double* g, int32_t ns, int32_t idx, double dx, double w) {
  g[idx] += w;
  g[ns + idx] += w * dx;
  g[2 * ns + idx] += w * dx * dx;
  g[3 * ns + idx] += w * dx * dx * dx;
}
static void spl_add_deriv(double* g, int32_t ns, int32_t idx, double dx, double w) {
  g[ns + idx] += w;
  g[2 * ns + idx] += w * 2.0 * dx;
  g[3 * ns + idx] += w * 3.0 * dx * dx;
}

/* EAM: fpair_ij = -(phi'_p(r) + F'_i rho'_tj(r) + F'_j rho'_ti(r)) / r.
 * With the adjoint density weight
 *   w_a = -sum_j rho'_tj(r_aj) (G_a - G_j) . d_aj / r_aj
 * the gradient w.r.t. every coefficient (layout of orc_eam: F, rho, phi,
 * each spline a|b|c|d) is
 *   phi_p : -(q_ij + q_ji) * dphi'/dc at r_ij          (each pair)
 *   rho_tj: -(q_ij + q_ji) F'_i * drho'/dc at r_ij     (and i<->j)
 *           + w_i F''_i * drho/dc at r_ij              (and i<->j)
 *   F_ta  : w_a * dF'/dc at rho_a.
 * gF, grho, gphi are overwritten. */
double orc_eam_fm_loss_grad(const orc_eam* e, int32_t nsnap, int64_t n, const double* pos,
                            const int32_t* types, const orc_box* b, const double* target,
                            double* gF, double* grho, double* gphi) {
  const int32_t nt = e->ntypes;
  const int32_t npairs = nt * (nt + 1) / 2;
  const int32_t nsr = e->nr - 1, nsf = e->nrho - 1;
  memset(gF, 0, sizeof(double) * (size_t)nt * 4 * (size_t)nsf);
  memset(grho, 0, sizeof(double) * (size_t)nt * 4 * (size_t)nsr);
  memset(gphi, 0, sizeof(double) * (size_t)npairs * 4 * (size_t)nsr);
  const size_t nn = (size_t)(n > 0 ? n : 1);
  int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * nn);
  int32_t* offsets = (int32_t*)malloc(sizeof(int32_t) * nn);
  int64_t cap = 64 * (int64_t)nn;
  int32_t* nbrs = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
  double* f = (double*)malloc(sizeof(double) * 3 * nn);
  double* G = (double*)malloc(sizeof(double) * 3 * nn);
  double* rho = (double*)malloc(sizeof(double) * nn);
  double* fp = (double*)malloc(sizeof(double) * nn);
  double* w = (double*)malloc(sizeof(double) * nn);
  const double c = 1.0 / (3.0 * (double)nsnap * (double)n);
  const double rc_sq = e->cutoff * e->cutoff;
  double loss = 0.0;
  for (int32_t s = 0; s < nsnap; ++s) {
    const double* p = pos + (size_t)s * 3 * nn;
    const int32_t* ty = types + (size_t)s * nn;
    const double* t = target + (size_t)s * 3 * nn;
    fm_list(p, n, b, e->cutoff, counts, offsets, &nbrs, &cap);
    orc_eam_forces(e, p, ty, n, b, counts, offsets, nbrs, f, rho, fp, NULL, NULL, NULL);
    for (int64_t k = 0; k < 3 * n; ++k) {
      const double d = f[k] - t[k];
      loss += c * d * d;
      G[k] = 2.0 * c * d;
    }
    memset(w, 0, sizeof(double) * nn);
    /* pass A: phi and direct rho gradients, adjoint density weights */
    for (int64_t i = 0; i < n; ++i) {
      const int32_t ti = ty[i] - 1;
      for (int32_t k = 0; k < counts[i]; ++k) {
        const int32_t j = nbrs[offsets[i] + k];
        const int32_t tj = ty[j] - 1;
        double d[3] = {p[3 * i] - p[3 * j], p[3 * i + 1] - p[3 * j + 1], p[3 * i + 2] - p[3 * j + 2]};
        min_image(d, b);
        const double r2 = len_sq(d);
        if (r2 >= rc_sq) continue;
        const double r = sqrt(r2);
        const double qq = ((G[3 * i] - G[3 * j]) * d[0] + (G[3 * i + 1] - G[3 * j + 1]) * d[1] +
                           (G[3 * i + 2] - G[3 * j + 2]) * d[2]) / r;
        double dx;
        const int32_t idx = spl_idx(e->nr, e->dr, r, &dx);
        const int32_t pp = phi_index(ti, tj, nt);
        spl_add_deriv(gphi + (size_t)pp * 4 * nsr, nsr, idx, dx, -qq);
        spl_add_deriv(grho + (size_t)tj * 4 * nsr, nsr, idx, dx, -qq * fp[i]);
        spl_add_deriv(grho + (size_t)ti * 4 * nsr, nsr, idx, dx, -qq * fp[j]);
        const double drj = orc_spline_deriv(e->rho_coef + (size_t)tj * 4 * nsr, e->nr, e->dr, 0.0, r);
        const double dri = orc_spline_deriv(e->rho_coef + (size_t)ti * 4 * nsr, e->nr, e->dr, 0.0, r);
        w[i] -= drj * qq;
        w[j] -= dri * qq; /* (G_j - G_i) . d_ji = qq * r */
      }
    }
    /* F gradients at rho_a; F''(rho_a) for pass B */
    for (int64_t a = 0; a < n; ++a) {
      const int32_t ta = ty[a] - 1;
      const double* fc = e->F_coef + (size_t)ta * 4 * nsf;
      double dx;
      const int32_t idx = spl_idx(e->nrho, e->drho, rho[a], &dx);
      spl_add_deriv(gF + (size_t)ta * 4 * nsf, nsf, idx, dx, w[a]);
      const double fpp = 2.0 * fc[2 * nsf + idx] + 6.0 * fc[3 * nsf + idx] * dx;
      w[a] *= fpp; /* now w_a F''_a */
    }
    /* pass B: rho value gradients through rho_a */
    for (int64_t i = 0; i < n; ++i) {
      const int32_t ti = ty[i] - 1;
      for (int32_t k = 0; k < counts[i]; ++k) {
        const int32_t j = nbrs[offsets[i] + k];
        const int32_t tj = ty[j] - 1;
        double d[3] = {p[3 * i] - p[3 * j], p[3 * i + 1] - p[3 * j + 1], p[3 * i + 2] - p[3 * j + 2]};
        min_image(d, b);
        const double r2 = len_sq(d);
        if (r2 >= rc_sq) continue;
        const double r = sqrt(r2);
        double dx;
        const int32_t idx = spl_idx(e->nr, e->dr, r, &dx);
        spl_add_value(grho + (size_t)tj * 4 * nsr, nsr, idx, dx, w[i]);
        spl_add_value(grho + (size_t)ti * 4 * nsr, nsr, idx, dx, w[j]);
      }
    }
  }
  free(counts);
  free(offsets);
  free(nbrs);
  free(f);
  free(G);
  free(rho);
  free(fp);
  free(w);
  return loss;
}

/* Overwrites one spline's packed coefficients (kind 0 = F, 1 = rho,
 * 2 = phi), so a caller can evaluate the loss at perturbed coefficients. */
int32_t orc_eam_set_coeffs(orc_eam* e, int32_t kind, int32_t idx, const double* in) {
  const int32_t nt = e->ntypes;
  const int32_t npairs = nt * (nt + 1) / 2;
  if (kind == 0 && idx >= 0 && idx < nt) {
    memcpy(e->F_coef + (size_t)idx * 4 * (e->nrho - 1), in, sizeof(double) * 4 * (size_t)(e->nrho - 1));
    return 0;
  }
  if (kind == 1 && idx >= 0 && idx < nt) {
    memcpy(e->rho_coef + (size_t)idx * 4 * (e->nr - 1), in, sizeof(double) * 4 * (size_t)(e->nr - 1));
    return 0;
  }
  if (kind == 2 && idx >= 0 && idx < npairs) {
    memcpy(e->phi_coef + (size_t)idx * 4 * (e->nr - 1), in, sizeof(double) * 4 * (size_t)(e->nr - 1));
    return 0;
  }
  return 1;
}
