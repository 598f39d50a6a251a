/*
 * tdmd_b200.h -- C ABI of the B200-native TDMD force + integration path.
 *
 * Plain C: pointers, sizes, opaque handles and int status codes.  No CUDA or
 * torch types appear in a signature; CUDA streams travel as `void*`
 * (a cudaStream_t, NULL = legacy default stream) and device arrays as typed
 * pointers.  Every call returns TDMD_OK (0) or a tdmd_status code and leaves
 * a message for tdmd_last_error() (thread-local).
 *
 * Each entry point names the reference interface it replaces
 * (tdmd_Claude, path:line).  The header-only C++ layer in tdmd_b200.hpp puts
 * the reference's class and function names back on top of these calls.
 *
 * Array layouts follow the reference's role types (src/core/types.hpp:63-79):
 *   positions, velocities : double[3*n]  (Vec3D, AoS)
 *   forces                : double[3*n] (FP64) or float[3*n] (mixed), AoS
 *   types                 : int32[n], 1-based
 *   ids                   : int32[n]
 *   masses                : double[ntypes+1], indexed by the 1-based type
 */
#ifndef TDMD_B200_H
#define TDMD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDMD_B200_ABI_VERSION 3

typedef enum tdmd_status {
  TDMD_OK = 0,
  TDMD_ERR_INVALID_ARGUMENT = 1,
  TDMD_ERR_CUDA = 2,
  TDMD_ERR_OUT_OF_MEMORY = 3,
  TDMD_ERR_PARSE = 4,          /* malformed setfl / data input            */
  TDMD_ERR_STATE = 5,          /* call order (e.g. run_until before upload) */
  TDMD_ERR_NLIST_OVERFLOW = 6, /* neighbor capacity exceeded, retry failed  */
  TDMD_ERR_TIMEOUT = 7,        /* a bounded device-side wait gave up        */
  TDMD_ERR_UNSUPPORTED = 8,
  TDMD_ERR_IO = 9              /* a file could not be opened or written     */
} tdmd_status;

/* Arithmetic of the force path.  FP64: everything double (the reference's
 * TDMD_PRECISION=fp64 build).  MIXED: pair distances, splines and forces in
 * FP32 with compensated FP32 per-atom accumulation; positions, velocities,
 * energies, virial and the thermostat chain in FP64. */
typedef enum tdmd_precision { TDMD_FP64 = 0, TDMD_MIXED = 1 } tdmd_precision;

/* PotentialKind, src/scheduler/fast_pipeline_scheduler.cuh:36-39 */
typedef enum tdmd_potential_kind { TDMD_POT_MORSE = 0, TDMD_POT_EAM = 1 } tdmd_potential_kind;

/* Box, src/core/box.hpp:17-26 (orthorhombic, periodic flags per axis). */
typedef struct tdmd_box {
  double lo[3];
  double hi[3];
  int32_t periodic[3];
} tdmd_box;

/* MorseParams, src/potentials/device_morse.cuh:14-20 */
typedef struct tdmd_morse_params {
  double d;
  double alpha;
  double r0;
  double rc;
  double rc_sq;
} tdmd_morse_params;

/* FastPipelineConfig, src/scheduler/fast_pipeline_scheduler.cuh:42-46, plus
 * the precision chosen per scheduler at run time (the reference fixes it at
 * compile time), the CUDA-graph switch, NVT and adaptive-dt settings
 * (PipelineConfig, src/scheduler/pipeline_scheduler.cuh:26-45). */
typedef struct tdmd_fast_pipeline_config {
  double dt;              /* ps, default 0.001                               */
  double r_skin;          /* A, default 1.0                                  */
  int32_t rebuild_every;  /* default 10                                      */
  int32_t precision;      /* tdmd_precision                                  */
  int32_t use_graphs;     /* capture rebuild windows as CUDA graphs (1)      */
  int32_t lanes_per_atom; /* 0 = autotuned choice, else 1,2,4,8,16 or 32     */
  /* NVT (Nose-Hoover chain) -- enabled when t_target > 0. */
  double t_target;        /* K                                               */
  double t_period;        /* ps                                              */
  int32_t nhc_length;     /* chain length                                    */
  /* Adaptive dt: dt = clamp(c2*rc/vmax, dt_min, dt_max) at each step start. */
  int32_t adaptive_dt;
  double dt_min;
  double dt_max;
  double c2;
  /* Energy log: every `energy_every` steps (0 = off) the step's potential
   * energy, kinetic energy (integer time) and virial are reduced on the
   * device (FP64) into a log read by tdmd_sched_energy_log. */
  int32_t energy_every;
  int32_t energy_log_capacity;
  /* Neighbors each lane loads per sweep in the gather passes: 0 = chosen by
   * the autotuner (4 when it does not run), else 2 or 4.  Results are
   * bit-reproducible for a fixed (lanes_per_atom, nbr_batch) pair. */
  int32_t nbr_batch;
} tdmd_fast_pipeline_config;

/* FastPipelineStats, src/scheduler/fast_pipeline_scheduler.cuh:49-53, plus
 * graph and neighbor-capacity counters. */
typedef struct tdmd_fast_pipeline_stats {
  int64_t ticks;
  int64_t kernel_launches; /* kernels enqueued (graph nodes counted per replay) */
  int64_t rebuilds;
  int64_t graph_launches;
  int64_t nlist_retries;   /* windows re-run after a capacity overflow        */
  int64_t nlist_capacity;  /* neighbor slots per atom currently allocated     */
  /* Launch shapes in use (after any autotuning): the pair-force pass and,
   * for EAM, the density pass (0 for Morse). */
  int32_t lanes_per_atom;
  int32_t nbr_batch;
  int32_t density_lanes_per_atom;
  int32_t density_nbr_batch;
} tdmd_fast_pipeline_stats;

/* ------------------------------------------------------------------------ */
/* Library                                                                   */
/* ------------------------------------------------------------------------ */
const char* tdmd_last_error(void);
int32_t tdmd_abi_version(void);
/* Copies `bytes` between any two host/device pointers (cudaMemcpyDefault)
 * on `stream` and waits for it.  Lets FFI callers read back the device
 * arrays the list/force entry points fill (no reference counterpart: the
 * reference's DeviceBuffer::copy_to_host, src/core/device_buffer.cuh:80-95,
 * is a member of its RAII buffer). */
int32_t tdmd_copy(void* dst, const void* src, size_t bytes, void* stream);
/* Fills cfg with the reference defaults (dt 0.001, skin 1.0, rebuild 10,
 * FP64, graphs on, NVE, no energy log). */
void tdmd_fast_pipeline_config_default(tdmd_fast_pipeline_config* cfg);

/* ------------------------------------------------------------------------ */
/* EAM/alloy tables -- EamAlloy, src/potentials/eam_alloy.hpp:47-93          */
/* ------------------------------------------------------------------------ */
typedef struct tdmd_eam tdmd_eam;

/* EamAlloy::read_setfl, src/potentials/eam_alloy.cpp:90-192. */
int32_t tdmd_eam_read_setfl(const char* path, tdmd_eam** out);
/* Same tables from raw setfl arrays: F[ntypes*nrho], rho[ntypes*nr],
 * rphi[npairs*nr] (r*phi(r), pairs i<=j in setfl order). */
int32_t tdmd_eam_create(int32_t ntypes, int32_t nrho, double drho, int32_t nr, double dr,
                        double cutoff, const double* F, const double* rho, const double* rphi,
                        tdmd_eam** out);
/* Same tables from the sampled functions as the reference's EamAlloy holds
 * them after read_setfl (eam_alloy.cpp:150-189, the SplineTable values of
 * embedding(), density() and phi()): F[ntypes*nrho], rho[ntypes*nr] and
 * phi[npairs*nr] = phi(k*dr) itself (the setfl's r*phi over r, phi(0) = 0),
 * pairs i<=j in setfl order.  The splines are built from these samples
 * exactly as from read_setfl's. */
int32_t tdmd_eam_create_sampled(int32_t ntypes, int32_t nrho, double drho, int32_t nr,
                                double dr, double cutoff, const double* F, const double* rho,
                                const double* phi, tdmd_eam** out);
int32_t tdmd_eam_destroy(tdmd_eam* eam);
/* cutoff(), ntypes(); table sizes. */
int32_t tdmd_eam_info(const tdmd_eam* eam, int32_t* ntypes, int32_t* nrho, double* drho,
                      int32_t* nr, double* dr, double* cutoff);
/* Packed a|b|c|d coefficients of one spline (kind 0 = F, 1 = rho, 2 = phi),
 * SplineTable::build_splines, eam_alloy.cpp:19-50.  out holds 4*(n-1). */
int32_t tdmd_eam_coeffs(const tdmd_eam* eam, int32_t kind, int32_t index, double* out);

/* ------------------------------------------------------------------------ */
/* Cell list -- DeviceCellList, src/domain/device_cell_list.cuh:16           */
/* ------------------------------------------------------------------------ */
typedef struct tdmd_cell_list tdmd_cell_list;
int32_t tdmd_cell_list_create(tdmd_cell_list** out);
int32_t tdmd_cell_list_destroy(tdmd_cell_list* cl);
/* DeviceCellList::build, device_cell_list.cu:59-150: counting sort of the
 * atoms into nc = max(3, floor(L/r_list)) cells per axis, atoms ID-ascending
 * within each cell.  d_positions: double[3*n] on the device. */
int32_t tdmd_cell_list_build(tdmd_cell_list* cl, const double* d_positions, int64_t natoms,
                             const tdmd_box* box, double r_list, void* stream);
/* Device pointers: cell_atoms[n], cell_offsets[ncells], cell_counts[ncells],
 * atom_cells[n]; grid dims nc[3]. */
int32_t tdmd_cell_list_get(const tdmd_cell_list* cl, const int32_t** cell_atoms,
                           const int32_t** cell_offsets, const int32_t** cell_counts,
                           const int32_t** atom_cells, int32_t nc[3]);

/* ------------------------------------------------------------------------ */
/* Neighbor list -- DeviceNeighborList, device_neighbor_list.cuh:20-65       */
/* ------------------------------------------------------------------------ */
typedef struct tdmd_nlist tdmd_nlist;
int32_t tdmd_nlist_create(tdmd_nlist** out);
int32_t tdmd_nlist_destroy(tdmd_nlist* nl);
/* DeviceNeighborList::build, device_neighbor_list.cu:158-278: full list
 * (both i->j and j->i), dense CSR.  Per-atom order is the reference's
 * ID-ordered-scatter order: stencil dz,dy,dx in -1..1, atoms of each cell
 * ID-ascending; pairs kept when the FP64 min-image r^2 < (r_cut+r_skin)^2. */
int32_t tdmd_nlist_build(tdmd_nlist* nl, const double* d_positions, int64_t natoms,
                         const tdmd_box* box, double r_cut, double r_skin, void* stream);
/* d_neighbors(), d_counts(), d_offsets(), max_neighbors(), plus total. */
int32_t tdmd_nlist_get(const tdmd_nlist* nl, const int32_t** d_neighbors,
                       const int32_t** d_offsets, const int32_t** d_counts,
                       int32_t* max_neighbors, int64_t* total_pairs);

/* ------------------------------------------------------------------------ */
/* Forces on caller-owned device arrays                                      */
/* ------------------------------------------------------------------------ */
/* compute_morse_gpu, src/potentials/device_morse.cuh:37-41.  Forces are
 * STORED (not accumulated); d_energy (nullable) is ACCUMULATED (+=) with the
 * potential energy in FP64; d_virial (nullable, 6 doubles xx,yy,zz,xy,xz,yz)
 * is accumulated likewise.  precision selects double or float d_forces.
 * Energies are reduced in a fixed order (no atomics). */
int32_t tdmd_morse_compute(const double* d_positions, void* d_forces, int32_t precision,
                           const int32_t* d_neighbors, const int32_t* d_offsets,
                           const int32_t* d_counts, int32_t natoms, const tdmd_box* box,
                           const tdmd_morse_params* params, double* d_energy, double* d_virial,
                           void* stream);

/* compute_morse_gpu_zone, src/potentials/device_morse_zone.cuh:13-23 (the
 * TD zone pipeline's force call): Morse forces of atoms
 * [first_atom, first_atom + atom_count) only, from the global positions and
 * the global neighbor list (dense CSR; neighbor indices are global).  Forces
 * are ADDED to d_forces[first_atom ..] (the reference's zone kernel
 * accumulates; zero the range first for the zone's forces); d_energy /
 * d_virial (nullable) are added to with the range's potential energy and
 * virial, reduced in a fixed order.  The ID-ordered energy mode does not
 * apply to this call. */
int32_t tdmd_morse_compute_zone(const double* d_positions, void* d_forces, int32_t precision,
                                const int32_t* d_neighbors, const int32_t* d_offsets,
                                const int32_t* d_counts, int32_t first_atom, int32_t atom_count,
                                const tdmd_box* box, const tdmd_morse_params* params,
                                double* d_energy, double* d_virial, void* stream);

/* No counterpart in the reference.  Same arguments and results as
 * tdmd_morse_compute, but it allocates no device memory: the per-block
 * energy/virial partials live in a fixed 1 MiB scratch array compiled into
 * the library, one per device.  For callers that size all device memory up
 * front and must not let a force call draw on the CUDA memory pool.
 *  - natoms above TDMD_MORSE_NOALLOC_MAX_ATOMS is rejected
 *    (TDMD_ERR_INVALID_ARGUMENT) before any launch;
 *  - d_energy / d_virial are added to (zero them for this call's totals);
 *    the scratch itself needs no zeroing;
 *  - two calls in flight on one device at the same time share the scratch
 *    and race: order them on one stream;
 *  - the first call on each device (made with that device current) that
 *    asks for an energy or a virial looks up the scratch address; make it
 *    before any stream capture begins.  Force-only and natoms == 0 calls
 *    use no scratch and do no look-up. */
#define TDMD_MORSE_NOALLOC_MAX_ATOMS 524288
int32_t tdmd_morse_compute_noalloc(const double* d_positions, void* d_forces, int32_t precision,
                                   const int32_t* d_neighbors, const int32_t* d_offsets,
                                   const int32_t* d_counts, int32_t natoms, const tdmd_box* box,
                                   const tdmd_morse_params* params, double* d_energy,
                                   double* d_virial, void* stream);

/* The ID-ordered energy mode, the run-time form of the reference's
 * TDMD_DETERMINISTIC_REDUCE build (src/core/determinism.hpp:20-24, ADR
 * 0010; sum_per_atom_kernel, src/potentials/device_morse.cu:16-30).
 * Process-wide, off by default.  While on, tdmd_morse_compute and
 * tdmd_device_eam_compute in TDMD_FP64 that ask for an energy or a virial
 * compute each atom's energy with the reference's per-atom arithmetic in
 * neighbor-row order and add the atoms' energies to *d_energy one after
 * another in atom-ID order (EAM: the embedding energies, then the pair
 * halves), the virial likewise: the energies equal the reference's
 * deterministic build bit for bit.  Slower (one thread per atom, one-thread
 * sums).  Mixed precision and the scheduler keep their fixed-order block
 * reductions, which are reproducible run to run. */
int32_t tdmd_set_deterministic_reduce(int32_t on);
int32_t tdmd_get_deterministic_reduce(int32_t* on);

/* ------------------------------------------------------------------------ */
/* File formats (host only).                                                */
/* ------------------------------------------------------------------------ */
/* read_lammps_data, src/io/lammps_data_reader.cpp:33-204: a LAMMPS
 * `atomic` data file into a host SystemState (ids 1-based, atom with id k
 * at index k-1, velocities 0 without a Velocities section, masses
 * [ntypes+1] with 1.0 where Masses gives none, periodic box).  A file that
 * cannot be opened returns TDMD_ERR_IO; parse errors return TDMD_ERR_PARSE;
 * so does an atom id outside 1..N or a Masses type outside 1..ntypes (where
 * the reference would index out of its arrays). */
typedef struct tdmd_system tdmd_system;
int32_t tdmd_read_lammps_data(const char* path, tdmd_system** out);
int32_t tdmd_system_destroy(tdmd_system* s);
/* The arrays of a read SystemState (owned by it): positions and velocities
 * double[3n], types and ids int32[n], masses double[ntypes+1].  Any output
 * may be null. */
int32_t tdmd_system_get(const tdmd_system* s, int64_t* natoms, int32_t* ntypes, tdmd_box* box,
                        const double** positions, const double** velocities,
                        const int32_t** types, const int32_t** ids, const double** masses);
/* No reference counterpart (the reference reads data files only): writes
 * a data file that read_lammps_data reads back exactly (17 significant
 * digits): title line, counts, box, Masses (masses[ntypes+1], nullable:
 * 1.0), "Atoms # atomic", and Velocities when velocities is non-null;
 * ids nullable (1..N). */
int32_t tdmd_write_lammps_data(const char* path, const char* title, int64_t natoms,
                               int32_t ntypes, const tdmd_box* box, const double* positions,
                               const double* velocities, const int32_t* types,
                               const int32_t* ids, const double* masses);
/* read_lammps_dump, src/io/dump_reader.cpp:15-55: a `dump custom id type x
 * y z fx fy fz` file, records sorted by id.  *natoms gets the count; with
 * every array null nothing else is read (size query), otherwise capacity
 * must be >= the count; each array may be null. */
int32_t tdmd_read_force_dump(const char* path, int64_t* natoms, int64_t capacity, int32_t* ids,
                             int32_t* types, double* positions, double* forces);
/* write_lammps_force_dump, src/drivers/tdmd_main.cpp:65-95: TIMESTEP,
 * NUMBER OF ATOMS, BOX BOUNDS pp pp pp, ATOMS id type x y z fx fy fz with
 * 17 significant digits; forces double[3n] (TDMD_FP64) or float[3n]
 * (TDMD_MIXED); ids nullable (1..N). */
int32_t tdmd_write_force_dump(const char* path, int64_t step, int64_t natoms,
                              const tdmd_box* box, const int32_t* ids, const int32_t* types,
                              const double* positions, const void* forces,
                              int32_t force_precision);
/* No reference counterpart (the reference reads setfl only): writes the
 * raw tables of an EAM in the setfl layout EamAlloy::read_setfl
 * (src/potentials/eam_alloy.cpp:90-192) reads, values with 17 significant
 * digits, so reading the file back gives the same tables and spline
 * coefficients bit for bit.  A table read from a setfl keeps its comment
 * and element header lines unless comment / masses (double[ntypes],
 * nullable) are given; elements (nullable) replaces the element names with
 * a space-separated list. */
int32_t tdmd_write_setfl(const char* path, const tdmd_eam* eam, const char* comment,
                         const double* masses, const char* elements);

/* DeviceEam, src/potentials/device_eam.cuh:26-75: device copy of the
 * tables plus rho/fp scratch. */
typedef struct tdmd_device_eam tdmd_device_eam;
/* DeviceEam::upload_tables, device_eam.cu:282-340. */
int32_t tdmd_device_eam_create(const tdmd_eam* eam, tdmd_device_eam** out);
int32_t tdmd_device_eam_destroy(tdmd_device_eam* de);
/* DeviceEam::compute, device_eam.cu:342-420: density -> embedding -> force.
 * Same store/accumulate contract as tdmd_morse_compute.  d_rho / d_fp
 * (nullable, double[n]) receive the per-atom density and F'(rho). */
int32_t tdmd_device_eam_compute(tdmd_device_eam* de, const double* d_positions, void* d_forces,
                                int32_t precision, const int32_t* d_types,
                                const int32_t* d_neighbors, const int32_t* d_offsets,
                                const int32_t* d_counts, int32_t natoms, const tdmd_box* box,
                                double* d_energy, double* d_virial, double* d_rho, double* d_fp,
                                void* stream);

/* ------------------------------------------------------------------------ */
/* Integrator -- src/integrator/device_velocity_verlet.cuh:13-59             */
/* force_precision says whether d_forces is double or float.                 */
/* ------------------------------------------------------------------------ */
int32_t tdmd_vv_half_kick(double* d_velocities, const void* d_forces, int32_t force_precision,
                          const int32_t* d_types, const double* d_masses, int32_t natoms,
                          double dt, void* stream);
int32_t tdmd_vv_drift(double* d_positions, const double* d_velocities, int32_t natoms, double dt,
                      const tdmd_box* box, void* stream);
/* full_kick = 0: device_fused_half_kick_drift; 1: device_fused_full_kick_drift. */
int32_t tdmd_vv_fused_kick_drift(double* d_velocities, double* d_positions, const void* d_forces,
                                 int32_t force_precision, const int32_t* d_types,
                                 const double* d_masses, int32_t natoms, double dt,
                                 const tdmd_box* box, int32_t full_kick, void* stream);
int32_t tdmd_vv_zero_forces(void* d_forces, int32_t force_precision, int32_t natoms,
                            void* stream);

/* ------------------------------------------------------------------------ */
/* Reductions + thermostat -- src/integrator/device_nose_hoover.cuh:26-88    */
/* All reductions are FP64, fixed-order (bit-reproducible), no atomics.      */
/* ------------------------------------------------------------------------ */
/* device_compute_ke: writes the result to *h_ke (host) after a stream sync. */
int32_t tdmd_reduce_ke(const double* d_velocities, const int32_t* d_types,
                       const double* d_masses, int32_t natoms, double* h_ke, void* stream);
/* device_compute_vmax: sqrt(max |v|^2). */
int32_t tdmd_reduce_vmax(const double* d_velocities, int32_t natoms, double* h_vmax,
                         void* stream);
/* device_scale_velocities. */
int32_t tdmd_scale_velocities(double* d_velocities, int32_t natoms, double factor, void* stream);

/* NoseHooverChain (host object), device_nose_hoover.cu:187-289. */
typedef struct tdmd_nhc tdmd_nhc;
int32_t tdmd_nhc_create(double t_target, double t_period, int32_t chain_length, double dt,
                        int32_t n_dof, tdmd_nhc** out);
int32_t tdmd_nhc_destroy(tdmd_nhc* nhc);
int32_t tdmd_nhc_half_step(tdmd_nhc* nhc, double ke_current, double* scale);
/* NoseHooverChain::set_t_target, device_nose_hoover.cuh:50: changes the
 * target temperature only (the chain masses are not recomputed). */
int32_t tdmd_nhc_set_t_target(tdmd_nhc* nhc, double t_target);
/* state out: eta[M], eta_v[M], eta_m[M]. */
int32_t tdmd_nhc_state(const tdmd_nhc* nhc, double* eta, double* eta_v, double* eta_m);

/* ------------------------------------------------------------------------ */
/* FastPipelineScheduler, src/scheduler/fast_pipeline_scheduler.cuh:76-192  */
/* ------------------------------------------------------------------------ */
typedef struct tdmd_sched tdmd_sched;
/* ctor (Box, natoms, MorseParams, FastPipelineConfig), .cu:15-26 */
int32_t tdmd_sched_create_morse(const tdmd_box* box, int32_t natoms,
                                const tdmd_morse_params* params,
                                const tdmd_fast_pipeline_config* cfg, tdmd_sched** out);
/* ctor (Box, natoms, EamAlloy, FastPipelineConfig), .cu:27-40 */
int32_t tdmd_sched_create_eam(const tdmd_box* box, int32_t natoms, const tdmd_eam* eam,
                              const tdmd_fast_pipeline_config* cfg, tdmd_sched** out);
int32_t tdmd_sched_destroy(tdmd_sched* s);
/* upload(), .cu:49-73.  forces may be NULL (zeros); its element type follows
 * the scheduler's precision.  Resets the step counter. */
int32_t tdmd_sched_upload(tdmd_sched* s, const double* positions, const double* velocities,
                          const void* forces, const int32_t* types, const int32_t* ids,
                          const double* masses, int32_t n_types);
/* run_until(), .cu:195-223: run_until(0) computes the initial forces only;
 * velocities are at integer time on return. */
int32_t tdmd_sched_run_until(tdmd_sched* s, int32_t target_step);
/* download(), .cu:75-85.  Any output pointer may be NULL. */
int32_t tdmd_sched_download(const tdmd_sched* s, double* positions, double* velocities,
                            void* forces, int32_t* types, int32_t* ids, int32_t natoms);
int32_t tdmd_sched_stats(const tdmd_sched* s, tdmd_fast_pipeline_stats* out);
int32_t tdmd_sched_current_step(const tdmd_sched* s, int32_t* step);
int32_t tdmd_sched_potential_kind(const tdmd_sched* s, int32_t* kind);
int32_t tdmd_sched_interaction_cutoff(const tdmd_sched* s, double* cutoff);
/* Potential energy, kinetic energy and virial (FP64) of the current state.
 * Runs an energy pass on the device; no state changes. */
int32_t tdmd_sched_energies(tdmd_sched* s, double* pe, double* ke, double* virial6);
/* Energy log (tdmd_fast_pipeline_config.energy_every): copies up to `cap`
 * records of 9 doubles {step, pe, ke, vxx, vyy, vzz, vxy, vxz, vyz}; *count
 * gets the number of records written since upload. */
int32_t tdmd_sched_energy_log(const tdmd_sched* s, double* records, int32_t cap, int32_t* count);
/* Current dt (adaptive) and NHC chain state (eta[M], eta_v[M]). */
int32_t tdmd_sched_thermostat_state(const tdmd_sched* s, double* dt, double* eta,
                                    double* eta_v);
/* Device pointers of the scheduler's state (for zero-copy callers):
 * positions as double4[n] {x,y,z,type}, velocities double[3n], forces
 * (double or float)[3n]; valid until the next upload/destroy.  The arrays
 * are in the scheduler's internal atom order (see tdmd_sched_atom_order). */
int32_t tdmd_sched_device_state(tdmd_sched* s, void** d_pos4, double** d_vel, void** d_forces);
/* No reference counterpart.  The scheduler holds the atoms in the cell
 * order of the uploaded positions, so that an atom's neighbors sit at
 * nearby indices whatever order the caller used; *d_order (device
 * int32[n]) gives, for each internal index, the caller's index.  Neighbor
 * rows and results are those of the caller's order (cells list their atoms
 * by the caller's index); upload and download convert. */
int32_t tdmd_sched_atom_order(const tdmd_sched* s, const int32_t** d_order);
/* No reference counterpart (the reference keeps its scheduler's
 * DeviceNeighborList private).  Copies the scheduler's current neighbor
 * list to host memory in the caller's atom order as dense CSR: counts[n]
 * (required), then, when neighbors is non-null, the rows back to back
 * (row i starts at the sum of counts[0..i)); *total (nullable) gets the
 * number of entries.  Needs a list (after run_until); synchronises the
 * scheduler's stream; TDMD_ERR_INVALID_ARGUMENT when capacity < total. */
int32_t tdmd_sched_neighbor_list(const tdmd_sched* s, int32_t* counts, int32_t* neighbors,
                                 int64_t capacity, int64_t* total);
/* Per-kernel timing (no reference counterpart; the reference profiles only
 * from outside with nsys/ncu).  While on, CUDA events bracket each phase:
 * windows replay graphs of their own whose event-record nodes surround each
 * phase (their kernels launch without programmatic serialization, so each
 * phase is timed alone), or, with use_graphs off, events recorded on the
 * scheduler's stream.  Results are those of an untimed run.  Averages in ms
 * per launch for the phases {kick+drift, neighbor rebuild, EAM density,
 * force, other} go to avg_ms[0..4], launch counts to counts[0..4]. */
int32_t tdmd_sched_set_profiling(tdmd_sched* s, int32_t on);
int32_t tdmd_sched_kernel_times(const tdmd_sched* s, double* avg_ms, int64_t* counts,
                                int32_t ncat);
/* Autotuner (no reference counterpart): times each gather pass of the
 * scheduler on its current state -- the EAM density pass, then the pair-force
 * pass -- for 1, 2, 4, 8, 16 and 32 lanes per atom and 2 or 4 neighbors per
 * lane sweep (only cfg.nbr_batch when that is fixed), keeps each pass's
 * fastest shape and recomputes the forces with them.  lanes2 / batch2
 * (nullable) get {density, force} (density 0 for Morse); ms24 (nullable)
 * the timings, ms24[12 * pass + 6 * (batch == 4) + k] for 2^k lanes, -1
 * where not measured.  Runs by itself on the first run_until when
 * cfg.lanes_per_atom == 0 and natoms >= 2048.  Results are bit-reproducible
 * for fixed shapes. */
int32_t tdmd_sched_autotune(tdmd_sched* s, int32_t* lanes2, int32_t* batch2, double* ms24);
/* Device time (ms) of the last run_until window: CUDA events recorded on the
 * scheduler's stream before its first and after its last enqueued kernel. */
int32_t tdmd_sched_last_window_ms(const tdmd_sched* s, double* ms);
/* The stream the scheduler enqueues on (a cudaStream_t). */
int32_t tdmd_sched_stream(const tdmd_sched* s, void** stream);

/* ------------------------------------------------------------------------ */
/* Batched replicas (no reference counterpart: the reference runs one       */
/* system per FastPipelineScheduler and only plans multi-step fusion,        */
/* docs gpu-strategy.md:67-82).  Many independent Morse or EAM systems of   */
/* sizes advance together: every phase is one launch over all replicas and  */
/* each run_until window is replayed as one CUDA graph.  Each replica       */
/* follows FastPipelineScheduler's NVE semantics (same step order, rebuild  */
/* every cfg.rebuild_every steps, velocities at integer time after          */
/* run_until); with equal lanes_per_atom its trajectory is bit-identical to */
/* a single scheduler's.  NVT and adaptive dt are rejected                  */
/* (TDMD_ERR_UNSUPPORTED).                                                  */
/* ------------------------------------------------------------------------ */
typedef struct tdmd_batch tdmd_batch;
/* boxes[nreplicas], natoms[nreplicas]; every periodic edge must exceed
 * 2 (rc + r_skin). */
int32_t tdmd_batch_create_morse(int32_t nreplicas, const tdmd_box* boxes, const int32_t* natoms,
                                const tdmd_morse_params* params,
                                const tdmd_fast_pipeline_config* cfg, tdmd_batch** out);
/* EAM replicas sharing one set of tables (each replica's trajectory equals
 * a single EAM FastPipelineScheduler's with the same lanes_per_atom). */
int32_t tdmd_batch_create_eam(int32_t nreplicas, const tdmd_box* boxes, const int32_t* natoms,
                              const tdmd_eam* eam, const tdmd_fast_pipeline_config* cfg,
                              tdmd_batch** out);
int32_t tdmd_batch_destroy(tdmd_batch* b);
/* Arrays hold all replicas back to back in replica order (positions and
 * velocities double[3*total], types int32[total]); masses[n_types] are
 * shared by all replicas.  Resets the step counter and the energy log. */
int32_t tdmd_batch_upload(tdmd_batch* b, const double* positions, const double* velocities,
                          const int32_t* types, const double* masses, int32_t n_types);
int32_t tdmd_batch_run_until(tdmd_batch* b, int32_t target_step);
/* Any pointer may be NULL; forces are float (mixed) or double (FP64). */
int32_t tdmd_batch_download(const tdmd_batch* b, double* positions, double* velocities,
                            void* forces);
/* Potential and kinetic energy per replica (double[nreplicas] each). */
int32_t tdmd_batch_energies(tdmd_batch* b, double* pe, double* ke);
/* Energy log: with cfg.energy_every > 0, every run_until window that ends
 * on a multiple of energy_every appends {step} and {pe, ke} per replica
 * (up to cfg.energy_log_capacity windows, default 1024).  Copies up to
 * `cap` windows: steps[cap], pe_ke[cap][nreplicas][2]; *count = windows
 * logged. */
int32_t tdmd_batch_energy_log(const tdmd_batch* b, double* steps, double* pe_ke, int32_t cap,
                              int32_t* count);
int32_t tdmd_batch_stats(const tdmd_batch* b, tdmd_fast_pipeline_stats* out);
int32_t tdmd_batch_info(const tdmd_batch* b, int32_t* nreplicas, int64_t* natoms_total,
                        int32_t* lanes_per_atom, int32_t* current_step);
/* As tdmd_sched_autotune for the batched passes (runs by itself on the
 * first run_until when cfg.lanes_per_atom is 0 and the batch has >= 2048
 * atoms). */
int32_t tdmd_batch_autotune(tdmd_batch* b, int32_t* lanes2, int32_t* batch2, double* ms24);
/* Device time of the last run_until window (events on the batch's stream). */
int32_t tdmd_batch_last_window_ms(const tdmd_batch* b, double* ms);
int32_t tdmd_batch_stream(const tdmd_batch* b, void** stream);

/* ------------------------------------------------------------------------ */
/* Force matching (no reference counterpart: the reference computes no      */
/* gradients).  Loss over nsnap snapshots of natoms atoms in one box,       */
/*   L = 1/(3 nsnap natoms) * sum |F_i(theta) - T_i|^2,                     */
/* with the Morse or EAM forces of this library, and its gradient by the   */
/* adjoint of the force expressions (FP64 accumulation).  Parameters,      */
/* coefficients, loss and gradients are DEVICE pointers, so a fitting loop  */
/* runs without host round trips; calls on one tdmd_fit share its scratch  */
/* and must be ordered on one stream.                                       */
/* ------------------------------------------------------------------------ */
typedef struct tdmd_fit tdmd_fit;
/* Host positions double[nsnap*natoms*3], types int32[nsnap*natoms]
 * (1-based); neighbor lists with r_list = cutoff are built here once. */
int32_t tdmd_fit_create(int32_t nsnap, int32_t natoms, const tdmd_box* box,
                        const double* positions, const int32_t* types, double cutoff,
                        int32_t precision, tdmd_fit** out);
int32_t tdmd_fit_destroy(tdmd_fit* f);
/* Target forces, host double[nsnap*natoms*3]. */
int32_t tdmd_fit_set_targets(tdmd_fit* f, const double* targets);
/* Morse (cutoff = the fit's cutoff): d_params = {D, alpha, r0}; writes
 * *d_loss and d_grad[3] = dL/d{D, alpha, r0} (nullable: loss only) and the
 * predicted forces d_forces[3*M] (nullable). */
int32_t tdmd_fit_morse(tdmd_fit* f, const double* d_params, double* d_loss, double* d_grad,
                       double* d_forces, void* stream);
/* EAM with spline coefficients packed a|b|c|d per spline as
 * tdmd_eam_coeffs gives them: d_F[ntypes][4(nrho-1)], d_rho[ntypes][4(nr-1)],
 * d_phi[npairs][4(nr-1)]; the fit's cutoff must not exceed the r tables'
 * range (nr-1)*dr.  Gradients have the same layout and are overwritten;
 * pass all three or none. */
int32_t tdmd_fit_eam(tdmd_fit* f, int32_t ntypes, int32_t nrho, double drho, int32_t nr,
                     double dr, const double* d_F, const double* d_rho, const double* d_phi,
                     double* d_loss, double* d_gF, double* d_grho, double* d_gphi,
                     double* d_forces, void* stream);
int32_t tdmd_fit_info(const tdmd_fit* f, int64_t* natoms_total, int32_t* lanes_per_atom);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* TDMD_B200_H */
