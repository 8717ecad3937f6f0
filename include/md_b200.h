/* md_b200.h — C-ABI of libmdgpu.so, the B200 (sm_100a) implementation of the per-step Lennard-Jones hot path
 * of nhantran1711/molecular-dynamics: cell list -> Verlet neighbour list -> truncated-shifted LJ forces ->
 * velocity Verlet with periodic wrap -> rescale / Bussi thermostat -> g(r).
 *
 * Plain pointers and sizes only. Every entry point returns an md_status; md_last_error() describes the
 * last failure on the calling thread. Host pointers passed in are read or written synchronously unless a
 * function says otherwise. Handles are not thread-safe: calls on one system are serialised on its stream.
 *
 * Array layouts (the reference's System layout, include/System.hpp:12-136):
 *   pos4   n x 4 doubles, particle i at pos4[4 i + k] for k = 0, 1, 2 and a pad at 4 i + 3
 *   vel3   3 x n doubles, component k of particle i at vel3[k n + i] (likewise force3)
 *   mass   n doubles;  ids  n uint64 (ids[i] = original index of the particle stored at i)
 */
#ifndef MD_B200_H
#define MD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum md_status {
    MD_OK = 0,
    MD_ERR_INVALID = 1,          /* bad argument: null handle or pointer, size mismatch, bad mode */
    MD_ERR_CUTOFF = 2,           /* 2 r_c > L (src/Forcefield.cpp:18-22) */
    MD_ERR_LIST_RADIUS = 3,      /* 2 (r_c + skin) > L (src/NeighbourList.cpp:57-59) */
    MD_ERR_NO_REVERSE_INDEX = 4, /* deterministic forces need a reverse index (src/Forcefield.cpp:217-219) */
    MD_ERR_CAPACITY = 5,         /* a neighbour row overflowed inside a device-side run; state is undefined */
    MD_ERR_CUDA = 6,             /* a CUDA runtime call failed */
    MD_ERR_NO_DEVICE = 7,        /* no usable CUDA device */
    MD_ERR_STATE = 8,            /* call out of order, e.g. list forces before any list build */
    MD_ERR_TIMEOUT = 9           /* a bounded device wait gave up */
} md_status;

/* Precision of the list force kernel */
typedef enum md_precision {
    MD_PREC_FP64 = 0,   /* double throughout, bit-identical to the reference's deterministic path */
    MD_PREC_FP32FX = 1, /* float pair arithmetic, 64-bit fixed-point force accumulation */
    MD_PREC_FP32 = 2,   /* float pair arithmetic, float accumulation */
    MD_PREC_FX64 = 3,   /* exact separations from 32-bit fixed-point frames, double pair terms, 64-bit
                           fixed-point accumulation */
    MD_PREC_FX32 = 4    /* double pair terms on exact separations (32-bit fixed-point frames) for the pairs
                           closer than 1.2 sigma + skin at the list build (at most the 16 closest of a row), float
                           pair terms (MD_PREC_FP32FX's) for the rest; 64-bit fixed-point sums */
} md_precision;

typedef struct md_system md_system;         /* System (include/System.hpp:12) */
typedef struct md_cells md_cells;           /* CellList (include/CellList.hpp:11) */
typedef struct md_nlist md_nlist;           /* NeighbourList (include/NeighbourList.hpp:10) */
typedef struct md_forcefield md_forcefield; /* LennardJonesForceField (include/Forcefield.hpp:6) */
typedef struct md_rdf md_rdf;               /* RadialDistribution (include/RadialDistribution.hpp:8) */

/* ---- library ------------------------------------------------------------------------------------- */
const char* md_last_error(void);
/* Version string and the device the library was built for ("sm_100a"). */
const char* md_version(void);
/* Number of CUDA devices visible (0 on a host without a GPU; never fails). */
int md_device_count(void);

/* ---- System: include/System.hpp:15-125, src/System.cpp ---------------------------------------------- */
/* System(particles, boxLength) (src/System.cpp:9-29): n particles on `device`, box length L. Ids start at
 * 0..n-1; velocities, forces and positions start at zero and masses at 1 until uploaded. */
md_status md_system_create(int64_t n, double box_length, int device, md_system** out);
md_status md_system_destroy(md_system* s);
md_status md_system_size(const md_system* s, int64_t* n, double* box_length);
/* Copy host arrays to the device; any pointer may be NULL to leave that array unchanged. */
md_status md_system_upload(md_system* s, const double* pos4, const double* vel3, const double* force3,
                           const double* mass, const uint64_t* ids);
/* Copy device arrays to the host; any pointer may be NULL. */
md_status md_system_download(md_system* s, double* pos4, double* vel3, double* force3, double* mass,
                             uint64_t* ids);
/* System::reorder (src/System.cpp:42-64): new particle k is old particle order[k]. */
md_status md_system_reorder(md_system* s, const uint64_t* order);
/* System::kineticEnergy (src/System.cpp:67-76), same 1024-block summation order (include/Parallel.hpp:32-57). */
md_status md_kinetic_energy(md_system* s, double* out);
/* System::temperature (src/System.cpp:79-82). */
md_status md_temperature(md_system* s, double* out);
/* System::stateHash (src/System.cpp:85-105): FNV-1a of every position and velocity bit pattern. */
md_status md_state_hash(md_system* s, uint64_t* out);
/* Multiply every velocity component by `scale` (src/Thermostat.cpp:6-12). */
md_status md_scale_velocities(md_system* s, double scale);
/* rescaleVelocities (src/Thermostat.cpp:17-30), computed on the device from the device kinetic energy. */
md_status md_rescale_velocities(md_system* s, double target_temperature);
/* BussiThermostat::apply(system, dt) (src/Thermostat.cpp:36-58) for a thermostat of coupling time tau, with
 * the draws r1 ~ N(0,1) and chi2 ~ Gamma(0.5 (dof-1), 2) supplied by the caller (md_bussi_noise makes them
 * from the reference's seed). */
md_status md_bussi_apply(md_system* s, double temperature, double tau, double dt, double r1, double chi2);
/* The (r1, chi2) draws of `count` successive BussiThermostat::apply calls on a system of n particles from
 * std::mt19937_64(seed) (src/Thermostat.cpp:48-51): r1[k], chi2[k]. Host-only, no device needed. */
md_status md_bussi_noise(uint64_t seed, int64_t n, int64_t count, double* r1, double* chi2);

/* ---- Initialisation: include/Initialisation.hpp:9-12, src/Initialisation.cpp (host input set-up) ----- */
/* createFCCLattice (src/Initialisation.cpp:7-44): 4 cells^3 particles offset by a/4, into pos4 (host). */
md_status md_fcc_lattice(int cells, double lattice_constant, double* pos4);
/* initializeVelocities (src/Initialisation.cpp:47-76): Maxwell-Boltzmann draws from std::mt19937(seed) on the
 * host, centre-of-mass removal, then rescaleVelocities on the device. Uses the system's masses. */
md_status md_initialize_velocities(md_system* s, double temperature, uint32_t seed);

/* Kinetic energy for callers that may not allocate device memory. No counterpart in the reference: it
 * serves hosts that own all device memory themselves (an embedding runtime with its own pool, or a process
 * that must not call cudaMalloc/cudaFree while running). vel3 (3 x n, component-major), mass (n) and out (one
 * double) are device pointers the caller owns; the result is bit-identical to md_kinetic_energy's (same
 * 1024-particle blocked order). Work is queued on `stream` (a cudaStream_t; NULL = legacy default stream)
 * and the call returns without waiting. Scratch lives in a fixed 256 KB device array that every GPU loading
 * the library keeps until exit; n above 16,777,216 is rejected with MD_ERR_INVALID. The first call on a
 * device (and the first after a device reset, which gives the device a new context) looks that array up on
 * the current device (cudaGetSymbolAddress), so make the first call on each device before any stream
 * capture. That first call may also be what loads the library's device code (CUDA loads modules lazily by
 * default), and the driver backs the loaded code and the array with device memory; a host that must see no
 * allocation after start-up makes one warm-up call then, or runs with CUDA_MODULE_LOADING=EAGER. Later calls
 * make no allocating call (no cudaMalloc, cudaFree or allocating library routine). All calls share the one
 * array: calls that overlap on the GPU (on different streams, or from different host threads) race and must
 * be serialised by the caller. The current device must be the one holding the pointers. */
md_status md_kinetic_energy_noalloc(const double* vel3, const double* mass, int64_t n, double* out, void* stream);

/* writeXyzFrame's data (src/Trajectory.cpp:4-25) in id order: out6[6 id + k] = (x, y, z, vx, vy, vz)[k] of
 * the particle with that id, gathered through the ids on the device and copied to the host in one transfer on a
 * second stream. With wait = 0 the call returns once the copy is queued (out6 should then be pinned memory) and
 * the system's stream may keep stepping; md_system_frame_wait blocks until the copy has landed. A new frame
 * waits for the previous one's copy. */
md_status md_system_frame_by_id(md_system* s, double* out6, int wait);
md_status md_system_frame_wait(md_system* s);

/* ---- streams, timing and counters ---------------------------------------------------------------------- */
/* The cudaStream_t every call on this system is queued on (for CUDA events around calls). */
md_status md_system_stream(md_system* s, void** stream);
/* Wait for all work queued on the system's stream. */
md_status md_system_synchronize(md_system* s);
/* Kernels this system has launched so far (every kernel of this library counts one). */
md_status md_system_launch_count(const md_system* s, uint64_t* launches);
/* While enabled, md_run brackets each list force kernel with CUDA events on the system's stream;
 * md_profile_read returns their summed time (ms) and count since the last enable. */
md_status md_profile_enable(md_system* s, int enable);
md_status md_profile_read(md_system* s, double* force_ms, int64_t* force_launches);

/* ---- CellList: include/CellList.hpp:14-40, src/CellList.cpp ----------------------------------------- */
md_status md_cells_create(double min_cell_size, md_cells** out);
md_status md_cells_destroy(md_cells* c);
/* CellList::build (src/CellList.cpp:9-52) on the system's current positions (the system is not reordered). */
md_status md_cells_build(md_cells* c, md_system* s, int* cells_per_side);
/* particle_cell[n] = cellOf(i); cell_start[ncells + 1]; cell_particles[n] = sortedOrder(). Any may be NULL. */
md_status md_cells_download(md_cells* c, int* particle_cell, uint64_t* cell_start, uint64_t* cell_particles);

/* ---- NeighbourList: include/NeighbourList.hpp:15-49, src/NeighbourList.cpp -------------------------- */
/* NeighbourList(cutOff, skin, reverseIndex) (src/NeighbourList.cpp:5-8). */
md_status md_nlist_create(double cutoff, double skin, int reverse_index, md_nlist** out);
md_status md_nlist_destroy(md_nlist* nl);
/* NeighbourList::build (src/NeighbourList.cpp:55-134): sorts the system by cell (reorders it) and rebuilds. */
md_status md_nlist_build(md_nlist* nl, md_system* s);
/* NeighbourList::update (src/NeighbourList.cpp:11-36): rebuild if any particle moved more than skin/2. */
md_status md_nlist_update(md_nlist* nl, md_system* s, int* rebuilt);
/* getPairCount, getRebuildCount, the cell grid side of the last build, hasReverseIndex. Any may be NULL. */
md_status md_nlist_info(const md_nlist* nl, uint64_t* pair_count, int* rebuild_count, int* cells_per_side,
                        int* reverse_index);
/* Force kernel choice for one precision: -1 autotunes (the first force call of the list times every
 * available variant and keeps the fastest), 0 pins global gathers, 1 pins the shared-memory tile kernel (used
 * only while the list has tiles; FP64 and the float modes), 2 pins global gathers with the rows prefetched
 * (FP64: a quad of entries at a time, branch-free; float modes: a group of 8 ahead), 3 the float modes' variant 2
 * with registers capped for occupancy and 4 the same on a resident grid. MD_PREC_FX64 and MD_PREC_FX32 have one
 * kernel each (variant 0). Every variant gives the same bits. md_nlist_force_variant reports the variant in use
 * (-1 until the first force call). */
md_status md_nlist_set_force_variant(md_nlist* nl, int precision, int variant);
md_status md_nlist_force_variant(const md_nlist* nl, int precision, int* variant);
/* List build kernel: -1 uses the shared-memory tile build wherever the list has tiles, 0 pins one thread per
 * particle over global memory, 1 pins the tile build (while the list has tiles). Both write the same rows.
 * md_nlist_build_variant reports the kernel of the last build (-1 before the first). */
md_status md_nlist_set_build_variant(md_nlist* nl, int variant);
md_status md_nlist_build_variant(const md_nlist* nl, int* variant);
/* Layout of the last build (diagnostics): whether the shared-memory tile kernels are in use, the segment
 * length in cells, segments per cell column, the largest staged tile (particles) and the row capacity.
 * Any pointer may be NULL. */
md_status md_nlist_layout(const md_nlist* nl, int* use_tiles, int* segment_cells, int* segments_per_column,
                          int* max_staged, int* row_capacity);
/* The half list in the reference's CSR form: offsets[n + 1] (firstPairOf), neighbours[pairs]
 * (neighboursOf in candidate order) and, when the list has a reverse index, rev_offsets[n + 1] and
 * rev_pairs[pairs] (pairsAsSecond). Any may be NULL. */
md_status md_nlist_download(md_nlist* nl, uint64_t* offsets, uint64_t* neighbours, uint64_t* rev_offsets,
                            uint64_t* rev_pairs);
/* MD_PREC_FX32's split of the last build's rows (diagnostics; the reference has no counterpart): near_rows[n * 16]
 * and far_rows[n * row_capacity], row i's entries in order (j | cell code << 27, the sentinel j = n), groups[2 n]
 * = (near groups, far groups) of 8 entries, near2 = the squared radius that classified them. MD_ERR_STATE until
 * MD_PREC_FX32 forces have been computed on this build. Any pointer may be NULL. */
md_status md_nlist_fx32_rows(md_nlist* nl, uint32_t* near_rows, uint32_t* far_rows, int32_t* groups, double* near2);

/* ---- LennardJonesForceField: include/Forcefield.hpp:8-45, src/Forcefield.cpp ------------------------ */
/* LennardJonesForceField(epsilon, sigma, cut_off) (src/Forcefield.cpp:8-15). Precision starts at MD_PREC_FP64. */
md_status md_forcefield_create(double epsilon, double sigma, double cutoff, md_forcefield** out);
md_status md_forcefield_destroy(md_forcefield* ff);
/* getEnergyShift (include/Forcefield.hpp:21-24). */
md_status md_forcefield_shift(const md_forcefield* ff, double* shift);
/* Precision of the list path; setMixedPrecision(true) (include/Forcefield.hpp:39-41) maps to MD_PREC_FP32FX. */
md_status md_forcefield_set_precision(md_forcefield* ff, int precision);
/* setDeterministic (include/Forcefield.hpp:43-45): with it, list forces require a list built with
 * reverseIndex, as in the reference. Every precision is deterministic on the device regardless. */
md_status md_forcefield_set_deterministic(md_forcefield* ff, int deterministic);
/* computeForces(System&, const NeighbourList&) (src/Forcefield.cpp:81-326): writes the system's forces and
 * returns PE, the virial W (getVirial) and the inside-cutoff pair count (getInsidePairs). Outputs may be NULL. */
md_status md_forces_list(md_forcefield* ff, md_system* s, md_nlist* nl, double* pe, double* virial,
                         double* inside);
/* computeForces(System&), the O(N^2) path (src/Forcefield.cpp:39-78). */
md_status md_forces_all_pairs(md_forcefield* ff, md_system* s, double* pe, double* virial, double* inside);
/* getVirial / getInsidePairs (include/Forcefield.hpp:26-29): the virial and inside-cutoff pair count of the
 * force field's last evaluation, whether by md_forces_*, md_step_* or md_run. Outputs may be NULL. */
md_status md_forcefield_results(const md_forcefield* ff, double* virial, double* inside);

/* ---- VelocityVerletIntegrator: include/Integrator.hpp:9-19, src/Integrator.cpp --------------------- */
/* step(System&, const LennardJonesForceField&, NeighbourList&) (src/Integrator.cpp:18-30): half kick, drift
 * and wrap, list update, forces, half kick. Returns the new PE; `rebuilt` says whether the list was rebuilt. */
md_status md_step_list(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, double* pe, int* rebuilt);
/* step(System&, const LennardJonesForceField&) with O(N^2) forces (src/Integrator.cpp:7-16). */
md_status md_step_all_pairs(md_system* s, md_forcefield* ff, double dt, double* pe);

/* n_steps list steps (md_sim's loops, src/main.cpp:219-304). Per step, in order: step_list; then the optional
 * thermostat; then the optional g(r) sample. Outputs (each NULL or n_steps long, host memory): pe[k] the step's
 * PE, ke[k] the kinetic energy after the thermostat, virial[k].
 * On a list with shared-memory tiles a run executes as CUDA graphs of up to md_system_set_graph's chunk length
 * (64 steps by default) when it is at least two chunks long or md_run_prepare captured the graphs for its length:
 * every step, the thermostat, the g(r) sample and MD_PREC_FP64's ordered energy sums included, is in the graph,
 * and a list rebuild is decided on the device (a conditional node runs the rebuild when the half-skin test of the
 * step's drift flagged a particle), so the host waits once per chunk. A rebuild that outgrows the row capacity,
 * the recorded shared-memory tile or (MD_PREC_FP64) the energy records' buffers makes the library run that chunk
 * again on the host path from the chunk's starting state, growing what it must; results are the same bits either
 * way. MD_PREC_FP64 systems of more than 10^6 particles (whose ordered energy sums overlap the next steps better
 * on their own streams), small boxes and lists pinned to the global build take the host-driven loop, which reads
 * the half-skin flag after each drift. */
typedef struct md_run_options {
    int thermostat;             /* 0 none (NVE), 1 rescale, 2 Bussi */
    int rescale_every;          /* rescale when (first_step + k) % rescale_every == 0 */
    double rescale_temperature; /* target of the rescale */
    int melt_until;             /* rescale to melt_temperature instead while first_step + k <= melt_until */
    double melt_temperature;
    double bussi_temperature;   /* Bussi target temperature */
    double bussi_tau;           /* coupling time; c = exp(-dt / tau) as in src/Thermostat.cpp:46 */
    const double* bussi_r1;     /* n_steps draws (host), e.g. from md_bussi_noise */
    const double* bussi_chi2;
    md_rdf* rdf;                /* sample g(r) when (first_step + k) % rdf_every == 0 (NULL: never) */
    int rdf_every;
    int64_t first_step;         /* step number of the first step of this run (1-based, as md_sim counts) */
} md_run_options;
md_status md_run(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                 const md_run_options* opts, double* pe, double* ke, double* virial);
/* Capture and instantiate the graphs md_run would launch for the same arguments, without running a step (graph
 * set-up stays out of a timed run). record: bit 0 when pe or virial will be requested, bit 1 when ke will. */
md_status md_run_prepare(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                         const md_run_options* opts, int record);
/* md_run's graph chunk length (1..1024 steps; 0 runs every step from the host) and test flags:
 * MD_GRAPH_TEST_RERUN makes every list rebuild on the device report an overflow, so that each chunk with a rebuild
 * reruns on the host path from its starting state (for tests of that path; the results are the same bits).
 * Drops the system's cached graphs. */
#define MD_GRAPH_TEST_RERUN 1
md_status md_system_set_graph(md_system* s, int chunk_steps, int flags);
/* Graph chunk length, graphs cached, chunk graphs launched and chunks rerun on the host path. Any may be NULL. */
md_status md_system_graph_info(const md_system* s, int* chunk_steps, uint64_t* graphs, uint64_t* launches,
                               uint64_t* recoveries);

/* ---- RadialDistribution: include/RadialDistribution.hpp:10-20, src/RadialDistribution.cpp ----------- */
md_status md_rdf_create(double r_max, int bins, md_rdf** out);
md_status md_rdf_destroy(md_rdf* r);
/* RadialDistribution::sample (src/RadialDistribution.cpp:11-30) over the list's half pairs. */
md_status md_rdf_sample(md_rdf* r, md_system* s, md_nlist* nl);
/* radii (src/RadialDistribution.cpp:32-38) and values (:42-54); either may be NULL; bins long. */
md_status md_rdf_values(md_rdf* r, double* radii, double* g, int* samples);
/* The raw histogram of pair counts (bins long). */
md_status md_rdf_histogram(md_rdf* r, double* hist);

/* ---- batched replicas ----------------------------------------------------------------------------------
 * Many independent systems of uneven size, density and temperature advanced together: each replica follows
 * the reference's single-system step on its own box (System + NeighbourList(r_c, skin, true) +
 * LennardJonesForceField with setDeterministic(true) in FP64 + VelocityVerletIntegrator::step + the thermostat,
 * src/Integrator.cpp:18-30, src/Thermostat.cpp:17-58), with the same bits as that replica run alone through
 * md_system/md_nlist/md_run. The reference has no batched interface; this one replaces a loop over systems.
 * Rebuilds are decided per replica on the device, and a run executes as CUDA graphs of chunk_steps steps. */
typedef struct md_batch md_batch;

typedef struct md_batch_options {
    double epsilon, sigma, cutoff, skin, dt; /* shared by all replicas */
    int precision;        /* md_precision */
    int thermostat;       /* 0 none (NVE), 1 rescaleVelocities to each replica's temperature every rescale_every
                             steps of a run, 2 Bussi with bussi_tau, drawing per replica like md_bussi_noise */
    int rescale_every;
    double bussi_tau;
    int energy_every;     /* record potential energy, virial and kinetic energy (after the thermostat) of every
                             replica at every energy_every-th step of a run; 0 records nothing */
    int chunk_steps;      /* steps per CUDA graph (0: 100), rounded up to a multiple of the thermostat and
                             sampling periods */
    int initial_capacity; /* neighbour row capacity (0: estimated from the densest replica); grown on demand */
} md_batch_options;

/* replicas systems; replica r has n_atoms[r] particles in a box of side box_length[r], target temperature
 * temperature[r] (thermostats only) and Bussi seed seeds[r] (thermostat 2 only). pos4, vel3 and mass are the
 * replicas' reference arrays concatenated in replica order: 4 n (x, y, z, pad) positions, 3 n component-major
 * velocities per replica ([vx(n), vy(n), vz(n)]), n masses (NULL: 1). ids start as 0 .. n-1 per replica.
 * The list is built and the starting forces computed from it. */
md_status md_batch_create(int device, int replicas, const int64_t* n_atoms, const double* box_length,
                          const double* temperature, const uint64_t* seeds, const double* pos4, const double* vel3,
                          const double* mass, const md_batch_options* opts, md_batch** out);
md_status md_batch_destroy(md_batch* b);
/* Replicas, particles (sum of n), neighbour row capacity, kernels launched so far. Any may be NULL. */
md_status md_batch_info(const md_batch* b, int* replicas, int64_t* atoms, int* capacity, uint64_t* launches);
md_status md_batch_stream(md_batch* b, void** stream);
/* n_steps steps of every replica. With energy_every = k, row s of the records (replica r at [s * replicas + r])
 * is step (s + 1) k of this run; arrays hold n_steps / k rows each and may be NULL. */
md_status md_batch_run(md_batch* b, int64_t n_steps, double* pe, double* virial, double* ke);
/* md_batch_run that also records each sampled step's inside-cutoff pair count (getInsidePairs,
 * include/Forcefield.hpp:26-29) into inside (same layout; NULL to skip): the count that converts the shifted
 * potential energy to the unshifted one, as bench/validate.py:114-120 of the reference does. */
md_status md_batch_run_records(md_batch* b, int64_t n_steps, double* pe, double* virial, double* ke, double* inside);
/* Change the thermostat between runs (a protocol of phases, e.g. bench/validate.py:96-111's melt, cool and NVT
 * production): thermostat 0 none, 1 rescale every rescale_every steps to temperature[r], 2 Bussi with coupling
 * time bussi_tau at temperature[r], each replica's generator started afresh from seeds[r] (a new
 * BussiThermostat, src/Thermostat.cpp:36-44). temperature may be NULL to keep the targets (thermostat 0 needs
 * none). Steps of the next run are numbered from 1 again. */
md_status md_batch_set_thermostat(md_batch* b, int thermostat, int rescale_every, double bussi_tau,
                                  const double* temperature, const uint64_t* seeds);
/* Potential energy, virial, inside-cutoff pair count and kinetic energy of each replica's current state
 * (replicas entries each; any may be NULL). */
md_status md_batch_energy(md_batch* b, double* pe, double* virial, double* ke, double* inside);
/* One replica's arrays in the reference's layout (as md_system_download). Any output may be NULL. */
md_status md_batch_download(md_batch* b, int replica, double* pos4, double* vel3, double* force3, double* mass,
                            uint64_t* ids);
/* System::stateHash of every replica (src/System.cpp:85-105) into hashes[replicas]. */
md_status md_batch_state_hash(md_batch* b, uint64_t* hashes);
/* NeighbourList::getRebuildCount of every replica (the first build included) into rebuilds[replicas]. */
md_status md_batch_rebuilds(md_batch* b, uint64_t* rebuilds);
/* Force kernel shape: variant -1 autotunes (times every shape and keeps the fastest; done at creation), else
 * pins one. md_batch_force_variant reports the variant in use, how many there are, and its particles per block
 * and threads per particle. Every variant gives the same bits. */
md_status md_batch_set_force_variant(md_batch* b, int variant);
md_status md_batch_force_variant(const md_batch* b, int* variant, int* count, int* particles_per_block,
                                 int* threads_per_particle);
/* Average device time (ms) of the list force kernel alone over reps launches, CUDA events on the batch stream. */
md_status md_batch_time_forces(md_batch* b, int reps, double* ms);

/* ---- trajectory adjoint --------------------------------------------------------------------------------
 * Gradients of J = g_pe * mean_k U_k + g_pressure * mean_k P_k over an NVE velocity-Verlet trajectory of
 * `steps` steps (k = 1..steps; P = (2 KE + W) / 3V, W the virial) with respect to epsilon, sigma and the
 * initial positions and velocities. The reference has no adjoint; its step (src/Integrator.cpp:18-71), pair
 * terms (src/Forcefield.cpp:25-36) and list rule (src/NeighbourList.cpp:11-134) define the trajectory, in FP64,
 * with the particles kept in their input order. Checkpoints every checkpoint_every steps; the backward pass
 * recomputes each segment from its checkpoint. forward/backward have torch.autograd.Function semantics: forward
 * returns (mean U, mean P), backward takes their cotangents. */
typedef struct md_adjoint md_adjoint;

md_status md_adjoint_create(int device, int64_t n, double box_length, const double* pos4, const double* vel3,
                            const double* mass, double epsilon, double sigma, double cutoff, double skin, double dt,
                            int steps, int checkpoint_every, md_adjoint** out);
md_status md_adjoint_destroy(md_adjoint* a);
/* New epsilon and sigma, or a new initial state (pos4 / vel3 may be NULL to keep one); forward must follow. */
md_status md_adjoint_set_parameters(md_adjoint* a, double epsilon, double sigma);
md_status md_adjoint_set_state(md_adjoint* a, const double* pos4, const double* vel3);
/* Runs the trajectory: mean U and mean P, and optionally U_k, W_k, KE_k for k = 1..steps (arrays of steps). */
md_status md_adjoint_forward(md_adjoint* a, double* mean_pe, double* mean_pressure, double* pe_steps, double* w_steps,
                             double* ke_steps);
/* dJ/d epsilon, dJ/d sigma, dJ/d initial positions and velocities (3 x n component-major; NULL to skip) for the
 * cotangents (g_pe, g_pressure) of the last forward's outputs. */
md_status md_adjoint_backward(md_adjoint* a, double g_pe, double g_pressure, double* d_epsilon, double* d_sigma,
                              double* d_pos3, double* d_vel3);
/* Particles, steps, checkpoint interval, list builds of the last forward (the first included), kernels launched. */
md_status md_adjoint_info(const md_adjoint* a, int64_t* n, int* steps, int* checkpoint_every, int* rebuilds,
                          uint64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* MD_B200_H */
