/*
 * cellgpu_b200 -- C ABI of the B200 (sm_100a) implementation of cellGPU's per-timestep hot path.
 *
 * Two layers, both plain C (extern "C", plain pointers and sizes, int status codes, no exceptions):
 *
 *  1. Kernel callers on caller-owned device memory. These replace the reference's L1 "gpu_*" free
 *     functions (the .cuh headers of inc/models, inc/updaters and inc/utility), which take raw device
 *     pointers obtained from ArrayHandle<T>(..., access_location::device, ...). Each takes a
 *     cudaStream_t (0 = legacy default stream, as the reference used) and never allocates unless
 *     its comment says so.
 *  2. An opaque, device-resident system handle (cg_system) that owns one batch of independent
 *     monolayers (a single monolayer is a batch of one) and runs whole timesteps, FIRE minimizations
 *     and topology maintenance without per-step host round trips. It replaces the GPU branches of the
 *     reference's model/updater classes (Simple2DCell, voronoiModelBase, VoronoiQuadraticEnergy,
 *     vertexModelBase, VertexQuadraticEnergy, selfPropelledParticleDynamics,
 *     brownianParticleDynamics, EnergyMinimizerFIRE).
 *
 * Layouts follow the reference: positions are interleaved (x, y) doubles (Dscalar2 = double2,
 * inc/std_include.h:47-60); neighbour rows are per-cell contiguous, n_idx(k, c) = c*K + k
 * (inc/utility/indexer.h:38-41), counter-clockwise. Boxes are rectangular (Lx, Ly), as gpubox's
 * setSquare(x, y) (inc/utility/gpubox.h:83-93).
 *
 * Calls on one cg_system are not thread-safe; distinct systems may be used from distinct threads.
 */
#ifndef CELLGPU_B200_H
#define CELLGPU_B200_H

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------- */
#define CG_OK 0
#define CG_ERR_CUDA (-1)          /* a CUDA call failed; cg_last_error_string() has the text */
#define CG_ERR_ARG (-2)           /* invalid argument */
#define CG_ERR_CAPACITY (-3)      /* a neighbour/vertex row exceeded its capacity; regrow needed */
#define CG_ERR_TOPOLOGY (-4)      /* the triangulation could not be made consistent */
#define CG_ERR_TIMEOUT (-5)       /* a bounded device wait gave up */
#define CG_ERR_STATE (-6)         /* call not valid in the current state */

/* precision modes */
#define CG_FP64 0   /* plain FP64: the drop-in for the reference's Dscalar = double path */
#define CG_MIXED 1  /* FP32 geometry/forces relative to each cell, FP64 positions and predicates */

/* model kinds */
#define CG_MODEL_VORONOI 0
#define CG_MODEL_VERTEX 1

const char *cg_last_error_string(void);
int cg_version(void);

/* =========================================================================================
 * 1. Kernel callers (caller-owned device memory)
 * ========================================================================================= */

/* Voronoi geometry: area and perimeter of every cell's Voronoi polygon.
 * Replaces gpu_compute_voronoi_geometry (inc/models/voronoiModelBase.cuh:35-48,
 * src/models/voronoiModelBase.cu:115-201); the per-slot voroCur/voroLastNext scratch of the
 * reference is not materialised. AP[c] = (A, P). */
int cg_voronoi_geometry(const double *pos, const int *nn, const int *nbr, int K, int N, double Lx,
                        double Ly, double *AP, cudaStream_t stream);

/* Voronoi quadratic-energy forces, geometry included (one fused pass).
 * Replaces gpu_compute_voronoi_geometry + gpu_force_sets + gpu_sum_force_sets
 * (inc/models/voronoiQuadraticEnergy.cuh:20-54). F must be zeroed by the caller (forces are
 * accumulated with FP64 atomics, so the last bits of F can vary between calls; systems offer
 * order-independent sums, cg_set_deterministic); AP receives (A, P). APpref[c] = (A0, P0); KA, KP
 * are the uniform moduli the reference uses (inc/models/Simple2DCell.h:272-274). */
int cg_voronoi_forces(const double *pos, const int *nn, const int *nbr, int K, int N, double Lx,
                      double Ly, const double *APpref, double KA, double KP, double *AP, double *F,
                      cudaStream_t stream);

/* Exact local-Delaunay test of a stored triangulation: every triangle counter-clockwise and every
 * edge locally Delaunay. Cells touching a failing edge get flag[c] = 1 (flag is not cleared);
 * *any_fail is set to 1 if anything failed. Same role as gpu_test_circumcenters
 * (inc/models/voronoiModelBase.cuh:20-33) with exact predicates. */
int cg_voronoi_test_triangulation(const double *pos, const int *nn, const int *nbr, int K, int N,
                                  double Lx, double Ly, int *flag, int *any_fail, cudaStream_t stream);

/* Self-propelled particle step, CPU semantics of the reference
 * (src/updaters/selfPropelledParticleDynamics.cpp:67-101), fused with the move-and-wrap of
 * gpu_move_degrees_of_freedom (inc/models/Simple2DCell.cuh:22-40):
 *   v = v0 (cos th, sin th); pos <- wrap(pos + dt (v + mu F)); th <- atan2(v) + xi sqrt(2 dt Dr).
 * noise: one normal per cell (device pointer), or NULL to draw from the counter-based RNG with
 * (seed, step). motility[c] = (v0, Dr). Replaces gpu_spp_eom_integration
 * (inc/updaters/selfPropelledParticleDynamics.cuh:17-27). */
int cg_spp_step(double *pos, double *theta, const double *F, const double *motility, const double *noise,
                int N, double Lx, double Ly, double dt, double mu, uint64_t seed, uint32_t step,
                cudaStream_t stream);

/* Periodic Delaunay triangulation of N points on the device (exact predicates), written as
 * counter-clockwise neighbour rows that start at the smallest neighbour index. Replaces the CPU/CGAL
 * voronoiModelBase::globalTriangulationCGAL (src/models/voronoiModelBase.cpp:281-351).
 * Allocates and frees its own scratch (cell list, candidate buffers). The rows are the caller's, of
 * capacity K: a cell with more than K neighbours returns CG_ERR_CAPACITY (retry with a larger K,
 * as the reference grows neighMax). Synchronous: returns once the rows are written. */
int cg_voronoi_triangulate(const double *pos, int N, double Lx, double Ly, int K, int *nn, int *nbr,
                           cudaStream_t stream);

/* Allocation-free variant of cg_voronoi_triangulate. No counterpart in the reference: it exists
 * for callers that must not allocate device memory -- applications that give the library a fixed
 * device-memory budget up front (another framework's caching allocator owns the heap), loops where
 * cudaFree's implicit device synchronisation would stall every other stream, and host threads that
 * run while another thread captures a CUDA graph in global mode (cudaMalloc is illegal for every
 * thread then; call this on a cudaStreamNonBlocking stream, since the legacy default stream
 * synchronises with the capturing stream). Its scratch is a file-scope __device__ array of fixed
 * size (about 2.9 MB) that each GPU loading this library keeps until the process exits; inputs and
 * outputs remain the caller's. Limits: N <= CG_NOALLOC_MAX_CELLS and at most CG_NOALLOC_MAX_BINS
 * cell-list bins (about 1.56 bins per unit of box area); larger inputs get CG_ERR_CAPACITY, and so
 * does a cell with more than K neighbours. The call is synchronous: it waits on `stream` for the
 * status words, so it cannot itself be captured into a graph. Its first call on a device resolves
 * the array's address with cudaGetSymbolAddress (with that device current). All calls share the
 * array (each clears what must start at zero): calls that overlap on the GPU race, so serialise
 * them. Calls no cudaMalloc, cudaFree or allocating library routine. */
#define CG_NOALLOC_MAX_CELLS 65536
#define CG_NOALLOC_MAX_BINS 131072
int cg_voronoi_triangulate_noalloc(const double *pos, int N, double Lx, double Ly, int K, int *nn, int *nbr,
                                   cudaStream_t stream);

/* =========================================================================================
 * 2. Device-resident systems (batched; a single instance is the plain drop-in)
 * ========================================================================================= */
typedef struct cg_system cg_system;

/* Create a batch of n_inst Voronoi monolayers with N[i] cells in boxes (box[2i], box[2i+1]).
 * K is the neighbour-row capacity, a multiple of 4 up to 32; 16 covers nearly every cell of random
 * points. A cell with more than K neighbours makes the system widen its rows to 32 (the reference
 * grows neighMax the same way); cg_neighbor_capacity reports the current K.
 * precision: CG_FP64 or CG_MIXED. */
int cg_voronoi_create(int n_inst, const int *N, const double *box, int K, int precision,
                      cg_system **out);
/* Vertex model batch: n_inst monolayers with Nc[i] cells and Nv[i] = 2*Nc[i] three-valent vertices;
 * vmax is the vertex-row capacity per cell (the reference fixes 30,
 * src/models/vertexModelBase.cpp:209-210). FP64 only. Initialise with cg_vertex_from_voronoi or
 * cg_set_positions + cg_set_vertex_topology. */
int cg_vertex_create(int n_inst, const int *Nc, const double *box, int vmax, int precision,
                     cg_system **out);
int cg_destroy(cg_system *sys);

/* sizes and footprint */
int cg_num_cells(const cg_system *sys);
int cg_num_dofs(const cg_system *sys);      /* cells (Voronoi) or vertices (vertex model) */
int cg_num_instances(const cg_system *sys);
int cg_neighbor_capacity(const cg_system *sys);
size_t cg_device_bytes(const cg_system *sys);
/* bytes a system of this shape would hold on the device (admission control) */
size_t cg_voronoi_footprint(int n_inst, const int *N, int K);
size_t cg_vertex_footprint(int n_inst, const int *Nc, int vmax);
/* free and total device memory of the current device (admission budgets) */
int cg_device_memory(size_t *free_bytes, size_t *total_bytes);

/* host <-> device state (host buffers; copies are ordered on the system's stream and complete
 * before return for get_*) */
int cg_set_positions(cg_system *sys, const double *pos);     /* cells (Voronoi) / vertices (vertex) */
int cg_get_positions(cg_system *sys, double *pos);
int cg_set_cell_preferences(cg_system *sys, const double *APpref); /* (A0, P0) per cell */
int cg_set_moduli(cg_system *sys, double KA, double KP);
int cg_set_motility(cg_system *sys, const double *motility);  /* (v0, Dr) per cell */
int cg_set_directors(cg_system *sys, const double *theta);
int cg_get_directors(cg_system *sys, double *theta);
int cg_get_forces(cg_system *sys, double *F);                 /* per dof */
int cg_get_area_perimeter(cg_system *sys, double *AP);        /* per cell */
int cg_get_topology(cg_system *sys, int *nn, int *nbr);       /* Voronoi rows (N x cg_neighbor_capacity) */
int cg_set_topology(cg_system *sys, const int *nn, const int *nbr);
/* vertex model wiring (vertexModelBase arrays, inc/models/Simple2DCell.h:160-290): vn[3*Nv] vertex
 * neighbours, vcn[3*Nv] cells of each vertex, cvn[Nc] vertices per cell, cv[Nc*vmax] cell vertices
 * counter-clockwise */
int cg_get_vertex_topology(cg_system *sys, int *vn, int *vcn, int *cvn, int *cv);
int cg_set_vertex_topology(cg_system *sys, const int *vn, const int *vcn, const int *cvn, const int *cv);
/* per-instance energies E = sum KA (A-A0)^2 + KP (P-P0)^2 (computeEnergy,
 * src/models/voronoiQuadraticEnergy.cpp:384-397), accumulated in FP64 */
int cg_get_energies(cg_system *sys, double *E);
/* the stream the system enqueues on (its own non-blocking stream unless set; NULL restores it).
 * CUDA graphs are captured on it, so it must not be the legacy default stream. */
int cg_set_stream(cg_system *sys, cudaStream_t stream);
cudaStream_t cg_get_stream(cg_system *sys);
int cg_synchronize(cg_system *sys);

/* topology and forces */
int cg_triangulate(cg_system *sys);       /* full Delaunay triangulation (Voronoi) */
/* vertex model from the Delaunay triangulation of cell positions (Nc points, (x,y) pairs): one
 * vertex per Delaunay triangle at its circumcentre (vertexModelBase::setCellsVoronoiTesselation,
 * src/models/vertexModelBase.cpp:115-229) */
int cg_vertex_from_voronoi(cg_system *vertex_sys, const double *cell_pos);
int cg_compute_forces(cg_system *sys);    /* forces on the current topology, geometry included */
int cg_enforce_topology(cg_system *sys);  /* Voronoi: test+repair; vertex: T1 sweep */

/* dynamics: n_steps integrator steps, each = forces, integrate, move, topology.
 * noise == NULL: counter-based RNG with the system seed; else a device pointer with n_steps blocks of
 * per-step normals (SPP: N per step; Brownian: 2*Nv per step). */
/* Device noise: instance i draws with Philox key seed_i and counters made of its local cell (or
 * vertex) index and the step, so its noise does not depend on where it sits in a batch.
 * cg_set_seed sets seed_i = SplitMix64(seed, i) (also the default, seed = 0x5eed);
 * cg_set_instance_seeds sets every seed_i explicitly (n_inst values). */
int cg_set_seed(cg_system *sys, uint64_t seed);
int cg_set_instance_seeds(cg_system *sys, const uint64_t *seeds);
/* Deterministic force sums (the reference's kernels sum each cell's force sets in a fixed order,
 * src/models/voronoiQuadraticEnergy.cu:30-54; Simulation::setReproducible maps here). Off (the
 * default): floating-point atomics, whose order varies, so reruns agree only to rounding and a
 * chaotic trajectory then drifts apart. On: forces are summed in fixed point with integer atomics,
 * exact in any order, so the same inputs give bit-identical forces and trajectories. Four 64-bit
 * words per component: contributions below 2 in magnitude go to one word of 2^-56 units, larger
 * ones (any finite value below 2^98; beyond that the cell's force is NaN) to three words of 2^-64
 * resolution.
 * FIRE's per-instance power and norm sums are then taken in a fixed order (per-block partials
 * joined by one block per instance) instead of with atomics. Allocates 64 bytes per cell (Voronoi)
 * or vertex (vertex model) on first use; drops captured graphs. Both models. */
int cg_set_deterministic(cg_system *sys, int on);
int cg_get_deterministic(cg_system *sys);
int cg_spp_run(cg_system *sys, int n_steps, double dt, double mu, const double *noise_dev);
/* Enqueue n_steps RNG-driven SPP steps (one CUDA graph replay) with no host synchronisation.
 * A step that cannot finish on the device (a global rebuild is needed) sets a sticky halt flag and
 * the remaining enqueued steps do nothing; cg_poll reports completed steps and recovers. */
int cg_spp_enqueue(cg_system *sys, int n_steps, double dt, double mu);
int cg_poll(cg_system *sys, int *steps_done, int *halted, int recover_if_halted);
/* One step through host buffers: host_noise (N normals) is copied in, the per-instance energies of
 * the step's force evaluation (the configuration at the start of the step) are copied out to
 * host_energy (may be NULL); returns when they are available. */
int cg_spp_step_host(cg_system *sys, const double *host_noise, double dt, double mu, double *host_energy);
/* The same step, asynchronous: host_noise (N normals; pinned memory, or the copy is staged by the
 * driver) is copied on the system's copy stream into one of two device buffers, so the copy for the
 * next step overlaps this one; the step waits for its copy; host_energy (may be NULL) receives the
 * per-instance energies (page-locked host memory is written directly by the reduction kernel, other
 * memory through a device-to-host copy). Nothing is synchronised: both host buffers must stay
 * untouched until the step has completed (cg_poll, cg_synchronize, or an event recorded on the
 * system stream). Energies are those of cg_spp_step_host. Halts behave as for cg_spp_enqueue. */
int cg_spp_enqueue_host(cg_system *sys, const double *host_noise, double dt, double mu, double *host_energy);
/* The fused geometry + force (+ exact Delaunay test) pass alone, enqueued without synchronisation. */
int cg_launch_force_pass(cg_system *sys, int with_test);
/* number of this library's kernels launched for the system so far, graph replays and the repair
 * rounds run inside graph conditional nodes included (synchronises the system's stream) */
long long cg_kernels_launched(cg_system *sys);

/* Brownian dynamics of the vertex model (brownianParticleDynamics, src/updaters/
 * brownianParticleDynamics.cpp:92-109): two normals per vertex and step (x then y); noise_dev holds
 * n_steps*2*Nv normals or is NULL for the counter-based RNG. Each step: forces, integrate + move,
 * T1 sweep. */
int cg_brownian_run(cg_system *sys, int n_steps, double dt, double mu, double T, const double *noise_dev);
/* self-propelled vertex model (selfPropelledCellVertexDynamics, src/updaters/
 * selfPropelledCellVertexDynamics.cpp:81-122): noise_dev holds n_steps*Nc normals or NULL */
int cg_vertex_spp_run(cg_system *sys, int n_steps, double dt, double mu, const double *noise_dev);
/* T1 edge-length threshold (vertexModelBase::setT1Threshold; default 0.01) */
int cg_set_t1_threshold(cg_system *sys, double threshold);

/* FIRE minimisation (EnergyMinimizerFIRE::minimize, src/updaters/EnergyMinimizerFIRE2D.cpp:269-284)
 * with the CPU conventions of the reference (forceMax = max |F|^2; dt >= dt_min), every instance
 * independently (its own dt, alpha, counters). Each call starts a fresh minimisation (zero
 * velocities, dt, alpha_start). Defaults of the reference (:24-41): dt 0.01, dt_max 0.1,
 * dt_min 0.01*dt, dt_inc 1.05, dt_dec 0.95, alpha_start 0.99, alpha_dec 0.9, n_min 5,
 * force_cutoff 1e-7, max_iterations 1000. */
typedef struct {
    double dt, dt_max, dt_min, dt_inc, dt_dec, alpha_start, alpha_dec, force_cutoff;
    int n_min, max_iterations;
} cg_fire_params;
int cg_fire_minimize(cg_system *sys, const cg_fire_params *prm);
/* The same minimisation in pieces (EnergyMinimizerFIRE::minimize split at its loop head): cg_fire_begin
 * starts it (fresh per-instance state, forces of the current positions); cg_fire_advance runs up to
 * `iterations` more iterations, or until every instance has stopped (converged or at max_iterations;
 * *n_stopped receives their number, may be NULL). Stopped instances stay frozen, so a caller can
 * read an instance's result as soon as it stops while the others continue; pieces with the same
 * parameters give the same result as one cg_fire_minimize call. No counterpart in the reference
 * (its minimize runs to the end in one call); the serving loop uses it to return results early. */
int cg_fire_begin(cg_system *sys, const cg_fire_params *prm);
int cg_fire_advance(cg_system *sys, const cg_fire_params *prm, int iterations, int *n_stopped);
/* Fresh FIRE state for instances [first, first + count) only (the others keep theirs) and the forces
 * of the current state: instances admitted into a serving batch beside instances that are already
 * minimising. No counterpart in the reference. */
int cg_fire_begin_instances(cg_system *sys, const cg_fire_params *prm, int first, int count);

/* Continuous batching (no counterpart in the reference, which runs one monolayer per process): copy
 * the whole state of instances [src_first, src_first + count) of src into instances
 * [dst_first, dst_first + count) of dst -- positions, directors, preferences, motility, forces,
 * areas and perimeters, topology (relabelled to dst's indices), FIRE velocities and per-instance
 * FIRE state, cell types, exclusions, noise keys and step counts -- so they continue in dst exactly
 * where they stopped in src (the noise of an instance is keyed by its own seed and step count, not by
 * the system it runs in). Both systems must have the same model, precision, summation mode (and
 * vmax), and the instances the same sizes and boxes. Synchronises src's and dst's streams. */
int cg_copy_instances(cg_system *dst, int dst_first, cg_system *src, int src_first, int count);
/* per instance: iterations, sqrt(max |F|^2) (CPU convention) and sqrt(mean |F|^2) (the reference's
 * GPU convention, src/updaters/EnergyMinimizerFIRE2D.cpp:184) of the last iteration */
int cg_fire_state(cg_system *sys, int *iterations, double *fmax_cpu, double *fnorm_gpu);

/* Snapshots and exact resume. No counterpart in the reference, whose state files (netCDF,
 * src/databases/DatabaseNetCDFSPV.cpp:32-46, DatabaseNetCDFAVM.cpp:33-52) store no RNG state.
 * cg_snapshot writes the whole state of a system (instances with their boxes and noise keys,
 * positions, directors, motility, preferences, moduli, topology or vertex wiring, T1 threshold,
 * step counter) into a host buffer of cg_snapshot_size bytes; cg_restore builds a new system from
 * it. Device noise is keyed per instance and counted by step and local index, so the restored
 * system continues the original trajectory: bit for bit in the deterministic mode (recorded in
 * the snapshot and switched on by cg_restore), else up to the summation order of atomics. FIRE
 * velocities and derived quantities (forces, A/P) are not stored. */
size_t cg_snapshot_size(cg_system *sys);
int cg_snapshot(cg_system *sys, void *buf, size_t bytes);
int cg_restore(const void *buf, size_t bytes, cg_system **out);
/* instance sizes (cells) and boxes (Lx, Ly), n_inst entries each; model kind and precision */
int cg_get_instances(cg_system *sys, int *N, double *box);
int cg_model_kind(cg_system *sys);
int cg_precision(cg_system *sys);

/* Observables per instance, computed on the device. Shape statistics from the stored areas and
 * perimeters (those of the last force evaluation), as Simple2DCell::reportq / reportVarq /
 * reportMeanP / reportVarAP (src/models/Simple2DCell.cpp:699-765); mean squared displacement and
 * overlap function (fraction with minimum-image displacement < cutoff) as dynamicalFeatures
 * (src/analysis/dynamicalFeatures.cpp:17-50) against the positions captured by
 * cg_set_reference_positions (cells for the Voronoi model, vertices for the vertex model).
 * out: n_inst records of CG_OBS_FIELDS doubles: mean q, var q, mean A, mean P, var A, var P,
 * MSD, overlap (the last two NaN before any reference is set). */
#define CG_OBS_FIELDS 8
int cg_set_reference_positions(cg_system *sys);
int cg_observables(cg_system *sys, double cutoff, double *out);

/* Spatial re-sorting of a Voronoi batch (Simple2DCell::spatiallySortCells,
 * src/models/Simple2DCell.cpp:438-477): the cells of every instance are reordered along a Hilbert
 * curve over its box, so that neighbours sit near each other in memory. Every per-cell array and
 * the neighbour rows move with their cells (rows keep their smallest-neighbour-first rotation);
 * cells stay inside their instance's index range. cg_get_tags gives, for every current index, the
 * index the cell had when the system was created (the reference's idxToTag). */
int cg_spatial_sort(cg_system *sys);
int cg_get_tags(cg_system *sys, int *idx_to_tag);

/* Line tension (VoronoiQuadraticEnergyWithTension, src/models/voronoiQuadraticEnergyWithTension.cpp;
 * VertexQuadraticEnergyWithTension, src/models/vertexQuadraticEnergyWithTension.cpp;
 * Simple2DCell::setCellType): cells carry a type (>= 0, all 0 by default); every edge between
 * cells of different types carries gamma per unit length (cg_set_tension: setSurfaceTension(g); 0
 * switches tension off) or gamma[type_self * ntypes + type_other] (cg_set_tension_matrix:
 * setSurfaceTension(vector), a symmetric ntypes x ntypes matrix, CG_ERR_ARG otherwise; ntypes = 0
 * switches it off). Forces are the reference's: in the Voronoi model each cell's terms count its
 * unlike edges, in the vertex model each force set adds the edge to its cell's next vertex.
 * cg_get_energies counts each unlike edge once (the reference's Voronoi computeEnergy; the vertex
 * model's is unimplemented there, and this is the energy its forces are the gradient of). Both
 * models. */
int cg_set_cell_types(cg_system *sys, const int *types);
int cg_set_tension(cg_system *sys, double gamma);
int cg_set_tension_matrix(cg_system *sys, int ntypes, const double *gamma);

/* Particle exclusions (voronoiModelBase::setExclusions, src/models/voronoiModelBase.cpp:85-104, and
 * the force summation with exclusions, gpu_sum_force_sets_with_exclusions,
 * inc/models/voronoiQuadraticEnergy.cuh:41-54 / src/models/voronoiQuadraticEnergy.cpp:119-135,
 * 368-377): cells with excluded[c] != 0 get zero motility (v0 = Dr = 0) now, and after every force
 * evaluation their net force F is stored as the external force -F and F is set to 0, so they
 * neither self-propel nor respond to forces. excluded = NULL clears every flag (motility is left as
 * it is, as in the reference). The flags move with their cells under spatial sorting and are kept
 * in snapshots. cg_get_external_forces copies the external forces, (x, y) per cell (0 for cells
 * that are not excluded), to a host buffer of 2N doubles. Voronoi systems only. */
int cg_set_exclusions(cg_system *sys, const int *excluded);
int cg_get_external_forces(cg_system *sys, double *out);

/* Autotuner (no counterpart in the reference): times the runtime-selectable launch parameters on
 * the system's current state and keeps the fastest -- the fused force pass's launch shape (0: 8-lane
 * groups, 2 warps per block; 1: groups, 4 warps per block; 2: one thread per cell, timed only where
 * it applies: FP64 with atomic sums, no line tension, 16-slot rows) and the global triangulation's
 * cell-list bin side (0: 0.8, 1: 1.0, 2: 1.25 mean cell spacings). A new system starts with shape 2
 * where it applies, else shape 0. times_ms (6 values: force pass per shape, 0 for a shape not
 * timed; triangulation per bin side) and choice (2 values) may be NULL. Voronoi systems only (a no-op
 * for the vertex model). */
int cg_autotune(cg_system *sys, double *times_ms, int *choice);

/* Repair-launch autotuner (no counterpart in the reference): times the grids of the local repair
 * round's two launches (k_star_local: 148 x 5 or 148 x 2 blocks; k_commit_check: 148 x 4, 8 or 16)
 * on real SPP steps with device noise, `steps` steps twice per pair, and keeps the fastest. The
 * system ADVANCES by 12 x steps steps (run it in place of equilibration steps). The repair queues
 * hold every cell per round and cannot overflow, so they have no capacity to tune. times_ms (6
 * values, ms per step, star grid major) and choice (the two grids) may be NULL. Voronoi systems only
 * (a no-op for the vertex model). */
int cg_autotune_repair(cg_system *sys, int steps, double dt, double mu, double *times_ms, int *choice);

/* counters: topology repairs, global retriangulations, T1 flips, fallbacks (per system) */
int cg_counters(cg_system *sys, long long *out, int n);

#ifdef __cplusplus
}
#endif
#endif
