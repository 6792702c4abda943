/*
 * nsfsi.h -- C ABI of the B200 (sm_100a) time-marching path for the 3D-NS-FSI compressible
 * Navier-Stokes solver. Plain C types only; every call returns an nsf_status (0 = success).
 *
 * The reference (Frederik-Kris/3D-NS-FSI) is a pure C++ program with no foreign-function interface.
 * Each entry point below replaces one piece of its C++ call surface, cited as path:line in the
 * reference project; the C++ host classes in 3d-ns-fsi_b200/host/nsfsi_host.hpp (ConfigSettings, Solver,
 * Mesh, OutputManager, Simulation) are re-expressed on top of these calls.
 *
 * Memory model: the solver handle owns all device memory (allocated in nsf_create / nsf_initialize,
 * freed in nsf_destroy) and one CUDA stream. Fields stay resident in HBM in the reference's SoA layout
 * (one array per variable, index i*NJ*NK + j*NK + k, k fastest). Host buffers passed to the download /
 * upload calls belong to the caller. No device pointer escapes through this interface.
 * Threading: calls on one handle must be serialised by the caller (nsf_download_wait and
 * nsf_download_done excepted); different handles are independent.
 */
#ifndef NSFSI_H
#define NSFSI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NSF_ABI_VERSION 1

typedef enum nsf_status {
  NSF_OK = 0,
  NSF_ERR_CONFIG = 1,    /* ConfigFile / nsf_config problem (ConfigSettings::errorOccurred) */
  NSF_ERR_CUDA = 2,      /* a CUDA runtime call failed, or no usable sm_100 device */
  NSF_ERR_NONFINITE = 3, /* a conserved variable became NaN/Inf (Mesh::checkFinity) */
  NSF_ERR_GEOMETRY = 4,  /* a body leaves the mesh or bodies interact (cases the reference mishandles) */
  NSF_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
  NSF_ERR_ARG = 6,       /* bad argument (null pointer, wrong state, index out of range) */
  NSF_ERR_STATE = 7      /* call out of order (e.g. nsf_march before nsf_initialize) */
} nsf_status;

/* Boundary type per mesh face (the MeshEdgeBoundary subclasses, Boundary.h:80-181). */
typedef enum nsf_bc { NSF_BC_PERIODIC = 0, NSF_BC_SYMMETRY = 1, NSF_BC_INLET = 2, NSF_BC_OUTLET = 3 } nsf_bc;
/* Initial condition (Solver::applyStagnation_IC, Solver.cpp:31-51, and the seeded/analytic extensions). */
typedef enum nsf_ic { NSF_IC_STAGNATION = 0, NSF_IC_FREESTREAM_NOISE = 1, NSF_IC_TGV = 2 } nsf_ic;
/* Field indices for downloads: conserved (Solver.cpp:446-479 names), primitive, transport. */
enum {
  NSF_RHO = 0, NSF_RHO_U, NSF_RHO_V, NSF_RHO_W, NSF_RHO_E,
  NSF_U, NSF_V, NSF_W, NSF_P, NSF_T, NSF_MU, NSF_KAPPA, NSF_NUM_FIELDS
};

#define NSF_MAX_FILTER_INTERVALS 16
#define NSF_MAX_SPHERES 64
#define NSF_MAX_CYLINDERS 16

typedef struct nsf_sphere { double cx, cy, cz, r; } nsf_sphere;          /* SphereBody, Boundary.h:318-345 */
typedef struct nsf_cylinder { int32_t axis; double cx, cy, cz, r; } nsf_cylinder; /* CylinderBody, :287-316 */

/* Every ConfigSettings member (ConfigSettings.h:33-80) plus the case description that the reference
 * hard-codes in Mesh::setupBoundaries (Mesh.cpp:25-58) and Solver::initialize (Solver.cpp:22-28). */
typedef struct nsf_config {
  uint64_t NI, NJ, NK;
  int32_t stop_criterion; /* 0 = "timesteps", 1 = "end_time" */
  uint64_t stop_time_level;
  double t_end;
  double conv_stability_limit, visc_stability_limit;
  int32_t n_filter_intervals;
  uint32_t filter_intervals[NSF_MAX_FILTER_INTERVALS];
  int32_t n_filter_change_times;
  double filter_change_times[NSF_MAX_FILTER_INTERVALS];
  double status_report_interval;
  int32_t save_density, save_momentum, save_energy, save_velocity, save_pressure, save_temperature,
      save_viscosity, save_thermal_cond, save_ic, save_final, save_intervals;
  double save_period, save_intervals_start_time, save_intervals_end_time;
  int32_t conv_history; /* 0 "none", 1 "density", 2 "all" */
  double gamma, pr, r_gas, re, sutherlands_c1, sutherlands_c2, m0, t0, lx, ly, lz;
  double machine_precision_buffer; /* derived: DBL_EPSILON*(lx+ly+lz), ConfigSettings.cpp:160-163 */
  /* case description */
  int32_t shipped_case; /* 1: the reference's own hard-coded case (z-cylinder, symmetry y, in/out x) */
  int32_t bc[3][2];     /* [axis x,y,z][min,max] -> nsf_bc */
  int32_t n_spheres;
  nsf_sphere spheres[NSF_MAX_SPHERES];
  int32_t n_cylinders;
  nsf_cylinder cylinders[NSF_MAX_CYLINDERS];
  int32_t ic; /* nsf_ic */
  double noise_amp;
  uint64_t seed;
} nsf_config;

typedef struct nsf_solver nsf_solver;

/* ABI version of the loaded library. */
int32_t nsf_abi_version(void);

/* Fill *cfg with the values of the reference's shipped ConfigFile and its hard-coded case. */
nsf_status nsf_config_defaults(nsf_config* cfg);

/* Parse a ConfigFile (libconfig syntax) into *cfg.
 * Replaces ConfigSettings::ConfigSettings / loadSettings (ConfigSettings.cpp:11-33, :77-163):
 * same setting names, same strict int/float typing, same consistency check on the filter lists.
 * An optional `case = { ... }` group describes boundaries, bodies and the initial condition.
 * On failure returns NSF_ERR_CONFIG and writes a message into err (if err != NULL). */
nsf_status nsf_config_load(const char* path, nsf_config* cfg, char* err, size_t errlen);
nsf_status nsf_config_parse(const char* text, nsf_config* cfg, char* err, size_t errlen);

/* Allocate a solver on CUDA device `device`. Replaces Solver::Solver / Mesh::Mesh
 * (Solver.cpp:13-18, Mesh.cpp:10-21). device = -1 makes a host-only handle: nsf_initialize then runs
 * the host setup (classification, ghost and filter lists) and no GPU work; marching is refused. */
nsf_status nsf_create(const nsf_config* cfg, int32_t device, nsf_solver** out);

/* Replaces Solver::initialize (Solver.cpp:22-28): boundary setup and node classification on the host
 * (bit-exact with Mesh::categorizeNodes, Mesh.cpp:61-82), ghost-node interpolation weights solved on
 * the device, initial condition, initial dt. */
nsf_status nsf_initialize(nsf_solver* s);

/* Replaces `nsteps` calls of Solver::marchTimeStep(t, timeLevel) (Solver.cpp:130-167). Asynchronous:
 * the steps are queued on the handle's stream (one CUDA graph per step). In end_time mode, steps after
 * t reaches t_end are no-ops, as Simulation::run (Simulation.cpp:19-30) would not call them. */
nsf_status nsf_march(nsf_solver* s, uint64_t nsteps);

/* Wait for queued work; returns NSF_ERR_NONFINITE if a non-finite conserved value was seen. */
nsf_status nsf_sync(nsf_solver* s);

/* t, timeLevel and the dt of the next step (Simulation::t, ::timeLevel, Solver::dt). Synchronises. */
nsf_status nsf_get_time(nsf_solver* s, double* t, uint64_t* time_level, double* dt);

/* Copy selected fields (bit i of field_mask = field i, see NSF_RHO..NSF_KAPPA) to host memory, packed
 * in increasing field order, N doubles each, reference layout. Replaces reading Mesh's public arrays
 * (Mesh.h:82-86), as OutputManager does (OutputManager.cpp:152-258). Synchronises. */
nsf_status nsf_download(nsf_solver* s, uint32_t field_mask, double* host);

/* Snapshot output that overlaps the march (the writes of OutputManager::storeCurrentSolution,
 * OutputManager.cpp:101-106, called from processIntermediateOutput, :57-83). Queues, behind the steps
 * already marched, a device copy of the fields in field_mask (packed as nsf_download packs them) into one
 * of two staging buffers in HBM, then the copy of that buffer into `host` on a copy stream of its own, and
 * returns without waiting: the steps marched after the call run while the snapshot travels to the host.
 * `host` must be page-locked (nsf_host_alloc, or memory the caller pinned with CUDA) and hold
 * popcount(field_mask) * N doubles; it must not be read or freed before nsf_download_wait returns for
 * `*ticket`. The two staging buffers are used in turn: a third download waits on the device (not on the
 * host) until the first one's copy has left its buffer. The first download of a larger field set than
 * before allocates that buffer (and synchronises). Refused (NSF_ERR_STATE) for members of an ensemble or
 * x-slab group, whose steps run on the group's stream: use nsf_download there. */
nsf_status nsf_download_async(nsf_solver* s, uint32_t field_mask, double* host, uint64_t* ticket);
/* Blocks until the download `ticket` has landed in its host buffer. May be called from another thread
 * than the one marching the handle (e.g. a snapshot writer); it leaves nsf_last_error untouched. */
nsf_status nsf_download_wait(nsf_solver* s, uint64_t ticket);
/* *done = 1 if the download `ticket` has landed in its host buffer, else 0; never blocks. Thread rules as
 * nsf_download_wait. */
nsf_status nsf_download_done(nsf_solver* s, uint64_t ticket, int32_t* done);
/* Page-locked host memory for nsf_download_async (the caller needs no CUDA headers), and its release. */
nsf_status nsf_host_alloc(size_t bytes, void** out);
nsf_status nsf_host_free(void* p);

/* Overwrite the current conserved fields (5 x N doubles: rho, rho_u, rho_v, rho_w, rho_E) from host
 * memory at every node. The stored primitive state is not recomputed, exactly as writing
 * Mesh::conservedVariables directly would leave it. */
nsf_status nsf_upload_conserved(nsf_solver* s, const double* host);

/* Node classification (NodeTypeEnum values, Node.h:27-34), N bytes. */
nsf_status nsf_get_node_types(nsf_solver* s, uint8_t* out);
/* Grid spacing and origin offset, 6 doubles: dx, dy, dz, positionOffset x, y, z (Mesh::dx/dy/dz and
 * Mesh::positionOffset, set by boundary type in Mesh::setupBoundaries, Mesh.cpp:40-49). */
nsf_status nsf_get_geometry(nsf_solver* s, double* out);
/* Number of immersed bodies and, per body, ghost / filter counts and how many ghosts the image-point
 * closure loop added (Boundary.cpp:910-916). */
nsf_status nsf_get_num_bodies(nsf_solver* s, uint32_t* nbodies);
nsf_status nsf_get_body_counts(nsf_solver* s, uint32_t body, uint64_t* nghost, uint64_t* nfilter,
                               uint64_t* closure_added);
/* *interact = 1 if immersed bodies reach each other's nodes (a node in two bodies' ghost or filter lists, a
 * filter stencil or an image-point cell touching another body's ghost or filter nodes); such bodies act in
 * the reference's body order, one after another in every stage (Mesh.cpp:164-165). */
nsf_status nsf_get_body_interaction(nsf_solver* s, int32_t* interact);
/* Per ghost, 9 doubles: i, j, k, body-intercept x,y,z, image point x,y,z (GhostNode, Node.h:15-22). */
nsf_status nsf_get_ghosts(nsf_solver* s, uint32_t body, double* out);
/* Filter-node indices of a body (ImmersedBoundary::filterNodes, Boundary.h:208). */
nsf_status nsf_get_filter_nodes(nsf_solver* s, uint32_t body, uint64_t* out);

/* Per-step history rows [first, first+count): t after the step, dt used, and the five change norms
 * (Solver::storeNormsOfChange, Solver.cpp:510-530; -1 where the norm is not recorded). 7 doubles per row.
 * *available receives the number of recorded steps. Synchronises. */
nsf_status nsf_get_history(nsf_solver* s, uint64_t first, uint64_t count, double* out, uint64_t* available);

/* Instrumentation. nsf_march_timed: nsf_march with CUDA events recorded on the handle's stream around
 * the queued steps; waits and returns the elapsed device time. nsf_profile_steps: runs nsteps steps
 * (rounded up to a multiple of 10) as replays of a graph of 10 consecutive steps that also holds event
 * nodes around each of the four stage kernels; returns their mean durations (stage_ms[4]) and the mean
 * step time, both measured inside those replays. Both advance the solution. */
nsf_status nsf_march_timed(nsf_solver* s, uint64_t nsteps, double* elapsed_ms);
nsf_status nsf_profile_steps(nsf_solver* s, uint64_t nsteps, double* stage_ms, double* step_ms);
/* Kernel launches issued per RK4 step (for instrumentation). */
nsf_status nsf_launches_per_step(nsf_solver* s, uint64_t* launches);

/* End-of-step metrics for conserved fields the caller keeps in device memory, allocating nothing.
 * No counterpart in the reference: it exists for callers that cannot let a library allocate device
 * memory -- host frameworks that own all device memory, code running while a stream is captured into a
 * CUDA graph, real-time loops that must not allocate after start-up. d_old / d_new: 5 x N doubles
 * (rho, rho_u, rho_v, rho_w, rho_E, reference layout, N = NI*NJ*NK); d_types: N node-type bytes or NULL
 * (then every node off the mesh faces is interior); d_out: 6 doubles written on `stream` (a
 * cudaStream_t, NULL = default stream): the five change norms sqrt(dx*dy*dz*sum (old-new)^2) over
 * interior nodes, then the next dt from the primitive values of d_new at every node (what nsf_march
 * records when the case has no immersed body and stops on a step count). out[5] is the dt before the
 * end_time clip of Solver::updateTimeStepSize (Solver.cpp:85-87): a caller whose run stops at t_end
 * applies it itself, dt = t_end - t wherever t + out[5] > t_end. Scratch is a fixed 8 MiB device array inside the library,
 * so at most 29,826,048 nodes (larger grids: NSF_ERR_ARG). The first call on a device resolves that
 * array's device address (cudaGetSymbolAddress); make it before any stream capture. Calls that overlap
 * on the GPU share the array and race: serialise them. */
nsf_status nsf_step_metrics_noalloc(const nsf_config* cfg, const double* d_old, const double* d_new,
                                    const uint8_t* d_types, double* d_out, void* stream);

/* ---------------------------------------------------------------------------------------------------
 * Ensembles: n independent grids (each member its own case: grid shape, Mach, Re, bodies) advanced
 * together -- ONE CUDA graph per RK4 step for all members, each of the four stage launches a single
 * persistent kernel over the union of the members' work items. No counterpart in the reference; every
 * member advances exactly as Solver::marchTimeStep (Solver.cpp:130-167) advances its own grid.
 * tune_cache: NULL (default 32 x 8 tiles), or a file of autotuner results (created/extended as needed)
 * from which the stage-kernel tile shape is chosen: per device and composition of grid shapes, the
 * ensemble stage kernel's time per node with each tile shape (a composition not yet in it is timed first,
 * on throwaway ensembles of the same members).
 * Results: nsf_ensemble_member returns member m's handle (valid until nsf_ensemble_destroy; do not
 * destroy or march it) after waiting for the queued ensemble steps, for nsf_get_time / nsf_download / ... */
typedef struct nsf_ensemble nsf_ensemble;
nsf_status nsf_ensemble_create(const nsf_config* cfgs, uint32_t n, int32_t device, const char* tune_cache,
                               nsf_ensemble** out);
nsf_status nsf_ensemble_march(nsf_ensemble* e, uint64_t nsteps);
nsf_status nsf_ensemble_march_timed(nsf_ensemble* e, uint64_t nsteps, double* elapsed_ms);
/* nsteps steps launched one kernel at a time with events around the four stage launches: mean stage-kernel
 * times (stage_ms[4]) and mean step time. Advances every member. */
nsf_status nsf_ensemble_profile_steps(nsf_ensemble* e, uint64_t nsteps, double* stage_ms, double* step_ms);
/* Wait; NSF_ERR_NONFINITE / NSF_ERR_TIMEOUT if any member saw one. */
nsf_status nsf_ensemble_sync(nsf_ensemble* e);
nsf_status nsf_ensemble_member(nsf_ensemble* e, uint32_t m, nsf_solver** member);
/* Chosen tile shape (0: 32 x 8, 1: 16 x 16), kernel launches per step, stage work items. */
nsf_status nsf_ensemble_info(nsf_ensemble* e, int32_t* tile, uint64_t* launches_per_step, uint32_t* work_items);
const char* nsf_ensemble_last_error(nsf_ensemble* e);
void nsf_ensemble_destroy(nsf_ensemble* e);

/* Stage-kernel autotuner: times the stage kernels of this configuration's grid for each tile shape
 * (32 x 8 and 16 x 16 columns) on `device`, caches the result per device and grid shape in cache_path
 * (JSON lines; NULL: no cache) and returns the faster shape and the mean time per node and stage in
 * nanoseconds for both (ns_per_node[2]). A cached shape is not timed again. */
nsf_status nsf_autotune(const nsf_config* cfg, int32_t device, const char* cache_path, int32_t* tile,
                        double* ns_per_node);

/* ---------------------------------------------------------------------------------------------------
 * x-slab decomposition of one grid (no counterpart in the reference, whose grid is one array per field;
 * its k-fastest, i-slowest layout, Array3D.h:41-42, makes every i-plane contiguous). The interior planes
 * 1 .. NI-2 are split into nslabs near-equal contiguous ranges (nsf_slab_plan); each slab is a solver on its
 * planes plus a halo plane on each side, and a step exchanges the halo planes after every stage, the x
 * faces' periodic copies between the end slabs, and reduces the dt maxima and change norms over all slabs.
 * The result equals the single-grid solve node for node. Grids without immersed bodies; at least two
 * interior planes per slab. nsf_slab_group_create: all slabs in this process on one device (one CUDA graph
 * per step). nsf_slab_group_create_ranks: the slabs spread over `world` processes (one GPU each). */
typedef struct nsf_slab_group nsf_slab_group;
/* first[p], last[p]: the interior planes slab p computes (host only). */
nsf_status nsf_slab_plan(const nsf_config* cfg, int32_t nslabs, int32_t* first, int32_t* last);
nsf_status nsf_slab_group_create(const nsf_config* cfg, int32_t nslabs, int32_t device, nsf_slab_group** out);
nsf_status nsf_slab_group_march(nsf_slab_group* g, uint64_t nsteps);
nsf_status nsf_slab_group_march_timed(nsf_slab_group* g, uint64_t nsteps, double* elapsed_ms);
nsf_status nsf_slab_group_sync(nsf_slab_group* g);
/* Fields of the whole grid assembled from the slabs (as nsf_download). */
nsf_status nsf_slab_group_download(nsf_slab_group* g, uint32_t field_mask, double* host);
/* Slab p's solver handle (t, dt, history, ...; valid until nsf_slab_group_destroy; do not march it). */
nsf_status nsf_slab_group_solver(nsf_slab_group* g, int32_t slab, nsf_solver** s);
/* Slab count, the first plane each slab owns, launches per step. */
nsf_status nsf_slab_group_info(nsf_slab_group* g, int32_t* nslabs, int32_t* first_planes, uint64_t* launches_per_step);
const char* nsf_slab_group_last_error(nsf_slab_group* g);
void nsf_slab_group_destroy(nsf_slab_group* g);
/* A group over several processes: process `rank` of `world` (world <= nslabs) holds the consecutive slabs p
 * with p * world / nslabs == rank, on `device`; the planes that cross processes move by NCCL send/recv
 * inside the step graph, and every slab's dt maxima and change-norm sums are all-gathered and combined in
 * slab order (every process computes the same dt; the fields equal the single-grid solve's). Collective:
 * every process of the group calls it with the same cfg, nslabs, world and nccl_id (NSF_NCCL_ID_BYTES bytes
 * from nsf_slab_nccl_id on one of them, passed on by any host channel). flags: NSF_SLAB_NCCL_ALL also moves
 * the planes between slabs of the same process through NCCL (send/recv to itself; with world = 1 a check of
 * the NCCL path on one GPU). NCCL is loaded at run time (libnccl.so.2; NSF_ERR_CUDA without it). The other
 * nsf_slab_group_* calls see this process's slabs (info, solver, download: its own planes only). */
#define NSF_NCCL_ID_BYTES 128
#define NSF_SLAB_NCCL_ALL 1
nsf_status nsf_slab_nccl_id(uint8_t* id);
nsf_status nsf_slab_group_create_ranks(const nsf_config* cfg, int32_t nslabs, int32_t rank, int32_t world,
                                       const uint8_t* nccl_id, int32_t flags, int32_t device, nsf_slab_group** out);
/* Host only: owner[p] = the process of slab p for `world` processes, and the group's plane transfers in the
 * order every process issues them, 5 int32 each: list (0 halo of the stage output, 1 periodic x face,
 * 2 halo of the filtered density), from slab, its global plane, to slab, its global plane. *count: in, the
 * capacity of transfers (entries); out, the number of transfers. */
nsf_status nsf_slab_schedule(const nsf_config* cfg, int32_t nslabs, int32_t world, int32_t* owner,
                             int32_t* transfers, int32_t* count);

/* ---------------------------------------------------------------------------------------------------
 * Discrete adjoint (a forward / backward pair; no counterpart in the reference, whose marchTimeStep,
 * Solver.cpp:130-167, it differentiates). Objective of a run of stop_time_level steps from level 0:
 *   J = (1/n_avg) sum over the last n_avg steps of F_x(U_n),  F_x = -(dx dy dz)^(2/3) sum_g p(U_g) n_x(g)
 * over the ghost nodes g of the immersed bodies (p: the ghost's pressure, equal to its image point's;
 * n: the body's outward unit normal at the ghost's body-intercept point). Parameters: the conserved field
 * at level 0 (5 x N doubles, every node, reference layout) and the x-inlet velocity profile factor
 * (NJ x NK doubles, index j*NK + k; the inlet velocity is min(1, t/10) M0 times the factor; only the
 * inlet's own nodes j, k in [1, N-2] matter). Cases: periodic faces and x inlet / outlet faces, spheres
 * and cylinders; stopCriterion "timesteps".
 * The first nsf_adj_forward freezes its dt sequence; later runs (and the backward pass) use it.
 * nsf_adj_backward: gradients of dJ * J. When every step's snapshot set fits the tape limit
 * (nsf_adj_set_tape_limit), the forward run records them all and the backward run is the adjoint kernels
 * alone. Otherwise the forward run stores `snapshots` + 1 states (default 20 + the initial one): when two
 * segments' sets fit the limit (or one), a state every ceil(steps / (snapshots + 1)) steps, and the
 * backward run restores each segment's state, records that segment's sets and runs its adjoint kernels
 * (the recording of one segment overlaps the adjoint kernels of the next); else binomial checkpointing
 * with recomputation. The gradients are the same bit for bit either way. Both leave the handle's state at
 * some level of the run. */
nsf_status nsf_adj_configure(nsf_solver* s, uint32_t avg_last_steps, uint32_t snapshots);
/* Device memory the tape may take, in bytes: 0 never records one (checkpointing), UINT64_MAX (default)
 * allows up to half the device memory free at the first forward run. A tape larger than a new limit is
 * released. */
nsf_status nsf_adj_set_tape_limit(nsf_solver* s, uint64_t bytes);
/* Bytes of the tape the last forward run recorded (0: it checkpointed). */
nsf_status nsf_adj_tape_bytes(nsf_solver* s, uint64_t* bytes);
/* The segment tape the last forward run left for the backward run: its bytes and the steps per segment
 * (both 0: none, the run was taped whole or checkpoints binomially). */
nsf_status nsf_adj_segment_tape(nsf_solver* s, uint64_t* bytes, uint32_t* segment_steps);
nsf_status nsf_adj_forward(nsf_solver* s, const double* u0, const double* inflow, double* J);
nsf_status nsf_adj_backward(nsf_solver* s, double dJ, double* g_inflow, double* g_u0);
/* The frozen dt sequence (count values: dt of step n). */
nsf_status nsf_adj_get_dt(nsf_solver* s, double* dts, uint64_t* count);
/* Device time (ms, CUDA events) of the phases of one adjoint step, launched eagerly after a forward run:
 * ms[0] recomputation of the step with its stage snapshots, [2] ghost nodes (with the objective), near-body
 * filter, edge conditions, solid-node copies, RK4 combine and RHS input quantities (one launch per stage),
 * [7] transposed RHS, [8] density filter (summed over the four stages); [1] and [3]-[6] are 0. Gradients
 * are unaffected. */
nsf_status nsf_adj_profile_step(nsf_solver* s, uint64_t step, double* ms);

/* Self-check of the device reciprocal and square root the stage kernel uses for the primitive values
 * (Newton-Raphson refinement of the hardware approximations): for n positive inputs x, out[4 i .. 4 i + 3]
 * = the refined reciprocal, the IEEE 1/x, the refined square root, the IEEE sqrt(x). */
nsf_status nsf_math_selftest(int32_t device, uint64_t n, const double* x, double* out);

/* Test support for the bounded waits (no counterpart in the reference): every wait of the stage
 * kernel gives up after `polls` polls (0 restores the default of 2^22), and withhold_epilogue = 1 makes
 * the kernel's producer issue none of its epilogue loads, so the waits for them run out. A step that
 * ran with the switch on is invalid: nsf_sync then returns NSF_ERR_TIMEOUT and the handle should be
 * destroyed. Synchronises. */
nsf_status nsf_debug_wait_limit(nsf_solver* s, uint64_t polls, int32_t withhold_epilogue);

/* Text of the last error on this handle (static storage owned by the handle). */
const char* nsf_last_error(nsf_solver* s);

void nsf_destroy(nsf_solver* s);

#ifdef __cplusplus
}
#endif
#endif /* NSFSI_H */
