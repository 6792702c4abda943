// Device-side data structures shared by the kernels in nsf_kernels.cu and the host driver.
//
// Buffer model. The reference keeps two conserved-variable buffers, `conservedVariables` (the stage
// target, written in place by every stage) and `conservedVariablesOld` (U0, read only), and swaps them
// at the start of each step (Mesh::swapConservedVariables, Mesh.cpp:144-151). Values at non-interior
// nodes therefore persist across steps and are read stale by the near-body filter and the periodic
// copies. A fused stencil kernel cannot write its input in place, so here each field has THREE
// physical buffers whose roles (cons / old / scratch) rotate: stage s reads I_s and writes O_s, with
// O_1 = O_3 = the reference's `conservedVariables` and O_2 = O_4 = scratch; before the boundary
// conditions of stages 2-4 the solid-node values of I_s are copied into O_s, so every buffer holds,
// node for node, what the reference's buffer holds at that point. Roles are kept in device memory
// (StepCtl) so that one captured CUDA graph serves every step, including the ones where the global
// density filter swaps the density buffers (Mesh::applyFilter_ifAppropriate, Mesh.cpp:108-140).
#ifndef NSF_DEVICE_CUH
#define NSF_DEVICE_CUH

#include <cstdint>
#include <vector>

namespace nsf {

constexpr int MAX_HIST = 1 << 20;  // per-step history rows kept on the device (ring)

// Physical constants and the reference's precomputed stencil coefficients (Solver.cpp:202-360),
// evaluated on the host exactly as the reference writes them.
struct Consts {
  double gamma, gm1, pr, re, sc1, pf, h0, vmod, convLim, viscLim, m0, tEnd;
  double dx, dy, dz, dxdydz;
  // continuity / inviscid: -1/(2d)
  double ax, ay, az;
  // x-momentum: 2/(3dx^2), 1/(2dy^2), 1/(2dz^2), -1/(6dydx), 1/(4dxdy), -1/(6dzdx), 1/(4dxdz)
  double xm_xx, xm_yy, xm_zz, xm_yx, xm_xy, xm_zx, xm_xz;
  // y-momentum: 1/(2dx^2), 2/(3dy^2), 1/(2dz^2), -1/(6dxdy), 1/(4dydx), -1/(6dzdy), 1/(4dydz)
  double ym_xx, ym_yy, ym_zz, ym_xy, ym_yx, ym_zy, ym_yz;
  // z-momentum: 1/(2dx^2), 1/(2dy^2), 2/(3dz^2), 1/(4dzdx), -1/(6dxdz), 1/(4dzdy), -1/(6dydz)
  double zm_xx, zm_yy, zm_zz, zm_zx, zm_xz, zm_zy, zm_yz;
  // energy: 2/(3dx^2), 1/(2dx^2), -1/(6dydx), -1/(6dzdx), 1/(4dydx), 1/(4dzdx), 1/(2dy^2), 2/(3dy^2),
  //         -1/(6dzdy), 1/(4dzdy), 1/(2dz^2), 2/(3dz^2)
  double e_xx23, e_xx12, e_yx6, e_zx6, e_yx4, e_zx4, e_yy12, e_yy23, e_zy6, e_zy4, e_zz12, e_zz23;
  int endTime, convHistory;
  int nFilterIv, nChange;
  unsigned filterIv[16];
  double changeT[16];
};

// Per-step control block in device memory, updated by the prologue / finalize kernels.
struct StepCtl {
  // persistent state
  double t;               // simulated time (Simulation::t)
  double dt;              // dt of the coming step (Solver::dt)
  unsigned long long level;  // timeLevel
  int perm[5][3];         // per field: physical buffer of [cons, old, scratch]
  int nonFinite;          // sticky NaN/Inf flag (Mesh::checkFinity)
  // Test support for the bounded waits of the stage kernel (left at 0 in normal runs): withhold = 1 makes
  // its producer issue no epilogue-ring load, so the column warps' waits run out; waitLimit = polls
  // before a wait gives up (0: the kernel's default).
  int withhold;
  // per-step decisions (prologue)
  int active;             // 0: step is a no-op (end_time reached)
  int filterNow;          // global density filter on this step
  double* gfSrc;          // filter input (the reference's conservedVariables.rho before the swaps)
  double* gfDst;          // filter output (conservedVariablesOld.rho before the swaps)
  double* U0[5];
  double* I[4][5];
  double* O[4][5];
  double* R[4];           // density used for the primitive variables of the stage input
  int copyMask[4];        // fields whose solid-node values are copied I -> O before the stage's BCs
  int iPhys[4][5];        // physical buffer of each stage input field (selects its TMA descriptor)
  int rPhys[4];           // physical buffer of the density used for primitives
  int u0Phys[5];          // physical buffer of each U0 field
  int timeout;            // sticky: a bounded device wait gave up (the step's results are invalid)
  long long waitLimit;    // see withhold
  double stageT[4];       // boundary-condition time of each stage
  double dtUsed;
  // stage-4 reductions
  unsigned long long mx[4];  // bit patterns of non-negative maxima: c+|u|, c+|v|, c+|w|, mu/(1+rho)*mod
};

// Everything a kernel needs to know about one grid (one ensemble member).
struct Grid {
  int NI, NJ, NK;
  long long sI, sJ, N;
  Consts C;
  StepCtl* ctl;
  double* bufs[3][5];
  double* acc[5];
  int NKp;                // k pitch of the device layout (multiple of 4: rows start on 32-byte boundaries)
  const void* tmaps;      // device array of TMA descriptors (see nsf_stage_tma.cu)
  const uint8_t* type;    // NodeTypeEnum | FILTER_BIT | EDGE_PLANE_BIT | ZCOPY_UP_BIT | ZCOPY_DOWN_BIT
  const int* fidx;        // node -> filter slot (only read where FILTER_BIT is set)
  double* fpre;           // [F][2] pre-filter rho, rho_E of the last near-body filter
  double* fnew;           // [F][2] filtered values (written back after the ghost update)
  const uint8_t* fsolid;  // [F] bit q: stencil node q (centre, +i, -i, +j, -j, +k, -k) is a solid node off the faces
  // [F] filter slots are per (body, node) in body order; fmeta = the node's first slot, | FMETA_LAST on its
  // last slot (a node filtered by two bodies has two slots: the stage kernel's pre-filter values come from
  // the first, the stage-4 dt and norm terms from the last)
  const int* fmeta;
  const long long* fnode; // [F] node of each filter slot
  int nFilter;
  // ghost nodes
  int nGhost;
  const long long* gnode;   // [G]
  const long long* gcell;   // [G][8]
  const double* gw;         // [G][16]: Neumann weights (rho, rho_E) then Dirichlet weights (momenta)
  // [G][8]: per corner, the filter slot whose filtered rho, rho_E the ghost reads (the last slot of a body
  // up to the ghost's own in body order), or -1: read the node's current value
  const int* gsrc;
  const uint8_t* glast;     // [G]: 1 if no later ghost item writes the same node (it adds the stage-4 dt terms)
  // solid-node copy list (ghost + inactive) and the inactive nodes' stored primitive values
  int nSolid;
  const long long* snode;   // [S]
  int nInactive;
  const long long* inode;   // [Q] inactive nodes (not on a boundary plane)
  const double* iprim;      // [Q][5] u, v, w, p, mu as the reference holds them
  // boundary conditions in application order
  int nEdge;
  int eAxis[6], eSide[6], eBc[6];
  int eBox[6][6];           // owned box i0,i1,j0,j1,k0,k1
  // Both z faces periodic: the stage kernel also writes the periodic copy of each interior node it
  // computes at k = 1 and k = NK-2 into k = NK-1 and k = 0 (same values, same sectors), and the z edge
  // kernel handles only the rows the stage kernel does not (see edge_blocks).
  int zFused;
  int yFused;  // periodic y faces: the stage kernel writes the copies of its YCOPY_BIT nodes
  // gradient support (NULL / 0 for a plain run): an x-inlet velocity profile factor per (j, k) node of the
  // inlet plane, and a prescribed dt per step (the adjoint differentiates with the dt sequence frozen)
  const double* inflow;     // [NJ * NKp], index j * NKp + k
  const double* dtFrozen;   // [nDtFrozen]: dt of step n
  int nDtFrozen;
  StepCtl* ctlHist;         // [nCtlHist]: the control block of step n right after its prologue (roles)
  int nCtlHist;
  // reductions
  double* normPart;         // [nNormSlots][5]: stage-kernel CTAs first, then the near-body filter's blocks
  int nNormSlots;
  int normSlotFilter;       // first slot of the near-body filter's partial sums
  double* hist;             // [MAX_HIST][7]
};

// Stage-kernel tile shapes (one column thread per (j, k) column, 256 columns per CTA).
enum StageTile { STAGE_TILE_32x8 = 0, STAGE_TILE_16x16 = 1 };

struct StageItem {
  int j0, k0, i0, i1;  // tile origin (first computed j, k) and inclusive i range
  int g;               // ensemble member (0 for a single grid)
};

// Launch geometry of one step, fixed at initialisation.
// Edge-condition kernels: blocks of 32 x kEdgeRows threads over a face (small blocks spread a face's
// few thousand nodes over many SMs), listed one by one so that a launch holds only blocks with nodes
// (an ensemble's faces differ in size from member to member).
constexpr int kEdgeRows = 2;
struct EdgeBlock {
  int g;       // member (0 for a single grid)
  int e;       // edge (face) of that member
  int a0, b0;  // first in-plane coordinates of the block: (a, bb) = the two axes other than the face's
  unsigned long long mask;  // thread ty * 32 + tx works iff its bit is set
  // thread ty * 32 + tx reads a solid node off the mesh faces, whose value it takes from the solid-node
  // copy's source (set by the fused boundary kernel's plan; 0 for the separate kernels)
  unsigned long long solidSrc;
};
// The blocks of one axis' faces of a grid, in launch order, appended to out (member g). type: the host
// node types with their flag bits (k fastest), or NULL. With G.zFused and a type array, the z faces'
// blocks cover only the rows the stage kernel does not copy (rows on an x or y face plane, and rows
// whose source node is not an unfiltered interior fluid node).
void edge_blocks(const Grid& G, const uint8_t* type, int g, int axis, std::vector<EdgeBlock>& out);

// Arguments of one launch of the fused boundary kernel (k_bc, see nsf_kernels.cu): the stage's boundary
// work in dependency levels (nsf_bc_plan.cpp). Level L (0-based here) of member g: edge blocks
// edges[edgeStart[L * (M + 1) + g] ..), near-body filter items (class 0) and ghost-pass items (class 1, the
// encoding of ghost_pass_item) items[itemStart[(L * 2 + c) * (M + 1) + g] ..). Solid-node copies: level 0.
struct BcParams {
  const EdgeBlock* edges;
  const int* edgeStart;
  const int* items;
  const int* itemStart;
  // arrival counters: [1 + g] member g's blocks done (stage 4), [1 + members + g] member g's level barrier
  // (members share no boundary data, so each member's blocks wait for one another only)
  unsigned long long* sync;
  const int* blockStart;     // members + 1: the blocks of member g are blockStart[g] .. blockStart[g + 1] - 1
  const int* memberLevels;   // members: the levels member g has (at most `levels`)
  int levels, members;
};

// Boundary work of one grid split into levels (bc_plan_member), and several grids' levels flattened into
// the arrays BcParams points to (bc_flatten).
struct BcMemberLevels {
  int levels = 0;
  long long solid = 0;
  std::vector<std::vector<EdgeBlock>> edges;  // [level]
  std::vector<std::vector<int>> filter, ghost;
};
struct BcMemberInput {  // device node indices (the padded device layout)
  std::vector<long long> snode, fnode, gnode, gcell, inode;
  std::vector<int> fbody, gbody, gsrc;  // body of each filter slot and ghost; ghost corner sources (Grid::gsrc)
  std::vector<uint8_t> typeDev;  // node types with FILTER_BIT, per device node
  std::vector<int> fidx;         // filter slot per device node, or -1
};
struct BcFlat {
  int levels = 0;
  std::vector<int> memberLevels;  // each member's own level count
  long long maxWork = 1;         // threads one member needs in its busiest level (the largest over members)
  std::vector<long long> work;   // the same per member
  std::vector<EdgeBlock> edges;
  std::vector<int> edgeStart, items, itemStart;
};

struct LaunchPlan {
  int nSM;
  int tile;  // StageTile
  int stageBlocks;
  int nItems;
  StageItem* items;  // device; the items of CTA b are items[ctaStart[b] .. ctaStart[b + 1])
  int* ctaStart;     // device, stageBlocks + 1 entries
  EdgeBlock* edgeBlocks[3];  // device, per axis
  int nEdgeBlocks[3];
  int filterBlocks, ghostBlocks, solidBlocks, gfBlocks;
  // Fused boundary kernel: per stage one cooperative launch of bcBlocks blocks (bcBlockStart: each member's
  // range) that runs the stage's boundary work level by level with grid barriers between levels (and, on
  // stage 4, the end-of-step finalize). 0: separate launches.
  int bcBlocks;
  int* bcBlockStart;
  int bcLevels;
  int* bcMemberLevels;
  EdgeBlock* bcEdges;  // device arrays of BcParams
  int* bcEdgeStart;
  int* bcItems;
  int* bcItemStart;
  unsigned long long* bcSync;  // device, 1 + 2 members counters, zero at creation
  int nSlots;
  bool hasBodies;
  bool hasFilter, hasGhostWork, hasSolid;
};

// Host entry points of nsf_kernels.cu.
// Stage-kernel variant queries (v: StageTile).
size_t stage_smem_bytes(int v);
int stage_configure(int v);
int stage_tile_j(int v);
int stage_tile_k(int v);
int stage_type_box_width(int v);
int stage_threads(int v);
int stage_occupancy(int v);
int stage_num_maps();
// Registers per thread the stage kernel is launched with; stage_register_split_ok() checks that the
// kernel's setmaxnreg split fits in them (a split above the launch total would never be granted).
int stage_launch_registers(int v);
bool stage_register_split_ok(int v);
void launch_stage(const Grid& hg, const LaunchPlan& L, int s, void* stream);
void launch_stage_ensemble(const Grid* dGrids, const LaunchPlan& L, int s, void* stream);
// dg: the grid in device memory (read by the small kernels); hg: the same grid on the host (passed by
// value to the stage kernel, whose coefficients then come from the constant bank).
int enqueue_step(Grid* dg, const Grid& hg, const LaunchPlan& L, void* stream);
// Pieces of a step for callers that put work between them (x-slab groups, nsf_slab.cpp): the prologue and
// the density filter of one grid; the fused boundary kernel of stage s (fin: with the end-of-step finalize).
// Return the launches queued.
int enqueue_step_begin(Grid* dg, const LaunchPlan& L, void* stream);
int launch_bc_part(Grid* dg, const LaunchPlan& L, int s, bool fin, void* stream);
// Same sequence with events recorded around each of the four stage kernels (events[2*s], events[2*s+1]);
// used for per-kernel timing. inGraph: the stream is being captured, and the events become event-record
// nodes of the graph (so the kernels are timed inside graph replays, as the solver runs them).
int enqueue_step_profiled(Grid* dg, const Grid& hg, const LaunchPlan& L, void* stream, void* events,
                          bool inGraph = false);
// Callbacks of a step launched kernel by kernel (enqueue_step_hooked): after the prologue, before each
// stage kernel, and before each stage's edge boundary conditions (after the solid-node copy).
struct StepHook {
  virtual ~StepHook() = default;
  virtual void after_prologue() {}
  virtual void before_stage(int) {}
  virtual void before_edges(int) {}
  // false: before_edges does nothing for this step, so the stage's boundary work may run as the fused
  // boundary kernel (whose phases the hook cannot come between)
  virtual bool wants_before_edges() const { return true; }
};
// lastStage: NULL for a whole step, or a plan whose items stage 4 is limited to (the step then stops after
// that stage kernel: the adjoint's recomputation when only some planes of the step's result are read).
int enqueue_step_hooked(Grid* dg, const Grid& hg, const LaunchPlan& L, void* stream, StepHook* hook,
                        const LaunchPlan* lastStage = nullptr);
// recip_nr, 1/x, sqrt_nr, sqrt of n host values on the current device (4 x n results); a cudaError_t.
int math_selftest(long long n, const double* hostIn, double* hostOut);
// One RK4 step of every member of an ensemble (dGrids: device array of `members` grids; L: the ensemble's
// combined plan). events: NULL, or 8 events recorded around the four stage kernels.
int enqueue_ensemble_step(Grid* dGrids, int members, const LaunchPlan& L, void* stream, void* events);
// Blocks of 256 threads of the fused boundary kernel that can be resident on the device at once (its
// cooperative launches must not exceed this), or 0 if unknown.
int bc_capacity(int nSM);
// Dependency levels of one grid's boundary work (nsf_bc_plan.cpp); edgeBlocks: the grid's edge blocks per
// axis (edge_blocks). Returns the number of levels.
int bc_plan_member(const Grid& G, const std::vector<EdgeBlock> edgeBlocks[3], const BcMemberInput& in,
                   BcMemberLevels& out);
void bc_flatten(const std::vector<const BcMemberLevels*>& members, BcFlat& out);
// Blocks of 256 threads per member for a fused-kernel launch of at most `capacity` blocks, in proportion to
// the members' work (at least one each, never more than a member can use); returns the members + 1 range
// starts, empty if the members do not fit.
std::vector<int> bc_block_ranges(const BcFlat& fl, int capacity);
// The node a periodic face node finally copies (opposite interior plane, then further periodic faces).
void periodic_source_host(const Grid& G, int axis, int side, int ijk[3]);
void launch_ghost_weights(int nGhost, const double* pts, const double* nrm, const uint8_t* flags, const double* ipl,
                          double dx, double dy, double dz, double* w, void* stream);
// Downloads (nsf_download, nsf_download_async): per field (rho, rho_u, rho_v, rho_w, rho_E, u, v, w, p, T, mu,
// kappa) its slot in the packed snapshot, or -1 when it is not asked for.
constexpr int NSF_SNAP_FIELDS = 12;
struct SnapSlots {
  int slot[NSF_SNAP_FIELDS];
};
// Solid inactive nodes with stored primitive values (device node index, 7 values each): the list for time
// level 0 and the one for later levels.
struct SnapInactive {
  const long long* nodes;
  const double* p7;
  int count;
  const long long* nodesIc;
  const double* p7Ic;
  int countIc;
};
// Queues the snapshot of the slots' fields into `out` (packed, NI*NJ*NK doubles per slot) on `stream`.
void launch_snapshot(const Grid* dg, const SnapSlots& sl, const SnapInactive& in, double* out, int nSM, void* stream);

}  // namespace nsf
#endif
