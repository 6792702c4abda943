// Launchers of the discrete-adjoint kernels (nsf_adjoint.cu), used by the adjoint driver (nsf_adjoint.cpp).
#ifndef NSF_ADJOINT_H
#define NSF_ADJOINT_H

#include "nsf_device.cuh"

namespace nsf {

// Pointers one adjoint kernel works on (unused ones may be NULL).
struct AdjPtrs {
  double* lamO[5];         // adjoint of the forward kernel's output buffer
  double* lamI[5];         // adjoint of the stage's input buffer
  double* lamR;            // adjoint of the density the stage's primitives were computed from
  double* lamU0[5];        // adjoint of U0 (the step's starting state)
  double* lamAcc[5];       // adjoint of the RK4 accumulator
  double* lamFpre;         // [2F] adjoint of the pre-filter values
  double* lamFnew;         // [2F] adjoint of the filtered values
  const double* val[5];    // forward values the kernel read (from a snapshot)
  const double* valR;
  const double* valFpre;   // [2F]
};

void launch_objective(const Grid* dg, const double* nx, double dA, double weight, double* acc, void* stream);
void launch_fpre_init(const Grid* dg, int nFilter, const double* rho, const double* rE, int nSM, void* stream);
void launch_fpre_init_adj(const Grid* dg, int nFilter, const double* lamFpre, double* lamRho, double* lamRE, int nSM,
                          void* stream);
// Everything of a stage's adjoint before the transposed RHS: ghost nodes (and, with `objective`, the
// objective's adjoint at them), near-body filter and edge conditions in one cooperative launch (k_adj_bc),
// then the RK4 combine and RHS input quantities (k_adj_combine).
struct AdjBcParams {
  AdjPtrs A;
  // ghosts: image-point adjoints (5 x nGhost), reverse map of the image-point cells (CSR)
  double* ipbar;
  const long long* cnode;
  const int* coff;
  const int* cent;
  int ncell;
  // near-body filter: the nodes of the filter stencils and, per node, its own and its six neighbours'
  // filter slots (7 each, -1: none)
  const long long* fsNodes;
  const int* fsSlots;
  int nfs;
  // edge blocks per axis (k_edge_bc's), the values the edge conditions read (the stage output before
  // them), the inlet's per-node adjoints, the inflow profile's adjoint
  const EdgeBlock* edges[3];
  const double* edgeVal[5];
  int nEdge[3];
  int inletGather;
  double* fbar;
  double* lamInflow;
  const StepCtl* roles;  // device copy of the step's control block (stage times, dt)
  // combine: the stage's copy mask, RHS adjoint lam (5 x N) and input quantities V (11 x N; rows 4-10, the
  // primitives and transport values -- rows 0-3 would repeat the stage input's own values)
  int solidMask;
  double* lam;
  double* V;
  // objective (the last stage of a step whose result enters J): F_x's pressure at the ghost nodes
  int objective;
  const double* objVal[5];
  const double* nx;
  double dA, weight;
  unsigned long long* sync;  // [2] grid-barrier arrival counters (zero at creation, only grow)
  // non-zero: the bodies' nodes and the face planes are disjoint, so the body phases and the edge phases
  // run as two independent chains (the launcher sets the blocks of the body chain)
  int bodyBlocks;
  int* timeout;              // StepCtl::timeout of the solver: set when a barrier gives up
};
void launch_adj_bc(const Grid& hg, const AdjBcParams& P, int s, int nSM, void* stream);
// The transposed RHS (gather) and the chain rule through the primitives into the stage input's adjoints,
// from launch_adj_bc's lam and V.
void launch_adj_rhs(const Grid* dg, const Grid& hg, const AdjPtrs& A, const double* lam, const double* V, int nSM,
                    void* stream);
// Kernel attributes (shared-memory size of the transposed RHS); call once before the first launch.
int adj_kernels_init();
void launch_adj_density_filter(const Grid* dg, long long N, const double* lamDstConst, double* lamDst, double* lamSrc,
                               int nSM, void* stream);
// count (<= kMaxCopies) device-to-device copies of words[c] doubles in one launch.
constexpr int kMaxCopies = 16;
void launch_copies(const double* const* src, double* const* dst, const long long* words, int count, int nSM,
                   void* stream);

// Copies into the adjoint's tape (the snapshot sets of every step of a forward run), with the sources and
// the set resolved on the device from the live control block, so one captured step serves every step.
enum TapeSource : int {
  TAPE_I = 0,       // ctl->I[q][f]
  TAPE_R_SEP = 1,   // ctl->R[q], copied only when it is another buffer than ctl->I[q][0]
  TAPE_O = 2,       // ctl->O[q][f]
  TAPE_FIXED = 3,   // src as given
};
struct TapeCopy {
  int kind[kMaxCopies], q[kMaxCopies], f[kMaxCopies];
  const double* src[kMaxCopies];
  long long srcOff[kMaxCopies];  // added to the resolved source
  long long dstOff[kMaxCopies];  // within the step's set
  long long words[kMaxCopies];
  int n;
  double* tape;
  long long setWords;
  int levelOffset;  // set = (ctl->level + levelOffset) mod nSets (levelOffset -1 after the step, whose
                    // finalize advanced the level); nothing is written for a negative level + levelOffset
  int nSets;        // sets the tape holds: every step's, or a ring of checkpoint segments' sets
};
void launch_tape_copy(const StepCtl* ctl, const TapeCopy& T, int nSM, void* stream);

}  // namespace nsf
#endif
