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
void launch_adj_objective(const Grid* dg, const AdjPtrs& A, int nGhost, const double* nx, double dA, double weight,
                          int nSM, void* stream);
void launch_adj_ghost(const Grid* dg, const AdjPtrs& A, int nGhost, int nFilter, double* ipbar, const long long* cnode,
                      const int* coff, const int* cent, int ncell, int nSM, void* stream);
void launch_adj_filter(const Grid* dg, const AdjPtrs& A, const long long* nodes, int count, int nFilter, int nSM,
                       void* stream);
// roles: device copy of the step's control block (stage times, dt).
void launch_adj_edge(const Grid& hg, const AdjPtrs& A, const LaunchPlan& L, int axis, const StepCtl* roles, int s,
                     double* fbar, double* lamInflow, bool inletGather, void* stream);
// The stage kernel's adjoint: prepare = RK4 combine adjoint into lam, the RHS input quantities into V
// (11 x N) and, at solid nodes, the adjoint of the solid-node copy (solidMask: the stage's copy mask);
// rhs = transposed RHS gather and the chain rule into the stage input's adjoints.
void launch_adj_prepare(const Grid* dg, const Grid& hg, const AdjPtrs& A, int s, const StepCtl* roles, int solidMask,
                        double* lam, double* V, int nSM, void* stream);
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

}  // namespace nsf
#endif
