// The solver handle behind the C ABI (include/nsfsi.h), shared by nsf_capi.cpp and nsf_ensemble.cpp.
#ifndef NSF_SOLVER_IMPL_H
#define NSF_SOLVER_IMPL_H

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <string>
#include <vector>

#include "nsf_device.cuh"
#include "nsf_internal.h"

struct nsf_solver {
  nsf_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  nsf::HostSetup setup;
  std::vector<uint8_t> typeFlags;  // host node types with the edge-plane and filter bits (k fastest)
  bool initialized = false;
  bool hostOnly = false;  // device < 0: host setup only (classification queries), no GPU work
  std::vector<void*> allocs;
  nsf::Grid hGrid{};
  nsf::Grid* dGrid = nullptr;
  nsf::StepCtl* dCtl = nullptr;
  nsf::StepCtl* hCtl = nullptr;  // page-locked host copy of the control block (nsf_get_time, nsf_sync)
  nsf::LaunchPlan plan{};
  cudaGraphExec_t graphExec = nullptr;
  cudaGraph_t graph = nullptr;
  int launchesPerStep = 0;
  // instrumentation (nsf_profile_steps): a graph of kProfileSteps steps with event nodes around the stage
  // kernels, built on first use
  cudaGraphExec_t profExec = nullptr;
  cudaGraph_t profGraph = nullptr;
  std::vector<cudaEvent_t> profEv;
  int nSM = 0;
  // solid inactive nodes with stored primitive values (downloads)
  long long* dDlNode = nullptr;
  double* dDlPrim = nullptr;    // values after the first step (periodic copies applied)
  double* dDlPrimIc = nullptr;  // values before any step (each node's own initial values)
  long long* dDlNodeIc = nullptr;
  int nDl = 0, nDlIc = 0;
  std::string err;
  std::vector<CUtensorMap> hostMaps;
  void* encodeFn = nullptr;
  int tileRequest = -1;  // StageTile to use, or -1 for the default
  // x-slab member of a slab group (nsf_slab.cpp): the initial condition sliced from the whole grid's, and
  // node flags to add (EDGE_PLANE_BIT on halo planes and on the whole grid's edge planes); empty otherwise
  std::vector<double> slabCons, slabPrim;
  std::vector<uint8_t> slabFlags;
  std::vector<int> ghostOrder;   // device ghost slot -> position in the bodies' ghost lists
  nsf::BcMemberLevels bcLevels;  // dependency levels of the boundary work (fused boundary kernel)
  nsf::StepCtl ctlInit{};  // the control block at level 0 (the discrete adjoint restarts from it)
  struct AdjCtx* adj = nullptr;  // discrete-adjoint state (nsf_adjoint.cpp), created on first use
  // member of an ensemble or x-slab group: its steps are queued on the group's stream, not on `stream`
  bool grouped = false;
  // asynchronous downloads (nsf_download_async): a copy stream and two device staging buffers used in turn,
  // each with the events that mark its snapshot taken (on `stream`) and its copy to the host done (on
  // dlStream); ticket t uses buffer t & 1
  cudaStream_t dlStream = nullptr;
  double* dlStage[2] = {nullptr, nullptr};
  size_t dlCap[2] = {0, 0};  // doubles
  cudaEvent_t dlTaken[2] = {nullptr, nullptr};
  cudaEvent_t dlDone[2] = {nullptr, nullptr};
  std::atomic<uint64_t> dlIssued{0};  // tickets handed out; read by nsf_download_wait from other threads
};

// Frees the adjoint state of a handle (nsf_adjoint.cpp).
void nsf_adjoint_free(nsf_solver* s);
// Device set-up of a handle whose host setup (s->setup) is in place (nsf_capi.cpp), and the initial dt of a
// grid from its initial fields (Solver::updateTimeStepSize at t = 0).
nsf_status nsf_build_device(nsf_solver* s);
double nsf_initial_dt(const nsf_config& c, const nsf::HostSetup& S, const std::vector<double>& cons,
                      const std::vector<double>& prim);

#endif
