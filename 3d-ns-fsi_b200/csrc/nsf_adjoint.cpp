// Discrete adjoint driver (C ABI: nsf_adj_configure / nsf_adj_forward / nsf_adj_backward / nsf_adj_get_dt).
//
// Objective: J = (1/n_avg) sum over the last n_avg steps of F_x(U_n), the x-force of the pressure on the
// immersed bodies, F_x = -dA sum_g p(U_g) n_x(g) over the ghost nodes g (p from the ghost's conserved
// values, which equal the image point's pressure; n = unit normal of the body at the ghost's body-intercept
// point; dA = (dx dy dz)^(2/3)). Parameters: the conserved field at level 0 (every node) and a factor per
// (j, k) node of the x-inlet's velocity profile (the inlet velocity is min(1, t/10) M0 times the factor;
// 1 everywhere is the reference's uniform inflow). The dt sequence of the first forward run is frozen
// and used by every later run (forward, recomputation and finite-difference checks alike).
//
// Backward: binomial checkpointing over the steps (Griewank's schedule: with c free snapshots the longest
// reversible run in t sweeps is C(c+t, t)); a step whose adjoint is due is recomputed kernel by kernel
// from its snapshot, keeping each stage's inputs, and the adjoint kernels (nsf_adjoint.cu) then run in
// reverse kernel order on adjoint arrays that mirror the physical field buffers. The recomputation and
// the schedule's restores and advances run on the solver's stream, the adjoint kernels on a second
// stream, with two snapshot sets between them: the forward work of the next step overlaps the adjoint
// kernels of the current one (at the grid sizes of the adjoint both use a fraction of the GPU).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "nsf_adjoint.h"
#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_solver_impl.h"

using namespace nsf;

struct AdjCtx {
  int nsteps = 0, navg = 50, nsnap = 20;
  bool haveDt = false, haveForward = false;
  std::vector<double> dts;
  double* dDt = nullptr;
  double* dInflow = nullptr;
  double* dU0 = nullptr;  // 5 x Nd: the forward run's level-0 state
  double* dNx = nullptr;
  double dA = 0;
  double* dAcc = nullptr;
  long long* cnode = nullptr;
  int* coff = nullptr;
  int* cent = nullptr;
  int ncell = 0;
  long long* fsNodes = nullptr;
  int* fsSlots = nullptr;
  int nfs = 0;
  bool inletX = false;
  bool xInOut = false;  // an x face is an inlet or an outlet (its adjoint reads the planes next to it)
  // The x-planes the inlet / outlet adjoint reads (i = 1, 2, NI-3, NI-2, inside the faces' j, k range)
  // hold only unfiltered interior fluid nodes: no kernel after the stage kernel writes them, so the next
  // stage's input (or the step's result) has the values the edge conditions read, and no copy is taken.
  bool edgePlanesClean = false;
  double* lam = nullptr;  // 20 x Nd: adjoint of bufs[b][f] at (5 b + f) Nd, accumulator at (15 + f) Nd
  double* lamFpre = nullptr;
  double* lamFnew = nullptr;
  double* lamInflow = nullptr;
  double* tmpLam = nullptr;
  double* tmpV = nullptr;
  double* ipbar = nullptr;
  double* fbar = nullptr;
  unsigned long long* bcSync = nullptr;  // grid-barrier counters of k_adj_bc (one per chain)
  // No node of the bodies' adjoint work (ghosts, filter nodes, image-point cells, filter stencils) lies in
  // the planes the edge conditions' adjoint touches (the faces and the two planes inside each): the two
  // chains of the boundary kernel run side by side.
  bool bodiesClearOfFaces = false;
  int* dTimeout = nullptr;               // set when a barrier of k_adj_bc gives up (checked after the backward run)
  std::vector<double*> slot;
  std::vector<StepCtl*> slotCtl;
  // Two snapshot sets: the recomputation of one step fills one set (on the solver's stream) while the
  // adjoint kernels of the step before read the other (on adjStream). A set holds per stage
  // (11 Nd + 2F): I (5), R (1), O before the edge conditions (5), fpre; then the step's result O (5 Nd);
  // and the step's control block after its prologue.
  double* snapStage[2] = {nullptr, nullptr};
  double* snapResult[2] = {nullptr, nullptr};
  StepCtl* snapCtl[2] = {nullptr, nullptr};
  int nextSet = 0;
  cudaStream_t adjStream = nullptr;
  cudaEvent_t setReady[2] = {nullptr, nullptr};  // recorded on the solver's stream once a set is filled
  cudaEvent_t setFree[2] = {nullptr, nullptr};   // recorded on adjStream once the adjoint kernels read it
  StepCtl* dHist = nullptr;      // [nsteps]: each step's control block after its prologue (written on the device)
  std::vector<StepCtl> hist;     // host copy of dHist from the last forward run
  std::vector<std::pair<int, int>> chain;  // (level, slot) checkpoints the forward run stores
  bool chainStored = false;                // the slots still hold the last forward run's checkpoints
  // CUDA graphs per distinct pattern of buffer roles (the roles rotate with a short period) and snapshot
  // set: the recomputation (solver's stream) and the adjoint kernels (adjStream)
  std::map<std::vector<uintptr_t>, cudaGraphExec_t> graphs;
  // Stage 4 of a recomputed step whose result enters no objective term: only the x-planes the inlet /
  // outlet adjoint reads (i = 1, 2, NI-3, NI-2) are computed, and nothing after that stage kernel runs.
  LaunchPlan lastStagePlan{};
  // Tape: the snapshot set of every step, recorded by the forward run when nsteps sets fit the limit, so
  // the backward run is the adjoint kernels alone (no checkpoint restores, re-advancing or recomputation).
  // A set has the layout of a snapshot set; its control block is the step's entry of dHist.
  // Segment tape, when the whole run's sets exceed the limit: the forward run stores a checkpoint every
  // segLen steps in slots 0, 1, ... (segLen = ceil(nsteps / (nsnap + 1)), so the slots suffice), and the
  // backward run restores each segment's checkpoint, records that segment's sets with the tape step graph
  // and runs their adjoint kernels. The tape then holds two segments' sets (or one, when only one fits):
  // the recording of a segment on the solver's stream overlaps the adjoint kernels of the one after it.
  uint64_t tapeLimit = UINT64_MAX;   // bytes; UINT64_MAX: half the free device memory at the forward run
  double* tape = nullptr;
  size_t tapeSetWords = 0;
  int tapeSets = 0;                  // sets the tape holds (nsteps, or 1-2 segments of segLen)
  int segLen = 0;
  bool tapeValid = false;            // the tape holds the last forward run's sets
  bool segValid = false;             // the slots hold the last forward run's segment checkpoints
  cudaGraphExec_t tapeExec = nullptr;  // one step with its tape copies (sources and set resolved on the device)
  std::vector<void*> allocs;
};

namespace {

nsf_status fail(nsf_solver* s, nsf_status st, const std::string& msg) {
  s->err = msg;
  return st;
}

#define CKA(call)                                                                  \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) return fail(s, NSF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
nsf_status aalloc(nsf_solver* s, AdjCtx* a, T** p, size_t count) {
  void* q = nullptr;
  CKA(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  a->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return NSF_OK;
}

size_t nd(const nsf_solver* s) { return size_t(s->hGrid.N); }
size_t nf(const nsf_solver* s) { return size_t(s->hGrid.nFilter); }
size_t per_stage(const nsf_solver* s) { return 11 * nd(s) + 2 * nf(s); }

int phys(const nsf_solver* s, const double* p, int f) {
  for (int b = 0; b < 3; ++b)
    if (s->hGrid.bufs[b][f] == p) return b;
  return 0;
}

double* lamOf(const nsf_solver* s, const AdjCtx* a, int b, int f) { return a->lam + (size_t(b) * 5 + f) * nd(s); }

nsf_status push_grid(nsf_solver* s) {
  CKA(cudaMemcpy(s->dGrid, &s->hGrid, sizeof(Grid), cudaMemcpyHostToDevice));
  return NSF_OK;
}

nsf_status setup(nsf_solver* s) {
  if (s->adj) return NSF_OK;
  if (!s->initialized || s->hostOnly) return fail(s, NSF_ERR_STATE, "the adjoint needs an initialized device solver");
  const nsf_config& c = s->cfg;
  if (c.stop_criterion != 0) return fail(s, NSF_ERR_ARG, "the adjoint needs stopCriterion = \"timesteps\"");
  const HostSetup& S = s->setup;
  for (const auto& e : S.edges) {
    const bool ok = e.bc == NSF_BC_PERIODIC || (e.axis == 0 && (e.bc == NSF_BC_INLET || e.bc == NSF_BC_OUTLET));
    if (!ok) return fail(s, NSF_ERR_ARG, "the adjoint supports periodic faces and x-inlet/x-outlet faces only");
  }
  if (S.NI < 6 || S.NJ < 4 || S.NK < 4) return fail(s, NSF_ERR_ARG, "grid too small for the adjoint");
  if (S.bodiesInteract)
    return fail(s, NSF_ERR_ARG, "the adjoint supports immersed bodies that do not reach each other's nodes only");
  if (adj_kernels_init() != 0) return fail(s, NSF_ERR_CUDA, "adjoint kernel attributes could not be set");
  auto* a = new AdjCtx;
  s->adj = a;
  a->nsteps = int(c.stop_time_level);
  const Grid& G = s->hGrid;
  const size_t N = nd(s), F = nf(s), NG = size_t(G.nGhost), plane = size_t(G.NJ) * G.NKp;
  nsf_status st;
  for (const auto& e : S.edges) {
    a->inletX |= e.axis == 0 && e.bc == NSF_BC_INLET;
    a->xInOut |= e.axis == 0 && (e.bc == NSF_BC_INLET || e.bc == NSF_BC_OUTLET);
  }
  a->edgePlanesClean = true;
  for (size_t i : {size_t(1), size_t(2), S.NI - 3, S.NI - 2})
    for (size_t j = 1; j + 1 < S.NJ; ++j)
      for (size_t k = 1; k + 1 < S.NK; ++k) {
        const uint8_t t = s->typeFlags[(i * S.NJ + j) * S.NK + k];
        if ((t & TYPE_MASK) != FLUID_INTERIOR || (t & FILTER_BIT)) a->edgePlanesClean = false;
      }
  if ((st = aalloc(s, a, &a->dDt, size_t(a->nsteps) + 1)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->dInflow, plane)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->dU0, 5 * N)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->dAcc, 1)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->lam, 20 * N)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->lamFpre, 2 * F)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->lamFnew, 2 * F)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->lamInflow, plane)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->tmpLam, 5 * N)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->tmpV, 11 * N)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->ipbar, 5 * NG)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->fbar, 2 * plane)) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->bcSync, 2)) != NSF_OK) return st;
  CKA(cudaMemset(a->bcSync, 0, 2 * sizeof(unsigned long long)));
  if ((st = aalloc(s, a, &a->dTimeout, 1)) != NSF_OK) return st;
  CKA(cudaMemset(a->dTimeout, 0, sizeof(int)));
  for (int j = 0; j < 2; ++j) {
    if ((st = aalloc(s, a, &a->snapStage[j], 4 * per_stage(s))) != NSF_OK) return st;
    if ((st = aalloc(s, a, &a->snapResult[j], 5 * N)) != NSF_OK) return st;
    if ((st = aalloc(s, a, &a->snapCtl[j], 1)) != NSF_OK) return st;
    CKA(cudaEventCreateWithFlags(&a->setReady[j], cudaEventDisableTiming));
    CKA(cudaEventCreateWithFlags(&a->setFree[j], cudaEventDisableTiming));
  }
  CKA(cudaStreamCreateWithFlags(&a->adjStream, cudaStreamNonBlocking));
  if ((st = aalloc(s, a, &a->dHist, size_t(a->nsteps))) != NSF_OK) return st;
  {  // the partial stage-4 plan: the main plan's tiles over planes [1, 2] and [NI-3, NI-2], round robin
    LaunchPlan& P = a->lastStagePlan;
    P = s->plan;
    P.items = nullptr;
    P.ctaStart = nullptr;
    P.nItems = 0;
    P.stageBlocks = 0;
    std::vector<StageItem> items;
    if (a->xInOut) {
      const int TJ = stage_tile_j(s->plan.tile), TK = stage_tile_k(s->plan.tile);
      const int nj = int((S.NJ - 2 + TJ - 1) / TJ), nk = int((S.NK - 2 + TK - 1) / TK);
      std::vector<std::pair<int, int>> ranges = {{1, 2}, {int(S.NI) - 3, int(S.NI) - 2}};
      if (ranges[1].first <= ranges[0].second + 1) ranges = {{1, int(S.NI) - 2}};
      for (auto& r : ranges)
        for (int tj = 0; tj < nj; ++tj)
          for (int tk = 0; tk < nk; ++tk) items.push_back(StageItem{1 + tj * TJ, 1 + tk * TK, r.first, r.second, 0});
    }
    if (!items.empty()) {
      P.nItems = int(items.size());
      P.stageBlocks = std::min(P.nItems, s->nSM);
      std::vector<StageItem> ordered;
      std::vector<int> start(1, 0);
      for (int b = 0; b < P.stageBlocks; ++b) {
        for (int q = b; q < P.nItems; q += P.stageBlocks) ordered.push_back(items[q]);
        start.push_back(int(ordered.size()));
      }
      if ((st = aalloc(s, a, &P.items, ordered.size())) != NSF_OK) return st;
      if ((st = aalloc(s, a, &P.ctaStart, start.size())) != NSF_OK) return st;
      CKA(cudaMemcpy(P.items, ordered.data(), ordered.size() * sizeof(StageItem), cudaMemcpyHostToDevice));
      CKA(cudaMemcpy(P.ctaStart, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  s->hGrid.ctlHist = a->dHist;
  s->hGrid.nCtlHist = a->nsteps;
  // objective: body normals at the ghosts' body-intercept points (in the device's ghost order, gnode), area
  // weight
  std::vector<double> nxBody;
  for (const auto& b : S.bodies)
    for (const auto& g : b.ghosts) {
      double d[3] = {g.bi[0] - b.c[0], g.bi[1] - b.c[1], g.bi[2] - b.c[2]};
      if (!b.sphere) d[b.axis] = 0;
      const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      nxBody.push_back(len > 0 ? d[0] / len : 0.0);
    }
  std::vector<double> nx(nxBody.size());
  for (size_t q = 0; q < nx.size(); ++q) nx[q] = nxBody[size_t(s->ghostOrder[q])];
  a->dA = std::pow(S.d[0] * S.d[1] * S.d[2], 2.0 / 3.0);
  if ((st = aalloc(s, a, &a->dNx, nx.size())) != NSF_OK) return st;
  if (!nx.empty()) CKA(cudaMemcpy(a->dNx, nx.data(), nx.size() * sizeof(double), cudaMemcpyHostToDevice));
  // reverse map of the image-point cells: node -> (ghost, corner) entries with non-zero weights
  std::vector<long long> gcell(8 * NG);
  std::vector<uint8_t> type(N);
  if (NG) CKA(cudaMemcpy(gcell.data(), G.gcell, gcell.size() * sizeof(long long), cudaMemcpyDeviceToHost));
  CKA(cudaMemcpy(type.data(), G.type, N, cudaMemcpyDeviceToHost));
  std::map<long long, std::vector<int>> byNode;
  for (size_t q = 0; q < NG; ++q)
    for (int m = 0; m < 8; ++m) {
      const long long n = gcell[8 * q + m];
      if ((type[n] & TYPE_MASK) == SOLID_GHOST) continue;  // a body-intercept row: zero weight
      byNode[n].push_back(int(8 * q + m));
    }
  std::vector<long long> cn;
  std::vector<int> co(1, 0), ce;
  for (auto& kv : byNode) {
    cn.push_back(kv.first);
    ce.insert(ce.end(), kv.second.begin(), kv.second.end());
    co.push_back(int(ce.size()));
  }
  a->ncell = int(cn.size());
  if ((st = aalloc(s, a, &a->cnode, cn.size())) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->coff, co.size())) != NSF_OK) return st;
  if ((st = aalloc(s, a, &a->cent, ce.size())) != NSF_OK) return st;
  if (!cn.empty()) {
    CKA(cudaMemcpy(a->cnode, cn.data(), cn.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CKA(cudaMemcpy(a->cent, ce.data(), ce.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  CKA(cudaMemcpy(a->coff, co.data(), co.size() * sizeof(int), cudaMemcpyHostToDevice));
  // nodes of the near-body filter stencils
  std::vector<long long> fnode(F);
  if (F) CKA(cudaMemcpy(fnode.data(), G.fnode, F * sizeof(long long), cudaMemcpyDeviceToHost));
  std::set<long long> fs;
  for (long long n : fnode)
    for (long long o : {0LL, G.sI, -G.sI, G.sJ, -G.sJ, 1LL, -1LL}) fs.insert(n + o);
  std::vector<long long> fsv(fs.begin(), fs.end());
  a->nfs = int(fsv.size());
  if ((st = aalloc(s, a, &a->fsNodes, fsv.size())) != NSF_OK) return st;
  if (!fsv.empty()) CKA(cudaMemcpy(a->fsNodes, fsv.data(), fsv.size() * sizeof(long long), cudaMemcpyHostToDevice));
  {  // per stencil node: its own filter slot and its six neighbours' (the order of the filter's gather)
    std::map<long long, int> slotOf;
    for (size_t q = 0; q < fnode.size(); ++q) slotOf.emplace(fnode[q], int(q));
    const long long off[6] = {G.sI, -G.sI, G.sJ, -G.sJ, 1, -1};
    std::vector<int> slots(7 * fsv.size(), -1);
    for (size_t q = 0; q < fsv.size(); ++q)
      for (int d = 0; d < 7; ++d) {
        const long long n = d == 0 ? fsv[q] : fsv[q] + off[d - 1];
        if (n < 0 || n >= G.N) continue;
        const auto it = slotOf.find(n);
        if (it != slotOf.end()) slots[7 * q + size_t(d)] = it->second;
      }
    if ((st = aalloc(s, a, &a->fsSlots, slots.size())) != NSF_OK) return st;
    if (!slots.empty()) CKA(cudaMemcpy(a->fsSlots, slots.data(), slots.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  {  // the bodies' adjoint nodes against the face planes (device indices: k fastest, rows of NKp)
    std::vector<long long> gnode(NG);
    if (NG) CKA(cudaMemcpy(gnode.data(), G.gnode, NG * sizeof(long long), cudaMemcpyDeviceToHost));
    auto clear = [&](long long n) {
      const long long i = n / G.sI, j = (n % G.sI) / G.sJ, k = n % G.sJ;
      return i >= 3 && i <= G.NI - 4 && j >= 2 && j <= G.NJ - 3 && k >= 2 && k <= G.NK - 3;
    };
    bool ok = true;
    for (const auto* v : {&gnode, &fnode, &cn, &fsv})
      for (long long n : *v) ok = ok && clear(n);
    a->bodiesClearOfFaces = ok;
  }
  // inflow profile factor 1; the initial condition of the case as the default level-0 state
  std::vector<double> ones(plane, 1.0);
  CKA(cudaMemcpy(a->dInflow, ones.data(), plane * sizeof(double), cudaMemcpyHostToDevice));
  std::vector<double> cons, prim;
  initial_condition(c, S, cons, prim);
  const size_t hp = S.NK * sizeof(double), dp = size_t(G.NKp) * sizeof(double);
  CKA(cudaMemset(a->dU0, 0, 5 * N * sizeof(double)));
  for (int f = 0; f < 5; ++f)
    CKA(cudaMemcpy2D(a->dU0 + f * N, dp, cons.data() + f * S.N, hp, hp, S.NI * S.NJ, cudaMemcpyHostToDevice));
  s->hGrid.inflow = a->dInflow;
  return push_grid(s);
}

nsf_status alloc_slots(nsf_solver* s, AdjCtx* a) {
  const size_t words = 15 * nd(s) + 2 * nf(s);
  while (int(a->slot.size()) < a->nsnap + 1) {
    double* p;
    StepCtl* c;
    nsf_status st;
    if ((st = aalloc(s, a, &p, words)) != NSF_OK) return st;
    if ((st = aalloc(s, a, &c, 1)) != NSF_OK) return st;
    a->slot.push_back(p);
    a->slotCtl.push_back(c);
  }
  return NSF_OK;
}

// Level-0 state: bufs[0] = U0, the other buffers zero (the reference's zero-initialised second buffer),
// fpre from U0, the control block of initialisation (dt of step 0 from the frozen sequence, if any).
nsf_status reset(nsf_solver* s, AdjCtx* a) {
  const size_t N = nd(s);
  Grid& G = s->hGrid;
  CKA(cudaMemcpyAsync(G.bufs[0][0], a->dU0, 5 * N * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  CKA(cudaMemsetAsync(G.bufs[1][0], 0, 15 * N * sizeof(double), s->stream));  // buffers 1, 2 and the accumulator
  launch_fpre_init(s->dGrid, G.nFilter, G.bufs[0][0], G.bufs[0][4], s->nSM, s->stream);
  StepCtl c = s->ctlInit;
  if (a->haveDt) c.dt = a->dts[0];
  CKA(cudaMemcpyAsync(s->dCtl, &c, sizeof c, cudaMemcpyHostToDevice, s->stream));
  CKA(cudaStreamSynchronize(s->stream));
  return NSF_OK;
}

nsf_status save(nsf_solver* s, AdjCtx* a, int k) {
  const size_t N = nd(s), F = nf(s);
  CKA(cudaMemcpyAsync(a->slot[k], s->hGrid.bufs[0][0], 15 * N * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  if (F)
    CKA(cudaMemcpyAsync(a->slot[k] + 15 * N, s->hGrid.fpre, 2 * F * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  CKA(cudaMemcpyAsync(a->slotCtl[k], s->dCtl, sizeof(StepCtl), cudaMemcpyDeviceToDevice, s->stream));
  return NSF_OK;
}

nsf_status restore(nsf_solver* s, AdjCtx* a, int k) {
  const size_t N = nd(s), F = nf(s);
  CKA(cudaMemcpyAsync(s->hGrid.bufs[0][0], a->slot[k], 15 * N * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  if (F)
    CKA(cudaMemcpyAsync(s->hGrid.fpre, a->slot[k] + 15 * N, 2 * F * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  CKA(cudaMemcpyAsync(s->dCtl, a->slotCtl[k], sizeof(StepCtl), cudaMemcpyDeviceToDevice, s->stream));
  return NSF_OK;
}

nsf_status advance(nsf_solver* s, int n) {
  for (int q = 0; q < n; ++q) CKA(cudaGraphLaunch(s->graphExec, s->stream));
  return NSF_OK;
}

// What the adjoint kernels of a step read, all from one snapshot set, so the next step's recomputation may
// overwrite the working buffers meanwhile: per stage its input values I (and its density R when that is
// another buffer), the near-body filter's pre-values and, for x inlet / outlet faces whose neighbouring
// planes are not clean (AdjCtx::edgePlanesClean), the four x-planes next to them (i = 1, 2, NI-3, NI-2) of
// the stage output before the edge conditions; the step's result; the step's control block. The step's
// roles (which physical buffer plays which part) are known on the host from the forward run's record, so
// nothing waits here and the recomputation can be captured as a graph.
struct SnapSet {
  double* stage;  // 4 x per_stage
  double* result;  // 5 Nd
  StepCtl* ctl;
};
SnapSet snap_set(const AdjCtx* a, int j) { return SnapSet{a->snapStage[j], a->snapResult[j], a->snapCtl[j]}; }

struct SnapHook : StepHook {
  nsf_solver* s;
  AdjCtx* a;
  const StepCtl& R;
  SnapSet set;
  cudaError_t err = cudaSuccess;
  const double* src[kMaxCopies];
  double* dst[kMaxCopies];
  long long words[kMaxCopies];
  int n = 0;
  SnapHook(nsf_solver* s_, AdjCtx* a_, const StepCtl& r, SnapSet st) : s(s_), a(a_), R(r), set(st) {}
  void add(double* d, const double* sr, size_t w) {
    if (n == kMaxCopies) flush();
    src[n] = sr;
    dst[n] = d;
    words[n++] = (long long)w;
  }
  void flush() {
    launch_copies(src, dst, words, n, s->nSM, s->stream);
    n = 0;
  }
  void after_prologue() override {
    if (err == cudaSuccess) err = cudaMemcpyAsync(set.ctl, s->dCtl, sizeof(StepCtl), cudaMemcpyDeviceToDevice, s->stream);
  }
  void before_stage(int q) override {
    const size_t N = nd(s);
    double* base = set.stage + q * per_stage(s);
    for (int f = 0; f < 5; ++f) add(base + f * N, R.I[q][f], N);
    if (R.R[q] != R.I[q][0]) add(base + 5 * N, R.R[q], N);
    if (nf(s)) add(base + 11 * N, s->hGrid.fpre, 2 * nf(s));
    flush();
  }
  bool wants_before_edges() const override { return a->xInOut && !a->edgePlanesClean; }
  void before_edges(int q) override {
    if (!a->xInOut || a->edgePlanesClean) return;
    const size_t N = nd(s), plane = size_t(s->hGrid.sI), NI = size_t(s->hGrid.NI);
    double* base = set.stage + q * per_stage(s);
    for (size_t i : {size_t(1), size_t(2), NI - 3, NI - 2})
      for (int f = 0; f < 4; ++f) add(base + (6 + f) * N + i * plane, R.O[q][f] + i * plane, plane);
    flush();
  }
  // after the step: its result (the objective's pressure, the inlet / outlet adjoint of stage 4)
  void result() {
    const size_t N = nd(s);
    for (int f = 0; f < 5; ++f) add(set.result + f * N, R.O[3][f], N);
    flush();
  }
};

size_t tape_set_words(const nsf_solver* s) { return 4 * per_stage(s) + 5 * nd(s); }

// The tape set of step k (the tape holds every step's set, or a ring of segments' sets).
SnapSet tape_set(const nsf_solver* s, const AdjCtx* a, int k) {
  double* base = a->tape + size_t(k % a->tapeSets) * a->tapeSetWords;
  return SnapSet{base, base + 4 * per_stage(s), a->dHist + k};
}

// The copies of SnapHook, into the tape set of the running step: the forward run records every step's set
// with one captured step graph (the copy kernel reads the buffer roles and the time level from the control
// block).
struct TapeHook : StepHook {
  nsf_solver* s;
  AdjCtx* a;
  TapeCopy T{};
  TapeHook(nsf_solver* s_, AdjCtx* a_) : s(s_), a(a_) {
    T.tape = a->tape;
    T.setWords = (long long)a->tapeSetWords;
    T.nSets = a->tapeSets;
  }
  void add(int kind, int q, int f, const double* src, size_t srcOff, size_t dstOff, size_t words) {
    if (T.n == kMaxCopies) flush();
    const int c = T.n++;
    T.kind[c] = kind;
    T.q[c] = q;
    T.f[c] = f;
    T.src[c] = src;
    T.srcOff[c] = (long long)srcOff;
    T.dstOff[c] = (long long)dstOff;
    T.words[c] = (long long)words;
  }
  void flush() {
    launch_tape_copy(s->dCtl, T, s->nSM, s->stream);
    T.n = 0;
  }
  void before_stage(int q) override {
    const size_t N = nd(s), base = q * per_stage(s);
    for (int f = 0; f < 5; ++f) add(TAPE_I, q, f, nullptr, 0, base + f * N, N);
    add(TAPE_R_SEP, q, 0, nullptr, 0, base + 5 * N, N);
    if (nf(s)) add(TAPE_FIXED, q, 0, s->hGrid.fpre, 0, base + 11 * N, 2 * nf(s));
    flush();
  }
  bool wants_before_edges() const override { return a->xInOut && !a->edgePlanesClean; }
  void before_edges(int q) override {
    if (!wants_before_edges()) return;
    const size_t N = nd(s), plane = size_t(s->hGrid.sI), NI = size_t(s->hGrid.NI), base = q * per_stage(s);
    for (size_t i : {size_t(1), size_t(2), NI - 3, NI - 2})
      for (int f = 0; f < 4; ++f) add(TAPE_O, q, f, nullptr, i * plane, base + (6 + f) * N + i * plane, plane);
    flush();
  }
  // after the step (its finalize has advanced the level): the result
  void result() {
    const size_t N = nd(s);
    T.levelOffset = -1;
    for (int f = 0; f < 5; ++f) add(TAPE_O, 3, f, nullptr, 0, 4 * per_stage(s) + f * N, N);
    flush();
    T.levelOffset = 0;
  }
};

enum TapeMode { TAPE_NONE, TAPE_FULL, TAPE_SEGMENTS };

void release_tape(AdjCtx* a) {
  if (a->tapeExec) cudaGraphExecDestroy(a->tapeExec);
  a->tapeExec = nullptr;
  if (a->tape) cudaFree(a->tape);
  a->tape = nullptr;
  a->tapeSets = 0;
  a->tapeValid = false;
  a->segValid = false;
}

// The tape of the coming forward run under the limit (allocating it, and capturing the tape step graph, on
// first use): every step's set when they all fit (TAPE_FULL: recorded by the forward run); else two
// checkpoint segments' sets, or one, when the schedule has fewer slots than steps (TAPE_SEGMENTS: recorded
// by the backward run, segment by segment); else none (binomial checkpointing).
nsf_status prepare_tape(nsf_solver* s, AdjCtx* a, int* mode) {
  *mode = TAPE_NONE;
  if (a->tapeLimit == 0) return NSF_OK;
  const size_t words = tape_set_words(s);
  const double setBytes = double(words) * 8.0;
  double limit = double(a->tapeLimit);
  if (a->tapeLimit == UINT64_MAX) {
    size_t fr = 0, tot = 0;
    CKA(cudaMemGetInfo(&fr, &tot));
    limit = (double(fr) + setBytes * a->tapeSets) / 2;  // the free memory as it was before the tape
  }
  const int L = (a->nsteps + a->nsnap) / (a->nsnap + 1);
  int sets = 0, m = TAPE_NONE;
  if (setBytes * a->nsteps <= limit) {
    sets = a->nsteps;
    m = TAPE_FULL;
  } else if (L < a->nsteps && setBytes * L <= limit) {
    sets = setBytes * 2 * L <= limit ? 2 * L : L;
    m = TAPE_SEGMENTS;
  }
  if (m == TAPE_NONE) return NSF_OK;
  if (a->tape && a->tapeSets != sets) {
    CKA(cudaStreamSynchronize(a->adjStream));
    CKA(cudaStreamSynchronize(s->stream));
    release_tape(a);
  }
  if (!a->tape) {
    if (cudaMalloc(&a->tape, size_t(setBytes * sets)) != cudaSuccess) {
      cudaGetLastError();  // not enough memory after all: checkpoints instead
      a->tape = nullptr;
      return NSF_OK;
    }
    a->tapeSetWords = words;
    a->tapeSets = sets;
  }
  if (!a->tapeExec) {
    CKA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    TapeHook hook(s, a);
    enqueue_step_hooked(s->dGrid, s->hGrid, s->plan, s->stream, &hook, nullptr);
    hook.result();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return fail(s, NSF_ERR_CUDA, std::string("tape step capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&a->tapeExec, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return fail(s, NSF_ERR_CUDA, std::string("tape step graph: ") + cudaGetErrorString(e2));
  }
  a->segLen = m == TAPE_SEGMENTS ? L : 0;
  *mode = m;
  return NSF_OK;
}

// Phases of an adjoint step, for nsf_adj_profile_step.
// PH_BC: one launch per stage for ghosts, near-body filter, edge conditions and the RK4 combine (and, on
// steps whose result enters J, the objective); slots 1 and 3-6 stay, empty, for the layout of the result.
enum AdjPhase { PH_RECOMPUTE, PH_OBJECTIVE, PH_BC, PH_UNUSED3, PH_UNUSED4, PH_UNUSED5, PH_UNUSED6, PH_RHS, PH_DFILTER,
                PH_COUNT };

// Events recorded between the phases of an eagerly launched adjoint step.
struct PhaseTimer {
  cudaStream_t st;
  std::vector<cudaEvent_t> ev;
  std::vector<int> phase;
  void mark(int ph) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, st);
    ev.push_back(e);
    phase.push_back(ph);
  }
  void collect(double* ms) {
    for (size_t q = 1; q < ev.size(); ++q) {
      float t = 0;
      if (cudaEventElapsedTime(&t, ev[q - 1], ev[q]) == cudaSuccess) ms[phase[q]] += t;
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};

// Enqueues the recomputation of a step with roles R on the solver's stream, filling snapshot set `set`:
// the working state holds U_k on entry, U_{k+1} on exit. objective: F_x(U_{k+1}) enters J (the whole step
// runs; else stage 4 only where the inlet / outlet adjoint reads it). pt: NULL, or phase events.
nsf_status enqueue_recompute(nsf_solver* s, AdjCtx* a, const StepCtl& R, bool objective, int set,
                             PhaseTimer* pt = nullptr) {
  SnapHook hook(s, a, R, snap_set(a, set));
  if (pt) pt->mark(-1);
  enqueue_step_hooked(s->dGrid, s->hGrid, s->plan, s->stream, &hook, objective ? nullptr : &a->lastStagePlan);
  hook.result();
  if (pt) pt->mark(PH_RECOMPUTE);
  if (hook.err != cudaSuccess) return fail(s, NSF_ERR_CUDA, std::string("adjoint recomputation: ") + cudaGetErrorString(hook.err));
  CKA(cudaGetLastError());
  return NSF_OK;
}

// Enqueues the adjoint kernels of that step on `stream`, reading only snapshot set S (a pipelined set or the
// step's tape set) and fixed buffers: the adjoint arrays hold the adjoint of U_{k+1} on entry and of U_k on
// exit.
nsf_status enqueue_adjoint_kernels(nsf_solver* s, AdjCtx* a, const StepCtl& R, bool objective, const SnapSet& S,
                                   cudaStream_t st, PhaseTimer* pt = nullptr) {
  auto mark = [&](int ph) {
    if (pt) pt->mark(ph);
  };
  const Grid& G = s->hGrid;
  const size_t N = nd(s);
  const int nSM = s->nSM;
  for (int q = 3; q >= 0; --q) {
    const double* snap = S.stage + q * per_stage(s);
    AdjBcParams P{};
    AdjPtrs& A = P.A;
    for (int f = 0; f < 5; ++f) {
      A.lamO[f] = lamOf(s, a, phys(s, R.O[q][f], f), f);
      A.lamI[f] = lamOf(s, a, phys(s, R.I[q][f], f), f);
      A.lamU0[f] = lamOf(s, a, phys(s, R.U0[f], f), f);
      A.lamAcc[f] = a->lam + (15 + size_t(f)) * N;
    }
    A.lamR = lamOf(s, a, phys(s, R.R[q], 0), 0);
    A.lamFpre = a->lamFpre;
    A.lamFnew = a->lamFnew;
    // the objective's adjoint (F_x of the step's result) joins the ghost phase of the last stage
    P.objective = (objective && q == 3) ? 1 : 0;
    for (int f = 0; f < 5; ++f) P.objVal[f] = S.result + f * N;
    P.nx = a->dNx;
    P.dA = a->dA;
    P.weight = 1.0 / a->navg;
    // near-body filter and ghosts
    P.ipbar = a->ipbar;
    P.cnode = a->cnode;
    P.coff = a->coff;
    P.cent = a->cent;
    P.ncell = a->ncell;
    P.fsNodes = a->fsNodes;
    P.fsSlots = a->fsSlots;
    P.nfs = a->nfs;
    // edge conditions: z, y, then x (reads the stage output before the edge conditions: its copy, or,
    // where the planes it reads are clean, the next stage's input / the step's result)
    for (int f = 0; f < 5; ++f) {
      if (!a->edgePlanesClean)
        P.edgeVal[f] = snap + (6 + f) * N;
      else if (q == 3)
        P.edgeVal[f] = S.result + f * N;
      else
        P.edgeVal[f] = S.stage + (q + 1) * per_stage(s) + f * N;
    }
    for (int axis = 0; axis < 3; ++axis) {
      P.edges[axis] = s->plan.edgeBlocks[axis];
      P.nEdge[axis] = s->plan.nEdgeBlocks[axis];
    }
    P.inletGather = a->inletX ? 1 : 0;
    P.fbar = a->fbar;
    P.lamInflow = a->lamInflow;
    P.roles = S.ctl;
    // stage kernel: RK4 combine and the RHS inputs (from the stage input's values), then the transposed RHS
    for (int f = 0; f < 5; ++f) A.val[f] = snap + f * N;
    A.valR = R.R[q] != R.I[q][0] ? snap + 5 * N : snap;
    A.valFpre = snap + 11 * N;
    P.solidMask = G.nSolid ? R.copyMask[q] : 0;
    P.lam = a->tmpLam;
    P.V = a->tmpV;
    P.sync = a->bcSync;
    P.bodyBlocks = a->bodiesClearOfFaces ? 1 : 0;
    P.timeout = a->dTimeout;
    launch_adj_bc(G, P, q, nSM, st);
    mark(PH_BC);
    launch_adj_rhs(s->dGrid, G, A, a->tmpLam, a->tmpV, nSM, st);
    mark(PH_RHS);
  }
  if (R.filterNow) {
    double* dst = lamOf(s, a, phys(s, R.gfDst, 0), 0);
    double* src = lamOf(s, a, phys(s, R.gfSrc, 0), 0);
    launch_adj_density_filter(s->dGrid, (long long)N, dst, dst, src, nSM, st);
    mark(PH_DFILTER);
  }
  CKA(cudaGetLastError());
  return NSF_OK;
}

// Everything the enqueued work of an adjoint step depends on besides fixed buffers.
std::vector<uintptr_t> role_key(const StepCtl& R, bool objective) {
  std::vector<uintptr_t> key;
  auto put = [&](const void* p) { key.push_back(reinterpret_cast<uintptr_t>(p)); };
  for (int q = 0; q < 4; ++q) {
    for (int f = 0; f < 5; ++f) {
      put(R.I[q][f]);
      put(R.O[q][f]);
    }
    put(R.R[q]);
    key.push_back(uintptr_t(R.copyMask[q]));
  }
  for (int f = 0; f < 5; ++f) put(R.U0[f]);
  key.push_back(uintptr_t(R.filterNow));
  put(R.filterNow ? R.gfSrc : nullptr);
  put(R.filterNow ? R.gfDst : nullptr);
  key.push_back(uintptr_t(objective));
  return key;
}

// A cached graph of one part of an adjoint step (0: recomputation, 1: adjoint kernels) for a role pattern
// and snapshot set, captured on `st` at first use.
nsf_status step_graph(nsf_solver* s, AdjCtx* a, int k, int part, int set, cudaStream_t st, cudaGraphExec_t* out) {
  const StepCtl& R = a->hist[k];
  const bool objective = k + 1 > a->nsteps - a->navg;
  auto key = role_key(R, objective);
  key.push_back(uintptr_t(part));
  key.push_back(uintptr_t(set));
  auto it = a->graphs.find(key);
  if (it == a->graphs.end()) {
    CKA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const nsf_status r = part == 0 ? enqueue_recompute(s, a, R, objective, set)
                                   : enqueue_adjoint_kernels(s, a, R, objective, snap_set(a, set), st);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (r != NSF_OK) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if (e != cudaSuccess) return fail(s, NSF_ERR_CUDA, std::string("adjoint step capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t x = nullptr;
    const cudaError_t e2 = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return fail(s, NSF_ERR_CUDA, std::string("adjoint step graph: ") + cudaGetErrorString(e2));
    it = a->graphs.emplace(key, x).first;
  }
  *out = it->second;
  return NSF_OK;
}

// The adjoint of step k, pipelined over two streams: the recomputation fills the next snapshot set on the
// solver's stream (after the adjoint kernels that last read that set are done), and the adjoint kernels
// read it on adjStream. The solver's stream then goes on with the schedule (restoring and advancing
// towards the step before) while those kernels run: every adjoint kernel reads only its set and fixed
// buffers, and only the adjoint kernels write the adjoint arrays, in step order on one stream.
nsf_status adjoint_step(nsf_solver* s, AdjCtx* a, int k) {
  const int j = a->nextSet;
  a->nextSet ^= 1;
  cudaGraphExec_t rec = nullptr, adj = nullptr;
  nsf_status st = step_graph(s, a, k, 0, j, s->stream, &rec);
  if (st == NSF_OK) st = step_graph(s, a, k, 1, j, a->adjStream, &adj);
  if (st != NSF_OK) return st;
  CKA(cudaStreamWaitEvent(s->stream, a->setFree[j], 0));
  CKA(cudaGraphLaunch(rec, s->stream));
  CKA(cudaEventRecord(a->setReady[j], s->stream));
  CKA(cudaStreamWaitEvent(a->adjStream, a->setReady[j], 0));
  CKA(cudaGraphLaunch(adj, a->adjStream));
  CKA(cudaEventRecord(a->setFree[j], a->adjStream));
  return NSF_OK;
}

// The backward run over the segment tape: segments last first; each restores its checkpoint and records
// its steps' sets with the tape step graph on the solver's stream (after the adjoint kernels that last read
// that part of the tape), then its adjoint kernels run on adjStream, last step first, reading the sets.
nsf_status reverse_segments(nsf_solver* s, AdjCtx* a) {
  const int L = a->segLen, H = a->tapeSets / L, M = (a->nsteps + L - 1) / L;
  nsf_status st;
  for (int m = M - 1; m >= 0; --m) {
    const int h = m % H, k0 = m * L, k1 = std::min(a->nsteps, k0 + L);
    CKA(cudaStreamWaitEvent(s->stream, a->setFree[h], 0));
    if ((st = restore(s, a, m)) != NSF_OK) return st;
    for (int k = k0; k < k1; ++k) CKA(cudaGraphLaunch(a->tapeExec, s->stream));
    CKA(cudaEventRecord(a->setReady[h], s->stream));
    CKA(cudaStreamWaitEvent(a->adjStream, a->setReady[h], 0));
    for (int k = k1 - 1; k >= k0; --k)
      if ((st = enqueue_adjoint_kernels(s, a, a->hist[k], k + 1 > a->nsteps - a->navg, tape_set(s, a, k),
                                        a->adjStream)) != NSF_OK)
        return st;
    CKA(cudaEventRecord(a->setFree[h], a->adjStream));
  }
  return NSF_OK;
}

double binom(int n, int k) {
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

int split(int a0, int b, int c) {
  const int n = b - a0;
  int t = 0;
  while (binom(c + t, t) < n) ++t;
  const int right = int(std::min<double>(binom(c - 1 + t, t), n - 1));
  return a0 + std::max(1, n - right);
}

// The checkpoints of the schedule's first descent (state at `level` into `slot`): the forward run stores
// them as it passes, so the backward run starts at the last step without recomputing.
std::vector<std::pair<int, int>> first_descent(int n, int c) {
  std::vector<std::pair<int, int>> out;
  int a0 = 0, depth = 0;
  while (n - a0 > 1 && c > 0) {
    a0 = split(a0, n, c);
    out.push_back({a0, ++depth});
    --c;
  }
  return out;
}

// Reverse steps [a0, b) with c free snapshot slots above `depth`; slot `depth` holds the state at a0.
// stored: the checkpoints of this call's first descent are already in their slots.
nsf_status reverse(nsf_solver* s, AdjCtx* a, int a0, int b, int c, int depth, bool stored = false) {
  nsf_status st;
  if (b - a0 == 1) {
    if ((st = restore(s, a, depth)) != NSF_OK) return st;
    return adjoint_step(s, a, a0);
  }
  if (c == 0) {
    for (int k = b - 1; k >= a0; --k) {
      if ((st = restore(s, a, depth)) != NSF_OK) return st;
      if ((st = advance(s, k - a0)) != NSF_OK) return st;
      if ((st = adjoint_step(s, a, k)) != NSF_OK) return st;
    }
    return NSF_OK;
  }
  const int m = split(a0, b, c);
  if (!stored) {
    if ((st = restore(s, a, depth)) != NSF_OK) return st;
    if ((st = advance(s, m - a0)) != NSF_OK) return st;
    if ((st = save(s, a, depth + 1)) != NSF_OK) return st;
  }
  if ((st = reverse(s, a, m, b, c - 1, depth + 1, stored)) != NSF_OK) return st;
  return reverse(s, a, a0, m, c, depth);
}

}  // namespace

void nsf_adjoint_free(nsf_solver* s) {
  if (!s || !s->adj) return;
  AdjCtx* a = s->adj;
  if (a->adjStream) cudaStreamSynchronize(a->adjStream);
  for (auto& kv : a->graphs) cudaGraphExecDestroy(kv.second);
  release_tape(a);
  for (int j = 0; j < 2; ++j) {
    if (a->setReady[j]) cudaEventDestroy(a->setReady[j]);
    if (a->setFree[j]) cudaEventDestroy(a->setFree[j]);
  }
  if (a->adjStream) cudaStreamDestroy(a->adjStream);
  for (void* p : a->allocs) cudaFree(p);
  delete s->adj;
  s->adj = nullptr;
}

extern "C" {

nsf_status nsf_adj_configure(nsf_solver* s, uint32_t avg_last_steps, uint32_t snapshots) {
  if (!s) return NSF_ERR_ARG;
  nsf_status st = setup(s);
  if (st != NSF_OK) return st;
  AdjCtx* a = s->adj;
  if (avg_last_steps == 0 || int(avg_last_steps) > a->nsteps || snapshots == 0 || snapshots > 4096)
    return fail(s, NSF_ERR_ARG, "nsf_adj_configure: 1 <= avg_last_steps <= steps and 1 <= snapshots <= 4096");
  if (int(avg_last_steps) != a->navg) {  // the graphs hold the objective's weight
    for (auto& kv : a->graphs) cudaGraphExecDestroy(kv.second);
    a->graphs.clear();
  }
  a->navg = int(avg_last_steps);
  if (int(snapshots) != a->nsnap) a->chainStored = a->segValid = false;
  a->nsnap = int(snapshots);
  return NSF_OK;
}

nsf_status nsf_adj_set_tape_limit(nsf_solver* s, uint64_t bytes) {
  if (!s) return NSF_ERR_ARG;
  nsf_status st = setup(s);
  if (st != NSF_OK) return st;
  AdjCtx* a = s->adj;
  a->tapeLimit = bytes;
  if (a->tape && bytes != UINT64_MAX && double(a->tapeSetWords) * 8.0 * a->tapeSets > double(bytes)) {
    CKA(cudaSetDevice(s->device));
    CKA(cudaStreamSynchronize(a->adjStream));
    CKA(cudaStreamSynchronize(s->stream));
    release_tape(a);
  }
  return NSF_OK;
}

nsf_status nsf_adj_tape_bytes(nsf_solver* s, uint64_t* bytes) {
  if (!s || !bytes) return NSF_ERR_ARG;
  const AdjCtx* a = s->adj;
  *bytes = a && a->tapeValid ? uint64_t(tape_set_words(s)) * 8u * uint64_t(a->nsteps) : 0u;
  return NSF_OK;
}

nsf_status nsf_adj_segment_tape(nsf_solver* s, uint64_t* bytes, uint32_t* segment_steps) {
  if (!s || !bytes || !segment_steps) return NSF_ERR_ARG;
  const AdjCtx* a = s->adj;
  const bool on = a && a->segValid && a->tape;
  *bytes = on ? uint64_t(a->tapeSetWords) * 8u * uint64_t(a->tapeSets) : 0u;
  *segment_steps = on ? uint32_t(a->segLen) : 0u;
  return NSF_OK;
}

nsf_status nsf_adj_forward(nsf_solver* s, const double* u0, const double* inflow, double* J) {
  if (!s || !J) return NSF_ERR_ARG;
  nsf_status st = setup(s);
  if (st != NSF_OK) return st;
  AdjCtx* a = s->adj;
  a->navg = std::min(a->navg, a->nsteps);
  if ((st = alloc_slots(s, a)) != NSF_OK) return st;
  const HostSetup& S = s->setup;
  Grid& G = s->hGrid;
  const size_t N = nd(s), hp = S.NK * sizeof(double), dp = size_t(G.NKp) * sizeof(double);
  CKA(cudaSetDevice(s->device));
  CKA(cudaStreamSynchronize(s->stream));
  if (u0) {
    CKA(cudaMemset(a->dU0, 0, 5 * N * sizeof(double)));
    for (int f = 0; f < 5; ++f)
      CKA(cudaMemcpy2D(a->dU0 + f * N, dp, u0 + f * S.N, hp, hp, S.NI * S.NJ, cudaMemcpyHostToDevice));
  }
  if (inflow) {
    CKA(cudaMemcpy2D(a->dInflow, dp, inflow, hp, hp, S.NJ, cudaMemcpyHostToDevice));
  } else {
    std::vector<double> ones(size_t(G.NJ) * G.NKp, 1.0);
    CKA(cudaMemcpy(a->dInflow, ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  G.inflow = a->dInflow;
  G.dtFrozen = a->haveDt ? a->dDt : nullptr;
  G.nDtFrozen = a->haveDt ? a->nsteps : 0;
  if ((st = push_grid(s)) != NSF_OK) return st;
  if ((st = reset(s, a)) != NSF_OK) return st;
  if ((st = save(s, a, 0)) != NSF_OK) return st;
  CKA(cudaMemsetAsync(a->dAcc, 0, sizeof(double), s->stream));
  int mode = TAPE_NONE;
  a->tapeValid = a->segValid = false;
  if ((st = prepare_tape(s, a, &mode)) != NSF_OK) return st;
  const bool tape = mode == TAPE_FULL;
  a->chain.clear();
  if (mode == TAPE_SEGMENTS)  // a checkpoint at the start of every segment (level 0 is in slot 0)
    for (int m = 1; m * a->segLen < a->nsteps; ++m) a->chain.push_back({m * a->segLen, m});
  else if (mode == TAPE_NONE)
    a->chain = first_descent(a->nsteps, a->nsnap);
  size_t next = 0;
  for (int n = 0; n < a->nsteps; ++n) {
    CKA(cudaGraphLaunch(tape ? a->tapeExec : s->graphExec, s->stream));
    if (n + 1 > a->nsteps - a->navg) launch_objective(s->dGrid, a->dNx, a->dA, 1.0 / a->navg, a->dAcc, s->stream);
    if (next < a->chain.size() && a->chain[next].first == n + 1)
      if ((st = save(s, a, a->chain[next++].second)) != NSF_OK) return st;
  }
  CKA(cudaGetLastError());
  if ((st = nsf_sync(s)) != NSF_OK) return st;
  CKA(cudaMemcpy(J, a->dAcc, sizeof(double), cudaMemcpyDeviceToHost));
  a->hist.resize(a->nsteps);
  CKA(cudaMemcpy(a->hist.data(), a->dHist, a->nsteps * sizeof(StepCtl), cudaMemcpyDeviceToHost));
  if (!a->haveDt) {  // freeze the dt sequence of this run
    std::vector<double> rows(7 * size_t(a->nsteps));
    uint64_t avail = 0;
    if ((st = nsf_get_history(s, 0, uint64_t(a->nsteps), rows.data(), &avail)) != NSF_OK) return st;
    a->dts.resize(a->nsteps);
    for (int n = 0; n < a->nsteps; ++n) a->dts[n] = rows[7 * size_t(n) + 1];
    CKA(cudaMemcpy(a->dDt, a->dts.data(), a->nsteps * sizeof(double), cudaMemcpyHostToDevice));
    a->haveDt = true;
    G.dtFrozen = a->dDt;
    G.nDtFrozen = a->nsteps;
    if ((st = push_grid(s)) != NSF_OK) return st;
  }
  a->haveForward = true;
  a->chainStored = mode == TAPE_NONE;
  a->tapeValid = tape;
  a->segValid = mode == TAPE_SEGMENTS;
  return NSF_OK;
}

nsf_status nsf_adj_backward(nsf_solver* s, double dJ, double* g_inflow, double* g_u0) {
  if (!s) return NSF_ERR_ARG;
  AdjCtx* a = s->adj;
  if (!a || !a->haveForward) return fail(s, NSF_ERR_STATE, "nsf_adj_backward needs a preceding nsf_adj_forward");
  const HostSetup& S = s->setup;
  const Grid& G = s->hGrid;
  const size_t N = nd(s), F = nf(s), plane = size_t(G.NJ) * G.NKp;
  CKA(cudaSetDevice(s->device));
  nsf_status st = alloc_slots(s, a);
  if (st != NSF_OK) return st;
  CKA(cudaMemsetAsync(a->lam, 0, 20 * N * sizeof(double), s->stream));
  if (F) {
    CKA(cudaMemsetAsync(a->lamFpre, 0, 2 * F * sizeof(double), s->stream));
    CKA(cudaMemsetAsync(a->lamFnew, 0, 2 * F * sizeof(double), s->stream));
  }
  CKA(cudaMemsetAsync(a->lamInflow, 0, plane * sizeof(double), s->stream));
  CKA(cudaMemsetAsync(a->fbar, 0, 2 * plane * sizeof(double), s->stream));
  CKA(cudaMemsetAsync(a->dTimeout, 0, sizeof(int), s->stream));
  CKA(cudaStreamSynchronize(s->stream));  // the adjoint kernels on adjStream start from these
  if (a->tapeValid) {  // every step's set is on the tape: the adjoint kernels alone, last step first
    for (int k = a->nsteps - 1; k >= 0 && st == NSF_OK; --k)
      st = enqueue_adjoint_kernels(s, a, a->hist[k], k + 1 > a->nsteps - a->navg, tape_set(s, a, k), a->adjStream);
  } else if (a->segValid && a->tape) {  // each segment recorded from its checkpoint, then its adjoint kernels
    st = reverse_segments(s, a);
  } else {
    st = reverse(s, a, 0, a->nsteps, a->nsnap, 0, a->chainStored);
    a->chainStored = false;  // the schedule has reused the slots
  }
  if (st != NSF_OK) {
    cudaStreamSynchronize(a->adjStream);
    return st;
  }
  // level-0 fpre was copied from U0
  launch_fpre_init_adj(s->dGrid, G.nFilter, a->lamFpre, lamOf(s, a, 0, 0), lamOf(s, a, 0, 4), s->nSM, a->adjStream);
  CKA(cudaStreamSynchronize(a->adjStream));
  CKA(cudaStreamSynchronize(s->stream));
  StepCtl ctl;
  int adjTimeout = 0;
  CKA(cudaMemcpy(&ctl, s->dCtl, sizeof ctl, cudaMemcpyDeviceToHost));
  CKA(cudaMemcpy(&adjTimeout, a->dTimeout, sizeof adjTimeout, cudaMemcpyDeviceToHost));
  if (ctl.timeout) return fail(s, NSF_ERR_TIMEOUT, "a bounded wait in the stage kernel gave up during the adjoint");
  if (adjTimeout) return fail(s, NSF_ERR_TIMEOUT, "a grid barrier of the adjoint boundary kernel gave up");
  const size_t hp = S.NK * sizeof(double), dp = size_t(G.NKp) * sizeof(double);
  if (g_u0) {
    for (int f = 0; f < 5; ++f)
      CKA(cudaMemcpy2D(g_u0 + f * S.N, hp, lamOf(s, a, 0, f), dp, hp, S.NI * S.NJ, cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < 5 * S.N; ++q) g_u0[q] *= dJ;
  }
  if (g_inflow) {
    CKA(cudaMemcpy2D(g_inflow, hp, a->lamInflow, dp, hp, S.NJ, cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < S.NJ * S.NK; ++q) g_inflow[q] *= dJ;
  }
  return NSF_OK;
}

nsf_status nsf_adj_profile_step(nsf_solver* s, uint64_t step, double* ms) {
  if (!s || !ms) return NSF_ERR_ARG;
  AdjCtx* a = s->adj;
  if (!a || !a->haveForward) return fail(s, NSF_ERR_STATE, "nsf_adj_profile_step needs a preceding nsf_adj_forward");
  if (step >= uint64_t(a->nsteps)) return fail(s, NSF_ERR_ARG, "nsf_adj_profile_step: step out of range");
  CKA(cudaSetDevice(s->device));
  // the state at `step`: from level 0 (slot 0 keeps it for the whole forward/backward cycle)
  nsf_status st = restore(s, a, 0);
  if (st == NSF_OK) st = advance(s, int(step));
  if (st != NSF_OK) return st;
  PhaseTimer pt{s->stream, {}, {}};  // both parts on the solver's stream, one after the other
  const bool objective = int(step) + 1 > a->nsteps - a->navg;
  CKA(cudaStreamSynchronize(a->adjStream));
  st = enqueue_recompute(s, a, a->hist[step], objective, 0, &pt);
  if (st == NSF_OK) st = enqueue_adjoint_kernels(s, a, a->hist[step], objective, snap_set(a, 0), s->stream, &pt);
  CKA(cudaStreamSynchronize(s->stream));
  for (int q = 0; q < PH_COUNT; ++q) ms[q] = 0;
  pt.collect(ms);
  return st;
}

nsf_status nsf_adj_get_dt(nsf_solver* s, double* dts, uint64_t* count) {
  if (!s || !count) return NSF_ERR_ARG;
  AdjCtx* a = s->adj;
  if (!a || !a->haveDt) return fail(s, NSF_ERR_STATE, "no frozen dt sequence yet (run nsf_adj_forward first)");
  *count = uint64_t(a->nsteps);
  if (dts) std::memcpy(dts, a->dts.data(), a->nsteps * sizeof(double));
  return NSF_OK;
}

}  // extern "C"
