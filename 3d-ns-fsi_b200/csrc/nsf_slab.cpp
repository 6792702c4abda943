// x-slab decomposition of one grid (i is the slowest index, so an i-plane is contiguous).
//
// The interior planes 1 .. NI-2 are split into P contiguous ranges; slab p owns its range (slab 0 also owns
// the x-min face plane, slab P-1 the x-max face plane) and holds one more plane on each side: a halo (a copy
// of the neighbour's plane) or, at the ends, its own x face. Each slab is an ordinary solver handle on its
// planes -- same kernels, same node classification restricted to the slab, its edge conditions clipped to
// the planes it owns -- so the stage kernel computes exactly the slab's interior planes. Per RK4 step:
//
//   prologue + density filter of every slab;  exchange of the filtered density's halo planes
//   4 x { stage kernel of every slab;
//         periodic x faces: plane NI-2 -> slab 0's x-min face plane, plane 1 -> slab P-1's x-max face plane
//           (the x faces' periodic copy, PeriodicBoundary, Boundary.cpp:344-367; the slabs' own edge
//           conditions then treat the face planes' y/z rows, which read those copies, as the reference does);
//         fused boundary kernel of every slab (no finalize);
//         halo exchange: each slab's first and last owned planes -> its neighbours' halo planes }
//   global reductions (dt maxima, change-norm sums) and the end of step of every slab.
//
// A group lives in one process or spans several (one GPU each, nsf_slab_group_create_ranks): rank r holds
// the consecutive slabs p with p * world / P == r. Each process's slabs share one device and one stream,
// and a step is one CUDA graph; a transfer packs the plane into a staging buffer and unpacks it on the
// receiving side (the buffers each step's roles select are read on the device) -- within a process the
// two sides share the buffer, across processes NCCL send/recv moves it (captured in the graph, between
// the pack and the unpack launches). The global reductions gather every slab's partials (NCCL all-gather
// across processes) and combine them in slab order, so every process computes the same dt and norms.
// The node values and the dt sequence equal the single-grid solve's bit for bit:
// every node's dt terms are formed by the same kernel as in the whole grid (the periodic x faces' by their
// edge items, BC_SLAB_COPY), and maxima do not depend on the order; the change norms are summed slab by slab,
// so they agree to rounding. Immersed bodies are not supported across slabs (NSF_ERR_ARG).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "nsf_internal.h"
#include "nsf_nccl.h"
#include "nsf_slab.h"
#include "nsf_solver_impl.h"

using namespace nsf;

struct nsf_slab_group {
  nsf_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  HostSetup whole;                 // the grid's own host setup (partition, downloads)
  int P = 0;                       // slabs of the whole group
  int rank = 0, world = 1;         // this process among the group's processes
  int first = 0;                   // global index of this process's first slab (slabs[l] is slab first + l)
  bool ncclAll = false;            // route transfers within this process through NCCL too (self send/recv)
  std::vector<nsf_solver*> slabs;  // this process's slabs
  std::vector<int> a, b;           // slab p's interior planes a[p] .. b[p] (global), every slab of the group
  std::vector<int> lo, hi;         // the global planes slab p owns: its interior planes, plus the x faces at the ends
  std::vector<int> base;           // global plane of slab p's local plane 0 (= a[p] - 1)
  bool xPeriodic = false;
  Grid* dGrids = nullptr;          // copies of this process's slabs' grids, device
  double* dPart = nullptr;         // [9 x local slabs] this process's slab partials
  double* dGather = nullptr;       // [9 x maxLocal x world] every process's partials (several processes)
  int* dAt = nullptr;              // [P] where slab p's partials are (in dPart, or in dGather)
  int maxLocal = 0;
  double* dRed = nullptr;          // [9] global dt maxima and norm sums
  // transfers: pack tasks (this process's sending side) and unpack tasks (its receiving side), per list
  std::vector<SlabTask> packStage, unpackStage, packWrap, unpackWrap, packFilter, unpackFilter;
  SlabTask* dTasks = nullptr;      // all task lists, device, in the order above
  size_t offs[7] = {0, 0, 0, 0, 0, 0, 0};
  // NCCL moves of each list (0 halos, 1 periodic x faces, 2 filtered density), in the group's global order
  struct Move {
    bool send;   // send (else receive)
    int peer;    // the other process
    double* buf;
    size_t words;
  };
  std::vector<Move> moves[3];
  void* comm = nullptr;            // ncclComm_t (several processes, or ncclAll)
  long long planeWords = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  int launchesPerStep = 0;
  std::vector<void*> allocs;
  std::string err;
};

namespace {

nsf_status gfail(nsf_slab_group* g, nsf_status st, const std::string& m) {
  g->err = m;
  return st;
}
#define CKG(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return gfail(g, NSF_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
nsf_status galloc(nsf_slab_group* g, T** p, size_t count) {
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess)
    return gfail(g, NSF_ERR_CUDA, "cudaMalloc failed (slab group)");
  g->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return NSF_OK;
}

// Host setup of slab p: the whole grid's planes base .. base + n - 1, edge conditions clipped to the planes
// the slab owns (the x faces' periodic copies come from the exchange instead), halo planes typed as edge
// nodes (no kernel computes or filters them; their values arrive from the neighbour).
void slab_setup(const nsf_slab_group* g, int p, HostSetup& S, std::vector<uint8_t>& flags) {
  const HostSetup& W = g->whole;
  const int P = int(g->lo.size());
  const int b0 = g->base[p], n = g->b[p] - g->a[p] + 3;
  const size_t plane = W.NJ * W.NK;
  S = HostSetup{};
  S.NI = size_t(n);
  S.NJ = W.NJ;
  S.NK = W.NK;
  S.N = S.NI * plane;
  std::memcpy(S.d, W.d, sizeof S.d);
  std::memcpy(S.off, W.off, sizeof S.off);
  S.type.assign(W.type.begin() + size_t(b0) * plane, W.type.begin() + size_t(b0 + n) * plane);
  flags.assign(S.N, 0);
  const int ownLo = p == 0 ? 0 : 1, ownHi = p == P - 1 ? n - 1 : n - 2;  // local planes the slab owns
  for (int li : {0, n - 1})
    if (li < ownLo || li > ownHi) {  // halo plane
      for (size_t q = 0; q < plane; ++q) {
        S.type[size_t(li) * plane + q] = FLUID_EDGE;
        flags[size_t(li) * plane + q] = EDGE_PLANE_BIT;
      }
    }
  for (const EdgeBC& e : W.edges) {
    // every node of the whole grid's edge planes keeps its edge-plane flag (the density filter copies them)
    for (size_t i = e.owned.i0; i <= e.owned.i1; ++i) {
      const int li = int(i) - b0;
      if (li < 0 || li >= n) continue;
      for (size_t j = e.owned.j0; j <= e.owned.j1; ++j)
        for (size_t k = e.owned.k0; k <= e.owned.k1; ++k) flags[size_t(li) * plane + j * W.NK + k] |= EDGE_PLANE_BIT;
    }
    const int i0 = std::max(int(e.owned.i0) - b0, ownLo), i1 = std::min(int(e.owned.i1) - b0, ownHi);
    if (i0 > i1) continue;
    EdgeBC c = e;
    // a periodic x face's values come from the exchange; its edge items only add the dt terms
    if (e.axis == 0 && e.bc == NSF_BC_PERIODIC) c.bc = BC_SLAB_COPY;
    c.owned.i0 = size_t(i0);
    c.owned.i1 = size_t(i1);
    S.edges.push_back(c);
  }
}

// The process that holds slab p: consecutive slabs per process, p * world / P.
int slab_owner(int p, int P, int world) { return int((long long)p * world / P); }

// One plane transfer of a step: list 0 halos (stage output), 1 periodic x faces (stage output), 2 the
// filtered density's halos; planes local to each slab (local plane l of slab p is global plane a[p] - 1 + l).
struct SlabXfer {
  int list, from, fromPlane, to, toPlane, which;
};

// Every transfer of a group, in the order every process walks them (NCCL pairs a process's sends to a peer
// with the peer's receives in issue order).
std::vector<SlabXfer> slab_transfers(const std::vector<int>& a, const std::vector<int>& b, bool xPeriodic) {
  const int P = int(a.size());
  std::vector<SlabXfer> out;
  auto n = [&](int p) { return b[size_t(p)] - a[size_t(p)] + 3; };  // local planes of slab p
  for (int which : {SLAB_STAGE, SLAB_FILTER})
    for (int p = 0; p + 1 < P; ++p) {  // last owned plane -> next slab's plane 0; first owned -> previous's last
      const int list = which == SLAB_STAGE ? 0 : 2;
      out.push_back(SlabXfer{list, p, n(p) - 2, p + 1, 0, which});
      out.push_back(SlabXfer{list, p + 1, 1, p, n(p) - 1, which});
    }
  if (xPeriodic) {  // global plane NI-2 -> slab 0's plane 0; global plane 1 -> slab P-1's last plane
    out.push_back(SlabXfer{1, P - 1, n(P - 1) - 2, 0, 0, SLAB_STAGE});
    out.push_back(SlabXfer{1, 0, 1, P - 1, n(P - 1) - 1, SLAB_STAGE});
  }
  return out;
}

// The partition of the interior planes 1 .. NI-2 into P near-equal ranges.
void slab_partition(const HostSetup& W, int P, std::vector<int>& a, std::vector<int>& b) {
  const int interior = int(W.NI) - 2;
  a.clear();
  b.clear();
  for (int p = 0; p < P; ++p) {
    a.push_back(1 + p * interior / P);
    b.push_back((p + 1) * interior / P);
  }
}

bool has_x_periodic(const HostSetup& W) {
  for (const EdgeBC& e : W.edges)
    if (e.axis == 0 && e.bc == NSF_BC_PERIODIC) return true;
  return false;
}

nsf_status build_group(nsf_slab_group* g, int P, const void* ncclId) {
  const nsf_config& cfg = g->cfg;
  std::string err;
  nsf_status st = build_setup(cfg, g->whole, err);
  if (st != NSF_OK) return gfail(g, st, err);
  const HostSetup& W = g->whole;
  if (!W.bodies.empty()) return gfail(g, NSF_ERR_ARG, "x-slab groups support grids without immersed bodies");
  const int interior = int(W.NI) - 2;
  if (P < 2 || interior < 2 * P) return gfail(g, NSF_ERR_ARG, "x-slabs: 2 <= slabs and at least 2 interior planes per slab");
  if (g->world < 1 || g->world > P || g->rank < 0 || g->rank >= g->world)
    return gfail(g, NSF_ERR_ARG, "x-slabs: 0 <= rank < world <= slabs");
  g->P = P;
  g->xPeriodic = has_x_periodic(W);
  slab_partition(W, P, g->a, g->b);
  for (int p = 0; p < P; ++p) {
    g->lo.push_back(p == 0 ? 0 : g->a[size_t(p)]);
    g->hi.push_back(p == P - 1 ? int(W.NI) - 1 : g->b[size_t(p)]);
    g->base.push_back(g->a[size_t(p)] - 1);
  }
  // this process's slabs, and the most any process holds
  std::vector<int> count(size_t(g->world), 0);
  for (int p = 0; p < P; ++p) ++count[size_t(slab_owner(p, P, g->world))];
  g->maxLocal = *std::max_element(count.begin(), count.end());
  g->first = 0;
  while (slab_owner(g->first, P, g->world) != g->rank) ++g->first;
  const int nLocal = count[size_t(g->rank)];
  const bool useNccl = g->world > 1 || g->ncclAll;
  const NcclApi* nccl = nullptr;
  if (useNccl) {
    std::string why;
    if (!(nccl = nccl_api(&why))) return gfail(g, NSF_ERR_CUDA, why);
    if (!ncclId) return gfail(g, NSF_ERR_ARG, "x-slabs over NCCL need the communicator id");
  }
  // the whole grid's initial condition, sliced per slab; its initial dt for every slab
  std::vector<double> cons, prim;
  initial_condition(cfg, W, cons, prim);
  const double dt0 = nsf_initial_dt(cfg, W, cons, prim);
  const size_t plane = W.NJ * W.NK;
  CKG(cudaSetDevice(g->device));
  for (int p = g->first; p < g->first + nLocal; ++p) {
    nsf_solver* s = nullptr;
    st = nsf_create(&cfg, g->device, &s);
    if (st != NSF_OK) {
      if (s) nsf_destroy(s);
      return gfail(g, st, "slab solver");
    }
    s->grouped = true;
    g->slabs.push_back(s);
    slab_setup(g, p, s->setup, s->slabFlags);
    const size_t n = s->setup.NI, N = s->setup.N;
    s->slabCons.resize(5 * N);
    s->slabPrim.resize(7 * N);
    for (int f = 0; f < 5; ++f)
      std::memcpy(s->slabCons.data() + f * N, cons.data() + f * W.N + size_t(g->base[p]) * plane, N * sizeof(double));
    for (int f = 0; f < 7; ++f)
      std::memcpy(s->slabPrim.data() + f * N, prim.data() + f * W.N + size_t(g->base[p]) * plane, N * sizeof(double));
    (void)n;
    st = nsf_build_device(s);
    if (st != NSF_OK) return gfail(g, st, "slab " + std::to_string(p) + ": " + s->err);
    s->initialized = true;
    s->ctlInit.dt = dt0;
    CKG(cudaMemcpy(&s->dCtl->dt, &dt0, sizeof dt0, cudaMemcpyHostToDevice));
    s->slabCons.clear();
    s->slabPrim.clear();
  }
  // device copies of the slabs' grids (the reductions read them)
  std::vector<Grid> hg;
  for (nsf_solver* s : g->slabs) hg.push_back(s->hGrid);
  if ((st = galloc(g, &g->dGrids, hg.size())) != NSF_OK) return st;
  CKG(cudaMemcpy(g->dGrids, hg.data(), hg.size() * sizeof(Grid), cudaMemcpyHostToDevice));
  if ((st = galloc(g, &g->dRed, 9)) != NSF_OK) return st;
  if ((st = galloc(g, &g->dPart, size_t(9) * size_t(g->maxLocal))) != NSF_OK) return st;
  CKG(cudaMemset(g->dPart, 0, size_t(9) * size_t(g->maxLocal) * sizeof(double)));
  {  // where each slab's partials are read: this process's own (one process), or the gathered copies
    std::vector<int> at(static_cast<size_t>(P));
    std::vector<int> firstOf(size_t(g->world), -1);
    for (int p = 0; p < P; ++p) {
      const int r = slab_owner(p, P, g->world);
      if (firstOf[size_t(r)] < 0) firstOf[size_t(r)] = p;
      at[size_t(p)] = useNccl ? r * g->maxLocal + (p - firstOf[size_t(r)]) : p;
    }
    if ((st = galloc(g, &g->dAt, at.size())) != NSF_OK) return st;
    CKG(cudaMemcpy(g->dAt, at.data(), at.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (useNccl && (st = galloc(g, &g->dGather, size_t(9) * g->maxLocal * g->world)) != NSF_OK) return st;
  }
  // transfers, in the group's global order: within this process one staging buffer per transfer (pack and
  // unpack share it); across processes (or all of them with ncclAll) a send buffer on the sending side and
  // a receive buffer on the receiving side, moved by NCCL
  g->planeWords = g->slabs[0]->hGrid.sI;
  auto local = [&](int p) { return slab_owner(p, P, g->world) == g->rank; };
  auto gridOf = [&](int p) { return g->slabs[size_t(p - g->first)]->dGrid; };
  for (const SlabXfer& x : slab_transfers(g->a, g->b, g->xPeriodic)) {
    auto& pk = x.list == 0 ? g->packStage : x.list == 1 ? g->packWrap : g->packFilter;
    auto& up = x.list == 0 ? g->unpackStage : x.list == 1 ? g->unpackWrap : g->unpackFilter;
    const size_t words = size_t(x.which == SLAB_STAGE ? 5 : 1) * size_t(g->planeWords);
    const bool fromHere = local(x.from), toHere = local(x.to);
    if (fromHere && toHere && !g->ncclAll) {
      double* buf = nullptr;
      if ((st = galloc(g, &buf, words)) != NSF_OK) return st;
      pk.push_back(SlabTask{gridOf(x.from), x.fromPlane, x.which, buf});
      up.push_back(SlabTask{gridOf(x.to), x.toPlane, x.which, buf});
      continue;
    }
    if (fromHere) {
      double* buf = nullptr;
      if ((st = galloc(g, &buf, words)) != NSF_OK) return st;
      pk.push_back(SlabTask{gridOf(x.from), x.fromPlane, x.which, buf});
      g->moves[x.list].push_back(nsf_slab_group::Move{true, slab_owner(x.to, P, g->world), buf, words});
    }
    if (toHere) {
      double* buf = nullptr;
      if ((st = galloc(g, &buf, words)) != NSF_OK) return st;
      up.push_back(SlabTask{gridOf(x.to), x.toPlane, x.which, buf});
      g->moves[x.list].push_back(nsf_slab_group::Move{false, slab_owner(x.from, P, g->world), buf, words});
    }
  }
  if (useNccl) {  // the communicator (every process of the group joins here)
    ncclUniqueId id;
    std::memcpy(&id, ncclId, sizeof id);
    ncclComm_t comm = nullptr;
    const ncclResult_t r = nccl->commInitRank(&comm, g->world, id, g->rank);
    if (r != ncclSuccess) return gfail(g, NSF_ERR_CUDA, std::string("ncclCommInitRank: ") + nccl->errorString(r));
    g->comm = comm;
  }
  std::vector<SlabTask> all;
  const std::vector<SlabTask>* lists[6] = {&g->packStage, &g->unpackStage, &g->packWrap, &g->unpackWrap,
                                           &g->packFilter, &g->unpackFilter};
  for (int q = 0; q < 6; ++q) {
    g->offs[q] = all.size();
    all.insert(all.end(), lists[q]->begin(), lists[q]->end());
  }
  g->offs[6] = all.size();
  if ((st = galloc(g, &g->dTasks, all.size())) != NSF_OK) return st;
  CKG(cudaMemcpy(g->dTasks, all.data(), all.size() * sizeof(SlabTask), cudaMemcpyHostToDevice));
  CKG(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  CKG(cudaDeviceSynchronize());
  // one step as a CUDA graph
  CKG(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
  int launches = 0;
  auto copies = [&](int list, int s, int dir) {
    const int n = int(g->offs[list + 1] - g->offs[list]);
    if (n > 0) {
      launch_slab_copy(g->dTasks + g->offs[list], n, g->planeWords, s, dir, g->stream);
      ++launches;
    }
  };
  ncclResult_t nr = ncclSuccess;
  auto move = [&](int list) {  // this process's NCCL sends and receives of one list, as one group
    if (g->moves[list].empty() || nr != ncclSuccess) return;
    const ncclComm_t comm = static_cast<ncclComm_t>(g->comm);
    nr = nccl->groupStart();
    for (const auto& m : g->moves[list]) {
      if (nr != ncclSuccess) break;
      nr = m.send ? nccl->send(m.buf, m.words, ncclDouble, m.peer, comm, g->stream)
                  : nccl->recv(m.buf, m.words, ncclDouble, m.peer, comm, g->stream);
    }
    const ncclResult_t e = nccl->groupEnd();
    if (nr == ncclSuccess) nr = e;
  };
  for (nsf_solver* s : g->slabs) launches += enqueue_step_begin(s->dGrid, s->plan, g->stream);
  copies(4, 0, 0);  // filtered density halos (filter steps)
  move(2);
  copies(5, 0, 1);
  for (int q = 0; q < 4; ++q) {
    for (nsf_solver* s : g->slabs) {
      launch_stage(s->hGrid, s->plan, q, g->stream);
      ++launches;
    }
    copies(2, q, 0);  // periodic x faces
    move(1);
    copies(3, q, 1);
    for (nsf_solver* s : g->slabs) launches += launch_bc_part(s->dGrid, s->plan, q, false, g->stream);
    copies(0, q, 0);  // halos
    move(0);
    copies(1, q, 1);
  }
  launch_slab_partials(g->dGrids, nLocal, g->dPart, g->stream);
  if (useNccl && nr == ncclSuccess)
    nr = nccl->allGather(g->dPart, g->dGather, size_t(9) * g->maxLocal, ncclDouble, static_cast<ncclComm_t>(g->comm),
                         g->stream);
  launch_slab_combine(useNccl ? g->dGather : g->dPart, g->dAt, P, g->dRed, g->stream);
  launch_slab_finalize(g->dGrids, nLocal, g->dRed, g->stream);
  launches += 3;
  if (nr != ncclSuccess) {
    cudaGraph_t dropped = nullptr;
    cudaStreamEndCapture(g->stream, &dropped);
    if (dropped) cudaGraphDestroy(dropped);
    return gfail(g, NSF_ERR_CUDA, std::string("NCCL in the slab step: ") + nccl->errorString(nr));
  }
  const cudaError_t e1 = cudaGetLastError();
  const cudaError_t e2 = cudaStreamEndCapture(g->stream, &g->graph);
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return gfail(g, NSF_ERR_CUDA, std::string("slab step capture: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  CKG(cudaGraphInstantiate(&g->graphExec, g->graph, 0));
  g->launchesPerStep = launches;
  return NSF_OK;
}

}  // namespace

extern "C" {

nsf_status nsf_slab_plan(const nsf_config* cfg, int32_t nslabs, int32_t* first, int32_t* last) {
  if (!cfg || !first || !last || nslabs < 2) return NSF_ERR_ARG;
  const int interior = int(cfg->NI) - 2;
  if (interior < 2 * nslabs) return NSF_ERR_ARG;
  for (int p = 0; p < nslabs; ++p) {
    first[p] = 1 + p * interior / nslabs;
    last[p] = (p + 1) * interior / nslabs;
  }
  return NSF_OK;
}

nsf_status nsf_slab_group_create(const nsf_config* cfg, int32_t nslabs, int32_t device, nsf_slab_group** out) {
  if (!cfg || !out || device < 0) return NSF_ERR_ARG;
  *out = nullptr;
  auto* g = new nsf_slab_group;
  g->cfg = *cfg;
  g->device = device;
  nsf_status st = build_group(g, nslabs, nullptr);
  *out = g;
  return st;
}

nsf_status nsf_slab_nccl_id(uint8_t* id) {
  if (!id) return NSF_ERR_ARG;
  const NcclApi* nccl = nccl_api(nullptr);
  if (!nccl) return NSF_ERR_CUDA;
  ncclUniqueId u;
  if (nccl->getUniqueId(&u) != ncclSuccess) return NSF_ERR_CUDA;
  static_assert(sizeof(u) == NSF_NCCL_ID_BYTES, "NCCL unique id size");
  std::memcpy(id, &u, sizeof u);
  return NSF_OK;
}

nsf_status nsf_slab_group_create_ranks(const nsf_config* cfg, int32_t nslabs, int32_t rank, int32_t world,
                                       const uint8_t* nccl_id, int32_t flags, int32_t device, nsf_slab_group** out) {
  if (!cfg || !out || !nccl_id || device < 0) return NSF_ERR_ARG;
  *out = nullptr;
  auto* g = new nsf_slab_group;
  g->cfg = *cfg;
  g->device = device;
  g->rank = rank;
  g->world = world;
  g->ncclAll = (flags & NSF_SLAB_NCCL_ALL) != 0;
  nsf_status st = build_group(g, nslabs, nccl_id);
  *out = g;
  return st;
}

nsf_status nsf_slab_schedule(const nsf_config* cfg, int32_t nslabs, int32_t world, int32_t* owner,
                             int32_t* transfers, int32_t* count) {
  if (!cfg || !count || nslabs < 2 || world < 1 || world > nslabs) return NSF_ERR_ARG;
  HostSetup W;
  std::string err;
  const nsf_status st = build_setup(*cfg, W, err);
  if (st != NSF_OK) return st;
  if (int(W.NI) - 2 < 2 * nslabs) return NSF_ERR_ARG;
  std::vector<int> a, b;
  slab_partition(W, nslabs, a, b);
  if (owner)
    for (int p = 0; p < nslabs; ++p) owner[p] = slab_owner(p, nslabs, world);
  const std::vector<SlabXfer> xs = slab_transfers(a, b, has_x_periodic(W));
  const int cap = *count;
  *count = int32_t(xs.size());
  if (transfers && cap >= int(xs.size()))
    for (size_t q = 0; q < xs.size(); ++q) {
      int32_t* t = transfers + 5 * q;
      t[0] = xs[q].list;
      t[1] = xs[q].from;
      t[2] = a[size_t(xs[q].from)] - 1 + xs[q].fromPlane;
      t[3] = xs[q].to;
      t[4] = a[size_t(xs[q].to)] - 1 + xs[q].toPlane;
    }
  return NSF_OK;
}

nsf_status nsf_slab_group_march(nsf_slab_group* g, uint64_t nsteps) {
  if (!g) return NSF_ERR_ARG;
  if (!g->graphExec) return NSF_ERR_STATE;
  CKG(cudaSetDevice(g->device));
  for (uint64_t q = 0; q < nsteps; ++q) CKG(cudaGraphLaunch(g->graphExec, g->stream));
  return NSF_OK;
}

nsf_status nsf_slab_group_march_timed(nsf_slab_group* g, uint64_t nsteps, double* elapsed_ms) {
  if (!g || !elapsed_ms) return NSF_ERR_ARG;
  if (!g->graphExec) return NSF_ERR_STATE;
  CKG(cudaSetDevice(g->device));
  cudaEvent_t a, b;
  CKG(cudaEventCreate(&a));
  CKG(cudaEventCreate(&b));
  CKG(cudaEventRecord(a, g->stream));
  for (uint64_t q = 0; q < nsteps; ++q) CKG(cudaGraphLaunch(g->graphExec, g->stream));
  CKG(cudaEventRecord(b, g->stream));
  CKG(cudaEventSynchronize(b));
  float ms = 0;
  CKG(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *elapsed_ms = ms;
  return NSF_OK;
}

nsf_status nsf_slab_group_sync(nsf_slab_group* g) {
  if (!g) return NSF_ERR_ARG;
  if (!g->graphExec) return NSF_ERR_STATE;
  CKG(cudaSetDevice(g->device));
  CKG(cudaStreamSynchronize(g->stream));
  nsf_status worst = NSF_OK;
  for (nsf_solver* s : g->slabs) {
    const nsf_status st = nsf_sync(s);
    if (st == NSF_ERR_TIMEOUT) return gfail(g, st, s->err);
    if (st != NSF_OK) {
      worst = st;
      g->err = s->err;
    }
  }
  return worst;
}

nsf_status nsf_slab_group_solver(nsf_slab_group* g, int32_t slab, nsf_solver** s) {
  if (!g || !s || slab < 0 || slab >= int32_t(g->slabs.size())) return NSF_ERR_ARG;
  CKG(cudaSetDevice(g->device));
  CKG(cudaStreamSynchronize(g->stream));
  *s = g->slabs[size_t(slab)];
  return NSF_OK;
}

nsf_status nsf_slab_group_info(nsf_slab_group* g, int32_t* nslabs, int32_t* first_planes, uint64_t* launches_per_step) {
  if (!g) return NSF_ERR_ARG;
  if (nslabs) *nslabs = int32_t(g->slabs.size());
  if (first_planes)
    for (size_t l = 0; l < g->slabs.size(); ++l) first_planes[l] = g->lo[size_t(g->first) + l];
  if (launches_per_step) *launches_per_step = uint64_t(g->launchesPerStep);
  return NSF_OK;
}

nsf_status nsf_slab_group_download(nsf_slab_group* g, uint32_t mask, double* host) {
  if (!g || !host || g->slabs.empty()) return NSF_ERR_ARG;
  CKG(cudaSetDevice(g->device));
  CKG(cudaStreamSynchronize(g->stream));
  const HostSetup& W = g->whole;
  const size_t plane = W.NJ * W.NK;
  int nf = 0;
  for (int f = 0; f < NSF_NUM_FIELDS; ++f) nf += (mask >> f) & 1;
  for (size_t l = 0; l < g->slabs.size(); ++l) {
    const size_t p = size_t(g->first) + l;
    nsf_solver* s = g->slabs[l];
    std::vector<double> loc(size_t(nf) * s->setup.N);
    const nsf_status st = nsf_download(s, mask, loc.data());
    if (st != NSF_OK) return gfail(g, st, s->err);
    const int b0 = g->base[p];
    for (int q = 0; q < nf; ++q)
      for (int i = g->lo[p]; i <= g->hi[p]; ++i)
        std::memcpy(host + size_t(q) * W.N + size_t(i) * plane, loc.data() + size_t(q) * s->setup.N + size_t(i - b0) * plane,
                    plane * sizeof(double));
  }
  return NSF_OK;
}

const char* nsf_slab_group_last_error(nsf_slab_group* g) { return g ? g->err.c_str() : "null slab group"; }

void nsf_slab_group_destroy(nsf_slab_group* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->graphExec) cudaGraphExecDestroy(g->graphExec);  // the graph holds NCCL work: before the communicator
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->comm) {
    const NcclApi* nccl = nccl_api(nullptr);
    if (nccl) nccl->commDestroy(static_cast<ncclComm_t>(g->comm));
  }
  for (nsf_solver* s : g->slabs) nsf_destroy(s);
  for (void* p : g->allocs) cudaFree(p);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

}  // extern "C"
