// Ensembles of independent grids advanced together (C ABI, include/nsfsi.h: nsf_ensemble_*), and the
// stage-kernel autotuner (nsf_autotune).
//
// Every member is an ordinary solver handle (host setup, device fields, TMA descriptors, lists); the
// ensemble adds one combined launch plan and captures ONE CUDA graph per RK4 step for all members: the
// small kernels carry the member in a grid dimension and each of the four stage launches is a single
// persistent kernel over the union of the members' work items (a tile and a chunk of i-planes each),
// distributed over the CTAs by longest-processing-time-first. The reference has no counterpart; each
// member advances exactly as Solver::marchTimeStep (Solver.cpp:130-167) advances its own grid.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_solver_impl.h"

using namespace nsf;

struct nsf_ensemble {
  int device = 0;
  int nSM = 0;
  cudaStream_t stream = nullptr;
  std::vector<nsf_solver*> members;
  std::vector<Grid> hGrids;
  Grid* dGrids = nullptr;
  LaunchPlan plan{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  int launchesPerStep = 0;
  std::vector<void*> allocs;
  std::string err;
  int tile = STAGE_TILE_32x8;
  int forceTile = -1;  // >= 0: this tile shape, no tuning (the tuner's own ensembles)
};

namespace {

#define CKE(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      e->err = std::string(#call) + ": " + cudaGetErrorString(e_);         \
      return NSF_ERR_CUDA;                                                 \
    }                                                                      \
  } while (0)

template <class T>
nsf_status ens_alloc(nsf_ensemble* e, T** p, size_t count) {
  void* q = nullptr;
  CKE(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  e->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return NSF_OK;
}

// Work items of one member: TJ x TK tiles of its interior columns and chunks of `len` i-planes.
void member_items(const HostSetup& S, int g, int TJ, int TK, int len, std::vector<StageItem>& out) {
  const int nj = int((S.NJ - 2 + TJ - 1) / TJ), nk = int((S.NK - 2 + TK - 1) / TK), planes = int(S.NI - 2);
  for (int c0 = 1; c0 <= planes; c0 += len)
    for (int tj = 0; tj < nj; ++tj)
      for (int tk = 0; tk < nk; ++tk)
        out.push_back(StageItem{1 + tj * TJ, 1 + tk * TK, c0, std::min(planes, c0 + len - 1), g});
}

// Longest processing time first: items sorted by cost (planes streamed, i.e. chunk + 2 halo planes)
// go one by one to the least-loaded CTA. Returns the makespan; fills the per-CTA ordered list.
double lpt(std::vector<StageItem> items, int ctas, std::vector<StageItem>& ordered, std::vector<int>& start) {
  auto cost = [](const StageItem& w) { return double(w.i1 - w.i0 + 3); };
  std::stable_sort(items.begin(), items.end(), [&](const StageItem& a, const StageItem& b) { return cost(a) > cost(b); });
  std::vector<double> load(ctas, 0.0);
  std::vector<std::vector<StageItem>> per(ctas);
  for (const StageItem& w : items) {
    const int b = int(std::min_element(load.begin(), load.end()) - load.begin());
    load[b] += cost(w);
    per[b].push_back(w);
  }
  ordered.clear();
  start.assign(1, 0);
  for (auto& v : per) {
    ordered.insert(ordered.end(), v.begin(), v.end());
    start.push_back(int(ordered.size()));
  }
  return *std::max_element(load.begin(), load.end());
}

// ------------------------------------------------------------------------------------------- autotune
std::string device_name(int device) {
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown";
  std::string n = p.name;
  for (char& c : n)
    if (c == ' ' || c == '"') c = '_';
  return n;
}

std::string shape_key(int device, const nsf_config& c) {
  std::ostringstream k;
  k << device_name(device) << "/" << c.NI << "x" << c.NJ << "x" << c.NK;
  return k.str();
}

struct Tuned {
  int tile = STAGE_TILE_32x8;
  double nsPerNode[2] = {0, 0};  // mean stage-kernel time per node and stage, per tile shape
};

// Cache file: one JSON object per line, {"key": "...", "tile": t, "ns_per_node": [a, b]}.
bool cache_lookup(const char* path, const std::string& key, Tuned& out) {
  if (!path) return false;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    const std::string tag = "\"key\": \"" + key + "\"";
    if (line.find(tag) == std::string::npos) continue;
    const size_t pt = line.find("\"tile\": "), pn = line.find("\"ns_per_node\": [");
    if (pt == std::string::npos || pn == std::string::npos) continue;
    out.tile = std::atoi(line.c_str() + pt + 8);
    if (std::sscanf(line.c_str() + pn + 16, "%lf, %lf", &out.nsPerNode[0], &out.nsPerNode[1]) != 2) continue;
    return true;
  }
  return false;
}

void cache_store(const char* path, const std::string& key, const Tuned& t) {
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  char buf[512];
  std::snprintf(buf, sizeof buf, "{\"key\": \"%s\", \"tile\": %d, \"ns_per_node\": [%.6g, %.6g]}\n", key.c_str(), t.tile,
                t.nsPerNode[0], t.nsPerNode[1]);
  f << buf;
}

// Time the stage kernels of a solo solver of this configuration for each tile shape.
nsf_status tune(const nsf_config& cfg, int device, const char* cache, Tuned& out, std::string& err) {
  const std::string key = shape_key(device, cfg);
  if (cache_lookup(cache, key, out)) return NSF_OK;
  const double nodes = double(cfg.NI) * double(cfg.NJ) * double(cfg.NK);
  for (int tile = 0; tile < 2; ++tile) {
    nsf_solver* s = nullptr;
    nsf_status st = nsf_create(&cfg, device, &s);
    if (st == NSF_OK) {
      s->tileRequest = tile;
      st = nsf_initialize(s);
    }
    double stage[4] = {0, 0, 0, 0}, step = 0;
    if (st == NSF_OK) st = nsf_profile_steps(s, 2, stage, &step);
    if (st == NSF_OK) st = nsf_profile_steps(s, 4, stage, &step);
    if (st != NSF_OK) {
      err = std::string("autotune: ") + (s ? nsf_last_error(s) : "nsf_create failed");
      nsf_destroy(s);
      return st;
    }
    nsf_destroy(s);
    out.nsPerNode[tile] = 1e6 * (stage[0] + stage[1] + stage[2] + stage[3]) / 4 / nodes;
  }
  out.tile = out.nsPerNode[1] < out.nsPerNode[0] ? STAGE_TILE_16x16 : STAGE_TILE_32x8;
  cache_store(cache, key, out);
  return NSF_OK;
}

nsf_status create_ensemble(const nsf_config* cfgs, uint32_t n, int32_t device, const char* tune_cache, int forceTile,
                           nsf_ensemble** out);

// The ensemble's tile shape: the stage kernels of throwaway ensembles of the same members are timed with
// each tile shape (the ensemble kernel's cost per node depends on the mix of members, not only on each
// member's shape). Cached per device and composition under "<device>/ensemble/<count>x<NI>x<NJ>x<NK>+...".
nsf_status tune_ensemble(const nsf_config* cfgs, uint32_t n, int device, const char* cache, Tuned& out,
                         std::string& err) {
  std::map<std::string, int> shapes;
  double nodes = 0;
  for (uint32_t m = 0; m < n; ++m) {
    std::ostringstream k;
    k << cfgs[m].NI << "x" << cfgs[m].NJ << "x" << cfgs[m].NK;
    ++shapes[k.str()];
    nodes += double(cfgs[m].NI) * double(cfgs[m].NJ) * double(cfgs[m].NK);
  }
  std::ostringstream k;
  k << device_name(device) << "/ensemble/";
  bool first = true;
  for (const auto& kv : shapes) {
    k << (first ? "" : "+") << kv.second << "x" << kv.first;
    first = false;
  }
  const std::string key = k.str();
  if (cache_lookup(cache, key, out)) return NSF_OK;
  for (int tile = 0; tile < 2; ++tile) {
    nsf_ensemble* t = nullptr;
    nsf_status st = create_ensemble(cfgs, n, device, nullptr, tile, &t);
    double stage[4] = {0, 0, 0, 0}, step = 0;
    if (st == NSF_OK) st = nsf_ensemble_profile_steps(t, 2, stage, &step);
    if (st == NSF_OK) st = nsf_ensemble_profile_steps(t, 4, stage, &step);
    if (st != NSF_OK) {
      err = std::string("ensemble autotune: ") + (t ? t->err : std::string("create failed"));
      nsf_ensemble_destroy(t);
      return st;
    }
    nsf_ensemble_destroy(t);
    out.nsPerNode[tile] = 1e6 * (stage[0] + stage[1] + stage[2] + stage[3]) / 4 / nodes;
  }
  out.tile = out.nsPerNode[1] < out.nsPerNode[0] ? STAGE_TILE_16x16 : STAGE_TILE_32x8;
  cache_store(cache, key, out);
  return NSF_OK;
}

nsf_status build_ensemble(nsf_ensemble* e, const char* cache) {
  const int M = int(e->members.size());
  // tile shape: chosen by create_ensemble (forced or tuned), 32 x 8 without a cache
  (void)cache;
  if (e->forceTile >= 0) e->tile = e->forceTile;
  // members: ordinary solver handles on this device with the chosen tile shape
  for (nsf_solver* s : e->members) {
    s->tileRequest = e->tile;
    nsf_status st = nsf_initialize(s);
    if (st != NSF_OK) {
      e->err = "ensemble member: " + s->err;
      return st;
    }
  }
  CKE(cudaSetDevice(e->device));
  CKE(cudaDeviceSynchronize());
  LaunchPlan& L = e->plan;
  L = LaunchPlan{};
  L.nSM = e->nSM;
  L.tile = e->tile;
  const int TJ = stage_tile_j(e->tile), TK = stage_tile_k(e->tile);
  const int ctas = e->nSM * std::max(1, stage_occupancy(e->tile));
  // chunk length (planes per item, the same for every member): the one with the smallest LPT makespan
  int maxPlanes = 1;
  for (nsf_solver* s : e->members) maxPlanes = std::max(maxPlanes, int(s->setup.NI) - 2);
  std::vector<StageItem> ordered;
  std::vector<int> start;
  double best = 1e300;
  int bestLen = maxPlanes;
  for (int len = maxPlanes; len >= 4; len = len > 16 ? len - 4 : len - 2) {
    std::vector<StageItem> items;
    for (int g = 0; g < M; ++g) member_items(e->members[g]->setup, g, TJ, TK, len, items);
    std::vector<StageItem> o;
    std::vector<int> st;
    const double span = lpt(items, std::min(ctas, int(items.size())), o, st);
    if (span < best - 1e-9) {
      best = span;
      bestLen = len;
      ordered.swap(o);
      start.swap(st);
    }
  }
  (void)bestLen;
  L.nItems = int(ordered.size());
  L.stageBlocks = int(start.size()) - 1;
  nsf_status st;
  if ((st = ens_alloc(e, &L.items, ordered.size())) != NSF_OK) return st;
  CKE(cudaMemcpy(L.items, ordered.data(), ordered.size() * sizeof(StageItem), cudaMemcpyHostToDevice));
  if ((st = ens_alloc(e, &L.ctaStart, start.size())) != NSF_OK) return st;
  CKE(cudaMemcpy(L.ctaStart, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
  // small kernels: block counts = maxima over the members
  L.gfBlocks = std::max(8, 4 * e->nSM / M);  // grid-stride over each member's nodes
  for (int a = 0; a < 3; ++a) {  // edge blocks: every member's own, member-major
    std::vector<EdgeBlock> eb;
    for (int g = 0; g < M; ++g) edge_blocks(e->members[g]->hGrid, e->members[g]->typeFlags.data(), g, a, eb);
    L.nEdgeBlocks[a] = int(eb.size());
    L.edgeBlocks[a] = nullptr;
    if (eb.empty()) continue;
    if ((st = ens_alloc(e, &L.edgeBlocks[a], eb.size())) != NSF_OK) return st;
    CKE(cudaMemcpy(L.edgeBlocks[a], eb.data(), eb.size() * sizeof(EdgeBlock), cudaMemcpyHostToDevice));
  }
  for (nsf_solver* s : e->members) {
    const LaunchPlan& P = s->plan;
    L.filterBlocks = std::max(L.filterBlocks, P.filterBlocks);
    L.ghostBlocks = std::max(L.ghostBlocks, P.ghostBlocks);
    L.solidBlocks = std::max(L.solidBlocks, P.solidBlocks);
    L.hasFilter |= P.hasFilter;
    L.hasGhostWork |= P.hasGhostWork;
    L.hasSolid |= P.hasSolid;
  }
  {  // fused boundary kernel: bcBlocks blocks per member, all members' blocks resident at once
    std::vector<const BcMemberLevels*> lv;
    for (nsf_solver* s : e->members) lv.push_back(&s->bcLevels);
    BcFlat fl;
    bc_flatten(lv, fl);
    const std::vector<int> ranges = bc_block_ranges(fl, bc_capacity(e->nSM));
    L.bcBlocks = ranges.empty() ? 0 : ranges.back();
    L.bcLevels = fl.levels;
    if (L.bcBlocks == 0)
      for (nsf_solver* s : e->members)
        if (s->setup.bodiesInteract) {
          e->err = "ensemble members with interacting immersed bodies need the fused boundary kernel, and the "
                   "members do not fit one launch of it";
          return NSF_ERR_GEOMETRY;
        }
    if (L.bcBlocks > 0) {
      int widest = 1;  // the most blocks one member has: its norm slots
      for (int g = 0; g < M; ++g) widest = std::max(widest, ranges[size_t(g) + 1] - ranges[size_t(g)]);
      L.filterBlocks = std::max(L.filterBlocks, widest);
      auto up = [&](auto** p, const auto& v) -> nsf_status {
        nsf_status r = ens_alloc(e, p, v.size());
        if (r != NSF_OK) return r;
        if (!v.empty() && cudaMemcpy(*p, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice) != cudaSuccess) {
          e->err = "could not upload the fused boundary kernel's plan";
          return NSF_ERR_CUDA;
        }
        return NSF_OK;
      };
      if ((st = up(&L.bcBlockStart, ranges)) != NSF_OK) return st;
      if ((st = up(&L.bcMemberLevels, fl.memberLevels)) != NSF_OK) return st;
      if ((st = up(&L.bcEdges, fl.edges)) != NSF_OK) return st;
      if ((st = up(&L.bcEdgeStart, fl.edgeStart)) != NSF_OK) return st;
      if ((st = up(&L.bcItems, fl.items)) != NSF_OK) return st;
      if ((st = up(&L.bcItemStart, fl.itemStart)) != NSF_OK) return st;
      if ((st = ens_alloc(e, &L.bcSync, 2 * size_t(M) + 1)) != NSF_OK) return st;
      CKE(cudaMemset(L.bcSync, 0, (2 * size_t(M) + 1) * sizeof(unsigned long long)));
    }
  }
  // member grids: the stage kernel adds its norm partials into slot 0 of each member, the near-body
  // filter's blocks (or the fused boundary kernel's) use slots 1 .. filterBlocks
  e->hGrids.resize(M);
  for (int g = 0; g < M; ++g) {
    Grid G = e->members[g]->hGrid;
    const int slots = 1 + L.filterBlocks;
    double* norm = nullptr;
    if ((st = ens_alloc(e, &norm, 5 * size_t(slots))) != NSF_OK) return st;
    CKE(cudaMemset(norm, 0, 5 * size_t(slots) * sizeof(double)));
    G.normPart = norm;
    G.nNormSlots = slots;
    G.normSlotFilter = 1;
    e->hGrids[g] = G;
  }
  if ((st = ens_alloc(e, &e->dGrids, size_t(M))) != NSF_OK) return st;
  CKE(cudaMemcpy(e->dGrids, e->hGrids.data(), M * sizeof(Grid), cudaMemcpyHostToDevice));
  CKE(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  e->launchesPerStep = enqueue_ensemble_step(e->dGrids, M, L, e->stream, nullptr);
  CKE(cudaStreamEndCapture(e->stream, &e->graph));
  CKE(cudaGraphInstantiate(&e->graphExec, e->graph, 0));
  return NSF_OK;
}

}  // namespace

extern "C" {

nsf_status nsf_autotune(const nsf_config* cfg, int32_t device, const char* cache_path, int32_t* tile,
                        double* ns_per_node) {
  if (!cfg || device < 0) return NSF_ERR_ARG;
  Tuned t;
  std::string err;
  nsf_status st = tune(*cfg, device, cache_path, t, err);
  if (st != NSF_OK) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return st;
  }
  if (tile) *tile = t.tile;
  if (ns_per_node) {
    ns_per_node[0] = t.nsPerNode[0];
    ns_per_node[1] = t.nsPerNode[1];
  }
  return NSF_OK;
}

nsf_status nsf_ensemble_create(const nsf_config* cfgs, uint32_t n, int32_t device, const char* tune_cache,
                               nsf_ensemble** out) {
  return create_ensemble(cfgs, n, device, tune_cache, -1, out);
}

}  // extern "C"

namespace {
nsf_status create_ensemble(const nsf_config* cfgs, uint32_t n, int32_t device, const char* tune_cache, int forceTile,
                           nsf_ensemble** out) {
  if (!cfgs || !out || n == 0 || device < 0) return NSF_ERR_ARG;
  auto* e = new nsf_ensemble;
  *out = e;
  e->device = device;
  if (forceTile < 0 && tune_cache) {  // throwaway ensembles time both tile shapes (once per composition)
    Tuned t;
    const nsf_status st = tune_ensemble(cfgs, n, device, tune_cache, t, e->err);
    if (st != NSF_OK) return st;
    forceTile = t.tile;
  }
  e->forceTile = forceTile;
  cudaDeviceProp prop{};
  if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess ||
      prop.major != 10) {
    e->err = "no sm_100 (B200) device for the ensemble";
    return NSF_ERR_CUDA;
  }
  e->nSM = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
    e->err = "could not create a CUDA stream";
    return NSF_ERR_CUDA;
  }
  for (uint32_t m = 0; m < n; ++m) {
    nsf_solver* s = nullptr;
    nsf_status st = nsf_create(&cfgs[m], device, &s);
    if (s) s->grouped = true;
    e->members.push_back(s);
    if (st != NSF_OK) {
      e->err = "ensemble member " + std::to_string(m) + ": " + (s ? s->err : std::string("nsf_create failed"));
      return st;
    }
  }
  return build_ensemble(e, tune_cache);
}
}  // namespace

extern "C" {

nsf_status nsf_ensemble_march(nsf_ensemble* e, uint64_t nsteps) {
  if (!e) return NSF_ERR_ARG;
  if (!e->graphExec) return NSF_ERR_STATE;
  CKE(cudaSetDevice(e->device));
  for (uint64_t q = 0; q < nsteps; ++q) CKE(cudaGraphLaunch(e->graphExec, e->stream));
  return NSF_OK;
}

nsf_status nsf_ensemble_march_timed(nsf_ensemble* e, uint64_t nsteps, double* ms) {
  if (!e || !ms) return NSF_ERR_ARG;
  if (!e->graphExec) return NSF_ERR_STATE;
  CKE(cudaSetDevice(e->device));
  cudaEvent_t a, b;
  CKE(cudaEventCreate(&a));
  CKE(cudaEventCreate(&b));
  CKE(cudaEventRecord(a, e->stream));
  for (uint64_t q = 0; q < nsteps; ++q) CKE(cudaGraphLaunch(e->graphExec, e->stream));
  CKE(cudaEventRecord(b, e->stream));
  CKE(cudaEventSynchronize(b));
  float f = 0;
  CKE(cudaEventElapsedTime(&f, a, b));
  *ms = f;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return NSF_OK;
}

nsf_status nsf_ensemble_profile_steps(nsf_ensemble* e, uint64_t nsteps, double* stage_ms, double* step_ms) {
  if (!e || !stage_ms || !step_ms) return NSF_ERR_ARG;
  if (!e->graphExec) return NSF_ERR_STATE;
  CKE(cudaSetDevice(e->device));
  std::vector<cudaEvent_t> ev(2 + 8 * nsteps);
  for (auto& x : ev) CKE(cudaEventCreate(&x));
  CKE(cudaEventRecord(ev[0], e->stream));
  for (uint64_t q = 0; q < nsteps; ++q)
    enqueue_ensemble_step(e->dGrids, int(e->members.size()), e->plan, e->stream, &ev[2 + 8 * q]);
  CKE(cudaGetLastError());
  CKE(cudaEventRecord(ev[1], e->stream));
  CKE(cudaEventSynchronize(ev[1]));
  float ms = 0;
  CKE(cudaEventElapsedTime(&ms, ev[0], ev[1]));
  *step_ms = ms / double(nsteps ? nsteps : 1);
  for (int s = 0; s < 4; ++s) {
    double tot = 0;
    for (uint64_t q = 0; q < nsteps; ++q) {
      float m = 0;
      CKE(cudaEventElapsedTime(&m, ev[2 + 8 * q + 2 * s], ev[2 + 8 * q + 2 * s + 1]));
      tot += m;
    }
    stage_ms[s] = tot / double(nsteps ? nsteps : 1);
  }
  for (auto& x : ev) cudaEventDestroy(x);
  return NSF_OK;
}

nsf_status nsf_ensemble_sync(nsf_ensemble* e) {
  if (!e) return NSF_ERR_ARG;
  if (!e->graphExec) return NSF_ERR_STATE;
  CKE(cudaStreamSynchronize(e->stream));
  for (size_t m = 0; m < e->members.size(); ++m) {
    nsf_status st = nsf_sync(e->members[m]);
    if (st != NSF_OK) {
      e->err = "member " + std::to_string(m) + ": " + e->members[m]->err;
      return st;
    }
  }
  return NSF_OK;
}

nsf_status nsf_ensemble_member(nsf_ensemble* e, uint32_t m, nsf_solver** member) {
  if (!e || !member || m >= e->members.size() || !e->graphExec) return NSF_ERR_ARG;
  CKE(cudaStreamSynchronize(e->stream));  // the member's own calls then see the ensemble's steps
  *member = e->members[m];
  return NSF_OK;
}

nsf_status nsf_ensemble_info(nsf_ensemble* e, int32_t* tile, uint64_t* launches_per_step, uint32_t* work_items) {
  if (!e) return NSF_ERR_ARG;
  if (!e->graphExec) return NSF_ERR_STATE;
  if (tile) *tile = e->tile;
  if (launches_per_step) *launches_per_step = uint64_t(e->launchesPerStep);
  if (work_items) *work_items = uint32_t(e->plan.nItems);
  return NSF_OK;
}

const char* nsf_ensemble_last_error(nsf_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

void nsf_ensemble_destroy(nsf_ensemble* e) {
  if (!e) return;
  if (e->stream) {
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
  }
  if (e->graphExec) cudaGraphExecDestroy(e->graphExec);
  if (e->graph) cudaGraphDestroy(e->graph);
  for (void* p : e->allocs) cudaFree(p);
  for (nsf_solver* s : e->members) nsf_destroy(s);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

}  // extern "C"
