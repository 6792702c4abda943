// C ABI implementation (include/nsfsi.h): the solver handle, device residency of all fields, the
// device-side lists built from the host setup, and one captured CUDA graph per RK4 step.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "nsf_device.cuh"
#include "nsf_internal.h"

using namespace nsf;

#include "nsf_solver_impl.h"

namespace {

nsf_status cuda_fail(nsf_solver* s, cudaError_t e, const char* what) {
  s->err = std::string(what) + ": " + cudaGetErrorString(e);
  return NSF_ERR_CUDA;
}
#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(s, e_, #call);    \
  } while (0)

template <class T>
nsf_status dalloc(nsf_solver* s, T** p, size_t count) {
  void* q = nullptr;
  CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  s->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return NSF_OK;
}
template <class T>
nsf_status upload(nsf_solver* s, T** p, const std::vector<T>& v) {
  nsf_status st = dalloc(s, p, v.size());
  if (st != NSF_OK) return st;
  if (!v.empty()) CK(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return NSF_OK;
}

// Physical and stencil constants, each evaluated as the reference writes it (Solver.cpp:202-360).
Consts make_consts(const nsf_config& c, const HostSetup& s) {
  Consts K{};
  const double dx = s.d[0], dy = s.d[1], dz = s.d[2];
  K.gamma = c.gamma;
  K.gm1 = c.gamma - 1;
  K.pr = c.pr;
  K.re = c.re;
  K.sc1 = 1 + c.sutherlands_c2 / c.t0;
  K.pf = 1 / (K.gm1 * c.pr);
  K.h0 = 1. / (c.gamma - 1);
  K.vmod = std::max(4. / 3, c.gamma / c.pr);
  K.convLim = std::fabs(c.conv_stability_limit);
  K.viscLim = std::fabs(c.visc_stability_limit);
  K.m0 = c.m0;
  K.tEnd = c.t_end;
  K.dx = dx;
  K.dy = dy;
  K.dz = dz;
  K.dxdydz = dx * dy * dz;
  K.ax = -1. / (2 * dx);
  K.ay = -1. / (2 * dy);
  K.az = -1. / (2 * dz);
  K.xm_xx = 2. / (3 * dx * dx);
  K.xm_yy = 1. / (2 * dy * dy);
  K.xm_zz = 1. / (2 * dz * dz);
  K.xm_yx = -1. / (6 * dy * dx);
  K.xm_xy = 1. / (4 * dx * dy);
  K.xm_zx = -1. / (6 * dz * dx);
  K.xm_xz = 1. / (4 * dx * dz);
  K.ym_xx = 1. / (2 * dx * dx);
  K.ym_yy = 2. / (3 * dy * dy);
  K.ym_zz = 1. / (2 * dz * dz);
  K.ym_xy = -1. / (6 * dx * dy);
  K.ym_yx = 1. / (4 * dy * dx);
  K.ym_zy = -1. / (6 * dz * dy);
  K.ym_yz = 1. / (4 * dy * dz);
  K.zm_xx = 1. / (2 * dx * dx);
  K.zm_yy = 1. / (2 * dy * dy);
  K.zm_zz = 2. / (3 * dz * dz);
  K.zm_zx = 1. / (4 * dz * dx);
  K.zm_xz = -1. / (6 * dx * dz);
  K.zm_zy = 1. / (4 * dz * dy);
  K.zm_yz = -1. / (6 * dy * dz);
  K.e_xx23 = 2. / (3 * dx * dx);
  K.e_xx12 = 1. / (2 * dx * dx);
  K.e_yx6 = -1. / (6 * dy * dx);
  K.e_zx6 = -1. / (6 * dz * dx);
  K.e_yx4 = 1. / (4 * dy * dx);
  K.e_zx4 = 1. / (4 * dz * dx);
  K.e_yy12 = 1. / (2 * dy * dy);
  K.e_yy23 = 2. / (3 * dy * dy);
  K.e_zy6 = -1. / (6 * dz * dy);
  K.e_zy4 = 1. / (4 * dz * dy);
  K.e_zz12 = 1. / (2 * dz * dz);
  K.e_zz23 = 2. / (3 * dz * dz);
  K.endTime = c.stop_criterion == 1;
  K.convHistory = c.conv_history;
  K.nFilterIv = c.n_filter_intervals;
  for (int q = 0; q < c.n_filter_intervals; ++q) K.filterIv[q] = c.filter_intervals[q];
  K.nChange = c.n_filter_change_times;
  for (int q = 0; q < c.n_filter_change_times; ++q) K.changeT[q] = c.filter_change_times[q];
  return K;
}

// Solver::updateTimeStepSize at t = 0 (Solver.cpp:80-126), on the host from the initial fields.
double initial_dt(const nsf_config& c, const HostSetup& s, const std::vector<double>& cons,
                  const std::vector<double>& prim) {
  const size_t N = s.N;
  double mX = 0, mY = 0, mZ = 0, mNu = 0;
  const double mod = std::max(4. / 3, c.gamma / c.pr);
  for (size_t i = 0; i < N; ++i) {
    double ci = std::sqrt((1 + c.gamma * prim[3 * N + i]) / (1 + cons[i]));
    mX = std::max(mX, ci + std::fabs(prim[i]));
    mY = std::max(mY, ci + std::fabs(prim[N + i]));
    mZ = std::max(mZ, ci + std::fabs(prim[2 * N + i]));
    mNu = std::max(mNu, prim[5 * N + i] / (cons[i] + 1) * mod);
  }
  double conv = std::fabs(c.conv_stability_limit) / (mX / s.d[0] + mY / s.d[1] + mZ / s.d[2]);
  double dx2 = s.d[0] * s.d[0], dy2 = s.d[1] * s.d[1], dz2 = s.d[2] * s.d[2];
  double visc = std::fabs(c.visc_stability_limit) / (mNu * (1 / dx2 + 1 / dy2 + 1 / dz2));
  double dt = std::min(conv, visc);
  if (c.stop_criterion == 1 && 0 + dt > c.t_end) dt = c.t_end - 0;
  return dt;
}

// Device layout: the reference's i/j/k order with the k rows padded to a pitch NKp (a multiple of 16),
// so every row of doubles starts on a 128-byte boundary, every row of node-type bytes on a 16-byte
// boundary, and TMA boxes can start at any tile origin.
long long dev_index(const HostSetup& S, size_t NKp, size_t n) {
  const size_t i = n / (S.NJ * S.NK), j = n % (S.NJ * S.NK) / S.NK, k = n % S.NK;
  return (long long)(i * S.NJ * NKp + j * NKp + k);
}

nsf_status build_device(nsf_solver* s) {
  const HostSetup& S = s->setup;
  const nsf_config& cfg = s->cfg;
  const size_t N = S.N;
  const size_t NKp = (S.NK + 15) / 16 * 16;
  const size_t Nd = S.NI * S.NJ * NKp;
  auto dev = [&](size_t n) { return dev_index(S, NKp, n); };
  Grid& G = s->hGrid;
  G = Grid{};
  // stage-kernel tile shape: the handle's request (ensembles, tuned plans), else NSF_STAGE_TILE=16x16 or
  // 32x8 (default)
  const int tile = s->tileRequest >= 0 ? s->tileRequest : [] {
    const char* e = std::getenv("NSF_STAGE_TILE");
    return e && std::string(e) == "16x16" ? int(STAGE_TILE_16x16) : int(STAGE_TILE_32x8);
  }();
  G.NI = int(S.NI);
  G.NJ = int(S.NJ);
  G.NK = int(S.NK);
  G.NKp = int(NKp);
  G.sI = (long long)(S.NJ * NKp);
  G.sJ = (long long)NKp;
  G.N = (long long)Nd;
  G.C = make_consts(cfg, S);

  // initial condition
  std::vector<double> cons, prim;
  if (!s->slabCons.empty()) {  // an x-slab: its planes of the whole grid's initial condition
    cons = s->slabCons;
    prim = s->slabPrim;
  } else {
    initial_condition(cfg, S, cons, prim);
  }
  double* fields = nullptr;
  nsf_status st = dalloc(s, &fields, 20 * Nd);
  if (st != NSF_OK) return st;
  CK(cudaMemset(fields, 0, 20 * Nd * sizeof(double)));
  for (int b = 0; b < 3; ++b)
    for (int f = 0; f < 5; ++f) G.bufs[b][f] = fields + (size_t(b) * 5 + f) * Nd;
  for (int f = 0; f < 5; ++f) G.acc[f] = fields + (15 + size_t(f)) * Nd;
  for (int f = 0; f < 5; ++f)
    CK(cudaMemcpy2D(G.bufs[0][f], NKp * sizeof(double), cons.data() + f * N, S.NK * sizeof(double),
                    S.NK * sizeof(double), S.NI * S.NJ, cudaMemcpyHostToDevice));

  // TMA descriptors: staged planes (box (TK + 2) x (TJ + 2) x 1) and epilogue tiles ((TK + 2) x TJ x 1) of every
  // physical buffer field, and epilogue tiles of the accumulator.
  {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    CK(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &qr));
    if (!fn || qr != cudaDriverEntryPointSuccess) {
      s->err = "cuTensorMapEncodeTiled is not available from the driver";
      return NSF_ERR_CUDA;
    }
    auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    std::vector<CUtensorMap> maps(stage_num_maps());
    auto mk = [&](CUtensorMap* m, double* base, cuuint32_t rows) {
      cuuint64_t gdim[3] = {S.NK, S.NJ, S.NI};
      cuuint64_t gstr[2] = {NKp * sizeof(double), S.NJ * NKp * sizeof(double)};
      cuuint32_t box[3] = {cuuint32_t(stage_tile_k(tile) + 2), rows, 1};
      cuuint32_t es[3] = {1, 1, 1};
      return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    };
    const cuuint32_t haloRows = cuuint32_t(stage_tile_j(tile) + 2), tileRows = cuuint32_t(stage_tile_j(tile));
    bool okMaps = true;
    for (int b = 0; b < 3; ++b)
      for (int f = 0; f < 5; ++f) {
        okMaps &= mk(&maps[b * 5 + f], G.bufs[b][f], haloRows) == CUDA_SUCCESS;
        okMaps &= mk(&maps[15 + b * 5 + f], G.bufs[b][f], tileRows) == CUDA_SUCCESS;
      }
    for (int f = 0; f < 5; ++f) okMaps &= mk(&maps[30 + f], G.acc[f], tileRows) == CUDA_SUCCESS;
    if (!okMaps) {
      s->err = "cuTensorMapEncodeTiled rejected a field descriptor";
      return NSF_ERR_CUDA;
    }
    s->hostMaps = maps;
    s->encodeFn = fn;
  }

  // node types with the filter bit, filter slots
  std::vector<uint8_t> type = S.type;
  if (!s->slabFlags.empty())
    for (size_t n = 0; n < N; ++n) type[n] |= s->slabFlags[n];
  for (auto& e : S.edges)
    for (size_t i = e.owned.i0; i <= e.owned.i1; ++i)
      for (size_t j = e.owned.j0; j <= e.owned.j1; ++j)
        for (size_t k = e.owned.k0; k <= e.owned.k1; ++k) type[i * S.NJ * S.NK + j * S.NK + k] |= EDGE_PLANE_BIT;
  std::vector<long long> fnode;  // filter slots: one per (body, node), in body order
  std::vector<int> fbody;
  for (size_t q = 0; q < S.bodies.size(); ++q)
    for (size_t f : S.bodies[q].filter) {
      fnode.push_back((long long)f);
      fbody.push_back(int(q));
    }
  std::map<long long, std::vector<int>> slotsOf;  // host node -> its filter slots (body order)
  for (size_t q = 0; q < fnode.size(); ++q) slotsOf[fnode[q]].push_back(int(q));
  std::vector<double> fpre(2 * fnode.size());
  for (size_t q = 0; q < fnode.size(); ++q) {
    type[fnode[q]] |= FILTER_BIT;
    fpre[2 * q] = cons[fnode[q]];
    fpre[2 * q + 1] = cons[4 * N + fnode[q]];
  }
  {  // periodic y faces: the nodes whose periodic copies the stage kernel writes. The edge conditions run
     // x, y, z: every reader of a y-face node (later y rows, the z faces, the bodies) wants the value after
     // the y copy, and the copy's source, an unfiltered interior node, is final after the stage kernel.
    int yPer = 0;
    for (const auto& e : S.edges) yPer += e.axis == 1 && e.bc == NSF_BC_PERIODIC;
    G.yFused = yPer == 2 && S.NJ >= 4;
    if (G.yFused)
      for (size_t i = 1; i + 1 < S.NI; ++i)
        for (size_t js : {size_t(1), S.NJ - 2})
          for (size_t k = 1; k + 1 < S.NK; ++k) {
            uint8_t& t = type[(i * S.NJ + js) * S.NK + k];
            if ((t & TYPE_MASK) == FLUID_INTERIOR && !(t & FILTER_BIT)) t |= YCOPY_BIT;
          }
  }
  {  // periodic z faces: the nodes whose periodic copies the stage kernel writes
    int zPer = 0;
    for (const auto& e : S.edges) zPer += e.axis == 2 && e.bc == NSF_BC_PERIODIC;
    G.zFused = zPer == 2 && S.NK >= 4;
    if (G.zFused)
      for (size_t i = 1; i + 1 < S.NI; ++i)
        for (size_t j = 1; j + 1 < S.NJ; ++j)
          for (size_t ks : {size_t(1), S.NK - 2}) {
            uint8_t& t = type[(i * S.NJ + j) * S.NK + ks];
            if ((t & TYPE_MASK) == FLUID_INTERIOR && !(t & FILTER_BIT)) t |= ks == 1 ? ZCOPY_UP_BIT : ZCOPY_DOWN_BIT;
          }
  }
  s->typeFlags = type;
  std::vector<uint8_t> typeDev(Nd, SOLID_INACTIVE);  // pitch padding never takes part
  for (size_t n = 0; n < N; ++n) typeDev[dev(n)] = type[n];
  for (auto& f : fnode) f = dev(size_t(f));
  uint8_t* dType;
  if ((st = upload(s, &dType, typeDev)) != NSF_OK) return st;
  G.type = dType;
  {  // node-type boxes (row width x (TJ + 2) x 1 bytes) for the stage kernel, then all descriptors to the device
    auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(s->encodeFn);
    cuuint64_t gdim[3] = {S.NK, S.NJ, S.NI};
    cuuint64_t gstr[2] = {NKp, S.NJ * NKp};
    cuuint32_t box[3] = {cuuint32_t(stage_type_box_width(tile)), cuuint32_t(stage_tile_j(tile) + 2), 1};
    cuuint32_t es[3] = {1, 1, 1};
    if (encode(&s->hostMaps[stage_num_maps() - 1], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dType, gdim, gstr, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      s->err = "cuTensorMapEncodeTiled rejected the node-type descriptor";
      return NSF_ERR_CUDA;
    }
    CUtensorMap* dMaps = nullptr;
    if ((st = upload(s, &dMaps, s->hostMaps)) != NSF_OK) return st;
    G.tmaps = dMaps;
  }
  G.nFilter = int(fnode.size());
  std::vector<int> fidx;
  if (!fnode.empty()) {
    fidx.assign(Nd, -1);  // a node's first slot (the stage kernel takes its pre-filter values from it)
    for (size_t q = 0; q < fnode.size(); ++q)
      if (fidx[fnode[q]] < 0) fidx[fnode[q]] = int(q);
    int* dF;
    if ((st = upload(s, &dF, fidx)) != NSF_OK) return st;
    G.fidx = dF;
  }
  {  // per slot: the node's first slot, and whether this is its last
    std::vector<int> fmeta(fnode.size());
    for (const auto& kv : slotsOf)
      for (size_t r = 0; r < kv.second.size(); ++r)
        fmeta[size_t(kv.second[r])] = kv.second[0] | (r + 1 == kv.second.size() ? FMETA_LAST : 0);
    int* dFm;
    if ((st = upload(s, &dFm, fmeta)) != NSF_OK) return st;
    G.fmeta = dFm;
  }
  {  // stencil nodes of each filter node that are solid nodes off the mesh faces, read from the solid copy's
     // source -- unless an earlier body's ghost item has written the node by then
    std::map<long long, int> firstGhostBody;  // device node -> first body whose ghost list holds it
    for (size_t q = S.bodies.size(); q-- > 0;)
      for (auto& g : S.bodies[q].ghosts) firstGhostBody[dev(g.i * S.NJ * S.NK + g.j * S.NK + g.k)] = int(q);
    std::vector<uint8_t> fsolid(fnode.size(), 0);
    for (size_t q = 0; q < fnode.size(); ++q) {
      const long long n = fnode[q];
      const long long nb[7] = {n, n + G.sI, n - G.sI, n + G.sJ, n - G.sJ, n + 1, n - 1};
      for (int b = 0; b < 7; ++b) {
        const uint8_t t = typeDev[size_t(nb[b])], k = t & TYPE_MASK;
        auto it = firstGhostBody.find(nb[b]);
        const bool written = it != firstGhostBody.end() && it->second < fbody[q];
        if ((k == SOLID_GHOST || k == SOLID_INACTIVE) && !(t & EDGE_PLANE_BIT) && !written)
          fsolid[q] |= uint8_t(1u << b);
      }
    }
    uint8_t* dFs;
    if ((st = upload(s, &dFs, fsolid)) != NSF_OK) return st;
    G.fsolid = dFs;
  }
  long long* dFnode;
  double *dFpre, *dFnew;
  if ((st = upload(s, &dFnode, fnode)) != NSF_OK) return st;
  if ((st = upload(s, &dFpre, fpre)) != NSF_OK) return st;
  if ((st = upload(s, &dFnew, fpre)) != NSF_OK) return st;
  G.fnode = dFnode;
  G.fpre = dFpre;
  G.fnew = dFnew;

  // ghost nodes: cells and the points / normals the weight solve needs
  std::vector<long long> gnode, gcell;
  std::vector<double> pts, nrm, ipl;
  std::vector<uint8_t> gfl, glast;
  std::vector<int> gbody, gsrc;
  for (size_t bq = 0; bq < S.bodies.size(); ++bq)
    for (auto& g : S.bodies[bq].ghosts) {
      const auto& b = S.bodies[bq];
      gbody.push_back(int(bq));
      gnode.push_back(dev(g.i * S.NJ * S.NK + g.j * S.NK + g.k));
      Box box;
      surrounding_box(S, g.ip, box);
      int64_t cs[8];
      box_corners(S, box, cs);
      double lo[3];
      node_position(S, box.i0, box.j0, box.k0, lo);
      for (int q = 0; q < 3; ++q) ipl.push_back(g.ip[q]);
      for (int q = 0; q < 3; ++q) ipl.push_back(lo[q]);
      for (int m = 0; m < 8; ++m) {
        gcell.push_back(dev(size_t(cs[m])));
        const size_t cn = size_t(cs[m]);
        {  // filtered values this ghost reads at a filter corner: the last slot of a body up to its own
          int src = -1;
          auto it = slotsOf.find((long long)cn);
          if (it != slotsOf.end())
            for (int sl : it->second)
              if (fbody[size_t(sl)] <= int(bq)) src = sl;
          gsrc.push_back(src);
        }
        if (S.type[cn] == SOLID_GHOST) {
          const GhostRec& og = b.ghosts[b.ghostIndex.at(cn)];
          double d[3] = {og.ip[0] - og.bi[0], og.ip[1] - og.bi[1], og.ip[2] - og.bi[2]};
          double len = std::sqrt(std::pow(d[0], 2) + std::pow(d[1], 2) + std::pow(d[2], 2));
          for (int q = 0; q < 3; ++q) pts.push_back(og.bi[q]);
          for (int q = 0; q < 3; ++q) nrm.push_back(d[q] / len);
          gfl.push_back(1);
        } else {
          double p[3];
          size_t ci = cn / (S.NJ * S.NK), cj = cn % (S.NJ * S.NK) / S.NK, ck = cn % S.NK;
          node_position(S, ci, cj, ck, p);
          for (int q = 0; q < 3; ++q) pts.push_back(p[q]);
          for (int q = 0; q < 3; ++q) nrm.push_back(0);
          gfl.push_back(0);
        }
      }
    }
  {  // a ghost item is its node's last writer unless a later body's ghost list holds the node too
    glast.assign(gnode.size(), 1);
    std::map<long long, size_t> lastOf;
    for (size_t q = 0; q < gnode.size(); ++q) {
      auto it = lastOf.find(gnode[q]);
      if (it != lastOf.end()) glast[it->second] = 0;
      lastOf[gnode[q]] = q;
    }
  }
  {  // device order of the ghosts: by image-point cell (first corner), so the lanes of a warp gather
     // overlapping corner sets; s->ghostOrder[q] = the ghost's position in the bodies' own order
    const size_t ng = gnode.size();
    std::vector<int> ord(ng);
    for (size_t q = 0; q < ng; ++q) ord[q] = int(q);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return gcell[8 * size_t(a)] < gcell[8 * size_t(b)]; });
    auto permute = [&](auto& v, size_t per) {
      auto w = v;
      for (size_t q = 0; q < ng; ++q)
        for (size_t r = 0; r < per; ++r) w[q * per + r] = v[size_t(ord[q]) * per + r];
      v.swap(w);
    };
    permute(gnode, 1);
    permute(gcell, 8);
    permute(pts, 24);
    permute(nrm, 24);
    permute(ipl, 6);
    permute(gfl, 8);
    permute(gbody, 1);
    permute(glast, 1);
    permute(gsrc, 8);
    s->ghostOrder = ord;
  }
  G.nGhost = int(gnode.size());
  long long *dGnode, *dGcell;
  double *dPts, *dNrm, *dIpl, *dW;
  uint8_t* dFl;
  if ((st = upload(s, &dGnode, gnode)) != NSF_OK) return st;
  if ((st = upload(s, &dGcell, gcell)) != NSF_OK) return st;
  if ((st = upload(s, &dPts, pts)) != NSF_OK) return st;
  if ((st = upload(s, &dNrm, nrm)) != NSF_OK) return st;
  if ((st = upload(s, &dIpl, ipl)) != NSF_OK) return st;
  if ((st = upload(s, &dFl, gfl)) != NSF_OK) return st;
  if ((st = dalloc(s, &dW, 16 * gnode.size())) != NSF_OK) return st;
  launch_ghost_weights(G.nGhost, dPts, dNrm, dFl, dIpl, S.d[0], S.d[1], S.d[2], dW, s->stream);
  CK(cudaGetLastError());
  G.gnode = dGnode;
  G.gcell = dGcell;
  G.gw = dW;
  {
    int* dGs;
    uint8_t* dGl;
    if ((st = upload(s, &dGs, gsrc)) != NSF_OK) return st;
    if ((st = upload(s, &dGl, glast)) != NSF_OK) return st;
    G.gsrc = dGs;
    G.glast = dGl;
  }

  // solid nodes: copy list (ghost + inactive); inactive primitive values as the reference holds them
  std::vector<long long> snode, inode, dlNode, dlNodeIc;
  std::vector<double> iprim, dlPrim, dlPrimIc;
  // owner edge of every boundary-plane node, to follow periodic copies of solid nodes
  std::vector<int> edgeOf(N, -1);
  for (size_t e = 0; e < S.edges.size(); ++e) {
    const Box& b = S.edges[e].owned;
    for (size_t i = b.i0; i <= b.i1; ++i)
      for (size_t j = b.j0; j <= b.j1; ++j)
        for (size_t k = b.k0; k <= b.k1; ++k) edgeOf[i * S.NJ * S.NK + j * S.NK + k] = int(e);
  }
  for (size_t n = 0; n < N; ++n) {
    uint8_t t = S.type[n];
    if (t != SOLID_GHOST && t != SOLID_INACTIVE) continue;
    snode.push_back(dev(n));
    if (t != SOLID_INACTIVE) continue;
    // Follow periodic copies to the node whose primitive values land here (Boundary.cpp:344-367).
    size_t src = n;
    bool dynamic = false;
    for (int hop = 0; hop < 4 && edgeOf[src] >= 0; ++hop) {
      const EdgeBC& e = S.edges[edgeOf[src]];
      if (e.bc != NSF_BC_PERIODIC) {
        dynamic = true;
        break;
      }
      size_t ijk[3] = {src / (S.NJ * S.NK), src % (S.NJ * S.NK) / S.NK, src % S.NK};
      size_t nAx[3] = {S.NI, S.NJ, S.NK};
      ijk[e.axis] = e.side == 0 ? nAx[e.axis] - 2 : 1;
      src = ijk[0] * S.NJ * S.NK + ijk[1] * S.NK + ijk[2];
    }
    if (S.type[src] != SOLID_INACTIVE) dynamic = true;
    inode.push_back(dev(n));
    dlNodeIc.push_back(dev(n));
    for (int q = 0; q < 7; ++q) dlPrimIc.push_back(prim[q * N + n]);
    if (dynamic) {
      // values copied with the conserved ones from a node whose primitives follow its conserved values
      for (int q = 0; q < 5; ++q) iprim.push_back(std::nan(""));
    } else {
      iprim.push_back(prim[src]);
      iprim.push_back(prim[N + src]);
      iprim.push_back(prim[2 * N + src]);
      iprim.push_back(prim[3 * N + src]);
      iprim.push_back(prim[5 * N + src]);
      dlNode.push_back(dev(n));
      for (int q = 0; q < 7; ++q) dlPrim.push_back(prim[q * N + src]);
    }
  }
  G.nSolid = int(snode.size());
  G.nInactive = int(inode.size());
  long long *dS, *dI;
  double* dIp;
  if ((st = upload(s, &dS, snode)) != NSF_OK) return st;
  if ((st = upload(s, &dI, inode)) != NSF_OK) return st;
  if ((st = upload(s, &dIp, iprim)) != NSF_OK) return st;
  G.snode = dS;
  G.inode = dI;
  G.iprim = dIp;
  s->nDl = int(dlNode.size());
  if ((st = upload(s, &s->dDlNode, dlNode)) != NSF_OK) return st;
  if ((st = upload(s, &s->dDlPrim, dlPrim)) != NSF_OK) return st;
  s->nDlIc = int(dlNodeIc.size());
  if ((st = upload(s, &s->dDlNodeIc, dlNodeIc)) != NSF_OK) return st;
  if ((st = upload(s, &s->dDlPrimIc, dlPrimIc)) != NSF_OK) return st;

  // boundary conditions in application order
  G.nEdge = int(S.edges.size());
  for (size_t e = 0; e < S.edges.size(); ++e) {
    G.eAxis[e] = S.edges[e].axis;
    G.eSide[e] = S.edges[e].side;
    G.eBc[e] = S.edges[e].bc;
    const Box& b = S.edges[e].owned;
    int bx[6] = {int(b.i0), int(b.i1), int(b.j0), int(b.j1), int(b.k0), int(b.k1)};
    std::memcpy(G.eBox[e], bx, sizeof bx);
  }

  // launch plan: stage work items (tile x i-chunk), grids of the small kernels
  LaunchPlan& L = s->plan;
  L = LaunchPlan{};
  L.nSM = s->nSM;
  L.tile = tile;
  CK(cudaError_t(stage_configure(tile)));
  if (!stage_register_split_ok(tile)) {
    s->err = "stage kernel: its launch registers do not cover its setmaxnreg split";
    return NSF_ERR_CUDA;
  }
  const int occ = std::max(1, stage_occupancy(tile));
  const int TJ = stage_tile_j(tile), TK = stage_tile_k(tile);
  const int nj = int((S.NJ - 2 + TJ - 1) / TJ), nk = int((S.NK - 2 + TK - 1) / TK);
  const int tiles = nj * nk, planes = int(S.NI - 2);
  const int slots = s->nSM * occ;
  // i-chunk count: minimise the planes the busiest CTA streams (whole waves of items, each item
  // streaming its chunk plus two halo planes).
  int chunks = 1;
  double best = 1e300;
  for (int c = 1; c <= planes; ++c) {
    const int len = (planes + c - 1) / c;
    const double waves = std::ceil(double(tiles) * c / slots);
    const double cost = waves * (len + 2);
    if (cost < best - 1e-9) {
      best = cost;
      chunks = c;
    }
  }
  const int clen = (planes + chunks - 1) / chunks;
  std::vector<StageItem> items;
  for (int c0 = 1; c0 <= planes; c0 += clen)
    for (int tj = 0; tj < nj; ++tj)
      for (int tk = 0; tk < nk; ++tk)
        items.push_back(StageItem{1 + tj * TJ, 1 + tk * TK, c0, std::min(planes, c0 + clen - 1), 0});
  L.nItems = int(items.size());
  L.stageBlocks = std::min(L.nItems, slots);
  {  // CTA b takes items b, b + stageBlocks, ... (whole waves of equal items), stored contiguously
    std::vector<StageItem> ordered;
    std::vector<int> start(1, 0);
    for (int b = 0; b < L.stageBlocks; ++b) {
      for (int q = b; q < L.nItems; q += L.stageBlocks) ordered.push_back(items[q]);
      start.push_back(int(ordered.size()));
    }
    items.swap(ordered);
    if ((st = upload(s, &L.ctaStart, start)) != NSF_OK) return st;
  }
  if ((st = upload(s, &L.items, items)) != NSF_OK) return st;
  std::vector<EdgeBlock> ebAxis[3];
  for (int a = 0; a < 3; ++a) {
    std::vector<EdgeBlock>& eb = ebAxis[a];
    edge_blocks(G, type.data(), 0, a, eb);
    L.nEdgeBlocks[a] = int(eb.size());
    L.edgeBlocks[a] = nullptr;
    if (!eb.empty() && (st = upload(s, &L.edgeBlocks[a], eb)) != NSF_OK) return st;
  }
  {  // dependency levels of the stage's boundary work, for the fused boundary kernel
    BcMemberInput in;
    in.snode = snode;
    in.fnode = fnode;
    in.gnode = gnode;
    in.gcell = gcell;
    in.inode = inode;
    in.typeDev = typeDev;
    in.fidx = fidx;
    in.fbody = fbody;
    in.gbody = gbody;
    in.gsrc = gsrc;
    bc_plan_member(G, ebAxis, in, s->bcLevels);
  }
  L.hasFilter = G.nFilter > 0;
  L.filterBlocks = std::max(1, std::min(s->nSM, (G.nFilter + 255) / 256));
  L.hasSolid = G.nSolid > 0;
  L.solidBlocks = std::max(1, std::min(4 * s->nSM, (G.nSolid + 255) / 256));
  const int ghostWork = G.nGhost + G.nFilter + G.nInactive;
  L.hasGhostWork = ghostWork > 0;
  L.ghostBlocks = std::max(1, std::min(4 * s->nSM, (ghostWork + 255) / 256));
  L.gfBlocks = 4 * s->nSM;
  {  // fused boundary kernel: enough blocks for the busiest level, within what can be resident at once
    BcFlat fl;
    bc_flatten({&s->bcLevels}, fl);
    const std::vector<int> ranges = bc_block_ranges(fl, bc_capacity(s->nSM));
    L.bcBlocks = ranges.empty() ? 0 : ranges.back();
    L.bcLevels = fl.levels;
    if (L.bcBlocks > 0) {
      if ((st = upload(s, &L.bcBlockStart, ranges)) != NSF_OK) return st;
      if ((st = upload(s, &L.bcMemberLevels, fl.memberLevels)) != NSF_OK) return st;
      L.filterBlocks = std::max(L.filterBlocks, L.bcBlocks);  // one norm slot per block of the fused kernel
      if ((st = upload(s, &L.bcEdges, fl.edges)) != NSF_OK) return st;
      if ((st = upload(s, &L.bcEdgeStart, fl.edgeStart)) != NSF_OK) return st;
      if ((st = upload(s, &L.bcItems, fl.items)) != NSF_OK) return st;
      if ((st = upload(s, &L.bcItemStart, fl.itemStart)) != NSF_OK) return st;
      const std::vector<unsigned long long> zero(3, 0ull);
      if ((st = upload(s, &L.bcSync, zero)) != NSF_OK) return st;
    }
  }
  if (S.bodiesInteract && L.bcBlocks == 0) {  // the separate boundary kernels treat all bodies at once
    s->err = "interacting immersed bodies need the fused boundary kernel, which this device cannot host";
    return NSF_ERR_GEOMETRY;
  }
  L.nSlots = L.stageBlocks + (L.hasFilter ? L.filterBlocks : 0);
  double* dNorm;
  if ((st = dalloc(s, &dNorm, 5 * size_t(L.nSlots))) != NSF_OK) return st;
  CK(cudaMemset(dNorm, 0, 5 * size_t(L.nSlots) * sizeof(double)));
  G.normPart = dNorm;
  G.nNormSlots = L.nSlots;
  G.normSlotFilter = L.stageBlocks;
  double* dHist;
  if ((st = dalloc(s, &dHist, 7 * size_t(MAX_HIST))) != NSF_OK) return st;
  G.hist = dHist;

  // control block
  StepCtl ctl{};
  ctl.t = 0;
  ctl.dt = initial_dt(cfg, S, cons, prim);
  ctl.level = 0;
  for (int f = 0; f < 5; ++f) {
    ctl.perm[f][0] = 0;
    ctl.perm[f][1] = 1;
    ctl.perm[f][2] = 2;
  }
  s->ctlInit = ctl;
  if ((st = dalloc(s, &s->dCtl, 1)) != NSF_OK) return st;
  CK(cudaMemcpy(s->dCtl, &ctl, sizeof ctl, cudaMemcpyHostToDevice));
  G.ctl = s->dCtl;
  if ((st = dalloc(s, &s->dGrid, 1)) != NSF_OK) return st;
  CK(cudaMemcpy(s->dGrid, &G, sizeof G, cudaMemcpyHostToDevice));
  CK(cudaStreamSynchronize(s->stream));

  // one step as a CUDA graph
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  s->launchesPerStep = enqueue_step(s->dGrid, G, L, s->stream);
  CK(cudaStreamEndCapture(s->stream, &s->graph));
  CK(cudaGraphInstantiate(&s->graphExec, s->graph, 0));
  return NSF_OK;
}

// Slots of the asked-for fields in a packed download (increasing field order), and how many there are.
SnapSlots snap_slots(uint32_t mask, int* count) {
  SnapSlots sl;
  int q = 0;
  for (int f = 0; f < NSF_SNAP_FIELDS; ++f) sl.slot[f] = (mask >> f) & 1u ? q++ : -1;
  *count = q;
  return sl;
}

SnapInactive snap_inactive(const nsf_solver* s) {
  return SnapInactive{s->dDlNode, s->dDlPrim, s->nDl, s->dDlNodeIc, s->dDlPrimIc, s->nDlIc};
}


}  // namespace

// For the x-slab groups (nsf_slab.cpp): device set-up of a handle whose host setup is already in place,
// and the initial dt of a whole grid.
nsf_status nsf_build_device(nsf_solver* s) { return build_device(s); }
double nsf_initial_dt(const nsf_config& c, const nsf::HostSetup& S, const std::vector<double>& cons,
                      const std::vector<double>& prim) {
  return initial_dt(c, S, cons, prim);
}

extern "C" {

nsf_status nsf_create(const nsf_config* cfg, int32_t device, nsf_solver** out) {
  if (!cfg || !out) return NSF_ERR_ARG;
  *out = nullptr;
  auto* s = new nsf_solver;
  s->cfg = *cfg;
  s->device = device;
  if (device < 0) {
    s->hostOnly = true;
    *out = s;
    return NSF_OK;
  }
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= device || device < 0) {
    s->err = "no CUDA device available for the B200 time-marching path";
    *out = s;
    return NSF_ERR_CUDA;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    s->err = "device is not an sm_100 (Blackwell B200) GPU; this library is built for sm_100a only";
    *out = s;
    return NSF_ERR_CUDA;
  }
  s->nSM = prop.multiProcessorCount;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    s->err = "could not create a CUDA stream";
    *out = s;
    return NSF_ERR_CUDA;
  }
  *out = s;
  return NSF_OK;
}

nsf_status nsf_initialize(nsf_solver* s) {
  if (!s) return NSF_ERR_ARG;
  if (s->initialized) {
    s->err = "nsf_initialize called twice";
    return NSF_ERR_STATE;
  }
  std::string err;
  nsf_status st = build_setup(s->cfg, s->setup, err);
  if (st != NSF_OK) {
    s->err = err;
    return st;
  }
  if (s->hostOnly) {
    s->initialized = true;
    return NSF_OK;
  }
  if (!s->stream) return NSF_ERR_CUDA;
  CK(cudaSetDevice(s->device));
  st = build_device(s);
  if (st != NSF_OK) return st;
  s->initialized = true;
  return NSF_OK;
}

nsf_status nsf_march(nsf_solver* s, uint64_t nsteps) {
  if (!s) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) {
    s->err = s->hostOnly ? "host-only handle (device -1) cannot march" : "nsf_march before nsf_initialize";
    return NSF_ERR_STATE;
  }
  CK(cudaSetDevice(s->device));
  for (uint64_t q = 0; q < nsteps; ++q) CK(cudaGraphLaunch(s->graphExec, s->stream));
  return NSF_OK;
}

// The control block after everything queued on the solver's stream: one copy into page-locked memory
// queued behind that work, then one wait.
static nsf_status read_ctl(nsf_solver* s, StepCtl* out) {
  if (!s->hCtl) CK(cudaMallocHost(&s->hCtl, sizeof(StepCtl)));
  CK(cudaMemcpyAsync(s->hCtl, s->dCtl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *out = *s->hCtl;
  return NSF_OK;
}

nsf_status nsf_sync(nsf_solver* s) {
  if (!s || !s->initialized || s->hostOnly) return s ? NSF_ERR_STATE : NSF_ERR_ARG;
  StepCtl ctl;
  const nsf_status st = read_ctl(s, &ctl);
  if (st != NSF_OK) return st;
  if (ctl.timeout) {
    s->err = "a bounded wait in the stage kernel gave up; results of the affected steps are invalid";
    return NSF_ERR_TIMEOUT;
  }
  if (ctl.nonFinite) {
    s->err = "Non-finite value found in the conserved variables";
    return NSF_ERR_NONFINITE;
  }
  return NSF_OK;
}

nsf_status nsf_debug_wait_limit(nsf_solver* s, uint64_t polls, int32_t withhold_epilogue) {
  if (!s || !s->initialized || s->hostOnly) return s ? NSF_ERR_STATE : NSF_ERR_ARG;
  CK(cudaSetDevice(s->device));
  CK(cudaStreamSynchronize(s->stream));
  const long long lim = static_cast<long long>(polls);
  const int wh = withhold_epilogue ? 1 : 0;
  char* base = reinterpret_cast<char*>(s->dCtl);
  CK(cudaMemcpy(base + offsetof(StepCtl, waitLimit), &lim, sizeof lim, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(base + offsetof(StepCtl, withhold), &wh, sizeof wh, cudaMemcpyHostToDevice));
  return NSF_OK;
}

nsf_status nsf_get_body_interaction(nsf_solver* s, int32_t* interact) {
  if (!s || !interact) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  *interact = s->setup.bodiesInteract ? 1 : 0;
  return NSF_OK;
}

nsf_status nsf_get_time(nsf_solver* s, double* t, uint64_t* level, double* dt) {
  if (!s || !s->initialized || s->hostOnly) return s ? NSF_ERR_STATE : NSF_ERR_ARG;
  StepCtl ctl;
  const nsf_status st = read_ctl(s, &ctl);
  if (st != NSF_OK) return st;
  if (t) *t = ctl.t;
  if (level) *level = ctl.level;
  if (dt) *dt = ctl.dt;
  return NSF_OK;
}


nsf_status nsf_download(nsf_solver* s, uint32_t mask, double* host) {
  if (!s || !host) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  int nf = 0;
  const SnapSlots sl = snap_slots(mask, &nf);
  if (!nf) return NSF_OK;
  CK(cudaSetDevice(s->device));
  if ((mask & ~0x1Fu) == 0) {  // conserved fields only: copied straight from their current buffers
    StepCtl ctl;
    const nsf_status st = read_ctl(s, &ctl);
    if (st != NSF_OK) return st;
    const HostSetup& S = s->setup;
    const size_t hp = S.NK * sizeof(double), dp = size_t(s->hGrid.NKp) * sizeof(double);
    for (int f = 0; f < 5; ++f)
      if (sl.slot[f] >= 0)
        CK(cudaMemcpy2DAsync(host + size_t(sl.slot[f]) * S.N, hp, s->hGrid.bufs[ctl.perm[f][0]][f], dp, hp,
                             S.NI * S.NJ, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return NSF_OK;
  }
  const size_t bytes = size_t(nf) * s->setup.N * sizeof(double);
  double* tmp = nullptr;
  CK(cudaMalloc(&tmp, bytes));
  launch_snapshot(s->dGrid, sl, snap_inactive(s), tmp, s->nSM, s->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(s, e, "download");
  return NSF_OK;
}

nsf_status nsf_download_async(nsf_solver* s, uint32_t mask, double* host, uint64_t* ticket) {
  if (!s || !host || !ticket) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  if (s->grouped) {
    s->err = "nsf_download_async: the handle is a member of an ensemble or slab group (use nsf_download)";
    return NSF_ERR_STATE;
  }
  int nf = 0;
  const SnapSlots sl = snap_slots(mask, &nf);
  if (!nf) {
    s->err = "nsf_download_async: the field mask selects no field";
    return NSF_ERR_ARG;
  }
  CK(cudaSetDevice(s->device));
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, host) != cudaSuccess || pa.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    s->err = "nsf_download_async: the host buffer is not page-locked (nsf_host_alloc)";
    return NSF_ERR_ARG;
  }
  if (!s->dlStream) {
    CK(cudaStreamCreateWithFlags(&s->dlStream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      CK(cudaEventCreateWithFlags(&s->dlTaken[b], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&s->dlDone[b], cudaEventDisableTiming));
    }
  }
  const uint64_t t = s->dlIssued.load() + 1;
  const int b = int(t & 1u);
  const size_t count = size_t(nf) * s->setup.N;
  if (s->dlCap[b] < count) {
    CK(cudaEventSynchronize(s->dlDone[b]));  // the buffer's last copy to the host has finished
    if (s->dlStage[b]) CK(cudaFree(s->dlStage[b]));
    s->dlStage[b] = nullptr;
    s->dlCap[b] = 0;
    CK(cudaMalloc(&s->dlStage[b], count * sizeof(double)));
    s->dlCap[b] = count;
  }
  // the snapshot overwrites the buffer only after its previous copy to the host has left it
  CK(cudaStreamWaitEvent(s->stream, s->dlDone[b], 0));
  launch_snapshot(s->dGrid, sl, snap_inactive(s), s->dlStage[b], s->nSM, s->stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(s->dlTaken[b], s->stream));
  CK(cudaStreamWaitEvent(s->dlStream, s->dlTaken[b], 0));
  CK(cudaMemcpyAsync(host, s->dlStage[b], count * sizeof(double), cudaMemcpyDeviceToHost, s->dlStream));
  CK(cudaEventRecord(s->dlDone[b], s->dlStream));
  s->dlIssued.store(t);
  *ticket = t;
  return NSF_OK;
}

// Ticket t's copy is done once buffer (t & 1)'s done event has completed: that event marks t's copy or, if
// the buffer was reused since, a later copy that started after t's had finished.
nsf_status nsf_download_wait(nsf_solver* s, uint64_t ticket) {
  if (!s) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  if (ticket == 0 || ticket > s->dlIssued.load()) return NSF_ERR_ARG;
  if (cudaSetDevice(s->device) != cudaSuccess || cudaEventSynchronize(s->dlDone[ticket & 1u]) != cudaSuccess)
    return NSF_ERR_CUDA;
  return NSF_OK;
}

nsf_status nsf_download_done(nsf_solver* s, uint64_t ticket, int32_t* done) {
  if (!s || !done) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  if (ticket == 0 || ticket > s->dlIssued.load()) return NSF_ERR_ARG;
  if (cudaSetDevice(s->device) != cudaSuccess) return NSF_ERR_CUDA;
  const cudaError_t e = cudaEventQuery(s->dlDone[ticket & 1u]);
  if (e == cudaErrorNotReady) {
    *done = 0;
    return NSF_OK;
  }
  if (e != cudaSuccess) return NSF_ERR_CUDA;
  *done = 1;
  return NSF_OK;
}

nsf_status nsf_host_alloc(size_t bytes, void** out) {
  if (!out) return NSF_ERR_ARG;
  *out = nullptr;
  if (!bytes) return NSF_ERR_ARG;
  if (cudaHostAlloc(out, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return NSF_ERR_CUDA;
  }
  return NSF_OK;
}

nsf_status nsf_host_free(void* p) {
  if (p && cudaFreeHost(p) != cudaSuccess) return NSF_ERR_CUDA;
  return NSF_OK;
}

nsf_status nsf_upload_conserved(nsf_solver* s, const double* host) {
  if (!s || !host) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  StepCtl ctl;
  const nsf_status st = read_ctl(s, &ctl);
  if (st != NSF_OK) return st;
  const HostSetup& S = s->setup;
  const size_t N = S.N, NKp = size_t(s->hGrid.NKp);
  for (int f = 0; f < 5; ++f)
    CK(cudaMemcpy2DAsync(s->hGrid.bufs[ctl.perm[f][0]][f], NKp * sizeof(double), host + f * N, S.NK * sizeof(double),
                         S.NK * sizeof(double), S.NI * S.NJ, cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return NSF_OK;
}

nsf_status nsf_get_node_types(nsf_solver* s, uint8_t* out) {
  if (!s || !out) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  std::memcpy(out, s->setup.type.data(), s->setup.N);
  return NSF_OK;
}

nsf_status nsf_get_geometry(nsf_solver* s, double* out) {
  if (!s || !out) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  for (int a = 0; a < 3; ++a) {
    out[a] = s->setup.d[a];
    out[3 + a] = s->setup.off[a];
  }
  return NSF_OK;
}

nsf_status nsf_get_num_bodies(nsf_solver* s, uint32_t* nb) {
  if (!s || !nb) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  *nb = uint32_t(s->setup.bodies.size());
  return NSF_OK;
}

nsf_status nsf_get_body_counts(nsf_solver* s, uint32_t body, uint64_t* ng, uint64_t* nf, uint64_t* cl) {
  if (!s) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  if (body >= s->setup.bodies.size()) return NSF_ERR_ARG;
  const BodyRec& b = s->setup.bodies[body];
  if (ng) *ng = b.ghosts.size();
  if (nf) *nf = b.filter.size();
  if (cl) *cl = b.closureAdded;
  return NSF_OK;
}

nsf_status nsf_get_ghosts(nsf_solver* s, uint32_t body, double* out) {
  if (!s || !out) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  if (body >= s->setup.bodies.size()) return NSF_ERR_ARG;
  const BodyRec& b = s->setup.bodies[body];
  for (size_t q = 0; q < b.ghosts.size(); ++q) {
    const GhostRec& g = b.ghosts[q];
    double row[9] = {double(g.i), double(g.j), double(g.k), g.bi[0], g.bi[1], g.bi[2], g.ip[0], g.ip[1], g.ip[2]};
    std::memcpy(out + 9 * q, row, sizeof row);
  }
  return NSF_OK;
}

nsf_status nsf_get_filter_nodes(nsf_solver* s, uint32_t body, uint64_t* out) {
  if (!s || !out) return NSF_ERR_ARG;
  if (!s->initialized) return NSF_ERR_STATE;
  if (body >= s->setup.bodies.size()) return NSF_ERR_ARG;
  const BodyRec& b = s->setup.bodies[body];
  for (size_t q = 0; q < b.filter.size(); ++q) out[q] = b.filter[q];
  return NSF_OK;
}

nsf_status nsf_get_history(nsf_solver* s, uint64_t first, uint64_t count, double* out, uint64_t* available) {
  if (!s) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  CK(cudaStreamSynchronize(s->stream));
  StepCtl ctl;
  CK(cudaMemcpy(&ctl, s->dCtl, sizeof ctl, cudaMemcpyDeviceToHost));
  if (available) *available = ctl.level;
  if (!out || !count) return NSF_OK;
  if (first + count > ctl.level || ctl.level - first > (uint64_t)MAX_HIST) {
    s->err = "history rows out of range (only the last 2^20 steps are kept on the device)";
    return NSF_ERR_ARG;
  }
  for (uint64_t q = 0; q < count; ++q)
    CK(cudaMemcpy(out + 7 * q, s->hGrid.hist + 7 * ((first + q) % MAX_HIST), 7 * sizeof(double), cudaMemcpyDeviceToHost));
  return NSF_OK;
}

nsf_status nsf_march_timed(nsf_solver* s, uint64_t nsteps, double* elapsed_ms) {
  if (!s || !elapsed_ms) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  CK(cudaSetDevice(s->device));
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, s->stream));
  for (uint64_t q = 0; q < nsteps; ++q) CK(cudaGraphLaunch(s->graphExec, s->stream));
  CK(cudaEventRecord(b, s->stream));
  CK(cudaEventSynchronize(b));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *elapsed_ms = ms;
  return NSF_OK;
}

// Steps per replay of the profiling graph: the graph holds this many RK4 steps back to back, as
// consecutive replays of the step graph run them, with event nodes around the stage kernels.
constexpr int kProfileSteps = 10;

static nsf_status build_profile_graph(nsf_solver* s) {
  s->profEv.assign(2 + 8 * kProfileSteps, nullptr);
  for (auto& e : s->profEv) CK(cudaEventCreate(&e));
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaEventRecordWithFlags(s->profEv[0], s->stream, cudaEventRecordExternal);
  for (int q = 0; q < kProfileSteps && e == cudaSuccess; ++q) {
    enqueue_step_profiled(s->dGrid, s->hGrid, s->plan, s->stream, s->profEv.data() + 2 + 8 * q, true);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(s->profEv[1], s->stream, cudaEventRecordExternal);
  const cudaError_t e2 = cudaStreamEndCapture(s->stream, &s->profGraph);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s->profExec, s->profGraph, 0);
  if (e != cudaSuccess) return cuda_fail(s, e, "capture of the profiling graph");
  return NSF_OK;
}

nsf_status nsf_profile_steps(nsf_solver* s, uint64_t nsteps, double* stage_ms, double* step_ms) {
  if (!s || !stage_ms || !step_ms) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  CK(cudaSetDevice(s->device));
  if (!s->profExec) {
    const nsf_status st = build_profile_graph(s);
    if (st != NSF_OK) return st;
  }
  const uint64_t reps = (nsteps + kProfileSteps - 1) / kProfileSteps;
  double tot[4] = {0, 0, 0, 0}, whole = 0;
  for (uint64_t r = 0; r < reps; ++r) {
    CK(cudaGraphLaunch(s->profExec, s->stream));
    CK(cudaEventSynchronize(s->profEv[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, s->profEv[0], s->profEv[1]));
    whole += ms;
    for (int q = 0; q < kProfileSteps; ++q)
      for (int st = 0; st < 4; ++st) {
        CK(cudaEventElapsedTime(&ms, s->profEv[2 + 8 * q + 2 * st], s->profEv[2 + 8 * q + 2 * st + 1]));
        tot[st] += ms;
      }
  }
  const double n = double(reps ? reps * kProfileSteps : 1);
  *step_ms = whole / n;
  for (int st = 0; st < 4; ++st) stage_ms[st] = tot[st] / n;
  return NSF_OK;
}

nsf_status nsf_launches_per_step(nsf_solver* s, uint64_t* n) {
  if (!s || !n) return NSF_ERR_ARG;
  if (!s->initialized || s->hostOnly) return NSF_ERR_STATE;
  *n = uint64_t(s->launchesPerStep);
  return NSF_OK;
}

const char* nsf_last_error(nsf_solver* s) { return s ? s->err.c_str() : "null solver handle"; }

void nsf_destroy(nsf_solver* s) {
  if (!s) return;
  if (s->stream) {
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
  }
  if (s->graphExec) cudaGraphExecDestroy(s->graphExec);
  if (s->graph) cudaGraphDestroy(s->graph);
  if (s->profExec) cudaGraphExecDestroy(s->profExec);
  if (s->profGraph) cudaGraphDestroy(s->profGraph);
  for (cudaEvent_t e : s->profEv)
    if (e) cudaEventDestroy(e);
  nsf_adjoint_free(s);
  if (s->dlStream) {
    cudaStreamSynchronize(s->dlStream);
    for (int b = 0; b < 2; ++b) {
      if (s->dlStage[b]) cudaFree(s->dlStage[b]);
      if (s->dlTaken[b]) cudaEventDestroy(s->dlTaken[b]);
      if (s->dlDone[b]) cudaEventDestroy(s->dlDone[b]);
    }
    cudaStreamDestroy(s->dlStream);
  }
  for (void* p : s->allocs) cudaFree(p);
  if (s->hCtl) cudaFreeHost(s->hCtl);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

nsf_status nsf_math_selftest(int32_t device, uint64_t n, const double* x, double* out) {
  if (n && (!x || !out)) return NSF_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return NSF_ERR_CUDA;
  return math_selftest((long long)n, x, out) == 0 ? NSF_OK : NSF_ERR_CUDA;
}

}  // extern "C"
