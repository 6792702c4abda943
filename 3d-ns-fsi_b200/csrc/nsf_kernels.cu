// CUDA kernels (sm_100a, FP64) of the RK4 time-marching path. One RK4 step (Solver::marchTimeStep,
// Solver.cpp:130-167) is the launch sequence enqueue_step() builds:
//
//   k_prologue            stop criterion, filter decision, buffer roles        (Solver.cpp:133-135)
//   k_density_filter      global 2nd-order density filter, rare              (Mesh.cpp:108-140)
//   4 x { k_stage_ws      fused RHS + primitive recompute + RK4 combine      (Solver.cpp:141-159, 170-507;
//                         TMA-fed, warp-specialised: nsf_stage_ws.cu)
//         k_solid_copy    stale solid-node values, I -> O                    (buffer semantics, see nsf_device.cuh)
//         k_edge_bc x3    outlet/inlet, then y faces, then z faces           (Boundary.cpp:250-417)
//         k_body_filter   near-body filter of rho, rho_E                     (Boundary.cpp:618-652)
//         k_ghost         image-point interpolation with cached weights      (Boundary.cpp:427-457, 655-883) }
//   k_finalize            change norms, next dt, time, history              (Solver.cpp:80-126, 510-530)
//
// Stage 4 also carries the dt maxima, the change norms and the NaN check as block reductions, so no
// kernel re-reads the fields for them.
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cuda_runtime.h>

#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_physics.cuh"

namespace nsf {

// ----------------------------------------------------------------------------------------------
// Prologue: Simulation::checkStoppingCriterion (end_time), Mesh::checkFilterCondition (Mesh.cpp:85-103),
// the buffer swaps of Mesh.cpp:133-151 expressed as role changes, and per-stage buffer roles.
// Member m = blockIdx.x of the grid array (a single grid: one block).
__global__ void k_prologue(Grid* grids) {
  if (threadIdx.x != 0) return;
  Grid* g = grids + blockIdx.x;
  StepCtl* c = g->ctl;
  for (int f = 0; f < 5; ++f) g->normPart[f] = 0.0;  // slot 0: the ensemble stage kernel adds into it
  const Consts& C = g->C;
  c->active = C.endTime ? (c->t < C.tEnd) : 1;
  if (!c->active) return;
  int counter = 0;
  for (int q = 0; q < C.nChange; ++q)
    if (c->t > C.changeT[q]) ++counter;
  int filt = 0;
  if (counter < C.nFilterIv) {
    unsigned iv = C.filterIv[counter];
    if (iv > 0 && (c->level + 1) % iv == 0) filt = 1;
  }
  c->filterNow = filt;
  int cons[5], old[5], scr[5];
  for (int f = 0; f < 5; ++f) {
    cons[f] = c->perm[f][0];
    old[f] = c->perm[f][1];
    scr[f] = c->perm[f][2];
  }
  if (filt) {  // the filter writes rho into the old buffer, then the two rho buffers trade places
    c->gfSrc = g->bufs[cons[0]][0];
    c->gfDst = g->bufs[old[0]][0];
    int t = cons[0];
    cons[0] = old[0];
    old[0] = t;
  }
  for (int f = 0; f < 5; ++f) {  // swapConservedVariables
    int t = cons[f];
    cons[f] = old[f];
    old[f] = t;
  }
  int A[5], B[5];
  for (int f = 0; f < 5; ++f) {
    A[f] = cons[f];
    B[f] = scr[f];
  }
  if (filt) {  // stage 1 cannot write the unfiltered density it reads: it writes the scratch buffer
    A[0] = scr[0];
    B[0] = cons[0];
  }
  for (int f = 0; f < 5; ++f) {
    c->u0Phys[f] = old[f];
    c->iPhys[0][f] = old[f];
    c->iPhys[1][f] = A[f];
    c->iPhys[2][f] = B[f];
    c->iPhys[3][f] = A[f];
  }
  c->rPhys[0] = filt ? cons[0] : old[0];
  c->rPhys[1] = A[0];
  c->rPhys[2] = B[0];
  c->rPhys[3] = A[0];
  for (int f = 0; f < 5; ++f) {
    c->U0[f] = g->bufs[old[f]][f];
    c->I[0][f] = g->bufs[old[f]][f];
    c->O[0][f] = g->bufs[A[f]][f];
    c->I[1][f] = g->bufs[A[f]][f];
    c->O[1][f] = g->bufs[B[f]][f];
    c->I[2][f] = g->bufs[B[f]][f];
    c->O[2][f] = g->bufs[A[f]][f];
    c->I[3][f] = g->bufs[A[f]][f];
    c->O[3][f] = g->bufs[B[f]][f];
  }
  c->R[0] = filt ? g->bufs[cons[0]][0] : g->bufs[old[0]][0];
  c->R[1] = g->bufs[A[0]][0];
  c->R[2] = g->bufs[B[0]][0];
  c->R[3] = g->bufs[A[0]][0];
  c->copyMask[0] = filt ? 1 : 0;
  c->copyMask[1] = c->copyMask[2] = c->copyMask[3] = 31;
  const double dt = c->dt;
  c->dtUsed = dt;
  c->stageT[0] = c->t + dt / 2;
  c->stageT[1] = c->t + dt / 2;
  c->stageT[2] = c->t + dt;
  c->stageT[3] = c->t + dt;
  for (int f = 0; f < 5; ++f) {  // roles after the step: final state = B, scratch = A
    c->perm[f][0] = B[f];
    c->perm[f][1] = old[f];
    c->perm[f][2] = A[f];
  }
  for (int q = 0; q < 4; ++q) c->mx[q] = 0ull;
  if (g->ctlHist && c->level < (unsigned long long)g->nCtlHist) g->ctlHist[c->level] = *c;
}

// Mesh::applyFilter_ifAppropriate body (Mesh.cpp:110-134): interior nodes get the 7-point filter,
// every node of an edge boundary's owned box (whatever its type) and every solid-ghost node is copied,
// the remaining solid inactive nodes are left as they are.
__global__ void k_density_filter(const Grid* __restrict__ grids) {
  const Grid* g = grids + blockIdx.y;
  const StepCtl* c = g->ctl;
  if (!c->active || !c->filterNow) return;
  const double* __restrict__ src = c->gfSrc;
  double* __restrict__ dst = c->gfDst;
  const long long sI = g->sI, sJ = g->sJ;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g->N; n += (long long)gridDim.x * blockDim.x) {
    const uint8_t raw = g->type[n], t = raw & TYPE_MASK;
    if (t == FLUID_INTERIOR)
      dst[n] = (6 * src[n] + src[n + sI] + src[n - sI] + src[n + sJ] + src[n - sJ] + src[n + 1] + src[n - 1]) / 12;
    else if (t != SOLID_INACTIVE || (raw & EDGE_PLANE_BIT))
      dst[n] = src[n];
  }
}

// ----------------------------------------------------------------------------------------------
// Solid-node values the reference's stage buffer still holds from earlier writes (see nsf_device.cuh).
// One solid node q of a grid; the device functions here are shared by the separate kernels and the fused
// boundary kernel (k_bc), which reads fields written earlier in the same launch: those reads bypass L1.
__device__ __forceinline__ void solid_copy_item(const Grid& G, const StepCtl* c, int s, int mask, int q) {
  const long long n = G.snode[q];
  if (mask & 1) c->O[s][0][n] = __ldcg(c->R[s] + n);
  for (int f = 1; f < 5; ++f)
    if (mask & (1 << f)) c->O[s][f][n] = __ldcg(c->I[s][f] + n);
}

// Field f at node m as the stage's boundary work reads it after the solid-node copy. For a solid node off
// the mesh faces (solid = true; nothing but the copy writes it in a stage) the value comes from the copy's
// source, so the reader does not wait for the copy; the values are the same either way.
__device__ __forceinline__ double ld_res(const StepCtl* c, int s, int f, long long m, bool solid) {
  if (solid && (c->copyMask[s] & (1 << f))) return __ldcg((f == 0 ? c->R[s] : c->I[s][f]) + m);
  return __ldcg(c->O[s][f] + m);
}

__global__ void k_solid_copy(const Grid* __restrict__ grids, int s) {
  const Grid* g = grids + blockIdx.y;
  const StepCtl* c = g->ctl;
  if (!c->active) return;
  const int mask = c->copyMask[s];
  if (!mask) return;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < g->nSolid; q += gridDim.x * blockDim.x)
    solid_copy_item(*g, c, s, mask, q);
}

// ----------------------------------------------------------------------------------------------
// Mesh-edge boundary conditions of one axis (both faces; the faces of one axis never read each other's
// nodes). Launched for x, then y, then z: the reference's application order outlet/inlet (x), y-max,
// y-min, z-max, z-min (Mesh.cpp:155-167 after the reversal at Mesh.cpp:70). Each block comes from the
// launch plan's list (member, face, first in-plane coordinates, mask of the nodes it works on).
// periodic_source: the node a periodic face node finally copies -- the opposite interior-plane node, and if
// that node lies on another periodic face (which copied it earlier in the reference's order), that face's
// source, and so on (at most two more hops). The copies are exact, so reading the final source gives the
// value the reference copies; it lets chains of copies run together (nsf_bc_plan.cpp).
// edge_node: one node (thread tx, ty of an edge block) of a mesh-edge boundary condition; adds the stage-4
// dt terms and the NaN check of edge and ghost-typed nodes.
__device__ __forceinline__ void periodic_source(const Grid& G, int axis, int side, int ijk[3]) {
  const int nAx[3] = {G.NI, G.NJ, G.NK};
  ijk[axis] = side == 0 ? nAx[axis] - 2 : 1;
  for (int hop = 0; hop < 2; ++hop) {
    int found = -1;
    for (int e = 0; e < G.nEdge && found < 0; ++e) {
      const int* b = G.eBox[e];
      if (G.eBc[e] == NSF_BC_PERIODIC && ijk[0] >= b[0] && ijk[0] <= b[1] && ijk[1] >= b[2] && ijk[1] <= b[3] &&
          ijk[2] >= b[4] && ijk[2] <= b[5])
        found = e;
    }
    if (found < 0) return;
    const int a = G.eAxis[found];
    ijk[a] = G.eSide[found] == 0 ? nAx[a] - 2 : 1;
  }
}

__device__ __forceinline__ void edge_node(const Grid& G, const StepCtl* c, const EdgeBlock& eb, int tx, int ty, int s,
                                          int axis, DtAcc& dta, int& bad) {
  const Consts& C = G.C;
  const int e = eb.e;
  {
    const int* b = G.eBox[e];
    // in-plane coordinates: (a, bb) = the two axes other than `axis`, in (i, j, k) order
    const int ax1 = axis == 0 ? 1 : 0, ax2 = axis == 2 ? 1 : 2;
    const int a = eb.a0 + ty;
    const int bb = eb.b0 + tx;
    if (a <= b[2 * ax1 + 1] && bb <= b[2 * ax2 + 1] && ((eb.mask >> (ty * 32 + tx)) & 1)) {
      int ijk[3];
      ijk[axis] = b[2 * axis];
      ijk[ax1] = a;
      ijk[ax2] = bb;
      const long long st = axis == 0 ? G.sI : axis == 1 ? G.sJ : 1;
      const long long n = ijk[0] * G.sI + ijk[1] * G.sJ + ijk[2];
      const int side = G.eSide[e], bc = G.eBc[e];
      double* const* O = c->O[s];
      const bool solidSrc = (eb.solidSrc >> (ty * 32 + tx)) & 1;
      auto ld = [&](int f, long long m) { return ld_res(c, s, f, m, solidSrc); };
      const long long a1 = side == 0 ? n + st : n - st, a2 = side == 0 ? n + 2 * st : n - 2 * st;  // Boundary.cpp:74-108
      double cv[5];
      double u = 0, v = 0, w = 0, p = 0, T = 0;
      bool primKnown = false;
      if (bc == NSF_BC_INLET) {  // Boundary.cpp:250-296 with filterInletDensity :142-245
        // extrapolated density of this node and of its in-plane neighbours inside the owned box
        const long long s1 = ax1 == 0 ? G.sI : G.sJ, s2 = ax2 == 1 ? G.sJ : 1;
        auto ext = [&](long long m) { return 2 * ld(0, side == 0 ? m + st : m - st) - ld(0, side == 0 ? m + 2 * st : m - 2 * st); };
        double f = 0;
        unsigned nn = 0;
        if (a < b[2 * ax1 + 1]) { f += ext(n + s1); ++nn; }
        if (a > b[2 * ax1]) { f += ext(n - s1); ++nn; }
        if (bb < b[2 * ax2 + 1]) { f += ext(n + s2); ++nn; }
        if (bb > b[2 * ax2]) { f += ext(n - s2); ++nn; }
        f += nn * ext(n);
        f /= 2 * nn;
        const double rho = f;
        double vel = fmin(1., c->stageT[s] / 10.) * C.m0;
        if (G.inflow && axis == 0) vel *= G.inflow[a * G.NKp + bb];  // profile factor (1 in a plain run)
        if (side == 1) vel *= -1;
        u = axis == 0 ? vel : 0;
        v = axis == 1 ? vel : 0;
        w = axis == 2 ? vel : 0;
        T = 0;
        p = (T * (1 + rho) + rho) / C.gamma;
        cons_of(C, u, v, w, p, T, cv);
        primKnown = true;
      } else if (bc == NSF_BC_OUTLET) {  // Boundary.cpp:304-336
        const double rho = 2 * ld(0, a1) - ld(0, a2);
        const double ru = 2 * ld(1, a1) - ld(1, a2);
        const double rv = 2 * ld(2, a1) - ld(2, a2);
        const double rw = 2 * ld(3, a1) - ld(3, a2);
        p = 0;
        u = ru / (1 + rho);
        v = rv / (1 + rho);
        w = rw / (1 + rho);
        T = (C.gamma * p - rho) / (1 + rho);
        cv[0] = rho;
        cv[1] = ru;
        cv[2] = rv;
        cv[3] = rw;
        cv[4] = p / C.gm1 + (1 + rho) / 2 * (u * u + v * v + w * w);
        primKnown = true;
      } else if (bc == BC_SLAB_COPY) {  // an x-slab's periodic x face: already copied by the plane exchange
        for (int f = 0; f < 5; ++f) cv[f] = ld(f, n);
      } else if (bc == NSF_BC_PERIODIC) {  // Boundary.cpp:344-367, opposite index :111-133
        int src[3] = {ijk[0], ijk[1], ijk[2]};
        periodic_source(G, axis, side, src);
        const long long m = src[0] * G.sI + src[1] * G.sJ + src[2];
        for (int f = 0; f < 5; ++f) cv[f] = ld(f, m);
      } else {  // symmetry, Boundary.cpp:377-417: mirror the primitives of the second interior node
        const Prim q = prims_of(C, ld(0, a2), ld(1, a2), ld(2, a2), ld(3, a2), ld(4, a2));
        u = q.u;
        v = q.v;
        w = q.w;
        if (axis == 0) u = -q.u;
        if (axis == 1) v = -q.v;
        if (axis == 2) w = -q.w;
        p = q.p;
        T = q.T;
        cons_of(C, u, v, w, p, T, cv);
        primKnown = true;
      }
      for (int f = 0; f < 5; ++f) O[f][n] = cv[f];
      if (s == 3) {
        const uint8_t t = G.type[n] & TYPE_MASK;
        if (t == FLUID_EDGE || t == FLUID_GHOST) {
          double mu;
          if (primKnown) {
            mu = mu_of_T(C, T);
          } else {
            const Prim q = prims_of(C, cv[0], cv[1], cv[2], cv[3], cv[4]);
            u = q.u;
            v = q.v;
            w = q.w;
            p = q.p;
            mu = q.mu;
          }
          dta.add(C, cv[0], u, v, w, p, mu);
          for (int f = 0; f < 5; ++f) bad |= !isfinite(cv[f]);
        }
      }
    }
  }
}

__global__ void k_edge_bc(const Grid* __restrict__ grids, const EdgeBlock* __restrict__ blocks, int s, int axis) {
  __shared__ double red[4 * 32];
  const EdgeBlock eb = blocks[blockIdx.x];  // every listed block holds nodes of its face
  const Grid& G = grids[eb.g];
  StepCtl* c = G.ctl;
  if (!c->active) return;
  DtAcc dta;
  int bad = 0;
  edge_node(G, c, eb, threadIdx.x, threadIdx.y, s, axis, dta, bad);
  if (s == 3) {
    flush_dt(c, dta, red);
    if (bad) atomicOr(&c->nonFinite, 1);
  }
}

// ----------------------------------------------------------------------------------------------
// Near-body filter (ImmersedBoundary::filterClosestFluidNodes, Boundary.cpp:618-652). Jacobi: every
// filtered value is computed from unfiltered neighbours; results go to fnew and are written back by
// the ghost pass. The values before the filter go to fpre: the reference does not recompute the primitive
// variables of these nodes after filtering, so the next stage builds their primitives from fpre.
// filter_item: filter node f of a grid (stage-4 dt terms, change norms of rho and rho_E, NaN check).
__device__ __forceinline__ void filter_item(const Grid& G, const StepCtl* c, int s, int f, DtAcc& dta, double nsum[5],
                                            int& bad) {
  double* const* O = c->O[s];
  const long long n = G.fnode[f];
  const unsigned sb = G.fsolid ? G.fsolid[f] : 0u;
  auto r = [&](long long m, int q) { return ld_res(c, s, 0, m, (sb >> q) & 1); };
  auto e = [&](long long m, int q) { return ld_res(c, s, 4, m, (sb >> q) & 1); };
  const double r0 = r(n, 0), e0 = e(n, 0);
  const double rf =
      (6 * r0 + r(n + G.sI, 1) + r(n - G.sI, 2) + r(n + G.sJ, 3) + r(n - G.sJ, 4) + r(n + 1, 5) + r(n - 1, 6)) / 12;
  const double ef =
      (6 * e0 + e(n + G.sI, 1) + e(n - G.sI, 2) + e(n + G.sJ, 3) + e(n - G.sJ, 4) + e(n + 1, 5) + e(n - 1, 6)) / 12;
  G.fpre[2 * f] = r0;
  G.fpre[2 * f + 1] = e0;
  G.fnew[2 * f] = rf;
  G.fnew[2 * f + 1] = ef;
  // stage 4: the node's dt and change-norm terms, once, from its last slot (a node two bodies filter has
  // two): the final filtered values, and primitives from the values before the node's first filter
  const int meta = G.fmeta ? G.fmeta[f] : (f | FMETA_LAST);
  if (s == 3 && (meta & FMETA_LAST)) {
    const int first = meta & ~FMETA_LAST;
    const double p0 = first == f ? r0 : __ldcg(G.fpre + 2 * first);
    const double p4 = first == f ? e0 : __ldcg(G.fpre + 2 * first + 1);
    const Prim q = prims_of(G.C, p0, __ldcg(O[1] + n), __ldcg(O[2] + n), __ldcg(O[3] + n), p4);
    dta.add(G.C, rf, q.u, q.v, q.w, q.p, q.mu);
    const double d0 = c->U0[0][n] - rf, d4 = c->U0[4][n] - ef;
    nsum[0] += d0 * d0;
    nsum[4] += d4 * d4;
    bad |= !isfinite(rf) || !isfinite(ef);
  }
}

__global__ void k_body_filter(const Grid* __restrict__ grids, int s) {
  __shared__ double red[5 * 32];
  const Grid& G = grids[blockIdx.y];
  StepCtl* c = G.ctl;
  if (!c->active) return;
  DtAcc dta;
  double nsum[5] = {0, 0, 0, 0, 0};
  int bad = 0;
  // a block past this member's filter nodes never writes its norm slot, which stays zero
  if (int(blockIdx.x * blockDim.x) >= G.nFilter) return;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < G.nFilter; f += gridDim.x * blockDim.x)
    filter_item(G, c, s, f, dta, nsum, bad);
  if (s == 3) {
    flush_dt(c, dta, red);
    flush_norms(G.normPart + 5 * (G.normSlotFilter + blockIdx.x), nsum, red);
    if (bad) atomicOr(&c->nonFinite, 1);
  }
}

// Ghost nodes (Boundary.cpp:432-456): image-point value = cached weights x the 8 surrounding values
// (Neumann weights for rho and rho_E, Dirichlet weights for the momenta, zero weight on ghost corners);
// ghost value = image value with momentum negated (getGhostNodeBCVariables, :777-785). The ghost lists
// are stored sorted by image-point cell, so the lanes of a warp gather overlapping corner sets; every
// corner's five values are loaded before any is used (40 independent loads in flight per ghost) and summed
// in corner order, skipping corners whose two weights are both zero, as the reference's sums do.
// ghost_pass_item: item q of the ghost pass: q < nGhost a ghost, then the filter write-backs (ghosts read
// the filtered values through fnew), then on stage 4 the solid inactive nodes' dt terms (the reference
// never updates their primitive values).
__device__ __forceinline__ void ghost_pass_item(const Grid& G, const StepCtl* c, int s, int q, DtAcc& dta, int& bad) {
  double* const* O = c->O[s];
  const Consts& C = G.C;
  if (q < G.nGhost) {
    const long long* cell = G.gcell + 8 * (long long)q;
    const double* w = G.gw + 16 * (long long)q;
    double v[8][5], wn[8], wd[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const long long cn = cell[m];
      wn[m] = w[m];
      wd[m] = w[8 + m];
#pragma unroll
      for (int f = 0; f < 5; ++f) v[m][f] = __ldcg(O[f] + cn);
      const int fi = G.gsrc[8 * (long long)q + m];  // a filter corner: the filtered values it sees
      if (fi >= 0) {
        v[m][0] = __ldcg(G.fnew + 2 * fi);
        v[m][4] = __ldcg(G.fnew + 2 * fi + 1);
      }
    }
    double ip[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if (wn[m] == 0.0 && wd[m] == 0.0) continue;
      ip[0] += wn[m] * v[m][0];
      ip[4] += wn[m] * v[m][4];
      ip[1] += wd[m] * v[m][1];
      ip[2] += wd[m] * v[m][2];
      ip[3] += wd[m] * v[m][3];
    }
    const double gc[5] = {ip[0], -ip[1], -ip[2], -ip[3], ip[4]};
    const long long n = G.gnode[q];
    for (int f = 0; f < 5; ++f) O[f][n] = gc[f];
    if (s == 3 && G.glast[q]) {  // a node in two bodies' ghost lists: the dt terms of its final values
      const Prim p = prims_of(C, gc[0], gc[1], gc[2], gc[3], gc[4]);
      dta.add(C, gc[0], p.u, p.v, p.w, p.p, p.mu);
      for (int f = 0; f < 5; ++f) bad |= !isfinite(gc[f]);
    }
  } else if (q < G.nGhost + G.nFilter) {
    const int f = q - G.nGhost;
    const long long n = G.fnode[f];
    O[0][n] = __ldcg(G.fnew + 2 * f);
    O[4][n] = __ldcg(G.fnew + 2 * f + 1);
  } else {
    const int z = q - G.nGhost - G.nFilter;
    const long long n = G.inode[z];
    const double* pr = G.iprim + 5 * (long long)z;
    const double r0 = ld_res(c, s, 0, n, true);  // inactive nodes lie off the mesh faces
    if (isnan(pr[0])) {  // periodic copy of a node whose primitives follow its conserved values
      const Prim p = prims_of(C, r0, ld_res(c, s, 1, n, true), ld_res(c, s, 2, n, true), ld_res(c, s, 3, n, true),
                              ld_res(c, s, 4, n, true));
      dta.add(C, r0, p.u, p.v, p.w, p.p, p.mu);
    } else {
      dta.add(C, r0, pr[0], pr[1], pr[2], pr[3], pr[4]);
    }
  }
}

__device__ __forceinline__ int ghost_pass_count(const Grid& G, int s) {
  return G.nGhost + G.nFilter + (s == 3 ? G.nInactive : 0);
}

__global__ void k_ghost(const Grid* __restrict__ grids, int s) {
  __shared__ double red[4 * 32];
  const Grid& G = grids[blockIdx.y];
  StepCtl* c = G.ctl;
  if (!c->active) return;
  DtAcc dta;
  int bad = 0;
  const int total = ghost_pass_count(G, s);
  if (int(blockIdx.x * blockDim.x) >= total) return;  // the whole block is past this member's work
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x)
    ghost_pass_item(G, c, s, q, dta, bad);
  if (s == 3) {
    flush_dt(c, dta, red);
    if (bad) atomicOr(&c->nonFinite, 1);
  }
}

// ----------------------------------------------------------------------------------------------
// End of step: change norms (Mesh::getNormOfChange, Mesh.cpp:171-178), next dt
// (Solver::updateTimeStepSize, Solver.cpp:80-126), t += dt, ++timeLevel, history row. Called by every
// thread of one block (block reductions); red: 5 x 32 doubles of shared memory.
__device__ void finalize_grid(Grid* g, double* red) {
  __shared__ double tot[5];
  const int nSlots = g->nNormSlots;
  StepCtl* c = g->ctl;
  const Consts& C = g->C;
  double s[5] = {0, 0, 0, 0, 0};
  for (int q = threadIdx.x; q < nSlots; q += blockDim.x)
    for (int f = 0; f < 5; ++f) s[f] += __ldcg(g->normPart + 5 * q + f);
  flush_norms(tot, s, red);
  if (threadIdx.x != 0) return;
  double mx[4];
  for (int q = 0; q < 4; ++q) mx[q] = __longlong_as_double(static_cast<long long>(atomicAdd(&c->mx[q], 0ull)));
  const double conv = C.convLim / (mx[0] / C.dx + mx[1] / C.dy + mx[2] / C.dz);
  const double dx2 = C.dx * C.dx, dy2 = C.dy * C.dy, dz2 = C.dz * C.dz;
  const double visc = C.viscLim / (mx[3] * (1 / dx2 + 1 / dy2 + 1 / dz2));
  const double tNew = c->t + c->dtUsed;
  double dt = (visc < conv) ? visc : conv;
  if (C.endTime && tNew + dt > C.tEnd) dt = C.tEnd - tNew;
  if (g->dtFrozen && c->level + 1 < (unsigned long long)g->nDtFrozen) dt = g->dtFrozen[c->level + 1];
  double* h = g->hist + 7 * (c->level % MAX_HIST);
  h[0] = tNew;
  h[1] = c->dtUsed;
  for (int f = 0; f < 5; ++f) {
    const bool kept = (f == 0 && C.convHistory != 0) || C.convHistory == 2;
    h[2 + f] = kept ? sqrt(C.dxdydz * tot[f]) : -1.0;
  }
  c->t = tNew;
  c->dt = dt;
  c->level += 1;
}

__global__ void k_finalize(Grid* grids) {
  __shared__ double red[5 * 32];
  Grid* g = grids + blockIdx.x;
  if (!g->ctl->active) return;
  finalize_grid(g, red);
}

// ----------------------------------------------------------------------------------------------
// Setup: interpolation weights of every ghost node, solved once. For image-point cells whose eight
// nodes are all fluid the weights are those of the reference's nested linear interpolation
// (Boundary.cpp:732-757). Otherwise the reference solves V c = phi with the Vandermonde rows
// [1, x, y, z, xy, xz, yz, xyz] (Neumann rows [0, n, ...] at ghost corners, Boundary.cpp:788-817) and
// evaluates b^T c at the image point; the value is w^T phi with V^T w = b. The system is solved here in
// cell-local scaled coordinates x' = (x - x0)/dx (the bilinear basis is invariant under per-axis affine
// maps; a Neumann row transforms with n'_a = n_a/d_a), which keeps its condition number near 10 instead
// of ~1e6 for the raw coordinates. Gaussian elimination with partial pivoting, in registers, one thread
// per ghost.
__device__ void solve8T(double A[8][8], double b[8]) {
  // solve A^T x = b in place (x returned in b)
  double M[8][8];
  for (int r = 0; r < 8; ++r)
    for (int q = 0; q < 8; ++q) M[r][q] = A[q][r];
  for (int k = 0; k < 8; ++k) {
    int piv = k;
    double best = fabs(M[k][k]);
    for (int r = k + 1; r < 8; ++r)
      if (fabs(M[r][k]) > best) {
        best = fabs(M[r][k]);
        piv = r;
      }
    if (piv != k) {
      for (int q = 0; q < 8; ++q) {
        double t = M[k][q];
        M[k][q] = M[piv][q];
        M[piv][q] = t;
      }
      double t = b[k];
      b[k] = b[piv];
      b[piv] = t;
    }
    for (int r = k + 1; r < 8; ++r) {
      const double l = M[r][k] / M[k][k];
      for (int q = k; q < 8; ++q) M[r][q] -= l * M[k][q];
      b[r] -= l * b[k];
    }
  }
  for (int k = 7; k >= 0; --k) {
    double acc = b[k];
    for (int q = k + 1; q < 8; ++q) acc -= M[k][q] * b[q];
    b[k] = acc / M[k][k];
  }
}

// in: per ghost 8 x (x, y, z) corner points (node position, or body-intercept point for a ghost corner),
// 8 x (nx, ny, nz) unit normals (ghost corners only), 8 flags, image point, lower cell node position.
__global__ void k_ghost_weights(int nGhost, const double* __restrict__ pts, const double* __restrict__ nrm,
                                const uint8_t* __restrict__ flags, const double* __restrict__ ipl,
                                double dx, double dy, double dz, double* __restrict__ wout) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nGhost) return;
  const double* P = pts + 24 * (long long)q;
  const double* Nn = nrm + 24 * (long long)q;
  const uint8_t* fl = flags + 8 * (long long)q;
  const double* L = ipl + 6 * (long long)q;  // image point, lower node position
  const double X = (L[0] - L[3]) / dx, Y = (L[1] - L[4]) / dy, Z = (L[2] - L[5]) / dz;
  double* w = wout + 16 * (long long)q;
  bool anyGhost = false;
  for (int m = 0; m < 8; ++m) anyGhost |= fl[m] != 0;
  if (!anyGhost) {
    // corner m = (di, dj, dk) in asIndexList order: m = 4*di + 2*dj + dk
    for (int m = 0; m < 8; ++m) {
      const int di = m >> 2, dj = (m >> 1) & 1, dk = m & 1;
      const double wv = (di ? X : 1 - X) * (dj ? Y : 1 - Y) * (dk ? Z : 1 - Z);
      w[m] = wv;
      w[8 + m] = wv;
    }
    return;
  }
  for (int set = 0; set < 2; ++set) {  // 0: Neumann rows at ghost corners, 1: Dirichlet everywhere
    double V[8][8], b[8];
    for (int m = 0; m < 8; ++m) {
      const double x = (P[3 * m] - L[3]) / dx, y = (P[3 * m + 1] - L[4]) / dy, z = (P[3 * m + 2] - L[5]) / dz;
      if (set == 0 && fl[m]) {
        const double nx = Nn[3 * m] / (1.0 / dx), ny = Nn[3 * m + 1] / (1.0 / dy), nz = Nn[3 * m + 2] / (1.0 / dz);
        // gradient of the basis in scaled coordinates: d/dx = (1/dx) d/dx'; the row is n . grad
        const double ax = nx / (dx * dx), ay = ny / (dy * dy), az = nz / (dz * dz);
        V[m][0] = 0;
        V[m][1] = ax;
        V[m][2] = ay;
        V[m][3] = az;
        V[m][4] = x * ay + y * ax;
        V[m][5] = x * az + z * ax;
        V[m][6] = y * az + z * ay;
        V[m][7] = x * y * az + x * z * ay + y * z * ax;
      } else {
        V[m][0] = 1;
        V[m][1] = x;
        V[m][2] = y;
        V[m][3] = z;
        V[m][4] = x * y;
        V[m][5] = x * z;
        V[m][6] = y * z;
        V[m][7] = x * y * z;
      }
    }
    b[0] = 1;
    b[1] = X;
    b[2] = Y;
    b[3] = Z;
    b[4] = X * Y;
    b[5] = X * Z;
    b[6] = Y * Z;
    b[7] = X * Y * Z;
    solve8T(V, b);
    for (int m = 0; m < 8; ++m) w[8 * set + m] = fl[m] ? 0.0 : b[m];
  }
}

// Snapshot of the fields a download asks for, packed in the reference's layout (k fastest, no row padding):
// field f goes to out + slot[f] * NI*NJ*NK, or nowhere for slot -1. Conserved fields are the current
// buffers; primitive / transport fields are recomputed from them as the reference holds them, except at
// filtered nodes (values before the last near-body filter) and solid inactive nodes (never updated by the
// reference; k_snapshot_inactive writes their stored values). The buffers are found through the control
// block, so the kernel can be queued behind any number of steps without the host reading it.
__global__ void k_snapshot(const Grid* __restrict__ gp, SnapSlots sl, double* __restrict__ out) {
  const Grid& G = *gp;
  const StepCtl* c = G.ctl;
  const Consts& C = G.C;
  const double* U[5];
  for (int f = 0; f < 5; ++f) U[f] = G.bufs[c->perm[f][0]][f];
  bool prim = false;
#pragma unroll
  for (int f = 5; f < NSF_SNAP_FIELDS; ++f) prim |= sl.slot[f] >= 0;
  const long long NK = G.NK, M = (long long)G.NI * G.NJ * NK;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M; q += (long long)gridDim.x * blockDim.x) {
    const long long n = (q / NK) * G.NKp + q % NK;
    double v[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      v[f] = U[f][n];
      if (sl.slot[f] >= 0) out[sl.slot[f] * M + q] = v[f];
    }
    if (!prim) continue;
    if (G.type[n] & FILTER_BIT) {
      const int f = G.fidx[n];
      v[0] = G.fpre[2 * f];
      v[4] = G.fpre[2 * f + 1];
    }
    const Prim p = prims_of(C, v[0], v[1], v[2], v[3], v[4]);
    const double pv[7] = {p.u, p.v, p.w, p.p, p.T, p.mu, p.ka};
#pragma unroll
    for (int f = 0; f < 7; ++f)
      if (sl.slot[5 + f] >= 0) out[sl.slot[5 + f] * M + q] = pv[f];
  }
}

// Solid inactive nodes of a snapshot: their stored primitive values, from the list for the time level the
// control block holds (level 0: each node's own initial values; later: the values after the first step).
__global__ void k_snapshot_inactive(const Grid* __restrict__ gp, SnapSlots sl, SnapInactive in,
                                    double* __restrict__ out) {
  const Grid& G = *gp;
  const bool ic = G.ctl->level == 0;
  const long long* nodes = ic ? in.nodesIc : in.nodes;
  const double* p7 = ic ? in.p7Ic : in.p7;
  const int count = ic ? in.countIc : in.count;
  const long long NK = G.NK, M = (long long)G.NI * G.NJ * NK;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    const long long n = nodes[q], cq = (n / G.NKp) * NK + n % G.NKp;
#pragma unroll
    for (int f = 0; f < 7; ++f)
      if (sl.slot[5 + f] >= 0) out[sl.slot[5 + f] * M + cq] = p7[7 * (long long)q + f];
  }
}

// ----------------------------------------------------------------------------------------------
// Fused boundary kernel: everything a stage does after its stage kernel, in one cooperative launch of
// bcBlocks blocks (a consecutive range of them per member, sized by its work), in the dependency levels of
// nsf_bc_plan.cpp: level 0
// holds the solid-node copies and every edge, filter and ghost-pass item whose inputs are final after the
// stage kernel; each later level reads what earlier levels wrote anywhere in the member's grid, so a barrier
// over the member's blocks separates levels (members share nothing, an ensemble's members do not wait for
// one another, and each member runs only its own levels) and those reads go through L2 (__ldcg in the item
// functions). The member's Grid and control block are copied to shared memory first (every item reads
// them). Stage 4 then flushes the dt maxima, change norms and NaN flag, and the member's last block to
// finish runs the end-of-step finalize. Every block of a member passes every barrier of that member (an
// inactive member's blocks do no work), so the launch is cooperative (all blocks resident).

// Resident blocks of the fused boundary kernel per SM (its registers are capped to fit): the kernel is
// latency-bound, each member's items spread over its blocks' threads.
constexpr int kBcBlocksPerSM = 4;

// LAST: stage 4 (s == 3), the one stage with dt terms, change norms and the NaN check; stages 1-3 run the
// other instantiation, whose item functions see s <= 2 and drop that work and its registers.
template <bool LAST>
__global__ void __launch_bounds__(256, kBcBlocksPerSM) k_bc(Grid* grids, const __grid_constant__ BcParams P, int sArg,
                                                            int fin) {
  const int s = LAST ? 3 : min(sArg, 2);
  __shared__ double red[5 * 32];
  __shared__ __align__(16) unsigned char gsm[sizeof(Grid)];
  __shared__ __align__(16) unsigned char csm[sizeof(StepCtl)];
  __shared__ int gShared;
  const int M = P.members, tid = threadIdx.x;
  if (tid == 0) {  // this block's member: blocks blockStart[g] .. blockStart[g + 1] - 1 work for member g
    int lo = 0, hi = M;
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (P.blockStart[mid] <= int(blockIdx.x)) lo = mid; else hi = mid;
    }
    gShared = lo;
  }
  __syncthreads();
  const int g = gShared;
  const int bx = int(blockIdx.x) - P.blockStart[g], nbx = P.blockStart[g + 1] - P.blockStart[g];
  Grid* gp = grids + g;
  StepCtl* c = gp->ctl;  // global: atomics, flags and finalize write here
  {
    static_assert(sizeof(Grid) % 8 == 0 && sizeof(StepCtl) % 8 == 0, "copied as 8-byte words");
    const unsigned long long* a = reinterpret_cast<const unsigned long long*>(gp);
    const unsigned long long* b = reinterpret_cast<const unsigned long long*>(c);
    for (int q = tid; q < int(sizeof(Grid) / 8); q += blockDim.x) reinterpret_cast<unsigned long long*>(gsm)[q] = a[q];
    for (int q = tid; q < int(sizeof(StepCtl) / 8); q += blockDim.x)
      reinterpret_cast<unsigned long long*>(csm)[q] = b[q];
  }
  __syncthreads();
  const Grid& G = *reinterpret_cast<const Grid*>(gsm);
  const StepCtl& cs = *reinterpret_cast<const StepCtl*>(csm);  // read-only copy for the item functions
  const bool active = cs.active != 0;
  const int gtid = bx * blockDim.x + tid, nthr = nbx * blockDim.x;
  DtAcc dta;
  double nsum[5] = {0, 0, 0, 0, 0};
  int bad = 0;
  const int ghostCount = ghost_pass_count(G, s);
  // A level's items of every kind form one index range -- solid copies (level 0), edge-block threads (64
  // per block), filter items, ghost-pass items -- and each thread takes every nthr-th index, so items of
  // different kinds run side by side rather than one list after another.
  const int levels = P.memberLevels[g];
  for (int L = 0; L < levels; ++L) {
    if (L > 0) grid_barrier(P.sync + 1 + M + g, unsigned(nbx), &c->timeout);
    if (!active) continue;
    const int mask = cs.copyMask[s];
    const int nS = (L == 0 && mask) ? G.nSolid : 0;
    const int* es = P.edgeStart + L * (M + 1) + g;
    const int* fs = P.itemStart + (L * 2) * (M + 1) + g;
    const int* hs = fs + (M + 1);
    const int e0 = es[0], nE = 64 * (es[1] - e0), f0 = fs[0], nF = fs[1] - f0, h0 = hs[0], nH = hs[1] - h0;
    const int total = nS + nE + nF + nH;
    for (int v = gtid; v < total; v += nthr) {
      if (v < nS) {
        solid_copy_item(G, &cs, s, mask, v);
      } else if (v < nS + nE) {
        const int t = v - nS, lane = t & 63;
        const EdgeBlock eb = P.edges[e0 + (t >> 6)];
        edge_node(G, &cs, eb, lane & 31, lane >> 5, s, G.eAxis[eb.e], dta, bad);
      } else if (v < nS + nE + nF) {
        filter_item(G, &cs, s, P.items[f0 + v - nS - nE], dta, nsum, bad);
      } else {
        const int item = P.items[h0 + v - nS - nE - nF];
        if (item < ghostCount) ghost_pass_item(G, &cs, s, item, dta, bad);
      }
    }
  }
  if (s == 3) {
    flush_dt(c, dta, red);
    // one norm slot per block (a member has 1 + bcBlocks slots or more when a filter exists)
    if (G.nFilter > 0) flush_norms(gp->normPart + 5 * (G.normSlotFilter + bx), nsum, red);
    if (bad) atomicOr(&c->nonFinite, 1);
  }
  if (fin) {  // the member's last block to get here runs its end-of-step finalize (no waiting)
    __shared__ int last;
    __syncthreads();
    if (tid == 0) {
      const unsigned long long old = atom_add_release(P.sync + 1 + g, 1ull);
      last = (old + 1) % (unsigned long long)nbx == 0;
      if (last) (void)ld_acquire(P.sync + 1 + g);
    }
    __syncthreads();
    if (last && active) finalize_grid(gp, red);
  }
}

static void launch_bc(Grid* dg, int members, const LaunchPlan& L, int s, bool fin, cudaStream_t st) {
  BcParams P{};
  P.edges = L.bcEdges;
  P.edgeStart = L.bcEdgeStart;
  P.items = L.bcItems;
  P.itemStart = L.bcItemStart;
  P.sync = L.bcSync;
  P.blockStart = L.bcBlockStart;
  P.memberLevels = L.bcMemberLevels;
  P.levels = L.bcLevels;
  P.members = members;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(unsigned(L.bcBlocks));
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (s == 3)
    cudaLaunchKernelEx(&cfg, k_bc<true>, dg, P, s, fin ? 1 : 0);
  else
    cudaLaunchKernelEx(&cfg, k_bc<false>, dg, P, s, fin ? 1 : 0);
}

int bc_capacity(int nSM) {
  int nb = 0;
  int nb2 = 0;  // both instantiations run the same plan: the smaller residency bounds it
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bc<true>, 256, 0) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k_bc<false>, 256, 0) != cudaSuccess) return 0;
  nb = nb2 < nb ? nb2 : nb;
  return nb * nSM;
}

// ----------------------------------------------------------------------------------------------
// Host-side launch helpers (called from nsf_capi.cpp).

void edge_blocks(const Grid& G, const uint8_t* type, int g, int axis, std::vector<EdgeBlock>& out) {
  const int ax1 = axis == 0 ? 1 : 0, ax2 = axis == 2 ? 1 : 2;
  // periodic faces whose copies the stage kernel writes: those nodes leave the blocks (z: (a, bb) = (i, j),
  // y: (a, bb) = (i, k))
  const bool fused = type && ((axis == 2 && G.zFused) || (axis == 1 && G.yFused));
  for (int e = 0; e < G.nEdge; ++e) {
    if (G.eAxis[e] != axis) continue;
    const int* b = G.eBox[e];
    const int ks = G.eSide[e] == 0 ? G.NK - 2 : 1;  // the periodic source plane
    const int js = G.eSide[e] == 0 ? G.NJ - 2 : 1;
    for (int a0 = b[2 * ax1]; a0 <= b[2 * ax1 + 1]; a0 += kEdgeRows)
      for (int b0 = b[2 * ax2]; b0 <= b[2 * ax2 + 1]; b0 += 32) {
        unsigned long long mask = ~0ull;
        if (fused && G.eBc[e] == NSF_BC_PERIODIC) {
          mask = 0;
          for (int ty = 0; ty < kEdgeRows; ++ty)
            for (int tx = 0; tx < 32; ++tx) {
              const int a = a0 + ty, bb = b0 + tx;
              if (a > b[2 * ax1 + 1] || bb > b[2 * ax2 + 1]) continue;
              const bool copiedByStage =
                  axis == 2 ? (type[(size_t(a) * G.NJ + bb) * G.NK + ks] & (ZCOPY_UP_BIT | ZCOPY_DOWN_BIT)) != 0
                            : (type[(size_t(a) * G.NJ + js) * G.NK + bb] & YCOPY_BIT) != 0;
              if (!copiedByStage) mask |= 1ull << (ty * 32 + tx);
            }
          if (!mask) continue;
        }
        out.push_back(EdgeBlock{g, e, a0, b0, mask, 0ull});
      }
  }
}

// One RK4 step for `members` grids (dg: device array of them). hg: the grid on the host for a single-grid
// solver (its stage kernel takes the grid by value), or NULL for an ensemble (the ensemble stage kernel
// reads every member from dg). The small kernels carry the member in a grid dimension, their block
// counts in L being the maxima over the members; the edge kernels run the listed blocks of every member.
// lastStage: NULL, or the plan of a partial stage 4 (single grid): stage 4 then runs the stage kernel over
// that plan's items only and the step ends there (no stage-4 boundary conditions, no finalize).
// ev: NULL, or 8 events recorded around the four stage kernels; evExternal: record them as event nodes of
// a graph being captured (cudaEventRecordExternal) rather than as plain stream events.
static int enqueue_impl(Grid* dg, const Grid* hg, int members, const LaunchPlan& L, cudaStream_t st, cudaEvent_t* ev,
                        StepHook* hook = nullptr, const LaunchPlan* lastStage = nullptr, bool evExternal = false) {
  auto record = [&](cudaEvent_t e) {
    if (evExternal)
      cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else
      cudaEventRecord(e, st);
  };
  int launches = 0;
  const unsigned M = unsigned(members);
  // the fused boundary kernel, unless a hook must run between the solid-node copy and the edge conditions
  // (a partial last stage ends before its boundary work, fused or not)
  const bool fused = L.bcBlocks > 0 && (!hook || !hook->wants_before_edges());
  k_prologue<<<M, 32, 0, st>>>(dg);
  ++launches;
  if (hook) hook->after_prologue();
  k_density_filter<<<dim3(L.gfBlocks, M), 256, 0, st>>>(dg);
  ++launches;
  for (int s = 0; s < 4; ++s) {
    if (ev) record(ev[2 * s]);
    if (hook) hook->before_stage(s);
    if (s == 3 && lastStage && hg) {
      if (lastStage->nItems > 0) {
        launch_stage(*hg, *lastStage, s, st);
        ++launches;
      }
      if (hook) hook->before_edges(s);
      return launches;
    }
    if (hg)
      launch_stage(*hg, L, s, st);
    else
      launch_stage_ensemble(dg, L, s, st);
    if (ev) record(ev[2 * s + 1]);
    ++launches;
    if (fused) {
      if (L.bcLevels > 0 || s == 3) {
        launch_bc(dg, members, L, s, s == 3, st);
        ++launches;
      }
      continue;
    }
    if (L.hasSolid) {
      k_solid_copy<<<dim3(L.solidBlocks, M), 256, 0, st>>>(dg, s);
      ++launches;
    }
    if (hook) hook->before_edges(s);
    for (int a = 0; a < 3; ++a)
      if (L.nEdgeBlocks[a] > 0) {
        k_edge_bc<<<L.nEdgeBlocks[a], dim3(32, kEdgeRows), 0, st>>>(dg, L.edgeBlocks[a], s, a);
        ++launches;
      }
    if (L.hasFilter) {
      k_body_filter<<<dim3(L.filterBlocks, M), 256, 0, st>>>(dg, s);
      ++launches;
    }
    if (L.hasGhostWork) {
      k_ghost<<<dim3(L.ghostBlocks, M), 256, 0, st>>>(dg, s);
      ++launches;
    }
  }
  if (!fused) {
    k_finalize<<<M, 256, 0, st>>>(dg);
    ++launches;
  }
  return launches;
}

int enqueue_step_begin(Grid* dg, const LaunchPlan& L, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_prologue<<<1, 32, 0, st>>>(dg);
  k_density_filter<<<dim3(L.gfBlocks, 1), 256, 0, st>>>(dg);
  return 2;
}

int launch_bc_part(Grid* dg, const LaunchPlan& L, int s, bool fin, void* stream) {
  if (L.bcBlocks <= 0 || (L.bcLevels == 0 && !fin)) return 0;
  launch_bc(dg, 1, L, s, fin, static_cast<cudaStream_t>(stream));
  return 1;
}

int enqueue_step(Grid* dg, const Grid& hg, const LaunchPlan& L, void* stream) {
  return enqueue_impl(dg, &hg, 1, L, static_cast<cudaStream_t>(stream), nullptr);
}

int enqueue_step_hooked(Grid* dg, const Grid& hg, const LaunchPlan& L, void* stream, StepHook* hook,
                        const LaunchPlan* lastStage) {
  return enqueue_impl(dg, &hg, 1, L, static_cast<cudaStream_t>(stream), nullptr, hook, lastStage);
}

int enqueue_ensemble_step(Grid* dGrids, int members, const LaunchPlan& L, void* stream, void* events) {
  return enqueue_impl(dGrids, nullptr, members, L, static_cast<cudaStream_t>(stream), static_cast<cudaEvent_t*>(events));
}

int enqueue_step_profiled(Grid* dg, const Grid& hg, const LaunchPlan& L, void* stream, void* events, bool inGraph) {
  return enqueue_impl(dg, &hg, 1, L, static_cast<cudaStream_t>(stream), static_cast<cudaEvent_t*>(events), nullptr,
                      nullptr, inGraph);
}

void launch_ghost_weights(int nGhost, const double* pts, const double* nrm, const uint8_t* flags, const double* ipl,
                          double dx, double dy, double dz, double* w, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (nGhost > 0) k_ghost_weights<<<(nGhost + 127) / 128, 128, 0, st>>>(nGhost, pts, nrm, flags, ipl, dx, dy, dz, w);
}

void launch_snapshot(const Grid* dg, const SnapSlots& sl, const SnapInactive& in, double* out, int nSM, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_snapshot<<<nSM * 8, 256, 0, st>>>(dg, sl, out);
  bool prim = false;
  for (int f = 5; f < NSF_SNAP_FIELDS; ++f) prim |= sl.slot[f] >= 0;
  const int most = in.count > in.countIc ? in.count : in.countIc;
  if (prim && most > 0) k_snapshot_inactive<<<(most + 255) / 256, 256, 0, st>>>(dg, sl, in, out);
}

// The Newton-Raphson reciprocal and square root next to the IEEE ones, for a check of their error.
__global__ void k_math_selftest(long long n, const double* __restrict__ x, double* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const double a = x[q];
    out[4 * q + 0] = recip_nr(a);
    out[4 * q + 1] = 1.0 / a;
    out[4 * q + 2] = sqrt_nr(a);
    out[4 * q + 3] = sqrt(a);
  }
}

int math_selftest(long long n, const double* hostIn, double* hostOut) {
  double *dx = nullptr, *dout = nullptr;
  cudaError_t e = cudaMalloc(&dx, (n > 0 ? n : 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dout, 4 * (n > 0 ? n : 1) * sizeof(double));
  if (e == cudaSuccess && n > 0) e = cudaMemcpy(dx, hostIn, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n > 0) {
    k_math_selftest<<<int((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), 256>>>(n, dx, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && n > 0) e = cudaMemcpy(hostOut, dout, 4 * n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  return int(e);
}

}  // namespace nsf
