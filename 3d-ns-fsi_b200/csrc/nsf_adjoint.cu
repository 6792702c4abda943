// Discrete adjoint of the RK4 time step: one kernel per forward kernel, in gather form.
//
// The forward step (nsf_kernels.cu, nsf_stage_ws.cu) is a sequence of kernels that read and write the
// physical field buffers (three per conserved field, the RK4 accumulator, the near-body filter's pre- and
// post-filter values). The adjoint keeps one adjoint array per physical buffer and runs the transpose of
// every kernel in reverse order: a kernel that overwrites values consumes (zeroes) their adjoints and adds
// its Jacobian-transposed contributions to the adjoints of the values it read. Because the adjoint state
// mirrors the physical buffers, the reference's stale-buffer semantics (values that persist across the
// buffer swaps, primitives of filter nodes taken before the near-body filter) are differentiated exactly
// as the forward path reproduces them. Every kernel writes only adjoints of its own nodes (gathers over
// precomputed reverse maps where the forward kernel scatters): no atomics, deterministic results.
//
// The dt sequence is frozen (the gradient does not differentiate the CFL limit), as the gradient checks
// against finite differences and the dual-number oracle do.
#include <cuda_runtime.h>

#include <algorithm>

#include "nsf_adjoint.h"
#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_physics.cuh"
#include "nsf_rhs_adjoint.cuh"

namespace nsf {
namespace {

// Pressure of conserved values (prims_of's p).
__device__ __forceinline__ double pressure(const Consts& C, const double u[5], double g[5]) {
  const double r1 = 1.0 / (u[0] + 1.0);
  const double vx = u[1] * r1, vy = u[2] * r1, vz = u[3] * r1;
  const double K = 0.5 * (vx * vx + vy * vy + vz * vz);
  if (g) {  // gradient of p with respect to the five conserved values
    g[0] = C.gm1 * K;
    g[1] = -C.gm1 * vx;
    g[2] = -C.gm1 * vy;
    g[3] = -C.gm1 * vz;
    g[4] = C.gm1;
  }
  return C.gm1 * (u[4] - (u[0] + 1.0) * K);
}

// --------------------------------------------------------------------------------------- objective
// F_x = -dA * sum_g p(U_g) n_x(g) over the ghost nodes of the current state (the buffers the step just
// finished in, StepCtl::perm[f][0]); one block, fixed summation order.
__global__ void k_objective(const Grid* __restrict__ gp, const double* __restrict__ nx, double dA, double weight,
                            double* acc) {
  __shared__ double red[32];
  const Grid& G = *gp;
  const StepCtl* c = G.ctl;
  double s = 0;
  for (int q = threadIdx.x; q < G.nGhost; q += blockDim.x) {
    const long long n = G.gnode[q];
    double u[5];
    for (int f = 0; f < 5; ++f) u[f] = G.bufs[c->perm[f][0]][f][n];
    s += -dA * nx[q] * pressure(G.C, u, nullptr);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
    *acc += weight * t;
  }
}

// The adjoint of the objective's pressure at ghost q (added to the adjoint of the step's result there).
__device__ __forceinline__ void adj_objective_term(const Grid& G, const double* const val[5], const double* nx,
                                                   double dA, double weight, int q, double lam[5]) {
  const long long n = G.gnode[q];
  double u[5], g[5];
  for (int f = 0; f < 5; ++f) u[f] = val[f][n];
  pressure(G.C, u, g);
  for (int f = 0; f < 5; ++f) lam[f] += weight * (-dA * nx[q]) * g[f];
}

// ------------------------------------------------------------------------------------------- ghosts
// k_ghost writes the ghost values (weights x cell values, momenta negated) and writes the filtered
// values back to the filter nodes. Phase 1: consume the adjoints of everything k_ghost wrote (with, on a
// step whose result enters J, the objective's adjoint at the ghost nodes first).
__device__ __forceinline__ void adj_ghost_consume_item(const Grid& G, const AdjPtrs& A, double* ipbar,
                                                       const AdjBcParams& P, int q) {
  if (q < G.nGhost) {
    const long long n = G.gnode[q];
    const double sgn[5] = {1, -1, -1, -1, 1};
    double lam[5];
    for (int f = 0; f < 5; ++f) lam[f] = A.lamO[f][n];
    if (P.objective) adj_objective_term(G, P.objVal, P.nx, P.dA, P.weight, q, lam);
    for (int f = 0; f < 5; ++f) {
      ipbar[f * (long long)G.nGhost + q] = sgn[f] * lam[f];
      A.lamO[f][n] = 0.0;
    }
  } else {
    const int f = q - G.nGhost;
    const long long n = G.fnode[f];
    A.lamFnew[2 * f] += A.lamO[0][n];
    A.lamFnew[2 * f + 1] += A.lamO[4][n];
    A.lamO[0][n] = 0.0;
    A.lamO[4][n] = 0.0;
  }
}

// Phase 2: every image-point cell node gathers weight x image-point adjoint from the ghosts that read it
// (reverse map in CSR form: entries 8 * ghost + corner).
__device__ __forceinline__ void adj_ghost_gather_item(const Grid& G, const AdjPtrs& A, const double* ipbar,
                                                      const AdjBcParams& P, int c) {
  const long long m = P.cnode[c];
  const int e0 = P.coff[c], e1 = P.coff[c + 1];
  // the node's own values first (they depend on m only), so their loads overlap the entries' loads
  const bool filt = (G.type[m] & FILTER_BIT) != 0;
  const int fi = filt ? G.fidx[m] : 0;
  double* const t0 = filt ? A.lamFnew + 2 * fi : A.lamO[0] + m;  // where the density's adjoint goes
  double* const t4 = filt ? A.lamFnew + 2 * fi + 1 : A.lamO[4] + m;
  double o[5];
  o[0] = *t0;
  o[4] = *t4;
  for (int f = 1; f < 4; ++f) o[f] = A.lamO[f][m];
  double a[5] = {0, 0, 0, 0, 0};
  for (int e = e0; e < e1; ++e) {
    const int q = P.cent[e] >> 3, slot = P.cent[e] & 7;
    const double wn = G.gw[16 * (long long)q + slot], wd = G.gw[16 * (long long)q + 8 + slot];
    a[0] += wn * ipbar[q];
    a[4] += wn * ipbar[4 * (long long)G.nGhost + q];
    for (int f = 1; f < 4; ++f) a[f] += wd * ipbar[f * (long long)G.nGhost + q];
  }
  *t0 = o[0] + a[0];  // filter node: k_ghost read its filtered values
  *t4 = o[4] + a[4];
  for (int f = 1; f < 4; ++f) A.lamO[f][m] = o[f] + a[f];
}

// ------------------------------------------------------------------------------- near-body filter
// k_body_filter: fpre = O at the filter node, fnew = (6 O[n] + sum of the 6 neighbours)/12 (rho, rho_E).
// Every node of the filter stencils gathers from the filter nodes whose stencil holds it. slots[7 q ..]:
// the node's own filter slot, then those of its neighbours at +-i, +-j, +-k (-1: not a filter node),
// listed at setup so that an item's loads take two round trips (indices, then values).
__device__ __forceinline__ void adj_filter_item(const AdjPtrs& A, const long long* nodes, const int* slots, int q) {
  const long long m = nodes[q];
  int sl[7];
  for (int d = 0; d < 7; ++d) sl[d] = slots[7 * (long long)q + d];
  double fn[7][2], fp[2] = {0, 0};
  for (int d = 0; d < 7; ++d)
    for (int c = 0; c < 2; ++c) fn[d][c] = sl[d] >= 0 ? A.lamFnew[2 * sl[d] + c] : 0.0;
  if (sl[0] >= 0)
    for (int c = 0; c < 2; ++c) fp[c] = A.lamFpre[2 * sl[0] + c];
  const double o0 = A.lamO[0][m], o4 = A.lamO[4][m];
  double ar = 0, ae = 0;
  if (sl[0] >= 0) {
    ar += 0.5 * fn[0][0] + fp[0];
    ae += 0.5 * fn[0][1] + fp[1];
  }
  for (int d = 1; d < 7; ++d) {
    if (sl[d] < 0) continue;
    ar += fn[d][0] / 12;
    ae += fn[d][1] / 12;
  }
  A.lamO[0][m] = o0 + ar;
  A.lamO[4][m] = o4 + ae;
}

// -------------------------------------------------------------------------------- edge boundaries
// One node of an edge block (k_edge_bc's geometry: 32 x kEdgeRows nodes, (tx, ty) within it). Phase 1
// (periodic, outlet, inlet part 1): consume the adjoint of the edge node; periodic and outlet add to their
// (one-to-one) source nodes, the inlet keeps the adjoint of its filtered extrapolated density per node for
// phase 2.
__device__ __forceinline__ void adj_edge_item(const Grid& G, const EdgeBlock& eb, int tx, int ty, const AdjPtrs& A,
                                              const double* const val[5], int axis, double stageT, double* fbar,
                                              double* lamInflow) {
  const Consts& C = G.C;
  const int e = eb.e;
  const int* b = G.eBox[e];
  const int ax1 = axis == 0 ? 1 : 0, ax2 = axis == 2 ? 1 : 2;
  const int a = eb.a0 + ty;
  const int bb = eb.b0 + tx;
  if (a > b[2 * ax1 + 1] || bb > b[2 * ax2 + 1]) return;
  int ijk[3];
  ijk[axis] = b[2 * axis];
  ijk[ax1] = a;
  ijk[ax2] = bb;
  const long long st = axis == 0 ? G.sI : axis == 1 ? G.sJ : 1;
  const long long n = ijk[0] * G.sI + ijk[1] * G.sJ + ijk[2];
  const int side = G.eSide[e], bc = G.eBc[e];
  // Every load of an item is issued before its first store (one memory round trip, not two): the nodes
  // an item reads and writes are its own -- no other item of the phase touches them.
  double lam[5];
  if (bc == NSF_BC_PERIODIC) {
    int src[3] = {ijk[0], ijk[1], ijk[2]};
    const int nAx = axis == 0 ? G.NI : axis == 1 ? G.NJ : G.NK;
    src[axis] = side == 0 ? nAx - 2 : 1;
    const long long m = src[0] * G.sI + src[1] * G.sJ + src[2];
    double acc[5];
    for (int f = 0; f < 5; ++f) {
      lam[f] = A.lamO[f][n];
      acc[f] = A.lamO[f][m];
    }
    for (int f = 0; f < 5; ++f) {
      A.lamO[f][n] = 0.0;
      A.lamO[f][m] = acc[f] + lam[f];
    }
    return;
  }
  if (bc == NSF_BC_OUTLET) {
    const long long a1 = side == 0 ? n + st : n - st, a2 = side == 0 ? n + 2 * st : n - 2 * st;
    double v1[4], v2[4], l1[4], l2[4];
    for (int f = 0; f < 5; ++f) lam[f] = A.lamO[f][n];
    for (int f = 0; f < 4; ++f) {
      v1[f] = val[f][a1];
      v2[f] = val[f][a2];
      l1[f] = A.lamO[f][a1];
      l2[f] = A.lamO[f][a2];
    }
    for (int f = 0; f < 5; ++f) A.lamO[f][n] = 0.0;
    const double rho = 2 * v1[0] - v2[0];
    double u[3];
    for (int f = 1; f < 4; ++f) u[f - 1] = (2 * v1[f] - v2[f]) / (1 + rho);
    // rho_E = (1 + rho)/2 |u|^2 with u = m/(1 + rho): d/drho = -|u|^2/2, d/dm = u
    const double rbar = lam[0] - 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * lam[4];
    A.lamO[0][a1] = l1[0] + 2 * rbar;
    A.lamO[0][a2] = l2[0] - rbar;
    for (int f = 1; f < 4; ++f) {
      const double mbar = lam[f] + u[f - 1] * lam[4];
      A.lamO[f][a1] = l1[f] + 2 * mbar;
      A.lamO[f][a2] = l2[f] - mbar;
    }
    return;
  }
  if (bc == NSF_BC_INLET) {
    // rho = f (filtered extrapolation); u_axis = ramp * M0 * profile; T = 0; p = rho / gamma
    for (int f = 0; f < 5; ++f) lam[f] = A.lamO[f][n];
    const long long s1 = ax1 == 0 ? G.sI : G.sJ, s2 = ax2 == 1 ? G.sJ : 1;
    auto ext = [&](long long m) {
      return 2 * val[0][side == 0 ? m + st : m - st] - val[0][side == 0 ? m + 2 * st : m - 2 * st];
    };
    double f = 0;
    unsigned nn = 0;
    if (a < b[2 * ax1 + 1]) { f += ext(n + s1); ++nn; }
    if (a > b[2 * ax1]) { f += ext(n - s1); ++nn; }
    if (bb < b[2 * ax2 + 1]) { f += ext(n + s2); ++nn; }
    if (bb > b[2 * ax2]) { f += ext(n - s2); ++nn; }
    f += nn * ext(n);
    f /= 2 * nn;
    const double ramp = fmin(1., stageT / 10.) * C.m0 * (side == 1 ? -1.0 : 1.0);
    const double prof = (G.inflow && axis == 0) ? G.inflow[a * G.NKp + bb] : 1.0;
    const double inflowBar = axis == 0 ? lamInflow[a * G.NKp + bb] : 0.0;
    for (int f = 0; f < 5; ++f) A.lamO[f][n] = 0.0;
    const double vel = ramp * prof;
    const double fb = lam[0] + vel * lam[axis + 1] + (1 / (C.gamma * C.gm1) + 0.5 * vel * vel) * lam[4];
    const double velbar = (1 + f) * (lam[axis + 1] + vel * lam[4]);
    if (axis == 0) lamInflow[a * G.NKp + bb] = inflowBar + velbar * ramp;
    fbar[(long long)a * G.NKp + bb + (side ? (long long)G.NJ * G.NKp : 0)] = fb;
    return;
  }
  for (int f = 0; f < 5; ++f) A.lamO[f][n] = 0.0;  // any other condition: the value is consumed
}

// Inlet phase 2 (x faces only): every node of the two planes behind the inlet gathers from the inlet
// nodes whose filtered extrapolation used it.
__device__ __forceinline__ void adj_inlet_gather_item(const Grid& G, const EdgeBlock& eb, int tx, int ty,
                                                      const AdjPtrs& A, const double* fbar) {
  const int e = eb.e;  // the x faces' blocks; only inlet faces gather
  if (G.eBc[e] != NSF_BC_INLET) return;
  const int* b = G.eBox[e];
  const int a = eb.a0 + ty;   // j
  const int bb = eb.b0 + tx;  // k
  if (a > b[3] || bb > b[5]) return;
  const int side = G.eSide[e];
  const long long base = side ? (long long)G.NJ * G.NKp : 0;
  auto nnOf = [&](int ca, int cb) {
    return unsigned(ca < b[3]) + unsigned(ca > b[2]) + unsigned(cb < b[5]) + unsigned(cb > b[4]);
  };
  double g = 0;
  const int da[5] = {0, 1, -1, 0, 0}, db[5] = {0, 0, 0, 1, -1};
  for (int c = 0; c < 5; ++c) {
    const int ca = a + da[c], cb = bb + db[c];
    if (ca < b[2] || ca > b[3] || cb < b[4] || cb > b[5]) continue;
    const unsigned nn = nnOf(ca, cb);
    const double w = c == 0 ? double(nn) / (2 * nn) : 1.0 / (2 * nn);
    g += w * fbar[base + (long long)ca * G.NKp + cb];
  }
  const long long n = (long long)b[0] * G.sI + (long long)a * G.sJ + bb;
  const long long st = G.sI;
  A.lamO[0][side == 0 ? n + st : n - st] += 2 * g;
  A.lamO[0][side == 0 ? n + 2 * st : n - 2 * st] -= g;
}

// ------------------------------------------------------------------------------------------ stage
// Before the stage kernel's adjoint: the RK4 combine's adjoint and the stage's RHS input quantities.
// Combine (interior fluid nodes; lam is zero elsewhere): with o = the adjoint of the stage output,
//   stage 1:    k = dt/2 o + acc, acc = 0      stages 2, 3: k = inc o + 2 acc      stage 4: k = dt/6 o, acc += k
// (inc = dt/2, dt), lam = k is the adjoint of the stage's RHS; U0 receives o, o is consumed.
// Values: momenta and rho_E from I, density from R, filter nodes' density and rho_E from fpre (for the
// primitives), then the primitives and transport properties, as the stage kernel stages them.
// With periodic z faces (Grid::zFused) the stage kernel also wrote the z copies of the nodes at k = 1 and
// k = NK-2 it computed, with periodic y faces (Grid::yFused) the y copies of those at j = 1 and j = NJ-2:
// their adjoints are gathered here, before the combine's (edge blocks left with only such nodes are not
// listed, so the edge phase has not consumed them).
// Solid nodes (ghost and inactive): the adjoint of k_solid_copy, which copied the stage input into the
// output of the fields in solidMask (bit 0: the density from R) before the edge conditions.
__device__ __forceinline__ void adj_prepare_item(const Grid& G, const AdjPtrs& A, int s, double dtUsed, int solidMask,
                                                 double* __restrict__ lam, double* __restrict__ V, long long n) {
  const double inc = s == 2 ? dtUsed : dtUsed / 2, dtF = dtUsed / 6;
  // every load first (about twenty independent loads in flight per thread), then the arithmetic
  const uint8_t ty = G.type[n];
  const bool interior = (ty & TYPE_MASK) == FLUID_INTERIOR;
  const double m1 = A.val[1][n], m2 = A.val[2][n], m3 = A.val[3][n], e4 = A.val[4][n];
  double rho = A.valR[n], rE = e4;
  double o[5], acc[5], u0[5], oz[5] = {0, 0, 0, 0, 0}, oy[5] = {0, 0, 0, 0, 0};
  // the z and y copies the stage kernel wrote with this node
  const bool zCopy = (ty & (ZCOPY_UP_BIT | ZCOPY_DOWN_BIT)) != 0;
  const long long nz = (ty & ZCOPY_UP_BIT) ? n + (G.NK - 2) : n - (G.NK - 2);
  const bool yCopy = (ty & YCOPY_BIT) != 0;
  const long long ny = (n % G.sI) / G.sJ == 1 ? n + (G.NJ - 2) * G.sJ : n - (G.NJ - 2) * G.sJ;
  if (interior)
    for (int f = 0; f < 5; ++f) {
      o[f] = A.lamO[f][n];
      acc[f] = A.lamAcc[f][n];
      u0[f] = A.lamU0[f][n];
      if (zCopy) oz[f] = A.lamO[f][nz];
      if (yCopy) oy[f] = A.lamO[f][ny];
    }
  if (ty & FILTER_BIT) {
    const int f = G.fidx[n];
    rho = A.valFpre[2 * f];
    rE = A.valFpre[2 * f + 1];
    // the near-body filter's adjoints were consumed by the filter phase: clear them for the transposed
    // RHS (fpre) and the previous stage's ghosts (fnew)
    A.lamFpre[2 * f] = 0.0;
    A.lamFpre[2 * f + 1] = 0.0;
    A.lamFnew[2 * f] = 0.0;
    A.lamFnew[2 * f + 1] = 0.0;
  }
  const Prim pr = prims_of_nr(G.C, rho, m1, m2, m3, rE);  // as the stage kernel's staging warps
  const double q[11] = {m1, m2, m3, e4, pr.u, pr.v, pr.w, pr.p, pr.T, pr.mu, pr.ka};
  for (int v = 4; v < 11; ++v) V[v * G.N + n] = q[v];  // 0..3 are the stage input's own values (A.val)
  if (!interior) {
    for (int f = 0; f < 5; ++f) lam[f * G.N + n] = 0.0;
    const uint8_t t = ty & TYPE_MASK;
    if (solidMask && (t == SOLID_GHOST || t == SOLID_INACTIVE)) {
      if (solidMask & 1) {
        A.lamR[n] += A.lamO[0][n];
        A.lamO[0][n] = 0.0;
      }
      for (int f = 1; f < 5; ++f)
        if (solidMask & (1 << f)) {
          A.lamI[f][n] += A.lamO[f][n];
          A.lamO[f][n] = 0.0;
        }
    }
    return;
  }
  if (zCopy)
    for (int f = 0; f < 5; ++f) {
      o[f] += oz[f];
      A.lamO[f][nz] = 0.0;
    }
  if (yCopy)
    for (int f = 0; f < 5; ++f) {
      o[f] += oy[f];
      A.lamO[f][ny] = 0.0;
    }
  for (int f = 0; f < 5; ++f) {
    double k;
    if (s == 0) {
      k = inc * o[f] + acc[f];
      A.lamAcc[f][n] = 0.0;
    } else if (s < 3) {
      k = inc * o[f] + 2 * acc[f];
    } else {
      k = dtF * o[f];
      A.lamAcc[f][n] = acc[f] + dtF * o[f];
    }
    lam[f * G.N + n] = k;
    A.lamU0[f][n] = u0[f] + o[f];
    A.lamO[f][n] = 0.0;
  }
}

// ----------------------------------------------------------------------- two launches per stage
// Everything of a stage's adjoint before the transposed RHS, in the forward kernels' reverse order. The
// boundary work runs as phases of one cooperative launch: ghost consume (and the objective) | ghost gather
// | near-body filter | edges z | y | x | inlet gather. Each phase reads what the one before it wrote
// anywhere in the grid, so a grid barrier (bounded: a wait that gives up marks the run invalid through
// StepCtl::timeout) separates non-empty phases. Every phase is a thread-stride loop over its items; an
// edge block counts 64 items (32 x kEdgeRows nodes). The RK4 combine and RHS inputs, one item per node,
// follow as a kernel of their own (measured faster than a last phase of the cooperative launch, whose
// grid is sized for the few boundary items).
constexpr int kAdjBcThreads = 256;  // the grid is sized by the largest phase: a few dozen blocks
__global__ void __launch_bounds__(kAdjBcThreads)
    k_adj_bc(const __grid_constant__ Grid G, const __grid_constant__ AdjBcParams P, int s) {
  const AdjPtrs& A = P.A;
  // One chain of phases over all blocks, or (P.bodyBlocks > 0: the host found the bodies' nodes and the
  // face planes disjoint) two independent chains -- the body phases on the first bodyBlocks blocks, the
  // edge phases on the rest -- each with its own barrier counter.
  const bool split = P.bodyBlocks > 0;
  const bool bodyChain = !split || int(blockIdx.x) < P.bodyBlocks;
  const bool edgeChain = !split || int(blockIdx.x) >= P.bodyBlocks;
  const int b0 = (split && edgeChain) ? P.bodyBlocks : 0;
  const int nb = split ? (bodyChain ? P.bodyBlocks : int(gridDim.x) - P.bodyBlocks) : int(gridDim.x);
  const int gtid = (int(blockIdx.x) - b0) * blockDim.x + threadIdx.x, nthr = nb * blockDim.x;
  unsigned long long* const sync = P.sync + ((split && edgeChain) ? 1 : 0);
  bool started = false;
  auto barrier = [&](long long count) {
    if (count == 0) return false;
    if (started) grid_barrier(sync, unsigned(nb), P.timeout);
    started = true;
    return true;
  };
  if (bodyChain) {
    if (barrier(G.nGhost + G.nFilter))
      for (int v = gtid; v < G.nGhost + G.nFilter; v += nthr) adj_ghost_consume_item(G, A, P.ipbar, P, v);
    if (barrier(P.ncell))
      for (int v = gtid; v < P.ncell; v += nthr) adj_ghost_gather_item(G, A, P.ipbar, P, v);
    if (barrier(P.nfs))
      for (int v = gtid; v < P.nfs; v += nthr) adj_filter_item(A, P.fsNodes, P.fsSlots, v);
  }
  if (!edgeChain) return;
  const double stageT = P.roles->stageT[s];
  for (int axis = 2; axis >= 0; --axis)  // z, y, then x
    if (barrier(P.nEdge[axis]))
      for (int v = gtid; v < 64 * P.nEdge[axis]; v += nthr) {
        const int lane = v & 63;
        adj_edge_item(G, P.edges[axis][v >> 6], lane & 31, lane >> 5, A, P.edgeVal, axis, stageT, P.fbar,
                      P.lamInflow);
      }
  if (barrier(P.inletGather ? P.nEdge[0] : 0))
    for (int v = gtid; v < 64 * P.nEdge[0]; v += nthr) {
      const int lane = v & 63;
      adj_inlet_gather_item(G, P.edges[0][v >> 6], lane & 31, lane >> 5, A, P.fbar);
    }
}

// The RK4 combine's adjoint and the RHS inputs: one thread per node.
__global__ void __launch_bounds__(256) k_adj_combine(const __grid_constant__ Grid G, const __grid_constant__ AdjBcParams P,
                                                     int s) {
  const double dtUsed = P.roles->dtUsed;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < G.N; n += (long long)gridDim.x * blockDim.x)
    adj_prepare_item(G, P.A, s, dtUsed, P.solidMask, P.lam, P.V, n);
}

// Several device-to-device copies in one launch (blockIdx.y: the copy).
struct CopySet {
  const double* src[kMaxCopies];
  double* dst[kMaxCopies];
  long long words[kMaxCopies];
};

__global__ void k_copy_set(CopySet S) {
  const int c = blockIdx.y;
  const double* __restrict__ src = S.src[c];
  double* __restrict__ dst = S.dst[c];
  const long long n = S.words[c];
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x)
    dst[m] = src[m];
}

// Tape copies (blockIdx.y: the copy), sources and set from the control block of the running step.
__global__ void k_tape_copy(const StepCtl* __restrict__ ctl, const __grid_constant__ TapeCopy T) {
  const int c = blockIdx.y;
  const StepCtl& C = *ctl;
  long long set = (long long)C.level + T.levelOffset;
  if (set < 0) return;
  set %= T.nSets;
  const int q = T.q[c], f = T.f[c];
  const double* src;
  switch (T.kind[c]) {
    case TAPE_I: src = C.I[q][f]; break;
    case TAPE_R_SEP:
      if (C.R[q] == C.I[q][0]) return;
      src = C.R[q];
      break;
    case TAPE_O: src = C.O[q][f]; break;
    default: src = T.src[c];
  }
  src += T.srcOff[c];
  double* __restrict__ dst = T.tape + set * T.setWords + T.dstOff[c];
  const long long n = T.words[c];
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x)
    dst[m] = src[m];
}

// Transposed RHS (generated gather) and the chain rule through the primitive / transport values.
// A block takes an 8 (j) x 32 (k) tile of nodes through a chunk of i-planes. The generated gather reads
// the RHS adjoints at the 19 RHS nodes around a node and u, v, w, T, mu, kappa at its 7-point stencil:
// those 11 fields are staged per plane with a one-node halo in a 3-plane ring in shared memory (so every
// read is a shared-memory load at a fixed offset), the other inputs (momenta, rho_E, p) are read at the
// node itself from global memory. Planes and halo nodes outside the grid are staged as zeros.
constexpr int RT_J = 8, RT_K = 32, RT_HK = RT_K + 2, RT_PLANE = (RT_J + 2) * RT_HK;
constexpr int RT_FIELDS = 11;                     // RHS adjoints 0..4, then u, v, w, T, mu, kappa
constexpr int RT_SLOT = RT_FIELDS * RT_PLANE;     // doubles per staged plane
constexpr int RT_SMEM = 3 * RT_SLOT * 8;          // bytes: 89,760
constexpr int kAdjRhsBlocks = 2;                  // resident blocks per SM (shared memory and registers)
__host__ __device__ constexpr int rt_field(int q) {  // input quantity q -> staged field, or -1
  return q == 4 ? 5 : q == 5 ? 6 : q == 6 ? 7 : q == 8 ? 8 : q == 9 ? 9 : q == 10 ? 10 : -1;
}

__global__ void __launch_bounds__(32 * RT_J, kAdjRhsBlocks)
    k_adj_rhs(const Grid* __restrict__ gp, const __grid_constant__ Consts C, AdjPtrs A, const double* __restrict__ lam,
              const double* __restrict__ V, int chunk) {
  extern __shared__ double sm[];
  const Grid& G = *gp;
  const long long N = G.N, sI = G.sI, sJ = G.sJ;
  const int NI = G.NI, NJ = G.NJ, NK = G.NK;
  const int tilesK = (NK + RT_K - 1) / RT_K;
  const int j0 = (blockIdx.x / tilesK) * RT_J, k0 = (blockIdx.x % tilesK) * RT_K;
  const int i0 = blockIdx.y * chunk, i1 = min(NI - 1, i0 + chunk - 1);
  if (i0 > i1) return;  // uniform over the block
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int j = j0 + ty, k = k0 + tx;
  auto stage = [&](int p, int slot) {
    double* s = sm + slot * RT_SLOT;
    for (int idx = tid; idx < RT_PLANE; idx += 32 * RT_J) {
      const int hj = idx / RT_HK, jj = j0 - 1 + hj, kk = k0 - 1 + (idx - hj * RT_HK);
      const bool in = p >= 0 && p < NI && jj >= 0 && jj < NJ && kk >= 0 && kk < NK;
      const long long n = in ? p * sI + jj * sJ + kk : 0;
      double v[RT_FIELDS];
#pragma unroll
      for (int e = 0; e < 5; ++e) v[e] = in ? lam[e * N + n] : 0.0;
      v[5] = in ? V[4 * N + n] : 0.0;
      v[6] = in ? V[5 * N + n] : 0.0;
      v[7] = in ? V[6 * N + n] : 0.0;
      v[8] = in ? V[8 * N + n] : 0.0;
      v[9] = in ? V[9 * N + n] : 0.0;
      v[10] = in ? V[10 * N + n] : 0.0;
#pragma unroll
      for (int f = 0; f < RT_FIELDS; ++f) s[f * RT_PLANE + idx] = v[f];
    }
  };
  stage(i0 - 1, 0);
  stage(i0, 1);
  int cur = 1;  // ring slot of plane i
  for (int i = i0; i <= i1; ++i) {
    const int nxt = cur == 2 ? 0 : cur + 1, prv = cur == 0 ? 2 : cur - 1;
    stage(i + 1, nxt);
    __syncthreads();
    if (j < NJ && k < NK) {
      const int sb[3] = {prv * RT_SLOT, cur * RT_SLOT, nxt * RT_SLOT};  // planes i-1, i, i+1
      const int c = (ty + 1) * RT_HK + tx + 1;
      const long long m = i * sI + j * sJ + k;
      auto lamAt = [&](int e, int di, int dj, int dk) { return sm[sb[di + 1] + e * RT_PLANE + c + dj * RT_HK + dk]; };
      // the inputs read at X only (momenta, rho_E, p) and the node's type: loaded before the gather, so
      // their latency overlaps it
      const double xv[5] = {A.val[1][m], A.val[2][m], A.val[3][m], A.val[4][m], V[7 * N + m]};
      const uint8_t tym = G.type[m];
      const bool filt = (tym & FILTER_BIT) != 0;
      const int fi = filt ? G.fidx[m] : 0;
      const double rho = filt ? A.valFpre[2 * fi] : A.valR[m];
      // the adjoints this node adds into (only this thread writes them in this kernel)
      double* const dR = filt ? A.lamFpre + 2 * fi : A.lamR + m;      // density's
      double* const dE = filt ? A.lamFpre + 2 * fi + 1 : nullptr;     // rho_E's, filter nodes
      const double aI1 = A.lamI[1][m], aI2 = A.lamI[2][m], aI3 = A.lamI[3][m], aI4 = A.lamI[4][m];
      const double aR = *dR, aE = filt ? *dE : 0.0;
      auto valAt = [&](int q, int di, int dj, int dk) {
        const int f = rt_field(q);
        return f >= 0 ? sm[sb[di + 1] + f * RT_PLANE + c + dj * RT_HK + dk] : xv[q == 7 ? 4 : q];
      };
      // the per-RHS-node conditions also bound the compiler's scheduling regions (without them it
      // interleaves all 19 blocks and runs out of registers)
      auto inner = [&](int di, int dj, int dk) {
        const int a = i - di, b = j - dj, d = k - dk;
        return a >= 1 && a <= NI - 2 && b >= 1 && b <= NJ - 2 && d >= 1 && d <= NK - 2;
      };
      double bar[11];
      rhs_adjoint_gather(C, lamAt, valAt, inner, bar);
      // chain rule: u = m r1, p = gm1 (rE - (rho+1) K), T = (gamma p - rho) r1, mu = x sqrt(x) sc1/(re (T+sc1)),
      // kappa = mu pf, with r1 = 1/(rho+1), K = |u|^2/2, x = 1 + T
      // the density of the primitives: the stage's density input, or the pre-filter copy at filter nodes
      const double r1 = recip_nr(rho + 1.0);
      const int cc = sb[1] + c;  // this node in the staged plane
      const double u = sm[cc + 5 * RT_PLANE], v = sm[cc + 6 * RT_PLANE], w = sm[cc + 7 * RT_PLANE],
                   T = sm[cc + 8 * RT_PLANE];
      const double K = 0.5 * (u * u + v * v + w * w);
      double ub = bar[4], vb = bar[5], wb = bar[6], pb = bar[7], Tb = bar[8], mub = bar[9];
      mub += C.pf * bar[10];
      const double x = 1.0 + T, sx = sqrt_nr(x), den = T + C.sc1;
      Tb += mub * C.sc1 * (1.5 * sx * den - x * sx) * recip_nr(C.re * den * den);
      pb += C.gamma * r1 * Tb;
      double rhob = -r1 * Tb - T * r1 * Tb;
      double rEb = C.gm1 * pb;
      rhob += -C.gm1 * K * pb;
      const double Kb = -C.gm1 * (rho + 1.0) * pb;
      ub += Kb * u;
      vb += Kb * v;
      wb += Kb * w;
      rhob += -(u * ub + v * vb + w * wb) * r1;
      A.lamI[1][m] = aI1 + (bar[0] + r1 * ub);
      A.lamI[2][m] = aI2 + (bar[1] + r1 * vb);
      A.lamI[3][m] = aI3 + (bar[2] + r1 * wb);
      *dR = aR + rhob;
      if (filt) {
        A.lamI[4][m] = aI4 + bar[3];
        *dE = aE + rEb;
      } else {
        A.lamI[4][m] = (aI4 + bar[3]) + rEb;
      }
    }
    __syncthreads();  // the next iteration restages the oldest slot
    cur = nxt;
  }
}

// ------------------------------------------------------------------------------- density filter
// k_density_filter: dst = (6 src + 6 neighbours)/12 at interior nodes, dst = src at edge-plane and ghost
// nodes; solid inactive nodes off the edge planes keep their value.
__device__ __forceinline__ int df_kind(uint8_t raw) {  // 2: filtered, 1: copied, 0: untouched
  const uint8_t t = raw & TYPE_MASK;
  return t == FLUID_INTERIOR ? 2 : (t != SOLID_INACTIVE || (raw & EDGE_PLANE_BIT)) ? 1 : 0;
}

__global__ void k_adj_density_filter(const Grid* __restrict__ gp, const double* __restrict__ lamDst,
                                     double* __restrict__ lamSrc) {
  const Grid& G = *gp;
  const long long off[6] = {G.sI, -G.sI, G.sJ, -G.sJ, 1, -1};
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < G.N; m += (long long)gridDim.x * blockDim.x) {
    const int kind = df_kind(G.type[m]);
    double a = kind == 2 ? 0.5 * lamDst[m] : kind == 1 ? lamDst[m] : 0.0;
    for (int d = 0; d < 6; ++d) {
      const long long n = m + off[d];
      if (n < 0 || n >= G.N) continue;
      if (df_kind(G.type[n]) == 2) a += lamDst[n] / 12;
    }
    lamSrc[m] += a;
  }
}

__global__ void k_adj_density_filter_clear(const Grid* __restrict__ gp, double* __restrict__ lamDst) {
  const Grid& G = *gp;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < G.N; m += (long long)gridDim.x * blockDim.x)
    if (df_kind(G.type[m])) lamDst[m] = 0.0;
}

int blocks_for(long long n, int nSM) {
  const long long b = (n + 255) / 256;
  return int(b < 8 * nSM ? (b > 0 ? b : 1) : 8 * nSM);
}

}  // namespace

// ------------------------------------------------------------------------------------ launchers
void launch_objective(const Grid* dg, const double* nx, double dA, double weight, double* acc, void* stream) {
  k_objective<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(dg, nx, dA, weight, acc);
}

// fpre = the density and rho_E of the filter nodes in buffer `U` (the state at level 0).
__global__ void k_fpre_init(const Grid* __restrict__ gp, const double* __restrict__ rho, const double* __restrict__ rE) {
  const Grid& G = *gp;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < G.nFilter; q += gridDim.x * blockDim.x) {
    G.fpre[2 * q] = rho[G.fnode[q]];
    G.fpre[2 * q + 1] = rE[G.fnode[q]];
  }
}

// The adjoint of that copy: the filter nodes' density / rho_E adjoints gather the fpre adjoints.
__global__ void k_fpre_init_adj(const Grid* __restrict__ gp, const double* __restrict__ lamFpre, double* lamRho,
                                double* lamRE) {
  const Grid& G = *gp;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < G.nFilter; q += gridDim.x * blockDim.x) {
    lamRho[G.fnode[q]] += lamFpre[2 * q];
    lamRE[G.fnode[q]] += lamFpre[2 * q + 1];
  }
}

void launch_fpre_init(const Grid* dg, int nFilter, const double* rho, const double* rE, int nSM, void* stream) {
  if (nFilter > 0) k_fpre_init<<<blocks_for(nFilter, nSM), 256, 0, static_cast<cudaStream_t>(stream)>>>(dg, rho, rE);
}

void launch_fpre_init_adj(const Grid* dg, int nFilter, const double* lamFpre, double* lamRho, double* lamRE, int nSM,
                          void* stream) {
  if (nFilter > 0)
    k_fpre_init_adj<<<blocks_for(nFilter, nSM), 256, 0, static_cast<cudaStream_t>(stream)>>>(dg, lamFpre, lamRho, lamRE);
}

void launch_adj_bc(const Grid& hg, const AdjBcParams& P, int s, int nSM, void* stream) {
  static int perSM = -1;
  if (perSM < 0) {
    int nb = 0;
    perSM = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_adj_bc, kAdjBcThreads, 0) == cudaSuccess ? nb : 0;
  }
  // enough blocks for the largest phase (of each chain when split), all resident (cooperative launch)
  auto blocks_of = [](long long items) { return std::max<long long>(1, (items + kAdjBcThreads - 1) / kAdjBcThreads); };
  const long long bodyItems = std::max<long long>(hg.nGhost + hg.nFilter, std::max(P.ncell, P.nfs));
  const long long edgeItems = 64ll * std::max(P.nEdge[0], std::max(P.nEdge[1], P.nEdge[2]));
  const long long cap = (long long)(perSM > 0 ? perSM : 1) * nSM;
  AdjBcParams Q = P;
  long long want = blocks_of(std::max(bodyItems, edgeItems));
  if (P.bodyBlocks > 0) {  // two chains: blocks for each (the request is a flag; the size is set here)
    const long long nbB = blocks_of(bodyItems), nbE = blocks_of(edgeItems);
    if (nbB + nbE <= cap) {
      Q.bodyBlocks = int(nbB);
      want = nbB + nbE;
    } else {
      Q.bodyBlocks = 0;
    }
  }
  const unsigned blocks = unsigned(want < cap ? want : cap);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kAdjBcThreads);
  cfg.stream = static_cast<cudaStream_t>(stream);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_adj_bc, hg, Q, s);
  k_adj_combine<<<blocks_for(hg.N, nSM), 256, 0, static_cast<cudaStream_t>(stream)>>>(hg, P, s);
}

int adj_kernels_init() {
  return int(cudaFuncSetAttribute(k_adj_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, RT_SMEM));
}

void launch_adj_rhs(const Grid* dg, const Grid& hg, const AdjPtrs& A, const double* lam, const double* V, int nSM,
                    void* stream) {
  // i-chunks: enough blocks for kAdjRhsBlocks per SM, each chunk at least 4 planes (a chunk of L planes
  // stages L + 2)
  const int tiles = ((hg.NJ + RT_J - 1) / RT_J) * ((hg.NK + RT_K - 1) / RT_K);
  int chunks = (kAdjRhsBlocks * nSM + tiles - 1) / tiles;
  chunks = std::max(1, std::min(chunks, hg.NI / 4));
  const int chunk = (hg.NI + chunks - 1) / chunks;
  chunks = (hg.NI + chunk - 1) / chunk;
  k_adj_rhs<<<dim3(tiles, chunks), dim3(32, RT_J), RT_SMEM, static_cast<cudaStream_t>(stream)>>>(dg, hg.C, A, lam, V,
                                                                                                   chunk);
}

void launch_copies(const double* const* src, double* const* dst, const long long* words, int count, int nSM,
                   void* stream) {
  if (count <= 0) return;
  CopySet S{};
  long long most = 1;
  for (int c = 0; c < count; ++c) {
    S.src[c] = src[c];
    S.dst[c] = dst[c];
    S.words[c] = words[c];
    most = words[c] > most ? words[c] : most;
  }
  const long long b = (most + 255) / 256, cap = 2LL * nSM;
  k_copy_set<<<dim3(unsigned(b < cap ? b : cap), count), 256, 0, static_cast<cudaStream_t>(stream)>>>(S);
}

void launch_tape_copy(const StepCtl* ctl, const TapeCopy& T, int nSM, void* stream) {
  if (T.n <= 0) return;
  long long most = 1;
  for (int c = 0; c < T.n; ++c) most = T.words[c] > most ? T.words[c] : most;
  const long long b = (most + 255) / 256, cap = 2LL * nSM;
  k_tape_copy<<<dim3(unsigned(b < cap ? b : cap), T.n), 256, 0, static_cast<cudaStream_t>(stream)>>>(ctl, T);
}

void launch_adj_density_filter(const Grid* dg, long long N, const double* lamDstConst, double* lamDst, double* lamSrc,
                               int nSM, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_adj_density_filter<<<blocks_for(N, nSM), 256, 0, st>>>(dg, lamDstConst, lamSrc);
  k_adj_density_filter_clear<<<blocks_for(N, nSM), 256, 0, st>>>(dg, lamDst);
}

}  // namespace nsf
