// Fused RK4 stage kernel for sm_100a: TMA-fed, warp-specialised, 2.5-D plane streaming.
// x-direction terms use per-node (G) and per-face (F) quantities carried in registers along the thread's
// column (see x_node / x_face in nsf_physics.cuh), so each staged value is read from shared memory once
// per plane by its own column; y/z terms read the in-plane neighbours from shared memory.
//
// One CTA (eight warps, one thread per (j, k) column of a TJ x TK tile) per SM, persistent over a static
// list of work items (a tile and a chunk of i-planes):
//   thread 0 issues cp.async.bulk.tensor (TMA) loads ahead of use -- for every i-plane of the item, the
//     five conserved fields and the node types of the tile plus a one-node halo (box 34 x 10) into a
//     6-slot ring (up to three planes ahead), and for every computed plane the U0 and RK4-accumulator tile
//     (box 34 x 8) into a 2-slot ring (one plane ahead). Each slot has a "full" mbarrier (TMA transaction
//     bytes) and an "empty" mbarrier (one arrival per warp when the slot's data is no longer needed);
//   all threads, in each interval between named barriers: the primitive and transport values of the
//     340 staged nodes of plane p are computed once into a 4-slot ring (filtered nodes take their values
//     from before the near-body filter, as the reference does), the column's x quantities of plane p-1
//     are formed, and the RHS and RK4 combine of plane p-2 are computed in registers and written with
//     coalesced 256-byte row stores. Staging and RHS of one interval are independent, so the scheduler
//     can interleave them.
// A dedicated producer warp is not used: with nine warps one SM sub-partition would hold three warps and
// cap registers at 168 per thread, which spills this kernel.
// All mbarrier waits are bounded; a wait that gives up sets StepCtl::timeout and the whole CTA stops at
// the next named barrier, after thread 0 has waited for every copy it issued.
// Conserved ring: 6 slots (plane being staged, the planes the x and y/z terms read, three in flight).
//
// Algorithmic HBM bytes per node: stage 1 reads U0 (40) and writes U1 and acc (80); stages 2-3 read
// U_s, U0, acc (120) and write U_{s+1}, acc (80); stage 4 reads U3, U0, acc (120) and writes U_new (40).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_physics.cuh"

namespace nsf {
namespace tma {
constexpr int TK = 32, TJ = 8, NCOMP = TK * TJ;  // threads (one per column of the tile)
constexpr int NTHREADS = NCOMP;
constexpr int HK = TK + 2, HJ = TJ + 2, HP = HK * HJ;
constexpr int FS = 352;                         // doubles per staged field (2816 B, a multiple of 128 B)
constexpr int EFS = HK * TJ;                    // doubles per epilogue field (2176 B = 17 x 128 B)
constexpr int NC = 6, NP = 4, NE = 2;           // conserved / primitive / epilogue ring depths
constexpr int TYW = 48;                         // row width of the staged node-type box (bytes, >= HK)
constexpr uint32_t CONS_BOX_BYTES = HK * HJ * 8;
constexpr uint32_t TYPE_BOX_BYTES = TYW * HJ;
constexpr uint32_t EPI_BOX_BYTES = HK * TJ * 8;
constexpr size_t TYPE_OFF = size_t(5) * FS * 8;  // node types follow the five fields in a staged slot
constexpr size_t CONS_SLOT = TYPE_OFF + 512;
constexpr size_t PRIM_SLOT = size_t(7) * FS * 8;
constexpr size_t EPI_SLOT = size_t(10) * EFS * 8;
constexpr size_t OFF_CONS = 0;
constexpr size_t OFF_PRIM = OFF_CONS + NC * CONS_SLOT;
constexpr size_t OFF_EPI = OFF_PRIM + NP * PRIM_SLOT;
constexpr size_t OFF_BAR = OFF_EPI + NE * EPI_SLOT;
constexpr size_t OFF_RED = OFF_BAR + 32 * 8;
constexpr size_t OFF_GRID = OFF_RED + 5 * 32 * 8;
constexpr size_t OFF_CTL = OFF_GRID + ((sizeof(Grid) + 127) / 128) * 128;
constexpr size_t SMEM = OFF_CTL + ((sizeof(StepCtl) + 127) / 128) * 128;
static_assert(OFF_PRIM % 128 == 0 && OFF_EPI % 128 == 0 && CONS_SLOT % 128 == 0 && TYPE_OFF % 128 == 0,
              "TMA destinations need 128 B alignment");
static_assert(TYPE_BOX_BYTES <= 512, "type box fits its slot region");
static_assert(SMEM <= 227 * 1024, "shared memory budget");
constexpr int MAP_CONS = 0, MAP_EPI = 15, MAP_ACC = 30, MAP_TYPE = 35, NMAPS = 36;
constexpr long long WAIT_LIMIT = 1ll << 22;  // try_wait polls before a wait is declared failed
}  // namespace tma

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  for (long long it = 0; it < tma::WAIT_LIMIT; ++it)
    if (mbar_try(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load3(void* dst, const void* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// Named barrier 1 over the eight compute warps, returning the OR of `v` over them.
__device__ __forceinline__ bool compute_bar_or(bool v) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred pi, po;\n setp.ne.u32 pi, %1, 0;\n bar.red.or.pred po, 1, 256, pi;\n selp.u32 %0, 1, 0, po;\n}\n"
      : "=r"(r)
      : "r"(v ? 1u : 0u)
      : "memory");
  return r != 0;
}

}  // namespace

__global__ void __launch_bounds__(tma::NTHREADS, 1)
    k_stage_tma(const Grid* __restrict__ gp, const StageItem* __restrict__ items, int nItems, int s) {
  using namespace tma;
  extern __shared__ __align__(1024) unsigned char sm[];
  uint64_t* consFull = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint64_t* consEmpty = consFull + NC;
  uint64_t* epiFull = consEmpty + NC;
  uint64_t* epiEmpty = epiFull + NE;
  double* red = reinterpret_cast<double*>(sm + OFF_RED);
  Grid& G = *reinterpret_cast<Grid*>(sm + OFF_GRID);
  StepCtl& ctl = *reinterpret_cast<StepCtl*>(sm + OFF_CTL);
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) {
    G = *gp;
    ctl = *gp->ctl;
    for (int q = 0; q < NC; ++q) {
      mbar_init(&consFull[q], 1);
      mbar_init(&consEmpty[q], 8);
    }
    for (int q = 0; q < NE; ++q) {
      mbar_init(&epiFull[q], 1);
      mbar_init(&epiEmpty[q], 8);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (!ctl.active) return;
  const Consts& C = G.C;
  DtAcc dta;
  double nsum[5] = {0, 0, 0, 0, 0};
  int bad = 0;

  // ---------------------------------------------------------------------- TMA issue (thread 0)
  // Two cursors walk this CTA's plane sequence: every staged plane (conserved ring, issued two planes
  // ahead of its use) and every computed plane (epilogue ring, issued one plane ahead).
  const CUtensorMap* maps = static_cast<const CUtensorMap*>(G.tmaps);
  int cIt = blockIdx.x, cP = cIt < nItems ? items[cIt].i0 - 1 : 0;  // next staged plane to issue
  int eIt = blockIdx.x, eP = eIt < nItems ? items[eIt].i0 : 0;      // next computed plane to issue
  uint32_t cIssued = 0, eIssued = 0;
  bool issueFailed = false;
  const int epiFields = s == 0 ? 5 : 10;
  auto issue_cons = [&]() {
    if (cIt >= nItems || issueFailed) return;
    const StageItem w = items[cIt];
    const uint32_t q = cIssued, sl = q % NC;
    if (q >= NC && !mbar_wait(&consEmpty[sl], ((q / NC) - 1) & 1)) {
      issueFailed = true;
      return;
    }
    unsigned char* dst = sm + OFF_CONS + sl * CONS_SLOT;
    mbar_expect_tx(&consFull[sl], 5 * CONS_BOX_BYTES + TYPE_BOX_BYTES);
    tma_load3(dst, &maps[MAP_CONS + ctl.rPhys[s] * 5 + 0], w.k0 - 1, w.j0 - 1, cP, &consFull[sl]);
    for (int f = 1; f < 5; ++f)
      tma_load3(dst + size_t(f) * FS * 8, &maps[MAP_CONS + ctl.iPhys[s][f] * 5 + f], w.k0 - 1, w.j0 - 1, cP,
                &consFull[sl]);
    tma_load3(dst + TYPE_OFF, &maps[MAP_TYPE], w.k0 - 1, w.j0 - 1, cP, &consFull[sl]);
    ++cIssued;
    if (++cP > w.i1 + 1) {
      cIt += gridDim.x;
      if (cIt < nItems) cP = items[cIt].i0 - 1;
    }
  };
  auto issue_epi = [&]() {
    if (eIt >= nItems || issueFailed) return;
    const StageItem w = items[eIt];
    const uint32_t e = eIssued, se = e % NE;
    if (e >= NE && !mbar_wait(&epiEmpty[se], ((e / NE) - 1) & 1)) {
      issueFailed = true;
      return;
    }
    unsigned char* dst = sm + OFF_EPI + se * EPI_SLOT;
    mbar_expect_tx(&epiFull[se], epiFields * EPI_BOX_BYTES);
    for (int f = 0; f < 5; ++f)
      tma_load3(dst + size_t(f) * EFS * 8, &maps[MAP_EPI + ctl.u0Phys[f] * 5 + f], w.k0 - 1, w.j0, eP, &epiFull[se]);
    if (s > 0)
      for (int f = 0; f < 5; ++f)
        tma_load3(dst + size_t(5 + f) * EFS * 8, &maps[MAP_ACC + f], w.k0 - 1, w.j0, eP, &epiFull[se]);
    ++eIssued;
    if (++eP > w.i1) {
      eIt += gridDim.x;
      if (eIt < nItems) eP = items[eIt].i0;
    }
  };
  // Thread 0 keeps the conserved ring LOOK planes ahead of staging. It only issues into a slot whose
  // previous plane its own warp has released; the other warps release it without depending on thread 0,
  // so an issue wait always ends.
  constexpr uint32_t LOOK = 4;  // 6 slots: staged, read by x, read by the RHS, three in flight
  uint32_t released = 0;  // number of staged planes (in sequence order) released by all warps so far
  auto top_up = [&](uint32_t stagedNext) {
    while (cIt < nItems && cIssued < stagedNext + LOOK && cIssued < released + NC) issue_cons();
  };
  if (tid == 0) {
    top_up(0);
    issue_epi();
  }
  {
    // ------------------------------------------------------------------ all threads: stage, x, RHS
    const int tx = tid % TK, ty = tid / TK;
    const int cidx = (ty + 1) * HK + (tx + 1);  // this column's node in a staged plane
    const int eidx = ty * HK + tx + 1;          // ... in an epilogue tile
    const int tcix = (ty + 1) * TYW + (tx + 1); // ... in a staged type box
    // staged nodes of this thread: idx0 for every thread, idx1 for the first HP - 256 threads
    const int idx0 = tid, hj0 = idx0 / HK, hk0 = idx0 - hj0 * HK;
    const bool has1 = tid + NCOMP < HP;
    const int idx1 = has1 ? tid + NCOMP : tid, hj1 = idx1 / HK, hk1 = idx1 - hj1 * HK;
    const double dtUsed = ctl.dtUsed;
    const double inc = (s == 2) ? dtUsed : dtUsed / 2;
    const double dtFactor = dtUsed / 6;
    const double* __restrict__ fpre = G.fpre;
    double* const out0 = ctl.O[s][0];
    double* const out1 = ctl.O[s][1];
    double* const out2 = ctl.O[s][2];
    double* const out3 = ctl.O[s][3];
    double* const out4 = ctl.O[s][4];
    double* const accb = G.acc[0];  // accumulator fields are contiguous, G.N doubles apart
    const long long NdF = G.N;
    unsigned char* const consBase = sm + OFF_CONS;
    unsigned char* const primBase = sm + OFF_PRIM;
    uint32_t qc = 0, qe = 0;
    bool abort = false;
    // Stage one node: primitive / transport values from the landed conserved values (filtered nodes use
    // their values from before the near-body filter). Nodes past the mesh read TMA zero fill; their values
    // are finite and never used.
    auto stage_node = [&](const double* cs, double* ps, const uint8_t* ts, int idx, int hj, int hk, int pS,
                          int j0, int k0) {
      const uint8_t ty8 = ts[hj * TYW + hk];
      double rho = cs[0 * FS + idx], rE = cs[4 * FS + idx];
      if (ty8 & FILTER_BIT) {
        const long long n = (long long)pS * G.sI + (long long)(j0 - 1 + hj) * G.sJ + (k0 - 1 + hk);
        const int f = __ldg(G.fidx + n);
        rho = fpre[2 * f];
        rE = fpre[2 * f + 1];
      }
      const Prim pr = prims_of(C, rho, cs[1 * FS + idx], cs[2 * FS + idx], cs[3 * FS + idx], rE);
      ps[0 * FS + idx] = pr.u;
      ps[1 * FS + idx] = pr.v;
      ps[2 * FS + idx] = pr.w;
      ps[3 * FS + idx] = pr.p;
      ps[4 * FS + idx] = pr.T;
      ps[5 * FS + idx] = pr.mu;
      ps[6 * FS + idx] = pr.ka;
    };
    int pSl = 0;  // primitive-ring slot of the next staged plane, continues across items
    for (int it = blockIdx.x; it < nItems && !abort; it += gridDim.x) {
      const StageItem w = items[it];
      const int j = w.j0 + ty, k = w.k0 + tx;
      const bool inTile = (j <= G.NJ - 2) && (k <= G.NK - 2);
      const int L = w.i1 - w.i0 + 1;
      const uint32_t qb = qc;  // sequence number of plane i0-1
      // conserved-ring slot of the plane staged in iteration a (sequence qb + a), advanced incrementally
      int cS = int(qb % NC);
      uint32_t phS = (qb / NC) & 1;
      long long nR = (long long)(w.i0 - 3) * G.sI + (long long)j * G.sJ + k;  // node of plane i0-3+a
      // x-direction state of this thread's column, carried from plane to plane
      XNode gm1{}, gm2{};
      double fprev[5] = {0, 0, 0, 0, 0};
      XOwn ownPrev{};
      // Iteration a stages plane i0-1+a, builds the column's x quantities of plane i0-2+a and computes the
      // RHS of plane i0-3+a; a named barrier closes each iteration (the next iteration reads the plane
      // staged in this one and overwrites the primitive slot this one's RHS read last).
      for (int a = 0; a <= L + 2; ++a) {
        const int pS = w.i0 - 1 + a;
        const bool doS = a <= L + 1, doX = a >= 1, doR = a >= 3;
        const int cX = cS == 0 ? NC - 1 : cS - 1, cR = cX == 0 ? NC - 1 : cX - 1;
        const int pX = pSl == 0 ? NP - 1 : pSl - 1, pR = pX == 0 ? NP - 1 : pX - 1, pW = pR == 0 ? NP - 1 : pR - 1;
        if (tid == 0) {
          top_up(doS ? qb + a : qc);
          if (doR) issue_epi();  // the computed plane after the one this iteration finishes
        }
        bool ok = true;
        if (doS) {
          ++qc;
          ok = mbar_wait(&consFull[cS], phS);
          if (ok) {
            const double* cs = reinterpret_cast<const double*>(consBase + cS * CONS_SLOT);
            double* ps = reinterpret_cast<double*>(primBase + pSl * PRIM_SLOT);
            const uint8_t* ts = reinterpret_cast<const uint8_t*>(cs) + TYPE_OFF;
            stage_node(cs, ps, ts, idx0, hj0, hk0, pS, w.j0, w.k0);
            if (has1) stage_node(cs, ps, ts, idx1, hj1, hk1, pS, w.j0, w.k0);
          }
        }
        // x quantities of the column's node on plane pS-1 (staged in the previous iteration)
        XNode gcur{};
        XOwn ownCur{};
        double fcur[5] = {0, 0, 0, 0, 0};
        if (doX && ok) {
          constexpr int oN = HK, oU = 1;
          const double* cs = reinterpret_cast<const double*>(consBase + cX * CONS_SLOT);
          const double* ps = reinterpret_cast<const double*>(primBase + pX * PRIM_SLOT);
          ownCur = XOwn{ps[5 * FS + cidx], ps[0 * FS + cidx], ps[1 * FS + cidx], ps[2 * FS + cidx], ps[4 * FS + cidx],
                        ps[6 * FS + cidx]};
          gcur = x_node(C, cs[1 * FS + cidx], cs[2 * FS + cidx], cs[3 * FS + cidx], cs[4 * FS + cidx], ownCur.u,
                        ownCur.v, ownCur.w, ps[3 * FS + cidx], ownCur.mu,
                        ps[1 * FS + cidx + oN] - ps[1 * FS + cidx - oN], ps[0 * FS + cidx + oN] - ps[0 * FS + cidx - oN],
                        ps[2 * FS + cidx + oU] - ps[2 * FS + cidx - oU], ps[0 * FS + cidx + oU] - ps[0 * FS + cidx - oU]);
          if (a >= 2) x_face(C, ownPrev, ownCur, fcur);
          if (a == 1) {  // plane i0-1: its conserved values have no other reader
            __syncwarp();
            if (lane == 0) mbar_arrive(&consEmpty[cX]);
            if (tid == 0) released = qb + 1;
          }
        }
        if (doR && ok) {
          const uint32_t e = qe++;
          const bool eok = mbar_wait(&epiFull[e & 1], (e >> 1) & 1);
          const double* cP = reinterpret_cast<const double*>(consBase + cR * CONS_SLOT);
          const uint8_t tc = (reinterpret_cast<const uint8_t*>(cP) + TYPE_OFF)[tcix];
          const bool valid = eok && inTile && (tc & TYPE_MASK) == FLUID_INTERIOR;
          double kk5[5];
          yz_part<HK, FS>(C, cP, reinterpret_cast<const double*>(primBase + pW * PRIM_SLOT),
                          reinterpret_cast<const double*>(primBase + pR * PRIM_SLOT),
                          reinterpret_cast<const double*>(primBase + pX * PRIM_SLOT), cidx, ownPrev, kk5);
#pragma unroll
          for (int f = 0; f < 5; ++f) kk5[f] += (gcur.g[f] - gm2.g[f]) + (fcur[f] - fprev[f]);
          const double* ep = reinterpret_cast<const double*>(sm + OFF_EPI + (e & 1) * EPI_SLOT);
          double u0[5], res[5];
#pragma unroll
          for (int f = 0; f < 5; ++f) u0[f] = ep[f * EFS + eidx];
          if (s == 0) {
#pragma unroll
            for (int f = 0; f < 5; ++f) res[f] = u0[f] + inc * kk5[f];
            if (valid) {
#pragma unroll
              for (int f = 0; f < 5; ++f) accb[f * NdF + nR] = kk5[f];
            }
          } else if (s < 3) {
            double an[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
              an[f] = ep[(5 + f) * EFS + eidx] + 2 * kk5[f];
              res[f] = u0[f] + inc * kk5[f];
            }
            if (valid) {
#pragma unroll
              for (int f = 0; f < 5; ++f) accb[f * NdF + nR] = an[f];
            }
          } else {
#pragma unroll
            for (int f = 0; f < 5; ++f) res[f] = u0[f] + dtFactor * (ep[(5 + f) * EFS + eidx] + kk5[f]);
            const bool filtered = (tc & FILTER_BIT) != 0;  // rho, rho_E change again in the near-body filter
#pragma unroll
            for (int f = 0; f < 5; ++f) {
              const double d = u0[f] - res[f];
              nsum[f] += (valid && !(filtered && (f == 0 || f == 4))) ? d * d : 0.0;
            }
            bad |= valid && !(isfinite(res[0]) && isfinite(res[1]) && isfinite(res[2]) && isfinite(res[3]) &&
                              isfinite(res[4]));
            if (valid && !filtered) {
              const Prim pr = prims_of(C, res[0], res[1], res[2], res[3], res[4]);
              dta.add(C, res[0], pr.u, pr.v, pr.w, pr.p, pr.mu);
            }
          }
          if (valid) {
            out0[nR] = res[0];
            out1[nR] = res[1];
            out2[nR] = res[2];
            out3[nR] = res[3];
            out4[nR] = res[4];
          }
          ok = eok;
          __syncwarp();
          if (lane == 0) {
            mbar_arrive(&epiEmpty[e & 1]);
            mbar_arrive(&consEmpty[cR]);   // plane pS-2: its last reader was this RHS
          }
          if (tid == 0) released = qb + uint32_t(a) - 1;  // planes up to sequence qb+a-2 released
          if (a == L + 2) {                // the item's last plane: its conserved values have no other reader
            __syncwarp();
            if (lane == 0) mbar_arrive(&consEmpty[cX]);
            if (tid == 0) released = qc;
          }
        }
        if (compute_bar_or(!ok)) {  // some thread's wait gave up: the whole CTA stops here
          if (!ok) atomicExch(&gp->ctl->timeout, 1);
          abort = true;
          break;
        }
        if (doX) {
          gm2 = gm1;
          gm1 = gcur;
#pragma unroll
          for (int f = 0; f < 5; ++f) fprev[f] = fcur[f];
          ownPrev = ownCur;
        }
        nR += G.sI;
        if (doS) {
          if (++cS == NC) {
            cS = 0;
            phS ^= 1;
          }
          if (++pSl == NP) pSl = 0;
        }
      }
    }
  }
  if (tid == 0) {
    if (issueFailed) atomicExch(&gp->ctl->timeout, 1);
    // Every copy issued must have landed before the CTA exits: wait for the last phase of each slot.
    for (uint32_t sl = 0; sl < NC; ++sl)
      if (cIssued > sl) {
        const uint32_t last = cIssued - 1 - ((cIssued - 1 - sl) % NC);
        if (!mbar_wait(&consFull[sl], (last / NC) & 1)) atomicExch(&gp->ctl->timeout, 1);
      }
    for (uint32_t se = 0; se < NE; ++se)
      if (eIssued > se) {
        const uint32_t last = eIssued - 1 - ((eIssued - 1 - se) % NE);
        if (!mbar_wait(&epiFull[se], (last / NE) & 1)) atomicExch(&gp->ctl->timeout, 1);
      }
  }
  if (s == 3) {
    flush_dt(gp->ctl, dta, red);
    flush_norms(G.normPart + 5 * blockIdx.x, nsum, red);
    if (bad) atomicOr(&gp->ctl->nonFinite, 1);
  }
}

size_t stage_smem_bytes() { return tma::SMEM; }
int stage_configure() {
  return int(cudaFuncSetAttribute(k_stage_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma::SMEM)));
}
int stage_tile_j() { return tma::TJ; }
int stage_tile_k() { return tma::TK; }
int stage_threads() { return tma::NTHREADS; }
int stage_occupancy() {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stage_tma, tma::NTHREADS, tma::SMEM);
  return nb;
}
int stage_num_maps() { return tma::NMAPS; }
void launch_stage(const Grid* dg, const LaunchPlan& L, int s, void* stream) {
  k_stage_tma<<<L.stageBlocks, tma::NTHREADS, tma::SMEM, static_cast<cudaStream_t>(stream)>>>(dg, L.items, L.nItems, s);
}

}  // namespace nsf
