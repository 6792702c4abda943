// Fused RK4 stage kernel for sm_100a: TMA-fed, warp-specialised, 2.5-D plane streaming along i.
//
// One CTA of 384 threads per SM, persistent over a static list of work items (a TJ x TK tile of (j, k)
// columns and a chunk of i-planes). Three warpgroups with separate jobs, decoupled by mbarrier rings:
//
//   warpgroup 0, warp 0, lane 0 -- producer: issues cp.async.bulk.tensor (TMA) loads as soon as a ring
//     slot is free: for every staged i-plane the five conserved fields and the node types of the tile
//     plus a one-node halo (box 34 x 10) into the conserved ring, and for every computed plane the U0
//     and RK4-accumulator tile (box 34 x 8) into the epilogue ring. It never blocks on one slot, so no
//     ordering between the rings can deadlock.
//   warpgroup 0, warps 1-3 -- staging: the primitive and transport values (u, v, w, p, T, mu) of
//     the 340 staged nodes of each plane, once per plane, into the primitive ring. Filtered nodes take
//     their values from before the near-body filter, as the reference does (its primitives are not
//     recomputed after the filter).
//   warpgroups 1-2 -- columns: one thread per (j, k) column of the tile. For each plane the thread forms
//     its node's x-direction quantities (G of the node, F of the face towards the previous plane,
//     see x_node / x_face in nsf_physics.cuh) and carries them in registers along the column; the
//     RHS of the previous plane is then G/F differences plus the y/z terms read from the staged planes,
//     and the RK4 combine is written with coalesced 256-byte row stores.
// Warpgroup 0 runs with 88 registers per thread and the column warpgroups with 208 (setmaxnreg), so
// the register-hungry RHS does not spill while the CTA still has twelve warps.
//
// Ring slots have a "full" and an "empty" mbarrier. Every wait is bounded: a wait that gives up sets
// StepCtl::timeout and a CTA-wide abort flag that ends every other wait at once; the producer then
// waits (bounded) for every copy it issued before the CTA exits.
//
// Algorithmic HBM bytes per node: stage 1 reads U0 (40) and writes U1 and acc (80); stages 2-3 read
// U_s, U0, acc (120) and write U_{s+1}, acc (80); stage 4 reads U3, U0, acc (120) and writes U_new (40).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>

#include <cstdint>

#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_physics.cuh"

namespace nsf {
namespace ws {
constexpr int NSTAGE = 96;                        // staging threads (warps 1-3)
constexpr int NC = 5, NP = 5, NE = 3;             // conserved / primitive / epilogue ring depths
constexpr int NPRIM = 6;                          // staged primitive fields: u, v, w, p, T, mu (kappa = pf mu)
constexpr int MAP_CONS = 0, MAP_EPI = 15, MAP_ACC = 30, MAP_TYPE = 35, NMAPS = 36;
constexpr long long WAIT_LIMIT = 1ll << 22;  // default polls before a wait is declared failed (StepCtl::waitLimit)
// Register split (setmaxnreg): the launch gives every thread 168 registers (384 x 168 = 64,512); the
// split must not exceed that total: 128 x 88 + 256 x 208 = 64,512.
constexpr int REG_LAUNCH = 168, REG_LOW = 88, REG_HIGH = 208;
// The ensemble's stage-4 instantiation (per-item coefficients and the dt / norm accumulators) gives its
// column threads 8 more: 128 x 72 + 256 x 216 = 64,512.
constexpr int REG_LOW_ENS4 = 72, REG_HIGH_ENS4 = 216;

constexpr int round_up(int x, int m) { return (x + m - 1) / m * m; }

// An ensemble column warp's per-item values, kept in shared memory and read where they are used (through
// volatile loads): held in registers across the item's loop they would push the column threads past their
// register budget.
struct ItemSm {
  double* out[5];  // stage output fields
  double* acc;     // accumulator fields (contiguous, N doubles apart)
  long long N, sI;
  double inc, dtFactor;
};

// Tile geometry of one kernel variant: TK x TJ columns (one column thread each, 256 in total).
template <int TK_, int TJ_>
struct Tile {
  static constexpr int TK = TK_, TJ = TJ_, NCOL = TK * TJ;
  static constexpr int NTHREADS = 128 + NCOL;
  static constexpr int HK = TK + 2, HJ = TJ + 2, HP = HK * HJ;
  static constexpr int FS = round_up(HP, 16);     // doubles per staged field (a multiple of 128 B)
  static constexpr int EFS = HK * TJ;             // doubles per epilogue field
  static constexpr int TYW = round_up(HK, 16);    // row width of the staged node-type box (bytes)
  static constexpr uint32_t CONS_BOX_BYTES = HK * HJ * 8;
  static constexpr uint32_t TYPE_BOX_BYTES = TYW * HJ;
  static constexpr uint32_t EPI_BOX_BYTES = HK * TJ * 8;
  static constexpr size_t TYPE_OFF = size_t(5) * FS * 8;  // node types follow the five fields in a slot
  static constexpr size_t CONS_SLOT = TYPE_OFF + size_t(round_up(TYW * HJ, 128));
  static constexpr size_t PRIM_SLOT = size_t(NPRIM) * FS * 8;
  static constexpr size_t EPI_SLOT = size_t(10) * EFS * 8;
  static constexpr size_t OFF_CONS = 0;
  static constexpr size_t OFF_PRIM = OFF_CONS + NC * CONS_SLOT;
  static constexpr size_t OFF_EPI = OFF_PRIM + NP * PRIM_SLOT;
  static constexpr size_t OFF_BAR = OFF_EPI + NE * EPI_SLOT;
  static constexpr size_t OFF_FLAG = OFF_BAR + 2 * (NC + NP + NE) * 8;
  static constexpr size_t OFF_RED = (OFF_FLAG + 16 + 127) / 128 * 128;
  static constexpr size_t OFF_CTL = OFF_RED + 5 * 32 * 8;
  // ensemble kernels: per column warp, a copy of the current member's Consts and of the item's output
  // pointers and step factors (ItemSm)
  static constexpr size_t CONSTS_BYTES = (sizeof(Consts) + 15) / 16 * 16;
  static constexpr size_t CSM_BYTES = CONSTS_BYTES + (sizeof(ItemSm) + 15) / 16 * 16;
  static constexpr size_t OFF_CSM = OFF_CTL + ((sizeof(StepCtl) + 127) / 128) * 128;
  static constexpr size_t SMEM = OFF_CSM + 8 * CSM_BYTES;
  static_assert(NCOL == 256, "two column warpgroups");
  static_assert(TK % 16 == 0, "box x coordinate k0 - 1 = TK * t must be 16-byte aligned for TMA");
  static_assert((EFS * 8) % 128 == 0 && (FS * 8) % 128 == 0, "TMA destinations need 128 B alignment");
  static_assert(OFF_PRIM % 128 == 0 && OFF_EPI % 128 == 0 && CONS_SLOT % 128 == 0 && TYPE_OFF % 128 == 0,
                "TMA destinations need 128 B alignment");
  static_assert(SMEM <= 227 * 1024, "shared memory budget");
  static_assert(NSTAGE * 4 >= HP, "four staging passes cover a plane");
  static_assert(128 * REG_LOW + NCOL * REG_HIGH <= NTHREADS * REG_LAUNCH, "register split exceeds the launch total");
  static_assert(128 * REG_LOW_ENS4 + NCOL * REG_HIGH_ENS4 <= NTHREADS * REG_LAUNCH, "register split exceeds the launch total");
};
}  // namespace ws

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
// Bounded wait for the completion of the phase with the given parity: at most *limit polls (the limit is
// read from shared memory only once the first poll has failed, so it holds no register on the fast path),
// and it gives up early when another thread has raised the CTA's abort flag.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, const volatile int* abortFlag,
                                          const long long* limit) {
  if (mbar_try(b, parity)) return true;
  const long long lim = *limit;
  for (long long it = 1; it < lim; ++it) {
    if (mbar_try(b, parity)) return true;
    if (*abortFlag) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_load3(void* dst, const void* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
template <int N>
__device__ __forceinline__ void reg_dealloc() {
  asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(N));
}
template <int N>
__device__ __forceinline__ void reg_alloc() {
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(N));
}

// dt-limit terms of a node of the new state (getInviscidTimeStepLimit / getViscousTimeStepLimit,
// Solver.cpp:91-126) with one reciprocal of 1 + rho for all the divisions by it, reciprocals and square
// roots by Newton-Raphson (recip_nr, sqrt_nr). The terms only enter maxima, so their last-bit rounding
// moves dt by at most an ulp or two.
__device__ __forceinline__ void dt_terms(const Consts& C, const double (&u)[5], DtAcc& a) {
  const double r1 = recip_nr(u[0] + 1.0);
  const double vx = u[1] * r1, vy = u[2] * r1, vz = u[3] * r1;
  const double p = C.gm1 * (u[4] - (u[0] + 1.0) * 0.5 * (vx * vx + vy * vy + vz * vz));
  const double T = (C.gamma * p - u[0]) * r1;
  const double x = 1.0 + T;
  const double c = sqrt_nr((1.0 + C.gamma * p) * r1);
  a.sx = fmax(a.sx, c + fabs(vx));
  a.sy = fmax(a.sy, c + fabs(vy));
  a.sz = fmax(a.sz, c + fabs(vz));
  a.nu = fmax(a.nu, x * sqrt_nr(x) * C.sc1 * r1 * recip_nr(C.re * (T + C.sc1)) * C.vmod);
}

}  // namespace

// ENS = false: one grid, passed by value (its stencil coefficients are then constant-bank operands).
// ENS = true: an ensemble; every work item names its member (StageItem::g) in the device array `grids`,
// and each member's StepCtl is read from device memory.
// Work items of CTA b: items[ctaStart[b] .. ctaStart[b + 1]).
// MODE: which stages an instantiation serves -- 0 any (s at run time), 1 stages 1-3, 2 stage 4 (s == 3, the
// only stage with dt maxima, change norms and the NaN check; mode 1 carries none of their registers). The
// single grid runs mode 0 for stages 1-3 and mode 2 for stage 4, an ensemble modes 1 and 2: the fastest
// pairing measured (mode 1 frees registers an ensemble needs, but its schedule is slower for one grid).
template <int TK_, int TJ_, bool ENS, int MODE>
__global__ void __launch_bounds__(ws::Tile<TK_, TJ_>::NTHREADS, 1)
    k_stage_ws(const __grid_constant__ Grid G0, const Grid* __restrict__ grids, const StageItem* __restrict__ items,
               const int* __restrict__ ctaStart, int s) {
  using namespace ws;
  using TL = Tile<TK_, TJ_>;
  constexpr int TK = TL::TK, NCOL = TL::NCOL, HK = TL::HK, HP = TL::HP, FS = TL::FS, EFS = TL::EFS,
                TYW = TL::TYW;
  constexpr uint32_t CONS_BOX_BYTES = TL::CONS_BOX_BYTES, TYPE_BOX_BYTES = TL::TYPE_BOX_BYTES,
                     EPI_BOX_BYTES = TL::EPI_BOX_BYTES;
  constexpr size_t TYPE_OFF = TL::TYPE_OFF, CONS_SLOT = TL::CONS_SLOT, PRIM_SLOT = TL::PRIM_SLOT,
                   EPI_SLOT = TL::EPI_SLOT, OFF_CONS = TL::OFF_CONS, OFF_PRIM = TL::OFF_PRIM, OFF_EPI = TL::OFF_EPI,
                   OFF_BAR = TL::OFF_BAR, OFF_FLAG = TL::OFF_FLAG, OFF_RED = TL::OFF_RED, OFF_CTL = TL::OFF_CTL,
                   OFF_CSM = TL::OFF_CSM, CSM_BYTES = TL::CSM_BYTES;
  extern __shared__ __align__(1024) unsigned char sm[];
  uint64_t* consFull = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint64_t* consEmpty = consFull + NC;
  uint64_t* primFull = consEmpty + NC;
  uint64_t* primEmpty = primFull + NP;
  uint64_t* epiFull = primEmpty + NP;
  uint64_t* epiEmpty = epiFull + NE;
  volatile int* abortFlag = reinterpret_cast<volatile int*>(sm + OFF_FLAG);
  int* withholdSm = reinterpret_cast<int*>(sm + OFF_FLAG + 4);
  long long* limitSm = reinterpret_cast<long long*>(sm + OFF_FLAG + 8);
  double* red = reinterpret_cast<double*>(sm + OFF_RED);
  StepCtl& ctl0 = *reinterpret_cast<StepCtl*>(sm + OFF_CTL);  // single grid: a copy of its StepCtl
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int itBegin = ctaStart[blockIdx.x], itEnd = ctaStart[blockIdx.x + 1];
  auto grid_of = [&](const StageItem& w) -> const Grid& {
    if constexpr (ENS) return grids[w.g];
    else return G0;
  };
  auto ctl_of = [&](const Grid& g) -> const StepCtl& {
    if constexpr (ENS) return *g.ctl;
    else return ctl0;
  };
  if (tid == 0) {
    if (!ENS) ctl0 = *G0.ctl;
    *abortFlag = 0;
    {  // wait limit and test switch: the grid's control block (an ensemble: its first member's)
      const StepCtl* c = ENS ? grids[0].ctl : G0.ctl;
      const long long l = c->waitLimit;
      *limitSm = l > 0 ? l : WAIT_LIMIT;
      *withholdSm = c->withhold;
    }
    for (int q = 0; q < NC; ++q) {
      mbar_init(&consFull[q], 1);
      mbar_init(&consEmpty[q], NCOL / 32);
    }
    for (int q = 0; q < NP; ++q) {
      mbar_init(&primFull[q], NSTAGE / 32);
      mbar_init(&primEmpty[q], NCOL / 32);
    }
    for (int q = 0; q < NE; ++q) {
      mbar_init(&epiFull[q], 1);
      mbar_init(&epiEmpty[q], NCOL / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (!ENS && !ctl0.active) return;
  const long long* const lim = limitSm;
  DtAcc dta;
  double nsum[5] = {0, 0, 0, 0, 0};
  int bad = 0;
  auto fail = [&](const Grid& g) {
    *abortFlag = 1;
    atomicExch(&g.ctl->timeout, 1);
  };
  // an ensemble member whose run has ended (end_time reached) is skipped by every role
  auto skip = [&](const StageItem& w) { return ENS && !ctl_of(grid_of(w)).active; };

  if (warp < 4) {
    reg_dealloc<(ENS && MODE == 2) ? REG_LOW_ENS4 : REG_LOW>();
    if (warp == 0) {
      // ------------------------------------------------------------------ producer (one thread)
      if (lane == 0) {
        const int epiFields = s == 0 ? 5 : 10;
        auto next_item = [&](int it) {
          while (it < itEnd && skip(items[it])) ++it;
          return it;
        };
        int cIt = next_item(itBegin), cP = cIt < itEnd ? items[cIt].i0 - 1 : 0;  // next staged plane
        int eIt = cIt, eP = eIt < itEnd ? items[eIt].i0 : 0;                     // next computed plane
        if (*withholdSm) eIt = itEnd;  // test switch: no epilogue load is ever issued
        uint32_t cq = 0, eq = 0;
        long long idle = 0;
        // descriptors of the item each cursor is in (reloaded only when the cursor moves to a new item)
        const CUtensorMap* cMaps = nullptr;
        const CUtensorMap* eMaps = nullptr;
        int cPhys[5] = {0, 0, 0, 0, 0}, ePhys[5] = {0, 0, 0, 0, 0};
        int cLoaded = -1, eLoaded = -1;
        while ((cIt < itEnd || eIt < itEnd) && !*abortFlag) {
          bool progressed = false;
          if (cIt < itEnd) {
            const uint32_t sl = cq % NC;
            if (cq < NC || mbar_try(&consEmpty[sl], ((cq / NC) - 1) & 1)) {
              const StageItem w = items[cIt];
              if (cLoaded != cIt) {
                const Grid& G = grid_of(w);
                const StepCtl& ctl = ctl_of(G);
                cMaps = static_cast<const CUtensorMap*>(G.tmaps);
                cPhys[0] = ctl.rPhys[s];
                for (int f = 1; f < 5; ++f) cPhys[f] = ctl.iPhys[s][f];
                cLoaded = cIt;
              }
              unsigned char* dst = sm + OFF_CONS + sl * CONS_SLOT;
              mbar_expect_tx(&consFull[sl], 5 * CONS_BOX_BYTES + TYPE_BOX_BYTES);
              for (int f = 0; f < 5; ++f)
                tma_load3(dst + size_t(f) * FS * 8, &cMaps[MAP_CONS + cPhys[f] * 5 + f], w.k0 - 1, w.j0 - 1, cP,
                          &consFull[sl]);
              tma_load3(dst + TYPE_OFF, &cMaps[MAP_TYPE], w.k0 - 1, w.j0 - 1, cP, &consFull[sl]);
              ++cq;
              if (++cP > w.i1 + 1) {
                cIt = next_item(cIt + 1);
                if (cIt < itEnd) cP = items[cIt].i0 - 1;
              }
              progressed = true;
            }
          }
          if (eIt < itEnd) {
            const uint32_t se = eq % NE;
            if (eq < NE || mbar_try(&epiEmpty[se], ((eq / NE) - 1) & 1)) {
              const StageItem w = items[eIt];
              if (eLoaded != eIt) {
                const Grid& G = grid_of(w);
                const StepCtl& ctl = ctl_of(G);
                eMaps = static_cast<const CUtensorMap*>(G.tmaps);
                for (int f = 0; f < 5; ++f) ePhys[f] = ctl.u0Phys[f];
                eLoaded = eIt;
              }
              unsigned char* dst = sm + OFF_EPI + se * EPI_SLOT;
              mbar_expect_tx(&epiFull[se], epiFields * EPI_BOX_BYTES);
              for (int f = 0; f < 5; ++f)
                tma_load3(dst + size_t(f) * EFS * 8, &eMaps[MAP_EPI + ePhys[f] * 5 + f], w.k0 - 1, w.j0, eP,
                          &epiFull[se]);
              if (s > 0)
                for (int f = 0; f < 5; ++f)
                  tma_load3(dst + size_t(5 + f) * EFS * 8, &eMaps[MAP_ACC + f], w.k0 - 1, w.j0, eP, &epiFull[se]);
              ++eq;
              if (++eP > w.i1) {
                eIt = next_item(eIt + 1);
                if (eIt < itEnd) eP = items[eIt].i0;
              }
              progressed = true;
            }
          }
          if (progressed) {
            idle = 0;
          } else if (++idle > *lim) {
            fail(grid_of(items[cIt < itEnd ? cIt : eIt]));
            break;
          }
        }
        // Every copy issued must have landed before the CTA exits: wait for the last phase of each slot.
        const volatile int never = 0;
        const Grid& Gf = ENS ? grids[0] : G0;  // where a failed drain is reported
        for (uint32_t sl = 0; sl < NC; ++sl)
          if (cq > sl) {
            const uint32_t last = cq - 1 - ((cq - 1 - sl) % NC);
            if (!mbar_wait(&consFull[sl], (last / NC) & 1, &never, lim)) atomicExch(&Gf.ctl->timeout, 1);
          }
        for (uint32_t se = 0; se < NE; ++se)
          if (eq > se) {
            const uint32_t last = eq - 1 - ((eq - 1 - se) % NE);
            if (!mbar_wait(&epiFull[se], (last / NE) & 1, &never, lim)) atomicExch(&Gf.ctl->timeout, 1);
          }
      }
    } else {
      // ------------------------------------------------------------------ staging (warps 1-3)
      const int st = tid - 32;
      uint32_t q = 0;  // staged-plane sequence number, continues across items
      bool ok = true;
      for (int it = itBegin; it < itEnd && ok; ++it) {
        const StageItem w = items[it];
        if (skip(w)) continue;
        const Grid& G = grid_of(w);
        const ThermoConsts C{G.C.gamma, G.C.gm1, G.C.sc1, G.C.re, G.C.pf};
        const double* __restrict__ fpre = G.fpre;
        const long long sIs = G.sI, sJs = G.sJ;
        for (int p = w.i0 - 1; p <= w.i1 + 1; ++p, ++q) {
          const uint32_t sl = q % NC, ps = q % NP;
          if (q >= NP) ok = mbar_wait(&primEmpty[ps], ((q / NP) - 1) & 1, abortFlag, lim);
          ok = ok && mbar_wait(&consFull[sl], (q / NC) & 1, abortFlag, lim);
          if (!ok) {
            fail(G);
            break;
          }
          const double* cs = reinterpret_cast<const double*>(sm + OFF_CONS + sl * CONS_SLOT);
          const uint8_t* ts = reinterpret_cast<const uint8_t*>(cs) + TYPE_OFF;
          double* pv = reinterpret_cast<double*>(sm + OFF_PRIM + ps * PRIM_SLOT);
          // Two nodes per pass (idx and idx + NSTAGE) so that their long dependency chains (reciprocal,
          // square root, division) overlap. Nodes past the mesh read TMA zero fill: finite values that
          // are never used. Slots past the plane (idx >= HP) compute a dummy node and store nothing.
#pragma unroll 1
          for (int idx = st; idx < HP; idx += 2 * NSTAGE) {
            const int idy = idx + NSTAGE, idyc = idy < HP ? idy : idx;
            double rho[2] = {cs[0 * FS + idx], cs[0 * FS + idyc]}, rE[2] = {cs[4 * FS + idx], cs[4 * FS + idyc]};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int id = h ? idyc : idx;
              const int hj = id / HK, hk = id - hj * HK;
              if (ts[hj * TYW + hk] & FILTER_BIT) {
                const long long n = (long long)p * sIs + (long long)(w.j0 - 1 + hj) * sJs + (w.k0 - 1 + hk);
                const int f = __ldg(G.fidx + n);
                rho[h] = fpre[2 * f];
                rE[h] = fpre[2 * f + 1];
              }
            }
            const Prim a0 = prims_of_nr(C, rho[0], cs[1 * FS + idx], cs[2 * FS + idx], cs[3 * FS + idx], rE[0]);
            const Prim a1 = prims_of_nr(C, rho[1], cs[1 * FS + idyc], cs[2 * FS + idyc], cs[3 * FS + idyc], rE[1]);
            pv[0 * FS + idx] = a0.u;
            pv[1 * FS + idx] = a0.v;
            pv[2 * FS + idx] = a0.w;
            pv[3 * FS + idx] = a0.p;
            pv[4 * FS + idx] = a0.T;
            pv[5 * FS + idx] = a0.mu;
            if (idy < HP) {
              pv[0 * FS + idy] = a1.u;
              pv[1 * FS + idy] = a1.v;
              pv[2 * FS + idy] = a1.w;
              pv[3 * FS + idy] = a1.p;
              pv[4 * FS + idy] = a1.T;
              pv[5 * FS + idy] = a1.mu;
            }
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&primFull[ps]);
        }
      }
    }
  } else {
    reg_alloc<(ENS && MODE == 2) ? REG_HIGH_ENS4 : REG_HIGH>();
    // -------------------------------------------------------------------- columns (warpgroups 1-2)
    const int ct = tid - 128, tx = ct % TK, ty = ct / TK;
    const int cidx = (ty + 1) * HK + (tx + 1);   // this column's node in a staged plane
    const int eidx = ty * HK + tx + 1;           // ... in an epilogue tile
    const int tcix = (ty + 1) * TYW + (tx + 1);  // ... in a staged type box
    const unsigned char* const consBase = sm + OFF_CONS;
    const unsigned char* const primBase = sm + OFF_PRIM;
    uint32_t q = 0, e = 0;  // staged-plane and computed-plane sequence numbers
    bool ok = true;
    for (int it = itBegin; it < itEnd && ok; ++it) {
      const StageItem w = items[it];
      if (skip(w)) continue;
      const Grid& G = grid_of(w);
      const StepCtl& ctl = ctl_of(G);
      Consts* const myC = reinterpret_cast<Consts*>(sm + OFF_CSM + (warp - 4) * CSM_BYTES);
      ItemSm* const myI = reinterpret_cast<ItemSm*>(sm + OFF_CSM + (warp - 4) * CSM_BYTES + TL::CONSTS_BYTES);
      const double dtUsed = ctl.dtUsed;
      if constexpr (ENS) {  // this warp's copy of the member's coefficients (shared-memory operands)
        __syncwarp();
        const double* src = reinterpret_cast<const double*>(&G.C);
        double* dst = reinterpret_cast<double*>(myC);
        for (int q = lane; q < int(sizeof(Consts) / 8); q += 32) dst[q] = src[q];
        if (lane == 0) {
          for (int f = 0; f < 5; ++f) myI->out[f] = ctl.O[s][f];
          myI->acc = G.acc[0];
          myI->N = G.N;
          myI->sI = G.sI;
          myI->inc = (s == 2) ? dtUsed : dtUsed / 2;
          myI->dtFactor = dtUsed / 6;
        }
        __syncwarp();
      }
      const Consts& C = ENS ? *myC : G.C;
      // single grid: registers; ensemble: shared-memory loads at each use
      const long long sIR = G.sI, NdR = G.N;
      const double incR = (s == 2) ? dtUsed : dtUsed / 2, dtFactorR = dtUsed / 6;
      double* const outR[5] = {ctl.O[s][0], ctl.O[s][1], ctl.O[s][2], ctl.O[s][3], ctl.O[s][4]};
      double* const accR = G.acc[0];
      const volatile ItemSm* const vI = myI;
      auto outp = [&](int f) -> double* {
        if constexpr (ENS) return vI->out[f];
        else return outR[f];
      };
      auto accp = [&]() -> double* {
        if constexpr (ENS) return vI->acc;
        else return accR;
      };
      auto nodes = [&]() -> long long {
        if constexpr (ENS) return vI->N;
        else return NdR;
      };
      auto planeStride = [&]() -> long long {
        if constexpr (ENS) return vI->sI;
        else return sIR;
      };
      auto incf = [&]() -> double {
        if constexpr (ENS) return vI->inc;
        else return incR;
      };
      auto dtFactorf = [&]() -> double {
        if constexpr (ENS) return vI->dtFactor;
        else return dtFactorR;
      };
      const int j = w.j0 + ty, k = w.k0 + tx;
      const bool inTile = (j <= G.NJ - 2) && (k <= G.NK - 2);
      const int L = w.i1 - w.i0 + 1;
      long long nR = (long long)w.i0 * planeStride() + (long long)j * G.sJ + k;  // node of the next computed plane
      XNode gm1{}, gm2{};
      double fprev[5] = {0, 0, 0, 0, 0};
      XOwn ownPrev{};
      constexpr int oN = HK, oU = 1;
      // x-direction quantities of the column's node in staged plane slot (cX, pX): G of the node, and F of
      // the face towards the previous plane (a >= 1)
      auto x_part = [&](int cX, int pX, bool face, XOwn& ownCur, XNode& gcur, double (&fcur)[5]) {
        const double* cs = reinterpret_cast<const double*>(consBase + cX * CONS_SLOT);
        const double* ps = reinterpret_cast<const double*>(primBase + pX * PRIM_SLOT);
        ownCur = XOwn{ps[5 * FS + cidx], ps[0 * FS + cidx], ps[1 * FS + cidx], ps[2 * FS + cidx], ps[4 * FS + cidx]};
        gcur = x_node(C, cs[1 * FS + cidx], cs[2 * FS + cidx], cs[3 * FS + cidx], cs[4 * FS + cidx], ownCur.u,
                      ownCur.v, ownCur.w, ps[3 * FS + cidx], ownCur.mu,
                      ps[1 * FS + cidx + oN] - ps[1 * FS + cidx - oN], ps[0 * FS + cidx + oN] - ps[0 * FS + cidx - oN],
                      ps[2 * FS + cidx + oU] - ps[2 * FS + cidx - oU], ps[0 * FS + cidx + oU] - ps[0 * FS + cidx - oU]);
#pragma unroll
        for (int f = 0; f < 5; ++f) fcur[f] = 0.0;
        if (face) x_face(C, ownPrev, ownCur, fcur);
      };
      // Planes i0-1 and i0: their x quantities only.
      for (int a = 0; a < 2; ++a) {
        const uint32_t qx = q + a;
        const int pX = qx % NP, cX = qx % NC;
        ok = mbar_wait(&primFull[pX], (qx / NP) & 1, abortFlag, lim) &&
             mbar_wait(&consFull[cX], (qx / NC) & 1, abortFlag, lim);
        if (!ok) {
          fail(G);
          break;
        }
        XNode gcur;
        XOwn ownCur;
        double fcur[5];
        x_part(cX, pX, a >= 1, ownCur, gcur, fcur);
        if (a == 0) {  // plane i0-1: its conserved values have no other reader
          __syncwarp();
          if (lane == 0) mbar_arrive(&consEmpty[cX]);
        }
        gm2 = gm1;
        gm1 = gcur;
#pragma unroll
        for (int f = 0; f < 5; ++f) fprev[f] = fcur[f];
        ownPrev = ownCur;
      }
      // Iteration a forms the x quantities of plane X = i0-1+a and the RHS of plane P = i0-2+a. Every wait
      // comes first, so the x quantities of X and the y/z terms of P (independent until their final sum)
      // are one block of straight-line arithmetic the compiler can interleave.
      for (int a = 2; a <= L + 1 && ok; ++a) {
        const uint32_t qx = q + a;
        const int pX = qx % NP, cX = qx % NC;
        const uint32_t se = e % NE;
        ok = mbar_wait(&primFull[pX], (qx / NP) & 1, abortFlag, lim) &&
             mbar_wait(&consFull[cX], (qx / NC) & 1, abortFlag, lim);
        // (the ensemble variant, short of registers, waits for the epilogue tile after the x quantities)
        if constexpr (!ENS) ok = ok && mbar_wait(&epiFull[se], (e / NE) & 1, abortFlag, lim);
        if (!ok) {
          fail(G);
          break;
        }
        const int pR = (qx - 1) % NP, pW = (qx - 2) % NP, cR = (qx - 1) % NC;
        XNode gcur;
        XOwn ownCur;
        double fcur[5];
        x_part(cX, pX, true, ownCur, gcur, fcur);
        if constexpr (ENS) {
          if (!mbar_wait(&epiFull[se], (e / NE) & 1, abortFlag, lim)) {
            ok = false;
            fail(G);
            break;
          }
        }
        const double* cP = reinterpret_cast<const double*>(consBase + cR * CONS_SLOT);
        const uint8_t tc = (reinterpret_cast<const uint8_t*>(cP) + TYPE_OFF)[tcix];
        const bool valid = inTile && (tc & TYPE_MASK) == FLUID_INTERIOR;
        double kk5[5];
        yz_part<HK, FS>(C, cP, reinterpret_cast<const double*>(primBase + pW * PRIM_SLOT),
                        reinterpret_cast<const double*>(primBase + pR * PRIM_SLOT),
                        reinterpret_cast<const double*>(primBase + pX * PRIM_SLOT), cidx, ownPrev, kk5);
#pragma unroll
        for (int f = 0; f < 5; ++f) kk5[f] += (gcur.g[f] - gm2.g[f]) + (fcur[f] - fprev[f]);
        const double* ep = reinterpret_cast<const double*>(sm + OFF_EPI + se * EPI_SLOT);
        double u0[5], res[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) u0[f] = ep[f * EFS + eidx];
        if (MODE != 2 && s == 0) {
          const double inc = incf();
#pragma unroll
          for (int f = 0; f < 5; ++f) res[f] = u0[f] + inc * kk5[f];
          if (valid) {
            double* const accb = accp();
            const long long NdF = nodes();
#pragma unroll
            for (int f = 0; f < 5; ++f) accb[f * NdF + nR] = kk5[f];
          }
        } else if (MODE == 1 || (MODE == 0 && s < 3)) {
          const double inc = incf();
          double an[5];
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            an[f] = ep[(5 + f) * EFS + eidx] + 2 * kk5[f];
            res[f] = u0[f] + inc * kk5[f];
          }
          if (valid) {
            double* const accb = accp();
            const long long NdF = nodes();
#pragma unroll
            for (int f = 0; f < 5; ++f) accb[f * NdF + nR] = an[f];
          }
        } else {
          const double dtFactor = dtFactorf();
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
          if (valid && !filtered) dt_terms(C, res, dta);
        }
        if (valid) {
          double* const out0 = outp(0);
          double* const out1 = outp(1);
          double* const out2 = outp(2);
          double* const out3 = outp(3);
          double* const out4 = outp(4);
          out0[nR] = res[0];
          out1[nR] = res[1];
          out2[nR] = res[2];
          out3[nR] = res[3];
          out4[nR] = res[4];
          if (tc & (ZCOPY_UP_BIT | ZCOPY_DOWN_BIT)) {
            // periodic z faces: this node's copy (PeriodicBoundary, Boundary.cpp:344-367) lands in the
            // 32-byte sector just written; k = 1 feeds k = NK-1, k = NK-2 feeds k = 0. (Rows whose
            // source is a filter node stay with the edge kernel, which adds the copy's dt terms.)
            const long long m = (tc & ZCOPY_UP_BIT) ? nR + (G.NK - 2) : nR - (G.NK - 2);
            out0[m] = res[0];
            out1[m] = res[1];
            out2[m] = res[2];
            out3[m] = res[3];
            out4[m] = res[4];
          }
          if (tc & YCOPY_BIT) {
            // periodic y faces likewise: j = 1 feeds j = NJ-1, j = NJ-2 feeds j = 0 (a row of the tile's
            // neighbour across the grid; the whole warp's row when the tile spans k)
            const long long m = j == 1 ? nR + (long long)(G.NJ - 2) * G.sJ : nR - (long long)(G.NJ - 2) * G.sJ;
            out0[m] = res[0];
            out1[m] = res[1];
            out2[m] = res[2];
            out3[m] = res[3];
            out4[m] = res[4];
          }
        }
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&epiEmpty[se]);
          mbar_arrive(&consEmpty[cR]);   // plane i0-3+a: its last reader was this RHS
          mbar_arrive(&primEmpty[pW]);   // plane i0-4+a: read for the last time as the west plane
          if (a == L + 1) {  // the item's last two planes' primitives, its last plane's conserved values
            mbar_arrive(&consEmpty[cX]);
            mbar_arrive(&primEmpty[pR]);
            mbar_arrive(&primEmpty[pX]);
          }
        }
        ++e;
        nR += planeStride();
        gm2 = gm1;
        gm1 = gcur;
#pragma unroll
        for (int f = 0; f < 5; ++f) fprev[f] = fcur[f];
        ownPrev = ownCur;
      }
      q += L + 2;
      if (ENS && MODE != 1 && s == 3) {
        // an ensemble CTA moves between members: hand this item's dt maxima, change norms and NaN flag
        // to its member now (warp reductions, then one atomic per warp and quantity)
        const double mx[4] = {warp_max(dta.sx), warp_max(dta.sy), warp_max(dta.sz), warp_max(dta.nu)};
        double sm5[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) sm5[f] = warp_sum(nsum[f]);
        const bool anyBad = __any_sync(0xffffffffu, bad);
        if (lane == 0) {
          for (int qm = 0; qm < 4; ++qm) atomic_max_pos(&G.ctl->mx[qm], mx[qm]);
          for (int f = 0; f < 5; ++f) atomicAdd(&G.normPart[f], sm5[f]);
          if (anyBad) atomicOr(&G.ctl->nonFinite, 1);
        }
        dta = DtAcc{};
#pragma unroll
        for (int f = 0; f < 5; ++f) nsum[f] = 0;
        bad = 0;
      }
    }
  }
  __syncwarp();
  if (!ENS && MODE != 1 && s == 3) {
    flush_dt(G0.ctl, dta, red);
    flush_norms(G0.normPart + 5 * blockIdx.x, nsum, red);
    if (bad) atomicOr(&G0.ctl->nonFinite, 1);
  }
}

// Kernel variants (tile shapes), selected per solver (see StageTile in nsf_device.cuh).
namespace {
struct VariantInfo {
  int tk, tj, threads, typeBoxW;
  size_t smem;
  const void* fn[2];     // single grid: stages 1-3 (mode 0), stage 4 (mode 2)
  const void* fnEns[2];  // ensemble: stages 1-3 (mode 1), stage 4 (mode 2)
};
template <int TK, int TJ>
VariantInfo variant_info() {
  using TL = ws::Tile<TK, TJ>;
  return VariantInfo{TK,
                     TJ,
                     TL::NTHREADS,
                     TL::TYW,
                     TL::SMEM,
                     {reinterpret_cast<const void*>(&k_stage_ws<TK, TJ, false, 0>),
                      reinterpret_cast<const void*>(&k_stage_ws<TK, TJ, false, 2>)},
                     {reinterpret_cast<const void*>(&k_stage_ws<TK, TJ, true, 1>),
                      reinterpret_cast<const void*>(&k_stage_ws<TK, TJ, true, 2>)}};
}
VariantInfo info(int v) { return v == STAGE_TILE_16x16 ? variant_info<16, 16>() : variant_info<32, 8>(); }

template <int TK, int TJ, bool ENS>
void launch_variant(const Grid& hg, const Grid* dGrids, const LaunchPlan& L, int s, cudaStream_t st) {
  using TL = ws::Tile<TK, TJ>;
  constexpr int early = ENS ? 1 : 0;  // the instantiation of stages 1-3
  if (s == 3)
    k_stage_ws<TK, TJ, ENS, 2><<<L.stageBlocks, TL::NTHREADS, TL::SMEM, st>>>(hg, dGrids, L.items, L.ctaStart, s);
  else
    k_stage_ws<TK, TJ, ENS, early><<<L.stageBlocks, TL::NTHREADS, TL::SMEM, st>>>(hg, dGrids, L.items, L.ctaStart, s);
}
}  // namespace

size_t stage_smem_bytes(int v) { return info(v).smem; }
int stage_configure(int v) {
  const VariantInfo vi = info(v);
  cudaError_t e = cudaSuccess;
  for (const void* fn : {vi.fn[0], vi.fn[1], vi.fnEns[0], vi.fnEns[1]})
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(vi.smem));
  return int(e);
}
int stage_tile_j(int v) { return info(v).tj; }
int stage_tile_k(int v) { return info(v).tk; }
int stage_type_box_width(int v) { return info(v).typeBoxW; }
int stage_threads(int v) { return info(v).threads; }
int stage_occupancy(int v) {
  const VariantInfo vi = info(v);
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, vi.fn[1], vi.threads, vi.smem);
  return nb;
}
int stage_num_maps() { return ws::NMAPS; }
// Registers per thread the kernels are launched with (the setmaxnreg split assumes ws::REG_LAUNCH); the
// smallest over the instantiations.
int stage_launch_registers(int v) {
  const VariantInfo vi = info(v);
  int r = 1 << 30;
  for (const void* fn : {vi.fn[0], vi.fn[1], vi.fnEns[0], vi.fnEns[1]}) {
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, fn) != cudaSuccess) return -1;
    r = a.numRegs < r ? a.numRegs : r;
  }
  return r;
}
bool stage_register_split_ok(int v) {
  const int r = stage_launch_registers(v);
  const int need = std::max(128 * ws::REG_LOW + 256 * ws::REG_HIGH, 128 * ws::REG_LOW_ENS4 + 256 * ws::REG_HIGH_ENS4);
  return r > 0 && need <= info(v).threads * r;
}
void launch_stage(const Grid& hg, const LaunchPlan& L, int s, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!hg.tmaps || !hg.ctl || !L.items || !L.ctaStart) return;  // never launch on an unbuilt grid
  if (L.tile == STAGE_TILE_16x16)
    launch_variant<16, 16, false>(hg, nullptr, L, s, st);
  else
    launch_variant<32, 8, false>(hg, nullptr, L, s, st);
}
void launch_stage_ensemble(const Grid* dGrids, const LaunchPlan& L, int s, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!dGrids || !L.items || !L.ctaStart) return;
  const Grid none{};
  if (L.tile == STAGE_TILE_16x16)
    launch_variant<16, 16, true>(none, dGrids, L, s, st);
  else
    launch_variant<32, 8, true>(none, dGrids, L, s, st);
}

}  // namespace nsf
