// Device helpers shared by the kernels: thermodynamics (primitive values from conserved values and
// back), dt-limit terms, block reductions, and the right-hand side of the reference's five flux loops.
#ifndef NSF_PHYSICS_CUH
#define NSF_PHYSICS_CUH

#include "nsf_device.cuh"

namespace nsf {

// ----------------------------------------------------------------------------------------------
// Thermodynamics (updatePrimitiveVariables, Solver.cpp:446-479; derive*, FlowVariableGroupStructs.h).
// pow(1+T, 1.5) is evaluated as x*sqrt(x); the three divisions by (1+rho) share one reciprocal.
// Both differ from the reference by rounding only.
struct Prim {
  double u, v, w, p, T, mu, ka;
};

// The constants prims_of reads, small enough to keep in registers.
struct ThermoConsts {
  double gamma, gm1, sc1, re, pf;
};

// CT: Consts, or any struct with the members gamma, gm1, sc1, re and pf (ThermoConsts).
template <class CT>
__device__ __forceinline__ Prim prims_of(const CT& C, double rho, double ru, double rv, double rw, double rE) {
  Prim q;
  const double r1 = 1.0 / (rho + 1.0);
  q.u = ru * r1;
  q.v = rv * r1;
  q.w = rw * r1;
  q.p = C.gm1 * (rE - (rho + 1.0) * 0.5 * (q.u * q.u + q.v * q.v + q.w * q.w));
  q.T = (C.gamma * q.p - rho) * r1;
  const double x = 1.0 + q.T;
  q.mu = x * sqrt(x) * C.sc1 / (C.re * (q.T + C.sc1));
  q.ka = q.mu * C.pf;
  return q;
}

// Reciprocal and square root by Newton-Raphson refinement of the hardware approximations
// (rcp.approx.ftz.f64, rsqrt.approx.ftz.f64): y <- y (2 - a y) and r <- r (3 - a r^2) / 2, each iteration
// doubling the correct bits, two of them from the approximation's ~20 bits, then one Heron correction of
// s = a r for the square root. Arguments are positive normal numbers here (1 + rho, 1 + T, and the
// viscosity denominator); results are within a couple of ulps of the correctly rounded ones.
__device__ __forceinline__ double recip_nr(double a) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  double e = fma(-a, y, 1.0);
  y = fma(y, e, y);
  e = fma(-a, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ double sqrt_nr(double a) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
  const double h = 0.5 * a;
  r = r * fma(-h * r, r, 1.5);
  r = r * fma(-h * r, r, 1.5);
  const double s = a * r;
  return fma(fma(-s, s, a), 0.5 * r, s);
}

// prims_of with the Newton-Raphson reciprocal and square root (the stage kernel's staging warps, where
// the IEEE division and square root sequences are the longest dependency chains of a plane).
template <class CT>
__device__ __forceinline__ Prim prims_of_nr(const CT& C, double rho, double ru, double rv, double rw, double rE) {
  Prim q;
  const double r1 = recip_nr(rho + 1.0);
  q.u = ru * r1;
  q.v = rv * r1;
  q.w = rw * r1;
  q.p = C.gm1 * (rE - (rho + 1.0) * 0.5 * (q.u * q.u + q.v * q.v + q.w * q.w));
  q.T = (C.gamma * q.p - rho) * r1;
  const double x = 1.0 + q.T;
  q.mu = x * sqrt_nr(x) * C.sc1 * recip_nr(C.re * (q.T + C.sc1));
  q.ka = q.mu * C.pf;
  return q;
}

__device__ __forceinline__ double mu_of_T(const Consts& C, double T) {
  const double x = 1.0 + T;
  return x * sqrt(x) * C.sc1 / (C.re * (T + C.sc1));
}

// Conserved values from primitive values (deriveConservedVariables, FlowVariableGroupStructs.h:152-161).
__device__ __forceinline__ void cons_of(const Consts& C, double u, double v, double w, double p, double T,
                                        double out[5]) {
  const double rho = (C.gamma * p - T) / (1.0 + T);
  out[0] = rho;
  out[1] = (1.0 + rho) * u;
  out[2] = (1.0 + rho) * v;
  out[3] = (1.0 + rho) * w;
  out[4] = p / C.gm1 + (1.0 + rho) * 0.5 * (u * u + v * v + w * w);
}

// Non-negative doubles compare like their bit patterns, so maxima reduce with integer atomicMax.
__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  if (v > 0) atomicMax(a, static_cast<unsigned long long>(__double_as_longlong(v)));
}

struct DtAcc {
  double sx = 0, sy = 0, sz = 0, nu = 0;
  __device__ __forceinline__ void add(const Consts& C, double rho, double u, double v, double w, double p, double mu) {
    // getInviscidTimeStepLimit / getViscousTimeStepLimit terms, Solver.cpp:100-122
    const double c = sqrt((1.0 + C.gamma * p) / (1.0 + rho));
    sx = fmax(sx, c + fabs(u));
    sy = fmax(sy, c + fabs(v));
    sz = fmax(sz, c + fabs(w));
    nu = fmax(nu, mu / (rho + 1.0) * C.vmod);
  }
};

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Linear thread index and thread count of the block (1-D or 2-D blocks).
__device__ __forceinline__ int block_tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ __forceinline__ int block_threads() { return blockDim.x * blockDim.y * blockDim.z; }

// Block-wide reduction of the four dt maxima into ctl->mx (order independent). Thread count % 32 == 0.
__device__ inline void flush_dt(StepCtl* ctl, DtAcc a, double* scratch /*[4*32]*/) {
  const int tid = block_tid(), lane = tid & 31, wid = tid >> 5, nw = block_threads() >> 5;
  double v[4] = {warp_max(a.sx), warp_max(a.sy), warp_max(a.sz), warp_max(a.nu)};
  __syncthreads();
  if (lane == 0)
    for (int q = 0; q < 4; ++q) scratch[q * 32 + wid] = v[q];
  __syncthreads();
  if (wid == 0) {
    for (int q = 0; q < 4; ++q) {
      double m = lane < nw ? scratch[q * 32 + lane] : 0.0;
      m = warp_max(m);
      if (lane == 0) atomic_max_pos(&ctl->mx[q], m);
    }
  }
  __syncthreads();
}

// Block-wide sums of the five change-norm partials into a per-block slot (fixed order: deterministic).
__device__ inline void flush_norms(double* slot, const double s[5], double* scratch /*[5*32]*/) {
  const int tid = block_tid(), lane = tid & 31, wid = tid >> 5, nw = block_threads() >> 5;
  double v[5];
  for (int q = 0; q < 5; ++q) v[q] = warp_sum(s[q]);
  __syncthreads();
  if (lane == 0)
    for (int q = 0; q < 5; ++q) scratch[q * 32 + wid] = v[q];
  __syncthreads();
  if (wid == 0)
    for (int q = 0; q < 5; ++q) {
      double m = lane < nw ? scratch[q * 32 + lane] : 0.0;
      m = warp_sum(m);
      if (lane == 0) slot[q] = m;
    }
  __syncthreads();
}


// Bounded grid barrier over nb blocks on a 64-bit arrival counter that only grows: every barrier instance
// takes exactly nb arrivals, so an arrival that reads `old` belongs to instance old / nb and waits until
// the counter reaches (old / nb + 1) * nb (release on arrival, acquire on the poll). A wait longer than
// kBarrierPolls polls sets *timeout (a StepCtl::timeout) and goes on: the run is then reported invalid,
// nothing hangs.
constexpr long long kBarrierPolls = 1ll << 24;
__device__ __forceinline__ unsigned long long atom_add_release(unsigned long long* a, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.release.gpu.u64 %0, [%1], %2;" : "=l"(old) : "l"(a), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* a) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
  return v;
}
__device__ inline void grid_barrier(unsigned long long* S, unsigned nb, int* timeout) {
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {  // one arrival per block, any block shape
    const unsigned long long old = atom_add_release(S, 1ull);
    const unsigned long long target = (old / nb + 1) * nb;
    long long it = 0;
    while (ld_acquire(S) < target) {
      if (++it > kBarrierPolls) {
        atomicExch(timeout, 1);
        break;
      }
      __nanosleep(32);
    }
    __threadfence();  // the block's later loads see what the other blocks wrote before they arrived
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------------------
// Right-hand side of the five flux loops (continuity Solver.cpp:181-196, x/y/z momentum :199-339, energy
// :342-418) split by direction, for kernels that stream along i and keep the thread's own (j, k) column in
// registers. For the x direction the reference's terms are differences of
// per-node quantities and of per-face quantities along the column:
//   x-part(P) = [G(E) - G(W)] + [F(P,E) - F(W,P)]
// with G the convective/inviscid flux and the mixed-derivative products of a node, and F the normal
// viscous and heat-flux products of an x-face, e.g. for x-momentum
//   G = ax (rho_u u + p) + xm_yx mu (v_N - v_S) + xm_zx mu (w_U - w_D),   F = xm_xx (mu_a + mu_b)(u_b - u_a).
// F(W,P) is the reference's (mu_W + mu_P)(u_P - u_W) (addition commutes); G differences regroup the
// reference's sums and differ from it by rounding only. Here and in yz_part the energy equation's mixed
// terms reuse the momentum equations' products (mu_N u_N (v_EN - v_WN) is formed as u_N [mu_N (v_EN - v_WN)])
// and the heat flux (kappa_a + kappa_b)(T_b - T_a) is formed as pf (mu_a + mu_b)(T_b - T_a), kappa = pf mu:
// the same sums, rounded differently.
struct XNode {  // G of one node for the five equations
  double g[5];
};
struct XOwn {  // a node's values that the next x-face needs
  double mu, u, v, w, T;
};

// G at one node. own: rho_u, rho_v, rho_w, rho_E, u, v, w, p, mu; d*: in-plane differences at the node
// (v_N - v_S, u_N - u_S, w_U - w_D, u_U - u_D).
// x_node and x_face spell out every rounding (__dmul_rn, __dadd_rn, __fma_rn are never contracted or
// reordered by the compiler): the stage kernel evaluates them in two places (the first planes of a work item
// and its main loop), and a plane's G and F must come out bit for bit the same in either, whatever the
// i-planes a work item covers (a grid run whole or in x-slabs gives identical values).
__device__ __forceinline__ XNode x_node(const Consts& C, double ru, double rv, double rw, double rE, double u,
                                        double v, double w, double p, double mu, double dyv, double dyu, double dzw,
                                        double dzu) {
  XNode n;
  const double myv = __dmul_rn(mu, dyv), mzw = __dmul_rn(mu, dzw), myu = __dmul_rn(mu, dyu), mzu = __dmul_rn(mu, dzu);
  n.g[0] = __dmul_rn(C.ax, ru);
  n.g[1] = __fma_rn(C.xm_zx, mzw, __fma_rn(C.xm_yx, myv, __dmul_rn(C.ax, __fma_rn(ru, u, p))));
  n.g[2] = __fma_rn(C.ym_yx, myu, __dmul_rn(C.ax, __dmul_rn(rv, u)));
  n.g[3] = __fma_rn(C.zm_zx, mzu, __dmul_rn(C.ax, __dmul_rn(rw, u)));
  const double h = __dmul_rn(__dadd_rn(__dadd_rn(C.h0, rE), p), u);
  double e4 = __dmul_rn(C.ax, h);
  e4 = __fma_rn(C.e_yx6, __dmul_rn(u, myv), e4);
  e4 = __fma_rn(C.e_zx6, __dmul_rn(u, mzw), e4);
  e4 = __fma_rn(C.e_yx4, __dmul_rn(v, myu), e4);
  n.g[4] = __fma_rn(C.e_zx4, __dmul_rn(w, mzu), e4);
  return n;
}

// F of the x-face between a (lower i) and b.
__device__ __forceinline__ void x_face(const Consts& C, const XOwn& a, const XOwn& b, double f[5]) {
  const double ms = __dadd_rn(a.mu, b.mu);
  const double du = __dsub_rn(b.u, a.u), dv = __dsub_rn(b.v, a.v), dw = __dsub_rn(b.w, a.w);
  f[0] = 0.0;
  f[1] = __dmul_rn(C.xm_xx, __dmul_rn(ms, du));
  f[2] = __dmul_rn(C.ym_xx, __dmul_rn(ms, dv));
  f[3] = __dmul_rn(C.zm_xx, __dmul_rn(ms, dw));
  const double su = __fma_rn(a.mu, a.u, __dmul_rn(b.mu, b.u));
  const double sv = __fma_rn(a.mu, a.v, __dmul_rn(b.mu, b.v));
  const double sw = __fma_rn(a.mu, a.w, __dmul_rn(b.mu, b.w));
  double e4 = __dmul_rn(C.e_xx23, __dmul_rn(su, du));
  e4 = __fma_rn(C.e_xx12, __dmul_rn(sv, dv), e4);
  e4 = __fma_rn(C.e_xx12, __dmul_rn(sw, dw), e4);
  f[4] = __fma_rn(C.e_xx12, __dmul_rn(C.pf, __dmul_rn(ms, __dsub_rn(b.T, a.T))), e4);
}

// y- and z-direction part of the right-hand side at P (the reference's terms not covered by G and F).
// cP/pP: staged centre plane; pE/pW: staged neighbour planes (only their N/S/U/D velocity values are
// read, for the mixed x-derivatives at the in-plane neighbours); own: P's own values. The staged planes
// hold u, v, w, p, T, mu (fields 0..5); kappa = pf mu is formed here, as prims_of forms it.
template <int HK, int FS>
__device__ __forceinline__ void yz_part(const Consts& C, const double* __restrict__ cP, const double* __restrict__ pW,
                                        const double* __restrict__ pP, const double* __restrict__ pE, int c,
                                        const XOwn& own, double out[5]) {
  enum { RU = 1, RV = 2, RW = 3, RE = 4 };
  enum { U = 0, V = 1, W = 2, P = 3, TT = 4, MU = 5 };
#define F_(b, v, o) (b)[(v)*FS + c + (o)]
  constexpr int oN = HK, oS = -HK, oU = 1, oD = -1;
  const double muP = own.mu, uP = own.u, vP = own.v, wP = own.w, TP = own.T;
  const double muN = F_(pP, MU, oN), muS = F_(pP, MU, oS), muU = F_(pP, MU, oU), muD = F_(pP, MU, oD);
  const double uN = F_(pP, U, oN), uS = F_(pP, U, oS), uU = F_(pP, U, oU), uD = F_(pP, U, oD);
  const double vN = F_(pP, V, oN), vS = F_(pP, V, oS), vU = F_(pP, V, oU), vD = F_(pP, V, oD);
  const double wN = F_(pP, W, oN), wS = F_(pP, W, oS), wU = F_(pP, W, oU), wD = F_(pP, W, oD);
  const double pN = F_(pP, P, oN), pS = F_(pP, P, oS), pU = F_(pP, P, oU), pD = F_(pP, P, oD);
  // face viscosity sums (mu_N + mu_P) ... of the normal viscous and heat-flux terms
  const double msN = muN + muP, msS = muS + muP, msU = muU + muP, msD = muD + muP;
  // mixed-derivative products mu_X (difference across X), shared by momentum and energy
  const double mNdxv = muN * (F_(pE, V, oN) - F_(pW, V, oN)), mSdxv = muS * (F_(pE, V, oS) - F_(pW, V, oS));
  const double mNdxu = muN * (F_(pE, U, oN) - F_(pW, U, oN)), mSdxu = muS * (F_(pE, U, oS) - F_(pW, U, oS));
  const double mUdxw = muU * (F_(pE, W, oU) - F_(pW, W, oU)), mDdxw = muD * (F_(pE, W, oD) - F_(pW, W, oD));
  const double mUdxu = muU * (F_(pE, U, oU) - F_(pW, U, oU)), mDdxu = muD * (F_(pE, U, oD) - F_(pW, U, oD));
  const double wNU = F_(pP, W, oN + oU), wND = F_(pP, W, oN + oD), wSU = F_(pP, W, oS + oU), wSD = F_(pP, W, oS + oD);
  const double vNU = F_(pP, V, oN + oU), vND = F_(pP, V, oN + oD), vSU = F_(pP, V, oS + oU), vSD = F_(pP, V, oS + oD);
  const double mNdzw = muN * (wNU - wND), mSdzw = muS * (wSU - wSD);  // w_U - w_D at N, S
  const double mUdyw = muU * (wNU - wSU), mDdyw = muD * (wND - wSD);  // w_N - w_S at U, D
  const double mNdzv = muN * (vNU - vND), mSdzv = muS * (vSU - vSD);  // v_U - v_D at N, S
  const double mUdyv = muU * (vNU - vSU), mDdyv = muD * (vND - vSD);  // v_N - v_S at U, D
  out[0] = C.ay * (F_(cP, RV, oN) - F_(cP, RV, oS)) + C.az * (F_(cP, RW, oU) - F_(cP, RW, oD));
  {
    const double ruN = F_(cP, RU, oN), ruS = F_(cP, RU, oS), ruU = F_(cP, RU, oU), ruD = F_(cP, RU, oD);
    const double cY = C.ay * (ruN * vN - ruS * vS);
    const double cZ = C.az * (ruU * wU - ruD * wD);
    const double vYY = C.xm_yy * (msN * (uN - uP) - msS * (uP - uS));
    const double vZZ = C.xm_zz * (msU * (uU - uP) - msD * (uP - uD));
    const double vXY = C.xm_xy * (mNdxv - mSdxv);
    const double vXZ = C.xm_xz * (mUdxw - mDdxw);
    out[1] = cY + cZ + vYY + vZZ + vXY + vXZ;
  }
  {
    const double rvN = F_(cP, RV, oN), rvS = F_(cP, RV, oS), rvU = F_(cP, RV, oU), rvD = F_(cP, RV, oD);
    const double cY = C.ay * (rvN * vN + pN - rvS * vS - pS);
    const double cZ = C.az * (rvU * wU - rvD * wD);
    const double vYY = C.ym_yy * (msN * (vN - vP) - msS * (vP - vS));
    const double vZZ = C.ym_zz * (msU * (vU - vP) - msD * (vP - vD));
    const double vXY = C.ym_xy * (mNdxu - mSdxu);
    const double vYZ = C.ym_yz * (mUdyw - mDdyw);
    const double vZY = C.ym_zy * (mNdzw - mSdzw);
    out[2] = cY + cZ + vYY + vZZ + vXY + vYZ + vZY;
  }
  {
    const double rwN = F_(cP, RW, oN), rwS = F_(cP, RW, oS), rwU = F_(cP, RW, oU), rwD = F_(cP, RW, oD);
    const double cY = C.ay * (rwN * vN - rwS * vS);
    const double cZ = C.az * (rwU * wU + pU - rwD * wD - pD);
    const double vYY = C.zm_yy * (msN * (wN - wP) - msS * (wP - wS));
    const double vZZ = C.zm_zz * (msU * (wU - wP) - msD * (wP - wD));
    const double vXZ = C.zm_xz * (mUdxu - mDdxu);
    const double vZY = C.zm_zy * (mNdzv - mSdzv);
    const double vYZ = C.zm_yz * (mUdyv - mDdyv);
    out[3] = cY + cZ + vYY + vZZ + vXZ + vZY + vYZ;
  }
  {
    const double H0 = C.h0;
    const double EN = F_(cP, RE, oN), ES = F_(cP, RE, oS), EU = F_(cP, RE, oU), ED = F_(cP, RE, oD);
    const double inv = C.ay * ((H0 + EN + pN) * vN - (H0 + ES + pS) * vS) + C.az * ((H0 + EU + pU) * wU - (H0 + ED + pD) * wD);
    const double vfY = C.e_yy12 * ((muN * uN + muP * uP) * (uN - uP) - (muS * uS + muP * uP) * (uP - uS)) +
                       C.e_yy23 * ((muN * vN + muP * vP) * (vN - vP) - (muS * vS + muP * vP) * (vP - vS)) +
                       C.e_yy12 * ((muN * wN + muP * wP) * (wN - wP) - (muS * wS + muP * wP) * (wP - wS)) +
                       C.e_yx6 * (vN * mNdxu - vS * mSdxu) + C.e_zy6 * (vN * mNdzw - vS * mSdzw) +
                       C.e_yx4 * (uN * mNdxv - uS * mSdxv) + C.e_zy4 * (wN * mNdzv - wS * mSdzv);
    const double vfZ = C.e_zz12 * ((muU * uU + muP * uP) * (uU - uP) - (muD * uD + muP * uP) * (uP - uD)) +
                       C.e_zz12 * ((muU * vU + muP * vP) * (vU - vP) - (muD * vD + muP * vP) * (vP - vD)) +
                       C.e_zz23 * ((muU * wU + muP * wP) * (wU - wP) - (muD * wD + muP * wP) * (wP - wD)) +
                       C.e_zx6 * (wU * mUdxu - wD * mDdxu) + C.e_zy6 * (wU * mUdyv - wD * mDdyv) +
                       C.e_zx4 * (uU * mUdxw - uD * mDdxw) + C.e_zy4 * (vU * mUdyw - vD * mDdyw);
    const double hf = C.e_yy12 * (C.pf * (msN * (F_(pP, TT, oN) - TP) - msS * (TP - F_(pP, TT, oS)))) +
                      C.e_zz12 * (C.pf * (msU * (F_(pP, TT, oU) - TP) - msD * (TP - F_(pP, TT, oD))));
    out[4] = inv + vfY + vfZ + hf;
  }
#undef F_
}

}  // namespace nsf
#endif
