// Generated by gen_rhs_adjoint.py from the RHS term table: do not edit. The transposed stencil of the
// right-hand side (Solver.cpp:181-418) in gather form: rhs_adjoint_gather(...) returns, for node
// X = (i, j, k), the adjoint of each input quantity (RU, RV, RW, RE, u, v, w, p, T, mu, ka) summed over
// every interior node whose RHS reads it. lam(e, di, dj, dk): RHS adjoint of equation e at node
// (i+di, j+dj, k+dk) (zero where no RHS is taken); val(q, di, dj, dk): input quantity q there (offsets
// within one node of X: the 7-point stencil for u, v, w, T, mu, ka, X itself for the others);
// inner(di, dj, dk): the node (i-di, j-dj, k-dk) is one whose RHS was taken (its whole stencil then
// lies inside the grid). All offsets are literals, so a caller's index arithmetic folds. The terms of
// one RHS node are grouped by equation and, within an equation, by coefficient.
#ifndef NSF_RHS_ADJOINT_CUH
#define NSF_RHS_ADJOINT_CUH

namespace nsf {

template <class Lam, class Val, class Inner>
__device__ __forceinline__ void rhs_adjoint_gather(const Consts& C, const Lam& lam, const Val& val,
                                                   const Inner& inner, double bar[11]) {
  for (int q = 0; q < 11; ++q) bar[q] = 0.0;
  asm volatile("" ::: "memory");
  if (inner(0, 0, 0)) {
    const double l1 = lam(1, 0, 0, 0);
    const double l2 = lam(2, 0, 0, 0);
    const double l3 = lam(3, 0, 0, 0);
    const double l4 = lam(4, 0, 0, 0);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w1 = val(5, -1, 0, 0);  // v (-1, 0, 0)
    const double w2 = val(6, -1, 0, 0);  // w (-1, 0, 0)
    const double w3 = val(8, -1, 0, 0);  // T (-1, 0, 0)
    const double w4 = val(9, -1, 0, 0);  // mu (-1, 0, 0)
    const double w5 = val(10, -1, 0, 0);  // ka (-1, 0, 0)
    const double w6 = val(4, 0, -1, 0);  // u (0, -1, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w8 = val(6, 0, -1, 0);  // w (0, -1, 0)
    const double w9 = val(8, 0, -1, 0);  // T (0, -1, 0)
    const double w10 = val(9, 0, -1, 0);  // mu (0, -1, 0)
    const double w11 = val(10, 0, -1, 0);  // ka (0, -1, 0)
    const double w12 = val(4, 0, 0, -1);  // u (0, 0, -1)
    const double w13 = val(5, 0, 0, -1);  // v (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w15 = val(8, 0, 0, -1);  // T (0, 0, -1)
    const double w16 = val(9, 0, 0, -1);  // mu (0, 0, -1)
    const double w17 = val(10, 0, 0, -1);  // ka (0, 0, -1)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w29 = val(4, 0, 0, 1);  // u (0, 0, 1)
    const double w30 = val(5, 0, 0, 1);  // v (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w32 = val(8, 0, 0, 1);  // T (0, 0, 1)
    const double w33 = val(9, 0, 0, 1);  // mu (0, 0, 1)
    const double w34 = val(10, 0, 0, 1);  // ka (0, 0, 1)
    const double w35 = val(4, 0, 1, 0);  // u (0, 1, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w37 = val(6, 0, 1, 0);  // w (0, 1, 0)
    const double w38 = val(8, 0, 1, 0);  // T (0, 1, 0)
    const double w39 = val(9, 0, 1, 0);  // mu (0, 1, 0)
    const double w40 = val(10, 0, 1, 0);  // ka (0, 1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w42 = val(5, 1, 0, 0);  // v (1, 0, 0)
    const double w43 = val(6, 1, 0, 0);  // w (1, 0, 0)
    const double w44 = val(8, 1, 0, 0);  // T (1, 0, 0)
    const double w45 = val(9, 1, 0, 0);  // mu (1, 0, 0)
    const double w46 = val(10, 1, 0, 0);  // ka (1, 0, 0)
    bar[4] += l1 * ((-2.0 * C.xm_xx + -2.0 * C.xm_yy + -2.0 * C.xm_zz) * (w27) + -C.xm_xx * (w45 + w4) + -C.xm_yy * (w39 + w10) + -C.xm_zz * (w33 + w16)) + l4 * ((-2.0 * C.e_xx23 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * w22 * (w27 + w27) + -C.e_xx23 * (w45 * w41 + w4 * w0) + C.e_xx23 * w27 * (w41 + w0) + -C.e_yy12 * (w39 * w35 + w10 * w6) + C.e_yy12 * w27 * (w35 + w6) + -C.e_zz12 * (w33 * w29 + w16 * w12) + C.e_zz12 * w27 * (w29 + w12));  // u
    bar[5] += l2 * ((-2.0 * C.ym_xx + -2.0 * C.ym_yy + -2.0 * C.ym_zz) * (w27) + -C.ym_xx * (w45 + w4) + -C.ym_yy * (w39 + w10) + -C.ym_zz * (w33 + w16)) + l4 * ((-2.0 * C.e_xx12 + -2.0 * C.e_yy23 + -2.0 * C.e_zz12) * w23 * (w27 + w27) + -C.e_xx12 * (w45 * w42 + w4 * w1) + C.e_xx12 * w27 * (w42 + w1) + -C.e_yy23 * (w39 * w36 + w10 * w7) + C.e_yy23 * w27 * (w36 + w7) + -C.e_zz12 * (w33 * w30 + w16 * w13) + C.e_zz12 * w27 * (w30 + w13));  // v
    bar[6] += l3 * ((-2.0 * C.zm_xx + -2.0 * C.zm_yy + -2.0 * C.zm_zz) * (w27) + -C.zm_xx * (w45 + w4) + -C.zm_yy * (w39 + w10) + -C.zm_zz * (w33 + w16)) + l4 * ((-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz23) * w24 * (w27 + w27) + -C.e_xx12 * (w45 * w43 + w4 * w2) + C.e_xx12 * w27 * (w43 + w2) + -C.e_yy12 * (w39 * w37 + w10 * w8) + C.e_yy12 * w27 * (w37 + w8) + -C.e_zz23 * (w33 * w31 + w16 * w14) + C.e_zz23 * w27 * (w31 + w14));  // w
    bar[8] += l4 * ((-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * (w28) + -C.e_xx12 * (w46 + w5) + -C.e_yy12 * (w40 + w11) + -C.e_zz12 * (w34 + w17));  // T
    bar[9] += l1 * ((-2.0 * C.xm_xx + -2.0 * C.xm_yy + -2.0 * C.xm_zz) * (w22) + C.xm_xx * (w41 + w0) + C.xm_yy * (w35 + w6) + C.xm_zz * (w29 + w12)) + l2 * ((-2.0 * C.ym_xx + -2.0 * C.ym_yy + -2.0 * C.ym_zz) * (w23) + C.ym_xx * (w42 + w1) + C.ym_yy * (w36 + w7) + C.ym_zz * (w30 + w13)) + l3 * ((-2.0 * C.zm_xx + -2.0 * C.zm_yy + -2.0 * C.zm_zz) * (w24) + C.zm_xx * (w43 + w2) + C.zm_yy * (w37 + w8) + C.zm_zz * (w31 + w14)) + l4 * ((-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz23) * (w24 * w24) + (-2.0 * C.e_xx12 + -2.0 * C.e_yy23 + -2.0 * C.e_zz12) * (w23 * w23) + C.e_xx12 * (w23 * w42 + w1 * w23 + w24 * w43 + w2 * w24) + (-2.0 * C.e_xx23 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * (w22 * w22) + C.e_xx23 * w22 * (w41 + w0) + C.e_yy12 * (w22 * w35 + w6 * w22 + w24 * w37 + w8 * w24) + C.e_yy23 * w23 * (w36 + w7) + C.e_zz12 * (w22 * w29 + w12 * w22 + w23 * w30 + w13 * w23) + C.e_zz23 * w24 * (w31 + w14));  // mu
    bar[10] += l4 * ((-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * (w26) + C.e_xx12 * (w44 + w3) + C.e_yy12 * (w38 + w9) + C.e_zz12 * (w32 + w15));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(-1, 0, 0)) {
    const double l0 = lam(0, 1, 0, 0);
    const double l1 = lam(1, 1, 0, 0);
    const double l2 = lam(2, 1, 0, 0);
    const double l3 = lam(3, 1, 0, 0);
    const double l4 = lam(4, 1, 0, 0);
    const double w6 = val(4, 0, -1, 0);  // u (0, -1, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w12 = val(4, 0, 0, -1);  // u (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w18 = val(0, 0, 0, 0);  // RU (0, 0, 0)
    const double w19 = val(1, 0, 0, 0);  // RV (0, 0, 0)
    const double w20 = val(2, 0, 0, 0);  // RW (0, 0, 0)
    const double w21 = val(3, 0, 0, 0);  // RE (0, 0, 0)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w25 = val(7, 0, 0, 0);  // p (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w29 = val(4, 0, 0, 1);  // u (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w35 = val(4, 0, 1, 0);  // u (0, 1, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w42 = val(5, 1, 0, 0);  // v (1, 0, 0)
    const double w43 = val(6, 1, 0, 0);  // w (1, 0, 0)
    const double w44 = val(8, 1, 0, 0);  // T (1, 0, 0)
    const double w45 = val(9, 1, 0, 0);  // mu (1, 0, 0)
    const double w46 = val(10, 1, 0, 0);  // ka (1, 0, 0)
    bar[0] += l0 * -C.ax + l1 * -C.ax * (w22);  // RU
    bar[1] += l2 * -C.ax * (w22);  // RV
    bar[2] += l3 * -C.ax * (w22);  // RW
    bar[3] += l4 * -C.ax * (w22);  // RE
    bar[4] += l1 * (-C.ax * (w18) + C.xm_xx * (w27 + w45)) + l2 * -C.ax * (w19) + l3 * -C.ax * (w20) + l4 * (-C.ax * (w21 + w25) + -C.ax * C.h0 + -C.e_xx23 * (w27 * w41) + C.e_xx23 * (w27 * w22 + w27 * w22 + w45 * w41) + -C.e_yx6 * (w27 * w36) + C.e_yx6 * (w27 * w7) + -C.e_zx6 * (w27 * w31) + C.e_zx6 * (w27 * w14));  // u
    bar[5] += l2 * C.ym_xx * (w27 + w45) + l4 * (-C.e_xx12 * (w27 * w42) + C.e_xx12 * (w27 * w23 + w27 * w23 + w45 * w42) + -C.e_yx4 * (w27 * w35) + C.e_yx4 * (w27 * w6));  // v
    bar[6] += l3 * C.zm_xx * (w27 + w45) + l4 * (-C.e_xx12 * (w27 * w43) + C.e_xx12 * (w27 * w24 + w27 * w24 + w45 * w43) + -C.e_zx4 * (w27 * w29) + C.e_zx4 * (w27 * w12));  // w
    bar[7] += l1 * -C.ax + l4 * -C.ax * (w22);  // p
    bar[8] += l4 * C.e_xx12 * (w28 + w46);  // T
    bar[9] += l1 * (-C.xm_xx * (w41) + C.xm_xx * (w22) + -C.xm_yx * (w36) + C.xm_yx * (w7) + -C.xm_zx * (w31) + C.xm_zx * (w14)) + l2 * (-C.ym_xx * (w42) + C.ym_xx * (w23) + -C.ym_yx * (w35) + C.ym_yx * (w6)) + l3 * (-C.zm_xx * (w43) + C.zm_xx * (w24) + -C.zm_zx * (w29) + C.zm_zx * (w12)) + l4 * (-C.e_xx12 * (w23 * w42 + w24 * w43) + C.e_xx12 * (w23 * w23 + w24 * w24) + -C.e_xx23 * (w22 * w41) + C.e_xx23 * (w22 * w22) + -C.e_yx4 * (w35 * w23) + C.e_yx4 * (w6 * w23) + -C.e_yx6 * (w22 * w36) + C.e_yx6 * (w22 * w7) + -C.e_zx4 * (w29 * w24) + C.e_zx4 * (w12 * w24) + -C.e_zx6 * (w22 * w31) + C.e_zx6 * (w22 * w14));  // mu
    bar[10] += l4 * (-C.e_xx12 * (w44) + C.e_xx12 * (w26));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(0, -1, 0)) {
    const double l0 = lam(0, 0, 1, 0);
    const double l1 = lam(1, 0, 1, 0);
    const double l2 = lam(2, 0, 1, 0);
    const double l3 = lam(3, 0, 1, 0);
    const double l4 = lam(4, 0, 1, 0);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w1 = val(5, -1, 0, 0);  // v (-1, 0, 0)
    const double w13 = val(5, 0, 0, -1);  // v (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w18 = val(0, 0, 0, 0);  // RU (0, 0, 0)
    const double w19 = val(1, 0, 0, 0);  // RV (0, 0, 0)
    const double w20 = val(2, 0, 0, 0);  // RW (0, 0, 0)
    const double w21 = val(3, 0, 0, 0);  // RE (0, 0, 0)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w25 = val(7, 0, 0, 0);  // p (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w30 = val(5, 0, 0, 1);  // v (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w35 = val(4, 0, 1, 0);  // u (0, 1, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w37 = val(6, 0, 1, 0);  // w (0, 1, 0)
    const double w38 = val(8, 0, 1, 0);  // T (0, 1, 0)
    const double w39 = val(9, 0, 1, 0);  // mu (0, 1, 0)
    const double w40 = val(10, 0, 1, 0);  // ka (0, 1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w42 = val(5, 1, 0, 0);  // v (1, 0, 0)
    bar[0] += l1 * -C.ay * (w23);  // RU
    bar[1] += l0 * -C.ay + l2 * -C.ay * (w23);  // RV
    bar[2] += l3 * -C.ay * (w23);  // RW
    bar[3] += l4 * -C.ay * (w23);  // RE
    bar[4] += l1 * C.xm_yy * (w27 + w39) + l4 * (-C.e_yx4 * (w27 * w42) + C.e_yx4 * (w27 * w1) + -C.e_yy12 * (w27 * w35) + C.e_yy12 * (w27 * w22 + w27 * w22 + w39 * w35));  // u
    bar[5] += l1 * -C.ay * (w18) + l2 * (-C.ay * (w19) + C.ym_yy * (w27 + w39)) + l3 * -C.ay * (w20) + l4 * (-C.ay * (w21 + w25) + -C.ay * C.h0 + -C.e_yx6 * (w27 * w41) + C.e_yx6 * (w27 * w0) + -C.e_yy23 * (w27 * w36) + C.e_yy23 * (w27 * w23 + w27 * w23 + w39 * w36) + -C.e_zy6 * (w27 * w31) + C.e_zy6 * (w27 * w14));  // v
    bar[6] += l3 * C.zm_yy * (w27 + w39) + l4 * (-C.e_yy12 * (w27 * w37) + C.e_yy12 * (w27 * w24 + w27 * w24 + w39 * w37) + -C.e_zy4 * (w27 * w30) + C.e_zy4 * (w27 * w13));  // w
    bar[7] += l2 * -C.ay + l4 * -C.ay * (w23);  // p
    bar[8] += l4 * C.e_yy12 * (w28 + w40);  // T
    bar[9] += l1 * (-C.xm_xy * (w42) + C.xm_xy * (w1) + -C.xm_yy * (w35) + C.xm_yy * (w22)) + l2 * (-C.ym_xy * (w41) + C.ym_xy * (w0) + -C.ym_yy * (w36) + C.ym_yy * (w23) + -C.ym_zy * (w31) + C.ym_zy * (w14)) + l3 * (-C.zm_yy * (w37) + C.zm_yy * (w24) + -C.zm_zy * (w30) + C.zm_zy * (w13)) + l4 * (-C.e_yx4 * (w22 * w42) + C.e_yx4 * (w22 * w1) + -C.e_yx6 * (w41 * w23) + C.e_yx6 * (w0 * w23) + -C.e_yy12 * (w22 * w35 + w24 * w37) + C.e_yy12 * (w22 * w22 + w24 * w24) + -C.e_yy23 * (w23 * w36) + C.e_yy23 * (w23 * w23) + -C.e_zy4 * (w30 * w24) + C.e_zy4 * (w13 * w24) + -C.e_zy6 * (w23 * w31) + C.e_zy6 * (w23 * w14));  // mu
    bar[10] += l4 * (-C.e_yy12 * (w38) + C.e_yy12 * (w26));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(0, 0, -1)) {
    const double l0 = lam(0, 0, 0, 1);
    const double l1 = lam(1, 0, 0, 1);
    const double l2 = lam(2, 0, 0, 1);
    const double l3 = lam(3, 0, 0, 1);
    const double l4 = lam(4, 0, 0, 1);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w2 = val(6, -1, 0, 0);  // w (-1, 0, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w8 = val(6, 0, -1, 0);  // w (0, -1, 0)
    const double w18 = val(0, 0, 0, 0);  // RU (0, 0, 0)
    const double w19 = val(1, 0, 0, 0);  // RV (0, 0, 0)
    const double w20 = val(2, 0, 0, 0);  // RW (0, 0, 0)
    const double w21 = val(3, 0, 0, 0);  // RE (0, 0, 0)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w25 = val(7, 0, 0, 0);  // p (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w29 = val(4, 0, 0, 1);  // u (0, 0, 1)
    const double w30 = val(5, 0, 0, 1);  // v (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w32 = val(8, 0, 0, 1);  // T (0, 0, 1)
    const double w33 = val(9, 0, 0, 1);  // mu (0, 0, 1)
    const double w34 = val(10, 0, 0, 1);  // ka (0, 0, 1)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w37 = val(6, 0, 1, 0);  // w (0, 1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w43 = val(6, 1, 0, 0);  // w (1, 0, 0)
    bar[0] += l1 * -C.az * (w24);  // RU
    bar[1] += l2 * -C.az * (w24);  // RV
    bar[2] += l0 * -C.az + l3 * -C.az * (w24);  // RW
    bar[3] += l4 * -C.az * (w24);  // RE
    bar[4] += l1 * C.xm_zz * (w27 + w33) + l4 * (-C.e_zx4 * (w27 * w43) + C.e_zx4 * (w27 * w2) + -C.e_zz12 * (w27 * w29) + C.e_zz12 * (w27 * w22 + w27 * w22 + w33 * w29));  // u
    bar[5] += l2 * C.ym_zz * (w27 + w33) + l4 * (-C.e_zy4 * (w27 * w37) + C.e_zy4 * (w27 * w8) + -C.e_zz12 * (w27 * w30) + C.e_zz12 * (w27 * w23 + w27 * w23 + w33 * w30));  // v
    bar[6] += l1 * -C.az * (w18) + l2 * -C.az * (w19) + l3 * (-C.az * (w20) + C.zm_zz * (w27 + w33)) + l4 * (-C.az * (w21 + w25) + -C.az * C.h0 + -C.e_zx6 * (w27 * w41) + C.e_zx6 * (w27 * w0) + -C.e_zy6 * (w27 * w36) + C.e_zy6 * (w27 * w7) + -C.e_zz23 * (w27 * w31) + C.e_zz23 * (w27 * w24 + w27 * w24 + w33 * w31));  // w
    bar[7] += l3 * -C.az + l4 * -C.az * (w24);  // p
    bar[8] += l4 * C.e_zz12 * (w28 + w34);  // T
    bar[9] += l1 * (-C.xm_xz * (w43) + C.xm_xz * (w2) + -C.xm_zz * (w29) + C.xm_zz * (w22)) + l2 * (-C.ym_yz * (w37) + C.ym_yz * (w8) + -C.ym_zz * (w30) + C.ym_zz * (w23)) + l3 * (-C.zm_xz * (w41) + C.zm_xz * (w0) + -C.zm_yz * (w36) + C.zm_yz * (w7) + -C.zm_zz * (w31) + C.zm_zz * (w24)) + l4 * (-C.e_zx4 * (w22 * w43) + C.e_zx4 * (w22 * w2) + -C.e_zx6 * (w41 * w24) + C.e_zx6 * (w0 * w24) + -C.e_zy4 * (w23 * w37) + C.e_zy4 * (w23 * w8) + -C.e_zy6 * (w36 * w24) + C.e_zy6 * (w7 * w24) + -C.e_zz12 * (w22 * w29 + w23 * w30) + C.e_zz12 * (w22 * w22 + w23 * w23) + -C.e_zz23 * (w24 * w31) + C.e_zz23 * (w24 * w24));  // mu
    bar[10] += l4 * (-C.e_zz12 * (w32) + C.e_zz12 * (w26));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(0, 0, 1)) {
    const double l0 = lam(0, 0, 0, -1);
    const double l1 = lam(1, 0, 0, -1);
    const double l2 = lam(2, 0, 0, -1);
    const double l3 = lam(3, 0, 0, -1);
    const double l4 = lam(4, 0, 0, -1);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w2 = val(6, -1, 0, 0);  // w (-1, 0, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w8 = val(6, 0, -1, 0);  // w (0, -1, 0)
    const double w12 = val(4, 0, 0, -1);  // u (0, 0, -1)
    const double w13 = val(5, 0, 0, -1);  // v (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w15 = val(8, 0, 0, -1);  // T (0, 0, -1)
    const double w16 = val(9, 0, 0, -1);  // mu (0, 0, -1)
    const double w17 = val(10, 0, 0, -1);  // ka (0, 0, -1)
    const double w18 = val(0, 0, 0, 0);  // RU (0, 0, 0)
    const double w19 = val(1, 0, 0, 0);  // RV (0, 0, 0)
    const double w20 = val(2, 0, 0, 0);  // RW (0, 0, 0)
    const double w21 = val(3, 0, 0, 0);  // RE (0, 0, 0)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w25 = val(7, 0, 0, 0);  // p (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w37 = val(6, 0, 1, 0);  // w (0, 1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w43 = val(6, 1, 0, 0);  // w (1, 0, 0)
    bar[0] += l1 * C.az * (w24);  // RU
    bar[1] += l2 * C.az * (w24);  // RV
    bar[2] += l0 * C.az + l3 * C.az * (w24);  // RW
    bar[3] += l4 * C.az * (w24);  // RE
    bar[4] += l1 * C.xm_zz * (w27 + w16) + l4 * (-C.e_zx4 * (w27 * w2) + C.e_zx4 * (w27 * w43) + -C.e_zz12 * (w27 * w12) + C.e_zz12 * (w27 * w22 + w27 * w22 + w16 * w12));  // u
    bar[5] += l2 * C.ym_zz * (w27 + w16) + l4 * (-C.e_zy4 * (w27 * w8) + C.e_zy4 * (w27 * w37) + -C.e_zz12 * (w27 * w13) + C.e_zz12 * (w27 * w23 + w27 * w23 + w16 * w13));  // v
    bar[6] += l1 * C.az * (w18) + l2 * C.az * (w19) + l3 * (C.az * (w20) + C.zm_zz * (w27 + w16)) + l4 * (C.az * (w21 + w25) + C.az * C.h0 + -C.e_zx6 * (w27 * w0) + C.e_zx6 * (w27 * w41) + -C.e_zy6 * (w27 * w7) + C.e_zy6 * (w27 * w36) + -C.e_zz23 * (w27 * w14) + C.e_zz23 * (w27 * w24 + w27 * w24 + w16 * w14));  // w
    bar[7] += l3 * C.az + l4 * C.az * (w24);  // p
    bar[8] += l4 * C.e_zz12 * (w28 + w17);  // T
    bar[9] += l1 * (-C.xm_xz * (w2) + C.xm_xz * (w43) + -C.xm_zz * (w12) + C.xm_zz * (w22)) + l2 * (-C.ym_yz * (w8) + C.ym_yz * (w37) + -C.ym_zz * (w13) + C.ym_zz * (w23)) + l3 * (-C.zm_xz * (w0) + C.zm_xz * (w41) + -C.zm_yz * (w7) + C.zm_yz * (w36) + -C.zm_zz * (w14) + C.zm_zz * (w24)) + l4 * (-C.e_zx4 * (w22 * w2) + C.e_zx4 * (w22 * w43) + -C.e_zx6 * (w0 * w24) + C.e_zx6 * (w41 * w24) + -C.e_zy4 * (w23 * w8) + C.e_zy4 * (w23 * w37) + -C.e_zy6 * (w7 * w24) + C.e_zy6 * (w36 * w24) + -C.e_zz12 * (w12 * w22 + w13 * w23) + C.e_zz12 * (w22 * w22 + w23 * w23) + -C.e_zz23 * (w14 * w24) + C.e_zz23 * (w24 * w24));  // mu
    bar[10] += l4 * (-C.e_zz12 * (w15) + C.e_zz12 * (w26));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(0, 1, 0)) {
    const double l0 = lam(0, 0, -1, 0);
    const double l1 = lam(1, 0, -1, 0);
    const double l2 = lam(2, 0, -1, 0);
    const double l3 = lam(3, 0, -1, 0);
    const double l4 = lam(4, 0, -1, 0);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w1 = val(5, -1, 0, 0);  // v (-1, 0, 0)
    const double w6 = val(4, 0, -1, 0);  // u (0, -1, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w8 = val(6, 0, -1, 0);  // w (0, -1, 0)
    const double w9 = val(8, 0, -1, 0);  // T (0, -1, 0)
    const double w10 = val(9, 0, -1, 0);  // mu (0, -1, 0)
    const double w11 = val(10, 0, -1, 0);  // ka (0, -1, 0)
    const double w13 = val(5, 0, 0, -1);  // v (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w18 = val(0, 0, 0, 0);  // RU (0, 0, 0)
    const double w19 = val(1, 0, 0, 0);  // RV (0, 0, 0)
    const double w20 = val(2, 0, 0, 0);  // RW (0, 0, 0)
    const double w21 = val(3, 0, 0, 0);  // RE (0, 0, 0)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w25 = val(7, 0, 0, 0);  // p (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w30 = val(5, 0, 0, 1);  // v (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w42 = val(5, 1, 0, 0);  // v (1, 0, 0)
    bar[0] += l1 * C.ay * (w23);  // RU
    bar[1] += l0 * C.ay + l2 * C.ay * (w23);  // RV
    bar[2] += l3 * C.ay * (w23);  // RW
    bar[3] += l4 * C.ay * (w23);  // RE
    bar[4] += l1 * C.xm_yy * (w27 + w10) + l4 * (-C.e_yx4 * (w27 * w1) + C.e_yx4 * (w27 * w42) + -C.e_yy12 * (w27 * w6) + C.e_yy12 * (w27 * w22 + w27 * w22 + w10 * w6));  // u
    bar[5] += l1 * C.ay * (w18) + l2 * (C.ay * (w19) + C.ym_yy * (w27 + w10)) + l3 * C.ay * (w20) + l4 * (C.ay * (w21 + w25) + C.ay * C.h0 + -C.e_yx6 * (w27 * w0) + C.e_yx6 * (w27 * w41) + -C.e_yy23 * (w27 * w7) + C.e_yy23 * (w27 * w23 + w27 * w23 + w10 * w7) + -C.e_zy6 * (w27 * w14) + C.e_zy6 * (w27 * w31));  // v
    bar[6] += l3 * C.zm_yy * (w27 + w10) + l4 * (-C.e_yy12 * (w27 * w8) + C.e_yy12 * (w27 * w24 + w27 * w24 + w10 * w8) + -C.e_zy4 * (w27 * w13) + C.e_zy4 * (w27 * w30));  // w
    bar[7] += l2 * C.ay + l4 * C.ay * (w23);  // p
    bar[8] += l4 * C.e_yy12 * (w28 + w11);  // T
    bar[9] += l1 * (-C.xm_xy * (w1) + C.xm_xy * (w42) + -C.xm_yy * (w6) + C.xm_yy * (w22)) + l2 * (-C.ym_xy * (w0) + C.ym_xy * (w41) + -C.ym_yy * (w7) + C.ym_yy * (w23) + -C.ym_zy * (w14) + C.ym_zy * (w31)) + l3 * (-C.zm_yy * (w8) + C.zm_yy * (w24) + -C.zm_zy * (w13) + C.zm_zy * (w30)) + l4 * (-C.e_yx4 * (w22 * w1) + C.e_yx4 * (w22 * w42) + -C.e_yx6 * (w0 * w23) + C.e_yx6 * (w41 * w23) + -C.e_yy12 * (w6 * w22 + w8 * w24) + C.e_yy12 * (w22 * w22 + w24 * w24) + -C.e_yy23 * (w7 * w23) + C.e_yy23 * (w23 * w23) + -C.e_zy4 * (w13 * w24) + C.e_zy4 * (w30 * w24) + -C.e_zy6 * (w23 * w14) + C.e_zy6 * (w23 * w31));  // mu
    bar[10] += l4 * (-C.e_yy12 * (w9) + C.e_yy12 * (w26));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(1, 0, 0)) {
    const double l0 = lam(0, -1, 0, 0);
    const double l1 = lam(1, -1, 0, 0);
    const double l2 = lam(2, -1, 0, 0);
    const double l3 = lam(3, -1, 0, 0);
    const double l4 = lam(4, -1, 0, 0);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w1 = val(5, -1, 0, 0);  // v (-1, 0, 0)
    const double w2 = val(6, -1, 0, 0);  // w (-1, 0, 0)
    const double w3 = val(8, -1, 0, 0);  // T (-1, 0, 0)
    const double w4 = val(9, -1, 0, 0);  // mu (-1, 0, 0)
    const double w5 = val(10, -1, 0, 0);  // ka (-1, 0, 0)
    const double w6 = val(4, 0, -1, 0);  // u (0, -1, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w12 = val(4, 0, 0, -1);  // u (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w18 = val(0, 0, 0, 0);  // RU (0, 0, 0)
    const double w19 = val(1, 0, 0, 0);  // RV (0, 0, 0)
    const double w20 = val(2, 0, 0, 0);  // RW (0, 0, 0)
    const double w21 = val(3, 0, 0, 0);  // RE (0, 0, 0)
    const double w22 = val(4, 0, 0, 0);  // u (0, 0, 0)
    const double w23 = val(5, 0, 0, 0);  // v (0, 0, 0)
    const double w24 = val(6, 0, 0, 0);  // w (0, 0, 0)
    const double w25 = val(7, 0, 0, 0);  // p (0, 0, 0)
    const double w26 = val(8, 0, 0, 0);  // T (0, 0, 0)
    const double w27 = val(9, 0, 0, 0);  // mu (0, 0, 0)
    const double w28 = val(10, 0, 0, 0);  // ka (0, 0, 0)
    const double w29 = val(4, 0, 0, 1);  // u (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w35 = val(4, 0, 1, 0);  // u (0, 1, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    bar[0] += l0 * C.ax + l1 * C.ax * (w22);  // RU
    bar[1] += l2 * C.ax * (w22);  // RV
    bar[2] += l3 * C.ax * (w22);  // RW
    bar[3] += l4 * C.ax * (w22);  // RE
    bar[4] += l1 * (C.ax * (w18) + C.xm_xx * (w27 + w4)) + l2 * C.ax * (w19) + l3 * C.ax * (w20) + l4 * (C.ax * (w21 + w25) + C.ax * C.h0 + -C.e_xx23 * (w27 * w0) + C.e_xx23 * (w27 * w22 + w27 * w22 + w4 * w0) + -C.e_yx6 * (w27 * w7) + C.e_yx6 * (w27 * w36) + -C.e_zx6 * (w27 * w14) + C.e_zx6 * (w27 * w31));  // u
    bar[5] += l2 * C.ym_xx * (w27 + w4) + l4 * (-C.e_xx12 * (w27 * w1) + C.e_xx12 * (w27 * w23 + w27 * w23 + w4 * w1) + -C.e_yx4 * (w27 * w6) + C.e_yx4 * (w27 * w35));  // v
    bar[6] += l3 * C.zm_xx * (w27 + w4) + l4 * (-C.e_xx12 * (w27 * w2) + C.e_xx12 * (w27 * w24 + w27 * w24 + w4 * w2) + -C.e_zx4 * (w27 * w12) + C.e_zx4 * (w27 * w29));  // w
    bar[7] += l1 * C.ax + l4 * C.ax * (w22);  // p
    bar[8] += l4 * C.e_xx12 * (w28 + w5);  // T
    bar[9] += l1 * (-C.xm_xx * (w0) + C.xm_xx * (w22) + -C.xm_yx * (w7) + C.xm_yx * (w36) + -C.xm_zx * (w14) + C.xm_zx * (w31)) + l2 * (-C.ym_xx * (w1) + C.ym_xx * (w23) + -C.ym_yx * (w6) + C.ym_yx * (w35)) + l3 * (-C.zm_xx * (w2) + C.zm_xx * (w24) + -C.zm_zx * (w12) + C.zm_zx * (w29)) + l4 * (-C.e_xx12 * (w1 * w23 + w2 * w24) + C.e_xx12 * (w23 * w23 + w24 * w24) + -C.e_xx23 * (w0 * w22) + C.e_xx23 * (w22 * w22) + -C.e_yx4 * (w6 * w23) + C.e_yx4 * (w35 * w23) + -C.e_yx6 * (w22 * w7) + C.e_yx6 * (w22 * w36) + -C.e_zx4 * (w12 * w24) + C.e_zx4 * (w29 * w24) + -C.e_zx6 * (w22 * w14) + C.e_zx6 * (w22 * w31));  // mu
    bar[10] += l4 * (-C.e_xx12 * (w3) + C.e_xx12 * (w26));  // ka
  }
  asm volatile("" ::: "memory");
  if (inner(-1, -1, 0)) {
    const double l1 = lam(1, 1, 1, 0);
    const double l2 = lam(2, 1, 1, 0);
    const double l4 = lam(4, 1, 1, 0);
    const double w35 = val(4, 0, 1, 0);  // u (0, 1, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w39 = val(9, 0, 1, 0);  // mu (0, 1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w42 = val(5, 1, 0, 0);  // v (1, 0, 0)
    const double w45 = val(9, 1, 0, 0);  // mu (1, 0, 0)
    bar[4] += l2 * (C.ym_xy * (w45) + C.ym_yx * (w39)) + l4 * (C.e_yx4 * (w39 * w36) + C.e_yx6 * (w45 * w42));  // u
    bar[5] += l1 * (C.xm_xy * (w45) + C.xm_yx * (w39)) + l4 * (C.e_yx4 * (w45 * w41) + C.e_yx6 * (w39 * w35));  // v
  }
  asm volatile("" ::: "memory");
  if (inner(-1, 0, -1)) {
    const double l1 = lam(1, 1, 0, 1);
    const double l3 = lam(3, 1, 0, 1);
    const double l4 = lam(4, 1, 0, 1);
    const double w29 = val(4, 0, 0, 1);  // u (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w33 = val(9, 0, 0, 1);  // mu (0, 0, 1)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w43 = val(6, 1, 0, 0);  // w (1, 0, 0)
    const double w45 = val(9, 1, 0, 0);  // mu (1, 0, 0)
    bar[4] += l3 * (C.zm_xz * (w45) + C.zm_zx * (w33)) + l4 * (C.e_zx4 * (w33 * w31) + C.e_zx6 * (w45 * w43));  // u
    bar[6] += l1 * (C.xm_xz * (w45) + C.xm_zx * (w33)) + l4 * (C.e_zx4 * (w45 * w41) + C.e_zx6 * (w33 * w29));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(-1, 0, 1)) {
    const double l1 = lam(1, 1, 0, -1);
    const double l3 = lam(3, 1, 0, -1);
    const double l4 = lam(4, 1, 0, -1);
    const double w12 = val(4, 0, 0, -1);  // u (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w16 = val(9, 0, 0, -1);  // mu (0, 0, -1)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w43 = val(6, 1, 0, 0);  // w (1, 0, 0)
    const double w45 = val(9, 1, 0, 0);  // mu (1, 0, 0)
    bar[4] += l3 * (-C.zm_xz * (w45) + -C.zm_zx * (w16)) + l4 * (-C.e_zx4 * (w16 * w14) + -C.e_zx6 * (w45 * w43));  // u
    bar[6] += l1 * (-C.xm_xz * (w45) + -C.xm_zx * (w16)) + l4 * (-C.e_zx4 * (w45 * w41) + -C.e_zx6 * (w16 * w12));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(-1, 1, 0)) {
    const double l1 = lam(1, 1, -1, 0);
    const double l2 = lam(2, 1, -1, 0);
    const double l4 = lam(4, 1, -1, 0);
    const double w6 = val(4, 0, -1, 0);  // u (0, -1, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w10 = val(9, 0, -1, 0);  // mu (0, -1, 0)
    const double w41 = val(4, 1, 0, 0);  // u (1, 0, 0)
    const double w42 = val(5, 1, 0, 0);  // v (1, 0, 0)
    const double w45 = val(9, 1, 0, 0);  // mu (1, 0, 0)
    bar[4] += l2 * (-C.ym_xy * (w45) + -C.ym_yx * (w10)) + l4 * (-C.e_yx4 * (w10 * w7) + -C.e_yx6 * (w45 * w42));  // u
    bar[5] += l1 * (-C.xm_xy * (w45) + -C.xm_yx * (w10)) + l4 * (-C.e_yx4 * (w45 * w41) + -C.e_yx6 * (w10 * w6));  // v
  }
  asm volatile("" ::: "memory");
  if (inner(0, -1, -1)) {
    const double l2 = lam(2, 0, 1, 1);
    const double l3 = lam(3, 0, 1, 1);
    const double l4 = lam(4, 0, 1, 1);
    const double w30 = val(5, 0, 0, 1);  // v (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w33 = val(9, 0, 0, 1);  // mu (0, 0, 1)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w37 = val(6, 0, 1, 0);  // w (0, 1, 0)
    const double w39 = val(9, 0, 1, 0);  // mu (0, 1, 0)
    bar[5] += l3 * (C.zm_yz * (w39) + C.zm_zy * (w33)) + l4 * (C.e_zy4 * (w33 * w31) + C.e_zy6 * (w39 * w37));  // v
    bar[6] += l2 * (C.ym_yz * (w39) + C.ym_zy * (w33)) + l4 * (C.e_zy4 * (w39 * w36) + C.e_zy6 * (w33 * w30));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(0, -1, 1)) {
    const double l2 = lam(2, 0, 1, -1);
    const double l3 = lam(3, 0, 1, -1);
    const double l4 = lam(4, 0, 1, -1);
    const double w13 = val(5, 0, 0, -1);  // v (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w16 = val(9, 0, 0, -1);  // mu (0, 0, -1)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w37 = val(6, 0, 1, 0);  // w (0, 1, 0)
    const double w39 = val(9, 0, 1, 0);  // mu (0, 1, 0)
    bar[5] += l3 * (-C.zm_yz * (w39) + -C.zm_zy * (w16)) + l4 * (-C.e_zy4 * (w16 * w14) + -C.e_zy6 * (w39 * w37));  // v
    bar[6] += l2 * (-C.ym_yz * (w39) + -C.ym_zy * (w16)) + l4 * (-C.e_zy4 * (w39 * w36) + -C.e_zy6 * (w16 * w13));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(0, 1, -1)) {
    const double l2 = lam(2, 0, -1, 1);
    const double l3 = lam(3, 0, -1, 1);
    const double l4 = lam(4, 0, -1, 1);
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w8 = val(6, 0, -1, 0);  // w (0, -1, 0)
    const double w10 = val(9, 0, -1, 0);  // mu (0, -1, 0)
    const double w30 = val(5, 0, 0, 1);  // v (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w33 = val(9, 0, 0, 1);  // mu (0, 0, 1)
    bar[5] += l3 * (-C.zm_yz * (w10) + -C.zm_zy * (w33)) + l4 * (-C.e_zy4 * (w33 * w31) + -C.e_zy6 * (w10 * w8));  // v
    bar[6] += l2 * (-C.ym_yz * (w10) + -C.ym_zy * (w33)) + l4 * (-C.e_zy4 * (w10 * w7) + -C.e_zy6 * (w33 * w30));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(0, 1, 1)) {
    const double l2 = lam(2, 0, -1, -1);
    const double l3 = lam(3, 0, -1, -1);
    const double l4 = lam(4, 0, -1, -1);
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w8 = val(6, 0, -1, 0);  // w (0, -1, 0)
    const double w10 = val(9, 0, -1, 0);  // mu (0, -1, 0)
    const double w13 = val(5, 0, 0, -1);  // v (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w16 = val(9, 0, 0, -1);  // mu (0, 0, -1)
    bar[5] += l3 * (C.zm_yz * (w10) + C.zm_zy * (w16)) + l4 * (C.e_zy4 * (w16 * w14) + C.e_zy6 * (w10 * w8));  // v
    bar[6] += l2 * (C.ym_yz * (w10) + C.ym_zy * (w16)) + l4 * (C.e_zy4 * (w10 * w7) + C.e_zy6 * (w16 * w13));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(1, -1, 0)) {
    const double l1 = lam(1, -1, 1, 0);
    const double l2 = lam(2, -1, 1, 0);
    const double l4 = lam(4, -1, 1, 0);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w1 = val(5, -1, 0, 0);  // v (-1, 0, 0)
    const double w4 = val(9, -1, 0, 0);  // mu (-1, 0, 0)
    const double w35 = val(4, 0, 1, 0);  // u (0, 1, 0)
    const double w36 = val(5, 0, 1, 0);  // v (0, 1, 0)
    const double w39 = val(9, 0, 1, 0);  // mu (0, 1, 0)
    bar[4] += l2 * (-C.ym_xy * (w4) + -C.ym_yx * (w39)) + l4 * (-C.e_yx4 * (w39 * w36) + -C.e_yx6 * (w4 * w1));  // u
    bar[5] += l1 * (-C.xm_xy * (w4) + -C.xm_yx * (w39)) + l4 * (-C.e_yx4 * (w4 * w0) + -C.e_yx6 * (w39 * w35));  // v
  }
  asm volatile("" ::: "memory");
  if (inner(1, 0, -1)) {
    const double l1 = lam(1, -1, 0, 1);
    const double l3 = lam(3, -1, 0, 1);
    const double l4 = lam(4, -1, 0, 1);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w2 = val(6, -1, 0, 0);  // w (-1, 0, 0)
    const double w4 = val(9, -1, 0, 0);  // mu (-1, 0, 0)
    const double w29 = val(4, 0, 0, 1);  // u (0, 0, 1)
    const double w31 = val(6, 0, 0, 1);  // w (0, 0, 1)
    const double w33 = val(9, 0, 0, 1);  // mu (0, 0, 1)
    bar[4] += l3 * (-C.zm_xz * (w4) + -C.zm_zx * (w33)) + l4 * (-C.e_zx4 * (w33 * w31) + -C.e_zx6 * (w4 * w2));  // u
    bar[6] += l1 * (-C.xm_xz * (w4) + -C.xm_zx * (w33)) + l4 * (-C.e_zx4 * (w4 * w0) + -C.e_zx6 * (w33 * w29));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(1, 0, 1)) {
    const double l1 = lam(1, -1, 0, -1);
    const double l3 = lam(3, -1, 0, -1);
    const double l4 = lam(4, -1, 0, -1);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w2 = val(6, -1, 0, 0);  // w (-1, 0, 0)
    const double w4 = val(9, -1, 0, 0);  // mu (-1, 0, 0)
    const double w12 = val(4, 0, 0, -1);  // u (0, 0, -1)
    const double w14 = val(6, 0, 0, -1);  // w (0, 0, -1)
    const double w16 = val(9, 0, 0, -1);  // mu (0, 0, -1)
    bar[4] += l3 * (C.zm_xz * (w4) + C.zm_zx * (w16)) + l4 * (C.e_zx4 * (w16 * w14) + C.e_zx6 * (w4 * w2));  // u
    bar[6] += l1 * (C.xm_xz * (w4) + C.xm_zx * (w16)) + l4 * (C.e_zx4 * (w4 * w0) + C.e_zx6 * (w16 * w12));  // w
  }
  asm volatile("" ::: "memory");
  if (inner(1, 1, 0)) {
    const double l1 = lam(1, -1, -1, 0);
    const double l2 = lam(2, -1, -1, 0);
    const double l4 = lam(4, -1, -1, 0);
    const double w0 = val(4, -1, 0, 0);  // u (-1, 0, 0)
    const double w1 = val(5, -1, 0, 0);  // v (-1, 0, 0)
    const double w4 = val(9, -1, 0, 0);  // mu (-1, 0, 0)
    const double w6 = val(4, 0, -1, 0);  // u (0, -1, 0)
    const double w7 = val(5, 0, -1, 0);  // v (0, -1, 0)
    const double w10 = val(9, 0, -1, 0);  // mu (0, -1, 0)
    bar[4] += l2 * (C.ym_xy * (w4) + C.ym_yx * (w10)) + l4 * (C.e_yx4 * (w10 * w7) + C.e_yx6 * (w4 * w1));  // u
    bar[5] += l1 * (C.xm_xy * (w4) + C.xm_yx * (w10)) + l4 * (C.e_yx4 * (w4 * w0) + C.e_yx6 * (w10 * w6));  // v
  }
}

}  // namespace nsf
#endif
