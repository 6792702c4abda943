// Generated by gen_rhs_adjoint.py from the RHS term table: do not edit. The transposed stencil of the
// right-hand side (rhs_eval, nsf_physics.cuh) in gather form: rhs_adjoint_gather(...) returns, for node
// (i, j, k), the adjoint of each input quantity (RU, RV, RW, RE, u, v, w, p, T, mu, ka) summed over every
// interior node whose RHS reads it. lam(e, b): RHS adjoint of equation e at linear node b (zero where no
// RHS is taken); val(q, b): input quantity q at node b; inner(di, dj, dk): the node (i-di, j-dj, k-dk)
// is one whose RHS was taken (its whole stencil then lies inside the grid).
#ifndef NSF_RHS_ADJOINT_CUH
#define NSF_RHS_ADJOINT_CUH

namespace nsf {

template <class Lam, class Val, class Inner>
__device__ __forceinline__ void rhs_adjoint_gather(const Consts& C, long long X, long long sI, long long sJ,
                                                   const Lam& lam, const Val& val, const Inner& inner,
                                                   double bar[11]) {
  for (int q = 0; q < 11; ++q) bar[q] = 0.0;
  if (inner(-1, -1, 0)) {
    const long long b = X - (-1 * sI + -1 * sJ + 0);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (-1 * sI + 0 * sJ + 0));  // mu (-1, 0, 0)
    const double v1 = val(9, b + (0 * sI + -1 * sJ + 0));  // mu (0, -1, 0)
    const double v2 = val(4, b + (-1 * sI + 0 * sJ + 0));  // u (-1, 0, 0)
    const double v3 = val(4, b + (0 * sI + -1 * sJ + 0));  // u (0, -1, 0)
    const double v4 = val(5, b + (-1 * sI + 0 * sJ + 0));  // v (-1, 0, 0)
    const double v5 = val(5, b + (0 * sI + -1 * sJ + 0));  // v (0, -1, 0)
    bar[4] += l2 * C.ym_yx * v0 + l2 * C.ym_xy * v1 + l4 * C.e_yx4 * v0 * v4 + l4 * C.e_yx6 * v1 * v5;  // u
    bar[5] += l1 * C.xm_xy * v1 + l1 * C.xm_yx * v0 + l4 * C.e_yx6 * v0 * v2 + l4 * C.e_yx4 * v1 * v3;  // v
  }
  if (inner(-1, 0, -1)) {
    const long long b = X - (-1 * sI + 0 * sJ + -1);
    const double l1 = lam(1, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (-1 * sI + 0 * sJ + 0));  // mu (-1, 0, 0)
    const double v1 = val(9, b + (0 * sI + 0 * sJ + -1));  // mu (0, 0, -1)
    const double v2 = val(4, b + (-1 * sI + 0 * sJ + 0));  // u (-1, 0, 0)
    const double v3 = val(4, b + (0 * sI + 0 * sJ + -1));  // u (0, 0, -1)
    const double v4 = val(6, b + (-1 * sI + 0 * sJ + 0));  // w (-1, 0, 0)
    const double v5 = val(6, b + (0 * sI + 0 * sJ + -1));  // w (0, 0, -1)
    bar[4] += l3 * C.zm_zx * v0 + l3 * C.zm_xz * v1 + l4 * C.e_zx4 * v0 * v4 + l4 * C.e_zx6 * v1 * v5;  // u
    bar[6] += l1 * C.xm_xz * v1 + l1 * C.xm_zx * v0 + l4 * C.e_zx6 * v0 * v2 + l4 * C.e_zx4 * v1 * v3;  // w
  }
  if (inner(-1, 0, 0)) {
    const long long b = X - (-1 * sI + 0 * sJ + 0);
    const double l0 = lam(0, b);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(3, b + (-1 * sI + 0 * sJ + 0));  // RE (-1, 0, 0)
    const double v1 = val(0, b + (-1 * sI + 0 * sJ + 0));  // RU (-1, 0, 0)
    const double v2 = val(1, b + (-1 * sI + 0 * sJ + 0));  // RV (-1, 0, 0)
    const double v3 = val(2, b + (-1 * sI + 0 * sJ + 0));  // RW (-1, 0, 0)
    const double v4 = val(8, b + (-1 * sI + 0 * sJ + 0));  // T (-1, 0, 0)
    const double v5 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v6 = val(10, b + (-1 * sI + 0 * sJ + 0));  // ka (-1, 0, 0)
    const double v7 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v8 = val(9, b + (-1 * sI + 0 * sJ + 0));  // mu (-1, 0, 0)
    const double v9 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v10 = val(7, b + (-1 * sI + 0 * sJ + 0));  // p (-1, 0, 0)
    const double v11 = val(4, b + (-1 * sI + -1 * sJ + 0));  // u (-1, -1, 0)
    const double v12 = val(4, b + (-1 * sI + 0 * sJ + -1));  // u (-1, 0, -1)
    const double v13 = val(4, b + (-1 * sI + 0 * sJ + 0));  // u (-1, 0, 0)
    const double v14 = val(4, b + (-1 * sI + 0 * sJ + 1));  // u (-1, 0, 1)
    const double v15 = val(4, b + (-1 * sI + 1 * sJ + 0));  // u (-1, 1, 0)
    const double v16 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v17 = val(5, b + (-1 * sI + -1 * sJ + 0));  // v (-1, -1, 0)
    const double v18 = val(5, b + (-1 * sI + 0 * sJ + 0));  // v (-1, 0, 0)
    const double v19 = val(5, b + (-1 * sI + 1 * sJ + 0));  // v (-1, 1, 0)
    const double v20 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v21 = val(6, b + (-1 * sI + 0 * sJ + -1));  // w (-1, 0, -1)
    const double v22 = val(6, b + (-1 * sI + 0 * sJ + 0));  // w (-1, 0, 0)
    const double v23 = val(6, b + (-1 * sI + 0 * sJ + 1));  // w (-1, 0, 1)
    const double v24 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    bar[0] += l0 * -C.ax + l1 * -C.ax * v13;  // RU
    bar[1] += l2 * -C.ax * v13;  // RV
    bar[2] += l3 * -C.ax * v13;  // RW
    bar[3] += l4 * -C.ax * v13;  // RE
    bar[4] += l1 * -C.ax * v1 + l1 * C.xm_xx * v8 + l1 * C.xm_xx * v9 + l2 * -C.ax * v2 + l3 * -C.ax * v3 + l4 * -C.ax * C.h0 + l4 * -C.ax * v0 + l4 * -C.ax * v10 + l4 * -C.e_xx23 * v8 * v16 + l4 * C.e_xx23 * v8 * v13 + l4 * C.e_xx23 * v8 * v13 + l4 * C.e_xx23 * v9 * v16 + l4 * -C.e_yx6 * v8 * v19 + l4 * C.e_yx6 * v8 * v17 + l4 * -C.e_zx6 * v8 * v23 + l4 * C.e_zx6 * v8 * v21;  // u
    bar[5] += l2 * C.ym_xx * v8 + l2 * C.ym_xx * v9 + l4 * -C.e_xx12 * v8 * v20 + l4 * C.e_xx12 * v8 * v18 + l4 * C.e_xx12 * v8 * v18 + l4 * C.e_xx12 * v9 * v20 + l4 * -C.e_yx4 * v8 * v15 + l4 * C.e_yx4 * v8 * v11;  // v
    bar[6] += l3 * C.zm_xx * v8 + l3 * C.zm_xx * v9 + l4 * -C.e_xx12 * v8 * v24 + l4 * C.e_xx12 * v8 * v22 + l4 * C.e_xx12 * v8 * v22 + l4 * C.e_xx12 * v9 * v24 + l4 * -C.e_zx4 * v8 * v14 + l4 * C.e_zx4 * v8 * v12;  // w
    bar[7] += l1 * -C.ax + l4 * -C.ax * v13;  // p
    bar[8] += l4 * C.e_xx12 * v6 + l4 * C.e_xx12 * v7;  // T
    bar[9] += l1 * -C.xm_xx * v16 + l1 * C.xm_xx * v13 + l1 * -C.xm_yx * v19 + l1 * C.xm_yx * v17 + l1 * -C.xm_zx * v23 + l1 * C.xm_zx * v21 + l2 * -C.ym_xx * v20 + l2 * C.ym_xx * v18 + l2 * -C.ym_yx * v15 + l2 * C.ym_yx * v11 + l3 * -C.zm_xx * v24 + l3 * C.zm_xx * v22 + l3 * -C.zm_zx * v14 + l3 * C.zm_zx * v12 + l4 * -C.e_xx23 * v13 * v16 + l4 * C.e_xx23 * v13 * v13 + l4 * -C.e_xx12 * v18 * v20 + l4 * C.e_xx12 * v18 * v18 + l4 * -C.e_xx12 * v22 * v24 + l4 * C.e_xx12 * v22 * v22 + l4 * -C.e_yx6 * v13 * v19 + l4 * C.e_yx6 * v13 * v17 + l4 * -C.e_zx6 * v13 * v23 + l4 * C.e_zx6 * v13 * v21 + l4 * -C.e_yx4 * v15 * v18 + l4 * C.e_yx4 * v11 * v18 + l4 * -C.e_zx4 * v14 * v22 + l4 * C.e_zx4 * v12 * v22;  // mu
    bar[10] += l4 * -C.e_xx12 * v5 + l4 * C.e_xx12 * v4;  // ka
  }
  if (inner(-1, 0, 1)) {
    const long long b = X - (-1 * sI + 0 * sJ + 1);
    const double l1 = lam(1, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (-1 * sI + 0 * sJ + 0));  // mu (-1, 0, 0)
    const double v1 = val(9, b + (0 * sI + 0 * sJ + 1));  // mu (0, 0, 1)
    const double v2 = val(4, b + (-1 * sI + 0 * sJ + 0));  // u (-1, 0, 0)
    const double v3 = val(4, b + (0 * sI + 0 * sJ + 1));  // u (0, 0, 1)
    const double v4 = val(6, b + (-1 * sI + 0 * sJ + 0));  // w (-1, 0, 0)
    const double v5 = val(6, b + (0 * sI + 0 * sJ + 1));  // w (0, 0, 1)
    bar[4] += l3 * -C.zm_zx * v0 + l3 * -C.zm_xz * v1 + l4 * -C.e_zx4 * v0 * v4 + l4 * -C.e_zx6 * v1 * v5;  // u
    bar[6] += l1 * -C.xm_xz * v1 + l1 * -C.xm_zx * v0 + l4 * -C.e_zx6 * v0 * v2 + l4 * -C.e_zx4 * v1 * v3;  // w
  }
  if (inner(-1, 1, 0)) {
    const long long b = X - (-1 * sI + 1 * sJ + 0);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (-1 * sI + 0 * sJ + 0));  // mu (-1, 0, 0)
    const double v1 = val(9, b + (0 * sI + 1 * sJ + 0));  // mu (0, 1, 0)
    const double v2 = val(4, b + (-1 * sI + 0 * sJ + 0));  // u (-1, 0, 0)
    const double v3 = val(4, b + (0 * sI + 1 * sJ + 0));  // u (0, 1, 0)
    const double v4 = val(5, b + (-1 * sI + 0 * sJ + 0));  // v (-1, 0, 0)
    const double v5 = val(5, b + (0 * sI + 1 * sJ + 0));  // v (0, 1, 0)
    bar[4] += l2 * -C.ym_yx * v0 + l2 * -C.ym_xy * v1 + l4 * -C.e_yx4 * v0 * v4 + l4 * -C.e_yx6 * v1 * v5;  // u
    bar[5] += l1 * -C.xm_xy * v1 + l1 * -C.xm_yx * v0 + l4 * -C.e_yx6 * v0 * v2 + l4 * -C.e_yx4 * v1 * v3;  // v
  }
  if (inner(0, -1, -1)) {
    const long long b = X - (0 * sI + -1 * sJ + -1);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + -1 * sJ + 0));  // mu (0, -1, 0)
    const double v1 = val(9, b + (0 * sI + 0 * sJ + -1));  // mu (0, 0, -1)
    const double v2 = val(5, b + (0 * sI + -1 * sJ + 0));  // v (0, -1, 0)
    const double v3 = val(5, b + (0 * sI + 0 * sJ + -1));  // v (0, 0, -1)
    const double v4 = val(6, b + (0 * sI + -1 * sJ + 0));  // w (0, -1, 0)
    const double v5 = val(6, b + (0 * sI + 0 * sJ + -1));  // w (0, 0, -1)
    bar[5] += l3 * C.zm_zy * v0 + l3 * C.zm_yz * v1 + l4 * C.e_zy4 * v0 * v4 + l4 * C.e_zy6 * v1 * v5;  // v
    bar[6] += l2 * C.ym_yz * v1 + l2 * C.ym_zy * v0 + l4 * C.e_zy6 * v0 * v2 + l4 * C.e_zy4 * v1 * v3;  // w
  }
  if (inner(0, -1, 0)) {
    const long long b = X - (0 * sI + -1 * sJ + 0);
    const double l0 = lam(0, b);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(3, b + (0 * sI + -1 * sJ + 0));  // RE (0, -1, 0)
    const double v1 = val(0, b + (0 * sI + -1 * sJ + 0));  // RU (0, -1, 0)
    const double v2 = val(1, b + (0 * sI + -1 * sJ + 0));  // RV (0, -1, 0)
    const double v3 = val(2, b + (0 * sI + -1 * sJ + 0));  // RW (0, -1, 0)
    const double v4 = val(8, b + (0 * sI + -1 * sJ + 0));  // T (0, -1, 0)
    const double v5 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v6 = val(10, b + (0 * sI + -1 * sJ + 0));  // ka (0, -1, 0)
    const double v7 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v8 = val(9, b + (0 * sI + -1 * sJ + 0));  // mu (0, -1, 0)
    const double v9 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v10 = val(7, b + (0 * sI + -1 * sJ + 0));  // p (0, -1, 0)
    const double v11 = val(4, b + (-1 * sI + -1 * sJ + 0));  // u (-1, -1, 0)
    const double v12 = val(4, b + (0 * sI + -1 * sJ + 0));  // u (0, -1, 0)
    const double v13 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v14 = val(4, b + (1 * sI + -1 * sJ + 0));  // u (1, -1, 0)
    const double v15 = val(5, b + (-1 * sI + -1 * sJ + 0));  // v (-1, -1, 0)
    const double v16 = val(5, b + (0 * sI + -1 * sJ + -1));  // v (0, -1, -1)
    const double v17 = val(5, b + (0 * sI + -1 * sJ + 0));  // v (0, -1, 0)
    const double v18 = val(5, b + (0 * sI + -1 * sJ + 1));  // v (0, -1, 1)
    const double v19 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v20 = val(5, b + (1 * sI + -1 * sJ + 0));  // v (1, -1, 0)
    const double v21 = val(6, b + (0 * sI + -1 * sJ + -1));  // w (0, -1, -1)
    const double v22 = val(6, b + (0 * sI + -1 * sJ + 0));  // w (0, -1, 0)
    const double v23 = val(6, b + (0 * sI + -1 * sJ + 1));  // w (0, -1, 1)
    const double v24 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    bar[0] += l1 * -C.ay * v17;  // RU
    bar[1] += l0 * -C.ay + l2 * -C.ay * v17;  // RV
    bar[2] += l3 * -C.ay * v17;  // RW
    bar[3] += l4 * -C.ay * v17;  // RE
    bar[4] += l1 * C.xm_yy * v8 + l1 * C.xm_yy * v9 + l4 * -C.e_yy12 * v8 * v13 + l4 * C.e_yy12 * v8 * v12 + l4 * C.e_yy12 * v8 * v12 + l4 * C.e_yy12 * v9 * v13 + l4 * -C.e_yx4 * v8 * v20 + l4 * C.e_yx4 * v8 * v15;  // u
    bar[5] += l1 * -C.ay * v1 + l2 * -C.ay * v2 + l2 * C.ym_yy * v8 + l2 * C.ym_yy * v9 + l3 * -C.ay * v3 + l4 * -C.ay * C.h0 + l4 * -C.ay * v0 + l4 * -C.ay * v10 + l4 * -C.e_yy23 * v8 * v19 + l4 * C.e_yy23 * v8 * v17 + l4 * C.e_yy23 * v8 * v17 + l4 * C.e_yy23 * v9 * v19 + l4 * -C.e_yx6 * v8 * v14 + l4 * C.e_yx6 * v8 * v11 + l4 * -C.e_zy6 * v8 * v23 + l4 * C.e_zy6 * v8 * v21;  // v
    bar[6] += l3 * C.zm_yy * v8 + l3 * C.zm_yy * v9 + l4 * -C.e_yy12 * v8 * v24 + l4 * C.e_yy12 * v8 * v22 + l4 * C.e_yy12 * v8 * v22 + l4 * C.e_yy12 * v9 * v24 + l4 * -C.e_zy4 * v8 * v18 + l4 * C.e_zy4 * v8 * v16;  // w
    bar[7] += l2 * -C.ay + l4 * -C.ay * v17;  // p
    bar[8] += l4 * C.e_yy12 * v6 + l4 * C.e_yy12 * v7;  // T
    bar[9] += l1 * -C.xm_yy * v13 + l1 * C.xm_yy * v12 + l1 * -C.xm_xy * v20 + l1 * C.xm_xy * v15 + l2 * -C.ym_yy * v19 + l2 * C.ym_yy * v17 + l2 * -C.ym_xy * v14 + l2 * C.ym_xy * v11 + l2 * -C.ym_zy * v23 + l2 * C.ym_zy * v21 + l3 * -C.zm_yy * v24 + l3 * C.zm_yy * v22 + l3 * -C.zm_zy * v18 + l3 * C.zm_zy * v16 + l4 * -C.e_yy12 * v12 * v13 + l4 * C.e_yy12 * v12 * v12 + l4 * -C.e_yy23 * v17 * v19 + l4 * C.e_yy23 * v17 * v17 + l4 * -C.e_yy12 * v22 * v24 + l4 * C.e_yy12 * v22 * v22 + l4 * -C.e_yx6 * v14 * v17 + l4 * C.e_yx6 * v11 * v17 + l4 * -C.e_zy6 * v17 * v23 + l4 * C.e_zy6 * v17 * v21 + l4 * -C.e_yx4 * v12 * v20 + l4 * C.e_yx4 * v12 * v15 + l4 * -C.e_zy4 * v18 * v22 + l4 * C.e_zy4 * v16 * v22;  // mu
    bar[10] += l4 * -C.e_yy12 * v5 + l4 * C.e_yy12 * v4;  // ka
  }
  if (inner(0, -1, 1)) {
    const long long b = X - (0 * sI + -1 * sJ + 1);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + -1 * sJ + 0));  // mu (0, -1, 0)
    const double v1 = val(9, b + (0 * sI + 0 * sJ + 1));  // mu (0, 0, 1)
    const double v2 = val(5, b + (0 * sI + -1 * sJ + 0));  // v (0, -1, 0)
    const double v3 = val(5, b + (0 * sI + 0 * sJ + 1));  // v (0, 0, 1)
    const double v4 = val(6, b + (0 * sI + -1 * sJ + 0));  // w (0, -1, 0)
    const double v5 = val(6, b + (0 * sI + 0 * sJ + 1));  // w (0, 0, 1)
    bar[5] += l3 * -C.zm_zy * v0 + l3 * -C.zm_yz * v1 + l4 * -C.e_zy4 * v0 * v4 + l4 * -C.e_zy6 * v1 * v5;  // v
    bar[6] += l2 * -C.ym_yz * v1 + l2 * -C.ym_zy * v0 + l4 * -C.e_zy6 * v0 * v2 + l4 * -C.e_zy4 * v1 * v3;  // w
  }
  if (inner(0, 0, -1)) {
    const long long b = X - (0 * sI + 0 * sJ + -1);
    const double l0 = lam(0, b);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(3, b + (0 * sI + 0 * sJ + -1));  // RE (0, 0, -1)
    const double v1 = val(0, b + (0 * sI + 0 * sJ + -1));  // RU (0, 0, -1)
    const double v2 = val(1, b + (0 * sI + 0 * sJ + -1));  // RV (0, 0, -1)
    const double v3 = val(2, b + (0 * sI + 0 * sJ + -1));  // RW (0, 0, -1)
    const double v4 = val(8, b + (0 * sI + 0 * sJ + -1));  // T (0, 0, -1)
    const double v5 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v6 = val(10, b + (0 * sI + 0 * sJ + -1));  // ka (0, 0, -1)
    const double v7 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v8 = val(9, b + (0 * sI + 0 * sJ + -1));  // mu (0, 0, -1)
    const double v9 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v10 = val(7, b + (0 * sI + 0 * sJ + -1));  // p (0, 0, -1)
    const double v11 = val(4, b + (-1 * sI + 0 * sJ + -1));  // u (-1, 0, -1)
    const double v12 = val(4, b + (0 * sI + 0 * sJ + -1));  // u (0, 0, -1)
    const double v13 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v14 = val(4, b + (1 * sI + 0 * sJ + -1));  // u (1, 0, -1)
    const double v15 = val(5, b + (0 * sI + -1 * sJ + -1));  // v (0, -1, -1)
    const double v16 = val(5, b + (0 * sI + 0 * sJ + -1));  // v (0, 0, -1)
    const double v17 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v18 = val(5, b + (0 * sI + 1 * sJ + -1));  // v (0, 1, -1)
    const double v19 = val(6, b + (-1 * sI + 0 * sJ + -1));  // w (-1, 0, -1)
    const double v20 = val(6, b + (0 * sI + -1 * sJ + -1));  // w (0, -1, -1)
    const double v21 = val(6, b + (0 * sI + 0 * sJ + -1));  // w (0, 0, -1)
    const double v22 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    const double v23 = val(6, b + (0 * sI + 1 * sJ + -1));  // w (0, 1, -1)
    const double v24 = val(6, b + (1 * sI + 0 * sJ + -1));  // w (1, 0, -1)
    bar[0] += l1 * -C.az * v21;  // RU
    bar[1] += l2 * -C.az * v21;  // RV
    bar[2] += l0 * -C.az + l3 * -C.az * v21;  // RW
    bar[3] += l4 * -C.az * v21;  // RE
    bar[4] += l1 * C.xm_zz * v8 + l1 * C.xm_zz * v9 + l4 * -C.e_zz12 * v8 * v13 + l4 * C.e_zz12 * v8 * v12 + l4 * C.e_zz12 * v8 * v12 + l4 * C.e_zz12 * v9 * v13 + l4 * -C.e_zx4 * v8 * v24 + l4 * C.e_zx4 * v8 * v19;  // u
    bar[5] += l2 * C.ym_zz * v8 + l2 * C.ym_zz * v9 + l4 * -C.e_zz12 * v8 * v17 + l4 * C.e_zz12 * v8 * v16 + l4 * C.e_zz12 * v8 * v16 + l4 * C.e_zz12 * v9 * v17 + l4 * -C.e_zy4 * v8 * v23 + l4 * C.e_zy4 * v8 * v20;  // v
    bar[6] += l1 * -C.az * v1 + l2 * -C.az * v2 + l3 * -C.az * v3 + l3 * C.zm_zz * v8 + l3 * C.zm_zz * v9 + l4 * -C.az * C.h0 + l4 * -C.az * v0 + l4 * -C.az * v10 + l4 * -C.e_zz23 * v8 * v22 + l4 * C.e_zz23 * v8 * v21 + l4 * C.e_zz23 * v8 * v21 + l4 * C.e_zz23 * v9 * v22 + l4 * -C.e_zx6 * v8 * v14 + l4 * C.e_zx6 * v8 * v11 + l4 * -C.e_zy6 * v8 * v18 + l4 * C.e_zy6 * v8 * v15;  // w
    bar[7] += l3 * -C.az + l4 * -C.az * v21;  // p
    bar[8] += l4 * C.e_zz12 * v6 + l4 * C.e_zz12 * v7;  // T
    bar[9] += l1 * -C.xm_zz * v13 + l1 * C.xm_zz * v12 + l1 * -C.xm_xz * v24 + l1 * C.xm_xz * v19 + l2 * -C.ym_zz * v17 + l2 * C.ym_zz * v16 + l2 * -C.ym_yz * v23 + l2 * C.ym_yz * v20 + l3 * -C.zm_zz * v22 + l3 * C.zm_zz * v21 + l3 * -C.zm_xz * v14 + l3 * C.zm_xz * v11 + l3 * -C.zm_yz * v18 + l3 * C.zm_yz * v15 + l4 * -C.e_zz12 * v12 * v13 + l4 * C.e_zz12 * v12 * v12 + l4 * -C.e_zz12 * v16 * v17 + l4 * C.e_zz12 * v16 * v16 + l4 * -C.e_zz23 * v21 * v22 + l4 * C.e_zz23 * v21 * v21 + l4 * -C.e_zx6 * v14 * v21 + l4 * C.e_zx6 * v11 * v21 + l4 * -C.e_zy6 * v18 * v21 + l4 * C.e_zy6 * v15 * v21 + l4 * -C.e_zx4 * v12 * v24 + l4 * C.e_zx4 * v12 * v19 + l4 * -C.e_zy4 * v16 * v23 + l4 * C.e_zy4 * v16 * v20;  // mu
    bar[10] += l4 * -C.e_zz12 * v5 + l4 * C.e_zz12 * v4;  // ka
  }
  if (inner(0, 0, 0)) {
    const long long b = X - (0 * sI + 0 * sJ + 0);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(8, b + (-1 * sI + 0 * sJ + 0));  // T (-1, 0, 0)
    const double v1 = val(8, b + (0 * sI + -1 * sJ + 0));  // T (0, -1, 0)
    const double v2 = val(8, b + (0 * sI + 0 * sJ + -1));  // T (0, 0, -1)
    const double v3 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v4 = val(8, b + (0 * sI + 0 * sJ + 1));  // T (0, 0, 1)
    const double v5 = val(8, b + (0 * sI + 1 * sJ + 0));  // T (0, 1, 0)
    const double v6 = val(8, b + (1 * sI + 0 * sJ + 0));  // T (1, 0, 0)
    const double v7 = val(10, b + (-1 * sI + 0 * sJ + 0));  // ka (-1, 0, 0)
    const double v8 = val(10, b + (0 * sI + -1 * sJ + 0));  // ka (0, -1, 0)
    const double v9 = val(10, b + (0 * sI + 0 * sJ + -1));  // ka (0, 0, -1)
    const double v10 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v11 = val(10, b + (0 * sI + 0 * sJ + 1));  // ka (0, 0, 1)
    const double v12 = val(10, b + (0 * sI + 1 * sJ + 0));  // ka (0, 1, 0)
    const double v13 = val(10, b + (1 * sI + 0 * sJ + 0));  // ka (1, 0, 0)
    const double v14 = val(9, b + (-1 * sI + 0 * sJ + 0));  // mu (-1, 0, 0)
    const double v15 = val(9, b + (0 * sI + -1 * sJ + 0));  // mu (0, -1, 0)
    const double v16 = val(9, b + (0 * sI + 0 * sJ + -1));  // mu (0, 0, -1)
    const double v17 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v18 = val(9, b + (0 * sI + 0 * sJ + 1));  // mu (0, 0, 1)
    const double v19 = val(9, b + (0 * sI + 1 * sJ + 0));  // mu (0, 1, 0)
    const double v20 = val(9, b + (1 * sI + 0 * sJ + 0));  // mu (1, 0, 0)
    const double v21 = val(4, b + (-1 * sI + 0 * sJ + 0));  // u (-1, 0, 0)
    const double v22 = val(4, b + (0 * sI + -1 * sJ + 0));  // u (0, -1, 0)
    const double v23 = val(4, b + (0 * sI + 0 * sJ + -1));  // u (0, 0, -1)
    const double v24 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v25 = val(4, b + (0 * sI + 0 * sJ + 1));  // u (0, 0, 1)
    const double v26 = val(4, b + (0 * sI + 1 * sJ + 0));  // u (0, 1, 0)
    const double v27 = val(4, b + (1 * sI + 0 * sJ + 0));  // u (1, 0, 0)
    const double v28 = val(5, b + (-1 * sI + 0 * sJ + 0));  // v (-1, 0, 0)
    const double v29 = val(5, b + (0 * sI + -1 * sJ + 0));  // v (0, -1, 0)
    const double v30 = val(5, b + (0 * sI + 0 * sJ + -1));  // v (0, 0, -1)
    const double v31 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v32 = val(5, b + (0 * sI + 0 * sJ + 1));  // v (0, 0, 1)
    const double v33 = val(5, b + (0 * sI + 1 * sJ + 0));  // v (0, 1, 0)
    const double v34 = val(5, b + (1 * sI + 0 * sJ + 0));  // v (1, 0, 0)
    const double v35 = val(6, b + (-1 * sI + 0 * sJ + 0));  // w (-1, 0, 0)
    const double v36 = val(6, b + (0 * sI + -1 * sJ + 0));  // w (0, -1, 0)
    const double v37 = val(6, b + (0 * sI + 0 * sJ + -1));  // w (0, 0, -1)
    const double v38 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    const double v39 = val(6, b + (0 * sI + 0 * sJ + 1));  // w (0, 0, 1)
    const double v40 = val(6, b + (0 * sI + 1 * sJ + 0));  // w (0, 1, 0)
    const double v41 = val(6, b + (1 * sI + 0 * sJ + 0));  // w (1, 0, 0)
    bar[4] += l1 * -C.xm_xx * v20 + l1 * (-2.0 * C.xm_xx + -2.0 * C.xm_yy + -2.0 * C.xm_zz) * v17 + l1 * -C.xm_xx * v14 + l1 * -C.xm_yy * v19 + l1 * -C.xm_yy * v15 + l1 * -C.xm_zz * v18 + l1 * -C.xm_zz * v16 + l4 * -C.e_xx23 * v20 * v27 + l4 * C.e_xx23 * v17 * v27 + l4 * (-2.0 * C.e_xx23 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * v17 * v24 + l4 * (-2.0 * C.e_xx23 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * v17 * v24 + l4 * -C.e_xx23 * v14 * v21 + l4 * C.e_xx23 * v17 * v21 + l4 * -C.e_yy12 * v19 * v26 + l4 * C.e_yy12 * v17 * v26 + l4 * -C.e_yy12 * v15 * v22 + l4 * C.e_yy12 * v17 * v22 + l4 * -C.e_zz12 * v18 * v25 + l4 * C.e_zz12 * v17 * v25 + l4 * -C.e_zz12 * v16 * v23 + l4 * C.e_zz12 * v17 * v23;  // u
    bar[5] += l2 * -C.ym_xx * v20 + l2 * (-2.0 * C.ym_xx + -2.0 * C.ym_yy + -2.0 * C.ym_zz) * v17 + l2 * -C.ym_xx * v14 + l2 * -C.ym_yy * v19 + l2 * -C.ym_yy * v15 + l2 * -C.ym_zz * v18 + l2 * -C.ym_zz * v16 + l4 * -C.e_xx12 * v20 * v34 + l4 * C.e_xx12 * v17 * v34 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy23 + -2.0 * C.e_zz12) * v17 * v31 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy23 + -2.0 * C.e_zz12) * v17 * v31 + l4 * -C.e_xx12 * v14 * v28 + l4 * C.e_xx12 * v17 * v28 + l4 * -C.e_yy23 * v19 * v33 + l4 * C.e_yy23 * v17 * v33 + l4 * -C.e_yy23 * v15 * v29 + l4 * C.e_yy23 * v17 * v29 + l4 * -C.e_zz12 * v18 * v32 + l4 * C.e_zz12 * v17 * v32 + l4 * -C.e_zz12 * v16 * v30 + l4 * C.e_zz12 * v17 * v30;  // v
    bar[6] += l3 * -C.zm_xx * v20 + l3 * (-2.0 * C.zm_xx + -2.0 * C.zm_yy + -2.0 * C.zm_zz) * v17 + l3 * -C.zm_xx * v14 + l3 * -C.zm_yy * v19 + l3 * -C.zm_yy * v15 + l3 * -C.zm_zz * v18 + l3 * -C.zm_zz * v16 + l4 * -C.e_xx12 * v20 * v41 + l4 * C.e_xx12 * v17 * v41 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz23) * v17 * v38 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz23) * v17 * v38 + l4 * -C.e_xx12 * v14 * v35 + l4 * C.e_xx12 * v17 * v35 + l4 * -C.e_yy12 * v19 * v40 + l4 * C.e_yy12 * v17 * v40 + l4 * -C.e_yy12 * v15 * v36 + l4 * C.e_yy12 * v17 * v36 + l4 * -C.e_zz23 * v18 * v39 + l4 * C.e_zz23 * v17 * v39 + l4 * -C.e_zz23 * v16 * v37 + l4 * C.e_zz23 * v17 * v37;  // w
    bar[8] += l4 * -C.e_xx12 * v13 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * v10 + l4 * -C.e_xx12 * v7 + l4 * -C.e_yy12 * v12 + l4 * -C.e_yy12 * v8 + l4 * -C.e_zz12 * v11 + l4 * -C.e_zz12 * v9;  // T
    bar[9] += l1 * C.xm_xx * v27 + l1 * (-2.0 * C.xm_xx + -2.0 * C.xm_yy + -2.0 * C.xm_zz) * v24 + l1 * C.xm_xx * v21 + l1 * C.xm_yy * v26 + l1 * C.xm_yy * v22 + l1 * C.xm_zz * v25 + l1 * C.xm_zz * v23 + l2 * C.ym_xx * v34 + l2 * (-2.0 * C.ym_xx + -2.0 * C.ym_yy + -2.0 * C.ym_zz) * v31 + l2 * C.ym_xx * v28 + l2 * C.ym_yy * v33 + l2 * C.ym_yy * v29 + l2 * C.ym_zz * v32 + l2 * C.ym_zz * v30 + l3 * C.zm_xx * v41 + l3 * (-2.0 * C.zm_xx + -2.0 * C.zm_yy + -2.0 * C.zm_zz) * v38 + l3 * C.zm_xx * v35 + l3 * C.zm_yy * v40 + l3 * C.zm_yy * v36 + l3 * C.zm_zz * v39 + l3 * C.zm_zz * v37 + l4 * C.e_xx23 * v24 * v27 + l4 * (-2.0 * C.e_xx23 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * v24 * v24 + l4 * C.e_xx23 * v21 * v24 + l4 * C.e_xx12 * v31 * v34 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy23 + -2.0 * C.e_zz12) * v31 * v31 + l4 * C.e_xx12 * v28 * v31 + l4 * C.e_xx12 * v38 * v41 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz23) * v38 * v38 + l4 * C.e_xx12 * v35 * v38 + l4 * C.e_yy12 * v24 * v26 + l4 * C.e_yy12 * v22 * v24 + l4 * C.e_yy23 * v31 * v33 + l4 * C.e_yy23 * v29 * v31 + l4 * C.e_yy12 * v38 * v40 + l4 * C.e_yy12 * v36 * v38 + l4 * C.e_zz12 * v24 * v25 + l4 * C.e_zz12 * v23 * v24 + l4 * C.e_zz12 * v31 * v32 + l4 * C.e_zz12 * v30 * v31 + l4 * C.e_zz23 * v38 * v39 + l4 * C.e_zz23 * v37 * v38;  // mu
    bar[10] += l4 * C.e_xx12 * v6 + l4 * (-2.0 * C.e_xx12 + -2.0 * C.e_yy12 + -2.0 * C.e_zz12) * v3 + l4 * C.e_xx12 * v0 + l4 * C.e_yy12 * v5 + l4 * C.e_yy12 * v1 + l4 * C.e_zz12 * v4 + l4 * C.e_zz12 * v2;  // ka
  }
  if (inner(0, 0, 1)) {
    const long long b = X - (0 * sI + 0 * sJ + 1);
    const double l0 = lam(0, b);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(3, b + (0 * sI + 0 * sJ + 1));  // RE (0, 0, 1)
    const double v1 = val(0, b + (0 * sI + 0 * sJ + 1));  // RU (0, 0, 1)
    const double v2 = val(1, b + (0 * sI + 0 * sJ + 1));  // RV (0, 0, 1)
    const double v3 = val(2, b + (0 * sI + 0 * sJ + 1));  // RW (0, 0, 1)
    const double v4 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v5 = val(8, b + (0 * sI + 0 * sJ + 1));  // T (0, 0, 1)
    const double v6 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v7 = val(10, b + (0 * sI + 0 * sJ + 1));  // ka (0, 0, 1)
    const double v8 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v9 = val(9, b + (0 * sI + 0 * sJ + 1));  // mu (0, 0, 1)
    const double v10 = val(7, b + (0 * sI + 0 * sJ + 1));  // p (0, 0, 1)
    const double v11 = val(4, b + (-1 * sI + 0 * sJ + 1));  // u (-1, 0, 1)
    const double v12 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v13 = val(4, b + (0 * sI + 0 * sJ + 1));  // u (0, 0, 1)
    const double v14 = val(4, b + (1 * sI + 0 * sJ + 1));  // u (1, 0, 1)
    const double v15 = val(5, b + (0 * sI + -1 * sJ + 1));  // v (0, -1, 1)
    const double v16 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v17 = val(5, b + (0 * sI + 0 * sJ + 1));  // v (0, 0, 1)
    const double v18 = val(5, b + (0 * sI + 1 * sJ + 1));  // v (0, 1, 1)
    const double v19 = val(6, b + (-1 * sI + 0 * sJ + 1));  // w (-1, 0, 1)
    const double v20 = val(6, b + (0 * sI + -1 * sJ + 1));  // w (0, -1, 1)
    const double v21 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    const double v22 = val(6, b + (0 * sI + 0 * sJ + 1));  // w (0, 0, 1)
    const double v23 = val(6, b + (0 * sI + 1 * sJ + 1));  // w (0, 1, 1)
    const double v24 = val(6, b + (1 * sI + 0 * sJ + 1));  // w (1, 0, 1)
    bar[0] += l1 * C.az * v22;  // RU
    bar[1] += l2 * C.az * v22;  // RV
    bar[2] += l0 * C.az + l3 * C.az * v22;  // RW
    bar[3] += l4 * C.az * v22;  // RE
    bar[4] += l1 * C.xm_zz * v9 + l1 * C.xm_zz * v8 + l4 * C.e_zz12 * v9 * v13 + l4 * C.e_zz12 * v9 * v13 + l4 * -C.e_zz12 * v9 * v12 + l4 * C.e_zz12 * v8 * v12 + l4 * C.e_zx4 * v9 * v24 + l4 * -C.e_zx4 * v9 * v19;  // u
    bar[5] += l2 * C.ym_zz * v9 + l2 * C.ym_zz * v8 + l4 * C.e_zz12 * v9 * v17 + l4 * C.e_zz12 * v9 * v17 + l4 * -C.e_zz12 * v9 * v16 + l4 * C.e_zz12 * v8 * v16 + l4 * C.e_zy4 * v9 * v23 + l4 * -C.e_zy4 * v9 * v20;  // v
    bar[6] += l1 * C.az * v1 + l2 * C.az * v2 + l3 * C.az * v3 + l3 * C.zm_zz * v9 + l3 * C.zm_zz * v8 + l4 * C.az * C.h0 + l4 * C.az * v0 + l4 * C.az * v10 + l4 * C.e_zz23 * v9 * v22 + l4 * C.e_zz23 * v9 * v22 + l4 * -C.e_zz23 * v9 * v21 + l4 * C.e_zz23 * v8 * v21 + l4 * C.e_zx6 * v9 * v14 + l4 * -C.e_zx6 * v9 * v11 + l4 * C.e_zy6 * v9 * v18 + l4 * -C.e_zy6 * v9 * v15;  // w
    bar[7] += l3 * C.az + l4 * C.az * v22;  // p
    bar[8] += l4 * C.e_zz12 * v7 + l4 * C.e_zz12 * v6;  // T
    bar[9] += l1 * C.xm_zz * v13 + l1 * -C.xm_zz * v12 + l1 * C.xm_xz * v24 + l1 * -C.xm_xz * v19 + l2 * C.ym_zz * v17 + l2 * -C.ym_zz * v16 + l2 * C.ym_yz * v23 + l2 * -C.ym_yz * v20 + l3 * C.zm_zz * v22 + l3 * -C.zm_zz * v21 + l3 * C.zm_xz * v14 + l3 * -C.zm_xz * v11 + l3 * C.zm_yz * v18 + l3 * -C.zm_yz * v15 + l4 * C.e_zz12 * v13 * v13 + l4 * -C.e_zz12 * v12 * v13 + l4 * C.e_zz12 * v17 * v17 + l4 * -C.e_zz12 * v16 * v17 + l4 * C.e_zz23 * v22 * v22 + l4 * -C.e_zz23 * v21 * v22 + l4 * C.e_zx6 * v14 * v22 + l4 * -C.e_zx6 * v11 * v22 + l4 * C.e_zy6 * v18 * v22 + l4 * -C.e_zy6 * v15 * v22 + l4 * C.e_zx4 * v13 * v24 + l4 * -C.e_zx4 * v13 * v19 + l4 * C.e_zy4 * v17 * v23 + l4 * -C.e_zy4 * v17 * v20;  // mu
    bar[10] += l4 * C.e_zz12 * v5 + l4 * -C.e_zz12 * v4;  // ka
  }
  if (inner(0, 1, -1)) {
    const long long b = X - (0 * sI + 1 * sJ + -1);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + 0 * sJ + -1));  // mu (0, 0, -1)
    const double v1 = val(9, b + (0 * sI + 1 * sJ + 0));  // mu (0, 1, 0)
    const double v2 = val(5, b + (0 * sI + 0 * sJ + -1));  // v (0, 0, -1)
    const double v3 = val(5, b + (0 * sI + 1 * sJ + 0));  // v (0, 1, 0)
    const double v4 = val(6, b + (0 * sI + 0 * sJ + -1));  // w (0, 0, -1)
    const double v5 = val(6, b + (0 * sI + 1 * sJ + 0));  // w (0, 1, 0)
    bar[5] += l3 * -C.zm_zy * v1 + l3 * -C.zm_yz * v0 + l4 * -C.e_zy4 * v1 * v5 + l4 * -C.e_zy6 * v0 * v4;  // v
    bar[6] += l2 * -C.ym_yz * v0 + l2 * -C.ym_zy * v1 + l4 * -C.e_zy6 * v1 * v3 + l4 * -C.e_zy4 * v0 * v2;  // w
  }
  if (inner(0, 1, 0)) {
    const long long b = X - (0 * sI + 1 * sJ + 0);
    const double l0 = lam(0, b);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(3, b + (0 * sI + 1 * sJ + 0));  // RE (0, 1, 0)
    const double v1 = val(0, b + (0 * sI + 1 * sJ + 0));  // RU (0, 1, 0)
    const double v2 = val(1, b + (0 * sI + 1 * sJ + 0));  // RV (0, 1, 0)
    const double v3 = val(2, b + (0 * sI + 1 * sJ + 0));  // RW (0, 1, 0)
    const double v4 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v5 = val(8, b + (0 * sI + 1 * sJ + 0));  // T (0, 1, 0)
    const double v6 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v7 = val(10, b + (0 * sI + 1 * sJ + 0));  // ka (0, 1, 0)
    const double v8 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v9 = val(9, b + (0 * sI + 1 * sJ + 0));  // mu (0, 1, 0)
    const double v10 = val(7, b + (0 * sI + 1 * sJ + 0));  // p (0, 1, 0)
    const double v11 = val(4, b + (-1 * sI + 1 * sJ + 0));  // u (-1, 1, 0)
    const double v12 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v13 = val(4, b + (0 * sI + 1 * sJ + 0));  // u (0, 1, 0)
    const double v14 = val(4, b + (1 * sI + 1 * sJ + 0));  // u (1, 1, 0)
    const double v15 = val(5, b + (-1 * sI + 1 * sJ + 0));  // v (-1, 1, 0)
    const double v16 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v17 = val(5, b + (0 * sI + 1 * sJ + -1));  // v (0, 1, -1)
    const double v18 = val(5, b + (0 * sI + 1 * sJ + 0));  // v (0, 1, 0)
    const double v19 = val(5, b + (0 * sI + 1 * sJ + 1));  // v (0, 1, 1)
    const double v20 = val(5, b + (1 * sI + 1 * sJ + 0));  // v (1, 1, 0)
    const double v21 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    const double v22 = val(6, b + (0 * sI + 1 * sJ + -1));  // w (0, 1, -1)
    const double v23 = val(6, b + (0 * sI + 1 * sJ + 0));  // w (0, 1, 0)
    const double v24 = val(6, b + (0 * sI + 1 * sJ + 1));  // w (0, 1, 1)
    bar[0] += l1 * C.ay * v18;  // RU
    bar[1] += l0 * C.ay + l2 * C.ay * v18;  // RV
    bar[2] += l3 * C.ay * v18;  // RW
    bar[3] += l4 * C.ay * v18;  // RE
    bar[4] += l1 * C.xm_yy * v9 + l1 * C.xm_yy * v8 + l4 * C.e_yy12 * v9 * v13 + l4 * C.e_yy12 * v9 * v13 + l4 * -C.e_yy12 * v9 * v12 + l4 * C.e_yy12 * v8 * v12 + l4 * C.e_yx4 * v9 * v20 + l4 * -C.e_yx4 * v9 * v15;  // u
    bar[5] += l1 * C.ay * v1 + l2 * C.ay * v2 + l2 * C.ym_yy * v9 + l2 * C.ym_yy * v8 + l3 * C.ay * v3 + l4 * C.ay * C.h0 + l4 * C.ay * v0 + l4 * C.ay * v10 + l4 * C.e_yy23 * v9 * v18 + l4 * C.e_yy23 * v9 * v18 + l4 * -C.e_yy23 * v9 * v16 + l4 * C.e_yy23 * v8 * v16 + l4 * C.e_yx6 * v9 * v14 + l4 * -C.e_yx6 * v9 * v11 + l4 * C.e_zy6 * v9 * v24 + l4 * -C.e_zy6 * v9 * v22;  // v
    bar[6] += l3 * C.zm_yy * v9 + l3 * C.zm_yy * v8 + l4 * C.e_yy12 * v9 * v23 + l4 * C.e_yy12 * v9 * v23 + l4 * -C.e_yy12 * v9 * v21 + l4 * C.e_yy12 * v8 * v21 + l4 * C.e_zy4 * v9 * v19 + l4 * -C.e_zy4 * v9 * v17;  // w
    bar[7] += l2 * C.ay + l4 * C.ay * v18;  // p
    bar[8] += l4 * C.e_yy12 * v7 + l4 * C.e_yy12 * v6;  // T
    bar[9] += l1 * C.xm_yy * v13 + l1 * -C.xm_yy * v12 + l1 * C.xm_xy * v20 + l1 * -C.xm_xy * v15 + l2 * C.ym_yy * v18 + l2 * -C.ym_yy * v16 + l2 * C.ym_xy * v14 + l2 * -C.ym_xy * v11 + l2 * C.ym_zy * v24 + l2 * -C.ym_zy * v22 + l3 * C.zm_yy * v23 + l3 * -C.zm_yy * v21 + l3 * C.zm_zy * v19 + l3 * -C.zm_zy * v17 + l4 * C.e_yy12 * v13 * v13 + l4 * -C.e_yy12 * v12 * v13 + l4 * C.e_yy23 * v18 * v18 + l4 * -C.e_yy23 * v16 * v18 + l4 * C.e_yy12 * v23 * v23 + l4 * -C.e_yy12 * v21 * v23 + l4 * C.e_yx6 * v14 * v18 + l4 * -C.e_yx6 * v11 * v18 + l4 * C.e_zy6 * v18 * v24 + l4 * -C.e_zy6 * v18 * v22 + l4 * C.e_yx4 * v13 * v20 + l4 * -C.e_yx4 * v13 * v15 + l4 * C.e_zy4 * v19 * v23 + l4 * -C.e_zy4 * v17 * v23;  // mu
    bar[10] += l4 * C.e_yy12 * v5 + l4 * -C.e_yy12 * v4;  // ka
  }
  if (inner(0, 1, 1)) {
    const long long b = X - (0 * sI + 1 * sJ + 1);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + 0 * sJ + 1));  // mu (0, 0, 1)
    const double v1 = val(9, b + (0 * sI + 1 * sJ + 0));  // mu (0, 1, 0)
    const double v2 = val(5, b + (0 * sI + 0 * sJ + 1));  // v (0, 0, 1)
    const double v3 = val(5, b + (0 * sI + 1 * sJ + 0));  // v (0, 1, 0)
    const double v4 = val(6, b + (0 * sI + 0 * sJ + 1));  // w (0, 0, 1)
    const double v5 = val(6, b + (0 * sI + 1 * sJ + 0));  // w (0, 1, 0)
    bar[5] += l3 * C.zm_zy * v1 + l3 * C.zm_yz * v0 + l4 * C.e_zy4 * v1 * v5 + l4 * C.e_zy6 * v0 * v4;  // v
    bar[6] += l2 * C.ym_yz * v0 + l2 * C.ym_zy * v1 + l4 * C.e_zy6 * v1 * v3 + l4 * C.e_zy4 * v0 * v2;  // w
  }
  if (inner(1, -1, 0)) {
    const long long b = X - (1 * sI + -1 * sJ + 0);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + -1 * sJ + 0));  // mu (0, -1, 0)
    const double v1 = val(9, b + (1 * sI + 0 * sJ + 0));  // mu (1, 0, 0)
    const double v2 = val(4, b + (0 * sI + -1 * sJ + 0));  // u (0, -1, 0)
    const double v3 = val(4, b + (1 * sI + 0 * sJ + 0));  // u (1, 0, 0)
    const double v4 = val(5, b + (0 * sI + -1 * sJ + 0));  // v (0, -1, 0)
    const double v5 = val(5, b + (1 * sI + 0 * sJ + 0));  // v (1, 0, 0)
    bar[4] += l2 * -C.ym_yx * v1 + l2 * -C.ym_xy * v0 + l4 * -C.e_yx4 * v1 * v5 + l4 * -C.e_yx6 * v0 * v4;  // u
    bar[5] += l1 * -C.xm_xy * v0 + l1 * -C.xm_yx * v1 + l4 * -C.e_yx6 * v1 * v3 + l4 * -C.e_yx4 * v0 * v2;  // v
  }
  if (inner(1, 0, -1)) {
    const long long b = X - (1 * sI + 0 * sJ + -1);
    const double l1 = lam(1, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + 0 * sJ + -1));  // mu (0, 0, -1)
    const double v1 = val(9, b + (1 * sI + 0 * sJ + 0));  // mu (1, 0, 0)
    const double v2 = val(4, b + (0 * sI + 0 * sJ + -1));  // u (0, 0, -1)
    const double v3 = val(4, b + (1 * sI + 0 * sJ + 0));  // u (1, 0, 0)
    const double v4 = val(6, b + (0 * sI + 0 * sJ + -1));  // w (0, 0, -1)
    const double v5 = val(6, b + (1 * sI + 0 * sJ + 0));  // w (1, 0, 0)
    bar[4] += l3 * -C.zm_zx * v1 + l3 * -C.zm_xz * v0 + l4 * -C.e_zx4 * v1 * v5 + l4 * -C.e_zx6 * v0 * v4;  // u
    bar[6] += l1 * -C.xm_xz * v0 + l1 * -C.xm_zx * v1 + l4 * -C.e_zx6 * v1 * v3 + l4 * -C.e_zx4 * v0 * v2;  // w
  }
  if (inner(1, 0, 0)) {
    const long long b = X - (1 * sI + 0 * sJ + 0);
    const double l0 = lam(0, b);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(3, b + (1 * sI + 0 * sJ + 0));  // RE (1, 0, 0)
    const double v1 = val(0, b + (1 * sI + 0 * sJ + 0));  // RU (1, 0, 0)
    const double v2 = val(1, b + (1 * sI + 0 * sJ + 0));  // RV (1, 0, 0)
    const double v3 = val(2, b + (1 * sI + 0 * sJ + 0));  // RW (1, 0, 0)
    const double v4 = val(8, b + (0 * sI + 0 * sJ + 0));  // T (0, 0, 0)
    const double v5 = val(8, b + (1 * sI + 0 * sJ + 0));  // T (1, 0, 0)
    const double v6 = val(10, b + (0 * sI + 0 * sJ + 0));  // ka (0, 0, 0)
    const double v7 = val(10, b + (1 * sI + 0 * sJ + 0));  // ka (1, 0, 0)
    const double v8 = val(9, b + (0 * sI + 0 * sJ + 0));  // mu (0, 0, 0)
    const double v9 = val(9, b + (1 * sI + 0 * sJ + 0));  // mu (1, 0, 0)
    const double v10 = val(7, b + (1 * sI + 0 * sJ + 0));  // p (1, 0, 0)
    const double v11 = val(4, b + (0 * sI + 0 * sJ + 0));  // u (0, 0, 0)
    const double v12 = val(4, b + (1 * sI + -1 * sJ + 0));  // u (1, -1, 0)
    const double v13 = val(4, b + (1 * sI + 0 * sJ + -1));  // u (1, 0, -1)
    const double v14 = val(4, b + (1 * sI + 0 * sJ + 0));  // u (1, 0, 0)
    const double v15 = val(4, b + (1 * sI + 0 * sJ + 1));  // u (1, 0, 1)
    const double v16 = val(4, b + (1 * sI + 1 * sJ + 0));  // u (1, 1, 0)
    const double v17 = val(5, b + (0 * sI + 0 * sJ + 0));  // v (0, 0, 0)
    const double v18 = val(5, b + (1 * sI + -1 * sJ + 0));  // v (1, -1, 0)
    const double v19 = val(5, b + (1 * sI + 0 * sJ + 0));  // v (1, 0, 0)
    const double v20 = val(5, b + (1 * sI + 1 * sJ + 0));  // v (1, 1, 0)
    const double v21 = val(6, b + (0 * sI + 0 * sJ + 0));  // w (0, 0, 0)
    const double v22 = val(6, b + (1 * sI + 0 * sJ + -1));  // w (1, 0, -1)
    const double v23 = val(6, b + (1 * sI + 0 * sJ + 0));  // w (1, 0, 0)
    const double v24 = val(6, b + (1 * sI + 0 * sJ + 1));  // w (1, 0, 1)
    bar[0] += l0 * C.ax + l1 * C.ax * v14;  // RU
    bar[1] += l2 * C.ax * v14;  // RV
    bar[2] += l3 * C.ax * v14;  // RW
    bar[3] += l4 * C.ax * v14;  // RE
    bar[4] += l1 * C.ax * v1 + l1 * C.xm_xx * v9 + l1 * C.xm_xx * v8 + l2 * C.ax * v2 + l3 * C.ax * v3 + l4 * C.ax * C.h0 + l4 * C.ax * v0 + l4 * C.ax * v10 + l4 * C.e_xx23 * v9 * v14 + l4 * C.e_xx23 * v9 * v14 + l4 * -C.e_xx23 * v9 * v11 + l4 * C.e_xx23 * v8 * v11 + l4 * C.e_yx6 * v9 * v20 + l4 * -C.e_yx6 * v9 * v18 + l4 * C.e_zx6 * v9 * v24 + l4 * -C.e_zx6 * v9 * v22;  // u
    bar[5] += l2 * C.ym_xx * v9 + l2 * C.ym_xx * v8 + l4 * C.e_xx12 * v9 * v19 + l4 * C.e_xx12 * v9 * v19 + l4 * -C.e_xx12 * v9 * v17 + l4 * C.e_xx12 * v8 * v17 + l4 * C.e_yx4 * v9 * v16 + l4 * -C.e_yx4 * v9 * v12;  // v
    bar[6] += l3 * C.zm_xx * v9 + l3 * C.zm_xx * v8 + l4 * C.e_xx12 * v9 * v23 + l4 * C.e_xx12 * v9 * v23 + l4 * -C.e_xx12 * v9 * v21 + l4 * C.e_xx12 * v8 * v21 + l4 * C.e_zx4 * v9 * v15 + l4 * -C.e_zx4 * v9 * v13;  // w
    bar[7] += l1 * C.ax + l4 * C.ax * v14;  // p
    bar[8] += l4 * C.e_xx12 * v7 + l4 * C.e_xx12 * v6;  // T
    bar[9] += l1 * C.xm_xx * v14 + l1 * -C.xm_xx * v11 + l1 * C.xm_yx * v20 + l1 * -C.xm_yx * v18 + l1 * C.xm_zx * v24 + l1 * -C.xm_zx * v22 + l2 * C.ym_xx * v19 + l2 * -C.ym_xx * v17 + l2 * C.ym_yx * v16 + l2 * -C.ym_yx * v12 + l3 * C.zm_xx * v23 + l3 * -C.zm_xx * v21 + l3 * C.zm_zx * v15 + l3 * -C.zm_zx * v13 + l4 * C.e_xx23 * v14 * v14 + l4 * -C.e_xx23 * v11 * v14 + l4 * C.e_xx12 * v19 * v19 + l4 * -C.e_xx12 * v17 * v19 + l4 * C.e_xx12 * v23 * v23 + l4 * -C.e_xx12 * v21 * v23 + l4 * C.e_yx6 * v14 * v20 + l4 * -C.e_yx6 * v14 * v18 + l4 * C.e_zx6 * v14 * v24 + l4 * -C.e_zx6 * v14 * v22 + l4 * C.e_yx4 * v16 * v19 + l4 * -C.e_yx4 * v12 * v19 + l4 * C.e_zx4 * v15 * v23 + l4 * -C.e_zx4 * v13 * v23;  // mu
    bar[10] += l4 * C.e_xx12 * v5 + l4 * -C.e_xx12 * v4;  // ka
  }
  if (inner(1, 0, 1)) {
    const long long b = X - (1 * sI + 0 * sJ + 1);
    const double l1 = lam(1, b);
    const double l3 = lam(3, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + 0 * sJ + 1));  // mu (0, 0, 1)
    const double v1 = val(9, b + (1 * sI + 0 * sJ + 0));  // mu (1, 0, 0)
    const double v2 = val(4, b + (0 * sI + 0 * sJ + 1));  // u (0, 0, 1)
    const double v3 = val(4, b + (1 * sI + 0 * sJ + 0));  // u (1, 0, 0)
    const double v4 = val(6, b + (0 * sI + 0 * sJ + 1));  // w (0, 0, 1)
    const double v5 = val(6, b + (1 * sI + 0 * sJ + 0));  // w (1, 0, 0)
    bar[4] += l3 * C.zm_zx * v1 + l3 * C.zm_xz * v0 + l4 * C.e_zx4 * v1 * v5 + l4 * C.e_zx6 * v0 * v4;  // u
    bar[6] += l1 * C.xm_xz * v0 + l1 * C.xm_zx * v1 + l4 * C.e_zx6 * v1 * v3 + l4 * C.e_zx4 * v0 * v2;  // w
  }
  if (inner(1, 1, 0)) {
    const long long b = X - (1 * sI + 1 * sJ + 0);
    const double l1 = lam(1, b);
    const double l2 = lam(2, b);
    const double l4 = lam(4, b);
    const double v0 = val(9, b + (0 * sI + 1 * sJ + 0));  // mu (0, 1, 0)
    const double v1 = val(9, b + (1 * sI + 0 * sJ + 0));  // mu (1, 0, 0)
    const double v2 = val(4, b + (0 * sI + 1 * sJ + 0));  // u (0, 1, 0)
    const double v3 = val(4, b + (1 * sI + 0 * sJ + 0));  // u (1, 0, 0)
    const double v4 = val(5, b + (0 * sI + 1 * sJ + 0));  // v (0, 1, 0)
    const double v5 = val(5, b + (1 * sI + 0 * sJ + 0));  // v (1, 0, 0)
    bar[4] += l2 * C.ym_yx * v1 + l2 * C.ym_xy * v0 + l4 * C.e_yx4 * v1 * v5 + l4 * C.e_yx6 * v0 * v4;  // u
    bar[5] += l1 * C.xm_xy * v0 + l1 * C.xm_yx * v1 + l4 * C.e_yx6 * v1 * v3 + l4 * C.e_yx4 * v0 * v2;  // v
  }
}

}  // namespace nsf
#endif
