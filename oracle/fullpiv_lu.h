// Oracle test infrastructure only. Dense LU with complete pivoting for the small (8x8) Vandermonde
// systems of the reference's image-point interpolation (Boundary.cpp:820-834 calls
// Eigen::FullPivLU::solve). Eigen is not installed on this image, so this textbook version
// (Golub & Van Loan, "Matrix Computations", 4th ed., Algorithm 3.4.2: Gaussian elimination with
// complete pivoting; then P*b, unit-lower forward substitution, upper back substitution, Q*c) stands in
// for it. Pivot choice: largest |a_ij| of the trailing block, first hit in column-major order.
// Results agree with Eigen's to rounding (a few ulp times the system's condition number); they are not
// pinned bit-for-bit against Eigen.
#ifndef ORACLE_FULLPIV_LU_H
#define ORACLE_FULLPIV_LU_H
#include <cmath>
#include <limits>

namespace oracle_lu {

template <int N>
struct FullPivLU {
  double lu[N][N];  // lu[row][col]
  int rowT[N];      // row transposition applied at step k
  int colT[N];      // column transposition applied at step k
  int rank = N;

  void compute(const double (&A)[N][N]) {
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < N; ++c) lu[r][c] = A[r][c];
    double maxPivot = 0;
    int nonzeroPivots = N;
    for (int k = 0; k < N; ++k) {
      int br = k, bc = k;
      double big = -1;
      for (int c = k; c < N; ++c)
        for (int r = k; r < N; ++r) {
          double a = std::fabs(lu[r][c]);
          if (a > big) {
            big = a;
            br = r;
            bc = c;
          }
        }
      if (big == 0) {
        nonzeroPivots = k;
        for (int q = k; q < N; ++q) rowT[q] = colT[q] = q;
        break;
      }
      if (big > maxPivot) maxPivot = big;
      rowT[k] = br;
      colT[k] = bc;
      if (br != k)
        for (int c = 0; c < N; ++c) {
          double t = lu[k][c];
          lu[k][c] = lu[br][c];
          lu[br][c] = t;
        }
      if (bc != k)
        for (int r = 0; r < N; ++r) {
          double t = lu[r][k];
          lu[r][k] = lu[r][bc];
          lu[r][bc] = t;
        }
      for (int r = k + 1; r < N; ++r) lu[r][k] /= lu[k][k];
      for (int c = k + 1; c < N; ++c)
        for (int r = k + 1; r < N; ++r) lu[r][c] -= lu[r][k] * lu[k][c];
    }
    const double thr = std::numeric_limits<double>::epsilon() * N;
    rank = 0;
    for (int i = 0; i < nonzeroPivots; ++i)
      if (std::fabs(lu[i][i]) > thr * maxPivot) ++rank;
  }

  // x = A^{-1} b. T may be double or a dual-number type supporting +,-,*,/ with double.
  template <class T>
  void solve(const T (&b)[N], T (&x)[N]) const {
    T c[N];
    for (int i = 0; i < N; ++i) c[i] = b[i];
    for (int k = 0; k < N; ++k)
      if (rowT[k] != k) {
        T t = c[k];
        c[k] = c[rowT[k]];
        c[rowT[k]] = t;
      }
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < i; ++j) c[i] = c[i] - lu[i][j] * c[j];
    for (int i = rank - 1; i >= 0; --i) {
      for (int j = i + 1; j < rank; ++j) c[i] = c[i] - lu[i][j] * c[j];
      c[i] = c[i] / lu[i][i];
    }
    for (int i = rank; i < N; ++i) c[i] = T(0.0);
    for (int k = N - 1; k >= 0; --k)
      if (colT[k] != k) {
        T t = c[k];
        c[k] = c[colT[k]];
        c[colT[k]] = t;
      }
    for (int i = 0; i < N; ++i) x[i] = c[i];
  }
};

}  // namespace oracle_lu
#endif
