/* Dense 3x3 solve used by the checkers' boundary-condition extrapolation
 * (test infrastructure only): A x = b, A row-major, Gaussian elimination with
 * partial pivoting (rows swap on a strictly larger |pivot|), back substitution.
 * The device kernel (mac_b200/csrc/mac_extrap_bc.cu) performs the same
 * operations in the same order. */
#ifndef MAC_ORACLE_SOLVE3_H
#define MAC_ORACLE_SOLVE3_H
#include <math.h>

static inline void mac_solve3(const double* A, const double* b, double* x) {
  double m[3][4];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) m[r][c] = A[3 * r + c];
    m[r][3] = b[r];
  }
  for (int c = 0; c < 3; ++c) {
    int p = c;
    for (int r = c + 1; r < 3; ++r)
      if (fabs(m[r][c]) > fabs(m[p][c])) p = r;
    if (p != c)
      for (int j = 0; j < 4; ++j) {
        const double t = m[c][j];
        m[c][j] = m[p][j];
        m[p][j] = t;
      }
    for (int r = c + 1; r < 3; ++r) {
      const double f = m[r][c] / m[c][c];
      for (int j = c; j < 4; ++j) m[r][j] = m[r][j] - f * m[c][j];
    }
  }
  for (int r = 2; r >= 0; --r) {
    double v = m[r][3];
    for (int j = r + 1; j < 3; ++j) v = v - m[r][j] * x[j];
    x[r] = v / m[r][r];
  }
}
#endif
