// The 4x4 inverse of the Khachiyan ellipsoid iteration, shared by the host (sd_synth.cc) and the
// device (sd_refpoint.cu) so that both compute the ligand reference point with the same operations.
//
// Inverse of a 4x4 matrix (column-major, a[c*4 + r]) in the operation order of the reference's
// MatrixXd::inverse() (its vendored Eigen 3.4: PartialPivLU, then solve against the identity):
//  * LU with partial pivoting, column by column: pivot = first row of largest |a(r,k)|, rows
//    swapped, the column below divided by the pivot, then a(r,c) -= a(r,k) * a(k,c);
//  * X = P I (the same row swaps applied to the identity);
//  * unit-lower solve, top to bottom: X(r,j) -= X(k,j) * L(r,k) for r > k;
//  * upper solve, bottom to top: X(i,j) *= 1 / U(i,i), then X(r,j) -= X(i,j) * U(r,i) for r < i.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define SD_MVEE_HD __host__ __device__ __forceinline__
#else
#define SD_MVEE_HD static inline
#endif

SD_MVEE_HD void sd_inverse4_lu(const double* a, double* x) {
  double lu[16];
  for (int k = 0; k < 16; ++k) lu[k] = a[k];
  int piv[4];
  for (int k = 0; k < 4; ++k) {
    int p = k;
    double best = fabs(lu[k * 4 + k]);
    for (int r = k + 1; r < 4; ++r)
      if (fabs(lu[k * 4 + r]) > best) {
        best = fabs(lu[k * 4 + r]);
        p = r;
      }
    piv[k] = p;
    if (best != 0.0) {
      if (p != k)
        for (int c = 0; c < 4; ++c) {
          const double v = lu[c * 4 + k];
          lu[c * 4 + k] = lu[c * 4 + p];
          lu[c * 4 + p] = v;
        }
      for (int r = k + 1; r < 4; ++r) lu[k * 4 + r] /= lu[k * 4 + k];
    }
    for (int c = k + 1; c < 4; ++c)
      for (int r = k + 1; r < 4; ++r) lu[c * 4 + r] -= lu[c * 4 + k] * lu[k * 4 + r];
  }
  for (int k = 0; k < 16; ++k) x[k] = (k % 5 == 0) ? 1.0 : 0.0;
  for (int k = 0; k < 4; ++k)
    if (piv[k] != k)
      for (int c = 0; c < 4; ++c) {
        const double v = x[c * 4 + k];
        x[c * 4 + k] = x[c * 4 + piv[k]];
        x[c * 4 + piv[k]] = v;
      }
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 4; ++j) {
      const double b = x[j * 4 + k];
      for (int r = k + 1; r < 4; ++r) x[j * 4 + r] -= b * lu[k * 4 + r];
    }
  for (int i = 3; i >= 0; --i) {
    const double inv = 1.0 / lu[i * 4 + i];
    for (int j = 0; j < 4; ++j) {
      x[j * 4 + i] *= inv;
      const double b = x[j * 4 + i];
      for (int r = 0; r < i; ++r) x[j * 4 + r] -= b * lu[i * 4 + r];
    }
  }
}
