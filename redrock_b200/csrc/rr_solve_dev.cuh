// Normal-equation solve and chi2 shared by the scan kernels (rr_scan.cu,
// rr_pairs.cu).
//
// Reference: solve_matrices (PCA) zscan.py:1131-1152 -- LAPACK gesv, an
// exactly singular system raises LinAlgError and the redshift gets
// HUGE_CHI2 (zscan.py:769-771); chi2 = sum w (f - Tb c)^2 (zscan.py:777-780).
#pragma once

#include <cmath>

#include "rr_common.cuh"

namespace rr {

// LDL^T of the packed lower triangle of a symmetric matrix (row-major,
// a[i(i+1)/2 + j], j <= i), then the solve for c.  Works on its own copy
// so the caller's accumulator stays in registers.  Returns false on an
// exactly zero pivot (redrock's singular case), leaving c unspecified.
template <int NB>
__device__ __forceinline__ bool ldlt_solve(const double (&m)[NB * (NB + 1) / 2],
                                           const double (&y)[NB], double (&c)[NB]) {
  constexpr int kTri = NB * (NB + 1) / 2;
  double a[kTri];
#pragma unroll
  for (int i = 0; i < kTri; ++i) a[i] = m[i];
#define A(i, j) a[(i) * ((i) + 1) / 2 + (j)]
  double d[NB];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    double v[NB];
    double dj = A(j, j);
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      if (k < j) {
        v[k] = A(j, k) * d[k];
        dj -= A(j, k) * v[k];
      }
    }
    ok = ok && (dj != 0.0);
    d[j] = dj;
    const double inv = 1.0 / dj;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      if (i > j) {
        double s = A(i, j);
#pragma unroll
        for (int k = 0; k < NB; ++k)
          if (k < j) s -= A(i, k) * v[k];
        A(i, j) = s * inv;
      }
    }
  }
  // L z = y
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    double s = y[i];
#pragma unroll
    for (int k = 0; k < NB; ++k)
      if (k < i) s -= A(i, k) * c[k];
    c[i] = s;
  }
#pragma unroll
  for (int i = 0; i < NB; ++i) c[i] /= d[i];
  // L^T c = z
#pragma unroll
  for (int ii = 0; ii < NB; ++ii) {
    const int i = NB - 1 - ii;
    double s = c[i];
#pragma unroll
    for (int k = 0; k < NB; ++k)
      if (k > i) s -= A(k, i) * c[k];
    c[i] = s;
  }
#undef A
  return ok;
}

// Relative accuracy assumed for the FP64 sums M, y and f^T W f (about 90
// ulp; calibrated against redrock's direct residual, whose measured error
// stays below a tenth of this bound), and the bound on the chi2 error above
// which a (target, z) is re-evaluated by the direct residual: 1e-4, a tenth
// of the |dchi2| <= 1e-3 acceptance bar.
constexpr double kSumEps = 1e-14;
#ifndef RR_CHI2_FIX_TOL
#define RR_CHI2_FIX_TOL 1e-4
#endif
constexpr double kChi2FixTol = RR_CHI2_FIX_TOL;

// Solve and chi2 for one (target, z) from its normal equations.
// chi2 = f^T W f - c^T y - c^T P c.  Also returns an upper estimate of that
// value's rounding error, kSumEps (sum_i |c_i| sqrt(M_ii) + sqrt(f^T W f))^2,
// which bounds |c^T dM c| + 2|c^T dy| + |d(f^T W f)| for relative errors
// kSumEps in the sums.  Returns false when the system is singular (or the
// target has no weight, or the method is unsupported).
template <int NB>
__device__ __forceinline__ bool solve_eval(int method, const double* __restrict__ prior,
                                           const double (&m)[NB * (NB + 1) / 2],
                                           const double (&y)[NB], double fwf, double wsum,
                                           double (&c)[NB], double& chi2, double& err) {
  constexpr int kTri = NB * (NB + 1) / 2;
  bool ok = (wsum != 0.0) && (method == RR_SOLVE_PCA);
  double s = 0.0;
  if (ok) {
    double mp[kTri];
#pragma unroll
    for (int i = 0; i < kTri; ++i) mp[i] = m[i];
    if (prior) {
#pragma unroll
      for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) mp[i * (i + 1) / 2 + j] += prior[i * NB + j];
    }
    ok = ldlt_solve<NB>(mp, y, c);
#pragma unroll
    for (int i = 0; i < NB; ++i) s = fma(fabs(c[i]), sqrt(fmax(m[i * (i + 1) / 2 + i], 0.0)), s);
  }
  if (!ok) {
#pragma unroll
    for (int i = 0; i < NB; ++i) c[i] = 0.0;
    chi2 = kHugeChi2;
    err = 0.0;
    return false;
  }
  double cy = 0.0;
#pragma unroll
  for (int i = 0; i < NB; ++i) cy = fma(c[i], y[i], cy);
  double cpc = 0.0;
  if (prior) {
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < NB; ++j) t = fma(prior[i * NB + j], c[j], t);
      cpc = fma(c[i], t, cpc);
    }
  }
  chi2 = fwf - cy - cpc;
  const double a = s + sqrt(fwf);
  err = kSumEps * a * a;
  return true;
}

}  // namespace rr
