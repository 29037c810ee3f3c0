// Bounded least squares for the non-PCA branches of redrock's
// solve_matrices (zscan.py:1153-1201): redrock hands the normal-equation
// pair (M, y) to scipy as a design matrix and right-hand side, so both
// solvers here minimise ||M x - y||_2 for the small square M (n <= 10):
//
//   nnls_solve  x >= 0: the active-set algorithm of Lawson & Hanson
//               ("Solving Least Squares Problems", 1974/1995, ch. 23), at
//               most 3 n subproblem solves (scipy.optimize.nnls's default
//               iteration limit; beyond it redrock sees an exception and
//               sets HUGE_CHI2).
//   bvls_solve  lo <= x <= hi: Stark & Parker's bounded-variable least
//               squares with the control flow of scipy's lsq_linear(...,
//               method='bvls'): start from the unconstrained solution
//               (returned as is when inside the bounds), clamp, free the
//               variables that the unconstrained subproblem keeps inside,
//               then at most n KKT steps (tolerance 1e-10 on the KKT
//               violation, or a relative cost decrease below 1e-10).
//
// Every subproblem is least squares on the free columns, solved by
// Householder QR (no normal equations: M is itself a Gram matrix).  A free
// set whose columns are exactly dependent makes the solve fail (redrock
// would return scipy's minimum-norm answer there; it does not arise for
// full-rank templates).
#pragma once
#include <cmath>

namespace rr {

// z[0..k) = argmin ||A[:, cols] z - r||, A row-major NB x NB.
template <int NB>
__device__ __forceinline__ bool lsq_cols(const double (&A)[NB][NB], const double (&r)[NB],
                                         const int (&cols)[NB], int k, double (&z)[NB]) {
  double W[NB][NB];
  double v[NB], diag[NB];
  for (int i = 0; i < NB; ++i) {
    v[i] = r[i];
    for (int j = 0; j < k; ++j) W[i][j] = A[i][cols[j]];
  }
  for (int j = 0; j < k; ++j) {
    double nrm2 = 0.0;
    for (int i = j; i < NB; ++i) nrm2 = fma(W[i][j], W[i][j], nrm2);
    const double nrm = sqrt(nrm2);
    if (!(nrm > 0.0)) return false;
    const double alpha = W[j][j] > 0.0 ? -nrm : nrm;
    W[j][j] -= alpha;  // Householder vector u = column - alpha e_j, rows j..
    double u2 = 0.0;
    for (int i = j; i < NB; ++i) u2 = fma(W[i][j], W[i][j], u2);
    diag[j] = alpha;
    if (u2 > 0.0) {
      for (int c = j + 1; c < k; ++c) {
        double s = 0.0;
        for (int i = j; i < NB; ++i) s = fma(W[i][j], W[i][c], s);
        const double f = 2.0 * s / u2;
        for (int i = j; i < NB; ++i) W[i][c] = fma(-f, W[i][j], W[i][c]);
      }
      double s = 0.0;
      for (int i = j; i < NB; ++i) s = fma(W[i][j], v[i], s);
      const double f = 2.0 * s / u2;
      for (int i = j; i < NB; ++i) v[i] = fma(-f, W[i][j], v[i]);
    }
  }
  for (int j = k - 1; j >= 0; --j) {
    double s = v[j];
    for (int c = j + 1; c < k; ++c) s = fma(-W[j][c], z[c], s);
    z[j] = s / diag[j];
  }
  return true;
}

// g = A^T (A x - b)
template <int NB>
__device__ __forceinline__ void lsq_grad(const double (&A)[NB][NB], const double (&b)[NB],
                                         const double (&x)[NB], double (&r)[NB],
                                         double (&g)[NB]) {
  for (int i = 0; i < NB; ++i) {
    double s = -b[i];
    for (int j = 0; j < NB; ++j) s = fma(A[i][j], x[j], s);
    r[i] = s;
  }
  for (int j = 0; j < NB; ++j) {
    double s = 0.0;
    for (int i = 0; i < NB; ++i) s = fma(A[i][j], r[i], s);
    g[j] = s;
  }
}

template <int NB>
__device__ bool nnls_solve(const double (&A)[NB][NB], const double (&b)[NB], double (&x)[NB]) {
  bool pset[NB];
  bool skip[NB];
  double r[NB], g[NB], z[NB];
  int cols[NB];
  double amax = 0.0, bmax = 0.0;
  for (int i = 0; i < NB; ++i) {
    x[i] = 0.0;
    pset[i] = false;
    skip[i] = false;
    bmax = fmax(bmax, fabs(b[i]));
    for (int j = 0; j < NB; ++j) amax = fmax(amax, fabs(A[i][j]));
  }
  // w_j below this is rounding noise of A^T (b - A x)
  const double tol = 100.0 * NB * 2.220446049250313e-16 * amax * bmax;
  int solves = 0;
  while (true) {
    // w = A^T (b - A x) = -g; the most positive w among bound variables
    lsq_grad<NB>(A, b, x, r, g);
    int t = -1;
    double best = tol;
    for (int j = 0; j < NB; ++j)
      if (!pset[j] && !skip[j] && -g[j] > best) {
        best = -g[j];
        t = j;
      }
    if (t < 0) return true;
    pset[t] = true;
    bool first = true;
    while (true) {
      if (++solves > 3 * NB) return false;
      int k = 0;
      for (int j = 0; j < NB; ++j)
        if (pset[j]) cols[k++] = j;
      double zc[NB];
      if (!lsq_cols<NB>(A, b, cols, k, zc)) return false;
      for (int j = 0; j < NB; ++j) z[j] = 0.0;
      for (int q = 0; q < k; ++q) z[cols[q]] = zc[q];
      if (first && z[t] <= 0.0) {
        // rounding made the new variable's solution non-positive: take it
        // back and try the next one (Lawson & Hanson's step)
        pset[t] = false;
        skip[t] = true;
        break;
      }
      first = false;
      bool feasible = true;
      double alpha = 2.0;
      int lim = -1;
      for (int j = 0; j < NB; ++j)
        if (pset[j] && z[j] <= 0.0) {
          feasible = false;
          const double den = x[j] - z[j];
          const double a = den > 0.0 ? x[j] / den : 0.0;
          if (a < alpha) {
            alpha = a;
            lim = j;
          }
        }
      if (feasible) {
        for (int j = 0; j < NB; ++j) x[j] = z[j];
        for (int j = 0; j < NB; ++j) skip[j] = false;
        break;
      }
      for (int j = 0; j < NB; ++j)
        if (pset[j]) x[j] = fma(alpha, z[j] - x[j], x[j]);
      for (int j = 0; j < NB; ++j)
        if (pset[j] && (j == lim || x[j] <= 0.0)) {
          x[j] = 0.0;
          pset[j] = false;
        }
    }
  }
}

// lo / hi point at the caller's bounds (read-only; in the plain chain the
// kernel's __grid_constant__ parameter, so no local copies are made).
template <int NB>
__device__ bool bvls_solve(const double (&A)[NB][NB], const double (&b)[NB],
                           const double* __restrict__ lo, const double* __restrict__ hi,
                           double (&x)[NB]) {
  constexpr double kTol = 1e-10;
  int onb[NB];  // -1 at lower bound, +1 at upper bound, 0 free
  int cols[NB];
  double r[NB], g[NB], zc[NB], rhs[NB];
  int all[NB];
  for (int j = 0; j < NB; ++j) all[j] = j;
  if (!lsq_cols<NB>(A, b, all, NB, x)) return false;
  bool inside = true;
  for (int j = 0; j < NB; ++j) inside = inside && x[j] >= lo[j] && x[j] <= hi[j];
  if (inside) return true;
  for (int j = 0; j < NB; ++j) {
    onb[j] = 0;
    if (x[j] <= lo[j]) {
      x[j] = lo[j];
      onb[j] = -1;
    } else if (x[j] >= hi[j]) {
      x[j] = hi[j];
      onb[j] = 1;
    }
  }
  // free-set rhs: b - A x over the variables at a bound
  auto free_rhs = [&](const int (&ob)[NB]) {
    for (int i = 0; i < NB; ++i) {
      double s = b[i];
      for (int j = 0; j < NB; ++j)
        if (ob[j] != 0) s = fma(-A[i][j], x[j], s);
      rhs[i] = s;
    }
  };
  // initialisation: free variables that stay inside, the rest to bounds
  bool fr[NB];
  for (int j = 0; j < NB; ++j) fr[j] = onb[j] == 0;
  int iteration = 0;
  while (true) {
    int k = 0;
    for (int j = 0; j < NB; ++j)
      if (fr[j]) cols[k++] = j;
    if (k == 0) break;
    ++iteration;
    int act[NB];
    for (int j = 0; j < NB; ++j) act[j] = fr[j] ? 0 : 1;
    free_rhs(act);
    if (!lsq_cols<NB>(A, rhs, cols, k, zc)) return false;
    bool any = false;
    for (int q = 0; q < k; ++q) {
      const int j = cols[q];
      if (zc[q] < lo[j]) {
        x[j] = lo[j];
        onb[j] = -1;
        fr[j] = false;
        any = true;
      } else if (zc[q] > hi[j]) {
        x[j] = hi[j];
        onb[j] = 1;
        fr[j] = false;
        any = true;
      } else {
        x[j] = zc[q];
      }
    }
    if (!any) break;
  }
  const int max_iter = NB + iteration;
  lsq_grad<NB>(A, b, x, r, g);
  double cost = 0.0;
  for (int i = 0; i < NB; ++i) cost = fma(r[i], r[i], cost);
  cost *= 0.5;
  bool done = false;
  for (int it = iteration; it < max_iter && !done; ++it) {
    double opt = 0.0;
    for (int j = 0; j < NB; ++j) opt = fmax(opt, onb[j] ? g[j] * onb[j] : fabs(g[j]));
    if (opt < kTol) break;
    int m = 0;
    double best = g[0] * onb[0];
    for (int j = 1; j < NB; ++j)
      if (g[j] * onb[j] > best) {
        best = g[j] * onb[j];
        m = j;
      }
    onb[m] = 0;
    for (int guard = 0;; ++guard) {
      if (guard > NB) return false;
      int k = 0;
      for (int j = 0; j < NB; ++j)
        if (onb[j] == 0) cols[k++] = j;
      free_rhs(onb);
      if (!lsq_cols<NB>(A, rhs, cols, k, zc)) return false;
      double alpha = 0.0;
      int lim = -1, side = 0;
      for (int q = 0; q < k; ++q) {
        const int j = cols[q];
        double a = 0.0;
        int sd = 0;
        if (zc[q] < lo[j]) {
          a = (lo[j] - x[j]) / (zc[q] - x[j]);
          sd = -1;
        } else if (zc[q] > hi[j]) {
          a = (hi[j] - x[j]) / (zc[q] - x[j]);
          sd = 1;
        }
        if (sd != 0 && (lim < 0 || a < alpha)) {
          alpha = a;
          lim = j;
          side = sd;
        }
      }
      if (lim < 0) {
        for (int q = 0; q < k; ++q) x[cols[q]] = zc[q];
        break;
      }
      for (int q = 0; q < k; ++q) {
        const int j = cols[q];
        x[j] = fma(alpha, zc[q], x[j] * (1.0 - alpha));
      }
      onb[lim] = side;
    }
    lsq_grad<NB>(A, b, x, r, g);
    double cnew = 0.0;
    for (int i = 0; i < NB; ++i) cnew = fma(r[i], r[i], cnew);
    cnew *= 0.5;
    if (cost - cnew < kTol * cost) done = true;
    cost = cnew;
  }
  return true;
}

}  // namespace rr
