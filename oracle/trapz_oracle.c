/*
 * Oracle (test infrastructure only): CPU restatement of redrock's
 * trapezoidal rebinning, used to check the CUDA kernels.  Not part of the
 * product; nothing in redrock_b200/ links or calls it.
 *
 * Follows redrock 0.22 py/redrock/rebin.py:
 *   _trapz_rebin_1d    rebin.py:126-176  (walk of input samples per bin)
 *   _trapz_rebin_batch rebin.py:178-209  (x * (1 + z) for each redshift,
 *                                         output [nz][nbin][nbasis])
 * Compiled without floating-point contraction (-ffp-contract=off) so the
 * operation order, and therefore every rounding, is redrock's.
 */
#include <stdint.h>

static void rebin_1d(const double* x, const double* y, const double* edges, int64_t nbin,
                     double* res, int64_t res_stride) {
  int64_t i = 0, j = 0;
  double yedge, area;
  for (i = 0; i < nbin; ++i) res[i * res_stride] = 0.0;
  for (i = 0; i < nbin; ++i) {
    while (x[j] <= edges[i]) j++;
    yedge = y[j - 1] + (edges[i] - x[j - 1]) * (y[j] - y[j - 1]) / (x[j] - x[j - 1]);
    if (x[j] < edges[i + 1]) {
      area = 0.5 * (y[j] + yedge) * (x[j] - edges[i]);
      res[i * res_stride] += area;
      while (x[j + 1] < edges[i + 1]) {
        j++;
        area = 0.5 * (y[j] + y[j - 1]) * (x[j] - x[j - 1]);
        res[i * res_stride] += area;
      }
      yedge = y[j] + (edges[i + 1] - x[j]) * (y[j + 1] - y[j]) / (x[j + 1] - x[j]);
      area = 0.5 * (yedge + y[j]) * (edges[i + 1] - x[j]);
      res[i * res_stride] += area;
    } else {
      double ylo = y[j] + (edges[i] - x[j]) * (y[j] - y[j - 1]) / (x[j] - x[j - 1]);
      double yhi = y[j] + (edges[i + 1] - x[j]) * (y[j] - y[j - 1]) / (x[j] - x[j - 1]);
      area = 0.5 * (ylo + yhi) * (edges[i + 1] - edges[i]);
      res[i * res_stride] += area;
    }
  }
  for (i = 0; i < nbin; ++i) res[i * res_stride] /= edges[i + 1] - edges[i];
}

/* out[nz][nbin][nbasis]; xs is caller scratch of nx doubles */
void oracle_trapz_rebin(const double* x, int64_t nx, const double* y, int64_t nbasis,
                        const double* edges, int64_t nbin, const double* z, int64_t nz,
                        double* out, double* xs) {
  for (int64_t iz = 0; iz < nz; ++iz) {
    for (int64_t k = 0; k < nx; ++k) xs[k] = x[k] * (1. + z[iz]);
    for (int64_t b = 0; b < nbasis; ++b)
      rebin_1d(xs, y + b * nx, edges, nbin, out + iz * nbin * nbasis + b, nbasis);
  }
}
