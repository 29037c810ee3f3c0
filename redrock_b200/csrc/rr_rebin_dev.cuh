// Device code shared by the basis builder (rr_basis.cu) and the pair scan
// (rr_pairs.cu): the trapezoid rebin of one output bin and the IGM
// transmission at one (z, wavelength).  Each translation unit that includes
// this header gets its own copy of the constant-memory tables and uploads
// them (once per device) before its first launch.
//
// Reference behaviour followed (redrock 0.22):
//   _trapz_rebin_1d  rebin.py:126-176   _trapz_rebin_batch rebin.py:178-209
//   Inoue14          igm.py:105-267     CaluraKamble       igm.py:321-364
#pragma once

#include <cmath>

#include "rr_common.cuh"
#include "rr_igm_table.h"

namespace rr {

static __constant__ double c_inoue_lam[RR_INOUE14_NLINES];
static __constant__ double c_inoue_laf[RR_INOUE14_NLINES][3];
static __constant__ double c_inoue_dla[RR_INOUE14_NLINES][2];

static int upload_igm_tables(cudaStream_t stream) {
  // constant-memory upload once per device
  static bool done[64] = {false};
  int dev = 0;
  RR_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 64 && done[dev]) return RR_OK;
  RR_CUDA_TRY(cudaMemcpyToSymbolAsync(c_inoue_lam, rr_inoue14_lam_h, sizeof(rr_inoue14_lam_h), 0,
                                      cudaMemcpyHostToDevice, stream));
  RR_CUDA_TRY(cudaMemcpyToSymbolAsync(c_inoue_laf, rr_inoue14_laf_h, sizeof(rr_inoue14_laf_h), 0,
                                      cudaMemcpyHostToDevice, stream));
  RR_CUDA_TRY(cudaMemcpyToSymbolAsync(c_inoue_dla, rr_inoue14_dla_h, sizeof(rr_inoue14_dla_h), 0,
                                      cudaMemcpyHostToDevice, stream));
  RR_CUDA_TRY(cudaStreamSynchronize(stream));
  if (dev < 64) done[dev] = true;
  return RR_OK;
}

// ---------------------------------------------------------------------------
// IGM transmission at one (z, observed wavelength)
// ---------------------------------------------------------------------------
constexpr double kLyA = 1215.67;   // constants.py:14
constexpr double kLamL = 911.8;    // Lyman limit used by Inoue14 (igm.py:172,202)

// Inoue et al. (2014) LAF + DLA, Lyman series and Lyman continuum.
// Expression order follows igm.py:105-267 term by term.
static __device__ double transmission_inoue14(double z, double lobs) {
  const double zp1 = dadd(1.0, z);
  const double lrest = ddiv(lobs, zp1);
  // --- Lyman series (sum over lines in table order) ---
  double t_laf = 0.0, t_dla = 0.0;
  if (lrest < c_inoue_lam[0]) {
    double p12 = -1.0, p37 = -1.0, p55 = -1.0, p3 = -1.0;
    const double l2sq = dmul(lobs, lobs);
    for (int j = 0; j < RR_INOUE14_NLINES; ++j) {
      const double l2 = c_inoue_lam[j];
      if (!(lrest < l2)) continue;  // masked terms add 0.0, which is exact
      double term;
      if (lobs < dmul(l2, dadd(1.0, 1.2))) {
        if (p12 < 0) p12 = pow(lobs, 1.2);
        term = dmul(c_inoue_laf[j][0], p12);
      } else if (lobs < dmul(l2, dadd(1.0, 4.7))) {
        if (p37 < 0) p37 = pow(lobs, 3.7);
        term = dmul(c_inoue_laf[j][1], p37);
      } else {
        if (p55 < 0) p55 = pow(lobs, 5.5);
        term = dmul(c_inoue_laf[j][2], p55);
      }
      t_laf = dadd(t_laf, term);
      if (lobs < dmul(l2, dadd(1.0, 2.0))) {
        term = dmul(c_inoue_dla[j][0], l2sq);
      } else {
        if (p3 < 0) p3 = pow(lobs, 3.0);
        term = dmul(c_inoue_dla[j][1], p3);
      }
      t_dla = dadd(t_dla, term);
    }
  }
  // --- Lyman continuum ---
  double t_lcdla = 0.0, t_lclaf = 0.0;
  if (lobs < dmul(kLamL, zp1)) {
    const double r = ddiv(lobs, kLamL);
    const double r_m03 = pow(r, -3e-1);
    // DLA (igm.py:167-192)
    if (z < 2.0) {
      const double a = dmul(zp1, zp1);
      const double b = pow(zp1, 2.3);
      t_lcdla = dsub(dsub(dmul(0.2113, a), dmul(dmul(0.07661, b), r_m03)), dmul(0.1347, dmul(r, r)));
    } else {
      const double e = pow(zp1, 3.0);
      const double f = pow(zp1, 3.3);
      if (lobs >= dmul(kLamL, dadd(1.0, 2.0))) {
        t_lcdla = dsub(dsub(dmul(0.04696, e), dmul(dmul(0.01779, f), r_m03)),
                       dmul(0.02916, pow(r, 3.0)));
      } else {
        t_lcdla = dsub(dsub(dsub(dadd(0.6340, dmul(0.04696, e)), dmul(dmul(0.01779, f), r_m03)),
                            dmul(0.1347, dmul(r, r))),
                       dmul(0.2905, r_m03));
      }
    }
    // LAF (igm.py:195-229).  In the reference the z < 1.2 assignment is
    // always overwritten by the z < 4.7 one (its mask contains it), so the
    // z < 4.7 formulas apply from z = 0 upwards.
    const double i21 = pow(r, 2.1);
    if (z < 4.7) {
      const double h = pow(zp1, 1.6);
      if (lobs >= dmul(kLamL, dadd(1.0, 1.2))) {
        t_lclaf = dmul(2.545e-2, dsub(dmul(h, i21), pow(r, 3.7)));
      } else {
        t_lclaf = dsub(dadd(dmul(dmul(2.545e-2, h), i21), dmul(0.3248, pow(r, 1.2))),
                       dmul(0.2496, i21));
      }
    } else {
      const double nn = pow(zp1, 3.4);
      if (lobs > dmul(kLamL, dadd(1.0, 4.7))) {
        t_lclaf = dmul(5.221e-4, dsub(dmul(nn, i21), pow(r, 5.5)));
      } else if (lobs >= dmul(kLamL, dadd(1.0, 1.2)) && lobs < dmul(kLamL, dadd(1.0, 4.7))) {
        t_lclaf = dsub(dadd(dmul(dmul(5.221e-4, nn), i21), dmul(0.2182, i21)),
                       dmul(2.545e-2, pow(r, 3.7)));
      } else if (lobs < dmul(kLamL, dadd(1.0, 1.2))) {
        t_lclaf = dsub(dadd(dmul(dmul(5.221e-4, nn), i21), dmul(0.3248, pow(r, 1.2))),
                       dmul(3.140e-2, i21));
      }
    }
  }
  const double tau_ls = dadd(t_laf, t_dla);
  const double tau_lc = dadd(t_lclaf, t_lcdla);
  const double tau = dadd(dadd(tau_lc, tau_ls), 0.0);
  return exp(dmul(-1.0, tau));
}

// Calura et al. (2012) / Kamble et al. (2020) effective optical depth of
// the Lyman series lines (constants.py:16-37, igm.py:321-364).
static __device__ double transmission_calura_kamble(int model, double z, double lobs) {
  const double lrest = dmul(ddiv(1.0, dadd(1.0, z)), lobs);
  double T = 1.0;
  if (model == RR_IGM_KAMBLE20) {
    const double line = kLyA;
    if (lrest < line) {
      const double zpix = dsub(ddiv(lobs, line), 1.0);
      const double tau = dmul(0.00554, pow(dadd(1.0, zpix), 3.182));
      T = dmul(T, exp(-tau));
    }
    return T;
  }
  const double lines[5] = {kLyA, 1025.72, 972.537, 949.7431, 937.8035};
  const double amp[5] = {0.0023, 0.0023 / 5.2615, 0.0023 / 14.356, 0.0023 / 29.85984,
                         0.0023 / 53.36202};
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    if (lrest < lines[l]) {
      const double zpix = dsub(ddiv(lobs, lines[l]), 1.0);
      const double tau = dmul(amp[l], pow(dadd(1.0, zpix), 3.64));
      T = dmul(T, exp(-tau));
    }
  }
  return T;
}

// d/dz of the Inoue14 Lyman-continuum optical depth at fixed observed
// wavelength (the smooth part of the z dependence; the Lyman-series terms
// depend on z only through their on/off masks).  Mirrors the branch
// structure of transmission_inoue14.
static __device__ double dtau_lc_dz_inoue14(double z, double lobs) {
  const double zp1 = dadd(1.0, z);
  if (!(lobs < dmul(kLamL, zp1))) return 0.0;
  const double r = ddiv(lobs, kLamL);
  const double r_m03 = pow(r, -3e-1);
  double d = 0.0;
  if (z < 2.0) {
    d += 2.0 * 0.2113 * zp1 - 0.07661 * 2.3 * pow(zp1, 1.3) * r_m03;
  } else {
    d += 3.0 * 0.04696 * zp1 * zp1 - 0.01779 * 3.3 * pow(zp1, 2.3) * r_m03;
  }
  const double i21 = pow(r, 2.1);
  if (z < 4.7) {
    d += 2.545e-2 * 1.6 * pow(zp1, 0.6) * i21;
  } else if (lobs > dmul(kLamL, dadd(1.0, 4.7)) || lobs < dmul(kLamL, dadd(1.0, 4.7))) {
    d += 5.221e-4 * 3.4 * pow(zp1, 2.4) * i21;
  }
  return d;
}

__device__ __forceinline__ double transmission(int model, double z, double lobs);

// Transmission and its smooth z derivative at one (z, wavelength).
// Calura12 / Kamble20 depend on z only through line masks: derivative 0.
__device__ __forceinline__ double transmission_dz(int model, double z, double lobs, double* dt) {
  const double t = transmission(model, z, lobs);
  *dt = (model == RR_IGM_INOUE14) ? -t * dtau_lc_dz_inoue14(z, lobs) : 0.0;
  return t;
}

__device__ __forceinline__ double transmission(int model, double z, double lobs) {
  if (model == RR_IGM_INOUE14) return transmission_inoue14(z, lobs);
  if (model == RR_IGM_CALURA12 || model == RR_IGM_KAMBLE20)
    return transmission_calura_kamble(model, z, lobs);
  return 1.0;
}


// ---------------------------------------------------------------------------
// trapezoid rebin of one output bin for all bases
// ---------------------------------------------------------------------------
constexpr int kMaxRebinBasis = 16;

// Returns false (and leaves res untouched) when the bin falls outside the
// redshifted input range; callers then report an error.
// y[b * ystride + j] holds basis b at sample j.
//
// With DZ, dres[b] also receives dT/dz of the rebinned value.  Writing the
// bin average as T = ((1+z)/w) * integral of the rest-frame interpolant over
// [e_lo/(1+z), e_hi/(1+z)] gives
//   dT/dz = (T - (e_hi y(e_hi) - e_lo y(e_lo)) / w) / (1+z),
// where y(e) is the redshifted interpolant at the bin edges -- the edge
// values the trapezoid sum already forms.  (T itself is unchanged, bit for
// bit, by the extra output.)
// First j in [0, nx) with x[j] (1+z) > e (nx if none), x increasing.  A
// guess from the mean sample spacing and a short walk find it with two or
// three dependent loads on the (usually uniform) template grids; a binary
// search over what is left covers uneven grids.  Every comparison is the
// exactly rounded x[j] (1+z) <= e, so the result is the binary search's.
__device__ __forceinline__ int64_t first_above(const double* __restrict__ x, int64_t nx,
                                               double zp1, double e) {
  int64_t lo = 0, hi = nx;  // the answer lies in [lo, hi]
  const double x0 = x[0];
  const double t = (e / zp1 - x0) / (x[nx - 1] - x0) * (double)(nx - 1);
  if (t > 0.0 && t < (double)(nx - 1)) {
    const int64_t g = (int64_t)t;
    if (dmul(x[g], zp1) <= e) {
      lo = g + 1;
      for (int k = 0; k < 8 && lo < hi; ++k) {
        if (dmul(x[lo], zp1) <= e) {
          ++lo;
        } else {
          hi = lo;
        }
      }
    } else {
      hi = g;
      for (int k = 0; k < 8 && lo < hi; ++k) {
        if (dmul(x[hi - 1], zp1) > e) {
          --hi;
        } else {
          lo = hi;
        }
      }
    }
  }
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (dmul(x[mid], zp1) <= e) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <bool DZ = false>
__device__ __forceinline__ bool rebin_bin_strided(const double* __restrict__ x, int64_t nx,
                                                  const double* __restrict__ y, int64_t ystride,
                                                  int nb, double zp1, double e_lo, double e_hi,
                                                  double* res, double* dres = nullptr) {
  double ylo_e[DZ ? kMaxRebinBasis : 1], yhi_e[DZ ? kMaxRebinBasis : 1];
  // first j with x[j] (1+z) > e_lo
  int64_t j = first_above(x, nx, zp1, e_lo);
  if (j < 1 || j >= nx) return false;
  double xj = dmul(x[j], zp1);
  const double xjm1 = dmul(x[j - 1], zp1);
  for (int b = 0; b < nb; ++b) res[b] = 0.0;
  if (xj < e_hi) {
    // lower edge to the first sample inside the bin
    for (int b = 0; b < nb; ++b) {
      const double* yb = y + (int64_t)b * ystride;
      const double yedge = dadd(yb[j - 1], ddiv(dmul(dsub(e_lo, xjm1), dsub(yb[j], yb[j - 1])),
                                                 dsub(xj, xjm1)));
      if (DZ) ylo_e[b] = yedge;
      res[b] = dadd(res[b], dmul(dmul(0.5, dadd(yb[j], yedge)), dsub(xj, e_lo)));
    }
    // interior samples
    while (true) {
      if (j + 1 >= nx) return false;
      const double xn = dmul(x[j + 1], zp1);
      if (!(xn < e_hi)) break;
      ++j;
      const double xprev = xj;
      xj = xn;
      for (int b = 0; b < nb; ++b) {
        const double* yb = y + (int64_t)b * ystride;
        res[b] = dadd(res[b], dmul(dmul(0.5, dadd(yb[j], yb[j - 1])), dsub(xj, xprev)));
      }
    }
    // upper edge
    const double xn = dmul(x[j + 1], zp1);
    for (int b = 0; b < nb; ++b) {
      const double* yb = y + (int64_t)b * ystride;
      const double yedge = dadd(yb[j], ddiv(dmul(dsub(e_hi, xj), dsub(yb[j + 1], yb[j])),
                                            dsub(xn, xj)));
      if (DZ) yhi_e[b] = yedge;
      res[b] = dadd(res[b], dmul(dmul(0.5, dadd(yedge, yb[j])), dsub(e_hi, xj)));
    }
  } else {
    // the samples span the whole bin
    for (int b = 0; b < nb; ++b) {
      const double* yb = y + (int64_t)b * ystride;
      const double slope_num = dsub(yb[j], yb[j - 1]);
      const double dx = dsub(xj, xjm1);
      const double ylo = dadd(yb[j], ddiv(dmul(dsub(e_lo, xj), slope_num), dx));
      const double yhi = dadd(yb[j], ddiv(dmul(dsub(e_hi, xj), slope_num), dx));
      if (DZ) {
        ylo_e[b] = ylo;
        yhi_e[b] = yhi;
      }
      res[b] = dadd(res[b], dmul(dmul(0.5, dadd(ylo, yhi)), dsub(e_hi, e_lo)));
    }
  }
  const double width = dsub(e_hi, e_lo);
  for (int b = 0; b < nb; ++b) res[b] = ddiv(res[b], width);
  if (DZ)
    for (int b = 0; b < nb; ++b)
      dres[b] = (res[b] - (e_hi * yhi_e[b] - e_lo * ylo_e[b]) / width) / zp1;
  return true;
}

__device__ __forceinline__ bool rebin_bin(const double* __restrict__ x, int64_t nx,
                                          const double* __restrict__ y, int nb, double zp1,
                                          double e_lo, double e_hi, double* res) {
  return rebin_bin_strided(x, nx, y, nx, nb, zp1, e_lo, e_hi, res);
}

}  // namespace rr
