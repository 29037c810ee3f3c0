// Coadd of a target's exposures per wavelength grid (redrock 0.22
// targets.py:267-373, Target.compute_coadd).
//
// For each (target, grid) group of nspec exposures with DIA resolution data
// data_s[d][j] (scipy convention: column j), ivar_s and flux_s:
//   weights[j]  = sum_s ivar_s[j]
//   flux[j]     = sum_s ivar_s[j] flux_s[j] / weights[j]
//                 (sum_s flux_s[j] / nspec where weights[j] == 0)
//   rdata[d][j] = sum_s data_s[d][j] ivar_s[j] / weights[j]   (/ 1 where 0)
// The sums run over the exposures in their list order with every product
// and sum rounded separately (no FMA contraction), which is numpy's order
// for these axis-0 reductions, so the results are bit-identical to
// redrock's.  One thread per (group, pixel).  With cosmic-ray rejection the
// resolution data keep the exposures' own ivar as weights (redrock sums
// them before rejecting), while ivar / flux use the masked ivar.
//
// Cosmic-ray rejection (cosmics_kernel, targets.py:310-354), one block per
// group of exposures on a common wavelength grid:
//   1. per exposure, the flux and ivar of pixels with ivar == 0 are linearly
//      interpolated in wavelength from the pixels with ivar > 0 (numpy's
//      interp: the end values beyond the first / last good pixel, else
//      slope * (x - x_j) + f_j with slope = (f_{j+1} - f_j) / (x_{j+1} -
//      x_j)); remaining ivar <= 0 take the smallest positive ivar;
//   2. grad_j = f_j - f_{j-1} (0 at j = 0), var_j = 1/ivar_j + 1/ivar_{j-1}
//      (1/ivar_0 at j = 0), gradivar = 1 / var;
//   3. for groups of >= 2 exposures: meangrad_j = sum_s gradivar grad / S
//      with S the sum of gradivar over ALL exposures and pixels (numpy's
//      pairwise sum order, as redrock writes it), chi2_j = sum_s gradivar
//      (grad - meangrad)^2 / (nspec - 1);
//   4. where chi2_j > nsig^2 the exposure with the largest
//      gradivar (grad - meangrad)^2 (first on ties) gets ivar 0 at j.
// All arithmetic is IEEE-rounded in numpy's order, so the mask and the
// coadd are bit-identical to redrock's.
#include "rr_common.cuh"

namespace rr {

__global__ void __launch_bounds__(256) coadd_kernel(const rr_coadd_group* __restrict__ groups,
                                                    const int64_t* __restrict__ exp_data,
                                                    const int64_t* __restrict__ exp_pix,
                                                    const double* __restrict__ rdata,
                                                    const double* __restrict__ ivar_r,
                                                    const double* __restrict__ ivar,
                                                    const double* __restrict__ flux,
                                                    double* __restrict__ rdata_out,
                                                    double* __restrict__ ivar_out,
                                                    double* __restrict__ flux_out) {
  const rr_coadd_group g = groups[blockIdx.y];
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.npix) return;
  double w = 0.0, uw = 0.0, wf = 0.0;
  for (int s = 0; s < g.nspec; ++s) {
    const int64_t e = g.first + s;
    const double iv = ivar[exp_pix[e] + j];
    const double fl = flux[exp_pix[e] + j];
    uw = s ? dadd(uw, fl) : fl;
    w = s ? dadd(w, iv) : iv;
    wf = s ? dadd(wf, dmul(iv, fl)) : dmul(iv, fl);
  }
  const bool bad = (w == 0.0);
  const double den = bad ? dadd(w, 1.0) : w;
  ivar_out[g.out_pix + j] = w;
  flux_out[g.out_pix + j] = bad ? ddiv(uw, (double)g.nspec) : ddiv(wf, den);
  for (int d = 0; d < g.ndiag; ++d) {
    double r = 0.0;
    for (int s = 0; s < g.nspec; ++s) {
      const int64_t e = g.first + s;
      const double v =
          dmul(rdata[exp_data[e] + (int64_t)d * g.npix + j], ivar_r[exp_pix[e] + j]);
      r = s ? dadd(r, v) : v;
    }
    rdata_out[g.out_data + (int64_t)d * g.npix + j] = ddiv(r, den);
  }
}


constexpr int kCosmicThreads = 256;

// numpy's pairwise summation of n doubles read through at(i): ranges of
// fewer than 8 summed in order from 0, ranges of up to 128 with 8
// interleaved partial sums combined ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7))
// plus the tail in order, larger ranges split at n/2 rounded down to a
// multiple of 8.  Iterative (explicit stack) so that one thread runs it.
template <class At>
__device__ double pairwise_sum(int64_t n, At at) {
  struct Frame {
    int64_t lo, n;
    double left;
    int stage;
  };
  Frame st[48];  // depth <= log2(n / 128) + 1
  int top = 0;
  st[0] = {0, n, 0.0, 0};
  double ret = 0.0;
  while (top >= 0) {
    Frame& f = st[top];
    if (f.n <= 128) {
      double res;
      if (f.n < 8) {
        res = 0.0;
        for (int64_t i = 0; i < f.n; ++i) res = dadd(res, at(f.lo + i));
      } else {
        double r[8];
        for (int k = 0; k < 8; ++k) r[k] = at(f.lo + k);
        int64_t i = 8;
        for (; i < f.n - (f.n % 8); i += 8)
          for (int k = 0; k < 8; ++k) r[k] = dadd(r[k], at(f.lo + i + k));
        res = dadd(dadd(dadd(r[0], r[1]), dadd(r[2], r[3])),
                   dadd(dadd(r[4], r[5]), dadd(r[6], r[7])));
        for (; i < f.n; ++i) res = dadd(res, at(f.lo + i));
      }
      ret = res;
      --top;
    } else if (f.stage == 0) {
      int64_t n2 = f.n / 2;
      n2 -= n2 % 8;
      f.stage = 1;
      st[top + 1] = {f.lo, n2, 0.0, 0};
      ++top;
    } else if (f.stage == 1) {
      f.left = ret;
      int64_t n2 = f.n / 2;
      n2 -= n2 % 8;
      f.stage = 2;
      st[top + 1] = {f.lo + n2, f.n - n2, 0.0, 0};
      ++top;
    } else {
      ret = dadd(f.left, ret);
      --top;
    }
  }
  return ret;
}

// Block-wide scans over per-thread chunk values: prev = the last index with
// ivar > 0 before the thread's chunk (-1 if none), next = the first one
// after it (none_hi if none); gfirst / glast of the whole row.
__device__ void chunk_neighbours(int64_t mylast, int64_t myfirst, int64_t none_hi,
                                 int64_t* sh_a, int64_t* sh_b, int64_t& prev, int64_t& next,
                                 int64_t& gfirst, int64_t& glast) {
  const int t = threadIdx.x;
  sh_a[t] = mylast;
  sh_b[t] = myfirst;
  __syncthreads();
  for (int off = 1; off < kCosmicThreads; off <<= 1) {
    const int64_t a = t >= off ? sh_a[t - off] : -1;
    const int64_t b = t + off < kCosmicThreads ? sh_b[t + off] : none_hi;
    __syncthreads();
    sh_a[t] = max(sh_a[t], a);
    sh_b[t] = min(sh_b[t], b);
    __syncthreads();
  }
  prev = t > 0 ? sh_a[t - 1] : -1;
  next = t + 1 < kCosmicThreads ? sh_b[t + 1] : none_hi;
  gfirst = sh_b[0];
  glast = sh_a[kCosmicThreads - 1];
  __syncthreads();
}

__global__ void __launch_bounds__(kCosmicThreads) cosmics_kernel(
    const rr_coadd_group* __restrict__ groups, const int64_t* __restrict__ exp_pix,
    const double* __restrict__ wave_all, const double* __restrict__ ivar,
    const double* __restrict__ flux, double thresh, double* __restrict__ ivar_out,
    double* __restrict__ work_f, double* __restrict__ work_v, int* status) {
  __shared__ int64_t sh_a[kCosmicThreads], sh_b[kCosmicThreads];
  __shared__ double sh_min[kCosmicThreads];
  __shared__ double sh_total;
  const rr_coadd_group g = groups[blockIdx.x];
  const int64_t N = g.npix;
  const int S = g.nspec;
  const int t = threadIdx.x;
  const double* wave = wave_all + g.out_pix;
  const int64_t C = (N + kCosmicThreads - 1) / kCosmicThreads;
  const int64_t lo = min(N, (int64_t)t * C), hi = min(N, lo + C);
  for (int s = 0; s < S; ++s) {
    const int64_t off = exp_pix[g.first + s];
    for (int64_t j = t; j < N; j += kCosmicThreads) ivar_out[off + j] = ivar[off + j];
    // 1. interpolation over ivar == 0 from the pixels with ivar > 0
    int64_t mylast = -1, myfirst = N;
    for (int64_t j = lo; j < hi; ++j)
      if (ivar[off + j] > 0.0) {
        if (myfirst == N) myfirst = j;
        mylast = j;
      }
    int64_t prev, next, gfirst, glast;
    chunk_neighbours(mylast, myfirst, N, sh_a, sh_b, prev, next, gfirst, glast);
    if (glast < 0) {  // the same for every thread: numpy has no sample points
      if (t == 0) set_status(status, RR_EINVAL);
      return;
    }
    double* tf = work_f + off;
    double* tv = work_v + off;
    // next good index of each ivar == 0 pixel, right to left (kept in tv)
    int64_t q = next;
    for (int64_t j = hi - 1; j >= lo; --j) {
      if (ivar[off + j] > 0.0) q = j;
      else tv[j] = (double)q;
    }
    int64_t p = prev;
    double mn = INFINITY;
    for (int64_t j = lo; j < hi; ++j) {
      const double iv = ivar[off + j];
      double f = flux[off + j], v = iv;
      if (iv > 0.0) {
        p = j;
      } else if (iv == 0.0) {
        const int64_t qq = (int64_t)tv[j];
        if (p < 0) {
          f = flux[off + gfirst];
          v = ivar[off + gfirst];
        } else if (qq >= N) {
          f = flux[off + glast];
          v = ivar[off + glast];
        } else {
          const double dx = dsub(wave[qq], wave[p]);
          const double x = dsub(wave[j], wave[p]);
          f = dadd(dmul(ddiv(dsub(flux[off + qq], flux[off + p]), dx), x), flux[off + p]);
          v = dadd(dmul(ddiv(dsub(ivar[off + qq], ivar[off + p]), dx), x), ivar[off + p]);
        }
      }
      tf[j] = f;
      tv[j] = v;
      if (v > 0.0) mn = fmin(mn, v);
    }
    // the smallest positive ivar of the exposure replaces ivar <= 0
    sh_min[t] = mn;
    __syncthreads();
    for (int w = kCosmicThreads / 2; w > 0; w >>= 1) {
      if (t < w) sh_min[t] = fmin(sh_min[t], sh_min[t + w]);
      __syncthreads();
    }
    const double minpos = sh_min[0];
    if (!(minpos < INFINITY)) {
      if (t == 0) set_status(status, RR_EINVAL);
      return;
    }
    for (int64_t j = lo; j < hi; ++j)
      if (tv[j] <= 0.0) tv[j] = minpos;
    // 2. gradient and its inverse variance, in place right to left; the
    //    left neighbour of each chunk is read before it is overwritten
    __syncthreads();
    const double fl = lo > 0 ? tf[lo - 1] : 0.0;
    const double vl = lo > 0 ? tv[lo - 1] : 1.0;
    __syncthreads();
    for (int64_t j = hi - 1; j >= lo; --j) {
      const double var = ddiv(1.0, tv[j]);
      if (j == 0) {
        tf[j] = 0.0;
        tv[j] = ddiv(1.0, var);
      } else {
        const double fp = j > lo ? tf[j - 1] : fl;
        const double vp = j > lo ? tv[j - 1] : vl;
        tf[j] = dsub(tf[j], fp);
        tv[j] = ddiv(1.0, dadd(var, ddiv(1.0, vp)));
      }
    }
    __syncthreads();
  }
  if (S < 2) return;
  // 3. the total of gradivar over all exposures and pixels, numpy's order
  if (t == 0) {
    const int64_t first = g.first;
    sh_total = pairwise_sum((int64_t)S * N, [&](int64_t e) {
      const int64_t s = e / N;
      return work_v[exp_pix[first + s] + (e - s * N)];
    });
  }
  __syncthreads();
  const double total = sh_total;
  // 4. per pixel: chi2 of the gradients across exposures, mask the worst
  for (int64_t j = t; j < N; j += kCosmicThreads) {
    double mg = 0.0;
    for (int s = 0; s < S; ++s) {
      const int64_t o = exp_pix[g.first + s] + j;
      const double v = dmul(work_v[o], work_f[o]);
      mg = s ? dadd(mg, v) : v;
    }
    mg = ddiv(mg, total);
    double c2 = 0.0, best = 0.0;
    int k = 0;
    bool nan_seen = false;
    for (int s = 0; s < S; ++s) {
      const int64_t o = exp_pix[g.first + s] + j;
      const double d = dsub(work_f[o], mg);
      const double v = dmul(work_v[o], dmul(d, d));
      c2 = s ? dadd(c2, v) : v;
      // numpy's argmax: the first maximum, a NaN counting as the maximum
      if (s == 0) {
        best = v;
        nan_seen = isnan(v);
      } else if (!nan_seen) {
        if (isnan(v)) {
          nan_seen = true;
          k = s;
        } else if (v > best) {
          best = v;
          k = s;
        }
      }
    }
    c2 = ddiv(c2, (double)(S - 1));
    if (c2 > thresh) ivar_out[exp_pix[g.first + k] + j] = 0.0;
  }
}

}  // namespace rr

using namespace rr;

extern "C" int rr_coadd_ex(const rr_coadd_group* groups, int64_t ngroup, int64_t max_npix,
                           const int64_t* exp_data, const int64_t* exp_pix, const double* rdata,
                           const double* ivar_rdata, const double* ivar, const double* flux,
                           double* rdata_out, double* ivar_out, double* flux_out,
                           rr_stream_t stream) {
  if (ngroup < 0 || ngroup > 65535 || max_npix < 0) return RR_EINVAL;
  if (ngroup == 0 || max_npix == 0) return RR_OK;
  if (!groups || !exp_data || !exp_pix || !rdata || !ivar || !flux || !rdata_out || !ivar_out ||
      !flux_out)
    return RR_EINVAL;
  if (!ivar_rdata) ivar_rdata = ivar;
  dim3 grid((unsigned)((max_npix + 255) / 256), (unsigned)ngroup);
  coadd_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(groups, exp_data, exp_pix, rdata,
                                                       ivar_rdata, ivar, flux, rdata_out,
                                                       ivar_out, flux_out);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_coadd(const rr_coadd_group* groups, int64_t ngroup, int64_t max_npix,
                        const int64_t* exp_data, const int64_t* exp_pix, const double* rdata,
                        const double* ivar, const double* flux, double* rdata_out,
                        double* ivar_out, double* flux_out, rr_stream_t stream) {
  return rr_coadd_ex(groups, ngroup, max_npix, exp_data, exp_pix, rdata, ivar, ivar, flux,
                     rdata_out, ivar_out, flux_out, stream);
}

extern "C" int rr_coadd_cosmics(const rr_coadd_group* groups, int64_t ngroup,
                                const int64_t* exp_pix, const double* wave, const double* ivar,
                                const double* flux, double nsig2, double* ivar_out, double* work,
                                int64_t npix_total, int* status, rr_stream_t stream) {
  if (ngroup < 0 || ngroup > 2147483647LL || npix_total < 0) return RR_EINVAL;
  if (ngroup == 0) return RR_OK;
  if (!groups || !exp_pix || !wave || !ivar || !flux || !ivar_out || !work) return RR_EINVAL;
  cosmics_kernel<<<(unsigned)ngroup, kCosmicThreads, 0, (cudaStream_t)stream>>>(
      groups, exp_pix, wave, ivar, flux, nsig2, ivar_out, work, work + npix_total, status);
  RR_CHECK_LAUNCH();
  return RR_OK;
}
