// Coadd of a target's exposures per wavelength grid (redrock 0.22
// targets.py:267-373, Target.compute_coadd with cosmics_nsig = 0).
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
// redrock's.  One thread per (group, pixel).
#include "rr_common.cuh"

namespace rr {

__global__ void __launch_bounds__(256) coadd_kernel(const rr_coadd_group* __restrict__ groups,
                                                    const int64_t* __restrict__ exp_data,
                                                    const int64_t* __restrict__ exp_pix,
                                                    const double* __restrict__ rdata,
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
      const double v = dmul(rdata[exp_data[e] + (int64_t)d * g.npix + j], ivar[exp_pix[e] + j]);
      r = s ? dadd(r, v) : v;
    }
    rdata_out[g.out_data + (int64_t)d * g.npix + j] = ddiv(r, den);
  }
}

}  // namespace rr

using namespace rr;

extern "C" int rr_coadd(const rr_coadd_group* groups, int64_t ngroup, int64_t max_npix,
                        const int64_t* exp_data, const int64_t* exp_pix, const double* rdata,
                        const double* ivar, const double* flux, double* rdata_out,
                        double* ivar_out, double* flux_out, rr_stream_t stream) {
  if (ngroup < 0 || ngroup > 65535 || max_npix < 0) return RR_EINVAL;
  if (ngroup == 0 || max_npix == 0) return RR_OK;
  if (!groups || !exp_data || !exp_pix || !rdata || !ivar || !flux || !rdata_out || !ivar_out ||
      !flux_out)
    return RR_EINVAL;
  dim3 grid((unsigned)((max_npix + 255) / 256), (unsigned)ngroup);
  coadd_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(groups, exp_data, exp_pix, rdata, ivar,
                                                       flux, rdata_out, ivar_out, flux_out);
  RR_CHECK_LAUNCH();
  return RR_OK;
}
