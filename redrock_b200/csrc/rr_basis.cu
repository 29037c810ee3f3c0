// Basis builder: trapezoidal rebinning of template bases onto camera pixel
// bins for every redshift, fused with the IGM (Lyman-series) transmission.
//
// Reference behaviour followed (redrock 0.22):
//   _trapz_rebin_1d     rebin.py:126-176   (per-bin walk over input samples)
//   _trapz_rebin_batch  rebin.py:178-209   (x * (1 + z) per redshift)
//   trapz_rebin         rebin.py:212-378   (range check, output layout)
//   Inoue14             igm.py:105-267     (LAF/DLA series + continuum)
//   CaluraKamble        igm.py:321-364
//   DistTemplate        templates.py:584-597 (rebin, then data *= T)
//
// Design: one thread per (z, output bin) computes every basis of that bin.
// The first input sample beyond the bin's lower edge is found by binary
// search on the redshifted grid (the reference walks it sequentially; both
// land on the first j with x[j](1+z) > edge).  All arithmetic of the rebin
// uses explicitly rounded operations in the reference's order, so results
// are bit-identical to redrock's CPU path.  The IGM factor of the bin's
// centre wavelength is computed in the same thread and multiplied in.
#include "rr_rebin_dev.cuh"

namespace rr {

__global__ void igm_kernel(int model, const double* __restrict__ z, int64_t nz,
                           const double* __restrict__ lobs, int64_t nwave, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t iz = blockIdx.y;
  if (i >= nwave || iz >= nz) return;
  out[iz * nwave + i] = transmission(model, z[iz], lobs[i]);
}

// out[(iz * z_stride) + ibin * bin_stride + b]
__global__ void trapz_rebin_kernel(const double* __restrict__ x, int64_t nx,
                                   const double* __restrict__ y, int nb,
                                   const double* __restrict__ edges, int64_t nbin,
                                   const double* __restrict__ z, int64_t nz, double* __restrict__ out,
                                   int64_t z_stride, int64_t bin_stride, int* status) {
  const int64_t ibin = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t iz = blockIdx.y;
  if (ibin >= nbin || iz >= nz) return;
  const double zp1 = dadd(1.0, z[iz]);
  double res[kMaxRebinBasis];
  double* o = out + iz * z_stride + ibin * bin_stride;
  if (!rebin_bin(x, nx, y, nb, zp1, edges[ibin], edges[ibin + 1], res)) {
    set_status(status, RR_ERANGE);
    for (int b = 0; b < nb; ++b) o[b] = nan("");
    return;
  }
  for (int b = 0; b < nb; ++b) o[b] = res[b];
}

// Fused builder for one grid: rebin + IGM into the padded basis layout.
// Threads cover the padded pixel range [pix_offset - 5, pix_offset +
// npix_pad + 5); pixels outside [pix_offset, pix_offset + npix) and basis
// columns >= nb are written as 0 so the scan's halo reads see zeros.
__global__ void build_basis_kernel(const double* __restrict__ x, int64_t nx,
                                   const double* __restrict__ y, int nb,
                                   const double* __restrict__ z, int64_t nz,
                                   const double* __restrict__ edges,
                                   const double* __restrict__ wave, int64_t npix, int64_t npix_pad,
                                   int64_t pix_offset, int igm_model, int apply_igm,
                                   double* __restrict__ basis, int64_t pix_stride,
                                   int basis_stride, int* status) {
  const int64_t span = npix_pad + 2 * kHalfBand;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // 0..span-1
  const int64_t iz = blockIdx.y;
  if (i >= span || iz >= nz) return;
  const int64_t ipix = i - kHalfBand;  // pixel index within the grid
  double* o = basis + (iz * pix_stride + pix_offset + ipix) * basis_stride;
  if (ipix < 0 || ipix >= npix) {
    for (int b = 0; b < basis_stride; ++b) o[b] = 0.0;
    return;
  }
  const double zz = z[iz];
  const double zp1 = dadd(1.0, zz);
  double res[kMaxRebinBasis];
  if (!rebin_bin(x, nx, y, nb, zp1, edges[ipix], edges[ipix + 1], res)) {
    set_status(status, RR_ERANGE);
    for (int b = 0; b < basis_stride; ++b) o[b] = nan("");
    return;
  }
  if (apply_igm) {
    const double t = transmission(igm_model, zz, wave[ipix]);
    for (int b = 0; b < nb; ++b) res[b] = dmul(res[b], t);
  }
  for (int b = 0; b < nb; ++b) o[b] = res[b];
  for (int b = nb; b < basis_stride; ++b) o[b] = 0.0;
}

}  // namespace rr

using namespace rr;

extern "C" int rr_trapz_rebin(const double* x, int64_t nx, const double* y, int64_t nbasis,
                              const double* edges, int64_t nbin, const double* z, int64_t nz,
                              double xmin, double xmax, double edge_min, double edge_max,
                              double* out, int* status, rr_stream_t stream) {
  if (nx < 2 || nbasis < 1 || nbasis > kMaxRebinBasis || nbin < 1 || nz < 0) return RR_EINVAL;
  if (!x || !y || !edges || (nz > 0 && (!z || !out))) return RR_EINVAL;
  if (edge_min < xmin || edge_max > xmax) return RR_ERANGE;
  if (nz == 0) return RR_OK;
  if (nz > 65535) return RR_ENOTSUP;
  dim3 block(128);
  dim3 grid((unsigned)((nbin + block.x - 1) / block.x), (unsigned)nz);
  trapz_rebin_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      x, nx, y, (int)nbasis, edges, nbin, z, nz, out, nbin * nbasis, nbasis, status);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_igm_transmission(int model, const double* z, int64_t nz, const double* lobs,
                                   int64_t nwave, double* out, rr_stream_t stream) {
  if (model < RR_IGM_NONE || model > RR_IGM_INOUE14) return RR_EINVAL;
  if (nz < 0 || nwave < 0) return RR_EINVAL;
  if (nz == 0 || nwave == 0) return RR_OK;
  if (!z || !lobs || !out) return RR_EINVAL;
  if (nz > 65535) return RR_ENOTSUP;
  int rc = upload_igm_tables((cudaStream_t)stream);
  if (rc) return rc;
  dim3 block(128);
  dim3 grid((unsigned)((nwave + block.x - 1) / block.x), (unsigned)nz);
  igm_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(model, z, nz, lobs, nwave, out);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_build_basis(const double* x, int64_t nx, const double* y, int64_t nbasis,
                              const double* z, int64_t nz, double xmin, double xmax,
                              const rr_grid_desc* grids, int ngrid, int igm_model,
                              int64_t pix_stride, int basis_stride, double* basis, int* status,
                              rr_stream_t stream) {
  if (nx < 2 || nbasis < 1 || nbasis > kMaxRebinBasis || nz < 0 || ngrid < 1 || !grids)
    return RR_EINVAL;
  if (basis_stride < nbasis || (basis_stride & 1)) return RR_EINVAL;
  if (igm_model < RR_IGM_NONE || igm_model > RR_IGM_INOUE14) return RR_EINVAL;
  if (nz > 65535) return RR_ENOTSUP;
  for (int g = 0; g < ngrid; ++g) {
    const rr_grid_desc& gd = grids[g];
    if (gd.npix < 1 || gd.npix_pad < gd.npix || (gd.npix_pad % RR_CHUNK) != 0) return RR_EINVAL;
    if (gd.pix_offset < kHalfBand || gd.pix_offset + gd.npix_pad + kHalfBand > pix_stride)
      return RR_EINVAL;
    if (gd.edge_min < xmin || gd.edge_max > xmax) return RR_ERANGE;
  }
  if (nz == 0) return RR_OK;
  int rc = upload_igm_tables((cudaStream_t)stream);
  if (rc) return rc;
  for (int g = 0; g < ngrid; ++g) {
    const rr_grid_desc& gd = grids[g];
    const int64_t span = gd.npix_pad + 2 * kHalfBand;
    dim3 block(128);
    dim3 grid((unsigned)((span + block.x - 1) / block.x), (unsigned)nz);
    build_basis_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
        x, nx, y, (int)nbasis, z, nz, gd.edges, gd.wave, gd.npix, gd.npix_pad, gd.pix_offset,
        igm_model, gd.apply_igm && igm_model != RR_IGM_NONE, basis, pix_stride, basis_stride,
        status);
    RR_CHECK_LAUNCH();
  }
  return RR_OK;
}
