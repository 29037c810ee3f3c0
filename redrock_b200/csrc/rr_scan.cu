// Redshift scan: chi2(z) and best-fit coefficients of every target against
// every template basis, with the [OII] penalty.
//
// Reference (redrock 0.22):
//   calc_zchi2_batch  zscan.py:626-781  Tb = R.T, M = Tb^T W Tb, y = Tb^T W f,
//                                        solve, chi2 = sum w (f - Tb c)^2
//   calc_zchi2        zscan.py:807-889  loop over targets, all-zero weights
//                                        -> HUGE_CHI2, [OII] penalty
//   solve_matrices    zscan.py:1107-1152 (PCA: LAPACK gesv; exactly
//                                        singular -> LinAlgError -> HUGE)
//   calc_negOII_penalty zscan.py:783-800
//
// Fused path (rr_zscan_fused).  A target's data is first packed as
//   rw[p][k] = sqrt(w_p) R[p, p+k-5]  (k < 11),  rw[p][11] = sqrt(w_p) f_p
// so that with Tb' = rw . T_z (the weighted resolution-convolved basis)
//   M = sum_p Tb'_p Tb'_p^T,  y = sum_p rw[p][11] Tb'_p,
// which are redrock's M and y.  chi2 = f^T W f - c^T y - c^T P c at the
// solution of (M + P) c = y equals redrock's sum w (f - Tb c)^2.
//
// One CTA = 8 warps; a tile is (template, block of 32 targets, 8 redshifts):
// warp w scans redshift z0 + w, lane l target l of the block, so each lane
// owns one (target, z) pair and keeps its 55 (n = 10) Gram entries and y in
// FP64 registers for the whole pixel sweep.  Pixels stream through shared
// memory in chunks of 16: one bulk (TMA) copy brings the block's packed
// resolution rows for the chunk (coalesced over lanes) and one copy per
// warp brings that redshift's basis window (chunk + 5-pixel halo each side);
// the basis values are read as warp-wide broadcasts.  Two stages alternate
// so the copy of chunk c+1 overlaps the arithmetic on chunk c.  Tiles are
// handed out by an atomic counter (persistent CTAs) across all templates, so
// templates with different nbasis / nz share one launch.  The epilogue
// solves the n x n system in registers (LDL^T, no pivoting; an exactly zero
// pivot is redrock's singular case) and writes chi2, coefficients and the
// penalty.
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "rr_common.cuh"
#include "rr_lsq_dev.cuh"
#include "rr_solve_dev.cuh"

#include "rr_fused.cuh"
#include "rr_lsq_dev.cuh"

namespace rr {
// ---------------------------------------------------------------------------
// packing
// ---------------------------------------------------------------------------

// One thread per (spectrum pixel): band row of R at that pixel from the DIA
// data, where data[d][j] = R[j - off_d, j] (scipy dia_matrix convention).
__device__ __forceinline__ void band_row(const double* __restrict__ rdata,
                                         const int32_t* __restrict__ roff,
                                         const rr_spectrum_desc& sd, int64_t i, double (&r)[kBand],
                                         int* status) {
#pragma unroll
  for (int k = 0; k < kBand; ++k) r[k] = 0.0;
  for (int d = 0; d < sd.ndiag; ++d) {
    const int off = roff[sd.diag_offset + d];
    if (off < -kHalfBand || off > kHalfBand) {
      // only reachable if the host check was bypassed; a nonzero band value
      // outside the kernel's band would be silently dropped
      const int64_t j = i + off;
      if (j >= 0 && j < sd.npix && rdata[sd.data_offset + (int64_t)d * sd.npix + j] != 0.0)
        set_status(status, RR_ENOTSUP);
      continue;
    }
    const int64_t j = i + off;
    if (j >= 0 && j < sd.npix) r[off + kHalfBand] += rdata[sd.data_offset + (int64_t)d * sd.npix + j];
  }
}

__global__ void pack_targets_kernel(const rr_spectrum_desc* __restrict__ specs, int64_t nspec,
                                    const double* __restrict__ rdata,
                                    const int32_t* __restrict__ roff,
                                    const double* __restrict__ ivar, const double* __restrict__ flux,
                                    const rr_segment_desc* __restrict__ segs, int64_t npix_block,
                                    double* __restrict__ rw, int* status) {
  const int64_t s = blockIdx.y;
  if (s >= nspec) return;
  const rr_spectrum_desc sd = specs[s];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= sd.npix) return;
  const rr_segment_desc seg = segs[sd.segment];
  if (i >= seg.npix_pad) { set_status(status, RR_EINVAL); return; }
  double r[kBand];
  band_row(rdata, roff, sd, i, r, status);
  const double w = ivar[sd.pix_offset + i];
  const double sw = sqrt(w);
  double* o = rw + ((int64_t)sd.block * npix_block + seg.rw_offset + i) * (RR_RW * RR_LANES) + sd.lane;
#pragma unroll
  for (int k = 0; k < kBand; ++k) o[k * RR_LANES] = sw * r[k];
  o[kBand * RR_LANES] = sw * flux[sd.pix_offset + i];
}

// Per-target sums f^T W f and sum w in FP64.  One CTA per target walks the
// target's spectra in order (spectra are grouped by target, target t owning
// specs[first[t] .. first[t+1])), so the summation order is fixed.
__global__ void pack_sums_kernel(const rr_spectrum_desc* __restrict__ specs,
                                 const int64_t* __restrict__ first, int64_t ntarget,
                                 const double* __restrict__ ivar, const double* __restrict__ flux,
                                 double* __restrict__ fwf, double* __restrict__ wsum) {
  const int64_t t = blockIdx.x;
  if (t >= ntarget) return;
  __shared__ double red[2][256];
  double tot_a = 0.0, tot_b = 0.0;
  int64_t slot = -1;
  for (int64_t s = first[t]; s < first[t + 1]; ++s) {
    const rr_spectrum_desc sd = specs[s];
    slot = (int64_t)sd.block * RR_LANES + sd.lane;
    double a = 0.0, b = 0.0;
    for (int64_t i = threadIdx.x; i < sd.npix; i += blockDim.x) {
      const double w = ivar[sd.pix_offset + i];
      const double f = flux[sd.pix_offset + i];
      a += w * f * f;
      b += w;
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) {
        red[0][threadIdx.x] += red[0][threadIdx.x + h];
        red[1][threadIdx.x] += red[1][threadIdx.x + h];
      }
      __syncthreads();
    }
    tot_a += red[0][0];
    tot_b += red[1][0];
    __syncthreads();
  }
  if (threadIdx.x == 0 && slot >= 0) {
    fwf[slot] = tot_a;
    wsum[slot] = tot_b;
  }
}

__global__ void pack_band_rows_kernel(const rr_spectrum_desc* __restrict__ specs, int64_t nspec,
                                      const double* __restrict__ rdata,
                                      const int32_t* __restrict__ roff, double* __restrict__ band,
                                      int* status) {
  const int64_t s = blockIdx.y;
  if (s >= nspec) return;
  const rr_spectrum_desc sd = specs[s];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= sd.npix) return;
  double r[kBand];
  band_row(rdata, roff, sd, i, r, status);
  double* o = band + (sd.pix_offset + i) * kBand;
#pragma unroll
  for (int k = 0; k < kBand; ++k) o[k] = r[k];
}

// ---------------------------------------------------------------------------
// plain per-target path
// ---------------------------------------------------------------------------

// Tb[z][p][b] = sum_k band[p][k] basis[z][pix_basis[p] + k - 5][b]
__global__ void plain_rt_kernel(const double* __restrict__ band, const int64_t* __restrict__ pix_basis,
                                int64_t npix, const double* __restrict__ basis, int64_t pix_stride,
                                int nz, int nb, int stride, double* __restrict__ tb, int* status) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)nz * npix * nb;
  if (i >= total) return;
  const int b = (int)(i % nb);
  const int64_t pz = i / nb;
  const int64_t p = pz % npix;
  const int64_t z = pz / npix;
  const int64_t pb = pix_basis[p];
  // the 11 basis rows of the band must lie inside this redshift's rows
  if (pb < kHalfBand || pb + kHalfBand >= pix_stride) {
    set_status(status, RR_EINVAL);
    tb[i] = 0.0;
    return;
  }
  const double* t = basis + (z * pix_stride + pb - kHalfBand) * stride + b;
  const double* r = band + p * kBand;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kBand; ++k) acc = fma(r[k], t[(int64_t)k * stride], acc);
  tb[i] = acc;
}

// One CTA per z: M = Tb^T W Tb (lower triangle) and y = Tb^T (w f),
// deterministic tree reduction.
template <int NB>
__global__ void plain_gram_kernel(const double* __restrict__ tb, const double* __restrict__ w,
                                  const double* __restrict__ wflux, int64_t npix,
                                  double* __restrict__ mout, double* __restrict__ yout) {
  constexpr int kTri = NB * (NB + 1) / 2;
  const int64_t z = blockIdx.x;
  const double* t = tb + z * npix * NB;
  double m[kTri], y[NB];
#pragma unroll
  for (int i = 0; i < kTri; ++i) m[i] = 0.0;
#pragma unroll
  for (int i = 0; i < NB; ++i) y[i] = 0.0;
  for (int64_t p = threadIdx.x; p < npix; p += blockDim.x) {
    double v[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) v[b] = t[p * NB + b];
    const double wp = w[p], wf = wflux[p];
#pragma unroll
    for (int a = 0; a < NB; ++a) {
      y[a] = fma(v[a], wf, y[a]);
      const double wa = wp * v[a];
#pragma unroll
      for (int b = 0; b <= a; ++b) m[a * (a + 1) / 2 + b] = fma(wa, v[b], m[a * (a + 1) / 2 + b]);
    }
  }
  __shared__ double red[128];
#pragma unroll 1
  for (int e = 0; e < kTri + NB; ++e) {
    red[threadIdx.x] = e < kTri ? m[e] : y[e - kTri];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (e < kTri) mout[z * kTri + e] = red[0];
      else yout[z * NB + (e - kTri)] = red[0];
    }
    __syncthreads();
  }
}

template <int NB>
__global__ void plain_solve_kernel(const double* __restrict__ mtri, const double* __restrict__ y,
                                   int nz, const double* __restrict__ prior, int method,
                                   double* __restrict__ zcoeff, unsigned char* __restrict__ bad) {
  constexpr int kTri = NB * (NB + 1) / 2;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= nz) return;
  double a[kTri], yy[NB], c[NB];
#pragma unroll
  for (int i = 0; i < kTri; ++i) a[i] = mtri[(int64_t)z * kTri + i];
#pragma unroll
  for (int i = 0; i < NB; ++i) yy[i] = y[(int64_t)z * NB + i];
  bool ok = method == RR_SOLVE_PCA;
  if (ok && prior) {
#pragma unroll
    for (int i = 0; i < NB; ++i)
#pragma unroll
      for (int j = 0; j <= i; ++j) a[i * (i + 1) / 2 + j] += prior[i * NB + j];
  }
  if (ok) ok = ldlt_solve<NB>(a, yy, c);
  if (!ok) {
#pragma unroll
    for (int i = 0; i < NB; ++i) c[i] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < NB; ++i) zcoeff[(int64_t)z * NB + i] = c[i];
  bad[z] = ok ? 0 : 1;
}

// Bounded solves of (M + prior) c ~ y in redrock's scipy sense (min
// ||(M + P) c - y||, rr_lsq_dev.cuh), one thread per z: RR_SOLVE_NNLS and
// RR_SOLVE_BVLS.  Separate from the PCA kernel so the common path keeps its
// registers.
template <int NB>
__global__ void plain_lsq_kernel(const double* __restrict__ mtri, const double* __restrict__ y,
                                 int nz, const double* __restrict__ prior, int method,
                                 const __grid_constant__ SolveBounds bounds,
                                 double* __restrict__ zcoeff, unsigned char* __restrict__ bad) {
  constexpr int kTri = NB * (NB + 1) / 2;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= nz) return;
  double full[NB][NB], yy[NB], c[NB];
  for (int i = 0; i < NB; ++i) {
    yy[i] = y[(int64_t)z * NB + i];
    for (int j = 0; j <= i; ++j) {
      double v = mtri[(int64_t)z * kTri + i * (i + 1) / 2 + j];
      if (prior) v += prior[i * NB + j];
      full[i][j] = full[j][i] = v;
    }
  }
  bool ok;
  if (method == RR_SOLVE_NNLS) {
    ok = nnls_solve<NB>(full, yy, c);
  } else {
    // the bounds are read in place from the parameter: with local copies
    // (double lo[NB], hi[NB] filled from it) nvcc 12.9 gave the copies
    // the same local-memory slots as the solver's own work arrays, and
    // BVLS read its bounds from the overwritten storage
    ok = bvls_solve<NB>(full, yy, bounds.lo, bounds.hi, c);
  }
  for (int i = 0; i < NB; ++i) zcoeff[(int64_t)z * NB + i] = ok ? c[i] : 0.0;
  bad[z] = ok ? 0 : 1;
}

// chi2[z] = sum_p w (f - Tb c)^2, deterministic reduction; HUGE if bad
// (for every method: the constrained solutions are not stationary points of
// f^T W f - c^T y, so chi2 is always the direct residual here).
template <int NB>
__global__ void plain_chi2_kernel(const double* __restrict__ tb, const double* __restrict__ w,
                                  const double* __restrict__ flux, int64_t npix,
                                  const double* __restrict__ zcoeff,
                                  const unsigned char* __restrict__ bad, double* __restrict__ zchi2) {
  const int64_t z = blockIdx.x;
  const double* t = tb + z * npix * NB;
  double c[NB];
#pragma unroll
  for (int i = 0; i < NB; ++i) c[i] = zcoeff[z * NB + i];
  double acc = 0.0;
  for (int64_t p = threadIdx.x; p < npix; p += blockDim.x) {
    double model = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) model = fma(t[p * NB + b], c[b], model);
    const double r = flux[p] - model;
    acc = fma(w[p], r * r, acc);
  }
  __shared__ double red[128];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) zchi2[z] = bad[z] ? kHugeChi2 : red[0];
}

__global__ void negoii_kernel(const double* __restrict__ coeff, int64_t nz, int nb,
                              const double* __restrict__ oii, double* __restrict__ pen) {
  const int64_t z = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (z >= nz) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s = fma(coeff[z * nb + b], oii[b], s);
  pen[z] = s < 0.0 ? -s : 0.0;
}

}  // namespace rr

using namespace rr;

static thread_local int g_last_cuda_error = 0;

extern "C" int rr_last_cuda_error(void) { return g_last_cuda_error; }

extern "C" int rr_version(void) { return 1; }

extern "C" int rr_scan_chunk(void) { return kChunk; }

extern "C" const char* rr_status_string(int status) {
  switch (status) {
    case RR_OK: return "ok";
    case RR_EINVAL: return "invalid argument";
    case RR_ERANGE: return "edges must be within input x range";
    case RR_ECUDA: return "CUDA runtime error";
    case RR_ETIMEOUT: return "bounded device wait timed out";
    case RR_ENOTSUP: return "unsupported input";
    case RR_ESCRATCH:
      return "request exceeds the fixed scratch of the no-allocation entry point";
    default: return "unknown status";
  }
}

#undef RR_CUDA_TRY
#define RR_CUDA_TRY(expr)                        \
  do {                                           \
    cudaError_t _e = (expr);                     \
    if (_e != cudaSuccess) {                     \
      g_last_cuda_error = (int)_e;               \
      return RR_ECUDA;                           \
    }                                            \
  } while (0)

#undef RR_CHECK_LAUNCH
#define RR_CHECK_LAUNCH() RR_CUDA_TRY(cudaGetLastError())


static int zscan_fused(const rr_scan_targets* targets, const rr_scan_template* templates,
                       int ntemplate, int* tile_counter, const rr_scan_options* opt, int* status,
                       rr_stream_t stream) {
  if (!targets || !templates || !tile_counter) return RR_EINVAL;
  if (ntemplate < 1 || ntemplate > RR_MAX_TEMPLATES) return RR_EINVAL;
  if (targets->nblock < 1 || targets->nseg < 1 || targets->nseg > 16) return RR_EINVAL;
  if (!targets->rw || !targets->fwf || !targets->wsum || !targets->rows || !targets->segs)
    return RR_EINVAL;
  if ((reinterpret_cast<uintptr_t>(targets->rw) & 15) != 0) return RR_EINVAL;
  int64_t rw_end = 0;
  for (int s = 0; s < targets->nseg; ++s) {
    const rr_segment_desc& sd = targets->segs[s];
    if (sd.npix_pad <= 0 || (sd.npix_pad % kChunk) != 0 || sd.basis_offset < kHalfBand ||
        sd.rw_offset < 0)
      return RR_EINVAL;
    rw_end = sd.rw_offset + sd.npix_pad > rw_end ? sd.rw_offset + sd.npix_pad : rw_end;
  }
  if (rw_end > targets->npix_block) return RR_EINVAL;
  int zt[kNGroups];
  for (int g = 0; g < kNGroups; ++g) zt[g] = kDefaultZt[g];
  int bgroup = 0;
  if (opt) {
    if (opt->block_group < 0) return RR_EINVAL;
    bgroup = opt->block_group;
    if (opt->zt_nbasis4 < 0 || opt->zt_nbasis4 > kMaxZt[1] || opt->zt_nbasis5 < 0 ||
        opt->zt_nbasis5 > kMaxZt[2])
      return RR_EINVAL;
    if (opt->zt_nbasis4) zt[1] = opt->zt_nbasis4;
    if (opt->zt_nbasis5) zt[2] = opt->zt_nbasis5;
  }
  // launch groups: (nbasis group, y_ext) -> one persistent launch each
  int group[2 * kNGroups][RR_MAX_TEMPLATES];
  int ng[2 * kNGroups] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = 0; t < ntemplate; ++t) {
    const rr_scan_template& tm = templates[t];
    if (tm.nbasis < 1 || tm.nbasis > RR_MAX_NBASIS || tm.nz < 0) return RR_EINVAL;
    if (tm.basis_stride < tm.nbasis || (tm.basis_stride & 1)) return RR_EINVAL;
    if (tm.nz > 0 && (!tm.basis || !tm.zchi2 || !tm.zcoeff)) return RR_EINVAL;
    if (tm.oii && !tm.penalty) return RR_EINVAL;
    if ((reinterpret_cast<uintptr_t>(tm.basis) & 15) != 0) return RR_EINVAL;
    for (int s = 0; s < targets->nseg; ++s)
      if (targets->segs[s].basis_offset + targets->segs[s].npix_pad + kHalfBand > tm.pix_stride)
        return RR_EINVAL;
    if (tm.y_ext && (reinterpret_cast<uintptr_t>(tm.y_ext) & 7) != 0) return RR_EINVAL;
    const int gi = group_of(tm.nbasis) + (tm.y_ext ? kNGroups : 0);
    group[gi][ng[gi]++] = t;
  }
  cudaStream_t st = (cudaStream_t)stream;
  // one zeroing of every counter before the first launch, so the launches
  // follow one another directly in the stream and each one after the first
  // can start on the SMs its predecessor's last tile wave leaves idle
  // (tile_counter[4 + g] hands out the tiles of launch g)
  RR_CUDA_TRY(cudaMemsetAsync(tile_counter, 0, RR_FUSED_COUNTERS * sizeof(int), st));
  int* resweep = tile_counter + 2;
  // Invariant of the programmatic dependent launches below: the group
  // launches are independent of one another -- each reads only the packed
  // targets, its own bases and y, all written before the first launch, and
  // writes only its own templates' outputs and its own tile counter (the
  // re-sweep counters are atomics).  That is why a dependent launch may
  // start before its predecessor finishes, and why each CTA can leave its
  // griddepcontrol.wait to the very end (it only orders completion for the
  // work after the last launch).  A change that makes one group read what
  // another writes must move that wait ahead of the read.
  int rc = RR_OK;
  bool overlap = false;
  typedef int (*group_fn)(bool, int, int, const rr_scan_targets*, const rr_scan_template*,
                          const int*, int, int*, int*, int*, bool, cudaStream_t);
  const group_fn fns[kNGroups] = {fused_group_0, fused_group_1, fused_group_2, fused_group_3};
  for (int gi = 0; gi < 2 * kNGroups && !rc; ++gi) {
    if (!ng[gi]) continue;
    const int g = gi % kNGroups;
    rc = fns[g](gi >= kNGroups, zt[g], bgroup, targets, templates, group[gi], ng[gi],
                tile_counter + 4 + gi, resweep, status, overlap, st);
    overlap = true;
  }
  return rc;
}

extern "C" int rr_zscan_fused(const rr_scan_targets* targets, const rr_scan_template* templates,
                              int ntemplate, int* tile_counter, int* status, rr_stream_t stream) {
  return zscan_fused(targets, templates, ntemplate, tile_counter, nullptr, status, stream);
}

extern "C" int rr_zscan_fused_opt(const rr_scan_targets* targets,
                                  const rr_scan_template* templates, int ntemplate,
                                  int* tile_counter, const rr_scan_options* opt, int* status,
                                  rr_stream_t stream) {
  return zscan_fused(targets, templates, ntemplate, tile_counter, opt, status, stream);
}

extern "C" int rr_pack_targets(const rr_spectrum_desc* specs, int64_t nspec,
                               const int64_t* target_first, int64_t ntarget, const double* rdata,
                               const int32_t* roffsets, const double* ivar, const double* flux,
                               const rr_segment_desc* segs, int nseg, int64_t npix_block,
                               int nblock, double* rw, double* fwf, double* wsum, int* status,
                               rr_stream_t stream) {
  if (nspec < 0 || ntarget < 0 || nseg < 1 || nblock < 1 || npix_block < 1) return RR_EINVAL;
  if (nspec == 0 || ntarget == 0) return RR_OK;
  if (!specs || !target_first || !rdata || !roffsets || !ivar || !flux || !segs || !rw || !fwf ||
      !wsum)
    return RR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  for (int64_t s0 = 0; s0 < nspec; s0 += 65535) {
    const int64_t n = nspec - s0 < 65535 ? nspec - s0 : 65535;
    dim3 block(128);
    dim3 grid((unsigned)((npix_block + block.x - 1) / block.x), (unsigned)n);
    pack_targets_kernel<<<grid, block, 0, st>>>(specs + s0, n, rdata, roffsets, ivar, flux, segs,
                                                npix_block, rw, status);
    RR_CHECK_LAUNCH();
  }
  pack_sums_kernel<<<(unsigned)ntarget, 256, 0, st>>>(specs, target_first, ntarget, ivar, flux, fwf,
                                                      wsum);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_pack_band_rows(const rr_spectrum_desc* specs, int64_t nspec, const double* rdata,
                                 const int32_t* roffsets, int64_t npix_total, double* band,
                                 int* status, rr_stream_t stream) {
  if (nspec < 0 || npix_total < 0) return RR_EINVAL;
  if (nspec == 0) return RR_OK;
  if (!specs || !rdata || !roffsets || !band || nspec > 65535) return RR_EINVAL;
  dim3 block(128);
  dim3 grid((unsigned)((npix_total + block.x - 1) / block.x), (unsigned)nspec);
  pack_band_rows_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(specs, nspec, rdata, roffsets,
                                                                  band, status);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// SIZE_MAX for sizes whose byte count does not fit (or negative sizes), so
// that every size check against it fails
extern "C" size_t rr_zchi2_batch_plain_workspace_bytes(int64_t npix_total, int32_t nz,
                                                       int32_t nbasis) {
  if (npix_total < 0 || nz < 0 || nbasis < 0) return SIZE_MAX;
  const size_t tri = (size_t)nbasis * (nbasis + 1) / 2;
  size_t tb = 0;
  if (__builtin_mul_overflow((size_t)nz, (size_t)npix_total, &tb) ||
      __builtin_mul_overflow(tb, (size_t)nbasis * sizeof(double), &tb) || tb > SIZE_MAX / 2)
    return SIZE_MAX;
  return align256(tb) + align256((size_t)nz * tri * sizeof(double)) +
         align256((size_t)nz * nbasis * sizeof(double)) + align256((size_t)nz);
}

template <int NB>
static int plain_launch(const double* band, const double* w, const double* wflux,
                        const double* flux, const int64_t* pix_basis, int64_t npix,
                        const double* basis, int64_t pix_stride, int nz, int stride,
                        const double* prior, int method, const SolveBounds& bounds,
                        double* zchi2, double* zcoeff, unsigned char* ws, int* status,
                        cudaStream_t st) {
  constexpr int kTri = NB * (NB + 1) / 2;
  double* tb = reinterpret_cast<double*>(ws);
  double* mtri = reinterpret_cast<double*>(ws + align256((size_t)nz * npix * NB * sizeof(double)));
  double* yv = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(mtri) +
                                         align256((size_t)nz * kTri * sizeof(double)));
  unsigned char* bad =
      reinterpret_cast<unsigned char*>(yv) + align256((size_t)nz * NB * sizeof(double));
  const int64_t total = (int64_t)nz * npix * NB;
  if ((total + 255) / 256 > (int64_t)INT32_MAX) return RR_EINVAL;
  plain_rt_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(band, pix_basis, npix, basis,
                                                                    pix_stride, nz, NB, stride, tb,
                                                                    status);
  RR_CHECK_LAUNCH();
  plain_gram_kernel<NB><<<nz, 128, 0, st>>>(tb, w, wflux, npix, mtri, yv);
  RR_CHECK_LAUNCH();
  if (method == RR_SOLVE_NNLS || method == RR_SOLVE_BVLS)
    plain_lsq_kernel<NB><<<(nz + 63) / 64, 64, 0, st>>>(mtri, yv, nz, prior, method, bounds,
                                                        zcoeff, bad);
  else
    plain_solve_kernel<NB><<<(nz + 127) / 128, 128, 0, st>>>(mtri, yv, nz, prior, method, zcoeff,
                                                              bad);
  RR_CHECK_LAUNCH();
  plain_chi2_kernel<NB><<<nz, 128, 0, st>>>(tb, w, flux, npix, zcoeff, bad, zchi2);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

static int plain_entry(const double* band, const double* w, const double* wflux,
                                    const double* flux, const int64_t* pix_basis,
                                    int64_t npix_total, const double* basis, int64_t pix_stride,
                                    int32_t nz, int32_t nbasis, int32_t basis_stride,
                                    const double* prior, int32_t method, double* zchi2,
                                    double* zcoeff, void* workspace, size_t workspace_bytes,
                                    int* status, rr_stream_t stream, const double* bounds) {
  SolveBounds sb;
  for (int i = 0; i < RR_MAX_NBASIS; ++i) {
    sb.lo[i] = -INFINITY;
    sb.hi[i] = INFINITY;
  }
  if (bounds && nbasis >= 1 && nbasis <= RR_MAX_NBASIS)
    for (int i = 0; i < nbasis; ++i) {
      sb.lo[i] = bounds[i];
      sb.hi[i] = bounds[nbasis + i];
      if (!(sb.lo[i] <= sb.hi[i])) return RR_EINVAL;
    }
  if (nz < 0 || npix_total < 1 || nbasis < 1 || nbasis > RR_MAX_NBASIS) return RR_EINVAL;
  if (basis_stride < nbasis) return RR_EINVAL;
  if (nz == 0) return RR_OK;
  if (!band || !w || !wflux || !flux || !pix_basis || !basis || !zchi2 || !zcoeff || !workspace)
    return RR_EINVAL;
  if (workspace_bytes < rr_zchi2_batch_plain_workspace_bytes(npix_total, nz, nbasis))
    return RR_EINVAL;
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  cudaStream_t st = (cudaStream_t)stream;
#define RR_PLAIN_CASE(N)                                                                          \
  case N:                                                                                         \
    return plain_launch<N>(band, w, wflux, flux, pix_basis, npix_total, basis, pix_stride, nz,    \
                           basis_stride, prior, method, sb, zchi2, zcoeff, ws, status, st);
  switch (nbasis) {
    RR_PLAIN_CASE(1)
    RR_PLAIN_CASE(2)
    RR_PLAIN_CASE(3)
    RR_PLAIN_CASE(4)
    RR_PLAIN_CASE(5)
    RR_PLAIN_CASE(6)
    RR_PLAIN_CASE(7)
    RR_PLAIN_CASE(8)
    RR_PLAIN_CASE(9)
    RR_PLAIN_CASE(10)
    default: return RR_EINVAL;
  }
#undef RR_PLAIN_CASE
}

extern "C" int rr_zchi2_batch_plain(const double* band, const double* w, const double* wflux,
                                    const double* flux, const int64_t* pix_basis,
                                    int64_t npix_total, const double* basis, int64_t pix_stride,
                                    int32_t nz, int32_t nbasis, int32_t basis_stride,
                                    const double* prior, int32_t method, double* zchi2,
                                    double* zcoeff, void* workspace, size_t workspace_bytes,
                                    int* status, rr_stream_t stream) {
  return plain_entry(band, w, wflux, flux, pix_basis, npix_total, basis, pix_stride, nz, nbasis,
                     basis_stride, prior, method, zchi2, zcoeff, workspace, workspace_bytes,
                     status, stream, nullptr);
}

extern "C" int rr_zchi2_batch_plain_ex(const double* band, const double* w, const double* wflux,
                                       const double* flux, const int64_t* pix_basis,
                                       int64_t npix_total, const double* basis, int64_t pix_stride,
                                       int32_t nz, int32_t nbasis, int32_t basis_stride,
                                       const double* prior, int32_t method, const double* bounds,
                                       double* zchi2, double* zcoeff, void* workspace,
                                       size_t workspace_bytes, int* status, rr_stream_t stream) {
  return plain_entry(band, w, wflux, flux, pix_basis, npix_total, basis, pix_stride, nz, nbasis,
                     basis_stride, prior, method, zchi2, zcoeff, workspace, workspace_bytes,
                     status, stream, bounds);
}

// ---------------------------------------------------------------------------
// No-allocation variant of the plain per-target chain.
//
// For callers that cannot allocate device memory themselves: programs whose
// own memory manager already owns the GPU's memory (a raw cudaMalloc there
// may fail or fragment it), or latency-bound loops in which a cudaMalloc /
// cudaFree could synchronise the device.  Its scratch is the file-scope
// array below, created when the library is loaded and kept on every GPU
// that loads the library until the process exits.
//
// * Maximum request: rr_zchi2_batch_plain_workspace_bytes(npix, nz, nbasis)
//   <= RR_NOALLOC_SCRATCH_BYTES (16 MiB; e.g. 15 redshifts x 8000 pixels x
//   10 bases); larger requests return RR_ESCRATCH before any launch.
// * All calls share the one array.  It keeps the previous call's contents;
//   every byte a call reads is written earlier in the same call, so nothing
//   needs clearing.  Calls that overlap on the GPU (different streams or
//   host threads, same device) race on it and must be serialised by the
//   caller.
// * The first call on each device looks up the array's device address
//   (cudaGetSymbolAddress) with that device current and caches it; make
//   that first call before any stream capture.  The cached address belongs
//   to that device's context: after cudaDeviceReset (or any teardown of
//   the primary context) it is stale, so do not call this entry point in a
//   process that resets a device it has already used it on.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char rr_noalloc_scratch[RR_NOALLOC_SCRATCH_BYTES];

static void* noalloc_scratch_ptr(int dev, int* rc) {
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static void* ptrs[kMaxDev] = {nullptr};
  *rc = RR_OK;
  if (dev < 0 || dev >= kMaxDev) {
    *rc = RR_EINVAL;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!ptrs[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, rr_noalloc_scratch);
    if (e != cudaSuccess) {
      g_last_cuda_error = (int)e;
      *rc = RR_ECUDA;
      return nullptr;
    }
    ptrs[dev] = p;
  }
  return ptrs[dev];
}

extern "C" int rr_zchi2_batch_plain_noalloc(const double* band, const double* w,
                                            const double* wflux, const double* flux,
                                            const int64_t* pix_basis, int64_t npix_total,
                                            const double* basis, int64_t pix_stride, int32_t nz,
                                            int32_t nbasis, int32_t basis_stride,
                                            const double* prior, int32_t method, double* zchi2,
                                            double* zcoeff, int* status, rr_stream_t stream) {
  if (nz < 0 || npix_total < 1 || nbasis < 1 || nbasis > RR_MAX_NBASIS) return RR_EINVAL;
  if (nz == 0) return RR_OK;
  const size_t need = rr_zchi2_batch_plain_workspace_bytes(npix_total, nz, nbasis);
  if (need > (size_t)RR_NOALLOC_SCRATCH_BYTES) return RR_ESCRATCH;
  int dev = 0;
  RR_CUDA_TRY(cudaGetDevice(&dev));
  int rc = RR_OK;
  void* ws = noalloc_scratch_ptr(dev, &rc);
  if (rc) return rc;
  return rr_zchi2_batch_plain(band, w, wflux, flux, pix_basis, npix_total, basis, pix_stride, nz,
                              nbasis, basis_stride, prior, method, zchi2, zcoeff, ws,
                              (size_t)RR_NOALLOC_SCRATCH_BYTES, status, stream);
}

extern "C" int rr_negoii_penalty(const double* coeff, int64_t nz, int32_t nbasis, const double* oii,
                                 double* penalty, rr_stream_t stream) {
  if (nz < 0 || nbasis < 1) return RR_EINVAL;
  if (nz == 0) return RR_OK;
  if (!coeff || !oii || !penalty) return RR_EINVAL;
  negoii_kernel<<<(unsigned)((nz + 127) / 128), 128, 0, (cudaStream_t)stream>>>(coeff, nz, nbasis,
                                                                                oii, penalty);
  RR_CHECK_LAUNCH();
  return RR_OK;
}
