// Pair scan: chi2, coefficients and [OII] penalty for an arbitrary list of
// (target, redshift) pairs, with the template rebinned on the fly.
//
// This is the batched form of redrock's fine-grid refinement (fitz.py:133-
// 395: for every coarse minimum, rebin_template + transmission_Lyman +
// calc_zchi2_batch on a 15-point grid, then a single-z fit at the parabola
// minimum).  Each target's fine redshifts are its own, so no basis is shared
// between targets: every CTA owns one pair, rebins the template for that
// redshift into shared memory chunk by chunk (the same bit-exact rebin and
// IGM code as the basis builder), and accumulates the banded R.T, the
// weighted Gram matrix and y in FP64 exactly as the fused scan does.
//
//   rows[t][p][12]: sqrt(w) R band rows and sqrt(w) f of target t, pixel p
//                   (rr_pack_rows; segment s starts at segs[s].rw_offset)
//
// Per chunk of 246 output pixels, thread i computes basis row c0 - 5 + i
// (256 rows = chunk + halo), then thread i < 246 forms Tb' for pixel c0 + i
// from shared rows i..i+10.  Template samples covering the chunk are staged
// in shared memory first, so the per-pixel search for the first sample
// beyond a bin edge runs on shared memory.
#include <cstring>

#include "rr_lsq_dev.cuh"
#include "rr_rebin_dev.cuh"
#include "rr_solve_dev.cuh"

namespace rr {

constexpr int kPairThreads = 256;
constexpr int kPairChunk = kPairThreads - 2 * kHalfBand;  // output pixels per chunk
constexpr int kPairMaxSeg = 16;
constexpr int kPairWin = 1536;  // template samples staged per chunk

struct PairsParams {
  rr_pair_template tm;
  rr_pair_segment segs[kPairMaxSeg];
  int nseg;
  const double* rows;
  const double* fwf;
  const double* wsum;
  int64_t npix_row;
  const int32_t* pair_target;
  const double* pair_z;
  int64_t npairs;
  double* chi2;
  double* coeff;
  double* penalty;
  // gradient mode (rr_zscan_pairs_grad)
  double* dchi2_dz;     // [npairs]
  double* d2chi2_dz2;   // [npairs]
  double* dchi2_dflux;  // [npairs][npix_row] or NULL
  double* dpen_dz;      // [npairs] d penalty / dz or NULL
  const double* sw;     // [ntarget][npix_row] sqrt(w), needed for dchi2_dflux
  int* status;
  // RR_SOLVE_BVLS bounds (+-inf when the caller gives none); read in place
  // by the solver, like the plain chain's
  double lo[RR_MAX_NBASIS];
  double hi[RR_MAX_NBASIS];
};

// odd row stride (doubles) of the shared basis rows: conflict-free 64-bit
// reads by consecutive threads
template <int NB>
constexpr int pair_stride() { return (NB & 1) ? NB : NB + 1; }

template <int NB>
struct PairSmem {
  double t[kPairThreads * pair_stride<NB>()];  // basis rows of the chunk + halo
  double dt[kPairThreads * pair_stride<NB>()]; // their z derivatives (gradient mode)
  double xs[kPairWin];                          // staged template wavelengths
  double ys[NB * kPairWin];                     // staged template fluxes
  double red[kPairThreads / 32][NB * (NB + 1) / 2 + NB];
  double c[NB];
  int64_t jlo, jhi, win;
  int fix;
  int bad;
};

// Fill the shared basis rows for output pixels [c0 - 5, c0 + kPairChunk + 5)
// of segment sg at redshift z.  Returns false if a bin fell outside the
// template (never for pairs that pass the host-side range check).
template <int NB, bool DZ>
__device__ bool fill_rows(const PairsParams& p, const rr_pair_segment& sg, int64_t c0, double z,
                          double zp1, bool igm, PairSmem<NB>& sm) {
  constexpr int S = pair_stride<NB>();
  const rr_pair_template& tm = p.tm;
  const int64_t first = c0 - kHalfBand;
  const int64_t last = min(c0 + kPairChunk + kHalfBand, sg.npix);  // exclusive
  // samples needed: from the one before the first edge to the one after
  // the last edge; the two searches (guess from the near-uniform sample
  // spacing, then a short walk: a few dependent loads instead of a binary
  // search's ~16) run in two warps at once
  if (threadIdx.x == 0) {
    const int64_t e0 = max(first, (int64_t)0);
    sm.jlo = max(first_above(tm.x, tm.nx, zp1, sg.edges[e0]) - 2, (int64_t)0);
  } else if (threadIdx.x == 32) {
    sm.jhi = min(first_above(tm.x, tm.nx, zp1, sg.edges[last]) + 2, tm.nx);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int64_t span = sm.jhi - sm.jlo;
    sm.win = (span > 0 && span <= kPairWin) ? span : 0;  // 0: use global arrays
  }
  __syncthreads();
  const int64_t jlo = sm.jlo, win = sm.win;
  for (int64_t i = threadIdx.x; i < win; i += kPairThreads) {
    sm.xs[i] = tm.x[jlo + i];
#pragma unroll
    for (int b = 0; b < NB; ++b) sm.ys[b * kPairWin + i] = tm.y[(int64_t)b * tm.nx + jlo + i];
  }
  __syncthreads();
  bool ok = true;
  const int64_t ip = first + threadIdx.x;
  double* row = sm.t + threadIdx.x * S;
  double* drow = sm.dt + threadIdx.x * S;
  if (ip < 0 || ip >= sg.npix) {
#pragma unroll
    for (int b = 0; b < NB; ++b) row[b] = 0.0;
    if (DZ)
#pragma unroll
      for (int b = 0; b < NB; ++b) drow[b] = 0.0;
  } else {
    double res[kMaxRebinBasis], dres[DZ ? kMaxRebinBasis : 1];
    bool got = false;
    if (win > 0) {
      // rebin on the staged window: the bin must have a sample before and
      // after it inside the window, else fall back to the global arrays
      got = rebin_bin_strided<DZ>(sm.xs, win, sm.ys, kPairWin, NB, zp1, sg.edges[ip],
                                  sg.edges[ip + 1], res, dres);
    }
    if (!got)
      got = rebin_bin_strided<DZ>(tm.x, tm.nx, tm.y, tm.nx, NB, zp1, sg.edges[ip],
                                  sg.edges[ip + 1], res, dres);
    if (!got) {
      ok = false;
#pragma unroll
      for (int b = 0; b < NB; ++b) res[b] = 0.0;
      if (DZ)
#pragma unroll
        for (int b = 0; b < NB; ++b) dres[b] = 0.0;
    }
    if (igm) {
      double dtr = 0.0;
      const double tr = DZ ? transmission_dz(tm.igm_model, z, sg.wave[ip], &dtr)
                           : transmission(tm.igm_model, z, sg.wave[ip]);
      if (DZ)
#pragma unroll
        for (int b = 0; b < NB; ++b) dres[b] = dres[b] * tr + res[b] * dtr;
#pragma unroll
      for (int b = 0; b < NB; ++b) res[b] = dmul(res[b], tr);
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) row[b] = res[b];
    if (DZ)
#pragma unroll
      for (int b = 0; b < NB; ++b) drow[b] = dres[b];
  }
  __syncthreads();
  return ok;
}

// Sweep modes over every pixel of the pair's target:
//   kGram:  Gram matrix m and y (forward);
//   kResid: residual sum (g - Tb'.c)^2 into acc[0];
//   kGrad:  residual sum, gradient and curvature accumulators with
//           dTb' = R' dT/dz:  acc[0] = sum res^2, acc[1] = sum res (dTb'.c),
//           acc[2] = sum (dTb'.c)^2, acc[3..3+NB) = u = dTb'^T res,
//           acc[3+NB..3+2NB) = v = Tb'^T (dTb'.c); and dchi2/dflux.
enum SweepMode { kGram = 0, kResid = 1, kGrad = 2 };

template <int NB, int MODE>
__device__ bool pair_sweep(const PairsParams& p, int64_t pr, int64_t t, double z,
                           double (&m)[NB * (NB + 1) / 2], double (&y)[NB], const double* c,
                           double* acc, PairSmem<NB>& sm) {
  constexpr int S = pair_stride<NB>();
  constexpr bool DZ = MODE == kGrad;
  const double zp1 = dadd(1.0, z);
  bool ok = true;
  for (int s = 0; s < p.nseg; ++s) {
    const rr_pair_segment& sg = p.segs[s];
    // redrock skips the IGM product when no redshift puts the grid's bluest
    // pixel below Lyman-alpha (igm.py:396-401); the transmission is exactly
    // 1 there anyway
    const bool igm = p.tm.igm_model != RR_IGM_NONE && !(ddiv(sg.wave_min, zp1) > kLyA);
    for (int64_t c0 = 0; c0 < sg.npix; c0 += kPairChunk) {
      ok = fill_rows<NB, DZ>(p, sg, c0, z, zp1, igm, sm) && ok;
      const int64_t ip = c0 + threadIdx.x;
      if (threadIdx.x < kPairChunk && ip < sg.npix) {
        const int64_t prow = (t * p.npix_row) + sg.row_offset + ip;
        const double* rr = p.rows + prow * RR_RW;
        double r[kBand];
#pragma unroll
        for (int k = 0; k < kBand; ++k) r[k] = rr[k];
        const double g = rr[kBand];
        double tb[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) tb[b] = 0.0;
#pragma unroll
        for (int k = 0; k < kBand; ++k) {
          const double* trow = sm.t + (threadIdx.x + k) * S;
#pragma unroll
          for (int b = 0; b < NB; ++b) tb[b] = fma(r[k], trow[b], tb[b]);
        }
        if (MODE == kGram) {
#pragma unroll
          for (int b = 0; b < NB; ++b) y[b] = fma(g, tb[b], y[b]);
#pragma unroll
          for (int a = 0; a < NB; ++a)
#pragma unroll
            for (int b = 0; b <= a; ++b)
              m[a * (a + 1) / 2 + b] = fma(tb[a], tb[b], m[a * (a + 1) / 2 + b]);
        } else {
          double model = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b) model = fma(tb[b], c[b], model);
          const double res = g - model;
          acc[0] = fma(res, res, acc[0]);
          if (MODE == kGrad) {
            double db[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) db[b] = 0.0;
#pragma unroll
            for (int k = 0; k < kBand; ++k) {
              const double* drow = sm.dt + (threadIdx.x + k) * S;
#pragma unroll
              for (int b = 0; b < NB; ++b) db[b] = fma(r[k], drow[b], db[b]);
            }
            double dm = 0.0;
#pragma unroll
            for (int b = 0; b < NB; ++b) dm = fma(db[b], c[b], dm);
            acc[1] = fma(res, dm, acc[1]);
            acc[2] = fma(dm, dm, acc[2]);
#pragma unroll
            for (int b = 0; b < NB; ++b) {
              acc[3 + b] = fma(db[b], res, acc[3 + b]);
              acc[3 + NB + b] = fma(tb[b], dm, acc[3 + NB + b]);
            }
            // d chi2 / d f_p = 2 w_p r_p = 2 sqrt(w_p) * (sqrt(w_p) r_p)
            if (p.dchi2_dflux)
              p.dchi2_dflux[pr * p.npix_row + sg.row_offset + ip] =
                  2.0 * p.sw[prow] * res;
          }
        }
      }
      __syncthreads();  // rows of this chunk fully consumed
    }
  }
  return ok;
}

// Deterministic block sum of v[0..n) (fixed shuffle tree, then warps in order).
template <int NB>
__device__ void block_sum(double* v, int n, PairSmem<NB>& sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int e = 0; e < n; ++e) {
    double x = v[e];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    if (lane == 0) sm.red[warp][e] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int e = 0; e < n; ++e) {
      double x = sm.red[0][e];
      for (int w = 1; w < kPairThreads / 32; ++w) x += sm.red[w][e];
      v[e] = x;
    }
  }
  __syncthreads();
}

// the plain chain's bounded solves (plain_lsq_kernel) on one pair's
// packed M and y: the full symmetric M + prior, then NNLS or BVLS
template <int NB>
__device__ __noinline__ bool bounded_solve(const PairsParams& p, const double (&mm)[NB * (NB + 1) / 2],
                                           const double (&yy)[NB], double (&c)[NB]) {
  double full[NB][NB], b[NB];
  for (int i = 0; i < NB; ++i) {
    b[i] = yy[i];
    for (int j = 0; j <= i; ++j) {
      double v = mm[i * (i + 1) / 2 + j];
      if (p.tm.prior) v += p.tm.prior[i * NB + j];
      full[i][j] = full[j][i] = v;
    }
  }
  bool ok;
  if (p.tm.method == RR_SOLVE_NNLS)
    ok = nnls_solve<NB>(full, b, c);
  else if (p.tm.method == RR_SOLVE_BVLS)
    ok = bvls_solve<NB>(full, b, p.lo, p.hi, c);
  else
    ok = false;
  if (!ok)
    for (int i = 0; i < NB; ++i) c[i] = 0.0;
  return ok;
}

template <int NB, bool GRAD>
__global__ void __launch_bounds__(kPairThreads, (NB <= 5 ? 2 : 1)) zscan_pairs_kernel(const __grid_constant__ PairsParams p) {
  extern __shared__ __align__(16) unsigned char pair_smem_raw[];
  PairSmem<NB>& sm = *reinterpret_cast<PairSmem<NB>*>(pair_smem_raw);
  constexpr int kTri = NB * (NB + 1) / 2;
  constexpr int kAcc = 3 + 2 * NB;
  for (int64_t pr = blockIdx.x; pr < p.npairs; pr += gridDim.x) {
    const int64_t t = p.pair_target[pr];
    const double z = p.pair_z[pr];
    double m[kTri + NB];
    double(&mm)[kTri] = *reinterpret_cast<double(*)[kTri]>(m);
    double(&yy)[NB] = *reinterpret_cast<double(*)[NB]>(m + kTri);
#pragma unroll
    for (int i = 0; i < kTri + NB; ++i) m[i] = 0.0;
    double acc[kAcc];
#pragma unroll
    for (int i = 0; i < kAcc; ++i) acc[i] = 0.0;
    bool ok = pair_sweep<NB, kGram>(p, pr, t, z, mm, yy, nullptr, acc, sm);
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) {
        set_status(p.status, RR_ERANGE);
        p.chi2[pr] = nan("");
        for (int b = 0; b < NB; ++b) p.coeff[pr * NB + b] = nan("");
        if (p.penalty) p.penalty[pr] = nan("");
        if (GRAD) {
          p.dchi2_dz[pr] = nan("");
          p.d2chi2_dz2[pr] = nan("");
          if (p.dpen_dz) p.dpen_dz[pr] = nan("");
        }
      }
      continue;
    }
    block_sum<NB>(m, kTri + NB, sm);
    bool solved = false;
    if (threadIdx.x == 0) {
      double c[NB], chi2 = 0.0, err = 0.0;
      if (GRAD || p.tm.method == RR_SOLVE_PCA) {
        solved = solve_eval<NB>(p.tm.method, p.tm.prior, mm, yy, p.fwf[t], p.wsum[t], c, chi2,
                                err);
        sm.fix = (solved && err > kChi2FixTol) ? 1 : 0;
      } else {
        // NMF / NNLS / BVLS (calc_zchi2_batch's bounded branches): the
        // solver on M + prior and y, then chi2 always as the direct
        // residual (a constrained c is no stationary point of
        // f^T W f - c^T y); a failed solve gives HUGE_CHI2, zero c
        solved = bounded_solve<NB>(p, mm, yy, c);
        chi2 = kHugeChi2;
        sm.fix = solved ? 1 : 0;
      }
      sm.bad = solved ? 0 : 1;
      for (int b = 0; b < NB; ++b) sm.c[b] = c[b];
      p.chi2[pr] = chi2;
      for (int b = 0; b < NB; ++b) p.coeff[pr * NB + b] = c[b];
      if (p.penalty) {
        double s = 0.0;
        if (p.tm.oii)
          for (int b = 0; b < NB; ++b) s = fma(c[b], p.tm.oii[b], s);
        p.penalty[pr] = (p.wsum[t] != 0.0 && s < 0.0) ? -s : 0.0;
      }
    }
    __syncthreads();
    if (GRAD) {
      if (sm.bad) {
        if (threadIdx.x == 0) {
          p.dchi2_dz[pr] = 0.0;
          p.d2chi2_dz2[pr] = 0.0;
          if (p.dpen_dz) p.dpen_dz[pr] = 0.0;
        }
        __syncthreads();
        continue;
      }
      // residual chi2 (exact), gradient and curvature in one more sweep
      pair_sweep<NB, kGrad>(p, pr, t, z, mm, yy, sm.c, acc, sm);
      block_sum<NB>(acc, kAcc, sm);
      if (threadIdx.x == 0) {
        // envelope curvature: 2 sum (dTb'.c)^2 - 2 (u - v)^T (M + P)^-1 (u - v)
        double mp[kTri], uv[NB], x[NB];
#pragma unroll
        for (int i = 0; i < kTri; ++i) mp[i] = mm[i];
        if (p.tm.prior)
#pragma unroll
          for (int i = 0; i < NB; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j) mp[i * (i + 1) / 2 + j] += p.tm.prior[i * NB + j];
#pragma unroll
        for (int b = 0; b < NB; ++b) uv[b] = acc[3 + b] - acc[3 + NB + b];
        double q = 0.0;
        const bool xok = ldlt_solve<NB>(mp, uv, x);
        if (xok)
#pragma unroll
          for (int b = 0; b < NB; ++b) q = fma(uv[b], x[b], q);
        p.chi2[pr] = acc[0];
        p.dchi2_dz[pr] = -2.0 * acc[1];
        p.d2chi2_dz2[pr] = 2.0 * acc[2] - 2.0 * q;
        if (p.dpen_dz) {
          // x = dc/dz = (M + P)^-1 (u - v); the penalty -c.oii (when the
          // [OII] model is negative) changes by -x.oii
          double s = 0.0, ds = 0.0;
          if (p.tm.oii)
            for (int b = 0; b < NB; ++b) {
              s = fma(sm.c[b], p.tm.oii[b], s);
              ds = fma(xok ? x[b] : 0.0, p.tm.oii[b], ds);
            }
          p.dpen_dz[pr] = (p.wsum[t] != 0.0 && s < 0.0) ? -ds : 0.0;
        }
      }
      __syncthreads();
      continue;
    }
    if (sm.fix) {
      // ill-conditioned: chi2 as the direct residual sum w (f - Tb c)^2
      acc[0] = 0.0;
      pair_sweep<NB, kResid>(p, pr, t, z, mm, yy, sm.c, acc, sm);
      block_sum<NB>(acc, 1, sm);
      if (threadIdx.x == 0) p.chi2[pr] = acc[0];
    }
    __syncthreads();
  }
}

// rows[t][p][12] for the pair scan; t = block * 32 + lane of the
// spectrum descriptor, row offset of segment s = segs[s].rw_offset.
__global__ void pack_rows_kernel(const rr_spectrum_desc* __restrict__ specs, int64_t nspec,
                                 const double* __restrict__ rdata, const int32_t* __restrict__ roff,
                                 const double* __restrict__ ivar, const double* __restrict__ flux,
                                 const rr_segment_desc* __restrict__ segs, int64_t npix_row,
                                 double* __restrict__ rows, double* __restrict__ sw_out,
                                 int* status) {
  const int64_t s = blockIdx.y;
  if (s >= nspec) return;
  const rr_spectrum_desc sd = specs[s];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= sd.npix) return;
  const rr_segment_desc seg = segs[sd.segment];
  if (seg.rw_offset + i >= npix_row) { set_status(status, RR_EINVAL); return; }
  double r[kBand];
#pragma unroll
  for (int k = 0; k < kBand; ++k) r[k] = 0.0;
  for (int d = 0; d < sd.ndiag; ++d) {
    const int off = roff[sd.diag_offset + d];
    const int64_t j = i + off;
    if (j < 0 || j >= sd.npix) continue;
    const double v = rdata[sd.data_offset + (int64_t)d * sd.npix + j];
    if (off < -kHalfBand || off > kHalfBand) {
      if (v != 0.0) set_status(status, RR_ENOTSUP);
      continue;
    }
    r[off + kHalfBand] += v;
  }
  const double sw = sqrt(ivar[sd.pix_offset + i]);
  const int64_t t = (int64_t)sd.block * RR_LANES + sd.lane;
  double* o = rows + ((t * npix_row) + seg.rw_offset + i) * RR_RW;
#pragma unroll
  for (int k = 0; k < kBand; ++k) o[k] = sw * r[k];
  o[kBand] = sw * flux[sd.pix_offset + i];
  if (sw_out) sw_out[(t * npix_row) + seg.rw_offset + i] = sw;
}

// f^T W f and sum w per target (spectra grouped by target, fixed order)
__global__ void pack_row_sums_kernel(const rr_spectrum_desc* __restrict__ specs,
                                     const int64_t* __restrict__ first, int64_t ntarget,
                                     const double* __restrict__ ivar,
                                     const double* __restrict__ flux, double* __restrict__ fwf,
                                     double* __restrict__ wsum) {
  const int64_t t = blockIdx.x;
  if (t >= ntarget) return;
  __shared__ double red[2][256];
  double ta = 0.0, tb = 0.0;
  for (int64_t s = first[t]; s < first[t + 1]; ++s) {
    const rr_spectrum_desc sd = specs[s];
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
    ta += red[0][0];
    tb += red[1][0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    fwf[t] = ta;
    wsum[t] = tb;
  }
}

template <int NB, bool GRAD>
static int launch_pairs(const PairsParams& p, cudaStream_t st) {
  const size_t smem = sizeof(PairSmem<NB>);
  if (cudaFuncSetAttribute(zscan_pairs_kernel<NB, GRAD>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return RR_ECUDA;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RR_ECUDA;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return RR_ECUDA;
  const int64_t grid = p.npairs < (int64_t)nsm * 4 ? p.npairs : (int64_t)nsm * 4;
  zscan_pairs_kernel<NB, GRAD><<<(unsigned)grid, kPairThreads, smem, st>>>(p);
  if (cudaGetLastError() != cudaSuccess) return RR_ECUDA;
  return RR_OK;
}

}  // namespace rr

using namespace rr;

extern "C" int rr_pack_rows(const rr_spectrum_desc* specs, int64_t nspec,
                            const int64_t* target_first, int64_t ntarget, const double* rdata,
                            const int32_t* roffsets, const double* ivar, const double* flux,
                            const rr_segment_desc* segs, int nseg, int64_t npix_row, double* rows,
                            double* sw, double* fwf, double* wsum, int* status,
                            rr_stream_t stream) {
  if (nspec < 0 || ntarget < 0 || nseg < 1 || npix_row < 1) return RR_EINVAL;
  if (nspec == 0 || ntarget == 0) return RR_OK;
  if (!specs || !target_first || !rdata || !roffsets || !ivar || !flux || !segs || !rows || !fwf ||
      !wsum)
    return RR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  for (int64_t s0 = 0; s0 < nspec; s0 += 65535) {
    const int64_t n = nspec - s0 < 65535 ? nspec - s0 : 65535;
    dim3 block(128);
    dim3 grid((unsigned)((npix_row + block.x - 1) / block.x), (unsigned)n);
    pack_rows_kernel<<<grid, block, 0, st>>>(specs + s0, n, rdata, roffsets, ivar, flux, segs,
                                             npix_row, rows, sw, status);
    if (cudaGetLastError() != cudaSuccess) return RR_ECUDA;
  }
  pack_row_sums_kernel<<<(unsigned)ntarget, 256, 0, st>>>(specs, target_first, ntarget, ivar, flux,
                                                          fwf, wsum);
  if (cudaGetLastError() != cudaSuccess) return RR_ECUDA;
  return RR_OK;
}

static int pairs_params(PairsParams& p, const rr_pair_template* tmpl, const rr_pair_segment* segs,
                        int nseg, const double* rows, const double* fwf, const double* wsum,
                        int64_t npix_row, const int32_t* pair_target, const double* pair_z,
                        int64_t npairs, double* chi2, double* coeff, double* penalty,
                        int* status) {
  if (!tmpl || !segs || nseg < 1 || nseg > kPairMaxSeg || npix_row < 1 || npairs < 0)
    return RR_EINVAL;
  if (npairs > 0 && (!rows || !fwf || !wsum || !pair_target || !pair_z || !chi2 || !coeff))
    return RR_EINVAL;
  if (!tmpl->x || !tmpl->y || tmpl->nx < 2 || tmpl->nbasis < 1 || tmpl->nbasis > RR_MAX_NBASIS)
    return RR_EINVAL;
  if (tmpl->igm_model < RR_IGM_NONE || tmpl->igm_model > RR_IGM_INOUE14) return RR_EINVAL;
  if (tmpl->oii && !penalty) return RR_EINVAL;
  if (tmpl->method < RR_SOLVE_PCA || tmpl->method > RR_SOLVE_BVLS) return RR_EINVAL;
  memset(&p, 0, sizeof(p));
  p.tm = *tmpl;
  for (int i = 0; i < RR_MAX_NBASIS; ++i) {
    p.lo[i] = -INFINITY;
    p.hi[i] = INFINITY;
  }
  if (tmpl->bounds)
    for (int i = 0; i < tmpl->nbasis; ++i) {
      p.lo[i] = tmpl->bounds[i];
      p.hi[i] = tmpl->bounds[tmpl->nbasis + i];
      if (!(p.lo[i] <= p.hi[i])) return RR_EINVAL;
    }
  p.tm.bounds = nullptr;  // host memory: not for the device
  p.nseg = nseg;
  for (int s = 0; s < nseg; ++s) {
    if (segs[s].npix < 1 || !segs[s].edges || !segs[s].wave || segs[s].row_offset < 0 ||
        segs[s].row_offset + segs[s].npix > npix_row)
      return RR_EINVAL;
    p.segs[s] = segs[s];
  }
  p.rows = rows;
  p.fwf = fwf;
  p.wsum = wsum;
  p.npix_row = npix_row;
  p.pair_target = pair_target;
  p.pair_z = pair_z;
  p.npairs = npairs;
  p.chi2 = chi2;
  p.coeff = coeff;
  p.penalty = penalty;
  p.status = status;
  return RR_OK;
}

template <bool GRAD>
static int dispatch_pairs(const PairsParams& p, int nbasis, cudaStream_t st) {
  int rc = upload_igm_tables(st);
  if (rc) return rc;
  switch (nbasis) {
    case 1: return launch_pairs<1, GRAD>(p, st);
    case 2: return launch_pairs<2, GRAD>(p, st);
    case 3: return launch_pairs<3, GRAD>(p, st);
    case 4: return launch_pairs<4, GRAD>(p, st);
    case 5: return launch_pairs<5, GRAD>(p, st);
    case 6: return launch_pairs<6, GRAD>(p, st);
    case 7: return launch_pairs<7, GRAD>(p, st);
    case 8: return launch_pairs<8, GRAD>(p, st);
    case 9: return launch_pairs<9, GRAD>(p, st);
    case 10: return launch_pairs<10, GRAD>(p, st);
    default: return RR_EINVAL;
  }
}

extern "C" int rr_zscan_pairs(const rr_pair_template* tmpl, const rr_pair_segment* segs, int nseg,
                              const double* rows, const double* fwf, const double* wsum,
                              int64_t npix_row, const int32_t* pair_target, const double* pair_z,
                              int64_t npairs, double* chi2, double* coeff, double* penalty,
                              int* status, rr_stream_t stream) {
  PairsParams p;
  int rc = pairs_params(p, tmpl, segs, nseg, rows, fwf, wsum, npix_row, pair_target, pair_z,
                        npairs, chi2, coeff, penalty, status);
  if (rc || npairs == 0) return rc;
  return dispatch_pairs<false>(p, tmpl->nbasis, (cudaStream_t)stream);
}

extern "C" int rr_zscan_pairs_grad(const rr_pair_template* tmpl, const rr_pair_segment* segs,
                                   int nseg, const double* rows, const double* sw,
                                   const double* fwf, const double* wsum, int64_t npix_row,
                                   const int32_t* pair_target, const double* pair_z,
                                   int64_t npairs, double* chi2, double* coeff, double* penalty,
                                   double* dchi2_dz, double* d2chi2_dz2, double* dchi2_dflux,
                                   double* dpenalty_dz, int* status, rr_stream_t stream) {
  PairsParams p;
  int rc = pairs_params(p, tmpl, segs, nseg, rows, fwf, wsum, npix_row, pair_target, pair_z,
                        npairs, chi2, coeff, penalty, status);
  if (rc || npairs == 0) return rc;
  if (!dchi2_dz || !d2chi2_dz2 || (dchi2_dflux && !sw)) return RR_EINVAL;
  if (tmpl->method != RR_SOLVE_PCA) return RR_ENOTSUP;
  if (tmpl->prior && dchi2_dflux) return RR_ENOTSUP;
  p.dchi2_dz = dchi2_dz;
  p.d2chi2_dz2 = d2chi2_dz2;
  p.dchi2_dflux = dchi2_dflux;
  p.dpen_dz = dpenalty_dz;
  p.sw = sw;
  return dispatch_pairs<true>(p, tmpl->nbasis, (cudaStream_t)stream);
}
