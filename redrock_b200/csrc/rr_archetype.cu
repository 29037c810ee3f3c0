// Batched archetype fits (redrock 0.22 archetypes.py:228-400 with the
// solves of zscan.py:245-348 / 626-781).
//
// redrock fits, for every refined redshift of every target, each archetype
// (or a combination of the nearest ones) together with Legendre nuisance
// columns: c = argmin || (M + P) c - y || under the bounds, with
//   M = Tb^T W Tb,  y = Tb^T W f,  Tb = R [a_1 .. a_m  L_1 .. L_nl]
// (a_t: an archetype rebinned to the target's grids at that redshift and
// multiplied by the IGM transmission; L_k: Legendre polynomials of the
// reduced wavelength, one set per camera or one for the spectrum), then
// chi2 = sum w (f - Tb c)^2.  One call here does all of that for many
// (target, redshift) pairs and many archetype selections ("jobs") at once.
//
// One warp per job: the lanes stride over the target's pixels and build
// each Tb column on the fly from the banded resolution rows (the same band
// rows as the plain chain: row p multiplies basis rows pix_basis[p] - 5 ..
// + 5), accumulating the lower triangle of M, y and f^T W f in registers;
// a shuffle tree reduces them into the caller's work array.  A second
// kernel, one thread per job, solves (PCA: LDL^T; NNLS / BVLS: the
// active-set solvers of rr_lsq_dev.cuh, bounds read in place from the
// kernel parameter) and writes chi2 = f^T W f - 2 c^T y + c^T M c (exact for
// any c, the prior excluded), or HUGE_CHI2 and zero coefficients when the
// solve fails, as redrock's calc_zchi2_batch does.
#include "rr_common.cuh"
#include "rr_lsq_dev.cuh"
#include "rr_solve_dev.cuh"

namespace rr {

struct ArchBounds {
  double lo[RR_MAX_NBASIS];
  double hi[RR_MAX_NBASIS];
};

struct ArchParams {
  const rr_arch_pair* pairs;
  int64_t npair;
  const double* band;
  const int64_t* pix_basis;
  const double* w;
  const double* wflux;
  const double* flux;
  const double* arch;
  const double* leg;
  int64_t pix_stride;
  int32_t narch;
  const int32_t* jobs;
  int32_t njob;
  int32_t m;
  int32_t nl;
  const double* prior;
  int32_t method;
  double* chi2;
  double* coeff;
};

constexpr int kArchWarps = 8;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int NB>
__global__ void __launch_bounds__(kArchWarps * 32)
    arch_gram_kernel(const __grid_constant__ ArchParams p, double* __restrict__ work) {
  constexpr int kTri = NB * (NB + 1) / 2;
  constexpr int kRec = kTri + NB + 2;  // M, y, f^T W f, index flag
  const int lane = threadIdx.x & 31;
  const int64_t job = (int64_t)blockIdx.x * kArchWarps + (threadIdx.x >> 5);
  if (job >= p.npair * p.njob) return;
  double* rec = work + job * kRec;
  const int64_t ip = job / p.njob;
  const rr_arch_pair pr = p.pairs[ip];
  // column sources: the job's archetypes, then the pair's Legendre set
  const int32_t* idx = p.jobs + job * p.m;
  bool in_range = true;
  for (int c = 0; c < p.m; ++c) in_range = in_range && idx[c] >= 0 && idx[c] < p.narch;
  if (!in_range) {  // the same for every lane of the warp
    if (lane == 0) rec[kRec - 1] = 1.0;
    return;
  }
  const double* col[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c)
    col[c] = c < p.m ? p.arch + pr.arch_off + (int64_t)idx[c] * p.pix_stride
                     : p.leg + pr.leg_off + (int64_t)(c - p.m) * p.pix_stride;
  double tri[kTri], yv[NB], ff = 0.0;
#pragma unroll
  for (int i = 0; i < kTri; ++i) tri[i] = 0.0;
#pragma unroll
  for (int i = 0; i < NB; ++i) yv[i] = 0.0;
  for (int64_t q = lane; q < pr.npix; q += 32) {
    const int64_t g = pr.pix_off + q;
    const double* r = p.band + g * kBand;
    const int64_t row = p.pix_basis[g] - kHalfBand;
    double v[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < kBand; ++k) acc = fma(r[k], col[c][row + k], acc);
      v[c] = acc;
    }
    const double wq = p.w[g], wf = p.wflux[g];
    ff = fma(wf, p.flux[g], ff);
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const double wv = wq * v[i];
      yv[i] = fma(v[i], wf, yv[i]);
#pragma unroll
      for (int j = 0; j <= i; ++j)
        tri[i * (i + 1) / 2 + j] = fma(wv, v[j], tri[i * (i + 1) / 2 + j]);
    }
  }
#pragma unroll
  for (int i = 0; i < kTri; ++i) tri[i] = warp_sum(tri[i]);
#pragma unroll
  for (int i = 0; i < NB; ++i) yv[i] = warp_sum(yv[i]);
  ff = warp_sum(ff);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < kTri; ++i) rec[i] = tri[i];
#pragma unroll
    for (int i = 0; i < NB; ++i) rec[kTri + i] = yv[i];
    rec[kTri + NB] = ff;
    rec[kRec - 1] = 0.0;
  }
}

// One thread per job: the solve of (M + prior) c ~ y and
// chi2 = f^T W f - 2 c^T y + c^T M c (M without the prior).
template <int NB>
__global__ void arch_solve_kernel(const __grid_constant__ ArchParams p,
                                  const __grid_constant__ ArchBounds bd,
                                  const double* __restrict__ work) {
  constexpr int kTri = NB * (NB + 1) / 2;
  constexpr int kRec = kTri + NB + 2;
  const int64_t job = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (job >= p.npair * p.njob) return;
  const double* rec = work + job * kRec;
  double c[NB];
  bool ok = rec[kRec - 1] == 0.0;
  if (ok) {
    double yv[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) yv[i] = rec[kTri + i];
    if (p.method == RR_SOLVE_PCA) {
      double mp[kTri];
#pragma unroll
      for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j)
          mp[i * (i + 1) / 2 + j] =
              rec[i * (i + 1) / 2 + j] + (p.prior ? p.prior[i * NB + j] : 0.0);
      ok = ldlt_solve<NB>(mp, yv, c);
    } else if (p.method == RR_SOLVE_NNLS || p.method == RR_SOLVE_BVLS) {
      double full[NB][NB];
      for (int i = 0; i < NB; ++i)
        for (int j = 0; j <= i; ++j) {
          const double v = rec[i * (i + 1) / 2 + j] + (p.prior ? p.prior[i * NB + j] : 0.0);
          full[i][j] = v;
          full[j][i] = v;
        }
      ok = p.method == RR_SOLVE_NNLS ? nnls_solve<NB>(full, yv, c)
                                     : bvls_solve<NB>(full, yv, bd.lo, bd.hi, c);
    } else {
      ok = false;
    }
    if (ok) {
      double cy = 0.0, cmc = 0.0;
      for (int i = 0; i < NB; ++i) {
        cy = fma(c[i], yv[i], cy);
        double s = 0.0;
        for (int j = 0; j < NB; ++j)
          s = fma(j <= i ? rec[i * (i + 1) / 2 + j] : rec[j * (j + 1) / 2 + i], c[j], s);
        cmc = fma(c[i], s, cmc);
      }
      p.chi2[job] = rec[kTri + NB] - 2.0 * cy + cmc;
    }
  }
  if (!ok) p.chi2[job] = RR_HUGE_CHI2;
  for (int i = 0; i < NB; ++i) p.coeff[job * NB + i] = ok ? c[i] : 0.0;
}

}  // namespace rr

using namespace rr;

extern "C" size_t rr_archetype_fit_work_bytes(int64_t npair, int32_t njob, int32_t nb) {
  if (npair < 0 || njob < 0 || nb < 1) return 0;
  return (size_t)npair * njob * (size_t)(nb * (nb + 1) / 2 + nb + 2) * sizeof(double);
}

extern "C" int rr_archetype_fit(const rr_arch_pair* pairs, int64_t npair, const double* band,
                                const int64_t* pix_basis, const double* w, const double* wflux,
                                const double* flux, const double* arch, int32_t narch,
                                const double* leg, int64_t pix_stride, const int32_t* jobs,
                                int32_t njob, int32_t m,
                                int32_t nl, const double* prior, int32_t method,
                                const double* bounds, double* chi2, double* coeff,
                                void* work, size_t work_bytes, rr_stream_t stream) {
  const int nb = m + nl;
  if (npair < 0 || njob < 0 || m < 1 || nl < 0 || nb > RR_MAX_NBASIS || pix_stride < 1 ||
      narch < 1)
    return RR_EINVAL;
  if (npair == 0 || njob == 0) return RR_OK;
  if (!pairs || !band || !pix_basis || !w || !wflux || !flux || !arch || !jobs || !chi2 ||
      !coeff || !work || (nl > 0 && !leg))
    return RR_EINVAL;
  if (work_bytes < rr_archetype_fit_work_bytes(npair, njob, nb)) return RR_EINVAL;
  if (method != RR_SOLVE_PCA && method != RR_SOLVE_NNLS && method != RR_SOLVE_BVLS &&
      method != RR_SOLVE_UNSUPPORTED)
    return RR_EINVAL;
  ArchParams p{pairs, npair, band, pix_basis, w, wflux, flux, arch, leg, pix_stride,
               narch, jobs, njob, m, nl, prior, method, chi2, coeff};
  ArchBounds bd;
  for (int i = 0; i < RR_MAX_NBASIS; ++i) {
    bd.lo[i] = -INFINITY;
    bd.hi[i] = INFINITY;
  }
  if (bounds)
    for (int i = 0; i < nb; ++i) {
      bd.lo[i] = bounds[i];
      bd.hi[i] = bounds[nb + i];
      if (!(bd.lo[i] <= bd.hi[i])) return RR_EINVAL;
    }
  const int64_t total = npair * (int64_t)njob;
  const int64_t blocks = (total + kArchWarps - 1) / kArchWarps;
  if (blocks > 2147483647LL) return RR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  double* wk = static_cast<double*>(work);
  const unsigned sblocks = (unsigned)((total + 127) / 128);
#define RR_ARCH_CASE(N)                                                               \
  case N:                                                                             \
    arch_gram_kernel<N><<<(unsigned)blocks, kArchWarps * 32, 0, st>>>(p, wk);         \
    RR_CHECK_LAUNCH();                                                                \
    arch_solve_kernel<N><<<sblocks, 128, 0, st>>>(p, bd, wk);                         \
    break;
  switch (nb) {
    RR_ARCH_CASE(1)
    RR_ARCH_CASE(2)
    RR_ARCH_CASE(3)
    RR_ARCH_CASE(4)
    RR_ARCH_CASE(5)
    RR_ARCH_CASE(6)
    RR_ARCH_CASE(7)
    RR_ARCH_CASE(8)
    RR_ARCH_CASE(9)
    RR_ARCH_CASE(10)
    default:
      return RR_EINVAL;
  }
#undef RR_ARCH_CASE
  RR_CHECK_LAUNCH();
  return RR_OK;
}
