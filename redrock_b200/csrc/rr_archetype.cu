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
// Three launches.  (1) One block per pair builds R L for the pair's
// Legendre columns once (the same for every archetype of the pair) and the
// pair's constants L^T W L, L^T W f and f^T W f.  (2) One warp per job: the
// lanes stride over the target's pixels, build only the job's archetype
// columns R a from the banded resolution rows (row p multiplies basis rows
// pix_basis[p] - 5 .. + 5, as in the plain chain), read R L, and accumulate
// the rows of M and y that involve an archetype; a shuffle tree reduces
// them and lane 0 writes the job's full M, y and f^T W f.  (3) One thread
// per job solves (PCA: LDL^T; NNLS / BVLS: the active-set solvers of
// rr_lsq_dev.cuh, bounds read in place from the kernel parameter) and writes
// chi2 = f^T W f - 2 c^T y + c^T M c (exact for any c, the prior excluded),
// or HUGE_CHI2 and zero coefficients when the solve fails, as redrock's
// calc_zchi2_batch does.
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
  int64_t max_npix;
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

// work layout (doubles): R L of every pair (nl x max_npix each), then each
// pair's constants (L^T W L lower triangle, L^T W f, f^T W f), then one
// record per job (M lower triangle, y, f^T W f, a flag set when the job's
// archetype indices are out of range).
__host__ __device__ constexpr int64_t arch_pair_consts(int nl) { return nl * (nl + 1) / 2 + nl + 1; }
__host__ __device__ constexpr int64_t arch_job_rec(int nb) { return nb * (nb + 1) / 2 + nb + 2; }

template <int NL>
__global__ void __launch_bounds__(256) arch_pair_kernel(const __grid_constant__ ArchParams p,
                                                        double* __restrict__ work) {
  constexpr int kLT = NL * (NL + 1) / 2;
  constexpr int kC = kLT + NL + 1;
  __shared__ double red[8][kC];
  const int64_t ip = blockIdx.x;
  const rr_arch_pair pr = p.pairs[ip];
  double* rl = work + ip * NL * p.max_npix;
  double* cst = work + p.npair * NL * p.max_npix + ip * kC;
  double acc[kC];
#pragma unroll
  for (int i = 0; i < kC; ++i) acc[i] = 0.0;
  for (int64_t q = threadIdx.x; q < pr.npix; q += blockDim.x) {
    const int64_t g = pr.pix_off + q;
    const double* r = p.band + g * kBand;
    const int64_t row = p.pix_basis[g] - kHalfBand;
    double v[NL > 0 ? NL : 1];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      const double* col = p.leg + pr.leg_off + (int64_t)k * p.pix_stride + row;
      double s = 0.0;
#pragma unroll
      for (int d = 0; d < kBand; ++d) s = fma(r[d], col[d], s);
      v[k] = s;
      rl[(int64_t)k * p.max_npix + q] = s;
    }
    const double wq = p.w[g], wf = p.wflux[g];
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const double wv = wq * v[i];
#pragma unroll
      for (int j = 0; j <= i; ++j) acc[i * (i + 1) / 2 + j] = fma(wv, v[j], acc[i * (i + 1) / 2 + j]);
      acc[kLT + i] = fma(v[i], wf, acc[kLT + i]);
    }
    acc[kC - 1] = fma(wf, p.flux[g], acc[kC - 1]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < kC; ++i) {
    const double v = warp_sum(acc[i]);
    if (lane == 0) red[warp][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < kC) {
    double s = 0.0;
    for (int w8 = 0; w8 < (int)(blockDim.x >> 5); ++w8) s += red[w8][threadIdx.x];
    cst[threadIdx.x] = s;
  }
}

// M = 1 for the fits of single archetypes (the rows of M involving the
// archetype are its column); M = 0: p.m archetypes (the nearest ones).
template <int NB, int M>
__global__ void __launch_bounds__(kArchWarps * 32)
    arch_gram_kernel(const __grid_constant__ ArchParams p, double* __restrict__ work) {
  constexpr int kTri = NB * (NB + 1) / 2;
  constexpr int kRec = arch_job_rec(NB);
  const int lane = threadIdx.x & 31;
  const int64_t job = (int64_t)blockIdx.x * kArchWarps + (threadIdx.x >> 5);
  if (job >= p.npair * p.njob) return;
  const int m = M ? M : p.m;
  const int nl = NB - m;
  const int64_t ip = job / p.njob;
  const rr_arch_pair pr = p.pairs[ip];
  const double* rl = work + ip * nl * p.max_npix;
  const double* cst = work + p.npair * nl * p.max_npix + ip * arch_pair_consts(nl);
  double* rec = work + p.npair * (nl * p.max_npix + arch_pair_consts(nl)) + job * kRec;
  const int32_t* idx = p.jobs + job * m;
  bool in_range = true;
  for (int c = 0; c < m; ++c) in_range = in_range && idx[c] >= 0 && idx[c] < p.narch;
  if (!in_range) {  // the same for every lane of the warp
    if (lane == 0) rec[kRec - 1] = 1.0;
    return;
  }
  const double* col[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c)
    col[c] = c < m ? p.arch + pr.arch_off + (int64_t)idx[c] * p.pix_stride : nullptr;
  double tri[kTri], yv[NB];
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
      if (c < m) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < kBand; ++k) acc = fma(r[k], col[c][row + k], acc);
        v[c] = acc;
      } else {
        v[c] = rl[(int64_t)(c - m) * p.max_npix + q];
      }
    }
    const double wq = p.w[g], wf = p.wflux[g];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      if (j < m) {
        const double wv = wq * v[j];
        yv[j] = fma(v[j], wf, yv[j]);
#pragma unroll
        for (int i = j; i < NB; ++i) tri[i * (i + 1) / 2 + j] = fma(wv, v[i], tri[i * (i + 1) / 2 + j]);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (j < m) {
#pragma unroll
      for (int i = j; i < NB; ++i) tri[i * (i + 1) / 2 + j] = warp_sum(tri[i * (i + 1) / 2 + j]);
      yv[j] = warp_sum(yv[j]);
    }
  }
  if (lane != 0) return;
  // the Legendre block and its y entries from the pair's constants
  for (int i = m; i < NB; ++i) {
    for (int j = m; j <= i; ++j) {
      const int a = i - m, b = j - m;
      tri[i * (i + 1) / 2 + j] = cst[a * (a + 1) / 2 + b];
    }
    yv[i] = cst[nl * (nl + 1) / 2 + (i - m)];
  }
#pragma unroll
  for (int i = 0; i < kTri; ++i) rec[i] = tri[i];
#pragma unroll
  for (int i = 0; i < NB; ++i) rec[kTri + i] = yv[i];
  rec[kTri + NB] = cst[arch_pair_consts(nl) - 1];
  rec[kRec - 1] = 0.0;
}

// One thread per job: the solve of (M + prior) c ~ y and
// chi2 = f^T W f - 2 c^T y + c^T M c (M without the prior).
template <int NB>
__global__ void arch_solve_kernel(const __grid_constant__ ArchParams p,
                                  const __grid_constant__ ArchBounds bd,
                                  const double* __restrict__ work) {
  constexpr int kTri = NB * (NB + 1) / 2;
  constexpr int kRec = arch_job_rec(NB);
  const int64_t job = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (job >= p.npair * p.njob) return;
  const int nl = NB - p.m;
  const double* rec = work + p.npair * (nl * p.max_npix + arch_pair_consts(nl)) + job * kRec;
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

extern "C" size_t rr_archetype_fit_work_bytes(int64_t npair, int32_t njob, int32_t m, int32_t nl,
                                              int64_t max_npix) {
  if (npair < 0 || njob < 0 || m < 1 || nl < 0 || max_npix < 0) return 0;
  return ((size_t)npair * (size_t)(nl * max_npix + arch_pair_consts(nl)) +
          (size_t)npair * njob * (size_t)arch_job_rec(m + nl)) * sizeof(double);
}

extern "C" int rr_archetype_fit(const rr_arch_pair* pairs, int64_t npair, const double* band,
                                const int64_t* pix_basis, const double* w, const double* wflux,
                                const double* flux, int64_t max_npix, const double* arch,
                                int32_t narch, const double* leg, int64_t pix_stride,
                                const int32_t* jobs,
                                int32_t njob, int32_t m,
                                int32_t nl, const double* prior, int32_t method,
                                const double* bounds, double* chi2, double* coeff,
                                void* work, size_t work_bytes, rr_stream_t stream) {
  const int nb = m + nl;
  if (npair < 0 || njob < 0 || m < 1 || nl < 0 || nb > RR_MAX_NBASIS || pix_stride < 1 ||
      narch < 1 || max_npix < 0)
    return RR_EINVAL;
  if (npair == 0 || njob == 0) return RR_OK;
  if (!pairs || !band || !pix_basis || !w || !wflux || !flux || !arch || !jobs || !chi2 ||
      !coeff || !work || (nl > 0 && !leg))
    return RR_EINVAL;
  if (work_bytes < rr_archetype_fit_work_bytes(npair, njob, m, nl, max_npix)) return RR_EINVAL;
  if (method != RR_SOLVE_PCA && method != RR_SOLVE_NNLS && method != RR_SOLVE_BVLS &&
      method != RR_SOLVE_UNSUPPORTED)
    return RR_EINVAL;
  ArchParams p{pairs, npair, band, pix_basis, w, wflux, flux, arch, leg, pix_stride,
               max_npix, narch, jobs, njob, m, nl, prior, method, chi2, coeff};
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
  if (blocks > 2147483647LL || npair > 2147483647LL) return RR_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  double* wk = static_cast<double*>(work);
  const unsigned sblocks = (unsigned)((total + 127) / 128);
#define RR_PAIR_CASE(N)                                                               \
  case N:                                                                             \
    arch_pair_kernel<N><<<(unsigned)npair, 256, 0, st>>>(p, wk);                      \
    break;
  switch (nl) {
    RR_PAIR_CASE(0)
    RR_PAIR_CASE(1)
    RR_PAIR_CASE(2)
    RR_PAIR_CASE(3)
    RR_PAIR_CASE(4)
    RR_PAIR_CASE(5)
    RR_PAIR_CASE(6)
    RR_PAIR_CASE(7)
    RR_PAIR_CASE(8)
    RR_PAIR_CASE(9)
    default:
      return RR_EINVAL;
  }
#undef RR_PAIR_CASE
  RR_CHECK_LAUNCH();
#define RR_ARCH_CASE(N)                                                               \
  case N:                                                                             \
    if (m == 1)                                                                       \
      arch_gram_kernel<N, 1><<<(unsigned)blocks, kArchWarps * 32, 0, st>>>(p, wk);    \
    else                                                                              \
      arch_gram_kernel<N, 0><<<(unsigned)blocks, kArchWarps * 32, 0, st>>>(p, wk);    \
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
