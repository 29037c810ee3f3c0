// fitz candidates on the device: the local minima of each target's coarse
// chi2 and the fine redshift grids around them, so that the coarse scan and
// the fine-grid pair scans of a whole target batch can run back to back
// (and be captured in one CUDA graph) without a host round trip.
//
// Reference behaviour followed (redrock 0.22):
//   find_minima  fitz.py:46-67    local minima including the edges, with
//                                 <= comparisons, sorted by value
//   fitz         fitz.py:226-240  zz = np.linspace(z[i-1], z[i+1], n),
//                                 indices clipped to the grid
//
// One warp per target row.  Each lane keeps the K + 1 smallest (value,
// index) minima of its strided share of the row in registers, then the
// warp merges them in K + 1 rounds of a (value, index) minimum.  numpy's
// argsort is not stable, so when two of the selected values are equal (or
// the K-th equals the next) the order redrock would see is not determined
// here: such rows are flagged and the caller sorts them on the host.
#include <cmath>
#include <cstdint>

#include "rr_common.cuh"

namespace rr {

constexpr int kMaxCand = 8;

struct Cand {
  double v;
  int32_t i;
};

__device__ __forceinline__ bool cand_less(const Cand& a, const Cand& b) {
  return a.v < b.v || (a.v == b.v && a.i < b.i);
}

// np.linspace(lo, hi, n)[k] for n >= 2: k * ((hi - lo) / (n - 1)) + lo,
// the last point exactly hi (separately rounded multiply and add, as
// numpy's ufuncs do); a zero step gives lo everywhere
__device__ __forceinline__ double linspace_at(double lo, double hi, int n, int k) {
  if (k == n - 1) return hi;
  const double step = ddiv(dsub(hi, lo), (double)(n - 1));
  if (step == 0.0) return lo;
  return dadd(dmul((double)k, step), lo);
}

__global__ void fitz_candidates_kernel(const double* __restrict__ zchi2,
                                       const double* __restrict__ penalty, int64_t ntarget,
                                       int64_t nz, const double* __restrict__ z, int K, int nfine,
                                       int32_t* __restrict__ cand, int32_t* __restrict__ count,
                                       int8_t* __restrict__ tie, double* __restrict__ pair_z,
                                       int32_t* __restrict__ pair_t) {
  const int lane = threadIdx.x & 31;
  const int64_t t = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (t >= ntarget) return;  // whole warps leave together
  const double* row = zchi2 + t * nz;
  const double* pen = penalty ? penalty + t * nz : nullptr;
  const int keep = K + 1;
  Cand best[kMaxCand + 1];
#pragma unroll
  for (int k = 0; k <= kMaxCand; ++k) best[k] = Cand{INFINITY, INT32_MAX};
  int nmin = 0;
  for (int64_t i = lane; i < nz; i += 32) {
    const double x = pen ? dadd(row[i], pen[i]) : row[i];
    bool is_min = true;
    if (i > 0) {
      const double xl = pen ? dadd(row[i - 1], pen[i - 1]) : row[i - 1];
      is_min = x <= xl;
    }
    if (is_min && i + 1 < nz) {
      const double xr = pen ? dadd(row[i + 1], pen[i + 1]) : row[i + 1];
      is_min = x <= xr;
    }
    if (!is_min) continue;
    ++nmin;
    Cand c{x, (int32_t)i};
    // insertion into the sorted register list (first `keep` entries used)
#pragma unroll
    for (int k = 0; k <= kMaxCand; ++k) {
      if (k < keep && cand_less(c, best[k])) {
        const Cand tmp = best[k];
        best[k] = c;
        c = tmp;
      }
    }
  }
  // total number of minima in the row
  int total = nmin;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
  // merge: keep rounds of the warp-wide (value, index) minimum of the heads
  Cand sel[kMaxCand + 1];
  int head = 0;
  for (int r = 0; r < keep; ++r) {
    Cand h = best[0];
#pragma unroll
    for (int k = 0; k <= kMaxCand; ++k)
      if (k == head) h = best[k];
    if (head >= keep) h = Cand{INFINITY, INT32_MAX};
    Cand m = h;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      Cand other;
      other.v = __shfl_xor_sync(0xffffffffu, m.v, o);
      other.i = __shfl_xor_sync(0xffffffffu, m.i, o);
      if (cand_less(other, m)) m = other;
    }
    if (h.i == m.i && h.v == m.v && m.i != INT32_MAX) ++head;
#pragma unroll
    for (int k = 0; k <= kMaxCand; ++k)
      if (k == r) sel[k] = m;
  }
  const int n = total < K ? total : K;
  bool ambiguous = false;
#pragma unroll
  for (int k = 0; k < kMaxCand; ++k)
    if (k + 1 < keep && k + 1 < total && k < n && sel[k].v == sel[k + 1].v) ambiguous = true;
  if (lane == 0) {
    count[t] = n;
    tie[t] = ambiguous ? 1 : 0;
  }
  // candidate k = lane (k < K): its index and fine grid; slots past the
  // count repeat candidate 0 so every pair is a valid evaluation
  if (lane < K) {
    Cand c = sel[0];
#pragma unroll
    for (int k = 0; k <= kMaxCand; ++k)
      if (k == lane && lane < n) c = sel[k];
    cand[t * K + lane] = lane < n ? c.i : -1;
    const int64_t im = c.i;
    const double lo = z[im > 0 ? im - 1 : 0];
    const double hi = z[im + 1 < nz ? im + 1 : nz - 1];
    double* pz = pair_z + (t * K + lane) * nfine;
    int32_t* pt = pair_t + (t * K + lane) * nfine;
    for (int q = 0; q < nfine; ++q) {
      pz[q] = nfine > 1 ? linspace_at(lo, hi, nfine, q) : lo;
      pt[q] = (int32_t)t;
    }
  }
}

}  // namespace rr

using namespace rr;

extern "C" int rr_fitz_candidates(const double* zchi2, const double* penalty, int64_t ntarget,
                                  int64_t nz, const double* redshifts, int32_t K, int32_t nfine,
                                  int32_t* cand, int32_t* count, int8_t* tie, double* pair_z,
                                  int32_t* pair_t, rr_stream_t stream) {
  if (ntarget < 0 || nz < 1 || K < 1 || K > kMaxCand || nfine < 1) return RR_EINVAL;
  if (nz > INT32_MAX - 1) return RR_EINVAL;
  if (ntarget == 0) return RR_OK;
  if (!zchi2 || !redshifts || !cand || !count || !tie || !pair_z || !pair_t) return RR_EINVAL;
  const int warps = 8;
  const int64_t blocks = (ntarget + warps - 1) / warps;
  if (blocks > INT32_MAX) return RR_EINVAL;
  fitz_candidates_kernel<<<(unsigned)blocks, warps * 32, 0, (cudaStream_t)stream>>>(
      zchi2, penalty, ntarget, nz, redshifts, K, nfine, cand, count, tie, pair_z, pair_t);
  RR_CHECK_LAUNCH();
  return RR_OK;
}
