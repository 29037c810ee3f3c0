// Fused redshift scan: device code and launch helpers shared by the
// per-group translation units rr_fused_g0.cu .. rr_fused_g3.cu (each
// instantiates the kernels of one nbasis group, so they compile in
// parallel).  The algorithm is described in rr_scan.cu.
#pragma once
#include <cmath>
#include <cstring>

#include "rr_common.cuh"
#include "rr_solve_dev.cuh"

namespace rr {

#ifndef RR_Q_UNROLL
#define RR_Q_UNROLL 1
#endif

#ifndef RR_SCAN_WARPS
#define RR_SCAN_WARPS 8
#endif
#ifndef RR_SCAN_STAGES
#define RR_SCAN_STAGES 2
#endif

#ifndef RR_PIX
#define RR_PIX 4
#endif
#ifndef RR_PIX_SMALL
#define RR_PIX_SMALL RR_PIX
#endif

constexpr int kQUnroll = RR_Q_UNROLL;
// pixels per step of the pixel loop: RR_PIX for the instantiations whose
// accumulators fill the register file (NB * ZT > 10), RR_PIX_SMALL for the
// others
template <int NB, int ZT>
constexpr int pix_per_step() {
  return NB * ZT > 10 ? RR_PIX : RR_PIX_SMALL;
}
constexpr int kWarps = RR_SCAN_WARPS;  // redshifts per tile (one per warp)
constexpr int kThreads = kWarps * 32;
constexpr int kChunk = RR_CHUNK;
static_assert(kChunk % RR_PIX == 0 && kChunk % RR_PIX_SMALL == 0,
              "chunk must hold whole pixel steps");
constexpr int kWin = kChunk + 2 * kHalfBand;  // basis rows per chunk window
constexpr int kStages = RR_SCAN_STAGES;      // copy pipeline depth
constexpr int kRwChunkDoubles = kChunk * RR_RW * RR_LANES;

// bounds of RR_SOLVE_BVLS (NNLS uses [0, inf) internally)
struct SolveBounds {
  double lo[RR_MAX_NBASIS];
  double hi[RR_MAX_NBASIS];
};

struct FusedParams {
  rr_scan_targets tg;
  rr_segment_desc segs[16];
  int nseg;
  int ntemplate;
  rr_scan_template tm[RR_MAX_TEMPLATES];
  int64_t tile_start[RR_MAX_TEMPLATES + 1];
  int64_t chunks_total;  // pixel chunks per block (over all segments)
  int max_stride;        // largest basis_stride
  int block_group;       // tile order: 0 = target blocks fastest; G > 0 = all z tiles of
                         // G blocks before the next G (their packed rows stay in L2)
  int* tile_counter;
  int* resweep_counter;  // [0] tiles swept a second time for the direct residual,
                         // [1] (target, z) lanes re-evaluated there
  int* status;
};

// Stage buffers live in the dynamic shared-memory array; stage s holds the
// packed resolution rows of a chunk (kRwChunkDoubles) followed by the basis
// windows of the tile's redshifts.  Addresses are formed from the
// __shared__ array itself so every read in the pixel loop is a shared load.
extern __shared__ __align__(128) double rr_stage_smem[];

struct StageBufs {
  int stage_doubles;  // doubles per stage
  uint64_t* full;     // kStages mbarriers
  __device__ __forceinline__ double* rw(int s) const { return rr_stage_smem + s * stage_doubles; }
  __device__ __forceinline__ double* t(int s) const {
    return rr_stage_smem + s * stage_doubles + kRwChunkDoubles;
  }
};

// phase parity of each stage barrier (bit s), kept in a register
struct Uses {
  uint32_t bits = 0;
  __device__ __forceinline__ uint32_t parity(int s) const { return (bits >> s) & 1u; }
  __device__ __forceinline__ void bump(int s) { bits ^= 1u << s; }
};

__device__ __forceinline__ void chunk_segment(const FusedParams& p, int64_t c, int& seg,
                                              int64_t& p0) {
  int s = 0;
  int64_t acc = 0;
  for (; s < p.nseg; ++s) {
    const int64_t n = p.segs[s].npix_pad / kChunk;
    if (c < acc + n) break;
    acc += n;
  }
  seg = s;
  p0 = (c - acc) * kChunk;
}

// Thread 0: start the copies of chunk c of (block, template, z0) into stage s.
__device__ __forceinline__ void issue_chunk(const FusedParams& p, const rr_scan_template& tm,
                                            int block, int z0, int nzt, int64_t c, int s,
                                            StageBufs& sb) {
  int seg;
  int64_t p0;
  chunk_segment(p, c, seg, p0);
  const rr_segment_desc& sd = p.segs[seg];
  const uint32_t rw_bytes = kRwChunkDoubles * sizeof(double);
  const uint32_t t_bytes = kWin * tm.basis_stride * sizeof(double);
  mbar_arrive_expect_tx(&sb.full[s], rw_bytes + nzt * t_bytes);
  const double* src_rw =
      p.tg.rw + ((int64_t)block * p.tg.npix_block + sd.rw_offset + p0) * (RR_RW * RR_LANES);
  bulk_g2s(sb.rw(s), src_rw, rw_bytes, &sb.full[s]);
  for (int w = 0; w < nzt; ++w) {
    const double* src_t =
        tm.basis + ((int64_t)(z0 + w) * tm.pix_stride + sd.basis_offset + p0 - kHalfBand) *
                       tm.basis_stride;
    bulk_g2s(sb.t(s) + (int64_t)w * kWin * tm.basis_stride, src_t, t_bytes, &sb.full[s]);
  }
}

template <int NB>
__device__ __forceinline__ void write_eval(const rr_scan_template& tm, int64_t row, int z,
                                           const double (&c)[NB], double chi2, double wsum) {
  tm.zchi2[row * tm.nz + z] = chi2;
  double* co = tm.zcoeff + (row * tm.nz + z) * NB;
#pragma unroll
  for (int i = 0; i < NB; ++i) co[i] = c[i];
  if (tm.oii) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NB; ++i) s = fma(c[i], tm.oii[i], s);
    // an all-zero-weight target is skipped before the penalty in redrock
    tm.penalty[row * tm.nz + z] = (wsum != 0.0 && s < 0.0) ? -s : 0.0;
  }
}

// One sweep of a tile's pixels through the two-stage copy pipeline.  Each
// thread owns ZT redshifts of its target (warp w scans z0 + w ZT + j,
// j < ZT); its packed-row loads serve all ZT of them.
// RESID = false: accumulate the Gram matrices m[j] (and y[j] unless EXTY).
// RESID = true:  accumulate the direct residual sums (g - Tb'.c)^2 into
//                acc[j] for the (lane, j) with active[j] set.
// Returns false (uniformly across the CTA) if a copy wait timed out.
template <int NB, bool RESID, bool EXTY, int ZT>
__device__ __forceinline__ bool sweep(const FusedParams& p, const rr_scan_template& tm, int block,
                                      int z0, int nzt, const bool (&active)[ZT], StageBufs& sb,
                                      Uses& uses, double (&m)[ZT][NB * (NB + 1) / 2],
                                      double (&y)[ZT][NB], const double (&c)[ZT][NB],
                                      double (&acc)[ZT]) {
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int stride = tm.basis_stride;
  const int64_t nchunk = p.chunks_total;
  bool any = false;
#pragma unroll
  for (int j = 0; j < ZT; ++j) any = any || active[j];
  // prologue: the first kStages - 1 chunks in flight
  if (threadIdx.x == 0)
    for (int i = 0; i < kStages - 1 && i < nchunk; ++i) issue_chunk(p, tm, block, z0, nzt, i, i, sb);
  int s = 0;
  for (int64_t ch = 0; ch < nchunk; ++ch) {
    const int64_t ahead = ch + kStages - 1;
    const bool more = ahead < nchunk;
    const int s_ahead = (s + kStages - 1) % kStages;
    if (threadIdx.x == 0 && more) issue_chunk(p, tm, block, z0, nzt, ahead, s_ahead, sb);
    const bool ok = mbar_wait(&sb.full[s], uses.parity(s), p.status);
    uses.bump(s);
    if (any && ok && RESID) {
      const double* rws = sb.rw(s) + lane;
#pragma unroll
      for (int j = 0; j < ZT; ++j) {
        if (!active[j]) continue;
        const double* ts = sb.t(s) + (warp * ZT + j) * kWin * stride;
        // model = R (T c): T c once per basis row of the window (n FMAs),
        // then the 11-tap band per pixel -- the coefficients are known
        // here, so the residual needs no full R.T product
        double tc[kWin];
#pragma unroll
        for (int r = 0; r < kWin; ++r) {
          const double* trow = ts + r * stride;
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b) v = fma(trow[b], c[j][b], v);
          tc[r] = v;
        }
#pragma unroll
        for (int q = 0; q < kChunk; ++q) {
          double mi = 0.0;
#pragma unroll
          for (int k = 0; k < kBand; ++k)
            mi = fma(rws[(q * RR_RW + k) * RR_LANES], tc[q + k], mi);
          const double res = rws[(q * RR_RW + kBand) * RR_LANES] - mi;
          acc[j] = fma(res, res, acc[j]);
        }
      }
    } else if (any && ok) {
      const double* rws = sb.rw(s) + lane;
      const double* ts = sb.t(s) + warp * ZT * kWin * stride;
      constexpr int kPix = pix_per_step<NB, ZT>();
      // kPix pixels per step: basis row q + k serves pixel q + i with band
      // index k - i, so each row is read once for all kPix pixels (and the
      // packed rows once for all ZT redshifts)
#pragma unroll kQUnroll
      for (int q = 0; q < kChunk; q += kPix) {
        double tp[ZT][kPix][NB];
#pragma unroll
        for (int j = 0; j < ZT; ++j)
#pragma unroll
          for (int i = 0; i < kPix; ++i)
#pragma unroll
            for (int b = 0; b < NB; ++b) tp[j][i][b] = 0.0;
#pragma unroll
        for (int k = 0; k < kBand + kPix - 1; ++k) {
          double rk[kPix];
#pragma unroll
          for (int i = 0; i < kPix; ++i)
            rk[i] = (k - i >= 0 && k - i < kBand) ? rws[((q + i) * RR_RW + k - i) * RR_LANES] : 0.0;
#pragma unroll
          for (int j = 0; j < ZT; ++j) {
            const double* trow = ts + (j * kWin + q + k) * stride;
#pragma unroll
            for (int b = 0; b + 1 < NB; b += 2) {
              const double2 tv = *reinterpret_cast<const double2*>(trow + b);
#pragma unroll
              for (int i = 0; i < kPix; ++i) {
                if (k - i >= 0 && k - i < kBand) {
                  tp[j][i][b] = fma(rk[i], tv.x, tp[j][i][b]);
                  tp[j][i][b + 1] = fma(rk[i], tv.y, tp[j][i][b + 1]);
                }
              }
            }
            if (NB & 1) {
              const double tv = trow[NB - 1];
#pragma unroll
              for (int i = 0; i < kPix; ++i)
                if (k - i >= 0 && k - i < kBand) tp[j][i][NB - 1] = fma(rk[i], tv, tp[j][i][NB - 1]);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < kPix; ++i) {
          const double gi = !EXTY ? rws[((q + i) * RR_RW + kBand) * RR_LANES] : 0.0;
#pragma unroll
          for (int j = 0; j < ZT; ++j) {
            if (!EXTY)
#pragma unroll
              for (int b = 0; b < NB; ++b) y[j][b] = fma(gi, tp[j][i][b], y[j][b]);
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
              for (int b = 0; b <= a; ++b)
                m[j][a * (a + 1) / 2 + b] = fma(tp[j][i][a], tp[j][i][b], m[j][a * (a + 1) / 2 + b]);
          }
        }
      }
    }
    // stage s is free for chunk ch + kStages once every warp is past this
    // point; a timed-out wait anywhere stops the whole CTA
    if (__syncthreads_or(!ok)) {
      // let the copies already issued land before leaving
      if (threadIdx.x == 0)
        for (int64_t i = ch + 1; i < nchunk && i <= ahead; ++i) {
          const int si = (int)((s + (i - ch)) % kStages);
          mbar_wait(&sb.full[si], uses.parity(si), p.status);
          uses.bump(si);
        }
      return false;
    }
    s = (s + 1 == kStages) ? 0 : s + 1;
  }
  return true;
}

// EXTY: y comes from tm.y_ext (rr_ygemm) instead of the pixel sweep.  ZT:
// redshifts per thread; the tile is 32 targets x kWarps ZT redshifts.
template <int NB, bool EXTY, int ZT>
__device__ void scan_tile(const FusedParams& p, const rr_scan_template& tm, int block, int z0,
                          StageBufs& sb, Uses& uses, bool& failed) {
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int nzt = min(kWarps * ZT, tm.nz - z0);
  constexpr int kTri = NB * (NB + 1) / 2;
  double m[ZT][kTri];
  double y[ZT][NB];
  double c[ZT][NB];
  double acc[ZT];
  bool inz[ZT];
#pragma unroll
  for (int j = 0; j < ZT; ++j) {
    acc[j] = 0.0;
    inz[j] = warp * ZT + j < nzt;
#pragma unroll
    for (int i = 0; i < kTri; ++i) m[j][i] = 0.0;
#pragma unroll
    for (int i = 0; i < NB; ++i) y[j][i] = 0.0;
  }
  const int32_t row = p.tg.rows[block * RR_LANES + lane];
  if (!sweep<NB, false, EXTY, ZT>(p, tm, block, z0, nzt, inz, sb, uses, m, y, c, acc)) {
    failed = true;
    return;
  }
  bool fix[ZT];
  bool anyfix = false;
  const double fwf = row >= 0 ? p.tg.fwf[block * RR_LANES + lane] : 0.0;
  const double wsum = row >= 0 ? p.tg.wsum[block * RR_LANES + lane] : 0.0;
#pragma unroll
  for (int j = 0; j < ZT; ++j) {
    fix[j] = false;
    const int z = z0 + warp * ZT + j;
    if (inz[j] && row >= 0) {
      if (EXTY) {
        const double* ye = tm.y_ext + ((int64_t)(block * RR_LANES + lane) * tm.nz + z) * NB;
#pragma unroll
        for (int b = 0; b < NB; ++b) y[j][b] = ye[b];
      }
      double chi2 = 0.0, err = 0.0;
      const bool ok = solve_eval<NB>(tm.method, tm.prior, m[j], y[j], fwf, wsum, c[j], chi2, err);
      fix[j] = ok && err > kChi2FixTol;
      write_eval<NB>(tm, row, z, c[j], chi2, wsum);
    }
    anyfix = anyfix || fix[j];
  }
  // ill-conditioned fits: re-evaluate chi2 as the direct weighted residual
  // sum w (f - Tb c)^2 (redrock's own formula, zscan.py:777-780), which does
  // not suffer the cancellation of f^T W f - c^T y
  if (__syncthreads_or(anyfix)) {
    if (threadIdx.x == 0 && p.resweep_counter) atomicAdd(p.resweep_counter, 1);
    int nfix = 0;
#pragma unroll
    for (int j = 0; j < ZT; ++j) nfix += __popc(__ballot_sync(0xffffffffu, fix[j]));
    if (lane == 0 && nfix && p.resweep_counter) atomicAdd(p.resweep_counter + 1, nfix);
#pragma unroll
    for (int j = 0; j < ZT; ++j) acc[j] = 0.0;
    if (!sweep<NB, true, EXTY, ZT>(p, tm, block, z0, nzt, fix, sb, uses, m, y, c, acc)) {
      failed = true;
      return;
    }
#pragma unroll
    for (int j = 0; j < ZT; ++j)
      if (fix[j]) tm.zchi2[(int64_t)row * tm.nz + z0 + warp * ZT + j] = acc[j];
  }
}

// (block, z tile) of tile `local` of a template with nzt z tiles.  G <= 0
// (or >= nblock): target blocks fastest, so the tiles running at one time
// share z tiles (basis windows) across blocks.  G > 0: the blocks form
// groups of G; all z tiles of one group come before the next group, blocks
// fastest within it, so a group's packed rows are reused by many z tiles
// while they sit in L2 (the last group may be smaller).
__device__ __forceinline__ void tile_coords(int64_t local, int64_t nzt, int nblock, int G,
                                            int& block, int64_t& zt) {
  if (G <= 0 || G >= nblock) {
    block = (int)(local % nblock);
    zt = local / nblock;
    return;
  }
  const int64_t full = nblock / G;
  const int64_t per = (int64_t)G * nzt;
  const int64_t g = local / per;
  if (g < full) {
    const int64_t r = local - g * per;
    block = (int)(g * G + r % G);
    zt = r / G;
  } else {
    const int gr = nblock - (int)full * G;
    const int64_t r = local - full * per;
    block = (int)(full * G + r % gr);
    zt = r / gr;
  }
}

// Launch groups of the fused kernel, one instantiation per (group,
// redshifts per thread ZT), so a group's register allocation does not
// depend on the others: nbasis 10 (GALAXY; ZT 1), 4 (QSO; ZT 1-3), 5
// (STAR; ZT 1-2), all other nbasis (ZT 1).  Several redshifts per thread
// share each packed-row load from shared memory: with one redshift the
// small bases are bound by shared-memory wavefronts rather than the FP64
// pipe.  The ZT of the small groups is a launch option (rr_scan_options),
// picked by the host autotuner; defaults below.
__host__ __device__ constexpr int group_of(int nb) {
  return nb == 10 ? 0 : (nb == 4 ? 1 : (nb == 5 ? 2 : 3));
}
constexpr int kNGroups = 4;
constexpr int kDefaultZt[kNGroups] = {1, 2, 2, 1};
constexpr int kMaxZt[kNGroups] = {1, 3, 2, 1};

template <int GROUP, bool EXTY, int ZT>
__global__ void __launch_bounds__(kThreads, (kWarps <= 4 ? 2 : 1)) zscan_fused_kernel(const __grid_constant__ FusedParams p) {
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ int64_t s_tile;
  StageBufs sb;
  sb.stage_doubles = kRwChunkDoubles + kWarps * ZT * kWin * p.max_stride;
  sb.full = full;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // the next group's launch (programmatic dependent launch) may start now:
  // its CTAs take the SMs this grid's CTAs leave in its last tile wave
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  Uses uses;
  bool failed = false;
  const int64_t ntiles = p.tile_start[p.ntemplate];
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(p.tile_counter, 1);
    __syncthreads();
    const int64_t tile = s_tile;
    __syncthreads();
    if (tile >= ntiles) break;
    int t = 0;
    while (t + 1 < p.ntemplate && tile >= p.tile_start[t + 1]) ++t;
    const rr_scan_template& tm = p.tm[t];
    const int64_t local = tile - p.tile_start[t];
    const int64_t nzt = (p.tile_start[t + 1] - p.tile_start[t]) / p.tg.nblock;
    int block;
    int64_t ztile;
    tile_coords(local, nzt, p.tg.nblock, p.block_group, block, ztile);
    const int z0 = (int)ztile * kWarps * ZT;
#define RR_TILE_CASE(N)                                                   \
  case N:                                                                 \
    if constexpr (group_of(N) == GROUP) {                                 \
      scan_tile<N, EXTY, ZT>(p, tm, block, z0, sb, uses, failed);         \
    } else {                                                              \
      set_status(p.status, RR_EINVAL);                                    \
      failed = true;                                                      \
    }                                                                     \
    break;
    switch (tm.nbasis) {
      RR_TILE_CASE(1) RR_TILE_CASE(2) RR_TILE_CASE(3) RR_TILE_CASE(4) RR_TILE_CASE(5)
      RR_TILE_CASE(6) RR_TILE_CASE(7) RR_TILE_CASE(8) RR_TILE_CASE(9) RR_TILE_CASE(10)
      default: set_status(p.status, RR_EINVAL); failed = true; break;
    }
#undef RR_TILE_CASE
    if (failed) break;  // uniform across the CTA
    __syncthreads();
  }
  // a grid launched as a dependent completes only after the grid before it
  // (no-op otherwise), so stream order still holds for whatever follows the
  // last launch
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

inline size_t fused_smem_bytes(int max_stride, int zt) {
  return (size_t)kStages * (kRwChunkDoubles + (size_t)kWarps * zt * kWin * max_stride) *
         sizeof(double);
}

// Launch one instantiation of the fused kernel over the templates selected
// by `pick` (indices into templates), using counter (zeroed by the caller) as
// its tile counter.  overlap: launch as a programmatic dependent of the
// previous kernel in the stream (the previous fused launch, whose tiles are
// independent of these).
template <int GROUP, bool EXTY, int ZT>
int launch_fused(const rr_scan_targets* targets, const rr_scan_template* templates,
                        const int* pick, int npick, int bgroup, int* counter, int* resweep,
                        int* status, bool overlap, cudaStream_t stream) {
  constexpr int kZt = ZT;
  FusedParams p;
  memset(&p, 0, sizeof(p));
  p.tg = *targets;
  p.nseg = targets->nseg;
  int64_t chunks = 0;
  for (int s = 0; s < p.nseg; ++s) {
    p.segs[s] = targets->segs[s];
    chunks += p.segs[s].npix_pad / kChunk;
  }
  p.chunks_total = chunks;
  p.ntemplate = npick;
  p.tile_start[0] = 0;
  int max_stride = 2;
  for (int i = 0; i < npick; ++i) {
    const rr_scan_template& tm = templates[pick[i]];
    p.tm[i] = tm;
    const int64_t zt = (tm.nz + kWarps * kZt - 1) / (kWarps * kZt);
    p.tile_start[i + 1] = p.tile_start[i] + zt * targets->nblock;
    max_stride = tm.basis_stride > max_stride ? tm.basis_stride : max_stride;
  }
  p.max_stride = max_stride;
  p.block_group = bgroup;
  p.tile_counter = counter;
  p.resweep_counter = resweep;
  p.status = status;
  const int64_t ntiles = p.tile_start[npick];
  if (ntiles == 0) return RR_OK;
  const size_t smem = fused_smem_bytes(max_stride, kZt);
  RR_CUDA_TRY(cudaFuncSetAttribute(zscan_fused_kernel<GROUP, EXTY, ZT>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 0;
  RR_CUDA_TRY(cudaGetDevice(&dev));
  RR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  int per_sm = 1;
  RR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, zscan_fused_kernel<GROUP, EXTY, ZT>,
                                                            kThreads, smem));
  if (per_sm < 1) per_sm = 1;
  const int64_t slots = (int64_t)nsm * per_sm;
  const int64_t grid = ntiles < slots ? ntiles : slots;
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = overlap ? 1 : 0;
  RR_CUDA_TRY(cudaLaunchKernelEx(&cfg, zscan_fused_kernel<GROUP, EXTY, ZT>, p));
  RR_CHECK_LAUNCH();
  return RR_OK;
}

// launch with the runtime ZT of a group (one of its compiled values)
template <int GROUP, bool EXTY>
int launch_group(int zt, int bgroup, const rr_scan_targets* targets,
                 const rr_scan_template* templates, const int* pick, int npick, int* counter,
                 int* resweep, int* status, bool overlap, cudaStream_t stream) {
  if (zt < 1 || zt > kMaxZt[GROUP]) return RR_EINVAL;
  if constexpr (kMaxZt[GROUP] >= 3)
    if (zt == 3)
      return launch_fused<GROUP, EXTY, (kMaxZt[GROUP] >= 3 ? 3 : 1)>(
          targets, templates, pick, npick, bgroup, counter, resweep, status, overlap, stream);
  if constexpr (kMaxZt[GROUP] >= 2)
    if (zt == 2)
      return launch_fused<GROUP, EXTY, (kMaxZt[GROUP] >= 2 ? 2 : 1)>(
          targets, templates, pick, npick, bgroup, counter, resweep, status, overlap, stream);
  return launch_fused<GROUP, EXTY, 1>(targets, templates, pick, npick, bgroup, counter, resweep,
                                      status, overlap, stream);
}

// one entry per group translation unit
#define RR_FUSED_GROUP_DECL(G)                                                                   \
  int fused_group_##G(bool exty, int zt, int bgroup, const rr_scan_targets* targets,             \
                      const rr_scan_template* templates, const int* pick, int npick,             \
                      int* counter, int* resweep, int* status, bool overlap,            \
                      cudaStream_t stream);
RR_FUSED_GROUP_DECL(0)
RR_FUSED_GROUP_DECL(1)
RR_FUSED_GROUP_DECL(2)
RR_FUSED_GROUP_DECL(3)
#undef RR_FUSED_GROUP_DECL

}  // namespace rr
