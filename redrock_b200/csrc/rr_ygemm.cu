// Tensor-core form of the y = Tb^T W f term of the redshift scan.
//
// With rw[p][k] = sqrt(w_p) R[p, p+k-5] and g_p = sqrt(w_p) f_p (the packed
// rows of rr_pack_targets), redrock's y (zscan.py:741-748, Tb^T (w f)) is
//   y_i(t, z) = sum_p g_p sum_k rw[p][k] T_z[p+k-5][i] = sum_q G[q][t] T_z[q][i]
// with G[., t] = R^T W f of target t, which does not depend on z.  So y for
// every (target, z, basis) of a template is one GEMM:
//   Y[t][(z, i)] = sum_q G[q][t] T[z][q][i]   (M = targets, N = (z, i),
//                                              K = padded basis pixel index).
// rr_pack_g builds G (and a power-of-two scale per target); the GEMM runs on
// the tcgen05 tensor cores; the fused scan then reads Y instead of summing y
// itself (rr_scan_template.y_ext).
//
// Operand tiles sit in shared memory in the canonical K-major, no-swizzle
// UMMA layout (8-row x 16-byte core matrices; unit u of a tile is the
// 16-byte core-matrix row at byte 16 u) and one thread issues the
// tcgen05.mma into TMEM accumulators.  Variants (rr_ygemm_variant):
//   BF16X3  (rr_ygemm) three bf16 slices per value (hi + mid + lo), the six
//           products of slice order <= 2, one FP32 accumulator (kind::f16).
//           Slicing happens while a tile is staged.
//   TF32X3  (rr_ygemm) two tf32 slices, hi*hi + hi*lo + lo*hi, FP32
//           accumulation (kind::tf32).
//   INT8X7  (rr_slice_g_i8 + rr_slice_basis_i8 + rr_ygemm_i8) Ozaki scheme:
//           each G column and basis column is scaled by a power of two and
//           rounded to a 49-bit integer X = sum_k a_k 128^(6-k) with seven
//           base-128 digits |a_k| <= 64 (kind::i8 operands).  The 28 digit
//           products of order i + j <= 6 accumulate EXACTLY in the int32
//           accumulator i + j and the seven accumulators combine in FP64.
//           The digits are written once per operand, already in the
//           shared-memory tile layout, and the GEMM streams them with 1-D
//           bulk copies (warp-specialised: one producer thread, one MMA
//           thread, four stages).  Error <= K 2^-45 2^(e_t + e_n) per
//           output for columns bounded by 2^e_t and 2^e_n.
#include <cuda_bf16.h>
#include <climits>
#include <cmath>

#include "rr_common.cuh"

namespace rr {
namespace yg {

constexpr int kTileM = 128;  // targets per tile (MMA M)
constexpr int kThreads = 256;
constexpr int kKpadAlign = 64;  // G rows padded to a multiple of every stage depth
constexpr int kExpBias = 4096;  // stored exponents are biased; 0 = all-zero row/column
constexpr double kExpMargin = 128.0 / 127.0;  // exponents bound max |x| by 127/128 2^e

// ---------------------------------------------------------------------------
// tcgen05 / descriptor helpers
// ---------------------------------------------------------------------------
// Shared-memory matrix descriptor: K-major, no swizzle; LBO = 128 B between
// the two core matrices along K of one instruction, SBO between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  return d;                // base offset 0, layout type 0 = SWIZZLE_NONE
}

// instruction descriptor: D format / A,B formats (fmt), K-major A and B, N, M
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt, int n, int m) {
  return fmt | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

enum Kind { kF16, kTF32, kI8 };

template <Kind K>
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accumulate) {
  if constexpr (K == kF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
  } else if constexpr (K == kTF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
  }
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// 8 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ int unbias(int e) { return e > 0 ? e - kExpBias : 0; }

// unit u of a tile with nkg core matrices along K: row and K group
__device__ __forceinline__ void unit_rc(int u, int nkg, int& r, int& kg) {
  r = (u & 7) + 8 * (u / (8 * nkg));
  kg = (u >> 3) % nkg;
}

// ===========================================================================
// BF16X3 / TF32X3: slices made while staging, FP32 accumulation
// ===========================================================================
template <int V>
struct Var;
template <>
struct Var<RR_YGEMM_BF16X3> {
  static constexpr int kEsz = 2, kSlices = 3, kKInst = 16, kNMax = 256, kKt = 32;
  static constexpr Kind kKind = kF16;
  static constexpr uint32_t kFmt = (1u << 4) | (1u << 7) | (1u << 10);  // D f32, A/B bf16
};
template <>
struct Var<RR_YGEMM_TF32X3> {
  static constexpr int kEsz = 4, kSlices = 2, kKInst = 8, kNMax = 256, kKt = 32;
  static constexpr Kind kKind = kTF32;
  static constexpr uint32_t kFmt = (1u << 4) | (2u << 7) | (2u << 10);  // D f32, A/B tf32
};

template <int V>
struct Geo {
  using P = Var<V>;
  static constexpr int kE = 16 / P::kEsz;            // elements per 16-byte core-matrix row
  static constexpr int kNkg = P::kKt / kE;           // core matrices along K per stage
  static constexpr int kSteps = P::kKt / P::kKInst;  // MMA instructions along K per stage
  static constexpr int kSbo = kNkg * 128;            // bytes between 8-row groups
  static constexpr int kASlice = kTileM * P::kKt * P::kEsz;
  static constexpr int kTmemCols = 256;
  static constexpr int kStages = 2;
  static __host__ __device__ constexpr int b_slice(int n) { return n * P::kKt * P::kEsz; }
  static __host__ __device__ constexpr int stage_bytes(int n) {
    return P::kSlices * (kASlice + b_slice(n));
  }
};

struct YParams {
  const double* g;      // [kpad][npos]
  const double* basis;  // [nz][pix_stride][basis_stride]
  double* y;            // [npos][nz][nbasis]
  int64_t npos, kpad, pix_stride;
  int nz, nbasis, basis_stride;
  int zt;    // redshifts per tile
  int n;     // MMA N (zt * nbasis rounded up to 16)
  int* status;
};

__device__ __forceinline__ uint32_t bf16_bits(double x, double& rest) {
  const __nv_bfloat16 h = __double2bfloat16(x);
  rest = x - (double)__bfloat162float(h);
  return (uint32_t)__bfloat16_as_ushort(h);
}
__device__ __forceinline__ uint32_t tf32_bits(double x, double& rest) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(__double2float_rn(x)));
  rest = x - (double)__uint_as_float(r);
  return r;
}

// Write the slices of v[0..kE) to dst + s * slice_bytes, s < kSlices.
template <int V>
__device__ __forceinline__ void store_slices(const double (&v)[Geo<V>::kE], unsigned char* dst,
                                             int slice_bytes) {
  constexpr int kE = Geo<V>::kE;
  if constexpr (V == RR_YGEMM_BF16X3) {
    uint32_t w[3][4];
#pragma unroll
    for (int j = 0; j < kE; j += 2) {
      double r0 = v[j], r1 = v[j + 1];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const uint32_t lo = bf16_bits(r0, r0);
        const uint32_t hi = bf16_bits(r1, r1);
        w[s][j / 2] = lo | (hi << 16);
      }
    }
#pragma unroll
    for (int s = 0; s < 3; ++s)
      *reinterpret_cast<uint4*>(dst + s * slice_bytes) = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
  } else {
    uint32_t w[2][4];
#pragma unroll
    for (int j = 0; j < kE; ++j) {
      double r = v[j];
      w[0][j] = tf32_bits(r, r);
      w[1][j] = tf32_bits(r, r);
    }
#pragma unroll
    for (int s = 0; s < 2; ++s)
      *reinterpret_cast<uint4*>(dst + s * slice_bytes) = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
  }
}

// Stage K-chunk (pixels q0 .. q0 + kKt) of the tile into shared memory.
template <int V>
__device__ __forceinline__ void stage_tile(const YParams& p, unsigned char* st, int64_t t0, int z0,
                                           int nzt, int64_t q0) {
  using G = Geo<V>;
  using P = Var<V>;
  constexpr int kE = G::kE;
  // A: G[q][t0 + r]
  for (int u = threadIdx.x; u < kTileM * G::kNkg; u += kThreads) {
    int r, kg;
    unit_rc(u, G::kNkg, r, kg);
    const double* src = p.g + (q0 + kg * kE) * p.npos + t0 + r;
    double v[kE];
#pragma unroll
    for (int j = 0; j < kE; ++j) v[j] = __ldg(src + (int64_t)j * p.npos);
    store_slices<V>(v, st + u * 16, G::kASlice);
  }
  // B: row n = (zl, i) of the basis, T[z0 + zl][q][i]
  unsigned char* sb = st + P::kSlices * G::kASlice;
  const int nused = nzt * p.nbasis;
  for (int u = threadIdx.x; u < p.n * G::kNkg; u += kThreads) {
    int r, kg;
    unit_rc(u, G::kNkg, r, kg);
    double v[kE];
    if (r < nused) {
      const int zl = r / p.nbasis;
      const int i = r - zl * p.nbasis;
      const int64_t q = q0 + kg * kE;
      const double* src = p.basis + ((int64_t)(z0 + zl) * p.pix_stride + q) * p.basis_stride + i;
#pragma unroll
      for (int j = 0; j < kE; ++j)
        v[j] = (q + j < p.pix_stride) ? __ldg(src + (int64_t)j * p.basis_stride) : 0.0;
    } else {
#pragma unroll
      for (int j = 0; j < kE; ++j) v[j] = 0.0;
    }
    store_slices<V>(v, sb + u * 16, G::b_slice(p.n));
  }
}

template <int V>
__global__ void __launch_bounds__(kThreads, 1) ygemm_kernel(const __grid_constant__ YParams p) {
  using G = Geo<V>;
  using P = Var<V>;
  constexpr int kStages = G::kStages;
  extern __shared__ __align__(1024) unsigned char ysm[];
  __shared__ __align__(8) uint64_t done[kStages];
  __shared__ uint32_t s_tmem;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t t0 = (int64_t)blockIdx.x * kTileM;
  const int z0 = blockIdx.y * p.zt;
  const int nzt = min(p.zt, p.nz - z0);

  if (warp == 0) tmem_alloc(&s_tmem, G::kTmemCols);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&done[s], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  const uint32_t idesc = instr_desc(P::kFmt, p.n, kTileM);
  const int stage_bytes = G::stage_bytes(p.n);
  const int64_t nchunk = p.kpad / P::kKt;
  bool ok = true;
  for (int64_t c = 0; c < nchunk; ++c) {
    const int s = (int)(c & 1);
    unsigned char* st = ysm + s * stage_bytes;
    // the MMAs of chunk c - 2 read this stage: wait for their commit
    if (c >= 2) {
      const bool w = mbar_wait(&done[s], (uint32_t)(((c >> 1) - 1) & 1), p.status);
      if (__syncthreads_or(!w)) {
        ok = false;
        break;
      }
    }
    stage_tile<V>(p, st, t0, z0, nzt, c * P::kKt);
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(st);
      const uint32_t b0 = a0 + P::kSlices * G::kASlice;
#pragma unroll 1
      for (int ks = 0; ks < G::kSteps; ++ks) {
        const uint32_t koff = ks * 256;
        // all slice products of order <= kSlices - 1, smallest first
#pragma unroll 1
        for (int d = P::kSlices - 1; d >= 0; --d)
#pragma unroll 1
          for (int i = 0; i <= d; ++i) {
            const uint64_t da = smem_desc(a0 + i * G::kASlice + koff, G::kSbo);
            const uint64_t db = smem_desc(b0 + (d - i) * G::b_slice(p.n) + koff, G::kSbo);
            const uint32_t acc = (c > 0 || ks > 0 || d != P::kSlices - 1 || i > 0) ? 1u : 0u;
            mma<P::kKind>(tmem, da, db, idesc, acc);
          }
      }
      mma_commit(&done[s]);
    }
  }
  // all MMAs done: the last commit covers every earlier one
  if (ok && nchunk > 0) {
    const int64_t last = nchunk - 1;
    ok = mbar_wait(&done[last & 1], (uint32_t)((last >> 1) & 1), p.status);
  }
  ok = __syncthreads_and(ok);
  if (ok) {
    tc_fence_after();
    const int lg = warp & 3;     // TMEM lanes 32 lg .. 32 lg + 31
    const int half = warp >> 2;  // column half
    const int64_t pos = t0 + 32 * lg + lane;
    const int ncol = p.n / 2;
    const int nused = nzt * p.nbasis;
    double* yrow = p.y + (pos * p.nz + z0) * p.nbasis;
    const uint32_t tl = tmem + ((uint32_t)(32 * lg) << 16);
    for (int c0 = half * ncol; c0 < (half + 1) * ncol; c0 += 8) {
      uint32_t v[8];
      tmem_ld8(tl + c0, v);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (pos < p.npos && c0 + j < nused) yrow[c0 + j] = (double)__uint_as_float(v[j]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, G::kTmemCols);
  }
}

template <int V>
static int launch_ygemm(YParams p, cudaStream_t stream) {
  using P = Var<V>;
  if (p.kpad % P::kKt) return RR_EINVAL;
  int zt = P::kNMax / p.nbasis;
  if (zt > p.nz) zt = p.nz;
  p.zt = zt;
  p.n = ((zt * p.nbasis + 15) / 16) * 16;
  if (p.n > P::kNMax) return RR_EINVAL;
  const size_t smem = (size_t)Geo<V>::kStages * Geo<V>::stage_bytes(p.n);
  RR_CUDA_TRY(cudaFuncSetAttribute(ygemm_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  dim3 grid((unsigned)(p.npos / kTileM), (unsigned)((p.nz + zt - 1) / zt));
  ygemm_kernel<V><<<grid, kThreads, smem, stream>>>(p);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

// ===========================================================================
// INT8X7: pre-sliced operands, exact integer accumulation
// ===========================================================================
namespace i8 {
constexpr int kKt = 32;                    // pixels per stage = one MMA K step
constexpr int kNkg = kKt / 16;             // 2 core matrices along K
constexpr int kSbo = kNkg * 128;           // 256 B between 8-row groups
constexpr int kASlice = kTileM * kKt;      // bytes of one digit plane of a G block
constexpr uint32_t kFmt = (2u << 4) | (1u << 7) | (1u << 10);  // D s32, A/B signed 8-bit

// The two digit schemes (rr_ygemm_variant):
//   INT8X7: X = rint(x 2^(48 - e)), seven balanced base-128 digits, the 28
//           products of order <= 6 -> 7 int32 accumulators of N = 64
//           columns; |digit| <= 64, so K <= 65536 keeps them exact.
//   INT8X6: X = rint(x 2^(47 - e)), six balanced base-256 digits, the 21
//           products of order <= 5 -> 6 accumulators of N = 80 columns
//           (480 of the 512 TMEM columns); |digit| <= 128, so K <= 21845.
// e is the column's exponent with a 128/127 margin (max |x| < 127/128 2^e),
// which keeps the leading base-256 digit within int8: |X| <= 127 2^40.
// Y = sum_d acc_d 2^(-bits d) 2^(e_t + e_n + shift), shift = 2 bits
// (digits - 1) - 2 mant.
template <int V>
struct Scheme;
template <>
struct Scheme<RR_YGEMM_INT8X7> {
  static constexpr int kDigits = 7, kBits = 7, kMant = 48, kN = 64, kStages = 4;
  static constexpr int64_t kMaxK = 65536;
};
template <>
struct Scheme<RR_YGEMM_INT8X6> {
  static constexpr int kDigits = 6, kBits = 8, kMant = 47, kN = 80, kStages = 5;
  static constexpr int64_t kMaxK = 21824;  // 6 * 128^2 * K < 2^31, K a multiple of 64
};
template <int V>
struct Tile {
  using S = Scheme<V>;
  static constexpr int kBSlice = S::kN * kKt;
  static constexpr int kABlock = S::kDigits * kASlice;  // bytes per (target tile, chunk)
  static constexpr int kBBlock = S::kDigits * kBSlice;  // bytes per (z tile, chunk)
  static constexpr int kStageBytes = kABlock + kBBlock;
  static constexpr int kShift = 2 * S::kBits * (S::kDigits - 1) - 2 * S::kMant;
  static_assert(S::kDigits * S::kN <= 512, "accumulators exceed TMEM");
  static_assert(S::kN % 16 == 0 && (S::kN / 2) % 8 == 0, "MMA N / epilogue split");
};

__host__ __device__ constexpr int zt_of(int v, int nbasis) {
  return (v == RR_YGEMM_INT8X6 ? Scheme<RR_YGEMM_INT8X6>::kN : Scheme<RR_YGEMM_INT8X7>::kN) /
         nbasis;
}
__host__ __device__ constexpr bool is_i8(int v) {
  return v == RR_YGEMM_INT8X7 || v == RR_YGEMM_INT8X6;
}

// Balanced digits of X = rint(x 2^(mant - e)): kDigits - 1 low digits in
// [-base/2, base/2 - 1] and the leading digit (|a_0| <= 64 for INT8X7,
// <= 127 for INT8X6 under the exponent margin).  One FP64 -> int64
// conversion; the digits are integer shifts and masks.  Digit k of element
// j goes to byte j of plane k.
template <int V>
__device__ __forceinline__ void digits16(const double (&v)[16], int e, unsigned char* dst,
                                         int plane_bytes) {
  using S = Scheme<V>;
  constexpr long long kHalf = 1ll << (S::kBits - 1);
  constexpr long long kMask = (1ll << S::kBits) - 1;
  // 2^(mant - e) as two factors so that neither overflows for tiny columns
  const int sh = S::kMant - e;
  const double f1 = ldexp(1.0, sh / 2), f2 = ldexp(1.0, sh - sh / 2);
  uint32_t w[S::kDigits][4];
#pragma unroll
  for (int k = 0; k < S::kDigits; ++k)
#pragma unroll
    for (int j = 0; j < 4; ++j) w[k][j] = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    long long x = __double2ll_rn((v[j] * f1) * f2);
#pragma unroll
    for (int k = S::kDigits - 1; k >= 1; --k) {
      const long long a = ((x + kHalf) & kMask) - kHalf;
      x = (x - a) >> S::kBits;  // exact: x - a is a multiple of the base
      w[k][j >> 2] |= ((uint32_t)a & 0xFFu) << (8 * (j & 3));
    }
    // the rest is the leading digit: the low digits sum to within about
    // +-base^(digits-1) / 2, so it stays inside int8 (no wrap, which would
    // drop a carry)
    w[0][j >> 2] |= ((uint32_t)x & 0xFFu) << (8 * (j & 3));
  }
#pragma unroll
  for (int k = 0; k < S::kDigits; ++k)
    *reinterpret_cast<uint4*>(dst + k * plane_bytes) = make_uint4(w[k][0], w[k][1], w[k][2], w[k][3]);
}

// G digits: one block per (target tile, chunk), one thread per unit
template <int V>
__global__ void __launch_bounds__(256) slice_g_kernel(const double* __restrict__ g,
                                                      const int* __restrict__ row_exp,
                                                      int64_t npos, int64_t nchunk,
                                                      unsigned char* __restrict__ out) {
  const int64_t tile = blockIdx.x;
  const int64_t c = blockIdx.y;
  const int u = threadIdx.x;  // < kTileM * kNkg
  int r, kg;
  unit_rc(u, kNkg, r, kg);
  const int64_t t = tile * kTileM + r;
  const double* src = g + (c * kKt + kg * 16) * npos + t;
  double v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __ldg(src + (int64_t)j * npos);
  digits16<V>(v, unbias(row_exp[t]), out + (tile * nchunk + c) * Tile<V>::kABlock + u * 16,
              kASlice);
}

// basis digits: one block per (z tile, chunk), one thread per unit
template <int V>
__global__ void __launch_bounds__(Scheme<V>::kN * kNkg) slice_basis_kernel(
    const double* __restrict__ basis, int nz, int64_t pix_stride, int nbasis, int basis_stride,
    const int* __restrict__ col_exp, int64_t nchunk, unsigned char* __restrict__ out) {
  const int zt = zt_of(V, nbasis);
  const int64_t tile = blockIdx.x;
  const int64_t c = blockIdx.y;
  const int u = threadIdx.x;  // < kN * kNkg
  int r, kg;
  unit_rc(u, kNkg, r, kg);
  const int z0 = (int)tile * zt;
  const int nused = min(zt, nz - z0) * nbasis;
  double v[16];
  int e = 0;
  if (r < nused) {
    const int zl = r / nbasis;
    const int i = r - zl * nbasis;
    const int64_t q = c * kKt + kg * 16;
    const double* src = basis + ((int64_t)(z0 + zl) * pix_stride + q) * basis_stride + i;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      v[j] = (q + j < pix_stride) ? __ldg(src + (int64_t)j * basis_stride) : 0.0;
    e = unbias(col_exp[(int64_t)(z0 + zl) * nbasis + i]);
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = 0.0;
  }
  digits16<V>(v, e, out + (tile * nchunk + c) * Tile<V>::kBBlock + u * 16, Tile<V>::kBSlice);
}

struct Params {
  const unsigned char* ga;  // G digits, [npos / 128][nchunk] blocks
  const unsigned char* tb;  // basis digits, [ztiles][nchunk] blocks
  const int* row_exp;
  const int* col_exp;
  double* y;  // [npos][nz][nbasis]
  int64_t npos, nchunk;
  int nz, nbasis, zt;
  int* status;
};

// grid (npos / 128, ztiles), 256 threads: thread 0 streams the digit blocks
// (1-D bulk copies), thread 32 issues the MMAs, all eight warps read TMEM.
template <int V>
__global__ void __launch_bounds__(kThreads, 1) ygemm_kernel(const __grid_constant__ Params p) {
  using S = Scheme<V>;
  using Gm = Tile<V>;
  constexpr int kStages = S::kStages;
  constexpr int kN = S::kN;
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ __align__(8) uint64_t acc_done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  __shared__ int s_rexp[kTileM];
  __shared__ int s_cexp[kN];

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t mt = blockIdx.x;
  const int64_t ztile = blockIdx.y;
  const int z0 = (int)ztile * p.zt;
  const int nused = min(p.zt, p.nz - z0) * p.nbasis;

  if (warp == 0) tmem_alloc(&s_tmem, 512);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&acc_done, 1);
    fence_mbar_init();
    s_fail = 0;
  }
  for (int r = threadIdx.x; r < kTileM; r += kThreads) s_rexp[r] = unbias(p.row_exp[mt * kTileM + r]);
  for (int r = threadIdx.x; r < kN; r += kThreads) {
    const int zl = r / p.nbasis;
    s_cexp[r] = r < nused ? unbias(p.col_exp[(int64_t)(z0 + zl) * p.nbasis + r - zl * p.nbasis]) : 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  if (threadIdx.x == 0) {
    // producer
    for (int64_t c = 0; c < p.nchunk; ++c) {
      const int s = (int)(c % kStages);
      const uint32_t use = (uint32_t)(c / kStages);
      if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1, p.status)) {
        s_fail = 1;
        break;
      }
      unsigned char* st = sm + s * Gm::kStageBytes;
      mbar_arrive_expect_tx(&full[s], Gm::kStageBytes);
      bulk_g2s(st, p.ga + (mt * p.nchunk + c) * Gm::kABlock, Gm::kABlock, &full[s]);
      bulk_g2s(st + Gm::kABlock, p.tb + (ztile * p.nchunk + c) * Gm::kBBlock, Gm::kBBlock,
               &full[s]);
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer: digit products (i, j), i + j = d < digits, into accumulator d
    const uint32_t idesc = instr_desc(kFmt, kN, kTileM);
    for (int64_t c = 0; c < p.nchunk; ++c) {
      const int s = (int)(c % kStages);
      const uint32_t use = (uint32_t)(c / kStages);
      if (!mbar_wait(&full[s], use & 1, p.status)) {
        s_fail = 1;
        break;
      }
      tc_fence_after();
      const uint32_t a0 = smem_u32(sm + s * Gm::kStageBytes);
      const uint32_t b0 = a0 + Gm::kABlock;
#pragma unroll 1
      for (int d = 0; d < S::kDigits; ++d)
#pragma unroll 1
        for (int i = 0; i <= d; ++i) {
          const uint64_t da = smem_desc(a0 + i * kASlice, kSbo);
          const uint64_t db = smem_desc(b0 + (d - i) * Gm::kBSlice, kSbo);
          mma<kI8>(tmem + d * kN, da, db, idesc, (c > 0 || i > 0) ? 1u : 0u);
        }
      mma_commit(&empty[s]);
    }
    mma_commit(&acc_done);
  }
  __syncthreads();
  bool ok = s_fail == 0;
  if (ok) ok = mbar_wait(&acc_done, 0, p.status);
  ok = __syncthreads_and(ok);
  if (ok) {
    tc_fence_after();
    const int lg = warp & 3;     // TMEM lanes 32 lg .. 32 lg + 31
    const int half = warp >> 2;  // column half
    const int row = 32 * lg + lane;
    const int64_t pos = mt * kTileM + row;
    double* yrow = p.y + (pos * p.nz + z0) * p.nbasis;
    const uint32_t tl = tmem + ((uint32_t)(32 * lg) << 16);
    for (int c0 = half * (kN / 2); c0 < (half + 1) * (kN / 2); c0 += 8) {
      double out[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) out[j] = 0.0;
      // X_t X_n = sum_d acc_d base^(2 (digits - 1) - d); smallest terms first
#pragma unroll 1
      for (int d = S::kDigits - 1; d >= 0; --d) {
        uint32_t v[8];
        tmem_ld8(tl + d * kN + c0, v);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 8; ++j) out[j] += ldexp((double)(int)v[j], -S::kBits * d);
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (c0 + j < nused)
          yrow[c0 + j] = ldexp(out[j], s_rexp[row] + s_cexp[c0 + j] + Gm::kShift);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

}  // namespace i8

// ---------------------------------------------------------------------------
// G = R^T W f per target, pixel-major, and the per-target exponent
// ---------------------------------------------------------------------------
struct GParams {
  const double* rw;
  int64_t npix_block;
  rr_segment_desc segs[16];
  int nseg;
  int64_t pix_stride, kpad, npos;
  double* g;
  int* row_exp;
};

// block (32 lanes, 8 pixels); grid (kpad / 8, nblock)
__global__ void __launch_bounds__(256) pack_g_kernel(const __grid_constant__ GParams p) {
  __shared__ int s_e[8][32];
  const int lane = threadIdx.x;
  const int64_t q = (int64_t)blockIdx.x * 8 + threadIdx.y;
  const int64_t b = blockIdx.y;
  double acc = 0.0;
  if (q < p.pix_stride) {
    for (int s = 0; s < p.nseg; ++s) {
      const rr_segment_desc& sd = p.segs[s];
      const int64_t base = q - sd.basis_offset + kHalfBand;
      for (int k = 0; k < kBand; ++k) {
        const int64_t px = base - k;
        if (px < 0 || px >= sd.npix_pad) continue;
        const double* row = p.rw + ((b * p.npix_block + sd.rw_offset + px) * RR_RW) * RR_LANES + lane;
        acc = fma(row[k * RR_LANES], row[kBand * RR_LANES], acc);
      }
    }
  }
  if (q < p.kpad) p.g[q * p.npos + b * RR_LANES + lane] = acc;
  if (p.row_exp) {
    int e = 0;
    if (acc != 0.0) {
      // exponent of |acc| 128/127: max |G| < 127/128 2^e (the digit
      // schemes' margin)
      frexp(fabs(acc) * kExpMargin, &e);
      e += kExpBias;
    }
    s_e[threadIdx.y][lane] = e;
    __syncthreads();
    if (threadIdx.y == 0) {
      int m = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) m = max(m, s_e[j][lane]);
      if (m > 0) atomicMax(p.row_exp + b * RR_LANES + lane, m);
    }
  }
}

// biased exponent of max_q |T[z][q][i]| per (z, i); one block per z, each
// thread keeps the running maxima of its rows (read once, contiguously)
__global__ void __launch_bounds__(256) col_exp_kernel(const double* __restrict__ basis,
                                                      int64_t pix_stride, int nbasis,
                                                      int basis_stride, int* col_exp) {
  __shared__ double s_m[RR_MAX_NBASIS][256];
  const int64_t z = blockIdx.x;
  const double* tz = basis + z * pix_stride * basis_stride;
  double m[RR_MAX_NBASIS];
#pragma unroll
  for (int i = 0; i < RR_MAX_NBASIS; ++i) m[i] = 0.0;
  for (int64_t q = threadIdx.x; q < pix_stride; q += blockDim.x) {
    const double* row = tz + q * basis_stride;
#pragma unroll
    for (int i = 0; i < RR_MAX_NBASIS; ++i)
      if (i < nbasis) m[i] = fmax(m[i], fabs(row[i]));
  }
#pragma unroll
  for (int i = 0; i < RR_MAX_NBASIS; ++i) s_m[i][threadIdx.x] = m[i];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int i = 0; i < nbasis; ++i)
        s_m[i][threadIdx.x] = fmax(s_m[i][threadIdx.x], s_m[i][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x < nbasis) {
    int e = 0;
    const double mx = s_m[threadIdx.x][0];
    if (mx > 0.0) {
      frexp(mx * kExpMargin, &e);
      e += kExpBias;
    }
    col_exp[z * nbasis + threadIdx.x] = e;
  }
}

}  // namespace yg
}  // namespace rr

using namespace rr;

extern "C" int64_t rr_ygemm_kpad(int64_t pix_stride) {
  return ((pix_stride + yg::kKpadAlign - 1) / yg::kKpadAlign) * yg::kKpadAlign;
}

extern "C" int rr_pack_g(const rr_scan_targets* targets, int64_t pix_stride, int64_t kpad,
                         int64_t npos, double* g, int* row_exp, int* status,
                         rr_stream_t stream) {
  (void)status;
  if (!targets || !g || pix_stride < 1 || kpad < pix_stride || kpad % yg::kKpadAlign) return RR_EINVAL;
  if (targets->nseg < 1 || targets->nseg > 16 || !targets->segs) return RR_EINVAL;
  if (npos % yg::kTileM || npos < (int64_t)targets->nblock * RR_LANES) return RR_EINVAL;
  if (!targets->rw || targets->nblock < 0) return RR_EINVAL;
  yg::GParams p;
  p.rw = targets->rw;
  p.npix_block = targets->npix_block;
  p.nseg = targets->nseg;
  for (int s = 0; s < p.nseg; ++s) {
    p.segs[s] = targets->segs[s];
    const rr_segment_desc& sd = p.segs[s];
    if (sd.npix_pad < 0 || sd.rw_offset < 0 || sd.rw_offset + sd.npix_pad > p.npix_block ||
        sd.basis_offset < kHalfBand || sd.basis_offset + sd.npix_pad + kHalfBand > pix_stride)
      return RR_EINVAL;
  }
  p.pix_stride = pix_stride;
  p.kpad = kpad;
  p.npos = npos;
  p.g = g;
  p.row_exp = row_exp;
  cudaStream_t st = (cudaStream_t)stream;
  // positions past the last block stay zero
  RR_CUDA_TRY(cudaMemsetAsync(g, 0, (size_t)kpad * npos * sizeof(double), st));
  if (row_exp) RR_CUDA_TRY(cudaMemsetAsync(row_exp, 0, (size_t)npos * sizeof(int), st));
  if (targets->nblock < 1) return RR_OK;
  dim3 grid((unsigned)(kpad / 8), (unsigned)targets->nblock);
  yg::pack_g_kernel<<<grid, dim3(32, 8), 0, st>>>(p);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_basis_col_exp(const double* basis, int64_t nz, int64_t pix_stride, int nbasis,
                                int basis_stride, int* col_exp, rr_stream_t stream) {
  if (!basis || !col_exp || nz < 0 || pix_stride < 1 || nbasis < 1 || basis_stride < nbasis)
    return RR_EINVAL;
  if (nz == 0) return RR_OK;
  yg::col_exp_kernel<<<(unsigned)nz, 256, 0, (cudaStream_t)stream>>>(basis, pix_stride, nbasis,
                                                                      basis_stride, col_exp);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_ygemm(int variant, const double* g, int64_t npos, int64_t kpad,
                        const double* basis, int64_t nz, int64_t pix_stride, int nbasis,
                        int basis_stride, double* y, int* status, rr_stream_t stream) {
  if (!g || !basis || !y || npos < yg::kTileM || npos % yg::kTileM) return RR_EINVAL;
  if (nz < 0 || nz > INT_MAX || nbasis < 1 || nbasis > RR_MAX_NBASIS || basis_stride < nbasis)
    return RR_EINVAL;
  if (kpad < pix_stride || kpad % yg::kKpadAlign || pix_stride < 1) return RR_EINVAL;
  if (nz == 0) return RR_OK;
  yg::YParams p;
  p.g = g;
  p.basis = basis;
  p.y = y;
  p.npos = npos;
  p.kpad = kpad;
  p.pix_stride = pix_stride;
  p.nz = (int)nz;
  p.nbasis = nbasis;
  p.basis_stride = basis_stride;
  p.status = status;
  cudaStream_t st = (cudaStream_t)stream;
  switch (variant) {
    case RR_YGEMM_BF16X3: return yg::launch_ygemm<RR_YGEMM_BF16X3>(p, st);
    case RR_YGEMM_TF32X3: return yg::launch_ygemm<RR_YGEMM_TF32X3>(p, st);
    default: return RR_EINVAL;  // the INT8 schemes run through rr_ygemm_i8
  }
}

extern "C" int64_t rr_ygemm_i8_g_bytes(int variant, int64_t npos, int64_t kpad) {
  if (!yg::i8::is_i8(variant)) return -1;
  if (npos < 0 || kpad < 0 || npos % yg::kTileM || kpad % yg::i8::kKt) return -1;
  const int64_t ablock = variant == RR_YGEMM_INT8X6 ? yg::i8::Tile<RR_YGEMM_INT8X6>::kABlock
                                                    : yg::i8::Tile<RR_YGEMM_INT8X7>::kABlock;
  return (npos / yg::kTileM) * (kpad / yg::i8::kKt) * ablock;
}

extern "C" int64_t rr_ygemm_i8_basis_bytes(int variant, int64_t nz, int nbasis, int64_t kpad) {
  if (!yg::i8::is_i8(variant)) return -1;
  if (nz < 0 || nbasis < 1 || nbasis > RR_MAX_NBASIS || kpad < 0 || kpad % yg::i8::kKt) return -1;
  const int zt = yg::i8::zt_of(variant, nbasis);
  const int64_t bblock = variant == RR_YGEMM_INT8X6 ? yg::i8::Tile<RR_YGEMM_INT8X6>::kBBlock
                                                    : yg::i8::Tile<RR_YGEMM_INT8X7>::kBBlock;
  return ((nz + zt - 1) / zt) * (kpad / yg::i8::kKt) * bblock;
}

extern "C" int64_t rr_ygemm_i8_max_kpad(int variant) {
  if (variant == RR_YGEMM_INT8X7) return yg::i8::Scheme<RR_YGEMM_INT8X7>::kMaxK;
  if (variant == RR_YGEMM_INT8X6) return yg::i8::Scheme<RR_YGEMM_INT8X6>::kMaxK;
  return -1;
}

extern "C" int rr_slice_g_i8(int variant, const double* g, const int* row_exp, int64_t npos,
                             int64_t kpad, void* g_digits, rr_stream_t stream) {
  if (!yg::i8::is_i8(variant)) return RR_EINVAL;
  if (!g || !row_exp || !g_digits || npos < yg::kTileM || npos % yg::kTileM) return RR_EINVAL;
  if (kpad < yg::kKpadAlign || kpad % yg::kKpadAlign || kpad / yg::i8::kKt > 65535) return RR_EINVAL;
  if ((reinterpret_cast<uintptr_t>(g_digits) & 15) != 0) return RR_EINVAL;
  const int64_t nchunk = kpad / yg::i8::kKt;
  dim3 grid((unsigned)(npos / yg::kTileM), (unsigned)nchunk);
  cudaStream_t st = (cudaStream_t)stream;
  if (variant == RR_YGEMM_INT8X6)
    yg::i8::slice_g_kernel<RR_YGEMM_INT8X6><<<grid, yg::kTileM * yg::i8::kNkg, 0, st>>>(
        g, row_exp, npos, nchunk, (unsigned char*)g_digits);
  else
    yg::i8::slice_g_kernel<RR_YGEMM_INT8X7><<<grid, yg::kTileM * yg::i8::kNkg, 0, st>>>(
        g, row_exp, npos, nchunk, (unsigned char*)g_digits);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

extern "C" int rr_slice_basis_i8(int variant, const double* basis, int64_t nz, int64_t pix_stride,
                                 int nbasis, int basis_stride, int64_t kpad, const int* col_exp,
                                 void* basis_digits, rr_stream_t stream) {
  if (!yg::i8::is_i8(variant)) return RR_EINVAL;
  if (!basis || !col_exp || !basis_digits || nz < 0 || nz > INT_MAX || pix_stride < 1)
    return RR_EINVAL;
  if (nbasis < 1 || nbasis > RR_MAX_NBASIS || basis_stride < nbasis) return RR_EINVAL;
  if (kpad < pix_stride || kpad % yg::kKpadAlign || kpad / yg::i8::kKt > 65535) return RR_EINVAL;
  if ((reinterpret_cast<uintptr_t>(basis_digits) & 15) != 0) return RR_EINVAL;
  if (nz == 0) return RR_OK;
  const int zt = yg::i8::zt_of(variant, nbasis);
  const int64_t nchunk = kpad / yg::i8::kKt;
  dim3 grid((unsigned)((nz + zt - 1) / zt), (unsigned)nchunk);
  cudaStream_t st = (cudaStream_t)stream;
  if (variant == RR_YGEMM_INT8X6)
    yg::i8::slice_basis_kernel<RR_YGEMM_INT8X6>
        <<<grid, yg::i8::Scheme<RR_YGEMM_INT8X6>::kN * yg::i8::kNkg, 0, st>>>(
            basis, (int)nz, pix_stride, nbasis, basis_stride, col_exp, nchunk,
            (unsigned char*)basis_digits);
  else
    yg::i8::slice_basis_kernel<RR_YGEMM_INT8X7>
        <<<grid, yg::i8::Scheme<RR_YGEMM_INT8X7>::kN * yg::i8::kNkg, 0, st>>>(
            basis, (int)nz, pix_stride, nbasis, basis_stride, col_exp, nchunk,
            (unsigned char*)basis_digits);
  RR_CHECK_LAUNCH();
  return RR_OK;
}

namespace rr {
namespace yg {
namespace i8 {
template <int V>
static int launch_ygemm_i8(const Params& p, int64_t npos, cudaStream_t st) {
  const size_t smem = (size_t)Scheme<V>::kStages * Tile<V>::kStageBytes;
  RR_CUDA_TRY(cudaFuncSetAttribute(ygemm_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  dim3 grid((unsigned)(npos / kTileM), (unsigned)((p.nz + p.zt - 1) / p.zt));
  ygemm_kernel<V><<<grid, kThreads, smem, st>>>(p);
  RR_CHECK_LAUNCH();
  return RR_OK;
}
}  // namespace i8
}  // namespace yg
}  // namespace rr

extern "C" int rr_ygemm_i8(int variant, const void* g_digits, const int* row_exp, int64_t npos,
                           int64_t kpad, const void* basis_digits, const int* col_exp, int64_t nz,
                           int nbasis, double* y, int* status, rr_stream_t stream) {
  if (!yg::i8::is_i8(variant)) return RR_EINVAL;
  if (!g_digits || !row_exp || !basis_digits || !col_exp || !y) return RR_EINVAL;
  if (npos < yg::kTileM || npos % yg::kTileM || nz < 0 || nz > INT_MAX) return RR_EINVAL;
  if (nbasis < 1 || nbasis > RR_MAX_NBASIS) return RR_EINVAL;
  if (kpad < yg::kKpadAlign || kpad % yg::kKpadAlign) return RR_EINVAL;
  // exact int32 accumulation: the scheme's pixel limit
  if (kpad > rr_ygemm_i8_max_kpad(variant)) return RR_ENOTSUP;
  if (((reinterpret_cast<uintptr_t>(g_digits) | reinterpret_cast<uintptr_t>(basis_digits)) & 15) != 0)
    return RR_EINVAL;
  if (nz == 0) return RR_OK;
  yg::i8::Params p;
  p.ga = (const unsigned char*)g_digits;
  p.tb = (const unsigned char*)basis_digits;
  p.row_exp = row_exp;
  p.col_exp = col_exp;
  p.y = y;
  p.npos = npos;
  p.nchunk = kpad / yg::i8::kKt;
  p.nz = (int)nz;
  p.nbasis = nbasis;
  p.zt = yg::i8::zt_of(variant, nbasis);
  p.status = status;
  cudaStream_t st = (cudaStream_t)stream;
  if (variant == RR_YGEMM_INT8X6)
    return yg::i8::launch_ygemm_i8<RR_YGEMM_INT8X6>(p, npos, st);
  return yg::i8::launch_ygemm_i8<RR_YGEMM_INT8X7>(p, npos, st);
}
