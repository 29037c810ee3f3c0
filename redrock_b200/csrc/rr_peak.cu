// FMA throughput microbenchmark, used as the roofline denominator of the
// FP64 CUDA-core-bound scan.  No counterpart in redrock.
#include "rr_common.cuh"

namespace rr {

template <typename T>
__global__ void fma_peak_kernel(T* out, int iters) {
  T a[8];
  const T b = (T)0.999999, c = (T)1e-7;
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = (T)(threadIdx.x + k);
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == (T)-1) out[0] = s;  // keeps the chains live; never true
}

}  // namespace rr

// FLOPs issued = 2 * 8 * 16 * iters * blocks * 256.  kind 0: FP64, 1: FP32.
extern "C" int rr_fma_peak(int kind, int blocks, int iters, void* out, rr_stream_t stream) {
  if (blocks < 1 || iters < 1 || !out) return RR_EINVAL;
  if (kind == 0)
    rr::fma_peak_kernel<double><<<blocks, 256, 0, (cudaStream_t)stream>>>((double*)out, iters);
  else
    rr::fma_peak_kernel<float><<<blocks, 256, 0, (cudaStream_t)stream>>>((float*)out, iters);
  if (cudaGetLastError() != cudaSuccess) return RR_ECUDA;
  return RR_OK;
}
