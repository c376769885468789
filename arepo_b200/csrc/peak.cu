// peak.cu -- CUDA-core fused multiply-add throughput (FP32 or FP64) of the
// current GPU: the denominator of the walk's roofline.  Each thread runs
// eight independent FMA chains in registers; nothing touches memory until the
// end.  One launch of 148 x 8 blocks of 256 threads, timed with CUDA events.
#include "internal.h"

namespace
{
template <class T>
__global__ void __launch_bounds__(256) k_fma(T seed, int iters, T *out)
{
  T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const T m = (T)0.999999, c = (T)1e-7;
  for(int i = 0; i < iters; i++)
    {
#pragma unroll
      for(int u = 0; u < 16; u++)
        {
          a0 = a0 * m + c;
          a1 = a1 * m + c;
          a2 = a2 * m + c;
          a3 = a3 * m + c;
          a4 = a4 * m + c;
          a5 = a5 * m + c;
          a6 = a6 * m + c;
          a7 = a7 * m + c;
        }
    }
  T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if(s == (T)-12345.0)  // never true; keeps the chains alive
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class T>
int run(int device, int iters, double *tflops)
{
  cudaSetDevice(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  T *out = nullptr;
  const int blocks = sms * 8;
  if(cudaMalloc(&out, (size_t)blocks * 256 * sizeof(T)) != cudaSuccess)
    return GPUGRAV_ERR_OOM;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_fma<T><<<blocks, 256>>>((T)1, iters / 4, out);  // warm-up
  cudaEventRecord(a);
  k_fma<T><<<blocks, 256>>>((T)1, iters, out);
  cudaEventRecord(b);
  cudaError_t e = cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if(e != cudaSuccess || ms <= 0)
    return GPUGRAV_ERR_CUDA;
  double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * 256.0;
  *tflops      = flops / (ms * 1e-3) / 1e12;
  return GPUGRAV_OK;
}
}  // namespace

extern "C" int32_t gpugrav_measure_fma_peak(int32_t device, int32_t precision, double *tflops)
{
  if(!tflops)
    return GPUGRAV_ERR_INVALID;
  int prev = 0;
  cudaGetDevice(&prev);
  int s = (precision == GPUGRAV_PREC_FP32) ? run<float>(device, 20000, tflops) : run<double>(device, 4000, tflops);
  cudaSetDevice(prev);
  return s;
}
