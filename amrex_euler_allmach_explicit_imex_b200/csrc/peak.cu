// FP64 FMA throughput of the GPU: the denominator of the explicit step's FP64
// roofline.  The step is a stencil with about 385 FP64 flops per cell, so
// beside its HBM fraction the bench reports its fraction of this number,
// measured on the same device rather than taken from a datasheet.
#include <cuda_runtime.h>

#include "ecg.h"

namespace {

constexpr int kChains = 8;   // independent FMA chains per thread
constexpr int kThreads = 256;

// Every thread runs kChains dependent chains x <- x * a + b for `iters`
// rounds; the chains are independent, so the FP64 pipe, not latency, bounds
// the rate.  The sum is stored so that no chain is dead code.
__global__ void __launch_bounds__(kThreads) fp64_fma_kernel(double* __restrict__ out, int iters, double a, double b)
{
  double x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = 1.0 + 1.0e-3 * (threadIdx.x + k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  out[blockIdx.x * kThreads + threadIdx.x] = s;
}

}  // namespace

extern "C" ecg_status ecg_measure_fp64_peak(int32_t device, double* tflops)
{
  if (!tflops) return ECG_ERR_BAD_ARG;
  *tflops = 0.0;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return ECG_ERR_NO_DEVICE;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return ECG_ERR_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = (sms > 0 ? sms : 1) * 8;  // 64 warps per SM
  const int iters = 4096;
  double* out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ecg_status st = ECG_OK;
  if (cudaMalloc(&out, sizeof(double) * blocks * kThreads) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    st = ECG_ERR_CUDA;
  } else {
    float best = 0.0f;
    for (int rep = 0; rep < 6 && st == ECG_OK; ++rep) {  // the first launch is a warm-up
      cudaEventRecord(e0, s);
      fp64_fma_kernel<<<blocks, kThreads, 0, s>>>(out, iters, 1.0 - 1.0e-9, 1.0e-9);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        st = ECG_ERR_CUDA;
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    if (st == ECG_OK && best > 0.0f) {
      const double flops = 2.0 * kChains * static_cast<double>(iters) * blocks * kThreads;
      *tflops = flops / (best * 1.0e-3) / 1.0e12;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (out) cudaFree(out);
  cudaSetDevice(prev);
  return st;
}
