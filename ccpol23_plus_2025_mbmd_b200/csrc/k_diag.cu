// k_diag.cu -- measured FMA-pipe peak of the device (diagnostics for the roofline).
//
// Every thread runs 8 independent fused multiply-add chains held in registers, so the
// kernel is bound by the FMA pipe alone; 2 flops per FMA.
#include <cuda_runtime.h>

#include <string>

#include "ccp_internal.h"

namespace {

template <typename T>
__global__ void k_fma_chain(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k) * (T)1e-3;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == (T)-1.2345) out[0] = s;  // keeps the chains alive; never true
}

// Special-function pipe: 8 independent chains x = exp(-x) through the hardware
// exponential (__expf: one MUFU ex2 and one multiply per step), values staying in (0, 1].
__global__ void k_mufu_chain(float *out, int iters) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = __expf(-x[k]);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == -1.2345f) out[0] = s;  // keeps the chains alive; never true
}

template <typename T, bool kMufu = false>
int run(int device, double *tflops) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CCP_ERR_CUDA;
  T *out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return CCP_ERR_CUDA;
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 2048;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 1e30;
  for (int rep = 0; rep < 6; rep++) {
    cudaEventRecord(e0);
    if (kMufu)
      k_mufu_chain<<<blocks, threads>>>(reinterpret_cast<float *>(out), iters);
    else
      k_fma_chain<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return CCP_ERR_CUDA;
  // 2 flops per FMA; 1 op per special-function evaluation
  const double flops = (kMufu ? 1.0 : 2.0) * 8.0 * 16.0 * (double)iters * threads * (double)blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return CCP_OK;
}

}  // namespace

extern "C" int ccp_device_fma_peak(int device, int precision, double *tflops) {
  if (!tflops) return CCP_ERR_BAD_INPUT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    ccp::set_error("no such CUDA device");
    return CCP_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return CCP_ERR_CUDA;
  return precision == CCP_FP64 ? run<double>(device, tflops) : run<float>(device, tflops);
}

extern "C" int ccp_device_mufu_peak(int device, double *tops) {
  if (!tops) return CCP_ERR_BAD_INPUT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    ccp::set_error("no such CUDA device");
    return CCP_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return CCP_ERR_CUDA;
  return run<float, true>(device, tops);
}
