// peaks.cu -- FP64 throughput calibration of the current GPU.
//
// The roofline of the batched GEMM is the FP64 tensor-core rate.  This
// measures it (and the FP64 FMA rate) with register-only loops of
// mma.sync.m16n8k8.f64 / fma.rn.f64, 8 independent accumulator chains per
// warp, 2 CTAs x 8 warps per SM, timed with CUDA events.
#include <cuda_runtime.h>

#include "ctx.h"

namespace {

__global__ void k_peak_dmma(double* out, int iters) {
  double c[8][4];
  for (int j = 0; j < 8; ++j)
    for (int v = 0; v < 4; ++v) c[j][v] = 0.0;
  const double a0 = threadIdx.x * 1e-3, a1 = 1.0, a2 = 2.0, a3 = 3.0, b0 = 0.5, b1 = 0.25;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
          "{%8,%9}, {%0,%1,%2,%3};"
          : "+d"(c[j][0]), "+d"(c[j][1]), "+d"(c[j][2]), "+d"(c[j][3])
          : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
  }
  double s = 0.0;
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1] + c[j][2] + c[j][3];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_peak_dfma(double* out, int iters) {
  double c[16];
  for (int j = 0; j < 16; ++j) c[j] = threadIdx.x * j;
  const double a = 1.000001, b = 1e-9;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 0; j < 16; ++j) c[j] = fma(c[j], a, b);
  }
  double s = 0.0;
  for (int j = 0; j < 16; ++j) s += c[j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int mpc_probe_fp64_peak(int device, double* dmma_tflops, double* dfma_tflops) {
  if (!dmma_tflops || !dfma_tflops) return mpc_fail(MPC_ERR_ARG, "null output");
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int grid = 2 * sms, block = 256;
  double* out = nullptr;
  CK(cudaMalloc(&out, sizeof(double) * grid * block));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 4000;
  float ms = 0.f;
  k_peak_dmma<<<grid, block>>>(out, 10);
  cudaEventRecord(e0);
  k_peak_dmma<<<grid, block>>>(out, iters);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  *dmma_tflops = (double)grid * (block / 32) * iters * 8 * 2048.0 / (ms * 1e-3) / 1e12;
  k_peak_dfma<<<grid, block>>>(out, 10);
  cudaEventRecord(e0);
  k_peak_dfma<<<grid, block>>>(out, 4 * iters);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  *dfma_tflops = (double)grid * block * 4.0 * iters * 16 * 2.0 / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const cudaError_t err = cudaGetLastError();
  cudaFree(out);
  if (err != cudaSuccess) return mpc_fail(MPC_ERR_CUDA, "peak probe: %s", cudaGetErrorString(err));
  return MPC_OK;
}
