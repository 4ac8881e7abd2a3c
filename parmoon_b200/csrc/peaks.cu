// Throughput probes of the arithmetic paths the kernels use: FP64 FMA on the
// CUDA cores, FP64 mma.sync m8n8k4 (DMMA: the assembly's contraction) and
// BF16 mma.sync m16n8k16 with FP32 accumulators (the stencil network's
// forward).  Registers only, 8 blocks of 256 threads per SM, each kernel timed
// once after a warm-up launch with CUDA events on the caller's current device.
#include "pmg_internal.h"

namespace pmg {

constexpr int PEAK_ITERS = 4096;

__global__ void __launch_bounds__(256) k_peak_fma(double *out, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < PEAK_ITERS; i++)
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_peak_dmma(double *out, double a) {
  const double A = a + threadIdx.x * 1e-6, B = a - threadIdx.x * 1e-6;
  double c[4][2] = {};
  for (int i = 0; i < PEAK_ITERS; i++)
#pragma unroll
    for (int k = 0; k < 4; k++)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[k][0]), "+d"(c[k][1])
                   : "d"(A), "d"(B));
  double s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) s += c[k][0] + c[k][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_peak_hmma(double *out, unsigned a) {
  const unsigned A0 = a ^ threadIdx.x, A1 = a + threadIdx.x, B0 = a - threadIdx.x;
  float c[4][4] = {};
  for (int i = 0; i < PEAK_ITERS; i++)
#pragma unroll
    for (int k = 0; k < 4; k++)
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
          "{%0,%1,%2,%3};"
          : "+f"(c[k][0]), "+f"(c[k][1]), "+f"(c[k][2]), "+f"(c[k][3])
          : "r"(A0), "r"(A1), "r"(A0), "r"(A1), "r"(B0), "r"(B0));
  float s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) s += c[k][0] + c[k][1] + c[k][2] + c[k][3];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace pmg

using namespace pmg;

extern "C" int pmg_measure_peaks(double *fp64_fma_tflops, double *fp64_dmma_tflops, double *bf16_mma_sync_tflops) {
  if (!fp64_fma_tflops || !fp64_dmma_tflops || !bf16_mma_sync_tflops) {
    set_error("pmg_measure_peaks: bad arguments");
    return PMG_ERR_ARG;
  }
  int dev = 0, sms = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256;
  const double nthreads = (double)blocks * threads, nwarps = nthreads / 32;
  DBuf<double> out;
  PMG_TRY(out.alloc((size_t)blocks * threads));
  cudaEvent_t e0, e1;
  PMG_CUDA(cudaEventCreate(&e0));
  PMG_CUDA(cudaEventCreate(&e1));
  float ms[3] = {0, 0, 0};
  for (int k = 0; k < 3; k++) {
    for (int rep = 0; rep < 2; rep++) {  // the first launch warms up
      if (rep == 1) PMG_CUDA(cudaEventRecord(e0, 0));
      if (k == 0) k_peak_fma<<<blocks, threads>>>(out.p, 0.999, 1e-3);
      if (k == 1) k_peak_dmma<<<blocks, threads>>>(out.p, 0.5);
      if (k == 2) k_peak_hmma<<<blocks, threads>>>(out.p, 0x3f803f80u);
      count_launches(1);
    }
    PMG_CUDA(cudaEventRecord(e1, 0));
    PMG_CUDA(cudaEventSynchronize(e1));
    PMG_CUDA(cudaEventElapsedTime(&ms[k], e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PMG_CUDA(cudaGetLastError());
  *fp64_fma_tflops = 2.0 * 8 * PEAK_ITERS * nthreads / (ms[0] * 1e9);
  *fp64_dmma_tflops = 2.0 * 8 * 8 * 4 * 4 * PEAK_ITERS * nwarps / (ms[1] * 1e9);
  *bf16_mma_sync_tflops = 2.0 * 16 * 8 * 16 * 4 * PEAK_ITERS * nwarps / (ms[2] * 1e9);
  return PMG_OK;
}
