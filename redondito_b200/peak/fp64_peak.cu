// fp64_peak.cu -- measures this GPU's FP64 tensor-core (DMMA) throughput.
//
// The HBM and bf16 peaks of the roofline come from a copy and a cuBLAS
// GEMM; there is no FP64 figure beside them, so the FP64 Legendre kernels
// are judged against this number: every SM runs independent
// mma.sync.m16n8k8.f64 chains on registers (no memory traffic) and the
// result is reported in TFLOP/s on stdout as one JSON line.
#include <cstdio>
#include <cuda_runtime.h>

__global__ void dmma_chain(double* out, int iters) {
  double c[8][4];
  double a0 = threadIdx.x * 1e-9, a1 = 1e-9, a2 = 2e-9, a3 = 3e-9, b0 = 1e-9, b1 = 2e-9;
  for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = c[i][2] = c[i][3] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
          "{%0,%1,%2,%3};"
          : "+d"(c[i][0]), "+d"(c[i][1]), "+d"(c[i][2]), "+d"(c[i][3])
          : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
  }
  double s = 0.0;
  for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1] + c[i][2] + c[i][3];
  if (s == 1234.5) out[0] = s;  // keeps the chains live; never true
}

int main() {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return 1;
  const int threads = 256, blocks = sms * 4, iters = 8192;
  dmma_chain<<<blocks, threads>>>(d, 64);
  cudaDeviceSynchronize();
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(a);
    dmma_chain<<<blocks, threads>>>(d, iters);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) best = ms;
  }
  cudaError_t e = cudaGetLastError();
  double flops = (double)blocks * threads / 32 * iters * 8 * 2.0 * 16 * 8 * 8;
  printf("{\"fp64_tensor_tflops\": %.3f, \"sms\": %d, \"status\": \"%s\"}\n", flops / (best * 1e-3) / 1e12,
         sms, cudaGetErrorString(e));
  cudaFree(d);
  return e == cudaSuccess ? 0 : 1;
}
