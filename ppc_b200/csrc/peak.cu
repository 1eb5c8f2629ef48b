// FP32 FMA and SFU throughputs of the device (the denominators of the propagation kernel's
// FP32/SFU issue roofline).  No counterpart in the reference.  Every thread runs 8
// independent chains (FFMA, or reciprocal square roots on the special-function unit) so the
// pipe stays full; the grid fills every SM at 1024 threads per SM.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/ppc_b200.h"

void ppcb_internal_set_error(const std::string& msg);

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_ffma(float* out, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; k++) x[k] = threadIdx.x * 1e-3f + k;
#pragma unroll 16
  for (int i = 0; i < kIters; i++) {
#pragma unroll
    for (int k = 0; k < kChains; k++) x[k] = fmaf(x[k], a, b);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; k++) s += x[k];
  if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

// one reciprocal square root (MUFU.RSQ) and one FADD per link; the FADDs go to the FMA pipe,
// four times faster than the special-function unit
__global__ void __launch_bounds__(256) k_mufu(float* out, float b) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; k++) x[k] = 1.f + threadIdx.x * 1e-3f + k;
#pragma unroll 16
  for (int i = 0; i < kIters; i++) {
#pragma unroll
    for (int k = 0; k < kChains; k++) x[k] = rsqrtf(x[k] + b);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; k++) s += x[k];
  if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

template <class L>
int time_best(int device, int repeats, const char* who, L launch, double* best_ms) {
  std::string tag(who);
  cudaDeviceProp p;
  if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&p, device) != cudaSuccess) {
    ppcb_internal_set_error(tag + ": no such device");
    return PPCB_ECUDA;
  }
  const int blocks = p.multiProcessorCount * 4, threads = 256;
  float* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&out, (size_t)blocks * threads * sizeof(float));
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double best = 1e30;
  for (int r = 0; e == cudaSuccess && r < repeats + 2; r++) {
    cudaEventRecord(e0);
    launch(blocks, threads, out);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float t = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (r >= 2 && t < best) best = t;  // two warm-up launches
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (out) cudaFree(out);
  if (e != cudaSuccess) {
    ppcb_internal_set_error(cudaGetErrorString(e));
    return PPCB_ECUDA;
  }
  *best_ms = best;
  return PPCB_OK;
}

int grid_threads(int device) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return 0;
  return p.multiProcessorCount * 4 * 256;
}

}  // namespace

extern "C" int ppcb_fp32_peak(int device, int repeats, double* tflops, double* ms) {
  if (!tflops || repeats <= 0) { ppcb_internal_set_error("ppcb_fp32_peak: bad argument"); return PPCB_EARG; }
  double best = 0;
  const int r = time_best(device, repeats, "ppcb_fp32_peak",
                          [](int b, int t, float* out) { k_ffma<<<b, t>>>(out, 0.999999f, 1e-6f); }, &best);
  if (r != PPCB_OK) return r;
  const double flops = 2.0 * kChains * kIters * (double)grid_threads(device);
  *tflops = flops / (best * 1e-3) / 1e12;
  if (ms) *ms = best;
  return PPCB_OK;
}

extern "C" int ppcb_sfu_peak(int device, int repeats, double* tops, double* ms) {
  if (!tops || repeats <= 0) { ppcb_internal_set_error("ppcb_sfu_peak: bad argument"); return PPCB_EARG; }
  double best = 0;
  const int r = time_best(device, repeats, "ppcb_sfu_peak",
                          [](int b, int t, float* out) { k_mufu<<<b, t>>>(out, 1e-3f); }, &best);
  if (r != PPCB_OK) return r;
  const double ops = (double)kChains * kIters * (double)grid_threads(device);
  *tops = ops / (best * 1e-3) / 1e12;
  if (ms) *ms = best;
  return PPCB_OK;
}
