// FP32 FMA throughput probe: the roofline denominator of the Debye pair
// kernel (FP32-pipe bound).  Eight independent register-resident FFMA chains
// per thread on every SM; FLOP counted as 2 per FMA.
#include <cuda_runtime.h>

#include <algorithm>

#include "engine.hpp"

namespace crab {
namespace {
constexpr int kIter = 4096;
__global__ void k_ffma_peak(float* out, float m, float c, int outer) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 1e-3f + k;
  for (int o = 0; o < outer; ++o)
    for (int it = 0; it < kIter; ++it) {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
    }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

double measure_fp32_peak(crab_ctx* ctx, double target_ms) {
  const int threads = 256, blocks = ctx->sm_count * 8;
  float* out = (float*)ctx->dev("probe.out", (size_t)threads * blocks * sizeof(float));
  cudaStream_t s = ctx->stream;
  // warm up and calibrate the loop count to roughly target_ms
  k_ffma_peak<<<blocks, threads, 0, s>>>(out, 0.9999f, 1e-4f, 1);
  CRAB_CUDA_CHECK(cudaGetLastError());
  CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_start, s));
  k_ffma_peak<<<blocks, threads, 0, s>>>(out, 0.9999f, 1e-4f, 1);
  CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_stop, s));
  CRAB_CUDA_CHECK(cudaEventSynchronize(ctx->ev_stop));
  float ms1 = 0.0f;
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&ms1, ctx->ev_start, ctx->ev_stop));
  const int outer = std::max(1, std::min(1000, (int)(target_ms / std::max(ms1, 1e-3f))));
  double best = 0.0;
  for (int rep = 0; rep < 3; ++rep) {
    CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_start, s));
    k_ffma_peak<<<blocks, threads, 0, s>>>(out, 0.9999f, 1e-4f, outer);
    CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_stop, s));
    CRAB_CUDA_CHECK(cudaEventSynchronize(ctx->ev_stop));
    float ms = 0.0f;
    CRAB_CUDA_CHECK(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
    const double flop = 2.0 * 8.0 * kIter * (double)outer * threads * (double)blocks;
    best = std::max(best, flop / (ms * 1e-3) / 1e12);
  }
  ctx->launches += 5;
  return best;
}

}  // namespace crab
