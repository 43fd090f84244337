// Throughput microbenchmarks of the two units that bound the compositing kernels: the FP32
// pipe (fused multiply-add) and the special-function unit (MUFU ex2, the fast exp's core,
// and rcp). They give the denominators of the compositing stages' roofline, which the
// copy-bandwidth and GEMM peaks do not cover.
//
// Each thread runs kChains independent dependency chains so that every scheduler always
// has an instruction ready; the grid is 8 blocks of 256 threads per SM. The kernel is
// timed with CUDA events on the context's stream around one launch after one untimed
// launch, so the figure is at whatever SM clock the GPU runs at; callers sample the clock
// beside it.
#include "common.cuh"
#include "kernels.cuh"

namespace splat {

namespace {
constexpr int kChains = 8;
constexpr int kPeakThreads = 256;

__global__ void __launch_bounds__(kPeakThreads) peak_fma_kernel(uint32_t iters, float b, float c,
                                                                 float* __restrict__ sink) {
  float a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) a[i] = (float)(threadIdx.x + i) * 1e-3f;
  for (uint32_t k = 0; k < iters; k++) {
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
      for (int i = 0; i < kChains; i++) a[i] = __fmaf_rn(a[i], b, c);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kChains; i++) s += a[i];
  if (s == 1234.5f) sink[threadIdx.x] = s;  // keeps the chains live; never true for these inputs
}

// ex2.approx of a negated argument keeps every value in (0, 1]: x -> 2^-x maps (0, 1] into
// [0.5, 1). The negation folds into the instruction's operand.
__global__ void __launch_bounds__(kPeakThreads) peak_ex2_kernel(uint32_t iters, float* __restrict__ sink) {
  float a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) a[i] = 0.5f + (float)((threadIdx.x + i) & 7) * 0.01f;
  for (uint32_t k = 0; k < iters; k++) {
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
      for (int i = 0; i < kChains; i++) asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(a[i]) : "f"(-a[i]));
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kChains; i++) s += a[i];
  if (s == 1234.5f) sink[threadIdx.x] = s;
}
}  // namespace

// unit 0: FP32 fused multiply-adds (2 FLOP each); unit 1: MUFU ex2 operations.
Status launch_diag_peak(Ctx* c, int unit, double* ops_per_s, float* ms_out) {
  float* sink = nullptr;
  SPLAT_TRY(arena_reserve(c, kPeakThreads * 4, (void**)&sink));
  const uint32_t blocks = (uint32_t)c->sm_count * 8;
  // About 2 ms per launch at the nominal peaks.
  const uint32_t iters = unit == 0 ? 8192 : 1024;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SPLAT_CUDA(cudaEventCreate(&e0));
  Status s = cuda_status(cudaEventCreate(&e1), "cudaEventCreate");
  for (int rep = 0; rep < 2 && s.good(); rep++) {
    if (rep == 1) s = cuda_status(cudaEventRecord(e0, c->stream), "cudaEventRecord");
    if (!s.good()) break;
    if (unit == 0)
      peak_fma_kernel<<<blocks, kPeakThreads, 0, c->stream>>>(iters, 0.999f, 1e-4f, sink);
    else
      peak_ex2_kernel<<<blocks, kPeakThreads, 0, c->stream>>>(iters, sink);
    c->launches.count++;
    s = cuda_status(cudaGetLastError(), unit == 0 ? "peak_fma_kernel" : "peak_ex2_kernel");
  }
  if (s.good()) s = cuda_status(cudaEventRecord(e1, c->stream), "cudaEventRecord");
  if (s.good()) s = cuda_status(cudaEventSynchronize(e1), "cudaEventSynchronize");
  float ms = 0.0f;
  if (s.good()) s = cuda_status(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
  cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!s.good()) return s;
  const double ops = (double)blocks * kPeakThreads * iters * 16 * kChains;
  *ops_per_s = (unit == 0 ? 2.0 * ops : ops) / (ms * 1e-3);
  *ms_out = ms;
  return Status::ok();
}

}  // namespace splat
