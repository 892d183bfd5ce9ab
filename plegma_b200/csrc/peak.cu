// FP64 FMA rate of the device: the roofline denominator of the plain form's
// FP64 kernels (site contraction and direct phase sum).  Each thread runs
// kChains independent FMA chains (enough to cover the FP64 pipe's latency),
// every SM holds several CTAs, and the time of kIters iterations is taken
// with CUDA events on the context's stream.
#include "ctx.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_fp64_fma_rate(double seed, double* sink) {
  double a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) a[i] = seed + threadIdx.x + i;
  const double m = 1.0 - 1e-12, c = 1e-13;
#pragma unroll 4
  for (int it = 0; it < kIters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i++) a[i] = fma(a[i], m, c);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < kChains; i++) s += a[i];
  if (s == -1.0) *sink = s;  // never true: keeps the chains live
}

}  // namespace

extern "C" p2_status p2_measure_fp64_rate(p2_ctx* c, double* tflops, double* ms) {
  if (!c || !tflops) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  const int blocks = c->nsm * 8, threads = 256;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  P2_TRY(c, cudaEventCreate(&e0), "event");
  cudaError_t e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return c->cuda(e, "event");
  }
  float best = 0.f;
  // warm-up launch, then the best of five
  for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {
    e = cudaEventRecord(e0, c->stream);
    if (e == cudaSuccess) {
      k_fp64_fma_rate<<<blocks, threads, 0, c->stream>>>(1.0 + rep, nullptr);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (e == cudaSuccess && rep > 0 && (best == 0.f || t < best)) best = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return c->cuda(e, "FP64 rate kernel");
  const double flop = 2.0 * kChains * (double)kIters * blocks * threads;
  *tflops = flop / (best * 1e-3) / 1e12;
  if (ms) *ms = best;
  return P2_OK;
}
