// FP64 direct summation (the error oracle of every result) and the FMA
// throughput probe used as the roofline denominator of the walk.
//
// The pair force is that of fortran/direct_forces.f90:24-26 and
// fortran/api3d.f90:54-59: f = G m_a m_b / (dist * dist2), dist2 = |d|^2 + eps^2,
// summed per target in source order (the Fortran pair loop with Newton's third
// law accumulates each target's terms in the same source order).  Sources are
// staged through shared memory in tiles of 256.
#include <math.h>

#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int kDirThreads = 256;

__global__ void __launch_bounds__(kDirThreads)
direct_kernel(const double *__restrict__ m, const double *__restrict__ x,
              const double *__restrict__ y, const double *__restrict__ z, int64_t n,
              const int64_t *__restrict__ targets, int64_t nt, double G, double eps2,
              int out_kind, double *__restrict__ out) {
  __shared__ double4 tile[kDirThreads];
  for (int64_t base = (int64_t)blockIdx.x * kDirThreads; base < nt;
       base += (int64_t)gridDim.x * kDirThreads) {
    const int64_t k = base + threadIdx.x;
    const bool valid = k < nt;
    int64_t a = valid ? (targets ? targets[k] : k) : 0;
    const bool bad = a < 0 || a >= n;  // invalid target index: NaN result
    if (bad) a = 0;
    const double xa = x[a], ya = y[a], za = z[a];
    const double ma = out_kind == 1 ? 1.0 : m[a];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int64_t src = 0; src < n; src += kDirThreads) {
      const int64_t j = src + threadIdx.x;
      tile[threadIdx.x] = j < n ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
      __syncthreads();
      const int cnt = (int)bh_min64(kDirThreads, n - src);
      for (int jj = 0; jj < cnt; ++jj) {
        if (src + jj == a) continue;
        const double4 s = tile[jj];
        const double dx = s.x - xa, dy = s.y - ya, dz = s.z - za;
        const double dist2 = dx * dx + dy * dy + dz * dz + eps2;
        const double dist = sqrt(dist2);
        const double f = G * ma * s.w / (dist * dist2);
        fx = fx + f * dx; fy = fy + f * dy; fz = fz + f * dz;
      }
      __syncthreads();
    }
    if (bad) fx = fy = fz = nan("");
    if (valid) { out[k] = fx; out[nt + k] = fy; out[2 * nt + k] = fz; }
  }
}

constexpr int kProbeIters = 4096;

template <typename T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T *sink, T a, T b) {
  T v0 = (T)threadIdx.x, v1 = v0 + 1, v2 = v0 + 2, v3 = v0 + 3, v4 = v0 + 4, v5 = v0 + 5,
    v6 = v0 + 6, v7 = v0 + 7;
#pragma unroll 16
  for (int i = 0; i < kProbeIters; ++i) {
    v0 = fma(v0, a, b); v1 = fma(v1, a, b); v2 = fma(v2, a, b); v3 = fma(v3, a, b);
    v4 = fma(v4, a, b); v5 = fma(v5, a, b); v6 = fma(v6, a, b); v7 = fma(v7, a, b);
  }
  T s = v0 + v1 + v2 + v3 + v4 + v5 + v6 + v7;
  if (s == (T)12345.678) sink[threadIdx.x] = s;  // keeps the chains alive
}

// The same chains with paired FP32 instructions (two FMAs per instruction).
__global__ void __launch_bounds__(256) fma2_probe_kernel(float *sink, float a, float b) {
  const float2 av = make_float2(a, a), bv = make_float2(b, b);
  const float f = (float)threadIdx.x;
  float2 v0 = make_float2(f, f + 1), v1 = make_float2(f + 2, f + 3), v2 = make_float2(f + 4, f + 5),
         v3 = make_float2(f + 6, f + 7);
#pragma unroll 16
  for (int i = 0; i < kProbeIters; ++i) {
    v0 = __ffma2_rn(v0, av, bv); v1 = __ffma2_rn(v1, av, bv);
    v2 = __ffma2_rn(v2, av, bv); v3 = __ffma2_rn(v3, av, bv);
  }
  const float s = v0.x + v0.y + v1.x + v1.y + v2.x + v2.y + v3.x + v3.y;
  if (s == 12345.678f) sink[threadIdx.x] = s;
}

}  // namespace

void launch_direct(const double *m, const double *x, const double *y, const double *z, int64_t n,
                   const int64_t *targets, int64_t ntargets, double G, double eps2, int out_kind,
                   double *out, cudaStream_t s) {
  const int64_t nt = targets ? ntargets : n;
  const int grid = grid_for(nt, kDirThreads, 148 * 64);
  direct_kernel<<<grid, kDirThreads, 0, s>>>(m, x, y, z, n, targets, nt, G, eps2, out_kind, out);
}

// GFLOP/s of FMA (2 flops each) on independent chains: [0] FP32, [1] FP64,
// [2] FP32 issued as paired (f32x2) instructions.
int probe_fma(double *gflops2) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256;
  float *fs = nullptr;
  double *ds = nullptr;
  if (cudaMalloc(&fs, threads * sizeof(float)) != cudaSuccess) return 1;
  if (cudaMalloc(&ds, threads * sizeof(double)) != cudaSuccess) { cudaFree(fs); return 1; }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const double flops = 2.0 * 8.0 * kProbeIters * (double)blocks * threads;
  for (int which = 0; which < 3; ++which) {
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
      cudaEventRecord(e0);
      if (which == 0) fma_probe_kernel<float><<<blocks, threads>>>(fs, 0.999f, 1e-3f);
      else if (which == 1) fma_probe_kernel<double><<<blocks, threads>>>(ds, 0.999, 1e-3);
      else fma2_probe_kernel<<<blocks, threads>>>(fs, 0.999f, 1e-3f);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms < best) best = ms;
    }
    gflops2[which] = flops / (best * 1e-3) / 1e9;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(fs);
  cudaFree(ds);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace bh
