// util.cuh -- small streaming kernels: update, conversion, deterministic
// reductions.  All grid-stride loops use 128-bit accesses where the type
// allows; reductions run over a fixed grid so their summation order, and
// hence their result, does not depend on timing.
#pragma once

#include "common.cuh"

namespace gfd {

constexpr int kRedBlocks = 1184;  // 8 per SM on 148 SMs
constexpr int kRedThreads = 256;

// y[i] = a * y[i] + b * x[i]   (mixed types allowed: X may be float)
template <class Y, class X>
__global__ void __launch_bounds__(256) axpby_kernel(Y* __restrict__ y, const X* __restrict__ x,
                                                    double a, double b, long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = Y(a * double(y[i]) + b * double(x[i]));
}

// y[i] = x[i] - c  (background removal; y may alias x)
template <class T>
__global__ void __launch_bounds__(256) sub_const_kernel(T* y, const T* x, double c, long long n) {
  pdl_enter();
  const T cc = T(c);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = x[i] - cc;
}

// y[i] = 0 (a kernel rather than a memset node, so the chain of kernels in
// a captured graph stays programmatic)
template <class T>
__global__ void __launch_bounds__(256) zero_kernel(T* __restrict__ y, long long n) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = T(0);
}

// y[i] = T(x[i])
template <class Y, class X>
__global__ void __launch_bounds__(256) convert_kernel(Y* __restrict__ y, const X* __restrict__ x,
                                                      long long n, Y* __restrict__ seed,
                                                      Y seed_scale) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const Y v = Y(x[i]);
    y[i] = v;
    if (seed) seed[i] = seed_scale * v;
  }
}

// out[b][i] += v[i] * in[b][i] for nb bands of n points (v real).
template <class V>
__global__ void __launch_bounds__(256) add_potential_kernel(V* __restrict__ out,
                                                            const V* __restrict__ in,
                                                            const typename vt<V>::S* __restrict__ v,
                                                            long long n, long long total) {
  pdl_enter();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    V o = out[i];
    madd(o, v[i % n], in[i]);
    out[i] = o;
  }
}

// y[i] *= target / *total (total on the device, computed by an earlier
// kernel on the stream).
static __global__ void __launch_bounds__(256) scale_to_total_kernel(double* __restrict__ y, long long n,
                                                             double target,
                                                             const double* __restrict__ total) {
  pdl_enter();
  const double x = target / *total;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] *= x;
}

// Per-block partial sums of a[i] (SQUARE: a[i]^2), in a fixed order.
template <class T, bool SQUARE>
__global__ void __launch_bounds__(kRedThreads) partial_sum_kernel(const T* __restrict__ a,
                                                                  long long n,
                                                                  double* __restrict__ partials) {
  pdl_enter();
  __shared__ double red[kRedThreads / 32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kRedThreads) {
    double v = double(a[i]);
    s += SQUARE ? v * v : v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kRedThreads / 32; w++) b += red[w];
    partials[blockIdx.x] = b;
  }
}

// out[0] = scale * sum(partials[0..n)), one block, fixed tree order.
static __global__ void __launch_bounds__(kRedThreads) final_sum_kernel(const double* __restrict__ partials,
                                                                int n, double scale,
                                                                double* __restrict__ out) {
  pdl_enter();
  __shared__ double red[kRedThreads];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += kRedThreads) s += partials[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] * scale;
}

// Launch helpers (host).
inline int grid_for(long long n, int threads = 256, int max_blocks = 148 * 16) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return int(b);
}

}  // namespace gfd
