// capi.cu -- error reporting, device queries, reductions and small streaming
// launches of libgpawfd.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "internal.h"
#include "util.cuh"

namespace gfd {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return GFD_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return set_error(GFD_ENOMEM, std::string(what) + ": " + cudaGetErrorString(e));
  }
  return set_error(GFD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_launch(const char* what) { return check_cuda(cudaGetLastError(), what); }

// Device allocations of the library go through dev_malloc.  A host-side
// fault hook (gfd_test_fail_alloc) can make the n-th next allocation fail as
// cudaMalloc would when memory is exhausted, without touching the device.
static std::mutex g_alloc_mu;
static long long g_fail_countdown = 0;  // 0: no failure planned

int dev_malloc(void** p, size_t bytes, const char* what) {
  {
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    if (g_fail_countdown > 0 && --g_fail_countdown == 0) {
      *p = nullptr;
      return set_error(GFD_ENOMEM, std::string(what) + ": out of memory (planned failure)");
    }
  }
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(e == cudaErrorMemoryAllocation ? GFD_ENOMEM : GFD_ECUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
  }
  return GFD_OK;
}

// Programmatic dependent launch is opt-in (GFD_PDL=1): in the Poisson solve
// graph, whose kernels are short, starting dependents early cost 3% of
// solves/s; the streaming kernels neither gain nor lose.
bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("GFD_PDL");
    return e && e[0] == '1';
  }();
  return on;
}

// Grids up to 300000 points (all bands) use the one-thread-per-point
// kernels, whose whole grid is in flight at once; larger ones the marching
// kernels.  GFD_DIRECT_MAX in the environment overrides the limit.
long long direct_max_points() {
  static const long long v = [] {
    const char* e = getenv("GFD_DIRECT_MAX");
    return e ? atoll(e) : 300000LL;
  }();
  return v;
}

bool split_enabled() {
  static const bool on = [] {
    const char* e = getenv("GFD_SPLIT");
    return !(e && e[0] == '0');
  }();
  return on;
}

int march_ctas_per_sm() {
  static const int v = [] {
    const char* e = getenv("GFD_MARCH_CTAS_PER_SM");
    const int x = e ? atoi(e) : 4;
    return x < 1 ? 1 : (x > 64 ? 64 : x);
  }();
  return v;
}

int zero_launch(int dtype, void* y, int64_t n, cudaStream_t s) {
  const int blocks = grid_for(n);
  if (dtype == GFD_FLOAT64)
    launch_k(zero_kernel<double>, blocks, 256, 0, s, static_cast<double*>(y), (long long)n);
  else if (dtype == GFD_FLOAT32)
    launch_k(zero_kernel<float>, blocks, 256, 0, s, static_cast<float*>(y), (long long)n);
  else
    return set_error(GFD_EINVAL, "zero: unsupported dtype");
  return check_launch("zero_kernel");
}

int num_sms() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cache[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

int reduce_launch(int dtype, const void* a, int64_t n, bool square, double scale,
                  double* partials, double* result, cudaStream_t s) {
  if (dtype == GFD_FLOAT64) {
    if (square)
      launch_k(partial_sum_kernel<double, true>, kRedBlocks, kRedThreads, 0, s, 
          static_cast<const double*>(a), n, partials);
    else
      launch_k(partial_sum_kernel<double, false>, kRedBlocks, kRedThreads, 0, s, 
          static_cast<const double*>(a), n, partials);
  } else if (dtype == GFD_FLOAT32) {
    if (square)
      launch_k(partial_sum_kernel<float, true>, kRedBlocks, kRedThreads, 0, s, 
          static_cast<const float*>(a), n, partials);
    else
      launch_k(partial_sum_kernel<float, false>, kRedBlocks, kRedThreads, 0, s, 
          static_cast<const float*>(a), n, partials);
  } else {
    return set_error(GFD_EINVAL, "reductions need a real dtype");
  }
  launch_k(final_sum_kernel, 1, kRedThreads, 0, s, partials, kRedBlocks, scale, result);
  return check_launch("partial_sum_kernel");
}

int final_sum_launch(const double* partials, int n, double scale, double* result,
                     cudaStream_t s) {
  launch_k(final_sum_kernel, 1, kRedThreads, 0, s, partials, n, scale, result);
  return check_launch("final_sum_kernel");
}

int axpby_launch(int ydtype, void* y, int xdtype, const void* x, double a, double b, int64_t n,
                 cudaStream_t s) {
  const int blocks = grid_for(n);
  if (ydtype == GFD_FLOAT64 && xdtype == GFD_FLOAT64)
    launch_k(axpby_kernel<double, double>, blocks, 256, 0, s, static_cast<double*>(y),
                                                        static_cast<const double*>(x), a, b, n);
  else if (ydtype == GFD_FLOAT64 && xdtype == GFD_FLOAT32)
    launch_k(axpby_kernel<double, float>, blocks, 256, 0, s, static_cast<double*>(y),
                                                       static_cast<const float*>(x), a, b, n);
  else if (ydtype == GFD_FLOAT32 && xdtype == GFD_FLOAT32)
    launch_k(axpby_kernel<float, float>, blocks, 256, 0, s, static_cast<float*>(y),
                                                      static_cast<const float*>(x), a, b, n);
  else
    return set_error(GFD_EINVAL, "axpby: unsupported dtype pair");
  return check_launch("axpby_kernel");
}

int sub_const_launch(int dtype, void* y, const void* x, double c, int64_t n, cudaStream_t s) {
  const int blocks = grid_for(n);
  if (dtype == GFD_FLOAT64)
    launch_k(sub_const_kernel<double>, blocks, 256, 0, s, static_cast<double*>(y),
                                                    static_cast<const double*>(x), c, n);
  else if (dtype == GFD_FLOAT32)
    launch_k(sub_const_kernel<float>, blocks, 256, 0, s, static_cast<float*>(y),
                                                   static_cast<const float*>(x), c, n);
  else
    return set_error(GFD_EINVAL, "sub_const: unsupported dtype");
  return check_launch("sub_const_kernel");
}

int add_potential_launch(int dtype, void* out, const void* in, const void* v, int64_t n,
                         int64_t nin, cudaStream_t s) {
  const long long total = (long long)n * nin;
  const int blocks = grid_for(total);
  switch (dtype) {
    case GFD_FLOAT64:
      launch_k(add_potential_kernel<double>, blocks, 256, 0, s, static_cast<double*>(out),
               static_cast<const double*>(in), static_cast<const double*>(v), (long long)n, total);
      break;
    case GFD_FLOAT32:
      launch_k(add_potential_kernel<float>, blocks, 256, 0, s, static_cast<float*>(out),
               static_cast<const float*>(in), static_cast<const float*>(v), (long long)n, total);
      break;
    case GFD_COMPLEX128:
      launch_k(add_potential_kernel<cplx<double>>, blocks, 256, 0, s,
               static_cast<cplx<double>*>(out), static_cast<const cplx<double>*>(in),
               static_cast<const double*>(v), (long long)n, total);
      break;
    case GFD_COMPLEX64:
      launch_k(add_potential_kernel<cplx<float>>, blocks, 256, 0, s,
               static_cast<cplx<float>*>(out), static_cast<const cplx<float>*>(in),
               static_cast<const float*>(v), (long long)n, total);
      break;
    default:
      return set_error(GFD_EINVAL, "unknown dtype");
  }
  return check_launch("add_potential_kernel");
}

int convert_launch(int ydtype, void* y, int xdtype, const void* x, int64_t n, cudaStream_t s,
                   void* seed, double seed_scale) {
  const int blocks = grid_for(n);
  if (ydtype == GFD_FLOAT32 && xdtype == GFD_FLOAT64)
    launch_k(convert_kernel<float, double>, blocks, 256, 0, s, static_cast<float*>(y),
             static_cast<const double*>(x), (long long)n, static_cast<float*>(seed),
             float(seed_scale));
  else if (ydtype == GFD_FLOAT64 && xdtype == GFD_FLOAT32)
    launch_k(convert_kernel<double, float>, blocks, 256, 0, s, static_cast<double*>(y),
             static_cast<const float*>(x), (long long)n, static_cast<double*>(seed), seed_scale);
  else
    return set_error(GFD_EINVAL, "convert: unsupported dtype pair");
  return check_launch("convert_kernel");
}

}  // namespace gfd

using namespace gfd;

extern "C" int gfd_test_fail_alloc(long long n) {
  if (n < 0) return set_error(GFD_EINVAL, "allocation count must be >= 0");
  std::lock_guard<std::mutex> lock(g_alloc_mu);
  g_fail_countdown = n;
  return GFD_OK;
}

extern "C" size_t gfd_last_error(char* buf, size_t len) {
  const std::string& m = g_last_error;
  if (buf && len > 0) {
    size_t n = m.size() < len - 1 ? m.size() : len - 1;
    std::memcpy(buf, m.data(), n);
    buf[n] = '\0';
  }
  return m.size();
}

extern "C" const char* gfd_version(void) { return "gpaw-fd-b200 0.1 sm_100a"; }

extern "C" int gfd_density_interpolate(gfd_transformer* tr, const double* nt_sG, double* nt_sg,
                                       int64_t nspins, double pseudo_charge, double dv_fine,
                                       int renormalize, void* stream) {
  if (!tr) return set_error(GFD_EINVAL, "null transformer");
  if (!tr->interpolate) return set_error(GFD_EINVAL, "the transformer must interpolate");
  if (!tr->real) return set_error(GFD_EINVAL, "densities are real");
  if (nspins < 0) return set_error(GFD_EINVAL, "negative spin count");
  if (nspins == 0) return GFD_OK;
  if (!nt_sG || !nt_sg) return set_error(GFD_EINVAL, "null array pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = tr_launch(tr, GFD_FLOAT64, nt_sG, nt_sg, nspins, nullptr, s);
  if (st) return st;
  // gpaw/density.py:229-235: only with a zero boundary on some axis and a
  // nonzero pseudo charge.
  if (!renormalize || std::fabs(pseudo_charge) <= 1.0e-14) return GFD_OK;
  const int64_t n = (int64_t)tr->nout[0] * tr->nout[1] * tr->nout[2] * nspins;
  double* buf = nullptr;
  if ((st = check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&buf),
                                       sizeof(double) * (kRedBlocks + 1), s),
                       "cudaMallocAsync(reduction)")))
    return st;
  st = reduce_launch(GFD_FLOAT64, nt_sg, n, false, dv_fine, buf, buf + kRedBlocks, s);
  if (!st) {
    launch_k(scale_to_total_kernel, grid_for(n), 256, 0, s, nt_sg, (long long)n, pseudo_charge,
             (const double*)(buf + kRedBlocks));
    st = check_launch("scale_to_total_kernel");
  }
  cudaFreeAsync(buf, s);
  return st;
}

extern "C" int gfd_grid_sum(const double* a, int64_t n, double scale, double* result,
                            void* stream) {
  if (!result) return set_error(GFD_EINVAL, "null result pointer");
  if (n < 0) return set_error(GFD_EINVAL, "negative size");
  if (n == 0) {
    *result = 0.0;
    return GFD_OK;
  }
  if (!a) return set_error(GFD_EINVAL, "null array pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* buf = nullptr;
  int st = check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&buf),
                                      sizeof(double) * (kRedBlocks + 1), s),
                      "cudaMallocAsync(reduction)");
  if (st) return st;
  st = reduce_launch(GFD_FLOAT64, a, n, false, scale, buf, buf + kRedBlocks, s);
  if (!st)
    st = check_cuda(cudaMemcpyAsync(result, buf + kRedBlocks, sizeof(double),
                                    cudaMemcpyDeviceToHost, s),
                    "cudaMemcpyAsync(sum)");
  cudaFreeAsync(buf, s);
  if (!st) st = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize(sum)");
  return st;
}
