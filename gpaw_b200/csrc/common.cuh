// common.cuh -- element types, halo mapping and error plumbing shared by the
// sm_100a kernels of libgpawfd.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <utility>

#include "gpaw_fd.h"

namespace gfd {

// ---------------------------------------------------------------------------
// Element types.  Complex values are interleaved (re, im) pairs, the layout
// of numpy / torch complex arrays; the 16-byte alignment lets one vector
// load move a complex128.
// ---------------------------------------------------------------------------
template <class S>
struct __align__(2 * sizeof(S)) cplx {
  S re, im;
};

template <class V> struct vt;
template <> struct vt<double> { using S = double; static constexpr int NC = 1; };
template <> struct vt<float> { using S = float; static constexpr int NC = 1; };
template <> struct vt<cplx<double>> { using S = double; static constexpr int NC = 2; };
template <> struct vt<cplx<float>> { using S = float; static constexpr int NC = 2; };

template <class V> __device__ __forceinline__ V vzero();
template <> __device__ __forceinline__ double vzero<double>() { return 0.0; }
template <> __device__ __forceinline__ float vzero<float>() { return 0.0f; }
template <> __device__ __forceinline__ cplx<double> vzero<cplx<double>>() { return {0.0, 0.0}; }
template <> __device__ __forceinline__ cplx<float> vzero<cplx<float>>() { return {0.0f, 0.0f}; }

// acc += c * v  (c real)
__device__ __forceinline__ void madd(double& a, double c, double v) { a = fma(c, v, a); }
__device__ __forceinline__ void madd(float& a, float c, float v) { a = fmaf(c, v, a); }
template <class S>
__device__ __forceinline__ void madd(cplx<S>& a, S c, const cplx<S>& v) {
  madd(a.re, c, v.re);
  madd(a.im, c, v.im);
}

__device__ __forceinline__ double vmul(double c, double v) { return c * v; }
__device__ __forceinline__ float vmul(float c, float v) { return c * v; }
template <class S>
__device__ __forceinline__ cplx<S> vmul(S c, const cplx<S>& v) { return {c * v.re, c * v.im}; }

__device__ __forceinline__ double vadd(double a, double b) { return a + b; }
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
template <class S>
__device__ __forceinline__ cplx<S> vadd(const cplx<S>& a, const cplx<S>& b) {
  return {a.re + b.re, a.im + b.im};
}
__device__ __forceinline__ double vsub(double a, double b) { return a - b; }
__device__ __forceinline__ float vsub(float a, float b) { return a - b; }
template <class S>
__device__ __forceinline__ cplx<S> vsub(const cplx<S>& a, const cplx<S>& b) {
  return {a.re - b.re, a.im - b.im};
}

// Complex phase times value; identity for real values.
template <class S>
__device__ __forceinline__ cplx<S> cmul(const cplx<S>& p, const cplx<S>& v) {
  return {p.re * v.re - p.im * v.im, p.re * v.im + p.im * v.re};
}
__device__ __forceinline__ double phase_mul(const cplx<double>&, double v) { return v; }
__device__ __forceinline__ float phase_mul(const cplx<float>&, float v) { return v; }
template <class S>
__device__ __forceinline__ cplx<S> phase_mul(const cplx<S>& p, const cplx<S>& v) {
  return cmul(p, v);
}

// Asynchronous global->shared copies (sm_80+ cp.async).  A source size of 0
// writes zeros (zero boundary points); the source address is then unused but
// kept valid.  16-byte copies use the L1-allocating form (.ca): measured on
// B200, the cache-bypass form (.cg) fetched one 32-byte L2 sector per lane
// and wrote shared memory one lane at a time (about 28 shared-store
// wavefronts per warp copy of 512 contiguous bytes, against 4.5 for .ca), so
// it moved twice the bytes from L2.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src, bool valid) {
  const unsigned d = smem_addr(dst);
  const int n = valid ? BYTES : 0;
  if constexpr (BYTES == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES),
                 "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Read-only global loads (one vector instruction per element).
__device__ __forceinline__ double ldro(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ldro(const float* p) { return __ldg(p); }
__device__ __forceinline__ cplx<double> ldro(const cplx<double>* p) {
  double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return {v.x, v.y};
}
__device__ __forceinline__ cplx<float> ldro(const cplx<float>* p) {
  float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return {v.x, v.y};
}

// Load policy of the per-point functions (stencil.cuh, transfer.cuh): the
// read-only path.
struct LoadRO {
  template <class T>
  __device__ __forceinline__ static T ld(const T* p) { return ldro(p); }
};

// Streaming store (output is not re-read by this kernel).
__device__ __forceinline__ void stcs(double* p, double v) { __stcs(p, v); }
__device__ __forceinline__ void stcs(float* p, float v) { __stcs(p, v); }
__device__ __forceinline__ void stcs(cplx<double>* p, const cplx<double>& v) {
  __stcs(reinterpret_cast<double2*>(p), make_double2(v.re, v.im));
}
__device__ __forceinline__ void stcs(cplx<float>* p, const cplx<float>& v) {
  __stcs(reinterpret_cast<float2*>(p), make_float2(v.re, v.im));
}

__device__ __forceinline__ double sq(double v) { return v * v; }
__device__ __forceinline__ double sq(float v) { return double(v) * double(v); }

// ---------------------------------------------------------------------------
// Halo mapping along one axis.  A coordinate u outside [0, n) is a zero
// point on a non-periodic axis and wraps on a periodic one (the host
// guarantees n >= halo width).  side: -1 inside, 1 low halo (takes
// phase_cd[c][1]), 0 high halo (takes phase_cd[c][0]); the convention of
// c/bc.c:234-249 where slab d is copied to the far side times phases[d].
// ---------------------------------------------------------------------------
// A tile that overhangs a short periodic axis asks for coordinates more than
// one period away (u >= 2n, e.g. a 32-wide tile on a 16-point axis).  Only
// outputs outside the domain use those cells, so any in-range index serves;
// the coordinate is reduced modulo n so every load stays inside the array.
__device__ __forceinline__ int wrap_axis(int u, int n, int periodic, int& side) {
  side = -1;
  if (u >= 0 && u < n) return u;
  if (!periodic) return -1;
  if (u < 0) {
    side = 1;
    u += n;
    return u >= 0 ? u : (u % n + n) % n;
  }
  side = 0;
  u -= n;
  return u < n ? u : u % n;
}

// The same for a plane index of a marching kernel, which lies in
// [-R, n + R) with n >= R on a periodic axis: one wrap at most.
__device__ __forceinline__ int wrap_plane(int u, int n, int periodic, int& side) {
  side = -1;
  if (u >= 0 && u < n) return u;
  if (!periodic) return -1;
  if (u < 0) {
    side = 1;
    return u + n;
  }
  side = 0;
  return u - n;
}

// Phases for the three axes: ph[c][d], d = 0 high halo, 1 low halo.
template <class S>
struct Phases {
  cplx<S> ph[3][2];
};

template <class S>
__device__ __forceinline__ cplx<S> phase_of(const Phases<S>& P, int c, int side) {
  return P.ph[c][side];
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  Every kernel of the library starts with
// pdl_enter(): it lets the next kernel on the stream be scheduled at once
// (so its launch overlaps this one), then waits until the previous kernel
// has completed and its writes are visible.  All global reads and writes
// come after the wait, so a dependent kernel never sees a predecessor's
// partial results.  Both instructions are no-ops for a normal launch.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

bool pdl_enabled();
// Complex bands on the lane-pair stencil kernel (GFD_SPLIT=0 turns it off).
bool split_enabled();
// Largest grid (points over all bands) for the one-thread-per-point kernels.
long long direct_max_points();
// CTAs per SM the marching kernels aim for when they split axis 0 into
// chunks (GFD_MARCH_CTAS_PER_SM, default 4).
int march_ctas_per_sm();

// Launch with the programmatic-stream-serialisation attribute when enabled
// (GFD_PDL=1 in the environment; off by default).
template <class... P, class... A>
inline cudaError_t launch_k(void (*kern)(P...), dim3 grid, dim3 block, size_t smem,
                            cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// ---------------------------------------------------------------------------
// Host-side error plumbing.
// ---------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
// cudaMalloc with the library's status codes (GFD_ENOMEM on exhaustion) and
// the planned-failure hook of gfd_test_fail_alloc.
int dev_malloc(void** p, size_t bytes, const char* what);
int check_cuda(cudaError_t e, const char* what);
int check_launch(const char* what);

inline int dtype_is_complex(int dtype) { return dtype == GFD_COMPLEX128 || dtype == GFD_COMPLEX64; }
template <class V>
constexpr int dtype_of() {
  return vt<V>::NC == 2 ? (sizeof(typename vt<V>::S) == 8 ? GFD_COMPLEX128 : GFD_COMPLEX64)
                        : (sizeof(typename vt<V>::S) == 8 ? GFD_FLOAT64 : GFD_FLOAT32);
}
inline int dtype_is_fp32(int dtype) { return dtype == GFD_FLOAT32 || dtype == GFD_COMPLEX64; }
inline size_t dtype_size(int dtype) {
  switch (dtype) {
    case GFD_FLOAT64: return 8;
    case GFD_COMPLEX128: return 16;
    case GFD_FLOAT32: return 4;
    case GFD_COMPLEX64: return 8;
  }
  return 0;
}

constexpr int kNumSMs = 148;

}  // namespace gfd
