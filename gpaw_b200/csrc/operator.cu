// operator.cu -- gfd_operator_*: the _gpaw.Operator replacement
// (c/operators.c:465-498 constructor, :316-405 apply, :49-91 relax,
// :408-421 get_diagonal_element).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "common.cuh"
#include "internal.h"
#include "stencil_launch.cuh"
#include "stencil_tmasplit.cuh"

GFD_DECLARE_STENCIL_ENTRY(f64)
GFD_DECLARE_STENCIL_ENTRY(f32)
GFD_DECLARE_STENCIL_ENTRY(c128)
GFD_DECLARE_STENCIL_ENTRY(c64)

namespace gfd {

static int check_dtype(const gfd_operator* op, int dtype) {
  if (dtype < GFD_FLOAT64 || dtype > GFD_COMPLEX64)
    return set_error(GFD_EINVAL, "unknown dtype " + std::to_string(dtype));
  if (op->real != !dtype_is_complex(dtype))
    return set_error(GFD_EINVAL, op->real ? "operator was built for real arrays"
                                          : "operator was built for complex arrays");
  return GFD_OK;
}

int op_launch(const gfd_operator* op, int dtype, int mode, const void* in, void* out,
              const void* rho, int64_t nin, const double* phase_cd, double w,
              double* partials, cudaStream_t s) {
  if (nin <= 0) return GFD_OK;
  const bool star = op->star;
  switch (dtype) {
    case GFD_FLOAT64:
      return star ? star_f64(op, mode, in, out, rho, nin, phase_cd, w, partials, s)
                  : general_f64(op, mode, in, out, rho, nin, phase_cd, w, partials, s);
    case GFD_FLOAT32:
      return star ? star_f32(op, mode, in, out, rho, nin, phase_cd, w, partials, s)
                  : general_f32(op, mode, in, out, rho, nin, phase_cd, w, partials, s);
    case GFD_COMPLEX128:
      return star ? star_c128(op, mode, in, out, rho, nin, phase_cd, w, partials, s)
                  : general_c128(op, mode, in, out, rho, nin, phase_cd, w, partials, s);
    case GFD_COMPLEX64:
      return star ? star_c64(op, mode, in, out, rho, nin, phase_cd, w, partials, s)
                  : general_c64(op, mode, in, out, rho, nin, phase_cd, w, partials, s);
  }
  return set_error(GFD_EINVAL, "unknown dtype");
}

int64_t op_partials(const gfd_operator* op, int /*dtype*/, int /*mode*/, int64_t nin) {
  return partials_count(op, nin);
}

// Smallest colour count for which no nonzero offset keeps the colour
// (i0 + i1 + i2) mod ncolor; 0 if none up to 2*mp + 2.
int op_gs_colors(const gfd_operator* op) {
  for (int nc = 2; nc <= 2 * op->mp + 2; nc++) {
    bool ok = true;
    for (int c = 1; c < op->ncoefs && ok; c++) {
      int s = op->off[3 * c] + op->off[3 * c + 1] + op->off[3 * c + 2];
      if (((s % nc) + nc) % nc == 0) ok = false;
    }
    if (ok) return nc;
  }
  return 0;
}

int op_gs_sweeps(const gfd_operator* op, int dtype, void* phi, const void* rho, int nsweeps,
                 void* frozen, cudaStream_t s) {
  int nc = op_gs_colors(op);
  if (nc == 0) return set_error(GFD_EUNSUPPORTED, "no valid colouring for this stencil");
  if (dtype == GFD_FLOAT64)
    return gs_typed<double>(op, static_cast<double*>(phi), static_cast<const double*>(rho),
                            nsweeps, static_cast<double*>(frozen), nc, s);
  if (dtype == GFD_FLOAT32)
    return gs_typed<float>(op, static_cast<float*>(phi), static_cast<const float*>(rho), nsweeps,
                           static_cast<float*>(frozen), nc, s);
  return set_error(GFD_EINVAL, "relaxation needs a real dtype");
}

static int ensure_scratch(gfd_operator* op, size_t bytes) {
  if (op->scratch && op->scratch_bytes >= bytes) return GFD_OK;
  if (op->scratch) {
    cudaFree(op->scratch);
    op->scratch = nullptr;
    op->scratch_bytes = 0;
  }
  int st = dev_malloc(&op->scratch, bytes, "cudaMalloc of relaxation scratch");
  if (st) return st;
  op->scratch_bytes = bytes;
  cudaGetDevice(&op->device);
  return GFD_OK;
}

// ---------------------------------------------------------------------------
// TMA-fed stencil support: the kernel's error flag, the switch, and the
// tensor maps.
// ---------------------------------------------------------------------------
// Set by a kernel whose bounded mbarrier wait expired.
__device__ int g_star_err = 0;

// The TMA-staged lane-pair kernel is the default for complex128 bands it
// can take; GFD_TMASPLIT=0 in the environment keeps them on the cp.async
// kernels (for comparisons).
bool tmasplit_enabled() {
  static const bool on = [] {
    const char* e = getenv("GFD_TMASPLIT");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Opt-in (GFD_STAR_TMA=1): on the 96^3 x 512-band complex128 workload the
// TMA-fed kernel measured 2.6 TB/s against 3.7 TB/s for star_kernel.
bool star_tma_enabled() {
  static const bool on = [] {
    const char* e = getenv("GFD_STAR_TMA");
    return e && e[0] == '1';
  }();
  return on;
}

int* star_error_flag() {
  static std::mutex mu;
  static int* ptr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_error(GFD_ECUDA, "cudaGetDevice failed");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!ptr[dev]) {
    void* p = nullptr;
    if (check_cuda(cudaGetSymbolAddress(&p, g_star_err), "cudaGetSymbolAddress(g_star_err)"))
      return nullptr;
    ptr[dev] = static_cast<int*>(p);
  }
  return ptr[dev];
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return EncodeTiledFn(nullptr);
    }
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// One 4-D map over nb complex128 bands viewed as doubles: (2*n2, n1, n0, nb),
// box (box0 doubles, box1 rows, 1, 1), zero fill outside.
static int encode_one(CUtensorMap* m, const void* base, const gfd_operator* op, int64_t nb,
                      int box0, int box1) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(GFD_ECUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t row = cuuint64_t(op->n[2]) * 16;
  cuuint64_t dims[4] = {cuuint64_t(2 * op->n[2]), cuuint64_t(op->n[1]), cuuint64_t(op->n[0]),
                        cuuint64_t(nb)};
  cuuint64_t strides[3] = {row, row * op->n[1], row * op->n[1] * op->n[0]};
  cuuint32_t box[4] = {cuuint32_t(box0), cuuint32_t(box1), 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(GFD_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return GFD_OK;
}

// Maps of star_tmasplit_kernel (stencil_tmasplit.cuh).  Bands as doubles
// (2, n2, n1, n0, nb) with element stride 2 on the column axis, so one box
// takes every second column: box (2, 2 pw, rows, 1, 1) stages pw values of
// one column parity for `rows` rows.
static int encode_parity(CUtensorMap* m, const void* base, const gfd_operator* op, int64_t nb,
                         int pw, int rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(GFD_ECUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t row = cuuint64_t(op->n[2]) * 16;
  cuuint64_t dims[5] = {2, cuuint64_t(op->n[2]), cuuint64_t(op->n[1]), cuuint64_t(op->n[0]),
                        cuuint64_t(nb)};
  cuuint64_t strides[4] = {16, row, row * op->n[1], row * op->n[1] * op->n[0]};
  cuuint32_t box[5] = {2, cuuint32_t(2 * pw), cuuint32_t(rows), 1, 1};
  cuuint32_t estr[5] = {1, 2, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(GFD_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return GFD_OK;
}

int encode_ts_maps(TsMaps* maps, const void* in, const void* rho, const void* pot,
                   const gfd_operator* op, int64_t nb, int R, int ng) {
  const int re = (R + 1) & ~1;
  const int pw = ts_pw(ng, re), sy = kTsBY + 2 * R;
  int st;
  if ((st = encode_parity(&maps->rows_full, in, op, nb, pw, sy))) return st;
  if ((st = encode_parity(&maps->rows_main, in, op, nb, pw, sy - R))) return st;
  if ((st = encode_parity(&maps->rows_own, in, op, nb, pw, kTsBY))) return st;
  if ((st = encode_parity(&maps->rows_halo, in, op, nb, pw, R))) return st;
  std::memset(&maps->rho, 0, sizeof maps->rho);
  std::memset(&maps->pot, 0, sizeof maps->pot);
  if (rho && (st = encode_parity(&maps->rho, rho, op, nb, ts_pwr(ng), kTsBY))) return st;
  if (pot) {
    // The potential: one real grid (n2, n1, n0), box (32 ng, BY, 1).
    EncodeTiledFn fn = encode_fn();
    if (!fn) return set_error(GFD_ECUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t row = cuuint64_t(op->n[2]) * 8;
    cuuint64_t dims[3] = {cuuint64_t(op->n[2]), cuuint64_t(op->n[1]), cuuint64_t(op->n[0])};
    cuuint64_t strides[2] = {row, row * op->n[1]};
    cuuint32_t box[3] = {cuuint32_t(32 * ng), cuuint32_t(kTsBY), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(&maps->pot, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(pot), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return set_error(GFD_ECUDA,
                       "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  }
  return GFD_OK;
}

int encode_tma_maps(TmaMaps* maps, const void* base, const gfd_operator* op, int64_t nb, int R,
                    int by) {
  int st;
  if ((st = encode_one(&maps->rows_halo, base, op, nb, 2 * kTmaBZ, R))) return st;
  if ((st = encode_one(&maps->rows_own, base, op, nb, 2 * kTmaBZ, by))) return st;
  return encode_one(&maps->side, base, op, nb, 2 * R, by);
}

}  // namespace gfd

namespace gfd {
// A wait that nothing completes: thread 0 initialises an mbarrier nobody
// arrives on, every thread waits on its first phase with the kernels'
// bounded wait (limit max_cycles) and, when the wait runs out, the kernel
// sets the device error flag exactly as the stencil kernels do.  No copy is
// in flight, so the early exit leaves nothing behind.
__global__ void wait_probe_kernel(int* err, long long max_cycles) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (!mbar_wait_bounded(&bar, 0u, &abort_flag, max_cycles)) {
    abort_flag = 1;
    if (threadIdx.x == 0) atomicExch(err, 1);
  }
}
}  // namespace gfd

using namespace gfd;

extern "C" int gfd_wait_selftest(long long max_cycles) {
  if (max_cycles < 1 || max_cycles > kSpinCycles)
    return set_error(GFD_EINVAL, "wait limit out of range");
  int* err = star_error_flag();
  if (!err) return GFD_ECUDA;
  wait_probe_kernel<<<1, 64>>>(err, max_cycles);
  int st = check_launch("wait_probe_kernel");
  if (st) return st;
  return check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize(wait probe)");
}

extern "C" int gfd_device_errors(int* flags) {
  if (!flags) return set_error(GFD_EINVAL, "null argument");
  int* p = star_error_flag();
  if (!p) return GFD_ECUDA;
  int st = check_cuda(cudaMemcpy(flags, p, sizeof(int), cudaMemcpyDeviceToHost),
                      "cudaMemcpy(error flag)");
  if (st) return st;
  const int zero = 0;
  return check_cuda(cudaMemcpy(p, &zero, sizeof(int), cudaMemcpyHostToDevice),
                    "cudaMemcpy(error flag)");
}

extern "C" int gfd_operator_create(int ncoefs, const double* coefs, const int64_t* offsets,
                                   const int64_t size[3], int range, const int64_t neighbors[6],
                                   int real, int cfd, gfd_operator** out) {
  if (!out) return set_error(GFD_EINVAL, "null output handle");
  *out = nullptr;
  if (ncoefs < 1 || !coefs || !offsets || !size || !neighbors)
    return set_error(GFD_EINVAL, "operator needs at least one coefficient and all arrays");
  gfd_operator* op = new (std::nothrow) gfd_operator();
  if (!op) return set_error(GFD_ENOMEM, "host allocation failed");
  op->ncoefs = ncoefs;
  op->coefs.assign(coefs, coefs + ncoefs);
  op->off.resize(3 * ncoefs);
  op->real = real ? 1 : 0;
  op->cfd = cfd ? 1 : 0;
  int mp = 0;
  for (int c = 0; c < ncoefs; c++)
    for (int a = 0; a < 3; a++) {
      int64_t o = offsets[3 * c + a];
      if (o < -kMaxR * 4 || o > kMaxR * 4) {
        delete op;
        return set_error(GFD_EINVAL, "stencil offset out of range");
      }
      op->off[3 * c + a] = (int)o;
      mp = std::max(mp, (int)std::llabs(o));
    }
  op->mp = mp;
  if (range < mp) {
    delete op;
    return set_error(GFD_EINVAL, "range is smaller than the largest offset");
  }
  for (int a = 0; a < 3; a++) {
    if (size[a] < 1 || size[a] > (1 << 20)) {
      delete op;
      return set_error(GFD_EINVAL, "grid size out of range");
    }
    op->n[a] = (int)size[a];
    int64_t lo = neighbors[2 * a], hi = neighbors[2 * a + 1];
    if (!((lo == 0 && hi == 0) || (lo == -1 && hi == -1))) {
      delete op;
      return set_error(GFD_EUNSUPPORTED,
                       "neighbors must be 0 (periodic, this domain) or -1 (zero boundary); "
                       "domain decomposition is not provided");
    }
    op->per[a] = (lo == 0) ? 1 : 0;
    if (op->per[a] && op->n[a] < mp) {
      delete op;
      return set_error(GFD_EINVAL, "periodic axis has fewer points than the stencil range");
    }
  }
  if ((double)op->n[0] * op->n[1] * op->n[2] >= 2147483647.0 / 16) {
    delete op;
    return set_error(GFD_EINVAL, "grid too large for one band");
  }
  // Zero-offset weight (the reference scans for offset 0, c/operators.c:414-417).
  for (int c = 0; c < ncoefs; c++)
    if (op->off[3 * c] == 0 && op->off[3 * c + 1] == 0 && op->off[3 * c + 2] == 0)
      op->diag = coefs[c];
  // Axis-aligned decomposition.
  bool star = mp <= kMaxR;
  for (int c = 0; c < ncoefs && star; c++) {
    int nz = (op->off[3 * c] != 0) + (op->off[3 * c + 1] != 0) + (op->off[3 * c + 2] != 0);
    if (nz > 1) star = false;
  }
  if (star) {
    op->c0 = 0.0;
    for (int c = 0; c < ncoefs; c++) {
      const int* o = &op->off[3 * c];
      if (o[0]) op->cx[kMaxR + o[0]] += coefs[c];
      else if (o[1]) op->cy[kMaxR + o[1]] += coefs[c];
      else if (o[2]) op->cz[kMaxR + o[2]] += coefs[c];
      else op->c0 += coefs[c];
    }
    op->R = std::max(mp, 1);
  }
  op->star = star;
  *out = op;
  return GFD_OK;
}

extern "C" int gfd_operator_destroy(gfd_operator* op) {
  if (!op) return GFD_OK;
  if (op->scratch) cudaFree(op->scratch);
  delete op;
  return GFD_OK;
}

extern "C" int gfd_operator_apply(gfd_operator* op, int dtype, const void* in, void* out,
                                  int64_t nin, const double* phase_cd, void* stream) {
  if (!op) return set_error(GFD_EINVAL, "null operator");
  int st = check_dtype(op, dtype);
  if (st) return st;
  if (nin < 0) return set_error(GFD_EINVAL, "negative band count");
  if (nin == 0) return GFD_OK;
  if (!in || !out) return set_error(GFD_EINVAL, "null array pointer");
  if (in == out) return set_error(GFD_EINVAL, "input and output must not overlap");
  return op_launch(op, dtype, OP_APPLY, in, out, nullptr, nin, phase_cd, 0.0, nullptr,
                   static_cast<cudaStream_t>(stream));
}

extern "C" int gfd_operator_apply_potential(gfd_operator* op, int dtype, const void* in,
                                            void* out, int64_t nin, const double* phase_cd,
                                            const void* v, void* stream) {
  if (!op) return set_error(GFD_EINVAL, "null operator");
  int st = check_dtype(op, dtype);
  if (st) return st;
  if (nin < 0) return set_error(GFD_EINVAL, "negative band count");
  if (nin == 0) return GFD_OK;
  if (!in || !out || !v) return set_error(GFD_EINVAL, "null array pointer");
  if (in == out) return set_error(GFD_EINVAL, "input and output must not overlap");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (op->star)
    return op_launch(op, dtype, OP_POTENTIAL, in, out, v, nin, phase_cd, 0.0, nullptr, s);
  // Other offset sets: the stencil, then the potential term in a second pass.
  if ((st = op_launch(op, dtype, OP_APPLY, in, out, nullptr, nin, phase_cd, 0.0, nullptr, s)))
    return st;
  return add_potential_launch(dtype, out, in, v, (int64_t)op->n[0] * op->n[1] * op->n[2], nin, s);
}

extern "C" int gfd_operator_relax(gfd_operator* op, int dtype, int relax_method, void* func,
                                  const void* source, int nrelax, double w, void* stream) {
  if (!op) return set_error(GFD_EINVAL, "null operator");
  if (dtype != GFD_FLOAT64 && dtype != GFD_FLOAT32)
    return set_error(GFD_EINVAL, "relaxation works on real arrays only");
  if (!op->real) return set_error(GFD_EINVAL, "operator was built for complex arrays");
  if (!func || !source) return set_error(GFD_EINVAL, "null array pointer");
  if (nrelax < 0) return set_error(GFD_EINVAL, "negative sweep count");
  if (nrelax == 0) return GFD_OK;
  if (op->off[0] != 0 || op->off[1] != 0 || op->off[2] != 0)
    return set_error(GFD_EINVAL, "relaxation needs the diagonal (zero offset) as coefs[0]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = (size_t)op->n[0] * op->n[1] * op->n[2] * dtype_size(dtype);
  int st = ensure_scratch(op, bytes);
  if (st) return st;
  if (relax_method == GFD_RELAX_GS) return op_gs_sweeps(op, dtype, func, source, nrelax, op->scratch, s);
  // Weighted Jacobi with w = 0 leaves func unchanged.
  if (w == 0.0) return GFD_OK;
  // Weighted Jacobi: ping-pong between func and the scratch grid.
  void* cur = func;
  void* nxt = op->scratch;
  for (int k = 0; k < nrelax; k++) {
    st = op_launch(op, dtype, OP_JACOBI, cur, nxt, source, 1, nullptr, w, nullptr, s);
    if (st) return st;
    std::swap(cur, nxt);
  }
  if (cur != func)
    return check_cuda(cudaMemcpyAsync(func, cur, bytes, cudaMemcpyDeviceToDevice, s),
                      "cudaMemcpyAsync(relax result)");
  return GFD_OK;
}

extern "C" int gfd_operator_get_diagonal_element(const gfd_operator* op, double* d) {
  if (!op || !d) return set_error(GFD_EINVAL, "null argument");
  *d = op->diag;
  return GFD_OK;
}
