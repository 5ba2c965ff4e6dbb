// transformer.cu -- gfd_transformer_*: the _gpaw.Transformer replacement
// (c/transformers.c:222-265 constructor, :127-185 apply).
#include <algorithm>
#include <new>
#include <string>

#include "common.cuh"
#include "internal.h"
#include "transfer.cuh"

namespace gfd {

template <class V, int NN>
static int restrict_go(const gfd_transformer* tr, const V* in, V* out, int64_t nin,
                       TrParams<typename vt<V>::S>& p, int cps, cudaStream_t s) {
  // Two coarse rows per thread (16 per CTA) stage fewer halo rows per output
  // row; complex128 keeps one, so two CTAs still fit on an SM.  Other shapes
  // measured slower on 256 float64 bands of 112^3 (nn = 3; 2800-2830 GB/s
  // for this one): 28 columns, which tile 112 exactly, 2580; one coarse row
  // per thread 2270; 32 rows per CTA 2410; 4 rows per thread 2490 (253
  // registers); three CTAs per SM (80 registers, spills) 1740.
  constexpr int BZC = 32, TYC = 8, VYC = sizeof(V) >= 16 ? 1 : 2, BYC = TYC * VYC;
  constexpr int W = 2 * NN - 1;
  constexpr int RY = 2 * BYC - 1 + 2 * W, RZ = 2 * BZC - 1 + 2 * W;
  const size_t smem = (size_t)(2 * RY * rst_row_pitch<V, RZ>() + 2 * RY * BZC) * sizeof(V);
  const int gx = (tr->nout[2] + BZC - 1) / BZC, gy = (tr->nout[1] + BYC - 1) / BYC;
  const int64_t tiles = (int64_t)gx * gy * nin;
  const int64_t target = (int64_t)(cps > 0 ? cps : march_ctas_per_sm()) * num_sms();
  int maxc = std::max(1, tr->nout[0] / 2);
  int nxc = (int)std::min<int64_t>(maxc, std::max<int64_t>(1, (target + tiles - 1) / tiles));
  p.x_chunk = (tr->nout[0] + nxc - 1) / nxc;
  p.nxc = (tr->nout[0] + p.x_chunk - 1) / p.x_chunk;
  auto kern = restrict_kernel<V, NN, BZC, TYC, VYC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(restrict_kernel)");
  const int64_t per_launch = std::max<int64_t>(1, 65535 / p.nxc);
  for (int64_t b0 = 0; b0 < nin; b0 += per_launch) {
    int64_t nb = std::min<int64_t>(per_launch, nin - b0);
    dim3 grid(gx, gy, (unsigned)(nb * p.nxc));
    launch_k(kern, grid, BZC * TYC, smem, s, in + b0 * p.band_in, out + b0 * p.band_out, p);
  }
  return check_launch("restrict_kernel");
}

template <class V, int NN>
static int interp_go(const gfd_transformer* tr, const V* in, V* out, const V* base, int64_t nin,
                     TrParams<typename vt<V>::S>& p, int cps, cudaStream_t s) {
  constexpr int BZF = 64, TYF = 4, VYF = 2, BYF = TYF * VYF;
  constexpr int CY = BYF / 2 + 2 * NN, CZ = BZF / 2 + 2 * NN;
  const size_t smem = (size_t)(2 * CY * CZ + 2 * CY * BZF) * sizeof(V);
  const int gx = (tr->nout[2] + BZF - 1) / BZF, gy = (tr->nout[1] + BYF - 1) / BYF;
  const int64_t tiles = (int64_t)gx * gy * nin;
  const int64_t target = (int64_t)(cps > 0 ? cps : march_ctas_per_sm()) * num_sms();
  int maxc = std::max(1, tr->nout[0] / 4);
  int nxc = (int)std::min<int64_t>(maxc, std::max<int64_t>(1, (target + tiles - 1) / tiles));
  p.x_chunk = (tr->nout[0] + nxc - 1) / nxc;
  p.nxc = (tr->nout[0] + p.x_chunk - 1) / p.x_chunk;
  auto kern = base ? interp_kernel<V, NN, BZF, TYF, VYF, true>
                   : interp_kernel<V, NN, BZF, TYF, VYF, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(interp_kernel)");
  const int64_t per_launch = std::max<int64_t>(1, 65535 / p.nxc);
  for (int64_t b0 = 0; b0 < nin; b0 += per_launch) {
    int64_t nb = std::min<int64_t>(per_launch, nin - b0);
    dim3 grid(gx, gy, (unsigned)(nb * p.nxc));
    launch_k(kern, grid, BZF * TYF, smem, s, in + b0 * p.band_in, out + b0 * p.band_out,
                                       base ? base + b0 * p.band_out : nullptr, p);
  }
  return check_launch("interp_kernel");
}

// Outputs (all bands) up to direct_max_points() use the one-thread-per-point
// forms.
template <class V, int NN>
static int direct_go(const gfd_transformer* tr, const V* in, V* out, const V* base, int64_t nin,
                     const TrParams<typename vt<V>::S>& p, cudaStream_t s) {
  const long long total = p.band_out * nin;
  long long b = (total + 255) / 256, cap = 8LL * num_sms();
  const int blocks = int(b < 1 ? 1 : (b > cap ? cap : b));
  if (!tr->interpolate)
    launch_k(restrict_direct_kernel<V, NN>, blocks, 256, 0, s, in, out, p, total);
  else if (base)
    launch_k(interp_direct_kernel<V, NN, true>, blocks, 256, 0, s, in, out, base, p, total);
  else
    launch_k(interp_direct_kernel<V, NN, false>, blocks, 256, 0, s, in, out, nullptr, p, total);
  return check_launch("transfer_direct_kernel");
}

template <class V>
static int tr_typed(const gfd_transformer* tr, const void* in, void* out, const void* base_v,
                    int64_t nin, const double* ph, cudaStream_t s, void* seed = nullptr,
                    double seed_scale = 0.0, double out_scale = 1.0) {
  using S = typename vt<V>::S;
  TrParams<S> p;
  tr_params(tr, ph, seed, seed_scale, out_scale, p);
  if (seed && tr->interpolate) return set_error(GFD_EINVAL, "seeded form is for restriction only");
  const V* vin = static_cast<const V*>(in);
  V* vout = static_cast<V*>(out);
  const V* base = static_cast<const V*>(base_v);
  if (base && !tr->interpolate)
    return set_error(GFD_EINVAL, "subtracting form is for interpolation only");
  TunePlan plan;
  const bool tuned = tune_lookup(tr_tune_key(tr, dtype_of<V>(), nin), &plan);
  const int cps = tuned ? plan.cps : 0;
  if (tuned ? plan.path == PLAN_DIRECT : p.band_out * nin <= direct_max_points()) {
    switch (tr->nn) {
      case 1: return direct_go<V, 1>(tr, vin, vout, base, nin, p, s);
      case 2: return direct_go<V, 2>(tr, vin, vout, base, nin, p, s);
      case 3: return direct_go<V, 3>(tr, vin, vout, base, nin, p, s);
      case 4: return direct_go<V, 4>(tr, vin, vout, base, nin, p, s);
    }
  }
  if (tr->interpolate) {
    switch (tr->nn) {
      case 1: return interp_go<V, 1>(tr, vin, vout, base, nin, p, cps, s);
      case 2: return interp_go<V, 2>(tr, vin, vout, base, nin, p, cps, s);
      case 3: return interp_go<V, 3>(tr, vin, vout, base, nin, p, cps, s);
      case 4: return interp_go<V, 4>(tr, vin, vout, base, nin, p, cps, s);
    }
  } else {
    if (base) return set_error(GFD_EINVAL, "subtracting form is for interpolation only");
    switch (tr->nn) {
      case 1: return restrict_go<V, 1>(tr, vin, vout, nin, p, cps, s);
      case 2: return restrict_go<V, 2>(tr, vin, vout, nin, p, cps, s);
      case 3: return restrict_go<V, 3>(tr, vin, vout, nin, p, cps, s);
      case 4: return restrict_go<V, 4>(tr, vin, vout, nin, p, cps, s);
    }
  }
  return set_error(GFD_EINVAL, "k must be 2, 4, 6 or 8");
}

int tr_launch_sub(const gfd_transformer* tr, int dtype, const void* in, void* out,
                  const void* base, int64_t nin, const double* phases, cudaStream_t s) {
  if (nin <= 0) return GFD_OK;
  switch (dtype) {
    case GFD_FLOAT64: return tr_typed<double>(tr, in, out, base, nin, phases, s);
    case GFD_FLOAT32: return tr_typed<float>(tr, in, out, base, nin, phases, s);
    case GFD_COMPLEX128: return tr_typed<cplx<double>>(tr, in, out, base, nin, phases, s);
    case GFD_COMPLEX64: return tr_typed<cplx<float>>(tr, in, out, base, nin, phases, s);
  }
  return set_error(GFD_EINVAL, "unknown dtype");
}

int tr_launch_seed(const gfd_transformer* tr, int dtype, const void* in, void* out, void* seed,
                   double seed_scale, cudaStream_t s) {
  return tr_launch_ex(tr, dtype, in, out, nullptr, 1, nullptr, 1.0, seed, seed_scale, s);
}

int tr_launch_ex(const gfd_transformer* tr, int dtype, const void* in, void* out,
                 const void* base, int64_t nin, const double* phases, double out_scale,
                 void* seed, double seed_scale, cudaStream_t s) {
  if (nin <= 0) return GFD_OK;
  switch (dtype) {
    case GFD_FLOAT64:
      return tr_typed<double>(tr, in, out, base, nin, phases, s, seed, seed_scale, out_scale);
    case GFD_FLOAT32:
      return tr_typed<float>(tr, in, out, base, nin, phases, s, seed, seed_scale, out_scale);
    case GFD_COMPLEX128:
      return tr_typed<cplx<double>>(tr, in, out, base, nin, phases, s, seed, seed_scale,
                                    out_scale);
    case GFD_COMPLEX64:
      return tr_typed<cplx<float>>(tr, in, out, base, nin, phases, s, seed, seed_scale,
                                   out_scale);
  }
  return set_error(GFD_EINVAL, "unknown dtype");
}

int tr_launch(const gfd_transformer* tr, int dtype, const void* in, void* out, int64_t nin,
              const double* phases, cudaStream_t s) {
  return tr_launch_sub(tr, dtype, in, out, nullptr, nin, phases, s);
}

}  // namespace gfd

using namespace gfd;

extern "C" int gfd_transformer_create(const int64_t size_in[3], const int64_t size_out[3], int k,
                                      const int64_t pad[6], const int64_t npad[6],
                                      const int64_t skip[6], const int64_t neighbors[6], int real,
                                      int interpolate, gfd_transformer** out) {
  if (!out) return set_error(GFD_EINVAL, "null output handle");
  *out = nullptr;
  if (!size_in || !size_out || !pad || !npad || !skip || !neighbors)
    return set_error(GFD_EINVAL, "null array argument");
  if (k != 2 && k != 4 && k != 6 && k != 8) return set_error(GFD_EINVAL, "k must be 2, 4, 6 or 8");
  gfd_transformer* tr = new (std::nothrow) gfd_transformer();
  if (!tr) return set_error(GFD_ENOMEM, "host allocation failed");
  tr->k = k;
  tr->nn = k / 2;
  tr->real = real ? 1 : 0;
  tr->interpolate = interpolate ? 1 : 0;
  for (int a = 0; a < 3; a++) {
    tr->nin[a] = (int)size_in[a];
    tr->nout[a] = (int)size_out[a];
    if (size_in[a] < 1 || size_out[a] < 1 || size_in[a] > (1 << 20) || size_out[a] > (1 << 20)) {
      delete tr;
      return set_error(GFD_EINVAL, "grid size out of range");
    }
    for (int d = 0; d < 2; d++) {
      if (pad[2 * a + d] < 0 || pad[2 * a + d] > 64 || skip[2 * a + d] < 0 || skip[2 * a + d] > 1) {
        delete tr;
        return set_error(GFD_EINVAL, "padding or skip out of range");
      }
      tr->pad[a][d] = (int)pad[2 * a + d];
      tr->skip[a][d] = interpolate ? (int)skip[2 * a + d] : 0;
    }
    int64_t lo = neighbors[2 * a], hi = neighbors[2 * a + 1];
    if (!((lo == 0 && hi == 0) || (lo == -1 && hi == -1))) {
      delete tr;
      return set_error(GFD_EUNSUPPORTED,
                       "neighbors must be 0 (periodic, this domain) or -1 (zero boundary); "
                       "domain decomposition is not provided");
    }
    tr->per[a] = lo == 0;
    if (tr->per[a] && (tr->pad[a][0] > tr->nin[a] || tr->pad[a][1] > tr->nin[a])) {
      delete tr;
      return set_error(GFD_EINVAL, "periodic axis has fewer points than the halo");
    }
    // Output size implied by the padding (c/bmgs/restrict.c:150-152,
    // c/bmgs/interpolate.c:158-167).
    int64_t s = size_in[a] + pad[2 * a] + pad[2 * a + 1];
    int64_t expect = interpolate
                         ? 2 * (s - (k - 1) + tr->skip[a][1]) - tr->skip[a][0] - tr->skip[a][1]
                         : (s - (2 * k - 3)) / 2;
    if (!interpolate && ((s - (2 * k - 3)) < 0 || (s - (2 * k - 3)) % 2)) expect = -1;
    if (expect != size_out[a]) {
      delete tr;
      return set_error(GFD_EINVAL, "size_out does not match size_in and the padding on axis " +
                                       std::to_string(a));
    }
  }
  *out = tr;
  return GFD_OK;
}

extern "C" int gfd_transformer_destroy(gfd_transformer* tr) {
  delete tr;
  return GFD_OK;
}

extern "C" int gfd_transformer_apply(gfd_transformer* tr, int dtype, const void* in, void* out,
                                     int64_t nin, const double* phases, void* stream) {
  if (!tr) return set_error(GFD_EINVAL, "null transformer");
  if (dtype < GFD_FLOAT64 || dtype > GFD_COMPLEX64) return set_error(GFD_EINVAL, "unknown dtype");
  if (tr->real != !dtype_is_complex(dtype))
    return set_error(GFD_EINVAL, tr->real ? "transformer was built for real arrays"
                                          : "transformer was built for complex arrays");
  if (nin < 0) return set_error(GFD_EINVAL, "negative band count");
  if (nin == 0) return GFD_OK;
  if (!in || !out) return set_error(GFD_EINVAL, "null array pointer");
  return tr_launch(tr, dtype, in, out, nin, phases, static_cast<cudaStream_t>(stream));
}
