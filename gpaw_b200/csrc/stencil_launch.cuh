// stencil_launch.cuh -- host-side tile selection and template dispatch for the
// stencil kernels.  Included by one translation unit per element type so the
// instantiations compile in parallel.
#pragma once

#include <algorithm>
#include <type_traits>

#include "internal.h"
#include "stencil.cuh"
#include "stencil_split.cuh"
#include "stencil_tma.cuh"
#include "stencil_tmasplit.cuh"

namespace gfd {

// Tile shapes (BZ x TY threads, VY rows per thread; TILE_* in internal.h).
// Wide tiles for grids whose fastest axis fills a warp, narrow ones for the
// small coarse multigrid levels.

inline int pick_tile(const gfd_operator* op) {
  if (op->R > 2) return TILE_WIDE;
  if (op->n[2] <= 8) return TILE_NARROW;
  if (op->n[2] <= 16) return TILE_MID;
  return TILE_WIDE;
}

struct TileDims {
  int BZ, BY, NT;
};
inline TileDims tile_dims(int tile) {
  switch (tile) {
    case TILE_NARROW: return {8, 8, 64};
    case TILE_MID: return {16, 16, 128};
    case TILE_SHORT: return {32, 8, 128};
    case TILE_SPLIT: return {32, 4 * GFD_SPLIT_VY, 128};
    case TILE_48: return {kTile48Z, 8, 4 * kTile48Z};
    default: return {32, 16, 128};
  }
}

constexpr int kStages = 4;

// Grids up to direct_max_points() (all bands) use the one-thread-per-point
// kernel: the marching kernel's plane pipeline only pays off on larger grids.
inline bool use_direct(const gfd_operator* op, int64_t nin) {
  return (long long)op->n[0] * op->n[1] * op->n[2] * nin <= direct_max_points();
}
inline int direct_blocks(long long total) {
  long long b = (total + 255) / 256;
  long long cap = 8LL * num_sms();
  return int(b < 1 ? 1 : (b > cap ? cap : b));
}

// Raise a kernel's dynamic shared-memory limit when it needs more than 48 KB.
template <class F>
int raise_smem_limit(F* kern, size_t bytes, const char* what) {
  if (bytes <= 48 * 1024) return GFD_OK;
  return check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes),
                    what);
}

struct LaunchGeom {
  dim3 grid;
  int nxc, x_chunk;
  int64_t bands_per_launch;
};

inline LaunchGeom star_geom(const gfd_operator* op, int tile, int64_t nin, int R,
                            int cps = 0) {
  TileDims td = tile_dims(tile);
  LaunchGeom g;
  int gx = (op->n[2] + td.BZ - 1) / td.BZ;
  int gy = (op->n[1] + td.BY - 1) / td.BY;
  int64_t tiles = (int64_t)gx * gy * std::max<int64_t>(nin, 1);
  int64_t target = (int64_t)(cps > 0 ? cps : march_ctas_per_sm()) * num_sms();
  int maxc = std::max(1, op->n[0] / std::max(4, 2 * R));
  int nxc = (int)std::min<int64_t>(maxc, std::max<int64_t>(1, (target + tiles - 1) / tiles));
  g.x_chunk = (op->n[0] + nxc - 1) / nxc;
  g.nxc = (op->n[0] + g.x_chunk - 1) / g.x_chunk;
  g.bands_per_launch = std::max<int64_t>(1, 65535 / g.nxc);
  g.grid = dim3(gx, gy, 1);
  return g;
}

template <class S>
void fill_phases(Phases<S>& P, const double* ph) {
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 2; d++) {
      P.ph[c][d].re = ph ? S(ph[4 * c + 2 * d]) : S(1);
      P.ph[c][d].im = ph ? S(ph[4 * c + 2 * d + 1]) : S(0);
    }
}

template <class V, int R, int BZ, int TY, int VY, int MODE, int S = kStages>
int star_go(const gfd_operator* op, const V* in, V* out, const V* rho, int64_t nin,
            const StarParams<typename vt<V>::S>& base, const LaunchGeom& g, double* partials,
            cudaStream_t s) {
  constexpr size_t smem = star_smem_bytes<BZ, TY, VY, R, S, V, MODE>();
  auto kern = star_kernel<V, R, BZ, TY, VY, S, MODE>;
  int st = raise_smem_limit(kern, smem, "cudaFuncSetAttribute(star_kernel)");
  if (st) return st;
  StarParams<typename vt<V>::S> p = base;
  const long long band = (long long)op->n[0] * op->n[1] * op->n[2];
  for (int64_t b0 = 0; b0 < nin; b0 += g.bands_per_launch) {
    int64_t nb = std::min<int64_t>(g.bands_per_launch, nin - b0);
    dim3 grid(g.grid.x, g.grid.y, (unsigned)(nb * g.nxc));
    p.partials = partials ? partials + b0 * g.nxc * g.grid.x * g.grid.y : nullptr;
    launch_k(kern, grid, BZ * TY, smem, s, in + b0 * band, out + b0 * band,
                                     rho ? rho + b0 * band : nullptr, p);
  }
  return check_launch("star_kernel");
}

// Wide tile: 32 columns x 16 rows; 4 rows per thread for 8-byte and
// smaller values, 2 rows per thread where 4 would exceed the register file
// (16-byte values or radius > 3).
// Complex Jacobi / residual sweeps (the band preconditioner) are built for
// radii up to 3 only, which keeps the number of kernels in check.
constexpr int kMaxComplexRelaxR = 3;

// The short tile exists for complex128 apply (and apply with a potential)
// up to radius 4 (beyond, its 2R + 1 partial sums per row do not fit the
// registers of three CTAs per SM).  It is the built-in choice for those
// launches where the 48-column tile below does not apply: on B200 (the
// 512-band 96^3 Laplace, one box) it measured 3730 GB/s at four CTAs of 128
// threads per SM, against 3120 for the 32 x 16 tile, 3100 for the lane-pair
// kernel and 3270 for its TMA-staged form; three CTAs per SM with up to 170
// registers took it to 3934.
constexpr int kMaxShortR = 4;
template <class V, int R, int MODE>
constexpr bool has_short_tile() {
  return sizeof(V) >= 16 && (MODE == MODE_APPLY || MODE == MODE_POTENTIAL) && R <= kMaxShortR;
}
// The 48-column tile: complex bands (complex128 and complex64), the same
// launches; the built-in choice for both where axis 2 is a multiple of 48.
template <class V, int R, int MODE>
constexpr bool has_tile48() {
  return vt<V>::NC == 2 && (MODE == MODE_APPLY || MODE == MODE_POTENTIAL) && R <= kMaxShortR;
}
// The 48-column tile (TILE_48) covers the same launches where axis 2 is a
// multiple of 48 and is then the built-in choice: 48 x 4 threads with 2
// rows each, two CTAs per SM.  On the 512-band 96^3 Laplace it measured
// 4010-4099 GB/s against 3730-3826 for the short tile at 4 CTAs per SM
// (3934 at 3)
// (apply with a potential: 3610-3750 against 3260-3380).  A 96-column tile
// measured slower at every thread shape tried (2110-3570 GB/s): one CTA per
// SM, or registers short of its 2R + 1 partial sums per row.

template <class V, int R, int MODE>
int star_wide(const gfd_operator* op, int tile, const V* in, V* out, const V* rho, int64_t nin,
              const StarParams<typename vt<V>::S>& p, const LaunchGeom& g, double* partials,
              cudaStream_t s) {
  if constexpr (has_short_tile<V, R, MODE>()) {
    if (tile == TILE_SHORT)
      return star_go<V, R, 32, 4, 2, MODE>(op, in, out, rho, nin, p, g, partials, s);
  }
  if constexpr (has_tile48<V, R, MODE>()) {
    if (tile == TILE_48)
      return star_go<V, R, kTile48Z, 4, 2, MODE>(op, in, out, rho, nin, p, g, partials, s);
  }
  if constexpr (sizeof(V) >= 16 || R > 3)
    return star_go<V, R, 32, 8, 2, MODE>(op, in, out, rho, nin, p, g, partials, s);
  else
    return star_go<V, R, 32, 4, 4, MODE>(op, in, out, rho, nin, p, g, partials, s);
}

template <class V, int MODE>
int star_dispatch(const gfd_operator* op, int tile, const V* in, V* out, const V* rho, int64_t nin,
                  const StarParams<typename vt<V>::S>& p, const LaunchGeom& g, double* partials,
                  cudaStream_t s) {
#define GFD_STAR_SMALL(RR)                                                                   \
  case RR:                                                                                   \
    if (tile == TILE_NARROW)                                                                 \
      return star_go<V, RR, 8, 8, 1, MODE>(op, in, out, rho, nin, p, g, partials, s);        \
    if (tile == TILE_MID)                                                                    \
      return star_go<V, RR, 16, 8, 2, MODE>(op, in, out, rho, nin, p, g, partials, s);       \
    return star_wide<V, RR, MODE>(op, tile, in, out, rho, nin, p, g, partials, s);
#define GFD_STAR_WIDE(RR)                                                                    \
  case RR:                                                                                   \
    if constexpr (RR > kMaxComplexRelaxR && vt<V>::NC == 2 && MODE != MODE_APPLY &&          \
                  MODE != MODE_POTENTIAL)                                                    \
      return set_error(GFD_EUNSUPPORTED, "complex Jacobi/residual sweeps need radius <= 3"); \
    else                                                                                     \
      return star_wide<V, RR, MODE>(op, tile, in, out, rho, nin, p, g, partials, s);
  switch (op->R) {
    GFD_STAR_SMALL(1)
    GFD_STAR_SMALL(2)
    GFD_STAR_WIDE(3)
    GFD_STAR_WIDE(4)
    GFD_STAR_WIDE(5)
    GFD_STAR_WIDE(6)
  }
#undef GFD_STAR_SMALL
#undef GFD_STAR_WIDE
  return set_error(GFD_EUNSUPPORTED, "star stencil radius out of range");
}

// ---------------------------------------------------------------------------
// Complex bands with the real and imaginary parts on lane pairs
// (stencil_split.cuh): 32 x 16 tile, 4 rows x 2 columns per lane, four
// pipeline stages (three with a staged source term), three CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int kSplitVY = GFD_SPLIT_VY, kSplitWY = 4;

// GFD_SPLIT=0 in the environment keeps complex bands on star_kernel (for
// comparisons); the lane-pair kernel is the default.

template <class V>
inline bool split_eligible(const gfd_operator* op) {
  return vt<V>::NC == 2 && op->R >= 1 && op->R <= kSplitMaxR && split_enabled();
}

template <class V, int R, int MODE>
int split_go(const gfd_operator* op, const V* in, V* out, const V* rho, int64_t nin,
             const StarParams<typename vt<V>::S>& p, const LaunchGeom& g, cudaStream_t s) {
  constexpr bool RHO = MODE == MODE_JACOBI || MODE == MODE_RESIDUAL;
  constexpr int S = RHO ? 3 : 4;
  constexpr size_t smem = split_smem_bytes<V, R, kSplitVY, kSplitWY, S, MODE>();
  auto kern = star_split_kernel<V, R, kSplitVY, kSplitWY, S, MODE>;
  int st = raise_smem_limit(kern, smem, "cudaFuncSetAttribute(star_split_kernel)");
  if (st) return st;
  if ((st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            int(cudaSharedmemCarveoutMaxShared)),
                       "cudaFuncSetAttribute(carveout)")))
    return st;
  const long long band = (long long)op->n[0] * op->n[1] * op->n[2];
  for (int64_t b0 = 0; b0 < nin; b0 += g.bands_per_launch) {
    int64_t nb = std::min<int64_t>(g.bands_per_launch, nin - b0);
    dim3 grid(g.grid.x, g.grid.y, (unsigned)(nb * g.nxc));
    launch_k(kern, grid, 32 * kSplitWY, smem, s, in + b0 * band, out + b0 * band,
             rho ? rho + b0 * band : nullptr, p);
  }
  return check_launch("star_split_kernel");
}

template <class V, int MODE>
int split_dispatch(const gfd_operator* op, const V* in, V* out, const V* rho, int64_t nin,
                   const StarParams<typename vt<V>::S>& p, const LaunchGeom& g, cudaStream_t s) {
  if constexpr (vt<V>::NC == 2) {
    switch (op->R) {
      case 1: return split_go<V, 1, MODE>(op, in, out, rho, nin, p, g, s);
      case 2: return split_go<V, 2, MODE>(op, in, out, rho, nin, p, g, s);
      case 3: return split_go<V, 3, MODE>(op, in, out, rho, nin, p, g, s);
    }
  }
  return set_error(GFD_EUNSUPPORTED, "lane-pair stencil: complex bands, radius <= 3");
}

// ---------------------------------------------------------------------------
// complex128 bands on full-row tiles staged by TMA, real and imaginary parts
// on lane pairs (stencil_tmasplit.cuh).  Takes grids up to 128 columns
// (32 ng, ng <= kTsMaxNG) whose rows tile evenly along a periodic axis 1, and
// a potential only on an even number of columns (its rows must start on a
// 16-byte boundary).
// ---------------------------------------------------------------------------
}  // namespace gfd
GFD_DECLARE_TS_ENTRY(1)
GFD_DECLARE_TS_ENTRY(2)
GFD_DECLARE_TS_ENTRY(3)
GFD_DECLARE_TS_ENTRY(4)
namespace gfd {

inline int ts_ng(const gfd_operator* op) { return (op->n[2] + 31) / 32; }

template <class V>
inline bool ts_eligible(const gfd_operator* op, int mode, const void* in, const void* rho) {
  if constexpr (!std::is_same_v<V, cplx<double>>) {
    return false;
  } else {
    if (!tmasplit_enabled() || op->R < 1 || op->R > kSplitMaxR) return false;
    if (ts_ng(op) > kTsMaxNG) return false;
    if (op->per[1] && op->n[1] % kTsBY) return false;
    if (mode == OP_POTENTIAL && (op->n[2] & 1)) return false;
    auto aligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    return aligned(in) && (!rho || aligned(rho));
  }
}

inline int ts_dispatch(const gfd_operator* op, int kmode, const cplx<double>* in,
                       cplx<double>* out, const cplx<double>* rho, const void* pot, int64_t nin,
                       const StarParams<double>& p, int cps, cudaStream_t s) {
  switch (ts_ng(op)) {
    case 1: return ts_launch_1(op, kmode, in, out, rho, pot, nin, p, cps, s);
    case 2: return ts_launch_2(op, kmode, in, out, rho, pot, nin, p, cps, s);
    case 3: return ts_launch_3(op, kmode, in, out, rho, pot, nin, p, cps, s);
    case 4: return ts_launch_4(op, kmode, in, out, rho, pot, nin, p, cps, s);
  }
  return set_error(GFD_EUNSUPPORTED, "TMA lane-pair stencil: at most 128 columns");
}

// ---------------------------------------------------------------------------
// TMA-fed kernel (stencil_tma.cuh): complex128 apply on grids whose plane
// holds whole 16 x 32 tiles along periodic axes (zero-boundary axes may end
// in a partial tile: the loads fill zeros past the edge).
// ---------------------------------------------------------------------------
constexpr int kTmaVY = 2, kTmaG = 8, kTmaBY = kTmaVY * kTmaG, kTmaStages = 8;

// Defined in operator.cu.
bool star_tma_enabled();
int* star_error_flag();
int encode_tma_maps(TmaMaps* maps, const void* base, const gfd_operator* op, int64_t nb, int R,
                    int by);

inline bool tma_eligible(const gfd_operator* op, const void* in) {
  if (!star_tma_enabled() || op->R < 1 || op->R > 3) return false;
  if (op->n[2] < kTmaBZ || op->n[1] < kTmaBY) return false;
  if (op->per[2] && op->n[2] % kTmaBZ) return false;
  if (op->per[1] && op->n[1] % kTmaBY) return false;
  return (reinterpret_cast<uintptr_t>(in) & 15) == 0;
}

template <int R>
int star_tma_go(const gfd_operator* op, const cplx<double>* in, cplx<double>* out, int64_t nin,
                const StarParams<double>& base, const LaunchGeom& g, cudaStream_t s) {
  constexpr size_t smem = star_tma_smem_bytes<R, kTmaBY, kTmaStages>();
  auto kern = star_tma_kernel<R, kTmaVY, kTmaG, kTmaStages>;
  int st = raise_smem_limit(kern, smem, "cudaFuncSetAttribute(star_tma_kernel)");
  if (st) return st;
  // Two CTAs per SM need the largest shared-memory carveout.
  if ((st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            int(cudaSharedmemCarveoutMaxShared)),
                       "cudaFuncSetAttribute(carveout)")))
    return st;
  int* err = star_error_flag();
  if (!err) return GFD_ECUDA;
  TmaMaps maps;
  if ((st = encode_tma_maps(&maps, in, op, nin, R, kTmaBY))) return st;
  const long long band = (long long)op->n[0] * op->n[1] * op->n[2];
  for (int64_t b0 = 0; b0 < nin; b0 += g.bands_per_launch) {
    int64_t nb = std::min<int64_t>(g.bands_per_launch, nin - b0);
    dim3 grid(g.grid.x, g.grid.y, (unsigned)(nb * g.nxc));
    launch_k(kern, grid, 32 * kTmaG, smem, s, out + b0 * band, base, maps, (int)b0, err);
  }
  return check_launch("star_tma_kernel");
}

inline int star_tma_dispatch(const gfd_operator* op, const cplx<double>* in, cplx<double>* out,
                             int64_t nin, const StarParams<double>& p, const LaunchGeom& g,
                             cudaStream_t s) {
  switch (op->R) {
    case 1: return star_tma_go<1>(op, in, out, nin, p, g, s);
    case 2: return star_tma_go<2>(op, in, out, nin, p, g, s);
    case 3: return star_tma_go<3>(op, in, out, nin, p, g, s);
  }
  return set_error(GFD_EUNSUPPORTED, "TMA stencil radius out of range");
}

template <class V, int MODE>
int direct_dispatch(const gfd_operator* op, const V* in, V* out, const V* rho,
                    const StarParams<typename vt<V>::S>& p, long long total, cudaStream_t s) {
  const int blocks = direct_blocks(total);
  if constexpr (vt<V>::NC == 2 && MODE != MODE_APPLY && MODE != MODE_POTENTIAL) {
    switch (op->R) {
      case 1: launch_k(star_direct_kernel<V, 1, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
      case 2: launch_k(star_direct_kernel<V, 2, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
      case 3: launch_k(star_direct_kernel<V, 3, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
      default: return set_error(GFD_EUNSUPPORTED, "complex Jacobi/residual sweeps need radius <= 3");
    }
    return check_launch("star_direct_kernel");
  }
  switch (op->R) {
    case 1: launch_k(star_direct_kernel<V, 1, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
    case 2: launch_k(star_direct_kernel<V, 2, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
    case 3: launch_k(star_direct_kernel<V, 3, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
    case 4: launch_k(star_direct_kernel<V, 4, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
    case 5: launch_k(star_direct_kernel<V, 5, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
    case 6: launch_k(star_direct_kernel<V, 6, MODE>, blocks, 256, 0, s, in, out, rho, p, total); break;
    default: return set_error(GFD_EUNSUPPORTED, "star stencil radius out of range");
  }
  return check_launch("star_direct_kernel");
}

// Stencil parameters of a star operator for one mode (weights in the
// element precision S; Jacobi folds (1 - w) phi into the centre weight, see
// star_kernel, and the negated sweep flips the sign of w / c0, exactly).
template <class S>
void star_params(const gfd_operator* op, int mode, double w, const double* phase_cd,
                 StarParams<S>& p) {
  p = StarParams<S>{};
  p.n0 = op->n[0]; p.n1 = op->n[1]; p.n2 = op->n[2];
  p.per0 = op->per[0]; p.per1 = op->per[1]; p.per2 = op->per[2];
  p.band = (long long)op->n[0] * op->n[1] * op->n[2];
  p.c0 = S(op->c0);
  for (int i = 0; i < 2 * kMaxR + 1; i++) {
    p.cx[i] = S(op->cx[i]);
    p.cy[i] = S(op->cy[i]);
    p.cz[i] = S(op->cz[i]);
  }
  if (mode == OP_JACOBI || mode == OP_JACOBI_NEG) {
    p.c0 = S(-(1.0 - w) * op->c0 / w);
    p.wc = S(w / op->c0);
    if (mode == OP_JACOBI_NEG) p.wc = -p.wc;
  }
  fill_phases(p.P, phase_cd);
  p.fix_yz = 0;
  if (phase_cd)
    for (int c = 1; c < 3; c++)
      for (int d = 0; d < 2; d++)
        if (op->per[c] && (phase_cd[4 * c + 2 * d] != 1.0 || phase_cd[4 * c + 2 * d + 1] != 0.0))
          p.fix_yz = 1;
}

template <class V>
int launch_star_typed(const gfd_operator* op, int mode, const void* in, void* out, const void* rho,
                      int64_t nin, const double* phase_cd, double w, double* partials,
                      cudaStream_t s) {
  using S = typename vt<V>::S;
  StarParams<S> p;
  star_params(op, mode, w, phase_cd, p);
  const V* vin = static_cast<const V*>(in);
  V* vout = static_cast<V*>(out);
  const V* vrho = static_cast<const V*>(rho);
  const bool relax_mode = mode == OP_JACOBI || mode == OP_JACOBI_NEG || mode == OP_RESIDUAL;
  if constexpr (vt<V>::NC == 2) {
    if (relax_mode && op->R > kMaxComplexRelaxR)
      return set_error(GFD_EUNSUPPORTED, "complex Jacobi/residual sweeps need radius <= 3");
  }
  if (mode == OP_POTENTIAL) p.pot = rho;  // the potential travels as the source argument
  TunePlan plan;
  const bool tuned =
      mode != OP_RESIDUAL && tune_lookup(star_tune_key(op, dtype_of<V>(), mode, nin), &plan);
  if (tuned ? plan.path == PLAN_DIRECT : use_direct(op, nin)) {
    p.partials = partials;
    const long long total = (long long)p.band * nin;
    if (mode == OP_POTENTIAL)
      return direct_dispatch<V, MODE_POTENTIAL>(op, vin, vout, nullptr, p, total, s);
    if (mode == OP_JACOBI || mode == OP_JACOBI_NEG)
      return direct_dispatch<V, MODE_JACOBI>(op, vin, vout, vrho, p, total, s);
    if (mode == OP_RESIDUAL)
      return direct_dispatch<V, MODE_RESIDUAL>(op, vin, vout, vrho, p, total, s);
    return direct_dispatch<V, MODE_APPLY>(op, vin, vout, nullptr, p, total, s);
  }
  if constexpr (std::is_same_v<V, cplx<double>>) {
    if (!tuned && mode == OP_APPLY && tma_eligible(op, in)) {
      LaunchGeom g = star_geom(op, TILE_WIDE, nin, op->R);
      p.nxc = g.nxc;
      p.x_chunk = g.x_chunk;
      return star_tma_dispatch(op, vin, vout, nin, p, g, s);
    }
  }
  // Radii above 2 have the wide tile only (and the short one for complex128
  // apply); complex bands up to radius 3 have the lane-pair tile, their
  // built-in choice wherever the wide tile would be picked.  Any other plan
  // tile falls back to the built-in choice, so the geometry always matches
  // the kernel launched.
  int tile = pick_tile(op);
  const bool split = split_eligible<V>(op);
  const bool tsplit = ts_eligible<V>(op, mode, in, rho);
  const bool shortok =
      sizeof(V) >= 16 && (mode == OP_APPLY || mode == OP_POTENTIAL) && op->R <= kMaxShortR;
  const bool t48ok = vt<V>::NC == 2 && (mode == OP_APPLY || mode == OP_POTENTIAL) &&
                     op->R <= kMaxShortR && tile48_eligible(op);
  if (shortok && tile == TILE_WIDE) tile = tile48_eligible(op) ? TILE_48 : TILE_SHORT;
  // complex64 (512-band 96^3 Laplace): 2970-2990 GB/s against 2905-2918 for
  // the 32 x 16 tile
  if (t48ok && !shortok && tile == TILE_WIDE) tile = TILE_48;
  if (tuned) {
    if (plan.tile == TILE_SHORT)
      tile = shortok ? TILE_SHORT : tile;
    else if (plan.tile == TILE_48)
      tile = t48ok ? TILE_48 : tile;
    else if (plan.tile == TILE_TMASPLIT)
      tile = tsplit ? TILE_TMASPLIT : tile;
    else if (plan.tile == TILE_SPLIT)
      tile = split ? TILE_SPLIT : tile;
    else if (op->R <= 2 || plan.tile == TILE_WIDE)
      tile = plan.tile;
  }
  if constexpr (std::is_same_v<V, cplx<double>>) {
    if (tile == TILE_TMASPLIT) {
      const int cps = tuned ? plan.cps : 0;
      if (mode == OP_POTENTIAL)
        return ts_dispatch(op, MODE_POTENTIAL, vin, vout, nullptr, rho, nin, p, cps, s);
      if (mode == OP_JACOBI || mode == OP_JACOBI_NEG)
        return ts_dispatch(op, MODE_JACOBI, vin, vout, vrho, nullptr, nin, p, cps, s);
      if (mode == OP_RESIDUAL)
        return ts_dispatch(op, MODE_RESIDUAL, vin, vout, vrho, nullptr, nin, p, cps, s);
      return ts_dispatch(op, MODE_APPLY, vin, vout, nullptr, nullptr, nin, p, cps, s);
    }
  }
  LaunchGeom g = star_geom(op, tile, nin, op->R, tuned ? plan.cps : 0);
  p.nxc = g.nxc;
  p.x_chunk = g.x_chunk;
  if (tile == TILE_SPLIT) {
    if (mode == OP_POTENTIAL)
      return split_dispatch<V, MODE_POTENTIAL>(op, vin, vout, nullptr, nin, p, g, s);
    if (mode == OP_JACOBI || mode == OP_JACOBI_NEG)
      return split_dispatch<V, MODE_JACOBI>(op, vin, vout, vrho, nin, p, g, s);
    if (mode == OP_RESIDUAL)
      return split_dispatch<V, MODE_RESIDUAL>(op, vin, vout, vrho, nin, p, g, s);
    return split_dispatch<V, MODE_APPLY>(op, vin, vout, nullptr, nin, p, g, s);
  }
  if (mode == OP_POTENTIAL)
    return star_dispatch<V, MODE_POTENTIAL>(op, tile, vin, vout, nullptr, nin, p, g, nullptr, s);
  if (mode == OP_JACOBI || mode == OP_JACOBI_NEG)
    return star_dispatch<V, MODE_JACOBI>(op, tile, vin, vout, vrho, nin, p, g, nullptr, s);
  if (mode == OP_RESIDUAL)
    return star_dispatch<V, MODE_RESIDUAL>(op, tile, vin, vout, vrho, nin, p, g, partials, s);
  return star_dispatch<V, MODE_APPLY>(op, tile, vin, vout, nullptr, nin, p, g, nullptr, s);
}

template <class V, int MODE>
int general_go(const gfd_operator* op, const V* in, V* out, const V* rho, int64_t nin,
               GenParams<typename vt<V>::S>& p, double* partials, cudaStream_t s) {
  constexpr int BZ = 32, TY = 4, VY = 2, BY = TY * VY;
  const int mp = std::max(op->mp, 0);
  const int gx = (op->n[2] + BZ - 1) / BZ, gy = (op->n[1] + BY - 1) / BY;
  gfd_operator tmp = *op;
  tmp.scratch = nullptr;  // geometry only
  LaunchGeom g = star_geom(op, TILE_WIDE, nin, std::max(mp, 1));
  g.grid = dim3(gx, gy, 1);
  p.nxc = g.nxc;
  p.x_chunk = g.x_chunk;
  size_t smem = (size_t)(2 * mp + 1) * (BY + 2 * mp) * (BZ + 2 * mp) * sizeof(V);
  if (smem > 227 * 1024) return set_error(GFD_EUNSUPPORTED, "stencil range too large");
  cudaError_t e = cudaFuncSetAttribute(general_kernel<V, BZ, TY, VY, MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(general_kernel)");
  const long long band = (long long)op->n[0] * op->n[1] * op->n[2];
  for (int64_t b0 = 0; b0 < nin; b0 += g.bands_per_launch) {
    int64_t nb = std::min<int64_t>(g.bands_per_launch, nin - b0);
    dim3 grid(gx, gy, (unsigned)(nb * g.nxc));
    p.partials = partials ? partials + b0 * g.nxc * gx * gy : nullptr;
    launch_k(general_kernel<V, BZ, TY, VY, MODE>, grid, BZ * TY, smem, s, 
        in + b0 * band, out + b0 * band, rho ? rho + b0 * band : nullptr, p, mp);
  }
  return check_launch("general_kernel");
}

template <class V>
int launch_general_typed(const gfd_operator* op, int mode, const void* in, void* out,
                         const void* rho, int64_t nin, const double* phase_cd, double w,
                         double* partials, cudaStream_t s) {
  using S = typename vt<V>::S;
  if (op->ncoefs > kMaxCoefs) return set_error(GFD_EUNSUPPORTED, "too many stencil coefficients");
  GenParams<S> p{};
  p.n0 = op->n[0]; p.n1 = op->n[1]; p.n2 = op->n[2];
  p.per0 = op->per[0]; p.per1 = op->per[1]; p.per2 = op->per[2];
  p.band = (long long)op->n[0] * op->n[1] * op->n[2];
  p.ncoefs = op->ncoefs;
  for (int c = 0; c < op->ncoefs; c++) {
    p.coefs[c] = S(op->coefs[c]);
    for (int a = 0; a < 3; a++) p.off[c][a] = (signed char)op->off[3 * c + a];
  }
  p.w = S(w);
  p.sign = mode == OP_JACOBI_NEG ? S(-1) : S(1);
  fill_phases(p.P, phase_cd);
  const V* vin = static_cast<const V*>(in);
  V* vout = static_cast<V*>(out);
  const V* vrho = static_cast<const V*>(rho);
  if (mode == OP_JACOBI || mode == OP_JACOBI_NEG)
    return general_go<V, MODE_JACOBI>(op, vin, vout, vrho, nin, p, nullptr, s);
  if (mode == OP_RESIDUAL)
    return general_go<V, MODE_RESIDUAL>(op, vin, vout, vrho, nin, p, partials, s);
  if (mode != OP_APPLY) return set_error(GFD_EUNSUPPORTED, "mode not available for this stencil");
  return general_go<V, MODE_APPLY>(op, vin, vout, nullptr, nin, p, nullptr, s);
}

inline int64_t partials_count(const gfd_operator* op, int64_t nin) {
  if (op->star && use_direct(op, nin))
    return direct_blocks((long long)op->n[0] * op->n[1] * op->n[2] * nin);
  if (op->star) {
    int tile = pick_tile(op);
    TileDims td = tile_dims(tile);
    LaunchGeom g = star_geom(op, tile, nin, op->R);
    int gx = (op->n[2] + td.BZ - 1) / td.BZ, gy = (op->n[1] + td.BY - 1) / td.BY;
    return (int64_t)gx * gy * g.nxc * nin;
  }
  const int BZ = 32, BY = 8;
  LaunchGeom g = star_geom(op, TILE_WIDE, nin, std::max(op->mp, 1));
  int gx = (op->n[2] + BZ - 1) / BZ, gy = (op->n[1] + BY - 1) / BY;
  return (int64_t)gx * gy * g.nxc * nin;
}

// Stencil parameters of a Gauss-Seidel colour pass (any offset set).
template <class S>
void gs_params(const gfd_operator* op, GenParams<S>& p) {
  p = GenParams<S>{};
  p.n0 = op->n[0]; p.n1 = op->n[1]; p.n2 = op->n[2];
  p.per0 = op->per[0]; p.per1 = op->per[1]; p.per2 = op->per[2];
  p.band = (long long)op->n[0] * op->n[1] * op->n[2];
  p.ncoefs = op->ncoefs;
  for (int c = 0; c < op->ncoefs; c++) {
    p.coefs[c] = S(op->coefs[c]);
    for (int a = 0; a < 3; a++) p.off[c][a] = (signed char)op->off[3 * c + a];
  }
}

template <class V>
int gs_typed(const gfd_operator* op, V* phi, const V* rho, int nsweeps, V* frozen, int ncolor,
             cudaStream_t s) {
  using S = typename vt<V>::S;
  GenParams<S> p;
  gs_params(op, p);
  const long long n = p.band;
  const bool any_per = op->per[0] || op->per[1] || op->per[2];
  const long long nq = (long long)op->n[0] * op->n[1] * gs_row_slots(op->n[2], ncolor);
  int blocks = (int)std::min<long long>((nq + 255) / 256, 148LL * 16);
  for (int sw = 0; sw < nsweeps; sw++) {
    if (any_per) {
      cudaError_t e = cudaMemcpyAsync(frozen, phi, n * sizeof(V), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return check_cuda(e, "cudaMemcpyAsync(frozen)");
    }
    for (int c = 0; c < ncolor; c++)
      launch_k(color_gs_kernel<V>, blocks, 256, 0, s, phi, rho, any_per ? frozen : phi, p, ncolor, c);
  }
  return check_launch("color_gs_kernel");
}

}  // namespace gfd

// One of these per element type, defined in stencil_<type>.cu.
#define GFD_DECLARE_STENCIL_ENTRY(NAME)                                                        \
  namespace gfd {                                                                             \
  int star_##NAME(const gfd_operator*, int, const void*, void*, const void*, int64_t,          \
                  const double*, double, double*, cudaStream_t);                              \
  int general_##NAME(const gfd_operator*, int, const void*, void*, const void*, int64_t,       \
                     const double*, double, double*, cudaStream_t);                           \
  }
