// internal.h -- handle layouts and launchers shared by the C-ABI entry points
// of libgpawfd (host code only).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <tuple>
#include <vector>

#include "gpaw_fd.h"

struct gfd_operator {
  int ncoefs = 0;
  std::vector<double> coefs;
  std::vector<int> off;  // ncoefs x 3
  int n[3] = {0, 0, 0};
  int mp = 0;            // halo width (largest |offset| component)
  int per[3] = {0, 0, 0};
  int real = 1;
  int cfd = 1;
  // Axis-aligned decomposition (star stencils).
  bool star = false;
  int R = 0;
  double c0 = 0.0;
  double cx[13] = {0}, cy[13] = {0}, cz[13] = {0};  // index 6 + k
  double diag = 0.0;     // weight of the zero offset
  // Device scratch of one grid for relaxation (Jacobi ping-pong / frozen
  // copy for periodic Gauss-Seidel), allocated on first use.
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  int device = -1;
};

struct gfd_transformer {
  int nin[3] = {0, 0, 0};
  int nout[3] = {0, 0, 0};
  int k = 2, nn = 1;
  int pad[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int skip[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int per[3] = {0, 0, 0};
  int real = 1;
  int interpolate = 0;
};

namespace gfd {

enum { OP_APPLY = 0, OP_JACOBI = 1, OP_RESIDUAL = 2, OP_POTENTIAL = 3, OP_JACOBI_NEG = 4 };

int num_sms();

// ---------------------------------------------------------------------------
// Launch plans (autotune.cu).  A plan fixes, for one kernel family, element
// type, mode, grid, stencil radius (or transfer order), boundary conditions
// and band-count class, the kernel form and the axis-0 split.  Launches use
// the cached plan when there is one and the built-in rules otherwise.
// ---------------------------------------------------------------------------
// Marching tiles 32 / 16 / 8 columns wide; TILE_SHORT: 32 columns by 8 rows
// (complex128 apply up to radius 4 only: 128 threads, three CTAs per SM).
// TILE_SPLIT: complex bands, radius <= 3, real and imaginary parts on lane
// pairs (star_split_kernel): 32 columns by 16 rows, 128 threads.
// TILE_TMASPLIT: complex128, radius <= 3, the same lane pairs on full-row
// tiles of 8 rows staged by TMA (star_tmasplit_kernel).
// TILE_48: complex apply (and apply with a potential) up to radius 4,
// 48 columns by 8 rows (48 x 4 threads, 2 rows each, two CTAs per SM), for
// axis-2 lengths that are multiples of 48: it stages 2R halo columns per 48
// where the 32-column tiles stage 2R per 32.
enum {
  TILE_WIDE = 0,
  TILE_MID = 1,
  TILE_NARROW = 2,
  TILE_SHORT = 3,
  TILE_SPLIT = 4,
  TILE_TMASPLIT = 5,
  TILE_48 = 6
};
inline bool tile48_eligible(const gfd_operator* op) {
  return op->star && op->R >= 1 && op->R <= 4 && op->n[2] % 48 == 0;
}
enum { PLAN_DIRECT = 0, PLAN_MARCH = 1 };               // one thread per point / marching
enum { TK_STAR = 0, TK_RESTRICT = 1, TK_INTERP = 2 };

struct TuneKey {
  int kind, dtype, mode, n0, n1, n2, order, per, nbc;
  bool operator<(const TuneKey& o) const {
    return std::tie(kind, dtype, mode, n0, n1, n2, order, per, nbc) <
           std::tie(o.kind, o.dtype, o.mode, o.n0, o.n1, o.n2, o.order, o.per, o.nbc);
  }
};
struct TunePlan {
  int path = PLAN_MARCH;
  int tile = TILE_WIDE;
  int cps = 4;       // target CTAs per SM of the axis-0 split
  double us = 0.0;   // measured time per launch
};
// Star operator launch of nin bands in mode OP_APPLY / OP_JACOBI(_NEG) /
// OP_POTENTIAL (residual sweeps keep the built-in rules: the Poisson solver
// sizes its partial-sum buffer from them).
TuneKey star_tune_key(const gfd_operator* op, int dtype, int mode, int64_t nin);
TuneKey tr_tune_key(const gfd_transformer* tr, int dtype, int64_t nin);
// The plan of an autotune run in progress on this thread, else the cached
// one; false: no plan, use the built-in rules.
bool tune_lookup(const TuneKey& k, TunePlan* plan);

// Stencil launch.  mode OP_APPLY: out = L in.  OP_JACOBI: out = Jacobi update
// of in with source rho and weight w.  OP_RESIDUAL: out = L in - rho and, if
// partials != nullptr, one sum of squares per CTA into partials.
// OP_JACOBI_NEG: minus the Jacobi update (exact sign flip).  Complex dtypes
// support the Jacobi / residual modes for radius <= 3.
// OP_POTENTIAL (star operators only): out = L in + v in with the real grid v
// (float64 for float64/complex128 bands, float32 otherwise) passed as rho.
// in/out/rho point to nin bands.  phase_cd: 12 doubles (host) or nullptr.
int op_launch(const gfd_operator* op, int dtype, int mode, const void* in, void* out,
              const void* rho, int64_t nin, const double* phase_cd, double w,
              double* partials, cudaStream_t s);
// Number of partial sums op_launch(OP_RESIDUAL) writes for nin bands.
int64_t op_partials(const gfd_operator* op, int dtype, int mode, int64_t nin);

// Multicolour Gauss-Seidel sweeps (real).  frozen: scratch of one grid.
int op_gs_sweeps(const gfd_operator* op, int dtype, void* phi, const void* rho, int nsweeps,
                 void* frozen, cudaStream_t s);
int op_gs_colors(const gfd_operator* op);

int tr_launch(const gfd_transformer* tr, int dtype, const void* in, void* out, int64_t nin,
              const double* phases, cudaStream_t s);
// Restriction of one real band that also writes seed = seed_scale * out
// (the first weighted-Jacobi sweep of the coarse level from a zero guess).
int tr_launch_seed(const gfd_transformer* tr, int dtype, const void* in, void* out, void* seed,
                   double seed_scale, cudaStream_t s);
// General form: out = out_scale * transfer(in) (interpolation with base:
// out = base - out_scale * interpolate(in)); restriction with seed also
// writes seed = seed_scale * out.  out_scale must be 1 or -1 (exact).
int tr_launch_ex(const gfd_transformer* tr, int dtype, const void* in, void* out,
                 const void* base, int64_t nin, const double* phases, double out_scale,
                 void* seed, double seed_scale, cudaStream_t s);
// Interpolation with the correction fused: out = base - interpolate(in)
// (in place when base == out).
int tr_launch_sub(const gfd_transformer* tr, int dtype, const void* in, void* out,
                  const void* base, int64_t nin, const double* phases, cudaStream_t s);

// Deterministic sum of n elements (float64 or float32 by dtype), SQUARE for
// the sum of squares; result (device) = scale * sum.  partials needs
// kRedBlocks doubles.
int reduce_launch(int dtype, const void* a, int64_t n, bool square, double scale,
                  double* partials, double* result, cudaStream_t s);
int final_sum_launch(const double* partials, int n, double scale, double* result,
                     cudaStream_t s);
int axpby_launch(int ydtype, void* y, int xdtype, const void* x, double a, double b, int64_t n,
                 cudaStream_t s);
int sub_const_launch(int dtype, void* y, const void* x, double c, int64_t n, cudaStream_t s);
// y = convert(x); with seed != nullptr also seed = seed_scale * y.
int convert_launch(int ydtype, void* y, int xdtype, const void* x, int64_t n, cudaStream_t s,
                   void* seed = nullptr, double seed_scale = 0.0);
int zero_launch(int dtype, void* y, int64_t n, cudaStream_t s);
// out[b][i] += v[i] * in[b][i] over nin bands of n points (v real: float64
// for float64/complex128, float32 otherwise).
int add_potential_launch(int dtype, void* out, const void* in, const void* v, int64_t n,
                         int64_t nin, cudaStream_t s);

}  // namespace gfd
