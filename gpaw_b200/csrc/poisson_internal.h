// poisson_internal.h -- the Poisson solver's handle, level hierarchy and
// solve controls, shared by poisson.cu (single solves and graph branches)
// and poisson_group.cu (grouped batches).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"

struct Level {
  gfd_operator* op = nullptr;
  int64_t n = 0;
  void* phi[2] = {nullptr, nullptr};
  void* rho = nullptr;
  void* res = nullptr;
  int pre = 0, post = 0;
  double w = 1.0;
};

// Solve controls shared by host and device.  The host writes the inputs
// (up to `charge`) before each launch and reads the outputs after it.
struct SolveCtrl {
  double eps;
  double maxcharge;
  double charge_arg;  // NaN: use the integral of rho
  int maxiter;
  int zero_init;      // charged branches start from phi = 0 (zero_initial_phi)
  const double* rho_gauss;  // L = 0 Gaussian of the non-periodic charged branch (or null)
  const double* phi_gauss;  // its potential
  double madelung;    // periodic charged branch: potential shift per unit charge (NaN: unset)
  int bc_kind;        // kBcPeriodic, kBcNone or kBcMixed (level-0 boundary conditions)
  int skip;           // an unused batch slot: no solve
  double charge;      // integral of rho times dv
  double bg;          // background charge density removed from rho
  double gq;          // non-periodic charged branch: the Gaussian's weight (charge / sqrt(4 pi))
  double shift;       // periodic charged branch: charge * madelung, added to phi
  double err;         // last residual norm sum(r^2) dv
  double sum;         // scratch scalar (sum of phi)
  int niter;
  int status;         // GFD_OK, GFD_EUNSUPPORTED (refused), GFD_ENEEDGAUSS
};

enum { kBcMixed = 0, kBcPeriodic = 1, kBcNone = 2 };

struct gfd_poisson {
  int levels = 0;
  std::vector<gfd_transformer*> restr, interp;
  int relax_method = GFD_RELAX_JACOBI;
  double dv = 1.0;
  int pbc_all = 0;
  int precision = GFD_POISSON_FP64;
  std::vector<Level> L;     // hierarchy in the V-cycle precision
  int vdtype = GFD_FLOAT64; // dtype of the V-cycle arrays
  // Float64 fine-grid arrays: the caller's rho and phi are copied here.
  double* rho_in = nullptr;
  double* phi64 = nullptr;  // mixed form: the float64 potential
  double* rho64 = nullptr;  // mixed form: rho - background
  double* r64 = nullptr;    // mixed form: float64 residual
  double* partials = nullptr;
  int64_t npartials = 0;
  SolveCtrl* dctrl = nullptr;
  SolveCtrl* hctrl = nullptr;  // pinned
  void* pool = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = -1;
  gfd_operator* B = nullptr;  // Mehrstellen right-hand side (not owned)
  int bc_kind = kBcMixed;
  // Charged branches (gpaw/poisson.py:139-191): the L = 0 Gaussian and its
  // potential on the level-0 grid (owned, allocated by gfd_poisson_load_gauss)
  // and the Madelung shift per unit charge (NaN until set).
  double* rho_gauss = nullptr;
  double* phi_gauss = nullptr;
  double madelung = 0.0;
  int zero_init = 0;
};

namespace gfd {

// Whether level l's first relaxation acts on a zero guess that the kernel
// writing its rho can seed, and the seed's scale (w / c0).
bool poisson_seedable(const gfd_poisson* ps, int l);
double poisson_seed_scale(const Level& lv);
// One solve's prologue on stream s: the charge integral, the controls
// (background, charged status; the loop conditional is left alone) and the
// level-0 source rho - background (B applied for Mehrstellen).
int poisson_prologue(gfd_poisson* ps, cudaStream_t s);
// Epilogue: the zero-mean potential of fully periodic systems.
int poisson_epilogue(gfd_poisson* ps, cudaStream_t s);

// Grouped solves (poisson_group.cu): solvers of one structure (levels,
// smoothing, weights, stencil radii or colourings, boundary conditions,
// transfer orders; float64, no Mehrstellen right-hand side) whose V-cycle
// steps run as one launch per step over all their grids.
struct PoissonGroup;
bool group_eligible(const gfd_poisson* ps);
bool group_same_structure(const gfd_poisson* a, const gfd_poisson* b, std::string* why);
int group_create(gfd_poisson* const* solvers, int n, PoissonGroup** out);
void group_destroy(PoissonGroup* g);
// On a capturing stream: the per-solve prologues, a `while` node (its body
// graph and handle returned, to fill after the outer capture ends) and the
// epilogues.
int group_capture_outer(PoissonGroup* g, cudaStream_t cs, cudaGraph_t* body,
                        cudaGraphConditionalHandle* loop);
int group_capture_body(PoissonGroup* g, cudaStream_t cs, cudaGraph_t body,
                       cudaGraphConditionalHandle loop);

}  // namespace gfd
