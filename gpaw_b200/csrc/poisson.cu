// poisson.cu -- gfd_poisson_*: the multigrid Poisson solver of
// gpaw/poisson.py:21-276 with the whole level hierarchy resident on the GPU.
//
// V-cycle (PoissonSolver.iterate2, gpaw/poisson.py:245-276), level l < L:
//   relax(presmooths[l]); r = L_l phi_l - rho_l; rho_{l+1} = restrict(r);
//   phi_{l+1} = 0; iterate2(l+1); phi_l -= interpolate(phi_{l+1});
// then relax(postsmooths[l]) and, on level 0, the residual norm
// sum(r^2) dv.  Weighted Jacobi sweeps ping-pong between two buffers per
// level, so no copy is needed between sweeps.
//
// GFD_POISSON_MIXED: defect correction.  The V-cycle is a linear iteration
// phi <- phi + B (rho - L phi), so running it in float32 on the defect
// (phi = 0, rho = L phi - rho) and subtracting the result from the float64
// phi gives the float64 iterate up to float32 rounding of the correction;
// the residual, the update and the norm stay float64.
#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "util.cuh"

namespace {

struct Level {
  gfd_operator* op = nullptr;
  int64_t n = 0;
  void* phi[2] = {nullptr, nullptr};  // level 0 (FP64 form): phi[0] is the caller's array
  int cur = 0;
  void* rho = nullptr;
  void* res = nullptr;
  int pre = 0, post = 0;
  double w = 1.0;
};

}  // namespace

struct gfd_poisson {
  int levels = 0;
  std::vector<gfd_transformer*> restr, interp;
  int relax_method = GFD_RELAX_JACOBI;
  double dv = 1.0;
  int pbc_all = 0;
  int precision = GFD_POISSON_FP64;
  std::vector<Level> L;     // hierarchy in the V-cycle precision
  int vdtype = GFD_FLOAT64; // dtype of the V-cycle arrays
  // Mixed form: float64 fine-grid residual and alternate phi.
  void* r64 = nullptr;
  void* phi64_alt = nullptr;
  double* partials = nullptr;
  int64_t npartials = 0;
  double* dscal = nullptr;  // device scalars: [0] err, [1] sum
  double* hscal = nullptr;  // pinned host mirror
  void* pool = nullptr;
};

namespace gfd {

static int relax_level(gfd_poisson* ps, Level& lv, int nsweeps, cudaStream_t s) {
  if (nsweeps <= 0) return GFD_OK;
  if (ps->relax_method == GFD_RELAX_GS)
    return op_gs_sweeps(lv.op, ps->vdtype, lv.phi[lv.cur], lv.rho, nsweeps, lv.phi[1 - lv.cur], s);
  for (int k = 0; k < nsweeps; k++) {
    int st = op_launch(lv.op, ps->vdtype, OP_JACOBI, lv.phi[lv.cur], lv.phi[1 - lv.cur], lv.rho, 1,
                       nullptr, lv.w, nullptr, s);
    if (st) return st;
    lv.cur = 1 - lv.cur;
  }
  return GFD_OK;
}

// One V-cycle from level l down.  final_norm: compute the level-0 residual
// norm into dscal[0] (FP64 form only).
static int iterate2(gfd_poisson* ps, int l, bool final_norm, cudaStream_t s) {
  Level& lv = ps->L[l];
  const size_t esz = dtype_size(ps->vdtype);
  int st;
  if (l < ps->levels) {
    Level& nx = ps->L[l + 1];
    if ((st = relax_level(ps, lv, lv.pre, s))) return st;
    if ((st = op_launch(lv.op, ps->vdtype, OP_RESIDUAL, lv.phi[lv.cur], lv.res, lv.rho, 1, nullptr,
                        0.0, nullptr, s)))
      return st;
    if ((st = tr_launch(ps->restr[l], ps->vdtype, lv.res, nx.rho, 1, nullptr, s))) return st;
    if ((st = check_cuda(cudaMemsetAsync(nx.phi[nx.cur], 0, nx.n * esz, s), "cudaMemsetAsync")))
      return st;
    if ((st = iterate2(ps, l + 1, false, s))) return st;
    if ((st = tr_launch(ps->interp[l], ps->vdtype, nx.phi[nx.cur], lv.res, 1, nullptr, s)))
      return st;
    if ((st = axpby_launch(ps->vdtype, lv.phi[lv.cur], ps->vdtype, lv.res, 1.0, -1.0, lv.n, s)))
      return st;
  }
  if ((st = relax_level(ps, lv, lv.post, s))) return st;
  if (l == 0 && final_norm) {
    if ((st = op_launch(lv.op, ps->vdtype, OP_RESIDUAL, lv.phi[lv.cur], lv.res, lv.rho, 1, nullptr,
                        0.0, ps->partials, s)))
      return st;
    if ((st = final_sum_launch(ps->partials, (int)ps->npartials, ps->dv, ps->dscal, s))) return st;
  }
  return GFD_OK;
}

static int read_scalar(gfd_poisson* ps, int idx, double* out, cudaStream_t s) {
  int st = check_cuda(cudaMemcpyAsync(ps->hscal + idx, ps->dscal + idx, sizeof(double),
                                      cudaMemcpyDeviceToHost, s),
                      "cudaMemcpyAsync(scalar)");
  if (st) return st;
  st = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (st) return st;
  *out = ps->hscal[idx];
  return GFD_OK;
}

}  // namespace gfd

using namespace gfd;

extern "C" int gfd_poisson_create(int levels, gfd_operator* const* ops,
                                  gfd_transformer* const* restrictors,
                                  gfd_transformer* const* interpolators, const int* presmooths,
                                  const int* postsmooths, const double* weights, int relax_method,
                                  double dv, int pbc_all, int precision, gfd_poisson** out) {
  if (!out) return set_error(GFD_EINVAL, "null output handle");
  *out = nullptr;
  if (levels < 0 || levels > 16 || !ops || !presmooths || !postsmooths || !weights)
    return set_error(GFD_EINVAL, "bad level description");
  if (levels > 0 && (!restrictors || !interpolators))
    return set_error(GFD_EINVAL, "missing transformers");
  if (precision != GFD_POISSON_FP64 && precision != GFD_POISSON_MIXED)
    return set_error(GFD_EINVAL, "unknown precision mode");
  for (int l = 0; l <= levels; l++) {
    if (!ops[l] || !ops[l]->real) return set_error(GFD_EINVAL, "level operators must be real");
    if (ops[l]->off[0] || ops[l]->off[1] || ops[l]->off[2])
      return set_error(GFD_EINVAL, "level operator needs the diagonal as coefs[0]");
    if (relax_method == GFD_RELAX_GS && op_gs_colors(ops[l]) == 0)
      return set_error(GFD_EUNSUPPORTED, "no valid Gauss-Seidel colouring for a level operator");
    if (l < levels) {
      const gfd_transformer* r = restrictors[l];
      const gfd_transformer* ip = interpolators[l];
      if (!r || !ip || r->interpolate || !ip->interpolate || !r->real || !ip->real)
        return set_error(GFD_EINVAL, "bad transformer for level " + std::to_string(l));
      for (int a = 0; a < 3; a++)
        if (r->nin[a] != ops[l]->n[a] || r->nout[a] != ops[l + 1]->n[a] ||
            ip->nin[a] != ops[l + 1]->n[a] || ip->nout[a] != ops[l]->n[a])
          return set_error(GFD_EINVAL, "transformer sizes do not match the level grids");
    }
  }
  gfd_poisson* ps = new (std::nothrow) gfd_poisson();
  if (!ps) return set_error(GFD_ENOMEM, "host allocation failed");
  ps->levels = levels;
  ps->relax_method = relax_method == GFD_RELAX_GS ? GFD_RELAX_GS : GFD_RELAX_JACOBI;
  ps->dv = dv;
  ps->pbc_all = pbc_all ? 1 : 0;
  ps->precision = precision;
  ps->vdtype = precision == GFD_POISSON_MIXED ? GFD_FLOAT32 : GFD_FLOAT64;
  ps->L.resize(levels + 1);
  for (int l = 0; l < levels; l++) {
    ps->restr.push_back(restrictors[l]);
    ps->interp.push_back(interpolators[l]);
  }
  const size_t esz = dtype_size(ps->vdtype);
  // Layout of one pool allocation, 256-byte aligned pieces.
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  std::vector<size_t> o_phi0(levels + 1), o_phi1(levels + 1), o_rho(levels + 1), o_res(levels + 1);
  for (int l = 0; l <= levels; l++) {
    Level& lv = ps->L[l];
    lv.op = ops[l];
    lv.n = (int64_t)ops[l]->n[0] * ops[l]->n[1] * ops[l]->n[2];
    lv.pre = presmooths[l];
    lv.post = postsmooths[l];
    lv.w = weights[l];
    const bool own_phi0 = (l > 0) || (precision == GFD_POISSON_MIXED);
    o_phi0[l] = own_phi0 ? take(lv.n * esz) : 0;
    o_phi1[l] = take(lv.n * esz);
    o_rho[l] = take(lv.n * esz);
    o_res[l] = take(lv.n * esz);
  }
  const int64_t n0 = ps->L[0].n;
  size_t o_r64 = 0, o_alt64 = 0;
  if (precision == GFD_POISSON_MIXED) {
    o_r64 = take(n0 * 8);
    o_alt64 = take(n0 * 8);
  }
  ps->npartials = std::max<int64_t>(op_partials(ops[0], GFD_FLOAT64, OP_RESIDUAL, 1), 1);
  size_t o_part = take(sizeof(double) * std::max<int64_t>(ps->npartials, (int64_t)kRedBlocks));
  size_t o_scal = take(sizeof(double) * 8);
  if (cudaMalloc(&ps->pool, off) != cudaSuccess) {
    cudaGetLastError();
    delete ps;
    return set_error(GFD_ENOMEM, "cudaMalloc of the level hierarchy failed");
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&ps->hscal), sizeof(double) * 8) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(ps->pool);
    delete ps;
    return set_error(GFD_ENOMEM, "cudaMallocHost failed");
  }
  char* base = static_cast<char*>(ps->pool);
  for (int l = 0; l <= levels; l++) {
    Level& lv = ps->L[l];
    const bool own_phi0 = (l > 0) || (precision == GFD_POISSON_MIXED);
    lv.phi[0] = own_phi0 ? base + o_phi0[l] : nullptr;
    lv.phi[1] = base + o_phi1[l];
    lv.rho = base + o_rho[l];
    lv.res = base + o_res[l];
  }
  if (precision == GFD_POISSON_MIXED) {
    ps->r64 = base + o_r64;
    ps->phi64_alt = base + o_alt64;
  }
  ps->partials = reinterpret_cast<double*>(base + o_part);
  ps->dscal = reinterpret_cast<double*>(base + o_scal);
  *out = ps;
  return GFD_OK;
}

extern "C" int gfd_poisson_destroy(gfd_poisson* ps) {
  if (!ps) return GFD_OK;
  if (ps->pool) cudaFree(ps->pool);
  if (ps->hscal) cudaFreeHost(ps->hscal);
  delete ps;
  return GFD_OK;
}

extern "C" int gfd_poisson_solve(gfd_poisson* ps, double* phi, const double* rho, double charge,
                                 double eps, double maxcharge, int maxiter, int* niter_out,
                                 double* error_out, void* stream) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  if (!phi || !rho) return set_error(GFD_EINVAL, "null array pointer");
  if (maxiter < 1) return set_error(GFD_EINVAL, "maxiter must be >= 1");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Level& L0 = ps->L[0];
  const int64_t n0 = L0.n;
  int st;
  // Charge and background (gpaw/poisson.py:130-138).
  double actual = 0.0;
  if ((st = reduce_launch(GFD_FLOAT64, rho, n0, false, ps->dv, ps->partials, ps->dscal + 1, s)))
    return st;
  if ((st = read_scalar(ps, 1, &actual, s))) return st;
  const double background = actual / ps->dv / double(n0);
  const double q = std::isnan(charge) ? actual : charge;
  if (std::fabs(q) > maxcharge)
    return set_error(GFD_EUNSUPPORTED,
                     "charged system: only the charge-neutral branch of solve() is provided");

  int niter = 1;
  double err = 0.0;
  if (ps->precision == GFD_POISSON_FP64) {
    // rhos[0] = rho - background; phis[0] = phi
    L0.phi[0] = phi;
    L0.cur = 0;
    if ((st = sub_const_launch(GFD_FLOAT64, L0.rho, rho, background, n0, s))) return st;
    while (true) {
      if ((st = iterate2(ps, 0, true, s))) return st;
      if ((st = read_scalar(ps, 0, &err, s))) return st;
      if (!(err > eps) || niter >= maxiter) break;
      niter++;
    }
    if (L0.cur != 0 &&
        (st = check_cuda(cudaMemcpyAsync(phi, L0.phi[L0.cur], n0 * 8, cudaMemcpyDeviceToDevice, s),
                         "cudaMemcpyAsync(phi)")))
      return st;
  } else {
    // Mixed: float64 rho0 in r64's sibling; residual r = L phi - rho0.
    double* rho0 = static_cast<double*>(ps->phi64_alt);
    double* r64 = static_cast<double*>(ps->r64);
    if ((st = sub_const_launch(GFD_FLOAT64, rho0, rho, background, n0, s))) return st;
    if ((st = op_launch(L0.op, GFD_FLOAT64, OP_RESIDUAL, phi, r64, rho0, 1, nullptr, 0.0, nullptr,
                        s)))
      return st;
    while (true) {
      if ((st = convert_launch(GFD_FLOAT32, L0.rho, GFD_FLOAT64, r64, n0, s))) return st;
      L0.cur = 0;
      if ((st = check_cuda(cudaMemsetAsync(L0.phi[0], 0, n0 * 4, s), "cudaMemsetAsync"))) return st;
      if ((st = iterate2(ps, 0, false, s))) return st;
      if ((st = axpby_launch(GFD_FLOAT64, phi, GFD_FLOAT32, L0.phi[L0.cur], 1.0, -1.0, n0, s)))
        return st;
      if ((st = op_launch(L0.op, GFD_FLOAT64, OP_RESIDUAL, phi, r64, rho0, 1, nullptr, 0.0,
                          ps->partials, s)))
        return st;
      if ((st = final_sum_launch(ps->partials, (int)ps->npartials, ps->dv, ps->dscal, s))) return st;
      if ((st = read_scalar(ps, 0, &err, s))) return st;
      if (!(err > eps) || niter >= maxiter) break;
      niter++;
    }
  }
  if (niter_out) *niter_out = niter;
  if (error_out) *error_out = err;
  if (niter == maxiter)
    return set_error(GFD_ENOCONV, "Poisson solver did not converge in " +
                                      std::to_string(maxiter) + " iterations!");
  // Zero mean potential for fully periodic systems (gpaw/poisson.py:212-216).
  if (ps->pbc_all) {
    double sum = 0.0;
    if ((st = reduce_launch(GFD_FLOAT64, phi, n0, false, 1.0, ps->partials, ps->dscal + 1, s)))
      return st;
    if ((st = read_scalar(ps, 1, &sum, s))) return st;
    if ((st = sub_const_launch(GFD_FLOAT64, phi, phi, sum / double(n0), n0, s))) return st;
  }
  return check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize(solve)");
}
