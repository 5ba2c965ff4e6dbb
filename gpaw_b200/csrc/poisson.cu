// poisson.cu -- gfd_poisson_*: the multigrid Poisson solver of
// gpaw/poisson.py:21-276 with the whole level hierarchy resident on the GPU.
//
// V-cycle (PoissonSolver.iterate2, gpaw/poisson.py:245-276), level l < L:
//   relax(presmooths[l]); r = L_l phi_l - rho_l; rho_{l+1} = restrict(r);
//   phi_{l+1} = 0; iterate2(l+1); phi_l -= interpolate(phi_{l+1});
// then relax(postsmooths[l]) and, on level 0, the residual norm
// sum(r^2) dv.  Weighted Jacobi sweeps ping-pong between two buffers per
// level.  On level 0 the correction phi -= interpolate(e) is written out of
// place (into the other buffer), so with 2 + 1 sweeps every V-cycle starts
// and ends in the same buffer; the coarser levels do an even number of
// sweeps and correct in place.
//
// A whole solve is one CUDA graph launch: the charge reduction, background
// subtraction and a `while` conditional node whose body is one V-cycle, the
// residual norm and a one-thread kernel applying the reference's stopping
// rule (gpaw/poisson.py:203-204) on the device.  The graph is captured on the
// first solve and reused; the caller's phi and rho are copied in and out
// around it, and the host waits once per solve.
//
// GFD_POISSON_MIXED: defect correction.  The V-cycle is a linear iteration
// phi <- phi + B (rho - L phi), so running it in float32 on the defect
// (phi = 0, rho = L phi - rho) and subtracting the result from the float64
// phi gives the float64 iterate up to float32 rounding of the correction;
// the residual, the update and the norm stay float64.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "poisson_internal.h"
#include "util.cuh"

namespace {

// The branch of PoissonSolver.solve (gpaw/poisson.py:124-191), from the
// integral of rho (c->charge, reduced just before):
//   |q| <= maxcharge      neutral: source rho - background;
//   charged, periodic     source rho - background, phi shifted by q madelung;
//   charged, non-periodic the monopole (the integral of rho) goes on the
//                         L = 0 Gaussian: source rho - gq g, no background,
//                         phi shifted by gq v, gq = charge / sqrt(4 pi);
//   charged, mixed        refused (NotImplementedError in the reference).
__global__ void prep_kernel(SolveCtrl* c, double npoints, double dv,
                            cudaGraphConditionalHandle loop, int in_graph) {
  gfd::pdl_enter();
  c->bg = c->charge / dv / npoints;
  c->gq = 0.0;
  c->shift = 0.0;
  const double q = isnan(c->charge_arg) ? c->charge : c->charge_arg;
  int status = GFD_OK;
  if (c->skip) {
    status = GFD_EUNSUPPORTED;
  } else if (fabs(q) > c->maxcharge) {
    if (c->bc_kind == kBcPeriodic) {
      if (isnan(c->madelung)) status = GFD_EUNSUPPORTED;
      else c->shift = q * c->madelung;
    } else if (c->bc_kind == kBcNone) {
      if (!c->rho_gauss || !c->phi_gauss) {
        status = GFD_ENEEDGAUSS;
      } else {
        c->gq = c->charge * 0.28209479177387814;  // 1 / sqrt(4 pi)
        c->bg = 0.0;
      }
    } else {
      status = GFD_EUNSUPPORTED;
    }
  }
  c->status = status;
  c->niter = 0;
  c->err = 0.0;
  if (status != GFD_OK && in_graph) cudaGraphSetConditional(loop, 0);
}

// One V-cycle done: count it and decide whether to run another
// (while iterate2() > eps and niter < maxiter).  in_graph = 0 (eager mode):
// only count; the host applies the rule.
__global__ void check_kernel(SolveCtrl* c, cudaGraphConditionalHandle loop, int in_graph) {
  gfd::pdl_enter();
  const int n = ++c->niter;
  if (in_graph) cudaGraphSetConditional(loop, (c->err > c->eps && n < c->maxiter) ? 1u : 0u);
}

// Level-0 source y = x - bg - gq g (background removal, or the Gaussian of
// the charged non-periodic branch) and, in the charged branches, the initial
// guess phi - shift - gq v (phi = 0 with zero_initial_phi); the controls
// hold the branch.
__global__ void __launch_bounds__(256) source_kernel(double* y, const double* x, double* phi,
                                                     const SolveCtrl* c, long long n) {
  gfd::pdl_enter();
  const double bg = c->bg, gq = c->gq, shift = c->shift;
  const bool charged = c->status == GFD_OK && (gq != 0.0 || shift != 0.0);
  const bool zero = charged && c->zero_init;
  const double* g = c->rho_gauss;
  const double* v = c->phi_gauss;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    y[i] = gq != 0.0 ? x[i] - bg - gq * g[i] : x[i] - bg;
    if (charged) phi[i] = zero ? 0.0 : (gq != 0.0 ? phi[i] - gq * v[i] : phi[i] - shift);
  }
}

// phi -= sum / n (zero mean potential in fully periodic systems), then
// + the charged periodic branch's shift (gpaw/poisson.py:157, 212-216).
__global__ void __launch_bounds__(256) sub_mean_kernel(double* phi, const SolveCtrl* c,
                                                       long long n) {
  gfd::pdl_enter();
  const double m = c->sum / double(n) - c->shift;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
    phi[i] -= m;
}

// Result to the caller: out = phi + gq v (the Gaussian's potential back on
// in the charged non-periodic branch, gpaw/poisson.py:185-186).
__global__ void __launch_bounds__(256) finish_kernel(double* out, const double* phi,
                                                     const SolveCtrl* c, long long n) {
  gfd::pdl_enter();
  const double gq = c->status == GFD_OK ? c->gq : 0.0;
  const double* v = c->phi_gauss;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
    out[i] = gq != 0.0 ? phi[i] + gq * v[i] : phi[i];
}

// The L = 0 Gaussian and its potential at every level-0 point
// (gpaw/utilities/gauss.py:22, 35, 67-82; coordinates of
// gpaw/utilities/tools.py:92-118): r_v = sum_c (i_c + beg_c) h_cv - center_v,
// r^2 clamped to 1e-12, g = sqrt(4 a^3) / pi exp(-a r^2),
// v = 2 sqrt(pi) erf(sqrt(a) r) / r.
struct GaussGeom {
  double h[9];
  double center[3];
  int beg[3];
  int n[3];
  double a;
};
__global__ void __launch_bounds__(256) gauss_kernel(double* g, double* v, const GaussGeom geo,
                                                    long long total) {
  gfd::pdl_enter();
  const double norm = sqrt(4.0 * geo.a * geo.a * geo.a) / 3.141592653589793;
  const double sa = sqrt(geo.a);
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < total;
       i += (long long)gridDim.x * 256) {
    const long long plane = (long long)geo.n[1] * geo.n[2];
    const int i0 = int(i / plane);
    const int r1 = int(i - i0 * plane);
    const int i1 = r1 / geo.n[2], i2 = r1 - i1 * geo.n[2];
    const double c0 = i0 + geo.beg[0], c1 = i1 + geo.beg[1], c2 = i2 + geo.beg[2];
    double r2 = 0.0;
    for (int d = 0; d < 3; d++) {
      const double x = c0 * geo.h[d] + c1 * geo.h[3 + d] + c2 * geo.h[6 + d] - geo.center[d];
      r2 += x * x;
    }
    if (r2 < 1e-12) r2 = 1e-12;
    const double r = sqrt(r2);
    g[i] = norm * exp(-geo.a * r2);
    v[i] = 2.0 * 1.7724538509055159 * erf(sa * r) / r;
  }
}

}  // namespace

namespace gfd {

static int relax_level(gfd_poisson* ps, Level& lv, int& cur, int nsweeps, cudaStream_t s) {
  if (nsweeps <= 0) return GFD_OK;
  if (ps->relax_method == GFD_RELAX_GS)
    return op_gs_sweeps(lv.op, ps->vdtype, lv.phi[cur], lv.rho, nsweeps, lv.phi[1 - cur], s);
  for (int k = 0; k < nsweeps; k++) {
    int st = op_launch(lv.op, ps->vdtype, OP_JACOBI, lv.phi[cur], lv.phi[1 - cur], lv.rho, 1,
                       nullptr, lv.w, nullptr, s);
    if (st) return st;
    cur = 1 - cur;
  }
  return GFD_OK;
}

// A level whose correction starts from zero can take its first weighted-
// Jacobi sweep, (w / c0) rho, from the kernel that writes its rho (seeded
// restriction or conversion): exactly the sweep's result, one pass less.
// Only the level's first relaxation acts on the zero guess: the
// pre-smoothing, or on the coarsest level (which has no pre-smoothing) the
// post-smoothing.
static bool seedable(const gfd_poisson* ps, int l) {
  const Level& lv = ps->L[l];
  return ps->relax_method != GFD_RELAX_GS && lv.op->star && lv.w != 0.0 &&
         (l < ps->levels ? lv.pre > 0 : lv.post > 0);
}
static double seed_scale(const Level& lv) { return lv.w / lv.op->c0; }
bool poisson_seedable(const gfd_poisson* ps, int l) { return seedable(ps, l); }
double poisson_seed_scale(const Level& lv) { return seed_scale(lv); }

// Enqueue one V-cycle from level l down; every level starts in phi[0] and
// ends there.  final_norm: the level-0 residual norm into dctrl->err.
// seeded: the level's first sweep is done already (phi[1] = (w/c0) rho from
// a zero guess).
static int iterate2(gfd_poisson* ps, int l, bool final_norm, cudaStream_t s,
                    bool seeded = false) {
  Level& lv = ps->L[l];
  const size_t esz = dtype_size(ps->vdtype);
  int cur = seeded ? 1 : 0;
  int pre = lv.pre, post = lv.post;
  if (seeded) {
    if (l < ps->levels) pre--;
    else post--;
  }
  int st;
  if (l < ps->levels) {
    Level& nx = ps->L[l + 1];
    if ((st = relax_level(ps, lv, cur, pre, s))) return st;
    if ((st = op_launch(lv.op, ps->vdtype, OP_RESIDUAL, lv.phi[cur], lv.res, lv.rho, 1, nullptr,
                        0.0, nullptr, s)))
      return st;
    const bool seed = seedable(ps, l + 1);
    if (seed) {
      if ((st = tr_launch_seed(ps->restr[l], ps->vdtype, lv.res, nx.rho, nx.phi[1],
                               seed_scale(nx), s)))
        return st;
    } else {
      if ((st = tr_launch(ps->restr[l], ps->vdtype, lv.res, nx.rho, 1, nullptr, s))) return st;
      if ((st = zero_launch(ps->vdtype, nx.phi[0], nx.n, s))) return st;
    }
    if ((st = iterate2(ps, l + 1, false, s, seed))) return st;
    // phi -= interpolate(e): out of place when the sweeps left level l in an
    // odd position, so the post-smoothing ends in phi[0].
    const bool flip = ((post & 1) != 0) != (cur != 0) && ps->relax_method != GFD_RELAX_GS;
    const int dst = flip ? 1 - cur : cur;
    if ((st = tr_launch_sub(ps->interp[l], ps->vdtype, nx.phi[0], lv.phi[dst], lv.phi[cur], 1,
                            nullptr, s)))
      return st;
    cur = dst;
  }
  if ((st = relax_level(ps, lv, cur, post, s))) return st;
  if (cur != 0) {
    // Only reachable for an odd total sweep count on a level without the
    // flip (possible with custom smoothing counts): copy back to phi[0].
    if ((st = check_cuda(cudaMemcpyAsync(lv.phi[0], lv.phi[cur], lv.n * esz,
                                         cudaMemcpyDeviceToDevice, s),
                         "cudaMemcpyAsync(phi)")))
      return st;
  }
  if (l == 0 && final_norm) {
    if ((st = op_launch(lv.op, ps->vdtype, OP_RESIDUAL, lv.phi[0], lv.res, lv.rho, 1, nullptr, 0.0,
                        ps->partials, s)))
      return st;
    if ((st = final_sum_launch(ps->partials,
                               (int)op_partials(lv.op, GFD_FLOAT64, OP_RESIDUAL, 1), ps->dv,
                               &ps->dctrl->err, s)))
      return st;
  }
  return GFD_OK;
}

// Level-0 source: rho_in - background (gpaw/poisson.py:128-138), or the
// charged branches' source and initial guess (source_kernel), and, for the
// Mehrstellen form, B applied to it (gpaw/poisson.py:196-199).
static int rhs_launch(gfd_poisson* ps, cudaStream_t s) {
  Level& L0 = ps->L[0];
  const int64_t n0 = L0.n;
  const bool fp64 = ps->precision == GFD_POISSON_FP64;
  double* rho0 = fp64 ? static_cast<double*>(L0.rho) : ps->rho64;
  double* dst = ps->B ? (fp64 ? static_cast<double*>(L0.res) : ps->r64) : rho0;
  double* phi_int = fp64 ? static_cast<double*>(L0.phi[0]) : ps->phi64;
  launch_k(source_kernel, grid_for(n0), 256, 0, s, dst, ps->rho_in, phi_int, ps->dctrl,
           (long long)n0);
  int st = check_launch("source_kernel");
  if (st || !ps->B) return st;
  return op_launch(ps->B, GFD_FLOAT64, OP_APPLY, dst, rho0, nullptr, 1, nullptr, 0.0, nullptr, s);
}

int poisson_prologue(gfd_poisson* ps, cudaStream_t s) {
  const int64_t n0 = ps->L[0].n;
  int st;
  if ((st = reduce_launch(GFD_FLOAT64, ps->rho_in, n0, false, ps->dv, ps->partials,
                          &ps->dctrl->charge, s)))
    return st;
  launch_k(prep_kernel, 1, 1, 0, s, ps->dctrl, double(n0), ps->dv,
           cudaGraphConditionalHandle(0), 0);
  if ((st = check_launch("prep_kernel"))) return st;
  return rhs_launch(ps, s);
}

int poisson_epilogue(gfd_poisson* ps, cudaStream_t s) {
  if (!ps->pbc_all) return GFD_OK;
  const int64_t n0 = ps->L[0].n;
  double* phi_final = ps->precision == GFD_POISSON_FP64 ? static_cast<double*>(ps->L[0].phi[0])
                                                        : ps->phi64;
  int st;
  if ((st = reduce_launch(GFD_FLOAT64, phi_final, n0, false, 1.0, ps->partials, &ps->dctrl->sum,
                          s)))
    return st;
  launch_k(sub_mean_kernel, grid_for(n0), 256, 0, s, phi_final, ps->dctrl, (long long)n0);
  return check_launch("sub_mean_kernel");
}

// Body of the solve loop: one iteration of the chosen form, ending with the
// stopping-rule kernel.
static int loop_body(gfd_poisson* ps, cudaGraphConditionalHandle loop, int in_graph,
                     cudaStream_t s) {
  int st;
  Level& L0 = ps->L[0];
  const int64_t n0 = L0.n;
  if (ps->precision == GFD_POISSON_FP64) {
    if ((st = iterate2(ps, 0, true, s))) return st;
  } else {
    // rho_V = float(L phi - rho); e = 0; one float32 V-cycle; phi -= e;
    // r = L phi - rho with its norm.
    const bool seed = seedable(ps, 0);
    if (seed) {
      if ((st = convert_launch(GFD_FLOAT32, L0.rho, GFD_FLOAT64, ps->r64, n0, s, L0.phi[1],
                               seed_scale(L0))))
        return st;
    } else {
      if ((st = convert_launch(GFD_FLOAT32, L0.rho, GFD_FLOAT64, ps->r64, n0, s))) return st;
      if ((st = zero_launch(GFD_FLOAT32, L0.phi[0], n0, s))) return st;
    }
    if ((st = iterate2(ps, 0, false, s, seed))) return st;
    if ((st = axpby_launch(GFD_FLOAT64, ps->phi64, GFD_FLOAT32, L0.phi[0], 1.0, -1.0, n0, s)))
      return st;
    if ((st = op_launch(L0.op, GFD_FLOAT64, OP_RESIDUAL, ps->phi64, ps->r64, ps->rho64, 1,
                        nullptr, 0.0, ps->partials, s)))
      return st;
    if ((st = final_sum_launch(ps->partials,
                               (int)op_partials(L0.op, GFD_FLOAT64, OP_RESIDUAL, 1), ps->dv,
                               &ps->dctrl->err, s)))
      return st;
  }
  launch_k(check_kernel, 1, 1, 0, s, ps->dctrl, loop, in_graph);
  return check_launch("check_kernel");
}

// Enqueue one solver's part of a graph on a capturing stream: prologue
// (charge, background, rho - background), a `while` conditional node and
// the epilogue (zero-mean potential when fully periodic).  Returns the
// loop's body graph and handle; the body is filled by capture_body once the
// outer capture has ended.
static int capture_solve(gfd_poisson* ps, cudaStream_t cs, cudaGraph_t* body_out,
                         cudaGraphConditionalHandle* loop_out) {
  Level& L0 = ps->L[0];
  const int64_t n0 = L0.n;
  const int blocks = grid_for(n0);
  int st;
  cudaGraphConditionalHandle loop;
  {
    cudaStreamCaptureStatus cst;
    unsigned long long id;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    if ((st = check_cuda(cudaStreamGetCaptureInfo(cs, &cst, &id, &g, &deps, &ndeps),
                         "cudaStreamGetCaptureInfo")))
      return st;
    if ((st = check_cuda(cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault),
                         "cudaGraphConditionalHandleCreate")))
      return st;
  }
  if ((st = reduce_launch(GFD_FLOAT64, ps->rho_in, n0, false, ps->dv, ps->partials,
                          &ps->dctrl->charge, cs)))
    return st;
  launch_k(prep_kernel, 1, 1, 0, cs, ps->dctrl, double(n0), ps->dv, loop, 1);
  if ((st = check_launch("prep_kernel"))) return st;
  if ((st = rhs_launch(ps, cs))) return st;
  if (ps->precision == GFD_POISSON_MIXED &&
      (st = op_launch(L0.op, GFD_FLOAT64, OP_RESIDUAL, ps->phi64, ps->r64, ps->rho64, 1, nullptr,
                      0.0, nullptr, cs)))
    return st;
  {
    cudaStreamCaptureStatus cst;
    unsigned long long id;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t g = nullptr;
    if ((st = check_cuda(cudaStreamGetCaptureInfo(cs, &cst, &id, &g, &deps, &ndeps),
                         "cudaStreamGetCaptureInfo")))
      return st;
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = loop;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if ((st = check_cuda(cudaGraphAddNode(&node, g, deps, ndeps, &np), "cudaGraphAddNode")))
      return st;
    *body_out = np.conditional.phGraph_out[0];
    if ((st = check_cuda(cudaStreamUpdateCaptureDependencies(cs, &node, 1,
                                                             cudaStreamSetCaptureDependencies),
                         "cudaStreamUpdateCaptureDependencies")))
      return st;
  }
  double* phi_final = ps->precision == GFD_POISSON_FP64 ? static_cast<double*>(L0.phi[0])
                                                        : ps->phi64;
  if (ps->pbc_all) {
    if ((st = reduce_launch(GFD_FLOAT64, phi_final, n0, false, 1.0, ps->partials, &ps->dctrl->sum,
                            cs)))
      return st;
    launch_k(sub_mean_kernel, blocks, 256, 0, cs, phi_final, ps->dctrl, (long long)n0);
    if ((st = check_launch("sub_mean_kernel"))) return st;
  }
  *loop_out = loop;
  return GFD_OK;
}

static int capture_body(gfd_poisson* ps, cudaStream_t cs, cudaGraph_t body,
                        cudaGraphConditionalHandle loop) {
  int st = check_cuda(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                                    cudaStreamCaptureModeThreadLocal),
                      "cudaStreamBeginCaptureToGraph");
  if (st) return st;
  st = loop_body(ps, loop, 1, cs);
  cudaGraph_t b2 = nullptr;
  int st2 = check_cuda(cudaStreamEndCapture(cs, &b2), "cudaStreamEndCapture(body)");
  return st ? st : st2;
}

static void abort_capture(cudaStream_t cs) {
  cudaStreamCaptureStatus cst;
  if (cudaStreamIsCapturing(cs, &cst) == cudaSuccess && cst != cudaStreamCaptureStatusNone) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(cs, &g);
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
}

// One branch of a batch graph: a solver alone, or a group of solvers whose
// V-cycle steps run as single launches (poisson_group.cu).
struct BatchUnit {
  gfd_poisson* ps = nullptr;
  gfd::PoissonGroup* group = nullptr;
};

// Capture the units as independent branches of one graph (one solver: that
// solver's own graph).
static int build_unit_graph(const std::vector<BatchUnit>& units, cudaGraph_t* graph_out,
                            cudaGraphExec_t* exec_out) {
  const int n = (int)units.size();
  std::vector<cudaStream_t> cs(n + 1, nullptr);
  for (auto& c : cs) {
    int st = check_cuda(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking), "cudaStreamCreate");
    if (st) {
      for (auto& d : cs) if (d) cudaStreamDestroy(d);
      return st;
    }
  }
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join(n, nullptr);
  std::vector<cudaGraph_t> bodies(n, nullptr);
  std::vector<cudaGraphConditionalHandle> loops(n);
  cudaGraph_t graph = nullptr;
  int st = check_cuda(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreate");
  for (int i = 0; i < n && !st; i++)
    st = check_cuda(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming), "cudaEventCreate");
  cudaStream_t origin = cs[n];
  if (!st)
    st = check_cuda(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal),
                    "cudaStreamBeginCapture");
  if (!st) st = check_cuda(cudaEventRecord(fork, origin), "cudaEventRecord");
  for (int i = 0; i < n && !st; i++) {
    st = check_cuda(cudaStreamWaitEvent(cs[i], fork, 0), "cudaStreamWaitEvent");
    if (!st)
      st = units[i].group ? group_capture_outer(units[i].group, cs[i], &bodies[i], &loops[i])
                          : capture_solve(units[i].ps, cs[i], &bodies[i], &loops[i]);
    if (!st) st = check_cuda(cudaEventRecord(join[i], cs[i]), "cudaEventRecord");
    if (!st) st = check_cuda(cudaStreamWaitEvent(origin, join[i], 0), "cudaStreamWaitEvent");
  }
  if (st) {
    for (auto& c : cs) abort_capture(c);
  } else {
    st = check_cuda(cudaStreamEndCapture(origin, &graph), "cudaStreamEndCapture");
  }
  for (int i = 0; i < n && !st; i++)
    st = units[i].group ? group_capture_body(units[i].group, cs[0], bodies[i], loops[i])
                        : capture_body(units[i].ps, cs[0], bodies[i], loops[i]);
  if (!st) {
    cudaGraphExec_t exec = nullptr;
    st = check_cuda(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
    if (!st) {
      *graph_out = graph;
      *exec_out = exec;
    }
  }
  if (st && graph) cudaGraphDestroy(graph);
  if (fork) cudaEventDestroy(fork);
  for (auto& e : join) if (e) cudaEventDestroy(e);
  for (auto& c : cs) cudaStreamDestroy(c);
  return st;
}

static int build_multi_graph(gfd_poisson* const* solvers, int n, cudaGraph_t* graph_out,
                             cudaGraphExec_t* exec_out) {
  std::vector<BatchUnit> units(n);
  for (int i = 0; i < n; i++) units[i].ps = solvers[i];
  return build_unit_graph(units, graph_out, exec_out);
}

static int build_graph(gfd_poisson* ps) {
  gfd_poisson* one[1] = {ps};
  return build_multi_graph(one, 1, &ps->graph, &ps->exec);
}

// Host-written part of the controls for one solve.
static void set_inputs(gfd_poisson* ps, SolveCtrl* h, double charge, double eps,
                       double maxcharge, int maxiter) {
  h->eps = eps;
  h->maxcharge = maxcharge;
  h->charge_arg = charge;
  h->maxiter = maxiter;
  h->zero_init = ps->zero_init;
  h->rho_gauss = ps->rho_gauss;
  h->phi_gauss = ps->phi_gauss;
  h->madelung = ps->madelung;
  h->bc_kind = ps->bc_kind;
  h->skip = 0;
}

// Copy-in of the controls, rho and phi (before a graph launch) and copy-out
// of phi and the controls (after it); the results are read by
// gfd_poisson_result once the stream has reached that point.
static int stage_in(gfd_poisson* ps, double* phi, const double* rho, double charge, double eps,
                    double maxcharge, int maxiter, cudaStream_t s) {
  const int64_t n0 = ps->L[0].n;
  double* phi_int = ps->precision == GFD_POISSON_FP64 ? static_cast<double*>(ps->L[0].phi[0])
                                                      : ps->phi64;
  SolveCtrl* h = ps->hctrl;
  set_inputs(ps, h, charge, eps, maxcharge, maxiter);
  int st;
  if ((st = check_cuda(cudaMemcpyAsync(ps->dctrl, h, offsetof(SolveCtrl, charge),
                                       cudaMemcpyHostToDevice, s),
                       "cudaMemcpyAsync(controls)")))
    return st;
  if ((st = check_cuda(cudaMemcpyAsync(ps->rho_in, rho, n0 * 8, cudaMemcpyDeviceToDevice, s),
                       "cudaMemcpyAsync(rho)")))
    return st;
  return check_cuda(cudaMemcpyAsync(phi_int, phi, n0 * 8, cudaMemcpyDeviceToDevice, s),
                    "cudaMemcpyAsync(phi)");
}

static int stage_out(gfd_poisson* ps, double* phi, cudaStream_t s) {
  const int64_t n0 = ps->L[0].n;
  double* phi_int = ps->precision == GFD_POISSON_FP64 ? static_cast<double*>(ps->L[0].phi[0])
                                                      : ps->phi64;
  int st;
  if (ps->rho_gauss) {
    // The charged non-periodic branch adds the Gaussian's potential back.
    launch_k(finish_kernel, grid_for(n0), 256, 0, s, phi, phi_int, ps->dctrl, (long long)n0);
    st = check_launch("finish_kernel");
  } else {
    st = check_cuda(cudaMemcpyAsync(phi, phi_int, n0 * 8, cudaMemcpyDeviceToDevice, s),
                    "cudaMemcpyAsync(phi)");
  }
  if (st) return st;
  return check_cuda(cudaMemcpyAsync(ps->hctrl, ps->dctrl, sizeof(SolveCtrl),
                                    cudaMemcpyDeviceToHost, s),
                    "cudaMemcpyAsync(controls)");
}

// The solve without a graph: prologue, host-driven loop, epilogue.
static int solve_eager(gfd_poisson* ps, cudaStream_t s) {
  Level& L0 = ps->L[0];
  const int64_t n0 = L0.n;
  const int blocks = grid_for(n0);
  int st;
  if ((st = reduce_launch(GFD_FLOAT64, ps->rho_in, n0, false, ps->dv, ps->partials,
                          &ps->dctrl->charge, s)))
    return st;
  launch_k(prep_kernel, 1, 1, 0, s, ps->dctrl, double(n0), ps->dv, cudaGraphConditionalHandle(0), 0);
  if ((st = check_launch("prep_kernel"))) return st;
  if ((st = rhs_launch(ps, s))) return st;
  if (ps->precision == GFD_POISSON_MIXED &&
      (st = op_launch(L0.op, GFD_FLOAT64, OP_RESIDUAL, ps->phi64, ps->r64, ps->rho64, 1, nullptr,
                      0.0, nullptr, s)))
    return st;
  SolveCtrl* h = ps->hctrl;
  if ((st = check_cuda(cudaMemcpyAsync(h, ps->dctrl, sizeof(SolveCtrl), cudaMemcpyDeviceToHost, s),
                       "cudaMemcpyAsync(controls)")) ||
      (st = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize")))
    return st;
  if (h->status == GFD_OK) {
    while (true) {
      if ((st = loop_body(ps, cudaGraphConditionalHandle(0), 0, s))) return st;
      if ((st = check_cuda(cudaMemcpyAsync(h, ps->dctrl, sizeof(SolveCtrl),
                                           cudaMemcpyDeviceToHost, s),
                           "cudaMemcpyAsync(controls)")) ||
          (st = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize")))
        return st;
      if (!(h->err > h->eps && h->niter < h->maxiter)) break;
    }
  }
  double* phi_final = ps->precision == GFD_POISSON_FP64 ? static_cast<double*>(L0.phi[0])
                                                        : ps->phi64;
  if (ps->pbc_all) {
    if ((st = reduce_launch(GFD_FLOAT64, phi_final, n0, false, 1.0, ps->partials, &ps->dctrl->sum,
                            s)))
      return st;
    launch_k(sub_mean_kernel, blocks, 256, 0, s, phi_final, ps->dctrl, n0);
    if ((st = check_launch("sub_mean_kernel"))) return st;
  }
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
    if (presmooths[l] < 0 || postsmooths[l] < 0)
      return set_error(GFD_EINVAL, "negative smoothing count");
    if (relax_method != GFD_RELAX_GS && weights[l] == 0.0)
      return set_error(GFD_EINVAL, "Jacobi weight must be nonzero");
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
    o_phi0[l] = take(lv.n * esz);
    o_phi1[l] = take(lv.n * esz);
    o_rho[l] = take(lv.n * esz);
    o_res[l] = take(lv.n * esz);
  }
  const int64_t n0 = ps->L[0].n;
  const size_t o_rho_in = take(n0 * 8);
  size_t o_phi64 = 0, o_rho64 = 0, o_r64 = 0;
  if (precision == GFD_POISSON_MIXED) {
    o_phi64 = take(n0 * 8);
    o_rho64 = take(n0 * 8);
    o_r64 = take(n0 * 8);
  }
  ps->npartials = std::max<int64_t>(op_partials(ops[0], GFD_FLOAT64, OP_RESIDUAL, 1), kRedBlocks);
  const size_t o_part = take(sizeof(double) * ps->npartials);
  const size_t o_ctrl = take(sizeof(SolveCtrl));
  if (int st = dev_malloc(&ps->pool, off, "cudaMalloc of the level hierarchy")) {
    delete ps;
    return st;
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&ps->hctrl), sizeof(SolveCtrl)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(ps->pool);
    delete ps;
    return set_error(GFD_ENOMEM, "cudaMallocHost failed");
  }
  cudaGetDevice(&ps->device);
  char* base = static_cast<char*>(ps->pool);
  for (int l = 0; l <= levels; l++) {
    Level& lv = ps->L[l];
    lv.phi[0] = base + o_phi0[l];
    lv.phi[1] = base + o_phi1[l];
    lv.rho = base + o_rho[l];
    lv.res = base + o_res[l];
  }
  ps->rho_in = reinterpret_cast<double*>(base + o_rho_in);
  if (precision == GFD_POISSON_MIXED) {
    ps->phi64 = reinterpret_cast<double*>(base + o_phi64);
    ps->rho64 = reinterpret_cast<double*>(base + o_rho64);
    ps->r64 = reinterpret_cast<double*>(base + o_r64);
  }
  ps->partials = reinterpret_cast<double*>(base + o_part);
  ps->dctrl = reinterpret_cast<SolveCtrl*>(base + o_ctrl);
  const int* per = ops[0]->per;
  ps->bc_kind = per[0] && per[1] && per[2] ? kBcPeriodic
                : !per[0] && !per[1] && !per[2] ? kBcNone
                                                 : kBcMixed;
  ps->madelung = std::nan("");
  *out = ps;
  return GFD_OK;
}

extern "C" int gfd_poisson_destroy(gfd_poisson* ps) {
  if (!ps) return GFD_OK;
  if (ps->exec) cudaGraphExecDestroy(ps->exec);
  if (ps->graph) cudaGraphDestroy(ps->graph);
  if (ps->pool) cudaFree(ps->pool);
  if (ps->hctrl) cudaFreeHost(ps->hctrl);
  if (ps->rho_gauss) cudaFree(ps->rho_gauss);
  delete ps;
  return GFD_OK;
}

extern "C" int gfd_poisson_load_gauss(gfd_poisson* ps, const double h_cv[9],
                                      const int64_t beg_c[3], const double center_v[3], double a,
                                      void* stream) {
  if (!ps || !h_cv || !beg_c || !center_v) return set_error(GFD_EINVAL, "null argument");
  if (!(a > 0.0)) return set_error(GFD_EINVAL, "the Gaussian's exponent must be positive");
  const gfd_operator* op = ps->L[0].op;
  const int64_t n0 = ps->L[0].n;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st;
  if (!ps->rho_gauss) {
    // One allocation for the Gaussian and its potential (phi_gauss follows).
    void* p = nullptr;
    if ((st = dev_malloc(&p, 2 * n0 * sizeof(double), "cudaMalloc(compensating Gaussian)")))
      return st;
    ps->rho_gauss = static_cast<double*>(p);
    ps->phi_gauss = ps->rho_gauss + n0;
  }
  GaussGeom geo;
  for (int i = 0; i < 9; i++) geo.h[i] = h_cv[i];
  for (int i = 0; i < 3; i++) {
    geo.center[i] = center_v[i];
    geo.beg[i] = (int)beg_c[i];
    geo.n[i] = op->n[i];
  }
  geo.a = a;
  launch_k(gauss_kernel, grid_for(n0), 256, 0, s, ps->rho_gauss, ps->phi_gauss, geo,
           (long long)n0);
  if ((st = check_launch("gauss_kernel"))) return st;
  return check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize(gauss)");
}

extern "C" int gfd_poisson_set_madelung(gfd_poisson* ps, double madelung) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  if (!std::isfinite(madelung)) return set_error(GFD_EINVAL, "Madelung shift must be finite");
  ps->madelung = madelung;
  return GFD_OK;
}

// madelung(cell_cv) of gpaw/utilities/ewald.py:148 with the Ewald class of
// ewald.py:12-146 evaluated at r = r_B = 0 for one probe charge q = -1 that
// is excluded from the central cell: real-space images erfc(G|l|)/|l| (l != 0,
// 3 shells either side), reciprocal sum pi/(V G^2) sum_g exp(-x)/x
// (x = g^2/(4 G^2), g != 0, 9 shells), minus the excluded charge's
// 2 G / sqrt(pi), plus the homogeneous background pi / (G^2 V);
// G = 5 / the longest lattice vector.
extern "C" int gfd_madelung(const double cell_cv[9], double* out) {
  if (!cell_cv || !out) return set_error(GFD_EINVAL, "null argument");
  const double* a1 = cell_cv;
  const double* a2 = cell_cv + 3;
  const double* a3 = cell_cv + 6;
  const double det = a1[0] * (a2[1] * a3[2] - a2[2] * a3[1]) -
                     a1[1] * (a2[0] * a3[2] - a2[2] * a3[0]) +
                     a1[2] * (a2[0] * a3[1] - a2[1] * a3[0]);
  const double vol = std::fabs(det);
  if (!(vol > 0.0)) return set_error(GFD_EINVAL, "singular cell");
  // Reciprocal vectors b_i = inv(cell).T rows: b1 = (a2 x a3) / det, ...
  auto cross = [](const double* u, const double* v, double* w) {
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
  };
  double b[3][3];
  cross(a2, a3, b[0]);
  cross(a3, a1, b[1]);
  cross(a1, a2, b[2]);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) b[i][j] /= det;
  double lmax = 0.0;
  for (int i = 0; i < 3; i++)
    lmax = std::max(lmax, cell_cv[3 * i] * cell_cv[3 * i] + cell_cv[3 * i + 1] * cell_cv[3 * i + 1] +
                              cell_cv[3 * i + 2] * cell_cv[3 * i + 2]);
  const double G = 5.0 / std::sqrt(lmax);
  const double pi = 3.141592653589793;
  const double q = -1.0;
  double e_r = 0.0;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        double l[3];
        for (int v = 0; v < 3; v++) l[v] = i * a1[v] + j * a2[v] + k * a3[v];
        const double d = std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
        if (d > 1e-5) e_r += std::erfc(G * d) / d;
      }
  double e_g = 0.0;
  for (int i = -9; i <= 9; i++)
    for (int j = -9; j <= 9; j++)
      for (int k = -9; k <= 9; k++) {
        double g[3];
        for (int v = 0; v < 3; v++) g[v] = 2.0 * pi * (i * b[0][v] + j * b[1][v] + k * b[2][v]);
        const double g2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
        if (g2 > 1e-10) {
          const double x = 0.25 * g2 / (G * G);
          e_g += std::exp(-x) / x;
        }
      }
  double e = q * e_r + q * pi / (vol * G * G) * e_g;
  e -= q * 2.0 * G / std::sqrt(pi);
  e += -q * pi / (G * G * vol);
  *out = e;
  return GFD_OK;
}

static void drop_graph(gfd_poisson* ps) {
  if (ps->exec) cudaGraphExecDestroy(ps->exec);
  if (ps->graph) cudaGraphDestroy(ps->graph);
  ps->exec = nullptr;
  ps->graph = nullptr;
}

extern "C" int gfd_poisson_set_rhs_operator(gfd_poisson* ps, gfd_operator* B) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  if (B) {
    const gfd_operator* A = ps->L[0].op;
    if (!B->real) return set_error(GFD_EINVAL, "right-hand-side operator must be real");
    if (B->n[0] != A->n[0] || B->n[1] != A->n[1] || B->n[2] != A->n[2])
      return set_error(GFD_EINVAL, "right-hand-side operator is on another grid");
  }
  ps->B = B;
  // The solve graph holds the old prologue: capture it again on the next solve.
  drop_graph(ps);
  return GFD_OK;
}

extern "C" int gfd_poisson_autotune(gfd_poisson* ps, int reps, void* stream) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  gfd_tune_plan plan;
  int st;
  // The level buffers are scratch between solves: the timed launches may
  // overwrite them.
  for (int l = 0; l <= ps->levels; l++) {
    Level& lv = ps->L[l];
    if (ps->relax_method != GFD_RELAX_GS && lv.op->star && lv.w != 0.0 &&
        (st = gfd_autotune_operator(lv.op, ps->vdtype, GFD_TUNE_JACOBI, lv.phi[0], lv.phi[1],
                                    lv.rho, 1, nullptr, lv.w, reps, stream, &plan)))
      return st;
    if (l < ps->levels) {
      Level& nx = ps->L[l + 1];
      if ((st = gfd_autotune_transformer(ps->restr[l], ps->vdtype, lv.res, nx.rho, 1, reps, stream,
                                         &plan)))
        return st;
      if ((st = gfd_autotune_transformer(ps->interp[l], ps->vdtype, nx.phi[0], lv.res, 1, reps,
                                         stream, &plan)))
        return st;
    }
  }
  drop_graph(ps);
  return GFD_OK;
}

static int solve_async_flags(gfd_poisson* ps, double* phi, const double* rho, double charge,
                             double eps, double maxcharge, int maxiter, void* stream);

extern "C" int gfd_poisson_solve_async(gfd_poisson* ps, double* phi, const double* rho,
                                       double charge, double eps, double maxcharge, int maxiter,
                                       void* stream) {
  if (ps) ps->zero_init = 0;
  return solve_async_flags(ps, phi, rho, charge, eps, maxcharge, maxiter, stream);
}

static int solve_async_flags(gfd_poisson* ps, double* phi, const double* rho, double charge,
                             double eps, double maxcharge, int maxiter, void* stream) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  if (!phi || !rho) return set_error(GFD_EINVAL, "null array pointer");
  if (maxiter < 1) return set_error(GFD_EINVAL, "maxiter must be >= 1");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st;
  if (!ps->exec && (st = build_graph(ps))) return st;
  if ((st = stage_in(ps, phi, rho, charge, eps, maxcharge, maxiter, s))) return st;
  if ((st = check_cuda(cudaGraphLaunch(ps->exec, s), "cudaGraphLaunch"))) return st;
  return stage_out(ps, phi, s);
}

extern "C" int gfd_poisson_result(const gfd_poisson* ps, int* niter, double* error) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  const SolveCtrl* h = ps->hctrl;
  if (h->status == GFD_ENEEDGAUSS)
    return set_error(GFD_ENEEDGAUSS,
                     "charged non-periodic system: load the compensating Gaussian first "
                     "(gfd_poisson_load_gauss); phi is unchanged");
  if (h->status == GFD_EUNSUPPORTED) {
    if (h->skip) return set_error(GFD_EUNSUPPORTED, "unused batch slot");
    if (ps->bc_kind == kBcPeriodic)
      return set_error(GFD_EUNSUPPORTED,
                       "charged periodic system: set the Madelung shift first "
                       "(gfd_poisson_set_madelung)");
    return set_error(GFD_EUNSUPPORTED,
                     "charged system with mixed boundary conditions is not supported");
  }
  if (niter) *niter = h->niter;
  if (error) *error = h->err;
  if (h->niter >= h->maxiter)
    return set_error(GFD_ENOCONV, "Poisson solver did not converge in " +
                                      std::to_string(h->maxiter) + " iterations!");
  return GFD_OK;
}

extern "C" int gfd_poisson_solve(gfd_poisson* ps, double* phi, const double* rho, double charge,
                                 double eps, double maxcharge, int maxiter, int* niter_out,
                                 double* error_out, void* stream) {
  return gfd_poisson_solve_ex(ps, phi, rho, charge, eps, maxcharge, maxiter, 0, niter_out,
                              error_out, stream);
}

extern "C" int gfd_poisson_solve_ex(gfd_poisson* ps, double* phi, const double* rho,
                                    double charge, double eps, double maxcharge, int maxiter,
                                    int flags, int* niter_out, double* error_out, void* stream) {
  if (!ps) return set_error(GFD_EINVAL, "null solver");
  if (flags & ~GFD_SOLVE_ZERO_INITIAL_PHI) return set_error(GFD_EINVAL, "unknown solve flags");
  ps->zero_init = (flags & GFD_SOLVE_ZERO_INITIAL_PHI) ? 1 : 0;
  if (!phi || !rho) return set_error(GFD_EINVAL, "null array pointer");
  if (maxiter < 1) return set_error(GFD_EINVAL, "maxiter must be >= 1");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // GFD_POISSON_EAGER=1: the same kernels launched one by one with a host
  // loop (one wait per V-cycle), for per-kernel profiling.
  static const bool eager = [] {
    const char* e = getenv("GFD_POISSON_EAGER");
    return e && e[0] == '1';
  }();
  int st;
  if (!eager) {
    if ((st = solve_async_flags(ps, phi, rho, charge, eps, maxcharge, maxiter, stream))) return st;
  } else {
    if ((st = stage_in(ps, phi, rho, charge, eps, maxcharge, maxiter, s))) return st;
    if ((st = solve_eager(ps, s))) return st;
    if ((st = stage_out(ps, phi, s))) return st;
  }
  if ((st = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize(solve)"))) return st;
  return gfd_poisson_result(ps, niter_out, error_out);
}

// ---------------------------------------------------------------------------
// Batches: several solvers (any grid sizes) as parallel branches of one graph.
// ---------------------------------------------------------------------------
struct gfd_poisson_batch {
  std::vector<gfd_poisson*> solvers;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<gfd::PoissonGroup*> groups;  // solvers of one structure, grouped
  int grouped = 0;                         // solvers inside groups
};

// GFD_BATCH_GROUPED=0: batches always use one graph branch per solver.
static bool grouping_enabled() {
  static const bool on = [] {
    const char* e = getenv("GFD_BATCH_GROUPED");
    return !(e && e[0] == '0');
  }();
  return on;
}

extern "C" int gfd_poisson_batch_create(int nsolvers, gfd_poisson* const* solvers,
                                        gfd_poisson_batch** out) {
  return gfd_poisson_batch_create_ex(nsolvers, solvers, 0, out);
}

extern "C" int gfd_poisson_batch_create_ex(int nsolvers, gfd_poisson* const* solvers, int flags,
                                           gfd_poisson_batch** out) {
  if (!out) return set_error(GFD_EINVAL, "null output handle");
  *out = nullptr;
  if (nsolvers < 1 || !solvers) return set_error(GFD_EINVAL, "a batch needs at least one solver");
  for (int i = 0; i < nsolvers; i++) {
    if (!solvers[i]) return set_error(GFD_EINVAL, "null solver in batch");
    for (int j = 0; j < i; j++)
      if (solvers[j] == solvers[i])
        return set_error(GFD_EINVAL, "a solver may appear only once in a batch");
  }
  gfd_poisson_batch* b = new (std::nothrow) gfd_poisson_batch();
  if (!b) return set_error(GFD_ENOMEM, "host allocation failed");
  b->solvers.assign(solvers, solvers + nsolvers);
  // Solvers of one structure form a group; the rest run alone.
  std::vector<std::vector<gfd_poisson*>> parts;
  for (gfd_poisson* s : b->solvers) {
    bool placed = false;
    if (!(flags & GFD_BATCH_NO_GROUPS) && grouping_enabled() && gfd::group_eligible(s) &&
        gfd::group_same_structure(s, s, nullptr))
      for (auto& part : parts)
        if (gfd::group_same_structure(part[0], s, nullptr)) {
          part.push_back(s);
          placed = true;
          break;
        }
    if (!placed) parts.push_back({s});
  }
  std::vector<BatchUnit> units;
  int st = GFD_OK;
  for (auto& part : parts) {
    BatchUnit u;
    if (part.size() >= 2) {
      if ((st = gfd::group_create(part.data(), (int)part.size(), &u.group))) break;
      b->groups.push_back(u.group);
      b->grouped += (int)part.size();
    } else {
      u.ps = part[0];
    }
    units.push_back(u);
  }
  if (!st) st = build_unit_graph(units, &b->graph, &b->exec);
  if (st) {
    for (auto* g : b->groups) gfd::group_destroy(g);
    delete b;
    return st;
  }
  *out = b;
  return GFD_OK;
}

extern "C" int gfd_poisson_batch_destroy(gfd_poisson_batch* b) {
  if (!b) return GFD_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto* g : b->groups) gfd::group_destroy(g);
  delete b;
  return GFD_OK;
}

extern "C" int gfd_poisson_batch_solve_async(gfd_poisson_batch* b, double* const* phis,
                                             const double* const* rhos, double eps,
                                             double maxcharge, int maxiter, void* stream) {
  if (!b) return set_error(GFD_EINVAL, "null batch");
  if (!phis || !rhos) return set_error(GFD_EINVAL, "null array list");
  if (maxiter < 1) return set_error(GFD_EINVAL, "maxiter must be >= 1");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = (int)b->solvers.size();
  int st;
  for (int i = 0; i < n; i++)
    if (!phis[i] != !rhos[i])
      return set_error(GFD_EINVAL, "phi and rho of a batch slot must both be given or both null");
  for (int i = 0; i < n; i++) {
    if (!phis[i]) {
      // Unused slot: marked skipped, so it runs no V-cycle; its arrays are
      // neither read nor written.
      gfd_poisson* ps = b->solvers[i];
      SolveCtrl* h = ps->hctrl;
      ps->zero_init = 0;
      set_inputs(ps, h, std::nan(""), eps, maxcharge, maxiter);
      h->skip = 1;
      if ((st = check_cuda(cudaMemcpyAsync(ps->dctrl, h, offsetof(SolveCtrl, charge),
                                           cudaMemcpyHostToDevice, s),
                           "cudaMemcpyAsync(controls)")))
        return st;
      continue;
    }
    b->solvers[i]->zero_init = 0;
    if ((st = stage_in(b->solvers[i], phis[i], rhos[i], std::nan(""), eps, maxcharge, maxiter, s)))
      return st;
  }
  if ((st = check_cuda(cudaGraphLaunch(b->exec, s), "cudaGraphLaunch(batch)"))) return st;
  for (int i = 0; i < n; i++)
    if (phis[i] && (st = stage_out(b->solvers[i], phis[i], s))) return st;
  return GFD_OK;
}

extern "C" int gfd_poisson_batch_grouped(const gfd_poisson_batch* b, int* grouped) {
  if (!b || !grouped) return set_error(GFD_EINVAL, "null argument");
  *grouped = b->grouped;
  return GFD_OK;
}
