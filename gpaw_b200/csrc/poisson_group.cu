// poisson_group.cu -- grouped batches of independent Poisson solves.
//
// A batch of solvers with one structure (same number of levels, smoothing
// counts, Jacobi weights, stencil radius or Gauss-Seidel colouring and
// boundary conditions per level, same transfer orders; grids of any sizes)
// runs its V-cycles in lockstep: each step of the V-cycle (a sweep, a
// residual, a restriction, ...) is ONE launch over every solve's grid of
// that level, instead of one launch per solve.  The V-cycle of
// gpaw/poisson.py:245-276 is unchanged per solve: the steps are those of
// iterate2 in poisson.cu, in the same order, with the same per-point
// arithmetic as the one-thread-per-point kernels.
//
// Work distribution: a step's grids are cut into tiles of kGTile points
// (item i owns tiles tile0[i] .. tile0[i] + ceil(n_i / kGTile) - 1).  A
// persistent grid of CTAs pulls tile indices from the step's atomic counter
// until the tiles run out, so big and small grids share the SMs without a
// per-grid launch.  The counters are reset before the loop and after every
// V-cycle.  A residual-norm step writes one partial sum per tile, and the
// check kernel adds each solve's partials in a fixed order (deterministic)
// and applies the reference's stopping rule (gpaw/poisson.py:203-209) per
// solve.  Converged solves drop out (their tiles are skipped); the graph's
// `while` node runs V-cycles until none is left.
//
// The prologue (charge, background, source) and the epilogue (zero-mean
// potential when fully periodic) stay per solve, as parallel graph branches.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "poisson_internal.h"
#include "stencil_launch.cuh"
#include "transfer.cuh"
#include "util.cuh"

namespace gfd {
namespace {

constexpr int kGTile = 1024;  // points per work tile
constexpr int kGThreads = 256;

struct GHead {
  long long n;  // points of this item's grid
  int tile0;    // first tile of the item within its step
  int solve;    // solver index (active flag)
};
struct GStar {
  GHead h;
  StarParams<double> p;
  const double* in;
  double* out;
  const double* rho;
};
struct GGs {
  GHead h;
  GenParams<double> p;
  double* phi;
  const double* rho;
  const double* frozen;
};
struct GTr {
  GHead h;
  TrParams<double> p;
  const double* in;
  double* out;
  const double* base;
};
struct GFill {
  GHead h;
  double* y;
  const double* x;  // nullptr: zero fill
};

// Next tile of the step for this CTA: t (>= ntiles when none is left) and
// the item that owns it.  Uniform across the CTA.
template <class Item>
__device__ __forceinline__ bool next_tile(const Item* items, int nitems, int ntiles,
                                          unsigned* ctr, int& t, int& i) {
  __shared__ int s_t, s_i;
  __syncthreads();  // every thread is done with the previous tile
  if (threadIdx.x == 0) {
    const int tt = int(atomicAdd(ctr, 1u));
    int lo = 0;
    if (tt < ntiles) {
      int hi = nitems - 1;  // last item whose first tile is <= tt
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].h.tile0 <= tt) lo = mid;
        else hi = mid - 1;
      }
    }
    s_t = tt;
    s_i = lo;
  }
  __syncthreads();
  t = s_t;
  i = s_i;
  return t < ntiles;
}

// Copy an item's parameter block to shared memory (8-byte words).
template <class P>
__device__ __forceinline__ void stage_params(P* dst, const P* src) {
  static_assert(sizeof(P) % 8 == 0, "parameter blocks are 8-byte multiples");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int k = threadIdx.x; k < int(sizeof(P) / 8); k += blockDim.x) d[k] = s[k];
  __syncthreads();
}

// Weighted-Jacobi sweep (MODE_JACOBI) or residual (MODE_RESIDUAL, with one
// sum of r^2 per tile into partials when it is not null).
template <int R, int MODE>
__global__ void __launch_bounds__(kGThreads)
g_star_kernel(const GStar* __restrict__ items, int nitems, int ntiles, unsigned* ctr,
              const int* __restrict__ active, double* __restrict__ partials) {
  pdl_enter();
  __shared__ __align__(16) StarParams<double> sp;
  __shared__ double red[kGThreads / 32];
  int t, i;
  while (next_tile(items, nitems, ntiles, ctr, t, i)) {
    const GStar& it = items[i];
    if (!active[it.h.solve]) continue;
    stage_params(&sp, &it.p);
    // One grid holds fewer than 2^31 points: 32-bit index arithmetic.
    const int plane = sp.n1 * sp.n2;
    const int g0 = (t - it.h.tile0) * kGTile;
    const int n = int(it.h.n);
    double sumsq = 0.0;
    for (int k = threadIdx.x; k < kGTile; k += kGThreads) {
      const int g = g0 + k;
      if (g >= n) break;
      const int i0 = g / plane;
      const int r1 = g - i0 * plane;
      const int i1 = r1 / sp.n2, i2 = r1 - i1 * sp.n2;
      const double v = star_point_at<double, R, MODE, LoadRO>(it.in, it.rho, sp, i0, i1, i2, g);
      it.out[g] = v;
      if constexpr (MODE == MODE_RESIDUAL) sumsq += v * v;
    }
    if constexpr (MODE == MODE_RESIDUAL) {
      if (partials) {
        const double sb = block_sum<kGThreads>(sumsq, red);
        if (threadIdx.x == 0) partials[t] = sb;
      }
    }
  }
}

// One colour of multicolour Gauss-Seidel.
__global__ void __launch_bounds__(kGThreads)
g_gs_kernel(const GGs* __restrict__ items, int nitems, int ntiles, unsigned* ctr,
            const int* __restrict__ active, int ncolor, int color) {
  pdl_enter();
  __shared__ __align__(16) GenParams<double> sp;
  int t, i;
  while (next_tile(items, nitems, ntiles, ctr, t, i)) {
    const GGs& it = items[i];
    if (!active[it.h.solve]) continue;
    stage_params(&sp, &it.p);
    // Item points are colour slots (gs_colour_point): n0 n1 ceil(n2 / ncolor).
    const int slots = gs_row_slots(sp.n2, ncolor);
    const int q0 = (t - it.h.tile0) * kGTile;
    const int nq = int(it.h.n);
    for (int k = threadIdx.x; k < kGTile; k += kGThreads) {
      const int q = q0 + k;
      if (q >= nq) break;
      int i0, i1, i2;
      if (gs_colour_point(q, slots, ncolor, color, sp.n1, sp.n2, i0, i1, i2))
        gs_point_at<double>(it.phi, it.rho, it.frozen, sp, i0, i1, i2);
    }
  }
}

// Restriction (with its seed output when p.seed is set) or interpolation
// subtracted from a base (out = base - interpolate(in)).
template <int NN, bool INTERP>
__global__ void __launch_bounds__(kGThreads)
g_tr_kernel(const GTr* __restrict__ items, int nitems, int ntiles, unsigned* ctr,
            const int* __restrict__ active) {
  pdl_enter();
  __shared__ __align__(16) TrParams<double> sp;
  int t, i;
  while (next_tile(items, nitems, ntiles, ctr, t, i)) {
    const GTr& it = items[i];
    if (!active[it.h.solve]) continue;
    stage_params(&sp, &it.p);
    const int plane = sp.no1 * sp.no2;
    const int g0 = (t - it.h.tile0) * kGTile;
    const int n = int(it.h.n);
    for (int k = threadIdx.x; k < kGTile; k += kGThreads) {
      const int g = g0 + k;
      if (g >= n) break;
      const int X = g / plane;
      const int r1 = g - X * plane;
      const int Y = r1 / sp.no2, Z = r1 - Y * sp.no2;
      if constexpr (INTERP) {
        it.out[g] = interp_point_at<double, NN, true, LoadRO>(it.in, it.base + g, X, Y, Z, sp);
      } else {
        const double v = restrict_point_at<double, NN, LoadRO>(it.in, X, Y, Z, sp);
        it.out[g] = v;
        if (sp.seed) static_cast<double*>(sp.seed)[g] = sp.seed_scale * v;
      }
    }
  }
}

__global__ void __launch_bounds__(kGThreads)
g_fill_kernel(const GFill* __restrict__ items, int nitems, int ntiles, unsigned* ctr,
              const int* __restrict__ active) {
  pdl_enter();
  int t, i;
  while (next_tile(items, nitems, ntiles, ctr, t, i)) {
    const GFill& it = items[i];
    if (!active[it.h.solve]) continue;
    const long long g0 = (long long)(t - it.h.tile0) * kGTile;
    for (int k = threadIdx.x; k < kGTile; k += kGThreads) {
      const long long g = g0 + k;
      if (g >= it.h.n) break;
      it.y[g] = it.x ? it.x[g] : 0.0;
    }
  }
}

// Before the loop: active = not charged; counters zero.
__global__ void g_init_kernel(SolveCtrl* const* ctrl, int* active, int nsolves, unsigned* ctrs,
                              int nctr) {
  pdl_enter();
  for (int k = threadIdx.x; k < nsolves; k += blockDim.x)
    active[k] = ctrl[k]->status == GFD_OK ? 1 : 0;
  for (int k = threadIdx.x; k < nctr; k += blockDim.x) ctrs[k] = 0;
}

// After each V-cycle: per active solve, err = dv * (its partials in tile
// order, lane-strided then a fixed shuffle tree), niter + 1, and the
// stopping rule; counters zero; loop again while any solve is active.
__global__ void __launch_bounds__(1024)
g_check_kernel(SolveCtrl* const* ctrl, int* active, const int* tile0, const int* ntile,
               const double* partials, const double* dv, int nsolves, unsigned* ctrs, int nctr,
               cudaGraphConditionalHandle loop) {
  pdl_enter();
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int s = warp; s < nsolves; s += nwarps) {
    if (!active[s]) continue;
    double v = 0.0;
    for (int k = lane; k < ntile[s]; k += 32) v += partials[tile0[s] + k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) {
      SolveCtrl* c = ctrl[s];
      c->err = v * dv[s];
      const int n = ++c->niter;
      const int more = (c->err > c->eps && n < c->maxiter) ? 1 : 0;
      active[s] = more;
      if (more) atomicOr(&any, 1);
    }
  }
  for (int k = threadIdx.x; k < nctr; k += blockDim.x) ctrs[k] = 0;
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(loop, any ? 1u : 0u);
}

enum { S_JACOBI, S_RESID, S_RESID_NORM, S_GS, S_RESTRICT, S_INTERP, S_FILL };

struct Step {
  int kind;
  int a, b;      // radius / order, or (ncolor, colour)
  size_t off;    // byte offset of the item array in the blob
  int nitems, ntiles;
};

}  // namespace

struct PoissonGroup {
  std::vector<gfd_poisson*> ps;
  std::vector<cudaStream_t> streams;  // prologue / epilogue branches while capturing
  std::vector<Step> steps;
  std::vector<unsigned char> blob;  // item arrays, host copy
  int norm_step = -1;
  void* mem = nullptr;              // device: items, counters, flags, partials, tables
  unsigned char* d_items = nullptr;
  unsigned* d_ctr = nullptr;
  int* d_active = nullptr;
  double* d_partials = nullptr;
  SolveCtrl** d_ctrl = nullptr;
  int* d_tile0 = nullptr;
  int* d_ntile = nullptr;
  double* d_dv = nullptr;
};

namespace {

// Append one step: make(i) returns solver i's item (h.n filled); tiles are
// numbered here.
template <class Item, class F>
void add_step(PoissonGroup* G, int kind, int a, int b, F make) {
  const int n = (int)G->ps.size();
  std::vector<Item> items(n);
  int tiles = 0;
  for (int i = 0; i < n; i++) {
    items[i] = make(i);
    items[i].h.tile0 = tiles;
    items[i].h.solve = i;
    tiles += int((items[i].h.n + kGTile - 1) / kGTile);
  }
  Step st;
  st.kind = kind;
  st.a = a;
  st.b = b;
  st.off = (G->blob.size() + 255) & ~size_t(255);
  st.nitems = n;
  st.ntiles = tiles;
  G->blob.resize(st.off + sizeof(Item) * n);
  std::memcpy(G->blob.data() + st.off, items.data(), sizeof(Item) * n);
  G->steps.push_back(st);
}

double* dptr(void* p) { return static_cast<double*>(p); }

void relax_steps(PoissonGroup* G, int l, int& cur, int nsweeps) {
  if (nsweeps <= 0) return;
  gfd_poisson* p0 = G->ps[0];
  const gfd_operator* op0 = p0->L[l].op;
  if (p0->relax_method == GFD_RELAX_GS) {
    const int nc = op_gs_colors(op0);
    const bool any_per = op0->per[0] || op0->per[1] || op0->per[2];
    const int c = cur;
    for (int sw = 0; sw < nsweeps; sw++) {
      if (any_per)  // wrapped neighbours read the values at the start of the sweep
        add_step<GFill>(G, S_FILL, 0, 0, [&](int i) {
          const Level& lv = G->ps[i]->L[l];
          GFill it{};
          it.h.n = lv.n;
          it.y = dptr(lv.phi[1 - c]);
          it.x = dptr(lv.phi[c]);
          return it;
        });
      for (int color = 0; color < nc; color++)
        add_step<GGs>(G, S_GS, nc, color, [&](int i) {
          const Level& lv = G->ps[i]->L[l];
          GGs it{};
          it.h.n = (long long)lv.op->n[0] * lv.op->n[1] * gs_row_slots(lv.op->n[2], nc);
          gs_params(lv.op, it.p);
          it.phi = dptr(lv.phi[c]);
          it.rho = dptr(lv.rho);
          it.frozen = any_per ? dptr(lv.phi[1 - c]) : dptr(lv.phi[c]);
          return it;
        });
    }
    return;
  }
  for (int k = 0; k < nsweeps; k++) {
    const int c = cur;
    add_step<GStar>(G, S_JACOBI, op0->R, 0, [&](int i) {
      const Level& lv = G->ps[i]->L[l];
      GStar it{};
      it.h.n = lv.n;
      star_params(lv.op, OP_JACOBI, lv.w, nullptr, it.p);
      it.in = dptr(lv.phi[c]);
      it.out = dptr(lv.phi[1 - c]);
      it.rho = dptr(lv.rho);
      return it;
    });
    cur = 1 - cur;
  }
}

void resid_step(PoissonGroup* G, int l, int src, bool norm) {
  add_step<GStar>(G, norm ? S_RESID_NORM : S_RESID, G->ps[0]->L[l].op->R, 0, [&](int i) {
    const Level& lv = G->ps[i]->L[l];
    GStar it{};
    it.h.n = lv.n;
    star_params(lv.op, OP_RESIDUAL, 0.0, nullptr, it.p);
    it.in = dptr(lv.phi[src]);
    it.out = dptr(lv.res);
    it.rho = dptr(lv.rho);
    return it;
  });
  if (norm) G->norm_step = (int)G->steps.size() - 1;
}

// The steps of iterate2 (poisson.cu) from level l down, float64.
void iterate2_steps(PoissonGroup* G, int l, bool final_norm, bool seeded) {
  gfd_poisson* p0 = G->ps[0];
  const Level& lv0 = p0->L[l];
  int cur = seeded ? 1 : 0;
  int pre = lv0.pre, post = lv0.post;
  if (seeded) {
    if (l < p0->levels) pre--;
    else post--;
  }
  if (l < p0->levels) {
    relax_steps(G, l, cur, pre);
    resid_step(G, l, cur, false);
    const bool seed = poisson_seedable(p0, l + 1);
    add_step<GTr>(G, S_RESTRICT, p0->restr[l]->nn, 0, [&](int i) {
      gfd_poisson* ps = G->ps[i];
      const Level& lv = ps->L[l];
      const Level& nx = ps->L[l + 1];
      GTr it{};
      it.h.n = nx.n;
      tr_params(ps->restr[l], nullptr, seed ? nx.phi[1] : nullptr,
                seed ? poisson_seed_scale(nx) : 0.0, 1.0, it.p);
      it.in = dptr(lv.res);
      it.out = dptr(nx.rho);
      return it;
    });
    if (!seed)
      add_step<GFill>(G, S_FILL, 0, 0, [&](int i) {
        const Level& nx = G->ps[i]->L[l + 1];
        GFill it{};
        it.h.n = nx.n;
        it.y = dptr(nx.phi[0]);
        return it;
      });
    iterate2_steps(G, l + 1, false, seed);
    const bool flip = ((post & 1) != 0) != (cur != 0) && p0->relax_method != GFD_RELAX_GS;
    const int dst = flip ? 1 - cur : cur;
    const int c = cur;
    add_step<GTr>(G, S_INTERP, p0->interp[l]->nn, 0, [&](int i) {
      gfd_poisson* ps = G->ps[i];
      const Level& lv = ps->L[l];
      const Level& nx = ps->L[l + 1];
      GTr it{};
      it.h.n = lv.n;
      tr_params(ps->interp[l], nullptr, nullptr, 0.0, 1.0, it.p);
      it.in = dptr(nx.phi[0]);
      it.out = dptr(lv.phi[dst]);
      it.base = dptr(lv.phi[c]);
      return it;
    });
    cur = dst;
  }
  relax_steps(G, l, cur, post);
  if (cur != 0) {
    const int c = cur;
    add_step<GFill>(G, S_FILL, 0, 0, [&](int i) {
      const Level& lv = G->ps[i]->L[l];
      GFill it{};
      it.h.n = lv.n;
      it.y = dptr(lv.phi[0]);
      it.x = dptr(lv.phi[c]);
      return it;
    });
  }
  if (l == 0 && final_norm) resid_step(G, 0, 0, true);
}

int step_blocks(const Step& st) { return std::max(1, std::min(st.ntiles, 8 * num_sms())); }

template <int R>
int launch_star_step(const PoissonGroup* G, const Step& st, int k, cudaStream_t s) {
  const GStar* items = reinterpret_cast<const GStar*>(G->d_items + st.off);
  if (st.kind == S_JACOBI)
    launch_k(g_star_kernel<R, MODE_JACOBI>, step_blocks(st), kGThreads, 0, s, items, st.nitems,
             st.ntiles, G->d_ctr + k, (const int*)G->d_active, (double*)nullptr);
  else
    launch_k(g_star_kernel<R, MODE_RESIDUAL>, step_blocks(st), kGThreads, 0, s, items,
             st.nitems, st.ntiles, G->d_ctr + k, (const int*)G->d_active,
             st.kind == S_RESID_NORM ? G->d_partials : (double*)nullptr);
  return check_launch("g_star_kernel");
}

template <int NN>
int launch_tr_step(const PoissonGroup* G, const Step& st, int k, cudaStream_t s) {
  const GTr* items = reinterpret_cast<const GTr*>(G->d_items + st.off);
  if (st.kind == S_INTERP)
    launch_k(g_tr_kernel<NN, true>, step_blocks(st), kGThreads, 0, s, items, st.nitems,
             st.ntiles, G->d_ctr + k, (const int*)G->d_active);
  else
    launch_k(g_tr_kernel<NN, false>, step_blocks(st), kGThreads, 0, s, items, st.nitems,
             st.ntiles, G->d_ctr + k, (const int*)G->d_active);
  return check_launch("g_tr_kernel");
}

int launch_step(const PoissonGroup* G, int k, cudaStream_t s) {
  const Step& st = G->steps[k];
  switch (st.kind) {
    case S_JACOBI:
    case S_RESID:
    case S_RESID_NORM:
      switch (st.a) {
        case 1: return launch_star_step<1>(G, st, k, s);
        case 2: return launch_star_step<2>(G, st, k, s);
        case 3: return launch_star_step<3>(G, st, k, s);
        case 4: return launch_star_step<4>(G, st, k, s);
        case 5: return launch_star_step<5>(G, st, k, s);
        case 6: return launch_star_step<6>(G, st, k, s);
      }
      return set_error(GFD_EUNSUPPORTED, "stencil radius out of range");
    case S_GS:
      launch_k(g_gs_kernel, step_blocks(st), kGThreads, 0, s,
               reinterpret_cast<const GGs*>(G->d_items + st.off), st.nitems, st.ntiles,
               G->d_ctr + k, (const int*)G->d_active, st.a, st.b);
      return check_launch("g_gs_kernel");
    case S_RESTRICT:
    case S_INTERP:
      switch (st.a) {
        case 1: return launch_tr_step<1>(G, st, k, s);
        case 2: return launch_tr_step<2>(G, st, k, s);
        case 3: return launch_tr_step<3>(G, st, k, s);
        case 4: return launch_tr_step<4>(G, st, k, s);
      }
      return set_error(GFD_EUNSUPPORTED, "transfer order out of range");
    case S_FILL:
      launch_k(g_fill_kernel, step_blocks(st), kGThreads, 0, s,
               reinterpret_cast<const GFill*>(G->d_items + st.off), st.nitems, st.ntiles,
               G->d_ctr + k, (const int*)G->d_active);
      return check_launch("g_fill_kernel");
  }
  return set_error(GFD_EINVAL, "unknown group step");
}

// Per-solve work as parallel branches off `origin` (capturing): f(i, stream).
template <class F>
int branches(int n, cudaStream_t origin, std::vector<cudaStream_t>& cs, F f) {
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join(n, nullptr);
  int st = check_cuda(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreate");
  for (int i = 0; i < n && !st; i++)
    st = check_cuda(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming), "cudaEventCreate");
  if (!st) st = check_cuda(cudaEventRecord(fork, origin), "cudaEventRecord");
  for (int i = 0; i < n && !st; i++) {
    st = check_cuda(cudaStreamWaitEvent(cs[i], fork, 0), "cudaStreamWaitEvent");
    if (!st) st = f(i, cs[i]);
    if (!st) st = check_cuda(cudaEventRecord(join[i], cs[i]), "cudaEventRecord");
    if (!st) st = check_cuda(cudaStreamWaitEvent(origin, join[i], 0), "cudaStreamWaitEvent");
  }
  if (fork) cudaEventDestroy(fork);
  for (auto& e : join)
    if (e) cudaEventDestroy(e);
  return st;
}

}  // namespace

int group_capture_outer(PoissonGroup* G, cudaStream_t cs, cudaGraph_t* body_out,
                        cudaGraphConditionalHandle* loop_out) {
  const int n = (int)G->ps.size();
  const int nctr = (int)G->steps.size();
  int st = branches(n, cs, G->streams, [&](int i, cudaStream_t c) {
    return poisson_prologue(G->ps[i], c);
  });
  if (st) return st;
  launch_k(g_init_kernel, 1, 256, 0, cs, (SolveCtrl* const*)G->d_ctrl, G->d_active, n, G->d_ctr,
           nctr);
  if ((st = check_launch("g_init_kernel"))) return st;
  cudaStreamCaptureStatus cst;
  unsigned long long id;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  if ((st = check_cuda(cudaStreamGetCaptureInfo(cs, &cst, &id, &g, &deps, &ndeps),
                       "cudaStreamGetCaptureInfo")))
    return st;
  cudaGraphConditionalHandle loop;
  if ((st = check_cuda(cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault),
                       "cudaGraphConditionalHandleCreate")))
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
  *loop_out = loop;
  if ((st = check_cuda(cudaStreamUpdateCaptureDependencies(cs, &node, 1,
                                                           cudaStreamSetCaptureDependencies),
                       "cudaStreamUpdateCaptureDependencies")))
    return st;
  return branches(n, cs, G->streams, [&](int i, cudaStream_t c) {
    return poisson_epilogue(G->ps[i], c);
  });
}

int group_capture_body(PoissonGroup* G, cudaStream_t cs, cudaGraph_t body,
                       cudaGraphConditionalHandle loop) {
  const int n = (int)G->ps.size();
  const int nctr = (int)G->steps.size();
  int st = check_cuda(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                                    cudaStreamCaptureModeThreadLocal),
                      "cudaStreamBeginCaptureToGraph");
  if (st) return st;
  for (int k = 0; k < nctr && !st; k++) st = launch_step(G, k, cs);
  if (!st) {
    launch_k(g_check_kernel, 1, 1024, 0, cs, (SolveCtrl* const*)G->d_ctrl, G->d_active,
             (const int*)G->d_tile0, (const int*)G->d_ntile, (const double*)G->d_partials,
             (const double*)G->d_dv, n, G->d_ctr, nctr, loop);
    st = check_launch("g_check_kernel");
  }
  cudaGraph_t b2 = nullptr;
  const int st2 = check_cuda(cudaStreamEndCapture(cs, &b2), "cudaStreamEndCapture(body)");
  return st ? st : st2;
}

// Solvers whose level-0 grid has at most GFD_GROUP_MAX_POINTS points join
// groups (default 32768, about 32^3).  Measured on B200, grouping beats
// graph branches for many small grids (128 solves of 32^3: 10.3K against
// 7.5K Gauss-Seidel solves/s) and loses from about 40^3 up (64 solves of
// 48^3: 4.6K against 5.0K), where the branches' concurrent kernels already
// fill the GPU and the queue's per-tile barriers cost more than the
// launches they save.  Up to the one-thread-per-point limit of the solve
// alone (300K points), a grouped solve computes exactly what it computes
// alone.
bool group_eligible(const gfd_poisson* ps) {
  static const long long limit = [] {
    const char* e = getenv("GFD_GROUP_MAX_POINTS");
    return e && e[0] ? atoll(e) : 32768LL;
  }();
  return ps->precision == GFD_POISSON_FP64 && !ps->B && ps->L[0].n <= limit;
}

bool group_same_structure(const gfd_poisson* a, const gfd_poisson* b, std::string* why) {
  auto no = [&](const char* w) {
    if (why) *why = w;
    return false;
  };
  for (const gfd_poisson* x : {a, b}) {
    if (x->precision != GFD_POISSON_FP64) return no("mixed precision");
    if (x->B) return no("Mehrstellen right-hand side");
  }
  if (b->device != a->device) return no("solvers on different devices");
  if (b->levels != a->levels || b->relax_method != a->relax_method)
    return no("different level counts or relaxation");
  for (int l = 0; l <= a->levels; l++) {
    const Level& x = a->L[l];
    const Level& y = b->L[l];
    if (x.pre != y.pre || x.post != y.post || x.w != y.w) return no("different smoothing");
    for (int c = 0; c < 3; c++)
      if (x.op->per[c] != y.op->per[c]) return no("different boundary conditions");
    // Sweeps and residuals use the star stencil form (Gauss-Seidel: any
    // offsets, same colouring).
    if (!x.op->star || !y.op->star || !x.op->real || !y.op->real || x.op->R != y.op->R ||
        x.op->R < 1 || x.op->R > 6)
      return no("stencils with cross terms or different radii");
    if (a->relax_method == GFD_RELAX_GS &&
        (op_gs_colors(x.op) != op_gs_colors(y.op) || op_gs_colors(x.op) == 0))
      return no("different colourings");
    if (l < a->levels &&
        (a->restr[l]->nn != b->restr[l]->nn || a->interp[l]->nn != b->interp[l]->nn ||
         a->restr[l]->nn > 4 || a->interp[l]->nn > 4))
      return no("different transfer orders");
  }
  return true;
}

void group_destroy(PoissonGroup* G) {
  if (!G) return;
  if (G->mem) cudaFree(G->mem);
  for (auto& c : G->streams)
    if (c) cudaStreamDestroy(c);
  delete G;
}

int group_create(gfd_poisson* const* solvers, int n, PoissonGroup** out) {
  *out = nullptr;
  std::string why;
  if (n < 1) return set_error(GFD_EINVAL, "empty group");
  for (int i = 0; i < n; i++)
    if (!group_same_structure(solvers[0], solvers[i], &why))
      return set_error(GFD_EINVAL, "cannot group: " + why);
  PoissonGroup* G = new (std::nothrow) PoissonGroup();
  if (!G) return set_error(GFD_ENOMEM, "host allocation failed");
  G->ps.assign(solvers, solvers + n);
  iterate2_steps(G, 0, true, false);
  const Step& ns = G->steps[G->norm_step];
  // Device memory: items, counters, active flags, partials, per-solve tables.
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_items = take(G->blob.size());
  const size_t o_ctr = take(sizeof(unsigned) * G->steps.size());
  const size_t o_active = take(sizeof(int) * n);
  const size_t o_part = take(sizeof(double) * ns.ntiles);
  const size_t o_ctrl = take(sizeof(SolveCtrl*) * n);
  const size_t o_tile0 = take(sizeof(int) * n);
  const size_t o_ntile = take(sizeof(int) * n);
  const size_t o_dv = take(sizeof(double) * n);
  if (int st = dev_malloc(&G->mem, off, "cudaMalloc of the batch tables")) {
    delete G;
    return st;
  }
  unsigned char* base = static_cast<unsigned char*>(G->mem);
  G->d_items = base + o_items;
  G->d_ctr = reinterpret_cast<unsigned*>(base + o_ctr);
  G->d_active = reinterpret_cast<int*>(base + o_active);
  G->d_partials = reinterpret_cast<double*>(base + o_part);
  G->d_ctrl = reinterpret_cast<SolveCtrl**>(base + o_ctrl);
  G->d_tile0 = reinterpret_cast<int*>(base + o_tile0);
  G->d_ntile = reinterpret_cast<int*>(base + o_ntile);
  G->d_dv = reinterpret_cast<double*>(base + o_dv);
  std::vector<SolveCtrl*> ctrl(n);
  std::vector<int> tile0(n), ntile(n);
  std::vector<double> dv(n);
  const GStar* nitems = reinterpret_cast<const GStar*>(G->blob.data() + ns.off);
  for (int i = 0; i < n; i++) {
    ctrl[i] = solvers[i]->dctrl;
    tile0[i] = nitems[i].h.tile0;
    ntile[i] = int((nitems[i].h.n + kGTile - 1) / kGTile);
    dv[i] = solvers[i]->dv;
  }
  int st = check_cuda(cudaMemcpy(G->d_items, G->blob.data(), G->blob.size(), cudaMemcpyHostToDevice),
                      "cudaMemcpy(batch items)");
  if (!st) st = check_cuda(cudaMemcpy(G->d_ctrl, ctrl.data(), sizeof(SolveCtrl*) * n,
                                      cudaMemcpyHostToDevice), "cudaMemcpy(batch tables)");
  if (!st) st = check_cuda(cudaMemcpy(G->d_tile0, tile0.data(), sizeof(int) * n,
                                      cudaMemcpyHostToDevice), "cudaMemcpy(batch tables)");
  if (!st) st = check_cuda(cudaMemcpy(G->d_ntile, ntile.data(), sizeof(int) * n,
                                      cudaMemcpyHostToDevice), "cudaMemcpy(batch tables)");
  if (!st) st = check_cuda(cudaMemcpy(G->d_dv, dv.data(), sizeof(double) * n,
                                      cudaMemcpyHostToDevice), "cudaMemcpy(batch tables)");
  G->streams.assign(n, nullptr);
  for (int i = 0; i < n && !st; i++)
    st = check_cuda(cudaStreamCreateWithFlags(&G->streams[i], cudaStreamNonBlocking),
                    "cudaStreamCreate");
  if (st) {
    group_destroy(G);
    return st;
  }
  *out = G;
  return GFD_OK;
}

}  // namespace gfd
