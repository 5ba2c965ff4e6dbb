// autotune.cu -- launch-plan autotuning and its cache.
//
// The reference has one CPU code path per operation; on the GPU the fastest
// kernel form depends on the grid, the stencil radius, the element type and
// how many bands go into one launch.  A plan (TunePlan, internal.h) fixes
//   * the kernel form: one thread per point (the small-grid form) or the
//     marching kernel, which streams planes along axis 0;
//   * the marching tile: 32, 16 or 8 columns wide (radius <= 2; larger radii
//     have the 32-wide tile only);
//   * the axis-0 split: a target number of CTAs per SM, which sets how many
//     planes each CTA marches through.
// gfd_autotune_operator / gfd_autotune_transformer time every candidate
// plan with CUDA events on the caller's buffers and stream and cache the
// fastest under the launch's key: kernel family, element type, mode, grid,
// radius or transfer order, boundary conditions and band-count class
// (floor(log2(bands))).  Every later launch with that key uses the plan;
// launches without an entry keep the built-in rules.  The cache can be saved
// to and loaded from a text file (GFD_TUNE_CACHE=<path> loads one on first
// use).  The marching candidates give bit-identical results; the
// one-thread-per-point form sums a stencil's terms in another order, so it
// differs from them at the rounding level (well inside the 1e-13 relative
// parity bound).
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace gfd {
namespace {

std::mutex g_mu;
std::map<TuneKey, TunePlan> g_cache;
std::atomic<int> g_size{0};
std::once_flag g_env_once;
// Set while an autotune run times one candidate on this thread.
thread_local const TunePlan* t_force = nullptr;

const int kCps[] = {1, 2, 4, 8};

int band_class(int64_t nin) {
  int c = 0;
  while (nin > 1) {
    nin >>= 1;
    ++c;
  }
  return c;
}

int per_mask(const int per[3]) { return (per[0] ? 1 : 0) | (per[1] ? 2 : 0) | (per[2] ? 4 : 0); }

bool plan_valid(const TunePlan& p) {
  return (p.path == PLAN_DIRECT || p.path == PLAN_MARCH) && p.tile >= TILE_WIDE &&
         p.tile <= TILE_48 && p.cps >= 1 && p.cps <= 64;
}

int load_file(const char* path);

void load_env_cache() {
  const char* e = getenv("GFD_TUNE_CACHE");
  if (e && e[0]) load_file(e);  // a missing or bad file leaves the cache empty
}

const char kMagic[] = "gfd-tune 1";

int load_file(const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return set_error(GFD_EINVAL, std::string("cannot open tune cache ") + path);
  char line[512];
  if (!fgets(line, sizeof line, f) || strncmp(line, kMagic, sizeof kMagic - 1) != 0) {
    fclose(f);
    return set_error(GFD_EINVAL, std::string("not a tune cache: ") + path);
  }
  std::map<TuneKey, TunePlan> got;
  int lineno = 1;
  while (fgets(line, sizeof line, f)) {
    ++lineno;
    if (line[0] == '#' || line[0] == '\n') continue;
    TuneKey k;
    TunePlan p;
    const int n = sscanf(line, "%d %d %d %d %d %d %d %d %d %d %d %d %lf", &k.kind, &k.dtype,
                         &k.mode, &k.n0, &k.n1, &k.n2, &k.order, &k.per, &k.nbc, &p.path, &p.tile,
                         &p.cps, &p.us);
    if (n != 13 || !plan_valid(p) || k.kind < TK_STAR || k.kind > TK_INTERP) {
      fclose(f);
      return set_error(GFD_EINVAL, std::string("bad tune cache line ") + std::to_string(lineno) +
                                       " in " + path);
    }
    got[k] = p;
  }
  fclose(f);
  std::lock_guard<std::mutex> g(g_mu);
  for (auto& kv : got) g_cache[kv.first] = kv.second;
  g_size.store((int)g_cache.size());
  return GFD_OK;
}

void store(const TuneKey& k, const TunePlan& p) {
  std::lock_guard<std::mutex> g(g_mu);
  g_cache[k] = p;
  g_size.store((int)g_cache.size());
}

int check_not_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  int st = check_cuda(cudaStreamIsCapturing(s, &cs), "cudaStreamIsCapturing");
  if (st) return st;
  if (cs != cudaStreamCaptureStatusNone)
    return set_error(GFD_EINVAL, "cannot autotune on a stream that is being captured");
  return GFD_OK;
}

// Time each candidate (one untimed launch, then reps timed ones) and return
// the fastest in *best.  launch(s) runs the operation once.
template <class Launch>
int time_candidates(const std::vector<TunePlan>& cands, int reps, cudaStream_t s, Launch launch,
                    TunePlan* best) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int st = check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
  if (!st) st = check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
  bool found = false;
  for (size_t i = 0; i < cands.size() && !st; i++) {
    t_force = &cands[i];
    st = launch(s);
    if (!st) st = check_cuda(cudaEventRecord(e0, s), "cudaEventRecord");
    for (int r = 0; r < reps && !st; r++) st = launch(s);
    if (!st) st = check_cuda(cudaEventRecord(e1, s), "cudaEventRecord");
    t_force = nullptr;
    if (!st) st = check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.f;
    if (!st) st = check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    if (st) break;
    const double us = 1000.0 * ms / reps;
    if (!found || us < best->us) {
      *best = cands[i];
      best->us = us;
      found = true;
    }
  }
  t_force = nullptr;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return st;
}

std::vector<TunePlan> march_candidates(const std::vector<int>& tiles) {
  std::vector<TunePlan> c;
  TunePlan d;
  d.path = PLAN_DIRECT;
  c.push_back(d);
  for (int t : tiles)
    for (int cps : kCps) {
      TunePlan p;
      p.path = PLAN_MARCH;
      p.tile = t;
      p.cps = cps;
      c.push_back(p);
    }
  return c;
}

}  // namespace

TuneKey star_tune_key(const gfd_operator* op, int dtype, int mode, int64_t nin) {
  TuneKey k;
  k.kind = TK_STAR;
  k.dtype = dtype;
  k.mode = mode == OP_JACOBI_NEG ? OP_JACOBI : mode;
  k.n0 = op->n[0];
  k.n1 = op->n[1];
  k.n2 = op->n[2];
  k.order = op->R;
  k.per = per_mask(op->per);
  k.nbc = band_class(nin);
  return k;
}

TuneKey tr_tune_key(const gfd_transformer* tr, int dtype, int64_t nin) {
  TuneKey k;
  k.kind = tr->interpolate ? TK_INTERP : TK_RESTRICT;
  k.dtype = dtype;
  k.mode = 0;
  k.n0 = tr->nin[0];
  k.n1 = tr->nin[1];
  k.n2 = tr->nin[2];
  k.order = tr->nn;
  k.per = per_mask(tr->per);
  k.nbc = band_class(nin);
  return k;
}

bool tune_lookup(const TuneKey& k, TunePlan* plan) {
  if (t_force) {
    *plan = *t_force;
    return true;
  }
  std::call_once(g_env_once, load_env_cache);
  if (g_size.load(std::memory_order_relaxed) == 0) return false;
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_cache.find(k);
  if (it == g_cache.end()) return false;
  *plan = it->second;
  return true;
}

}  // namespace gfd

using namespace gfd;

static void to_public(const TunePlan& p, gfd_tune_plan* out) {
  if (!out) return;
  out->form = p.path;
  out->tile = p.tile;
  out->ctas_per_sm = p.cps;
  out->us = p.us;
}

extern "C" int gfd_autotune_operator(gfd_operator* op, int dtype, int mode, const void* in,
                                     void* out, const void* src, int64_t nin,
                                     const double* phase_cd, double w, int reps, void* stream,
                                     gfd_tune_plan* best) {
  if (!op) return set_error(GFD_EINVAL, "null operator");
  if (!in || !out) return set_error(GFD_EINVAL, "null array pointer");
  if (nin < 1) return set_error(GFD_EINVAL, "autotuning needs at least one band");
  if (reps < 1 || reps > 1000) return set_error(GFD_EINVAL, "reps must be in 1..1000");
  if (dtype < GFD_FLOAT64 || dtype > GFD_COMPLEX64) return set_error(GFD_EINVAL, "unknown dtype");
  if (op->real != !dtype_is_complex(dtype))
    return set_error(GFD_EINVAL, op->real ? "operator was built for real arrays"
                                          : "operator was built for complex arrays");
  if (!op->star)
    return set_error(GFD_EUNSUPPORTED,
                     "launch plans are for axis-aligned stencils; this one has cross terms");
  if (mode != GFD_TUNE_APPLY && mode != GFD_TUNE_JACOBI && mode != GFD_TUNE_POTENTIAL)
    return set_error(GFD_EINVAL, "mode must be GFD_TUNE_APPLY, _JACOBI or _POTENTIAL");
  if (mode != GFD_TUNE_APPLY && !src)
    return set_error(GFD_EINVAL, "the Jacobi and potential modes need a source array");
  if (mode == GFD_TUNE_JACOBI && w == 0.0)
    return set_error(GFD_EINVAL, "a Jacobi sweep with weight 0 does no work to time");
  if (in == out) return set_error(GFD_EINVAL, "input and output must not alias");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = check_not_capturing(s);
  if (st) return st;
  const int imode = mode == GFD_TUNE_JACOBI ? OP_JACOBI
                    : mode == GFD_TUNE_POTENTIAL ? OP_POTENTIAL
                                                 : OP_APPLY;
  std::vector<int> tiles = {TILE_WIDE};
  if (op->R <= 2) tiles = {TILE_WIDE, TILE_MID, TILE_NARROW};
  // Where the 48-column tile applies it replaces the short tile as a
  // candidate: the two time alike in short bursts, but under sustained load
  // (the power cap lowering the SM clock) the 48-column tile kept 2.6% more
  // (512-band 96^3 Laplace, 200 steps: 3730 against 3636 GB/s).
  if (dtype == GFD_COMPLEX128 && (imode == OP_APPLY || imode == OP_POTENTIAL) && op->R <= 4 &&
      !tile48_eligible(op))
    tiles.push_back(TILE_SHORT);
  if (dtype_is_complex(dtype) && op->R <= 3) tiles.push_back(TILE_SPLIT);
  if (dtype == GFD_COMPLEX128 && op->R <= 3) tiles.push_back(TILE_TMASPLIT);
  if (dtype_is_complex(dtype) && (imode == OP_APPLY || imode == OP_POTENTIAL) &&
      tile48_eligible(op))
    tiles.push_back(TILE_48);
  const std::vector<TunePlan> cands = march_candidates(tiles);
  const double* ph = dtype_is_complex(dtype) ? phase_cd : nullptr;
  TunePlan pick;
  st = time_candidates(cands, reps, s,
                       [&](cudaStream_t ss) {
                         return op_launch(op, dtype, imode, in, out,
                                          imode == OP_APPLY ? nullptr : src, nin, ph, w, nullptr,
                                          ss);
                       },
                       &pick);
  if (st) return st;
  store(star_tune_key(op, dtype, imode, nin), pick);
  to_public(pick, best);
  return GFD_OK;
}

extern "C" int gfd_autotune_transformer(gfd_transformer* tr, int dtype, const void* in, void* out,
                                        int64_t nin, int reps, void* stream, gfd_tune_plan* best) {
  if (!tr) return set_error(GFD_EINVAL, "null transformer");
  if (!in || !out) return set_error(GFD_EINVAL, "null array pointer");
  if (nin < 1) return set_error(GFD_EINVAL, "autotuning needs at least one band");
  if (reps < 1 || reps > 1000) return set_error(GFD_EINVAL, "reps must be in 1..1000");
  if (dtype < GFD_FLOAT64 || dtype > GFD_COMPLEX64) return set_error(GFD_EINVAL, "unknown dtype");
  if (tr->real != !dtype_is_complex(dtype))
    return set_error(GFD_EINVAL, tr->real ? "transformer was built for real arrays"
                                          : "transformer was built for complex arrays");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = check_not_capturing(s);
  if (st) return st;
  const std::vector<TunePlan> cands = march_candidates({TILE_WIDE});
  TunePlan pick;
  st = time_candidates(cands, reps, s,
                       [&](cudaStream_t ss) {
                         return tr_launch(tr, dtype, in, out, nin, nullptr, ss);
                       },
                       &pick);
  if (st) return st;
  store(tr_tune_key(tr, dtype, nin), pick);
  to_public(pick, best);
  return GFD_OK;
}

extern "C" int gfd_autotune_operator_plan(const gfd_operator* op, int dtype, int mode,
                                          int64_t nin, gfd_tune_plan* plan, int* found) {
  if (!op || !found) return set_error(GFD_EINVAL, "null argument");
  const int imode = mode == GFD_TUNE_JACOBI ? OP_JACOBI
                    : mode == GFD_TUNE_POTENTIAL ? OP_POTENTIAL
                                                 : OP_APPLY;
  TunePlan p;
  *found = op->star && tune_lookup(star_tune_key(op, dtype, imode, nin), &p) ? 1 : 0;
  if (*found) to_public(p, plan);
  return GFD_OK;
}

extern "C" int gfd_autotune_transformer_plan(const gfd_transformer* tr, int dtype, int64_t nin,
                                             gfd_tune_plan* plan, int* found) {
  if (!tr || !found) return set_error(GFD_EINVAL, "null argument");
  TunePlan p;
  *found = tune_lookup(tr_tune_key(tr, dtype, nin), &p) ? 1 : 0;
  if (*found) to_public(p, plan);
  return GFD_OK;
}

extern "C" int gfd_autotune_count(int* n) {
  if (!n) return set_error(GFD_EINVAL, "null argument");
  std::call_once(g_env_once, load_env_cache);
  std::lock_guard<std::mutex> g(g_mu);
  *n = (int)g_cache.size();
  return GFD_OK;
}

extern "C" int gfd_autotune_clear(void) {
  std::call_once(g_env_once, [] {});  // a later lookup must not reload the file
  std::lock_guard<std::mutex> g(g_mu);
  g_cache.clear();
  g_size.store(0);
  return GFD_OK;
}

extern "C" int gfd_autotune_save(const char* path) {
  if (!path) return set_error(GFD_EINVAL, "null path");
  std::call_once(g_env_once, load_env_cache);
  std::map<TuneKey, TunePlan> snap;
  {
    std::lock_guard<std::mutex> g(g_mu);
    snap = g_cache;
  }
  FILE* f = fopen(path, "w");
  if (!f) return set_error(GFD_EINVAL, std::string("cannot write tune cache ") + path);
  fprintf(f, "%s\n", kMagic);
  fprintf(f, "# kind dtype mode n0 n1 n2 order per band_class form tile ctas_per_sm us\n");
  for (auto& kv : snap) {
    const TuneKey& k = kv.first;
    const TunePlan& p = kv.second;
    fprintf(f, "%d %d %d %d %d %d %d %d %d %d %d %d %.3f\n", k.kind, k.dtype, k.mode, k.n0, k.n1,
            k.n2, k.order, k.per, k.nbc, p.path, p.tile, p.cps, p.us);
  }
  const bool ok = fclose(f) == 0;
  return ok ? GFD_OK : set_error(GFD_EINVAL, std::string("error writing ") + path);
}

extern "C" int gfd_autotune_load(const char* path) {
  if (!path) return set_error(GFD_EINVAL, "null path");
  std::call_once(g_env_once, load_env_cache);
  return load_file(path);
}
