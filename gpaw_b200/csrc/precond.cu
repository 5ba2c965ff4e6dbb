// precond.cu -- gfd_preconditioner_*: the band preconditioner of
// gpaw/preconditioner.py:13-70 (two coarse levels, nn = 1 kinetic operators
// and transfers, Bloch phases) as eight device passes.
//
// The reference's nineteen array operations per call
// (gpaw/preconditioner.py:48-70) regroup exactly into:
//   r1 = -restrict(R),  d1 = 4 step r1              seeded restriction, sign -1
//   q1 = kin1 d1 - r1                                residual pass
//   r2 = restrict(q1),  d2 = 16 step r2              seeded restriction
//   d2 <- d2 - 16 step (kin2 d2 - r2)                one weighted-Jacobi pass
//   d1 <- d1 - interpolate(d2)                       interpolation, subtracting
//   d1 <- d1 - 4 step (kin1 d1 - r1)                 one weighted-Jacobi pass
//   d0 = -interpolate(d1)                            interpolation, sign -1
//   out = -(d0 - step (kin0 d0 - R))                 one negated Jacobi pass
// using d - s (L d - r) = (1 - w) d + (w / c0)(r - sum_{p != 0} c_p d_p)
// with w = s c0, the weighted-Jacobi update.  On the fine grid this reads R
// twice and d0 once and writes d0 and out once, instead of the reference's
// eleven fine-grid array passes.
#include <new>
#include <string>

#include "common.cuh"
#include "internal.h"

struct gfd_preconditioner {
  gfd_operator* kin[3] = {nullptr, nullptr, nullptr};  // not owned
  gfd_transformer* restr[2] = {nullptr, nullptr};       // 0 -> 1, 1 -> 2 (not owned)
  gfd_transformer* interp[2] = {nullptr, nullptr};      // 2 -> 1, 1 -> 0 (not owned)
  int dtype = GFD_FLOAT64;
  int64_t block = 0;
  int64_t n[3] = {0, 0, 0};  // points per band on each level
  double step = 0.0;
  // Scratch, `block` bands each: level 1 r1, d1, t1; level 2 r2, d2, t2;
  // level 0 d0.
  void* buf[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

namespace {

int64_t points(const int* n) { return (int64_t)n[0] * n[1] * n[2]; }

bool same(const int* a, const int* b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }

void release(gfd_preconditioner* pc) {
  for (void*& b : pc->buf) {
    if (b) cudaFree(b);
    b = nullptr;
  }
}

}  // namespace

using namespace gfd;

extern "C" int gfd_preconditioner_create(gfd_operator* kin0, gfd_operator* kin1,
                                         gfd_operator* kin2, gfd_transformer* restrict0,
                                         gfd_transformer* restrict1,
                                         gfd_transformer* interpolate2,
                                         gfd_transformer* interpolate1, int dtype,
                                         int64_t block, gfd_preconditioner** out) {
  if (!out) return set_error(GFD_EINVAL, "null output handle");
  *out = nullptr;
  if (!kin0 || !kin1 || !kin2 || !restrict0 || !restrict1 || !interpolate2 || !interpolate1)
    return set_error(GFD_EINVAL, "null operator or transformer");
  if (dtype < GFD_FLOAT64 || dtype > GFD_COMPLEX64) return set_error(GFD_EINVAL, "unknown dtype");
  if (block < 1) return set_error(GFD_EINVAL, "block must be at least 1");
  const int real = !dtype_is_complex(dtype);
  for (gfd_operator* k : {kin0, kin1, kin2})
    if (k->real != real) return set_error(GFD_EINVAL, "operator dtype does not match");
  for (gfd_transformer* t : {restrict0, restrict1, interpolate2, interpolate1})
    if (t->real != real) return set_error(GFD_EINVAL, "transformer dtype does not match");
  if (restrict0->interpolate || restrict1->interpolate || !interpolate2->interpolate ||
      !interpolate1->interpolate)
    return set_error(GFD_EINVAL, "restrictors and interpolators swapped");
  if (!same(restrict0->nin, kin0->n) || !same(restrict0->nout, kin1->n) ||
      !same(restrict1->nin, kin1->n) || !same(restrict1->nout, kin2->n) ||
      !same(interpolate2->nin, kin2->n) || !same(interpolate2->nout, kin1->n) ||
      !same(interpolate1->nin, kin1->n) || !same(interpolate1->nout, kin0->n))
    return set_error(GFD_EINVAL, "grid sizes of the levels do not chain");
  if (kin0->diag == 0.0 || kin1->diag == 0.0 || kin2->diag == 0.0)
    return set_error(GFD_EINVAL, "kinetic operators need a nonzero diagonal");
  if (kin0->off[0] || kin0->off[1] || kin0->off[2] || kin1->off[0] || kin1->off[1] ||
      kin1->off[2] || kin2->off[0] || kin2->off[1] || kin2->off[2])
    return set_error(GFD_EINVAL, "the diagonal (zero offset) must be the first coefficient");
  gfd_preconditioner* pc = new (std::nothrow) gfd_preconditioner();
  if (!pc) return set_error(GFD_ENOMEM, "host allocation failed");
  pc->kin[0] = kin0;
  pc->kin[1] = kin1;
  pc->kin[2] = kin2;
  pc->restr[0] = restrict0;
  pc->restr[1] = restrict1;
  pc->interp[0] = interpolate2;
  pc->interp[1] = interpolate1;
  pc->dtype = dtype;
  pc->block = block;
  pc->n[0] = points(kin0->n);
  pc->n[1] = points(kin1->n);
  pc->n[2] = points(kin2->n);
  // gpaw/preconditioner.py:23
  pc->step = 0.66666666 / kin0->diag;
  const size_t esz = dtype_size(dtype);
  const int64_t lv[7] = {pc->n[1], pc->n[1], pc->n[1], pc->n[2], pc->n[2], pc->n[2], pc->n[0]};
  for (int i = 0; i < 7; i++) {
    if (int st = dev_malloc(&pc->buf[i], size_t(lv[i]) * size_t(block) * esz,
                            "cudaMalloc of preconditioner scratch")) {
      release(pc);
      delete pc;
      return st;
    }
  }
  *out = pc;
  return GFD_OK;
}

extern "C" int gfd_preconditioner_destroy(gfd_preconditioner* pc) {
  if (!pc) return GFD_OK;
  release(pc);
  delete pc;
  return GFD_OK;
}

extern "C" int gfd_preconditioner_apply(gfd_preconditioner* pc, int dtype, const void* residuals,
                                        void* out, int64_t nb, const double* phase_cd,
                                        void* stream) {
  if (!pc) return set_error(GFD_EINVAL, "null preconditioner");
  if (dtype != pc->dtype) return set_error(GFD_EINVAL, "dtype differs from the one created for");
  if (nb < 0) return set_error(GFD_EINVAL, "negative band count");
  if (nb == 0) return GFD_OK;
  if (!residuals || !out) return set_error(GFD_EINVAL, "null array pointer");
  if (residuals == out) return set_error(GFD_EINVAL, "residuals and output must not overlap");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t esz = dtype_size(dtype);
  const double step = pc->step;
  void *r1 = pc->buf[0], *d1 = pc->buf[1], *t1 = pc->buf[2];
  void *r2 = pc->buf[3], *d2 = pc->buf[4], *t2 = pc->buf[5], *d0 = pc->buf[6];
  const double* ph = dtype_is_complex(dtype) ? phase_cd : nullptr;
  int st;
  for (int64_t b0 = 0; b0 < nb; b0 += pc->block) {
    const int64_t m = nb - b0 < pc->block ? nb - b0 : pc->block;
    const char* R = static_cast<const char*>(residuals) + size_t(b0) * pc->n[0] * esz;
    char* O = static_cast<char*>(out) + size_t(b0) * pc->n[0] * esz;
    if ((st = tr_launch_ex(pc->restr[0], dtype, R, r1, nullptr, m, ph, -1.0, d1, 4.0 * step, s)))
      return st;
    if ((st = op_launch(pc->kin[1], dtype, OP_RESIDUAL, d1, t1, r1, m, ph, 0.0, nullptr, s)))
      return st;
    if ((st = tr_launch_ex(pc->restr[1], dtype, t1, r2, nullptr, m, ph, 1.0, d2, 16.0 * step, s)))
      return st;
    if ((st = op_launch(pc->kin[2], dtype, OP_JACOBI, d2, t2, r2, m, ph,
                        16.0 * step * pc->kin[2]->diag, nullptr, s)))
      return st;
    if ((st = tr_launch_ex(pc->interp[0], dtype, t2, d1, d1, m, ph, 1.0, nullptr, 0.0, s)))
      return st;
    if ((st = op_launch(pc->kin[1], dtype, OP_JACOBI, d1, t1, r1, m, ph,
                        4.0 * step * pc->kin[1]->diag, nullptr, s)))
      return st;
    if ((st = tr_launch_ex(pc->interp[1], dtype, t1, d0, nullptr, m, ph, -1.0, nullptr, 0.0, s)))
      return st;
    if ((st = op_launch(pc->kin[0], dtype, OP_JACOBI_NEG, d0, O, R, m, ph,
                        step * pc->kin[0]->diag, nullptr, s)))
      return st;
  }
  return GFD_OK;
}
