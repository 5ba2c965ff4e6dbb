// stencil_tma.cuh -- TMA-fed star stencil for band-batched complex128 apply.
//
// Same operator as star_kernel (stencil.cuh): out[g] = sum_p coefs[p] *
// a[g + offsets[p]] over an axis-aligned offset set (c/bmgs/fd.c:16-51 on the
// halo-padded copy of c/bc.c:138-250, Bloch phases included), marching along
// axis 0 with 2R+1 partial sums per point in registers.  What changes is how
// planes reach shared memory and how warps synchronise:
//
//  * one producer thread loads each plane with five tensor-memory-accelerator
//    boxes -- the 2R + BY rows of the CTA's 32 columns (top halo, own rows,
//    bottom halo) and the R-column left / right halos of the own rows --
//    at wrapped coordinates on periodic axes; on zero-boundary axes the
//    coordinates run off the grid and the hardware fills zeros.  No thread
//    issues per-element copies and L2 sends whole lines.
//  * a ring of S stages with a full and an empty mbarrier each: consumer
//    warps wait for "plane landed" and release the stage when they have read
//    it, so warps drift apart instead of meeting at a CTA barrier per plane.
//  * each thread owns VY rows of one column; Bloch phases of wrapped halo
//    cells are applied when the cell is read (tiles on a wrapped boundary
//    take a separate, phased read path).
//
// Every mbarrier wait is bounded (iterations and SM cycles); on expiry the
// kernel sets *err, drains the loads it issued and returns.
#pragma once

#include <cuda.h>

#include "stencil.cuh"

namespace gfd {

constexpr int kTmaBZ = 32;                        // columns per CTA
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_addr(bar))
      : "memory");
}

// Stage layout (complex128 cells): rows [2R + BY][32] (top halo, own rows,
// bottom halo), then left [BY][R] and right [BY][R] halo columns.  Every
// region starts on a 128-byte boundary.
template <int R, int BY>
struct TmaStage {
  static constexpr int SY = BY + 2 * R;
  static constexpr int ROWS = SY * kTmaBZ;  // cells
  static constexpr int SIDE = BY * R;       // cells per side
  static constexpr int CELLS = ROWS + 2 * SIDE;
  static constexpr unsigned BYTES = unsigned(CELLS) * 16u;
  static_assert(BYTES % 128 == 0, "stage must keep 128-byte alignment");
};

template <int R, int BY, int S>
constexpr size_t star_tma_smem_bytes() {
  return size_t(S) * TmaStage<R, BY>::BYTES + 2 * S * sizeof(uint64_t) + 128;
}

struct TmaMaps {
  CUtensorMap rows_halo;  // box {2*32 doubles, R rows}
  CUtensorMap rows_own;   // box {2*32 doubles, BY rows}
  CUtensorMap side;       // box {2*R doubles, BY rows}
};

// In-plane part of one plane for a thread: sum[j] = c0 a + axis-1 and
// axis-2 neighbour terms of own row j, own[j] = the own cell.  PH: apply the
// Bloch phases of wrapped halos (flags w = top, bottom, left, right);
// without PH every read is a plain 16-byte load whose address is selected
// without branches, so the loads of a plane issue back to back.
template <int R, int VY, int BY, bool PH>
__device__ __forceinline__ void tma_plane(const cplx<double>* st, int g, int zt,
                                          const StarParams<double>& p, unsigned w,
                                          cplx<double> (&sum)[VY], cplx<double> (&own)[VY]) {
  using V = cplx<double>;
  using St = TmaStage<R, BY>;
  const V* left = st + St::ROWS;
  const V* right = left + St::SIDE;
  auto part = [&](const V* c, bool wrapped, const cplx<double>& ph) -> V {
    if constexpr (PH) return wrapped ? cmul(ph, *c) : *c;
    else return *c;
  };
  V col[VY + 2 * R];
#pragma unroll
  for (int m = 0; m < VY + 2 * R; m++) {
    const int r = VY * g + m;
    const bool wr = r < R ? (w & 1u) : (r >= R + BY ? (w & 2u) : false);
    col[m] = part(st + r * kTmaBZ + zt, wr, r < R ? p.P.ph[1][1] : p.P.ph[1][0]);
  }
#pragma unroll
  for (int j = 0; j < VY; j++) {
    own[j] = col[R + j];
    V sy = vmul(p.c0, col[R + j]);
    V sz = vzero<V>();
    const V* row = st + (R + VY * g + j) * kTmaBZ;
    const int side = (VY * g + j) * R;
#pragma unroll
    for (int k = 1; k <= R; k++) {
      madd(sy, p.cy[kMaxR - k], col[R + j - k]);
      madd(sy, p.cy[kMaxR + k], col[R + j + k]);
      const int za = zt - k, zb = zt + k;
      const V* ca = za >= 0 ? row + za : left + side + za + R;
      const V* cb = zb < kTmaBZ ? row + zb : right + side + zb - kTmaBZ;
      madd(sz, p.cz[kMaxR - k], part(ca, za < 0 && (w & 4u), p.P.ph[2][1]));
      madd(sz, p.cz[kMaxR + k], part(cb, zb >= kTmaBZ && (w & 8u), p.P.ph[2][0]));
    }
    sum[j] = vadd(sy, sz);
  }
}

// 32G threads: lane zt of warp g owns column zt of rows VY*g .. VY*g+VY-1
// of the CTA's BY = VY*G rows.  Thread 0 is also the producer: at plane i it
// loads plane i + S - 1 into the stage that plane i - 1 held, once every warp
// has released it; the other warps may run up to S - 1 planes ahead.
// blockIdx.z = band within this launch * nxc + axis-0 chunk; band0 is the
// first band's index in the tensor maps.
template <int R, int VY, int G, int S>
__global__ void __launch_bounds__(32 * G, 2)
star_tma_kernel(cplx<double>* __restrict__ out, const StarParams<double> p,
                const __grid_constant__ TmaMaps maps, int band0, int* err) {
  pdl_enter();
  using V = cplx<double>;
  constexpr int BY = VY * G, NT = 32 * G, NW = NT / 32, Q = 2 * R + 1;
  using St = TmaStage<R, BY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* sbase = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  V* stages = reinterpret_cast<V*>(sbase);
  uint64_t* full = reinterpret_cast<uint64_t*>(sbase + size_t(S) * St::BYTES);
  uint64_t* empty = full + S;
  __shared__ int abort_flag;  // set by the first thread whose wait expired

  const int t = threadIdx.x;
  const int z0 = blockIdx.x * kTmaBZ, y0 = blockIdx.y * BY;
  const int bl = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int x0 = xc * p.x_chunk, x1 = min(p.n0, x0 + p.x_chunk);
  const int pbeg = x0 - R, pend = x1 + R, nplanes = pend - pbeg;

  if (t == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NW);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // Plane i into stage i % S: own rows, halo rows and halo columns at wrapped
  // coordinates (periodic axes) or off-grid ones (zero boundaries).
  auto issue = [&](int i) {
    const int s = i % S;
    int xp = pbeg + i;
    int yt = y0 - R, yb = y0 + BY, zl = z0 - R, zr = z0 + kTmaBZ;
    if (p.per0) {
      if (xp < 0) xp += p.n0;
      else if (xp >= p.n0) xp -= p.n0;
    }
    if (p.per1) {
      if (yt < 0) yt += p.n1;
      if (yb >= p.n1) yb -= p.n1;
    }
    if (p.per2) {
      if (zl < 0) zl += p.n2;
      if (zr >= p.n2) zr -= p.n2;
    }
    const int band = band0 + bl;
    V* st = stages + s * St::CELLS;
    mbar_arrive_expect_tx(&full[s], St::BYTES);
    tma_load_4d(st, &maps.rows_halo, &full[s], 2 * z0, yt, xp, band);
    tma_load_4d(st + R * kTmaBZ, &maps.rows_own, &full[s], 2 * z0, y0, xp, band);
    tma_load_4d(st + (R + BY) * kTmaBZ, &maps.rows_halo, &full[s], 2 * z0, yb, xp, band);
    tma_load_4d(st + St::ROWS, &maps.side, &full[s], 2 * zl, y0, xp, band);
    tma_load_4d(st + St::ROWS + St::SIDE, &maps.side, &full[s], 2 * zr, y0, xp, band);
  };
  int issued = 0;
  if (t == 0)
    for (; issued < min(S - 1, nplanes); issued++) issue(issued);

  const int zt = t & (kTmaBZ - 1), g = t / 32, lane = t & 31;
  // Bloch phases of wrapped halos (tile-uniform; only with y/z phases).
  const bool fx = p.fix_yz != 0;
  const unsigned wflags = fx ? (unsigned(p.per1 && y0 == 0) | unsigned(p.per1 && y0 + BY >= p.n1) << 1 |
                                 unsigned(p.per2 && z0 == 0) << 2 |
                                 unsigned(p.per2 && z0 + kTmaBZ >= p.n2) << 3)
                              : 0u;
  const long long plane = (long long)p.n1 * p.n2;
  V* outb = out + bl * p.band;
  const int z = z0 + zt;
  unsigned own_ok = 0;
#pragma unroll
  for (int j = 0; j < VY; j++)
    if (y0 + VY * g + j < p.n1 && z < p.n2) own_ok |= 1u << j;
  const long long own_off = (long long)(y0 + VY * g) * p.n2 + z;

  V acc[VY][Q];
#pragma unroll
  for (int j = 0; j < VY; j++)
#pragma unroll
    for (int q = 0; q < Q; q++) acc[j][q] = vzero<V>();

  bool failed = false;
  for (int base = 0; base < nplanes; base += Q) {
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      const int i = base + u;
      if (i < nplanes) {
        const int s = i % S;
        if (t == 0 && !failed && i + S - 1 < nplanes) {
          const int j = i + S - 1;  // its stage held plane i - 1
          if (j >= S && !mbar_wait(&empty[j % S], unsigned(j / S + 1) & 1u, &abort_flag)) {
            failed = true;
            abort_flag = 1;
          } else {
            issue(j);
            issued = j + 1;
          }
        }
        if (!failed && !mbar_wait(&full[s], unsigned(i / S) & 1u, &abort_flag)) {
          failed = true;
          abort_flag = 1;
        }
        const V* st = stages + s * St::CELLS;
        const int pl = pbeg + i;
        int xside;
        const int xs = wrap_plane(pl, p.n0, p.per0, xside);
        V own[VY];
        if (!failed) {
          if (pl >= x0 && pl < x1) {
            V sum[VY];
            if (wflags) tma_plane<R, VY, BY, true>(st, g, zt, p, wflags, sum, own);
            else tma_plane<R, VY, BY, false>(st, g, zt, p, 0u, sum, own);
#pragma unroll
            for (int j = 0; j < VY; j++) acc[j][u] = vadd(acc[j][u], sum[j]);
          } else {
#pragma unroll
            for (int j = 0; j < VY; j++)
              own[j] = st[(R + VY * g + j) * kTmaBZ + zt];
          }
          if (xs >= 0 && xside >= 0) {
            // Own cells of a wrapped plane take the axis-0 phase.
#pragma unroll
            for (int j = 0; j < VY; j++)
              own[j] = cmul(p.P.ph[0][xside], own[j]);
          }
        }
        // Stage read (or abandoned): release it to the producer.
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);

        if (!failed) {
          if (xs >= 0) {
#pragma unroll
            for (int j = 0; j < VY; j++)
#pragma unroll
              for (int k = 1; k <= R; k++) {
                madd(acc[j][(u - k + Q) % Q], p.cx[kMaxR + k], own[j]);
                madd(acc[j][(u + k) % Q], p.cx[kMaxR - k], own[j]);
              }
          }
          const int q = pl - R;
          const int qs = (u - R + Q) % Q;  // slot of output pl - R
          if (q >= x0 && q < x1) {
            V* dst = outb + q * plane + own_off;
#pragma unroll
            for (int j = 0; j < VY; j++)
              if (own_ok >> j & 1u) stcs(dst + (long long)j * p.n2, acc[j][qs]);
          }
#pragma unroll
          for (int j = 0; j < VY; j++) acc[j][qs] = vzero<V>();
        }
      }
    }
  }
  if (failed) {
    atomicExch(err, 1);
    // Let the loads already issued land before the CTA exits.
    if (t == 0)
      for (int k = max(0, issued - S); k < issued; k++)
        mbar_wait(&full[k % S], unsigned(k / S) & 1u, nullptr);
  }
}

}  // namespace gfd
