// stencil_tmasplit.cuh -- complex128 star stencils: full-row tiles staged by
// TMA, real and imaginary parts on neighbouring lanes.
//
// Same computation as star_kernel (c/bmgs/fd.c:16-51 over the Bloch-phased
// halo of c/bc.c:138-250; Jacobi and residual modes of c/bmgs/relax.c) and
// the same arithmetic per point as star_split_kernel (stencil_split.cuh):
// lane 2k + c computes component c of columns 2k, 2k + 1 for VY rows, and
// staged rows are split by column parity so every shared load of a warp is
// 32 consecutive doubles.  What changes is the fill:
//
//  * A CTA covers BY rows by the whole row (n2 columns, in groups of 32 per
//    warp) and marches along axis 0.  Thread 0 stages each plane with tensor
//    (TMA) copies -- one box per column parity, taking every second column
//    (element stride 2 on the column axis), so the parity split costs no
//    instruction at all.  16-byte cp.async copies, in contrast, were found to
//    move one 32-byte L2 sector per lane in their cache-bypass form and to
//    write shared memory one lane at a time.
//  * Zero boundaries come from the copy's zero fill past the array's edge
//    (rows, columns and planes alike).  On a periodic axis 1 the box is split
//    by rows at the wrap; a periodic axis 0 is wrapped in the plane
//    coordinate.  The halo columns of a periodic axis 2 lie in the same row,
//    already staged: after the copy lands they are copied across within
//    shared memory.  Bloch phases are applied in the same pass, by the
//    thread that writes the cell, before the CTA barrier of the plane.
//  * One CTA barrier per plane orders the fix-up before the reads and every
//    read of a stage before thread 0 refills it.  (A form without it, with
//    an "empty" mbarrier per stage and per-warp fix-ups, measured slower: it
//    needs more registers and spilled.)
//  * Every wait on an mbarrier is bounded; a wait that runs out sets the
//    shared abort flag (which cuts the other threads' waits short), the CTA
//    leaves the march together at the plane's barrier (a barrier that ORs
//    every thread's failure), thread 0 drains the copies it issued and the
//    device error flag is set.
#pragma once

#include "internal.h"
#include "stencil_split.cuh"
#include "stencil_tma.cuh"

namespace gfd {

// Rows per lane (a build-time knob for measuring other shapes).
#ifndef GFD_TS_VY
#define GFD_TS_VY 4
#endif
constexpr int kTsVY = GFD_TS_VY;  // rows per lane
constexpr int kTsWY = 2;        // warps per column group
constexpr int kTsBY = kTsVY * kTsWY;
constexpr int kTsMaxNG = 4;     // column groups (n2 <= 128)


// Values per parity half-row, rounded up so every staged row starts on a
// 128-byte boundary (the alignment of a tensor copy's destination).
__host__ __device__ constexpr int ts_pw(int ng, int re) { return (16 * ng + re + 7) / 8 * 8; }
// Values per parity half-row of a staged source term (own columns only).
__host__ __device__ constexpr int ts_pwr(int ng) { return (16 * ng + 7) / 8 * 8; }

template <int R, int MODE>
struct TsLayout {
  static constexpr int RE = (R + 1) & ~1;
  static constexpr int SY = kTsBY + 2 * R;
  static constexpr bool RHO = MODE == MODE_JACOBI || MODE == MODE_RESIDUAL;
  static constexpr bool POT = MODE == MODE_POTENTIAL;
  static constexpr int S = (RHO || POT) ? 3 : 4;
  // Bytes of one stage for ng column groups: the planes's two parity
  // blocks [SY][PW], the source term's two parity blocks [BY][PWR], the
  // potential [BY][32 ng].
  __host__ __device__ static constexpr unsigned tile_bytes(int ng) {
    return unsigned(2 * SY * ts_pw(ng, RE) * 16);
  }
  __host__ __device__ static constexpr unsigned rho_bytes(int ng) {
    return RHO ? unsigned(2 * kTsBY * ts_pwr(ng) * 16) : 0u;
  }
  __host__ __device__ static constexpr unsigned pot_bytes(int ng) {
    return POT ? unsigned(kTsBY * 32 * ng * 8) : 0u;
  }
  __host__ __device__ static constexpr unsigned stage_bytes(int ng) {
    return tile_bytes(ng) + rho_bytes(ng) + pot_bytes(ng);
  }
  __host__ __device__ static constexpr size_t smem_bytes(int ng) {
    return size_t(S) * stage_bytes(ng) + 128;  // + S mbarriers and the abort flag
  }
};

// Tensor maps of one launch.  Input bands as doubles (2, n2, n1, n0, nb) with
// element stride 2 on the column axis: rows_full spans the SY staged rows of
// a tile, rows_main SY - R of them, rows_own BY and rows_halo R (the pieces
// of a tile whose rows wrap on a periodic axis 1).  rho: the source term's
// own rows, same form; pot: the potential as (n2, n1, n0) doubles, box
// (32 ng, BY, 1).
struct TsMaps {
  CUtensorMap rows_full, rows_main, rows_own, rows_halo, rho, pot;
};

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

// One step of the axis-0 ring for ring slot U (= plane index mod Q): add
// the in-plane part of output plane pl (inp), spread plane pl's own values
// (own) into the outputs pl - R .. pl + R, and write output pl - R, whose
// slot is complete.  The slot of output pl + R, (U + R) mod Q, is the one
// written at the previous step: it is assigned here, not accumulated, so no
// slot is ever cleared.
template <int R, int MODE, int U>
__device__ __forceinline__ void ts_ring_step(double (&acc)[kTsVY][2][2 * R + 1],
                                             const double (&inp)[kTsVY][2],
                                             const double (&own)[kTsVY][2],
                                             const double (&src)[kTsVY][2], bool add_inp,
                                             bool add_own, bool store,
                                             const StarParams<double>& p, cplx<double>* dst,
                                             int n2, unsigned okm, int c) {
  constexpr int Q = 2 * R + 1;
  constexpr int F = (U + R) % Q;      // slot of output pl + R
  constexpr int D = (U - R + Q) % Q;  // slot of output pl - R (complete)
#pragma unroll
  for (int j = 0; j < kTsVY; j++)
#pragma unroll
    for (int v = 0; v < 2; v++) {
      if (add_inp) acc[j][v][U] += inp[j][v];
      if (add_own) {
#pragma unroll
        for (int m = 1; m <= R; m++)
          acc[j][v][(U - m + Q) % Q] = fma(p.cx[kMaxR + m], own[j][v], acc[j][v][(U - m + Q) % Q]);
#pragma unroll
        for (int m = 1; m < R; m++)
          acc[j][v][(U + m) % Q] = fma(p.cx[kMaxR - m], own[j][v], acc[j][v][(U + m) % Q]);
      }
    }
  if (store) {
#pragma unroll
    for (int j = 0; j < kTsVY; j++) {
      double r0 = acc[j][0][D], r1 = acc[j][1][D];
      if constexpr (MODE == MODE_JACOBI) {
        r0 = p.wc * (src[j][0] - r0);
        r1 = p.wc * (src[j][1] - r1);
      } else if constexpr (MODE == MODE_RESIDUAL) {
        r0 = r0 - src[j][0];
        r1 = r1 - src[j][1];
      }
      // Lane c = 0 holds the real parts of columns 2k, 2k+1, lane 1 the
      // imaginary parts: swap so each lane writes one whole value.
      const double give = c ? r0 : r1;
      const double got = __shfl_xor_sync(0xffffffffu, give, 1);
      cplx<double> o;
      o.re = c ? got : r0;
      o.im = c ? r1 : got;
      if (okm >> (2 * j + c) & 1u) stcs(dst + (long long)j * n2 + c, o);
    }
  }
#pragma unroll
  for (int j = 0; j < kTsVY; j++)
#pragma unroll
    for (int v = 0; v < 2; v++) acc[j][v][F] = add_own ? p.cx[kMaxR - R] * own[j][v] : 0.0;
}

// NG = ceil(n2 / 32) column groups (a template parameter, so every staged
// offset is a compile-time constant); blockDim.x = 32 * kTsWY * NG.  Grid:
// (1, ceil(n1 / BY), bands * nxc).  The register cap keeps about 12 warps per
// SM (at most 168 registers a thread) up to three column groups; four
// groups run one CTA per SM.
template <int NG>
constexpr int ts_min_ctas() {
  return NG == 1 ? 6 : NG == 2 ? 3 : NG == 3 ? 2 : 1;
}

template <int R, int MODE, int NG>
__global__ void __launch_bounds__(32 * kTsWY * NG, ts_min_ctas<NG>())
star_tmasplit_kernel(cplx<double>* __restrict__ out, const StarParams<double> p,
                     const __grid_constant__ TsMaps maps, int* err) {
  pdl_enter();
  using V = cplx<double>;
  using L = TsLayout<R, MODE>;
  constexpr int VY = kTsVY, BY = kTsBY, RE = L::RE, SY = L::SY, S = L::S;
  constexpr int Q = 2 * R + 1;
  constexpr bool RHO = L::RHO, POT = L::POT;
  constexpr int ng = NG;
  constexpr int PW = ts_pw(ng, RE), PWR = ts_pwr(ng), PWV = 32 * ng;
  constexpr unsigned tile_b = L::tile_bytes(ng), rho_b = L::rho_bytes(ng),
                     stage_b = L::stage_bytes(ng);

  extern __shared__ __align__(128) unsigned char ts_smem[];
  unsigned char* stages = ts_smem;
  uint64_t* full = reinterpret_cast<uint64_t*>(ts_smem + size_t(S) * stage_b);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + S);

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int g = warp % ng, wy = warp / ng;
  const int k = lane >> 1, c = lane & 1;
  const int y0 = blockIdx.y * BY;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int x0 = xc * p.x_chunk, x1 = min(p.n0, x0 + p.x_chunk);
  const int pbeg = x0 - R, pend = x1 + R, nplanes = pend - pbeg;
  const long long plane = (long long)p.n1 * p.n2;

  if (t == 0) {
    for (int i = 0; i < S; i++) mbar_init(&full[i], 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // Row pieces of a tile on a periodic axis 1 (n1 a multiple of BY): the
  // first and last tiles take their wrapped halo rows from the far side.
  const bool ylo = p.per1 && y0 == 0, yhi = p.per1 && y0 + BY >= p.n1;

  // Stage plane i (of this CTA's march) into stage i % S.  Thread 0 only.
  auto issue = [&](int i) {
    const int st_i = i % S;
    const int P = pbeg + i;
    int xp = P;  // off-grid planes of a zero boundary read as zeros
    if (p.per0) xp = P < 0 ? P + p.n0 : (P >= p.n0 ? P - p.n0 : P);
    const int q = P - R;
    const bool rho_now = RHO && q >= x0 && q < x1;
    const bool pot_now = POT && P >= x0 && P < x1;
    unsigned char* st = stages + size_t(st_i) * stage_b;
    uint64_t* bar = &full[st_i];
    mbar_arrive_expect_tx(bar, tile_b + (rho_now ? rho_b : 0u) + (pot_now ? L::pot_bytes(ng) : 0u));
    for (int par = 0; par < 2; par++) {
      unsigned char* blk = st + size_t(par) * SY * PW * 16;
      const int col = par - RE;
      if (!ylo && !yhi) {
        tma_load_5d(blk, &maps.rows_full, bar, 0, col, y0 - R, xp, bnd);
      } else if (ylo && yhi) {
        tma_load_5d(blk, &maps.rows_halo, bar, 0, col, p.n1 - R, xp, bnd);
        tma_load_5d(blk + size_t(R) * PW * 16, &maps.rows_own, bar, 0, col, 0, xp, bnd);
        tma_load_5d(blk + size_t(R + BY) * PW * 16, &maps.rows_halo, bar, 0, col, 0, xp, bnd);
      } else if (ylo) {
        tma_load_5d(blk, &maps.rows_halo, bar, 0, col, p.n1 - R, xp, bnd);
        tma_load_5d(blk + size_t(R) * PW * 16, &maps.rows_main, bar, 0, col, 0, xp, bnd);
      } else {
        tma_load_5d(blk, &maps.rows_main, bar, 0, col, y0 - R, xp, bnd);
        tma_load_5d(blk + size_t(SY - R) * PW * 16, &maps.rows_halo, bar, 0, col, 0, xp, bnd);
      }
    }
    if constexpr (RHO) {
      if (rho_now) {
        unsigned char* rb = st + tile_b;
        tma_load_5d(rb, &maps.rho, bar, 0, 0, y0, q, bnd);
        tma_load_5d(rb + size_t(BY) * PWR * 16, &maps.rho, bar, 0, 1, y0, q, bnd);
      }
    }
    if constexpr (POT) {
      if (pot_now) tma_load_3d(st + tile_b + rho_b, &maps.pot, bar, 0, y0, P);
    }
  };

  int issued = 0;
  if (t == 0)
    for (; issued < min(S - 1, nplanes); issued++) issue(issued);

  // This lane's points: rows y0 + wy VY + j, columns 32 g + 2k + v.
  const int yb = y0 + wy * VY, zc = 32 * g + 2 * k;
  unsigned okm = 0;  // bit 2j + v: point (j, v) inside the grid
#pragma unroll
  for (int j = 0; j < VY; j++) {
    if (yb + j < p.n1 && zc < p.n2) okm |= 1u << (2 * j);
    if (yb + j < p.n1 && zc + 1 < p.n2) okm |= 1u << (2 * j + 1);
  }
  const long long own_off = (long long)(yb < p.n1 ? yb : 0) * p.n2 + (zc < p.n2 ? zc : 0);
  V* outb = out + bnd * p.band;

  // Bloch phases of wrapped halo rows (axis 1) that the fix-up applies.
  auto nontrivial = [](const cplx<double>& ph) { return ph.re != 1.0 || ph.im != 0.0; };
  const bool phy_lo = ylo && nontrivial(p.P.ph[1][1]);
  const bool phy_hi = yhi && nontrivial(p.P.ph[1][0]);

  double acc[VY][2][Q];
#pragma unroll
  for (int j = 0; j < VY; j++)
#pragma unroll
    for (int v = 0; v < 2; v++)
#pragma unroll
      for (int qq = 0; qq < Q; qq++) acc[j][v][qq] = 0.0;

  // Scalar view; column 2k + v of group g, staged row r, is at
  // ((par(v) SY + r) PW + 16 g + k + h(v)) 2 + c, par(v) = (v + RE) & 1,
  // h(v) = (v + RE) >> 1.
  const int lane_s = ((R + wy * VY) * PW + 16 * g + k) * 2 + c;
  constexpr int par_s = SY * PW * 2;
  constexpr int row_s = PW * 2;
  auto col_off = [](int v) { return ((v + RE) & 1) * par_s + ((v + RE) >> 1) * 2; };

  bool failed = false;
  int s = 0, slot = 0;   // plane index mod S and mod Q
  unsigned phase = 0;    // completed uses of stage s, mod 2
  for (int i = 0; i < nplanes; i++) {
    const int pl = pbeg + i;
    if (!failed && !mbar_wait_bounded(&full[s], phase, abort_flag)) {
      failed = true;
      *abort_flag = 1;
    }
    int xside;
    const int xs = wrap_plane(pl, p.n0, p.per0, xside);
    const bool out_plane = pl >= x0 && pl < x1;
    unsigned char* stp = stages + size_t(s) * stage_b;
    V* tile = reinterpret_cast<V*>(stp);
    if (!failed) {
      // Fix-up pass over the whole tile: halo columns of a periodic axis 2
      // from the same row, Bloch phases of wrapped rows (axis 1) and planes
      // (axis 0).
      const bool fz = p.per2 && out_plane;
      const bool fy = (phy_lo || phy_hi) && out_plane;
      const bool fx = xside >= 0 && nontrivial(p.P.ph[0][xside]);
      if (fz || fy || fx) {
        auto cell = [&](int r, int lc) -> V& {
          const int u2 = lc + RE;
          return tile[((u2 & 1) * SY + r) * PW + (u2 >> 1)];
        };
        constexpr int nt = 32 * kTsWY * NG;
        if (fz) {
          for (int e = t; e < BY * 2 * R; e += nt) {
            const int r = R + e / (2 * R), sd = e % (2 * R);
            const int lc = sd < R ? sd - R : p.n2 + (sd - R);
            const int side = sd < R ? 1 : 0;
            V v = cell(r, sd < R ? lc + p.n2 : lc - p.n2);
            if (nontrivial(p.P.ph[2][side])) v = cmul(p.P.ph[2][side], v);
            cell(r, lc) = v;
          }
        }
        if (fy) {
          for (int e = t; e < 2 * R * p.n2; e += nt) {
            const int rr = e / p.n2, lc = e % p.n2;
            const bool lo = rr < R;
            if (lo ? phy_lo : phy_hi) {
              const int r = lo ? rr : BY + rr;
              V& v = cell(r, lc);
              v = cmul(p.P.ph[1][lo ? 1 : 0], v);
            }
          }
        }
        if (fx) {
          const cplx<double> ph = p.P.ph[0][xside];
          for (int e = t; e < BY * p.n2; e += nt) {
            V& v = cell(R + e / p.n2, e % p.n2);
            v = cmul(ph, v);
          }
        }
      }
    }
    // One decision for the whole CTA: a thread's wait that ran out ends the
    // march for every thread at this barrier.  (The shared abort flag only
    // shortens the other threads' waits; reading it after a plain barrier
    // could race with a thread that already moved on to the next wait.)
    if (__syncthreads_or(failed)) {
      failed = true;
      break;
    }
    if (t == 0 && i + S - 1 < nplanes) {
      // The stage of plane i - 1: read (and patched) by every thread before
      // the barrier; the patches were generic-proxy writes.
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue(i + S - 1);
      issued = i + S;
    }

    // In-plane terms of output plane pl (8 independent chains, one per
    // point, interleaved) and the own values.
    const double* T = reinterpret_cast<const double*>(stp) + lane_s;
    double inp[VY][2], own[VY][2];
    if (out_plane) {
#pragma unroll
      for (int j = 0; j < VY; j++) {
        double row[2 + 2 * R];
#pragma unroll
        for (int v = -R; v <= 1 + R; v++) row[v + R] = T[j * row_s + col_off(v)];
        double pv0 = 0.0, pv1 = 0.0;
        if constexpr (POT) {
          const double2 pp = *reinterpret_cast<const double2*>(
              stp + tile_b + rho_b + size_t((wy * VY + j) * PWV + zc) * 8);
          pv0 = pp.x;
          pv1 = pp.y;
        }
        own[j][0] = row[R];
        own[j][1] = row[R + 1];
        inp[j][0] = (p.c0 + pv0) * row[R];
        inp[j][1] = (p.c0 + pv1) * row[R + 1];
#pragma unroll
        for (int m = 1; m <= R; m++)
#pragma unroll
          for (int v = 0; v < 2; v++) {
            inp[j][v] = fma(p.cz[kMaxR - m], row[R + v - m], inp[j][v]);
            inp[j][v] = fma(p.cz[kMaxR + m], row[R + v + m], inp[j][v]);
          }
      }
      // Axis-1 terms: the staged rows above and below the lane's block.
      double up[R][2], dn[R][2];
#pragma unroll
      for (int m = 1; m <= R; m++)
#pragma unroll
        for (int v = 0; v < 2; v++) {
          up[m - 1][v] = T[-m * row_s + col_off(v)];
          dn[m - 1][v] = T[(VY - 1 + m) * row_s + col_off(v)];
        }
#pragma unroll
      for (int m = 1; m <= R; m++)
#pragma unroll
        for (int j = 0; j < VY; j++)
#pragma unroll
          for (int v = 0; v < 2; v++) {
            const double lo = j - m >= 0 ? own[j - m][v] : up[m - j - 1][v];
            const double hi = j + m < VY ? own[j + m][v] : dn[j + m - VY][v];
            inp[j][v] = fma(p.cy[kMaxR - m], lo, inp[j][v]);
            inp[j][v] = fma(p.cy[kMaxR + m], hi, inp[j][v]);
          }
    } else {
#pragma unroll
      for (int j = 0; j < VY; j++) {
        own[j][0] = T[j * row_s + col_off(0)];
        own[j][1] = T[j * row_s + col_off(1)];
        inp[j][0] = inp[j][1] = 0.0;
      }
    }

    // Output plane pl - R: its source term (Jacobi / residual) and address.
    const int q = pl - R;
    const bool store = q >= x0 && q < x1;
    double src[VY][2];
#pragma unroll
    for (int j = 0; j < VY; j++) src[j][0] = src[j][1] = 0.0;
    if constexpr (RHO) {
      if (store) {
        const double* rt = reinterpret_cast<const double*>(stp + tile_b) +
                           ((wy * VY) * PWR + 16 * g + k) * 2 + c;
#pragma unroll
        for (int j = 0; j < VY; j++) {
          src[j][0] = rt[j * PWR * 2];                    // column 2k: even block
          src[j][1] = rt[j * PWR * 2 + BY * PWR * 2];     // column 2k + 1: odd block
        }
      }
    }
    V* dst = outb + q * plane + own_off;
    const bool add_own = xs >= 0;
    switch (slot) {
#define GFD_TS_STEP(UU)                                                                        \
  case UU:                                                                                     \
    if constexpr (UU < Q)                                                                      \
      ts_ring_step<R, MODE, (UU < Q ? UU : 0)>(acc, inp, own, src, out_plane, add_own, store, p, \
                                               dst, p.n2, okm, c);                             \
    break;
      GFD_TS_STEP(0)
      GFD_TS_STEP(1)
      GFD_TS_STEP(2)
      GFD_TS_STEP(3)
      GFD_TS_STEP(4)
      GFD_TS_STEP(5)
      GFD_TS_STEP(6)
#undef GFD_TS_STEP
    }
    if (++s == S) {
      s = 0;
      phase ^= 1u;
    }
    if (++slot == Q) slot = 0;
  }
  if (failed) {
    if (t == 0) {
      atomicExch(err, 1);
      // Let the copies already issued land before the CTA exits.
      for (int kk = max(0, issued - S); kk < issued; kk++)
        mbar_wait_bounded(&full[kk % S], unsigned(kk / S) & 1u, nullptr);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side.  Defined in operator.cu: the switch, the error flag and the maps.
// ---------------------------------------------------------------------------
bool tmasplit_enabled();
int* star_error_flag();
int encode_ts_maps(TsMaps* maps, const void* in, const void* rho, const void* pot,
                   const gfd_operator* op, int64_t nb, int R, int ng);

template <int R, int MODE, int NG>
int ts_go(const gfd_operator* op, const cplx<double>* in, cplx<double>* out,
          const cplx<double>* rho, const void* pot, int64_t nin, const StarParams<double>& base,
          int cps, cudaStream_t s) {
  using L = TsLayout<R, MODE>;
  constexpr size_t smem = L::smem_bytes(NG);
  auto kern = star_tmasplit_kernel<R, MODE, NG>;
  int st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem),
                      "cudaFuncSetAttribute(star_tmasplit_kernel)");
  if (st) return st;
  if ((st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            int(cudaSharedmemCarveoutMaxShared)),
                       "cudaFuncSetAttribute(carveout)")))
    return st;
  int* err = star_error_flag();
  if (!err) return GFD_ECUDA;
  // Axis-0 split as for the marching kernels: about cps CTAs per SM.
  const int gy = (op->n[1] + kTsBY - 1) / kTsBY;
  const int64_t tiles = (int64_t)gy * (nin > 1 ? nin : 1);
  const int64_t target = (int64_t)(cps > 0 ? cps : march_ctas_per_sm()) * num_sms();
  const int maxc = op->n[0] / (2 * R > 4 ? 2 * R : 4) > 1 ? op->n[0] / (2 * R > 4 ? 2 * R : 4) : 1;
  int64_t want = (target + tiles - 1) / tiles;
  int nxc = int(want < 1 ? 1 : (want > maxc ? maxc : want));
  StarParams<double> p = base;
  p.x_chunk = (op->n[0] + nxc - 1) / nxc;
  p.nxc = nxc = (op->n[0] + p.x_chunk - 1) / p.x_chunk;
  const int64_t per_launch = 65535 / nxc > 1 ? 65535 / nxc : 1;
  const long long band = (long long)op->n[0] * op->n[1] * op->n[2];
  for (int64_t b0 = 0; b0 < nin; b0 += per_launch) {
    const int64_t nb = nin - b0 < per_launch ? nin - b0 : per_launch;
    TsMaps maps;
    if ((st = encode_ts_maps(&maps, in + b0 * band, rho ? rho + b0 * band : nullptr, pot, op, nb,
                             R, NG)))
      return st;
    launch_k(kern, dim3(1, gy, (unsigned)(nb * nxc)), 32 * kTsWY * NG, smem, s, out + b0 * band,
             p, maps, err);
  }
  return check_launch("star_tmasplit_kernel");
}

// mode: MODE_APPLY / MODE_POTENTIAL (pot = the potential) / MODE_JACOBI /
// MODE_RESIDUAL (rho = the source term).
template <int NG>
int ts_launch_ng(const gfd_operator* op, int mode, const cplx<double>* in, cplx<double>* out,
                 const cplx<double>* rho, const void* pot, int64_t nin,
                 const StarParams<double>& p, int cps, cudaStream_t s) {
#define GFD_TS_MODES(RR)                                                                   \
  case RR:                                                                                 \
    switch (mode) {                                                                        \
      case MODE_APPLY: return ts_go<RR, MODE_APPLY, NG>(op, in, out, rho, pot, nin, p, cps, s); \
      case MODE_POTENTIAL:                                                                 \
        return ts_go<RR, MODE_POTENTIAL, NG>(op, in, out, rho, pot, nin, p, cps, s);       \
      case MODE_JACOBI: return ts_go<RR, MODE_JACOBI, NG>(op, in, out, rho, pot, nin, p, cps, s); \
      case MODE_RESIDUAL:                                                                  \
        return ts_go<RR, MODE_RESIDUAL, NG>(op, in, out, rho, pot, nin, p, cps, s);        \
    }                                                                                      \
    break;
  switch (op->R) {
    GFD_TS_MODES(1)
    GFD_TS_MODES(2)
    GFD_TS_MODES(3)
  }
#undef GFD_TS_MODES
  return set_error(GFD_EUNSUPPORTED, "TMA lane-pair stencil: radius <= 3");
}

}  // namespace gfd

// One translation unit per column-group count (stencil_ts<NG>.cu).
#define GFD_DECLARE_TS_ENTRY(NG)                                                            \
  namespace gfd {                                                                          \
  int ts_launch_##NG(const gfd_operator* op, int mode, const cplx<double>* in,             \
                     cplx<double>* out, const cplx<double>* rho, const void* pot, int64_t nin, \
                     const StarParams<double>& p, int cps, cudaStream_t s);                \
  }
#define GFD_DEFINE_TS_ENTRY(NG)                                                             \
  namespace gfd {                                                                          \
  int ts_launch_##NG(const gfd_operator* op, int mode, const cplx<double>* in,             \
                     cplx<double>* out, const cplx<double>* rho, const void* pot, int64_t nin, \
                     const StarParams<double>& p, int cps, cudaStream_t s) {               \
    return ts_launch_ng<NG>(op, mode, in, out, rho, pot, nin, p, cps, s);                  \
  }                                                                                        \
  }
