// stencil.cuh -- band-batched 3-D finite-difference stencils for sm_100a.
//
// Reference computation (c/bmgs/fd.c:16-51 over the halo-padded copy that
// c/bc.c:138-250 builds): out[g] = sum_p coefs[p] * a[g + offsets[p]], with
// zero or (Bloch-)periodic halos.  Here the padded copy does not exist: every
// kernel maps out-of-domain coordinates itself (wrap_axis), so a band is read
// from HBM once and written once.
//
// star_kernel  axis-aligned stencils (Laplace/Gradient on orthorhombic
//   grids, the reference's cfd case).  A CTA owns a BY x BZ column of
//   points and marches along axis 0 (the largest stride).  Each thread keeps
//   a shift register of 2R+1 partial sums for its points; a plane's own
//   values arrive in registers (prefetched D planes ahead) and contribute to
//   the 2R+1 outputs around it, so x-neighbours are never re-read.  The
//   in-plane (axis 1 / axis 2) neighbours come from a double-buffered shared
//   memory tile that the CTA fills with the plane's own values plus a halo
//   of R rows/columns.  One __syncthreads per plane.
//   MODE selects the epilogue: plain apply, weighted-Jacobi update
//   (c/bmgs/relax.c:46-71), or residual L a - rho with per-CTA sums of r^2.
//
// general_kernel  any offset set (cross terms of non-orthogonal cells,
//   Mehrstellen): a ring of 2*MP+1 shared-memory planes with full halos.
//
// color_gs_kernel  one colour of multicolour Gauss-Seidel.
#pragma once

#include "common.cuh"

namespace gfd {

constexpr int kMaxR = 6;      // largest star radius (stencil order 2*6)
constexpr int kMaxCoefs = 128;  // general kernel

enum { MODE_APPLY = 0, MODE_JACOBI = 1, MODE_RESIDUAL = 2, MODE_POTENTIAL = 3 };

template <class S>
struct StarParams {
  int n0, n1, n2;
  int per0, per1, per2;
  int x_chunk;      // outputs along axis 0 per CTA
  int nxc;          // number of axis-0 chunks
  long long band;   // elements per band
  S c0;             // centre weight (MODE_JACOBI: the folded centre weight, see below)
  S cx[2 * kMaxR + 1];  // weight of offset k along axis 0 at index kMaxR + k
  S cy[2 * kMaxR + 1];
  S cz[2 * kMaxR + 1];
  S wc;             // MODE_JACOBI: w / coefs[0] (negated for the negated sweep)
  int fix_yz;       // complex: the tile needs y/z Bloch phases on wrapped cells
  Phases<S> P;
  double* partials; // MODE_RESIDUAL: one sum of r^2 per CTA (or nullptr)
  const void* pot;  // MODE_POTENTIAL: real potential v (one grid, type S)
};

// mbarriers and bounded waits on their phases (the TMA-staged kernels).
constexpr int kSpinIters = 1 << 26;               // mbarrier wait: iterations
constexpr long long kSpinCycles = 4000000000LL;   // and SM cycles (about 2 s)

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of the given parity to complete; false when the limit
// expired first or *abort became nonzero.  test_wait never suspends the
// thread, so a waiting warp resumes as soon as the phase completes; the
// iteration count and the cycle counter bound the total time.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity,
                                          const volatile int* abort) {
  if (mbar_test_wait(b, parity)) return true;
  const long long t0 = clock64();
  for (int i = 0; i < kSpinIters; i++) {
    if (mbar_test_wait(b, parity)) return true;
    if ((abort && *abort) || clock64() - t0 > kSpinCycles) break;
  }
  return false;
}
// Bounded wait on an mbarrier phase.  try_wait suspends the thread for a
// while when the phase is not complete, so waiting warps take few issue
// slots; the iteration count and the cycle counter bound the total time.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, unsigned parity,
                                                  const volatile int* abort,
                                                  long long max_cycles = kSpinCycles) {
  if (mbar_try_wait(b, parity)) return true;
  const long long t0 = clock64();
  for (int i = 0; i < kSpinIters; i++) {
    if (mbar_try_wait(b, parity)) return true;
    if ((abort && *abort) || clock64() - t0 > max_cycles) break;
  }
  return false;
}

// Block-wide sum of one double per thread in a fixed order.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NT / 32; i++) s += red[i];
  return s;
}

template <int BZ, int TY, int VY, int R, int S, class V, int MODE>
constexpr size_t star_smem_bytes() {
  constexpr bool RHO = MODE == MODE_JACOBI || MODE == MODE_RESIDUAL;
  constexpr bool POT = MODE == MODE_POTENTIAL;
  return size_t(S) * ((TY * VY + 2 * R) * (BZ + 2 * R) + (RHO ? TY * VY * BZ : 0)) * sizeof(V) +
         (POT ? size_t(S) * TY * VY * BZ * sizeof(typename vt<V>::S) : 0);
}

// Axis-aligned ("star") stencil, marching along axis 0.
//
//  * A CTA owns BY = TY*VY rows (axis 1) by BZ columns (axis 2); thread
//    (tz, ty) owns the VY consecutive rows ty*VY .. ty*VY+VY-1 at column tz.
//  * Planes stream through an S-stage shared-memory ring filled by cp.async:
//    the plane's tile plus an R-wide halo (corners skipped), zero-filled on
//    zero boundaries and wrapped on periodic ones (Bloch phases applied by
//    the thread that copied the cell, after its copy landed).  Planes
//    outside this CTA's axis-0 chunk are copied without their halo.
//  * Axis-1 neighbours and the own values come from one column read of
//    VY+2R cells; axis-2 neighbours from 2R reads per point.
//  * Axis 0: each point keeps 2R+1 partial sums in registers; plane p adds
//    its own value into the sums of outputs p-R..p+R.  The plane loop is
//    unrolled by 2R+1 so the ring index of every sum is a compile-time
//    constant.
//  * MODE_JACOBI folds the (1-w) phi term into the centre weight:
//    phi_new = (w/c0) (rho - sum_{p>=1} c_p phi_p - c0' phi) with
//    c0' = -(1-w) c0 / w, which equals (1-w) phi + w (rho - sum) / c0.
//  * The source term of MODE_JACOBI / MODE_RESIDUAL travels in the same
//    pipeline stages.
// CTAs per SM the register allocation is sized for: the short tile
// (32 x 4 threads, 2 rows each) and the 48-column tile (48 x 4 threads,
// 2 rows each), both for complex128 apply up to radius 4.  Measured on the
// 512-band 96^3 complex128 Laplace: the short tile at 3 CTAs per SM (up to
// 170 registers) 3934 GB/s against 3744 at 4 (128 registers, the limit
// there) and 3232 at 2; the 48-column tile at 2 per SM 4010-4099, at 3
// (spilling) 2770.
constexpr int kShortTileZ = 32, kTile48Z = 48;
template <int BZ, int TY, int VY>
constexpr int star_min_ctas() {
  return TY == 4 && VY == 2 ? (BZ == kShortTileZ ? 3 : (BZ == kTile48Z ? 2 : 1)) : 1;
}

template <class V, int R, int BZ, int TY, int VY, int S, int MODE>
__global__ void __launch_bounds__(BZ * TY, star_min_ctas<BZ, TY, VY>())
star_kernel(const V* __restrict__ in, V* __restrict__ out, const V* __restrict__ rho,
            const StarParams<typename vt<V>::S> p) {
  pdl_enter();
  using Sc = typename vt<V>::S;
  constexpr int NT = BZ * TY, BY = TY * VY;
  constexpr int SY = BY + 2 * R, SZ = BZ + 2 * R, CELLS = SY * SZ;
  constexpr int CPT = (CELLS + NT - 1) / NT;
  constexpr int Q = 2 * R + 1;
  constexpr bool RHO = MODE == MODE_JACOBI || MODE == MODE_RESIDUAL;
  constexpr bool POT = MODE == MODE_POTENTIAL;
  constexpr int RCELLS = RHO ? BY * BZ : 0;
  static_assert(S >= 2, "pipeline needs two stages");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* tiles = reinterpret_cast<V*>(smem_raw);  // [S][CELLS]
  V* rtiles = tiles + S * CELLS;              // [S][BY*BZ] source terms
  Sc* vtiles = reinterpret_cast<Sc*>(rtiles + S * RCELLS);  // [S][BY*BZ] potential
  __shared__ double red[NT / 32 > 0 ? NT / 32 : 1];

  const int t = threadIdx.x, tz = t % BZ, ty = t / BZ;
  const int z0 = blockIdx.x * BZ, y0 = blockIdx.y * BY;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int x0 = xc * p.x_chunk;
  const int x1 = min(p.n0, x0 + p.x_chunk);
  const long long plane = (long long)p.n1 * p.n2;
  const V* inb = in + bnd * p.band;
  V* outb = out + bnd * p.band;
  const V* rhob = RHO ? rho + bnd * p.band : nullptr;
  const int pbeg = x0 - R, pend = x1 + R;

  // Cells this thread copies (all cells of the halo box, corners included,
  // so the copy loop has no branches): byte offset of the source within a
  // plane (a valid dummy offset 0 for zero points, flagged in czero) and the
  // byte offset of the destination within a stage.  Wrap sides are kept
  // only for Bloch phases (y side bits 0-1, z side bits 2-3).
  unsigned csrc[CPT];
  unsigned cdst[CPT];
  unsigned czero = 0, clive = 0;  // bit i: zero point / cell exists
  int ccode[CPT];
  bool fix = false;
#pragma unroll
  for (int i = 0; i < CPT; i++) {
    const int c = t + i * NT;
    csrc[i] = 0;
    cdst[i] = unsigned(c) * unsigned(sizeof(V));
    ccode[i] = 0;
    if (c < CELLS) {
      clive |= 1u << i;
      const int sy = c / SZ, sz = c % SZ;
      int ysd, zsd;
      const int ys = wrap_axis(y0 - R + sy, p.n1, p.per1, ysd);
      const int zs = wrap_axis(z0 - R + sz, p.n2, p.per2, zsd);
      if (ys >= 0 && zs >= 0) {
        csrc[i] = unsigned(ys * p.n2 + zs) * unsigned(sizeof(V));
        if (ysd >= 0 || zsd >= 0) fix = true;
      } else {
        czero |= 1u << i;
      }
      ccode[i] = (ysd + 1) | ((zsd + 1) << 2);
    }
  }
  fix = fix && p.fix_yz;
  bool own_in[VY];
  unsigned own_b[VY];  // byte offset of an own point within a plane
#pragma unroll
  for (int j = 0; j < VY; j++) {
    const int y = y0 + ty * VY + j, z = z0 + tz;
    own_in[j] = y < p.n1 && z < p.n2;
    own_b[j] = own_in[j] ? unsigned(y * p.n2 + z) * unsigned(sizeof(V)) : 0u;
  }
  const unsigned smem0 = smem_addr(tiles);
  const unsigned rsmem0 = smem_addr(rtiles);
  const unsigned vsmem0 = smem_addr(vtiles);
  const char* pot_c = reinterpret_cast<const char*>(p.pot);
  const size_t plane_b = size_t(plane) * sizeof(V);
  const char* inb_c = reinterpret_cast<const char*>(inb);
  const char* rho_c = reinterpret_cast<const char*>(rhob);

  // Copy plane P (and the source term of output plane P - R) into stage
  // (P - pbeg) % S; always commits one group.
  auto issue = [&](int P) {
    if (P < pend) {
      const int st = (P - pbeg) % S;
      const unsigned sbase = smem0 + unsigned(st * CELLS * sizeof(V));
      int xside;
      const int xs = wrap_plane(P, p.n0, p.per0, xside);
      const char* src = inb_c + size_t(xs >= 0 ? xs : 0) * plane_b;
      const unsigned zmask = xs >= 0 ? czero : ~0u;
#pragma unroll
      for (int i = 0; i < CPT; i++) {
        if (!(clive >> i & 1u)) continue;
        const unsigned n = (zmask >> i & 1u) ? 0u : unsigned(sizeof(V));
        if constexpr (sizeof(V) == 16)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sbase + cdst[i]),
                       "l"(src + csrc[i]), "r"(n)
                       : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sbase + cdst[i]),
                       "l"(src + csrc[i]), "n"(int(sizeof(V))), "r"(n)
                       : "memory");
      }
      if constexpr (RHO) {
        const int q = P - R;
        if (q >= x0 && q < x1) {
          const unsigned rbase = rsmem0 + unsigned((st * RCELLS + ty * VY * BZ + tz) * sizeof(V));
          const char* rsrc = rho_c + size_t(q) * plane_b;
#pragma unroll
          for (int j = 0; j < VY; j++) {
            const unsigned n = own_in[j] ? unsigned(sizeof(V)) : 0u;
            const unsigned d = rbase + unsigned(j * BZ * sizeof(V));
            if constexpr (sizeof(V) == 16)
              asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d),
                           "l"(rsrc + own_b[j]), "r"(n)
                           : "memory");
            else
              asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d),
                           "l"(rsrc + own_b[j]), "n"(int(sizeof(V))), "r"(n)
                           : "memory");
          }
        }
      }
      if constexpr (POT) {
        // The potential of this plane's own points (same stage as the plane).
        if (P >= x0 && P < x1) {
          const unsigned vbase = vsmem0 + unsigned((st * BY * BZ + ty * VY * BZ + tz) * sizeof(Sc));
          const char* vsrc = pot_c + size_t(P) * size_t(plane) * sizeof(Sc);
#pragma unroll
          for (int j = 0; j < VY; j++) {
            const unsigned n = own_in[j] ? unsigned(sizeof(Sc)) : 0u;
            const unsigned d = vbase + unsigned(j * BZ * sizeof(Sc));
            asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d),
                         "l"(vsrc + own_b[j] / vt<V>::NC), "n"(int(sizeof(Sc))), "r"(n)
                         : "memory");
          }
        }
      }
    }
    cp_async_commit();
  };

#pragma unroll
  for (int k = 0; k < S - 1; k++) issue(pbeg + k);

  V acc[VY][Q];
#pragma unroll
  for (int j = 0; j < VY; j++)
#pragma unroll
    for (int q = 0; q < Q; q++) acc[j][q] = vzero<V>();
  double sumsq = 0.0;
  char* out_c = reinterpret_cast<char*>(outb);

  for (int base = pbeg; base < pend; base += Q) {
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      const int pl = base + u;
      if (pl < pend) {
        const int st = (pl - pbeg) % S;
        V* tile = tiles + st * CELLS;
        cp_async_wait<S - 2>();
        if constexpr (vt<V>::NC == 2) {
          if (fix) {
#pragma unroll
            for (int i = 0; i < CPT; i++) {
              if (!(clive >> i & 1u) || (czero >> i & 1u)) continue;
              const int ys = (ccode[i] & 3) - 1, zs = ((ccode[i] >> 2) & 3) - 1;
              if (ys < 0 && zs < 0) continue;
              V v = tile[t + i * NT];
              if (ys >= 0) v = phase_mul(phase_of(p.P, 1, ys), v);
              if (zs >= 0) v = phase_mul(phase_of(p.P, 2, zs), v);
              tile[t + i * NT] = v;
            }
          }
        }
        __syncthreads();
        issue(pl + S - 1);

        // Own values and axis-1 neighbours: one column of VY + 2R cells.
        const V* colp = tile + (ty * VY) * SZ + R + tz;
        V own[VY];
        if (pl >= x0 && pl < x1) {
          V col[VY + 2 * R];
#pragma unroll
          for (int m = 0; m < VY + 2 * R; m++) col[m] = colp[m * SZ];
#pragma unroll
          for (int j = 0; j < VY; j++) {
            own[j] = col[R + j];
            const V* row = colp + (R + j) * SZ;
            Sc cc = p.c0;
            if constexpr (POT) cc += vtiles[st * BY * BZ + ty * VY * BZ + tz + j * BZ];
            V sy = vmul(cc, col[R + j]);
            V sz = vzero<V>();
#pragma unroll
            for (int k = 1; k <= R; k++) {
              madd(sy, p.cy[kMaxR - k], col[R + j - k]);
              madd(sz, p.cz[kMaxR - k], row[-k]);
              madd(sy, p.cy[kMaxR + k], col[R + j + k]);
              madd(sz, p.cz[kMaxR + k], row[k]);
            }
            acc[j][u] = vadd(acc[j][u], vadd(sy, sz));  // slot of output pl
          }
        } else {
#pragma unroll
          for (int j = 0; j < VY; j++) own[j] = colp[(R + j) * SZ];
        }

        int xside;
        const int xs = wrap_plane(pl, p.n0, p.per0, xside);
        if (xs >= 0) {
          if constexpr (vt<V>::NC == 2) {
            if (xside >= 0) {
#pragma unroll
              for (int j = 0; j < VY; j++) own[j] = phase_mul(phase_of(p.P, 0, xside), own[j]);
            }
          }
#pragma unroll
          for (int j = 0; j < VY; j++) {
#pragma unroll
            for (int k = 1; k <= R; k++) {
              madd(acc[j][(u - k + Q) % Q], p.cx[kMaxR + k], own[j]);  // output pl-k: offset +k
              madd(acc[j][(u + k) % Q], p.cx[kMaxR - k], own[j]);      // output pl+k: offset -k
            }
          }
        }

        const int q = pl - R;
        const int qs = (u - R + Q) % Q;  // slot of output pl - R
        if (q >= x0 && q < x1) {
          const V* rt = rtiles + st * RCELLS + ty * VY * BZ + tz;
          char* dstp = out_c + size_t(q) * plane_b;
#pragma unroll
          for (int j = 0; j < VY; j++) {
            V* dst = reinterpret_cast<V*>(dstp + own_b[j]);
            if constexpr (MODE == MODE_APPLY || MODE == MODE_POTENTIAL) {
              if (own_in[j]) stcs(dst, acc[j][qs]);
            } else if constexpr (MODE == MODE_JACOBI) {
              if (own_in[j]) stcs(dst, vmul(p.wc, vsub(rt[j * BZ], acc[j][qs])));
            } else {
              const V r = vsub(acc[j][qs], rt[j * BZ]);
              if (own_in[j]) {
                stcs(dst, r);
                if constexpr (vt<V>::NC == 1) sumsq += sq(r);
              }
            }
          }
        }
#pragma unroll
        for (int j = 0; j < VY; j++) acc[j][qs] = vzero<V>();
      }
    }
  }
  cp_async_wait<0>();

  if constexpr (MODE == MODE_RESIDUAL) {
    if (p.partials) {
      const double sblk = block_sum<NT>(sumsq, red);
      if (t == 0) {
        const long long cta = (long long)blockIdx.z * gridDim.y * gridDim.x +
                              (long long)blockIdx.y * gridDim.x + blockIdx.x;
        p.partials[cta] = sblk;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Direct star stencil: one thread per point, neighbours read through the L1
// cache.  For small grids (the coarse multigrid levels) the marching kernel
// is latency-bound -- each plane step waits for a memory round trip -- while
// this kernel finishes in about one round trip.  Same modes and arithmetic
// as star_kernel (folded Jacobi centre weight included).  Grid-stride over
// nin * n0 * n1 * n2 points with a fixed grid, so the per-CTA partial sums
// of MODE_RESIDUAL have a fixed order.
// ---------------------------------------------------------------------------
// One output point of the direct star stencil at (i0, i1, i2) of a band:
// base / rho_b point to the band, rem = (i0 n1 + i1) n2 + i2.  Every mode;
// LD is the load policy (common.cuh).
template <class V, int R, int MODE, class LD>
__device__ __forceinline__ V star_point_at(const V* __restrict__ base, const V* __restrict__ rho_b,
                                           const StarParams<typename vt<V>::S>& p, int i0, int i1,
                                           int i2, long long rem) {
  using Sc = typename vt<V>::S;
  const long long plane = (long long)p.n1 * p.n2;
  const int r1 = int(rem - i0 * plane);
  Sc cc = p.c0;
  if constexpr (MODE == MODE_POTENTIAL) cc += LD::ld(static_cast<const Sc*>(p.pot) + rem);
  V s = vmul(cc, LD::ld(base + rem));
#pragma unroll
  for (int k = -R; k <= R; k++) {
    if (k == 0) continue;
    int sd;
    int j = wrap_axis(i0 + k, p.n0, p.per0, sd);
    if (j >= 0) {
      V v = LD::ld(base + j * plane + r1);
      if constexpr (vt<V>::NC == 2) { if (sd >= 0) v = phase_mul(phase_of(p.P, 0, sd), v); }
      madd(s, p.cx[kMaxR + k], v);
    }
    j = wrap_axis(i1 + k, p.n1, p.per1, sd);
    if (j >= 0) {
      V v = LD::ld(base + i0 * plane + j * p.n2 + i2);
      if constexpr (vt<V>::NC == 2) { if (sd >= 0) v = phase_mul(phase_of(p.P, 1, sd), v); }
      madd(s, p.cy[kMaxR + k], v);
    }
    j = wrap_axis(i2 + k, p.n2, p.per2, sd);
    if (j >= 0) {
      V v = LD::ld(base + i0 * plane + i1 * p.n2 + j);
      if constexpr (vt<V>::NC == 2) { if (sd >= 0) v = phase_mul(phase_of(p.P, 2, sd), v); }
      madd(s, p.cz[kMaxR + k], v);
    }
  }
  if constexpr (MODE == MODE_JACOBI) return vmul(p.wc, vsub(LD::ld(rho_b + rem), s));
  else if constexpr (MODE == MODE_RESIDUAL) return vsub(s, LD::ld(rho_b + rem));
  else return s;
}

// The same at flat index g over all bands.
template <class V, int R, int MODE, class LD>
__device__ __forceinline__ V star_point(const V* __restrict__ in, const V* __restrict__ rho,
                                        const StarParams<typename vt<V>::S>& p, long long g) {
  const long long plane = (long long)p.n1 * p.n2;
  const long long b = g / p.band;
  const long long rem = g - b * p.band;
  const int i0 = int(rem / plane);
  const int r1 = int(rem - i0 * plane);
  const int i1 = r1 / p.n2, i2 = r1 - i1 * p.n2;
  return star_point_at<V, R, MODE, LD>(in + b * p.band, rho ? rho + b * p.band : nullptr, p, i0,
                                       i1, i2, rem);
}

template <class V, int R, int MODE>
__global__ void __launch_bounds__(256)
star_direct_kernel(const V* __restrict__ in, V* __restrict__ out, const V* __restrict__ rho,
                   const StarParams<typename vt<V>::S> p, long long total) {
  pdl_enter();
  __shared__ double red[8];
  double sumsq = 0.0;
  for (long long g = blockIdx.x * 256LL + threadIdx.x; g < total; g += (long long)gridDim.x * 256) {
    const V o = star_point<V, R, MODE, LoadRO>(in, rho, p, g);
    out[g] = o;
    if constexpr (MODE == MODE_RESIDUAL && vt<V>::NC == 1) sumsq += sq(o);
  }
  if constexpr (MODE == MODE_RESIDUAL) {
    if (p.partials) {
      const double sblk = block_sum<256>(sumsq, red);
      if (threadIdx.x == 0) p.partials[blockIdx.x] = sblk;
    }
  }
}

// ---------------------------------------------------------------------------
// General stencil: any offsets within +-MP on every axis.
// ---------------------------------------------------------------------------
template <class S>
struct GenParams {
  int n0, n1, n2;
  int per0, per1, per2;
  int x_chunk, nxc;
  long long band;
  int ncoefs;
  S coefs[kMaxCoefs];
  signed char off[kMaxCoefs][3];
  S w;
  S sign;           // MODE_JACOBI: +1, or -1 for the negated sweep (exact)
  Phases<S> P;
  double* partials;
};

template <class V, int BZ, int TY, int VY, int MODE>
__global__ void __launch_bounds__(BZ * TY)
general_kernel(const V* __restrict__ in, V* __restrict__ out, const V* __restrict__ rho,
               const GenParams<typename vt<V>::S> p, int mp) {
  pdl_enter();
  using S = typename vt<V>::S;
  constexpr int NT = BZ * TY, BY = TY * VY;
  const int SY = BY + 2 * mp, SZ = BZ + 2 * mp, NR = 2 * mp + 1;
  const int CELLS = SY * SZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* ring = reinterpret_cast<V*>(smem_raw);
  __shared__ double red[NT / 32];

  const int t = threadIdx.x, tz = t % BZ, ty = t / BZ;
  const int z0 = blockIdx.x * BZ, y0 = blockIdx.y * BY;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int x0 = xc * p.x_chunk, x1 = min(p.n0, x0 + p.x_chunk);
  const long long plane = (long long)p.n1 * p.n2;
  const V* inb = in + bnd * p.band;
  V* outb = out + bnd * p.band;
  const V* rhob = rho ? rho + bnd * p.band : nullptr;
  double sumsq = 0.0;

  for (int pl = x0 - mp; pl < x1 + mp; ++pl) {
    V* slot = ring + ((pl - (x0 - mp)) % NR) * CELLS;
    int xside;
    int xs = wrap_plane(pl, p.n0, p.per0, xside);
    for (int c = t; c < CELLS; c += NT) {
      int sy = c / SZ, sz = c % SZ;
      int ysd, zsd;
      int ys = wrap_axis(y0 - mp + sy, p.n1, p.per1, ysd);
      int zs = wrap_axis(z0 - mp + sz, p.n2, p.per2, zsd);
      V v = vzero<V>();
      if (xs >= 0 && ys >= 0 && zs >= 0) {
        v = ldro(inb + xs * plane + ys * p.n2 + zs);
        if constexpr (vt<V>::NC == 2) {
          if (xside >= 0) v = phase_mul(phase_of(p.P, 0, xside), v);
          if (ysd >= 0) v = phase_mul(phase_of(p.P, 1, ysd), v);
          if (zsd >= 0) v = phase_mul(phase_of(p.P, 2, zsd), v);
        }
      }
      slot[c] = v;
    }
    __syncthreads();
    const int q = pl - mp;
    if (q >= x0) {
      for (int j = 0; j < VY; j++) {
        const int y = y0 + ty + j * TY, z = z0 + tz;
        if (y >= p.n1 || z >= p.n2) continue;
        V s = vzero<V>();
        for (int c = 0; c < p.ncoefs; c++) {
          if (MODE == MODE_JACOBI && c == 0) continue;
          const int dx = p.off[c][0], dy = p.off[c][1], dz = p.off[c][2];
          const V* sl = ring + ((q + dx - (x0 - mp)) % NR) * CELLS;
          madd(s, p.coefs[c], sl[(mp + ty + j * TY + dy) * SZ + (mp + tz + dz)]);
        }
        V* dst = outb + q * plane + (long long)y * p.n2 + z;
        if constexpr (MODE == MODE_APPLY) {
          *dst = s;
        } else {
          V src = ldro(rhob + q * plane + (long long)y * p.n2 + z);
          if constexpr (MODE == MODE_JACOBI) {
            // coefs[0] is the diagonal (c/bmgs/relax.c:46-71)
            const V* sl = ring + ((q - (x0 - mp)) % NR) * CELLS;
            V ctr = sl[(mp + ty + j * TY) * SZ + (mp + tz)];
            if constexpr (vt<V>::NC == 1) {
              *dst = p.sign * ((S(1) - p.w) * ctr + p.w * (src - s) / p.coefs[0]);
            } else {
              const V d = vsub(src, s);
              *dst = {p.sign * ((S(1) - p.w) * ctr.re + p.w * d.re / p.coefs[0]),
                      p.sign * ((S(1) - p.w) * ctr.im + p.w * d.im / p.coefs[0])};
            }
          } else {
            V r = vsub(s, src);
            *dst = r;
            if constexpr (vt<V>::NC == 1) sumsq += sq(r);
          }
        }
      }
    }
    __syncthreads();
  }
  if constexpr (MODE == MODE_RESIDUAL) {
    if (p.partials) {
      double s = block_sum<NT>(sumsq, red);
      if (t == 0) {
        long long cta = (long long)blockIdx.z * gridDim.y * gridDim.x +
                        (long long)blockIdx.y * gridDim.x + blockIdx.x;
        p.partials[cta] = s;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// One colour of multicolour Gauss-Seidel for "L phi = rho" (real only):
// phi[g] = (rho[g] - sum_{p >= 1} c_p phi[g + o_p]) / c_0 for the
// points with (i0 + i1 + i2) mod ncolor == color.  Neighbours inside the
// domain are read from phi (current values); wrapped neighbours on periodic
// axes are read from `frozen`, a copy taken at the start of the sweep, as
// the reference's halo is filled once per sweep (c/operators.c:66-78).
// ---------------------------------------------------------------------------
// The update of point (i0, i1, i2).  phi and frozen may be the same array
// (no periodic axis).
template <class V>
__device__ __forceinline__ void gs_point_at(V* phi, const V* __restrict__ rho, const V* frozen,
                                            const GenParams<typename vt<V>::S>& p, int i0, int i1,
                                            int i2) {
  using S = typename vt<V>::S;
  S s = 0;
  for (int c = 1; c < p.ncoefs; c++) {
    int sd0, sd1, sd2;
    int j0 = wrap_axis(i0 + p.off[c][0], p.n0, p.per0, sd0);
    int j1 = wrap_axis(i1 + p.off[c][1], p.n1, p.per1, sd1);
    int j2 = wrap_axis(i2 + p.off[c][2], p.n2, p.per2, sd2);
    if (j0 < 0 || j1 < 0 || j2 < 0) continue;
    long long gg = ((long long)j0 * p.n1 + j1) * p.n2 + j2;
    bool wrapped = (sd0 >= 0) || (sd1 >= 0) || (sd2 >= 0);
    S v = wrapped ? frozen[gg] : phi[gg];
    s += v * p.coefs[c];
  }
  const long long g = ((long long)i0 * p.n1 + i1) * p.n2 + i2;
  phi[g] = (rho[g] - s) * (S(1) / p.coefs[0]);
}

// Points of one colour, enumerated without idle threads: index q covers
// the rows (i0, i1) times gs_row_slots() slots; slot j of a row is
// i2 = first + ncolor j, first = (color - i0 - i1) mod ncolor.  False for
// slots past the row's end.  32-bit index arithmetic (a grid holds fewer
// than 2^31 points).
__host__ __device__ inline int gs_row_slots(int n2, int ncolor) {
  return (n2 + ncolor - 1) / ncolor;
}
__device__ __forceinline__ bool gs_colour_point(int q, int slots, int ncolor, int color, int n1,
                                                int n2, int& i0, int& i1, int& i2) {
  const int row = q / slots, j = q - row * slots;
  i0 = row / n1;
  i1 = row - i0 * n1;
  int first = (color - i0 - i1) % ncolor;
  if (first < 0) first += ncolor;
  i2 = first + ncolor * j;
  return i2 < n2;
}

template <class V>
__global__ void __launch_bounds__(256)
color_gs_kernel(V* phi, const V* __restrict__ rho, const V* frozen,
                const GenParams<typename vt<V>::S> p, int ncolor, int color) {
  pdl_enter();
  const int slots = gs_row_slots(p.n2, ncolor);
  const int nq = p.n0 * p.n1 * slots;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    int i0, i1, i2;
    if (gs_colour_point(q, slots, ncolor, color, p.n1, p.n2, i0, i1, i2))
      gs_point_at<V>(phi, rho, frozen, p, i0, i1, i2);
  }
}

}  // namespace gfd
