// stencil_split.cuh -- axis-aligned ("star") stencils on complex bands with
// the real and imaginary parts on neighbouring lanes.
//
// Same computation as star_kernel (c/bmgs/fd.c:16-51 over the Bloch-phased
// halo of c/bc.c:138-250; Jacobi and residual modes of c/bmgs/relax.c), for
// complex128 / complex64 and radius R <= 3.  What changes is where the
// shared-memory bytes go.  star_kernel reads every in-plane neighbour of a
// complex point as one 16-byte load (10 per point at R = 3): with the
// partial-sum ring in registers it is bound by the shared-memory data path,
// not by HBM.  Here:
//
//  * The stencil weights are real, so the real and imaginary parts of a band
//    are two independent real stencils once the halo carries its phases.
//    Lane 2k + c of a warp computes component c (0 re, 1 im) of columns 2k
//    and 2k + 1, for VY consecutive rows.  A thread's 2 x VY block reuses
//    every in-plane value it loads along both axes: 1 + 2R (1/2 + 1/VY)
//    loads per point and component, 5.5 at R = 3 and VY = 4, of 8 (4) bytes.
//  * Staged rows are split by column parity: even columns first, then odd
//    ones.  Lane pair k reads column 2k + v of one parity at half-index
//    k + floor(v / 2), so a warp's load of component c is 32 consecutive
//    scalars -- conflict-free.  The 16-byte cp.async that stages one complex
//    value puts it straight into its half, so the split costs nothing.  The
//    copies take the L1-allocating form (see cp_async in stencil.cuh).
//  * Axis 0 is marched as in star_kernel: 2R + 1 partial sums per point in
//    registers, the plane loop unrolled by 2R + 1.  Bloch phases of all
//    three axes are applied where a copied cell lands (the copying thread,
//    after its copy is complete, before the CTA barrier), so the arithmetic
//    loop holds no phase logic: a plane outside [0, n0) is only ever an
//    axis-0 neighbour, and the whole staged plane takes the axis-0 phase.
//  * The lane pair swaps halves before the store (one shuffle per row), so
//    each lane writes one whole complex value and a warp writes 32
//    consecutive values.
#pragma once

#include "stencil.cuh"

namespace gfd {

constexpr int kSplitMaxR = 3;

// Rows per lane and the CTAs per SM the register budget is sized for
// (build-time knobs for measuring other shapes; the defaults are the ones
// the launch code is written for).
#ifndef GFD_SPLIT_VY
#define GFD_SPLIT_VY 4
#endif
#ifndef GFD_SPLIT_MINB
#define GFD_SPLIT_MINB 3
#endif

template <int R>
struct SplitShape {
  static constexpr int BZ = 32;              // columns of a tile
  static constexpr int RE = (R + 1) & ~1;    // R rounded up to even
  static constexpr int HW = BZ / 2 + RE;     // values per parity half-row
  static constexpr int RS = 2 * HW;          // values per staged row
};

template <class V, int R, int VY, int WY, int S, int MODE>
constexpr size_t split_smem_bytes() {
  using Sc = typename vt<V>::S;
  constexpr int BY = VY * WY, BZ = 32;
  constexpr bool RHO = MODE == MODE_JACOBI || MODE == MODE_RESIDUAL;
  constexpr bool POT = MODE == MODE_POTENTIAL;
  return size_t(S) * ((BY + 2 * R) * SplitShape<R>::RS * sizeof(V) +
                      (RHO ? BY * BZ * sizeof(V) : 0) + (POT ? BY * BZ * sizeof(Sc) : 0));
}

// 128 threads (WY = 4 warps of 2 x 4 points per lane) at three CTAs per SM:
// at most 168 registers per thread.
template <class V, int R, int VY, int WY, int S, int MODE>
__global__ void __launch_bounds__(32 * WY, GFD_SPLIT_MINB)
star_split_kernel(const V* __restrict__ in, V* __restrict__ out, const V* __restrict__ rho,
                  const StarParams<typename vt<V>::S> p) {
  pdl_enter();
  using Sc = typename vt<V>::S;
  static_assert(vt<V>::NC == 2, "complex values only");
  using Shp = SplitShape<R>;
  constexpr int BZ = Shp::BZ, RE = Shp::RE, HW = Shp::HW, RS = Shp::RS;
  constexpr int NT = 32 * WY, BY = VY * WY, SY = BY + 2 * R;
  constexpr int OWN = BY * BZ;                    // a plane's own cells
  constexpr int HALO = BY * 2 * R + 2 * R * BZ;   // side columns, then halo rows
  constexpr int CELLS = OWN + HALO;
  constexpr int CPT = (CELLS + NT - 1) / NT;
  constexpr int OWN_CPT = OWN / NT;
  static_assert(OWN % NT == 0, "own cells split evenly over the threads");
  constexpr int Q = 2 * R + 1;
  constexpr int STAGE = SY * RS;                  // values per staged plane
  constexpr bool RHO = MODE == MODE_JACOBI || MODE == MODE_RESIDUAL;
  constexpr bool POT = MODE == MODE_POTENTIAL;
  static_assert(S >= 2, "pipeline needs two stages");
  static_assert(R >= 1 && R <= kSplitMaxR, "radius");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* tiles = reinterpret_cast<V*>(smem_raw);            // [S][SY][2][HW]
  V* rtiles = tiles + S * STAGE;                        // [S][BY][2][16]: rho by parity
  Sc* vtiles = reinterpret_cast<Sc*>(rtiles + (RHO ? S * OWN : 0));  // [S][BY][32]

  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int k = lane >> 1, c = lane & 1;
  const int z0 = blockIdx.x * BZ, y0 = blockIdx.y * BY;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int x0 = xc * p.x_chunk;
  const int x1 = min(p.n0, x0 + p.x_chunk);
  const long long plane = (long long)p.n1 * p.n2;
  const size_t plane_b = size_t(plane) * sizeof(V);
  const char* inb_c = reinterpret_cast<const char*>(in + bnd * p.band);
  char* outb_c = reinterpret_cast<char*>(out + bnd * p.band);
  const char* rho_c = RHO ? reinterpret_cast<const char*>(rho + bnd * p.band) : nullptr;
  const char* pot_c = reinterpret_cast<const char*>(p.pot);
  const int pbeg = x0 - R, pend = x1 + R;

  // Cells this thread copies: source byte offset within a plane, destination
  // byte offset within a stage, zero / live flags and the Bloch wrap sides
  // (y side bits 0-1, z side bits 2-3 of a 4-bit code per cell).
  unsigned csrc[CPT], cdst[CPT];
  unsigned czero = 0, clive = 0, ccode = 0;
  bool fix_yz = false;
#pragma unroll
  for (int i = 0; i < CPT; i++) {
    const int cell = t + i * NT;
    csrc[i] = 0;
    cdst[i] = 0;
    if (cell < CELLS) {
      clive |= 1u << i;
      int sy, lc;  // staged row, column relative to z0
      if (cell < OWN) {
        sy = R + cell / BZ;
        lc = cell % BZ;
      } else if (cell < OWN + BY * 2 * R) {
        const int h = cell - OWN;
        sy = R + h / (2 * R);
        const int s = h % (2 * R);
        lc = s < R ? s - R : BZ + (s - R);
      } else {
        const int h = cell - OWN - BY * 2 * R;
        const int r = h / BZ;
        sy = r < R ? r : BY + r;
        lc = h % BZ;
      }
      const int u = lc + RE;
      cdst[i] = unsigned((sy * RS + (u & 1) * HW + (u >> 1)) * sizeof(V));
      int ysd, zsd;
      const int ys = wrap_axis(y0 - R + sy, p.n1, p.per1, ysd);
      const int zs = wrap_axis(z0 + lc, p.n2, p.per2, zsd);
      if (ys >= 0 && zs >= 0) {
        csrc[i] = unsigned(ys * p.n2 + zs) * unsigned(sizeof(V));
        if (ysd >= 0 || zsd >= 0) fix_yz = true;
      } else {
        czero |= 1u << i;
      }
      ccode |= unsigned((ysd + 1) | ((zsd + 1) << 2)) << (4 * i);
    }
  }
  fix_yz = fix_yz && p.fix_yz;

  // This lane's points: rows y0 + w VY + j, columns z0 + 2k + v.
  const int yb = y0 + w * VY;
  const int zc = z0 + 2 * k;
  bool ok[VY][2];
  unsigned own_b[VY];  // byte offset of column zc, row j within a plane
#pragma unroll
  for (int j = 0; j < VY; j++) {
    const int y = yb + j;
    own_b[j] = unsigned((y < p.n1 ? y : 0) * p.n2 + (zc < p.n2 ? zc : 0)) * unsigned(sizeof(V));
    ok[j][0] = y < p.n1 && zc < p.n2;
    ok[j][1] = y < p.n1 && zc + 1 < p.n2;
  }
  const unsigned smem0 = smem_addr(tiles);
  const unsigned rsmem0 = smem_addr(rtiles);
  const unsigned vsmem0 = smem_addr(vtiles);

  // Copy plane P into stage (P - pbeg) % S: all cells when P is an output
  // plane of this CTA, only the own cells otherwise (an axis-0 neighbour),
  // plus the source term of output plane P - R or the potential of plane P.
  // Always commits one group.
  auto issue = [&](int P) {
    if (P < pend) {
      const int st = (P - pbeg) % S;
      const unsigned sbase = smem0 + unsigned(st * STAGE * sizeof(V));
      int xside;
      const int xs = wrap_plane(P, p.n0, p.per0, xside);
      const char* src = inb_c + size_t(xs >= 0 ? xs : 0) * plane_b;
      const unsigned zmask = xs >= 0 ? czero : ~0u;
      const bool full = P >= x0 && P < x1;
#pragma unroll
      for (int i = 0; i < CPT; i++) {
        if (!(clive >> i & 1u)) continue;
        if (i >= OWN_CPT && !full) continue;
        const unsigned n = (zmask >> i & 1u) ? 0u : unsigned(sizeof(V));
        if constexpr (sizeof(V) == 16)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sbase + cdst[i]),
                       "l"(src + csrc[i]), "r"(n)
                       : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sbase + cdst[i]),
                       "l"(src + csrc[i]), "r"(n)
                       : "memory");
      }
      if constexpr (RHO) {
        // rho of output plane P - R, split by column parity like the tiles:
        // thread t copies the own cells t + i NT (row cell / 32, column
        // cell % 32) to [row][column parity][column / 2].
        const int q = P - R;
        if (q >= x0 && q < x1) {
          const unsigned rbase = rsmem0 + unsigned(st * OWN * sizeof(V));
          const char* rsrc = rho_c + size_t(q) * plane_b;
#pragma unroll
          for (int i = 0; i < OWN_CPT; i++) {
            const int cell = t + i * NT;
            const int r = cell / BZ, lc = cell % BZ;
            const int y = y0 + r, z = z0 + lc;
            const bool in_dom = y < p.n1 && z < p.n2;
            const unsigned d =
                rbase + unsigned((r * BZ + (lc & 1) * (BZ / 2) + (lc >> 1)) * sizeof(V));
            const char* s = rsrc + (in_dom ? size_t(y * p.n2 + z) * sizeof(V) : 0);
            const unsigned n = in_dom ? unsigned(sizeof(V)) : 0u;
            if constexpr (sizeof(V) == 16)
              asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(s),
                           "r"(n)
                           : "memory");
            else
              asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(s),
                           "r"(n)
                           : "memory");
          }
        }
      }
      if constexpr (POT) {
        // The potential of this plane's own points, natural layout
        // [row][column], one copy per value (zero-filled off the domain).
        if (full) {
          const unsigned vbase = vsmem0 + unsigned(st * OWN * sizeof(Sc));
          const char* vsrc = pot_c + size_t(P) * size_t(plane) * sizeof(Sc);
          constexpr int PAIRS = OWN / 2, PPT = (PAIRS + NT - 1) / NT;
#pragma unroll
          for (int i = 0; i < PPT; i++) {
            const int pr = t + i * NT;
            if (pr < PAIRS) {
              const int r = pr / (BZ / 2), lc = 2 * (pr % (BZ / 2));
              const int y = y0 + r, z = z0 + lc;
              const unsigned d = vbase + unsigned((r * BZ + lc) * sizeof(Sc));
#pragma unroll
              for (int e = 0; e < 2; e++) {
                const bool in_dom = y < p.n1 && z + e < p.n2;
                const char* s = vsrc + (in_dom ? size_t(y * p.n2 + z + e) * sizeof(Sc) : 0);
                const unsigned n = in_dom ? unsigned(sizeof(Sc)) : 0u;
                asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(
                                 d + unsigned(e * sizeof(Sc))),
                             "l"(s), "n"(int(sizeof(Sc))), "r"(n)
                             : "memory");
              }
            }
          }
        }
      }
    }
    cp_async_commit();
  };

#pragma unroll
  for (int i = 0; i < S - 1; i++) issue(pbeg + i);

  Sc acc[VY][2][Q];
#pragma unroll
  for (int j = 0; j < VY; j++)
#pragma unroll
    for (int v = 0; v < 2; v++)
#pragma unroll
      for (int q = 0; q < Q; q++) acc[j][v][q] = Sc(0);

  // Scalar view of the staged planes; lane base: row R + w VY, lane pair k,
  // component c.  Column 2k + v of staged row sy is at
  // sy RS + ((v + RE) & 1) HW + k + ((v + RE) >> 1) values from the stage.
  const Sc* tiles_s = reinterpret_cast<const Sc*>(tiles);
  const int lane_s = ((R + w * VY) * RS + k) * 2 + c;
  auto col_off = [](int v) { return (((v + RE) & 1) * HW + ((v + RE) >> 1)) * 2; };

  for (int base = pbeg; base < pend; base += Q) {
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      const int pl = base + u;
      if (pl < pend) {
        const int st = (pl - pbeg) % S;
        cp_async_wait<S - 2>();
        int xside;
        const int xs = wrap_plane(pl, p.n0, p.per0, xside);
        const bool out_plane = pl >= x0 && pl < x1;
        {
          // Bloch phases where this thread's copies landed: the axis-0 phase
          // on a plane from across the axis-0 boundary, the axis-1/2 phases on
          // wrapped halo cells of an output plane.
          const bool fx = xside >= 0 && (p.P.ph[0][xside].re != Sc(1) ||
                                          p.P.ph[0][xside].im != Sc(0));
          if (fx || (fix_yz && out_plane)) {
            V* tile = tiles + st * STAGE;
#pragma unroll
            for (int i = 0; i < CPT; i++) {
              if (!(clive >> i & 1u) || (czero >> i & 1u)) continue;
              if (i >= OWN_CPT && !out_plane) continue;
              const unsigned code = ccode >> (4 * i) & 15u;
              const int ys = int(code & 3u) - 1, zs = int(code >> 2) - 1;
              if (!fx && ys < 0 && zs < 0) continue;
              V* cellp = reinterpret_cast<V*>(reinterpret_cast<char*>(tile) + cdst[i]);
              V v = *cellp;
              if (fx) v = phase_mul(phase_of(p.P, 0, xside), v);
              if (ys >= 0) v = phase_mul(phase_of(p.P, 1, ys), v);
              if (zs >= 0) v = phase_mul(phase_of(p.P, 2, zs), v);
              *cellp = v;
            }
          }
        }
        __syncthreads();
        issue(pl + S - 1);

        const Sc* T = tiles_s + st * STAGE * 2 + lane_s;
        Sc own[VY][2];
        if (out_plane) {
          // In-plane terms of output plane pl.
          Sc up[R][2], dn[R][2];
#pragma unroll
          for (int m = 1; m <= R; m++)
#pragma unroll
            for (int v = 0; v < 2; v++) {
              up[m - 1][v] = T[-m * RS * 2 + col_off(v)];
              dn[m - 1][v] = T[(VY - 1 + m) * RS * 2 + col_off(v)];
            }
          Sc ctr[VY][2];
          Sc pv[VY][2];
#pragma unroll
          for (int j = 0; j < VY; j++) {
            Sc row[2 + 2 * R];
#pragma unroll
            for (int v = -R; v <= 1 + R; v++) row[v + R] = T[j * RS * 2 + col_off(v)];
            ctr[j][0] = row[R];
            ctr[j][1] = row[R + 1];
            if constexpr (POT) {
              const Sc* vt = reinterpret_cast<const Sc*>(vtiles) + st * OWN +
                             (w * VY + j) * BZ + 2 * k;
              if constexpr (sizeof(Sc) == 8) {
                const double2 pp = *reinterpret_cast<const double2*>(vt);
                pv[j][0] = pp.x;
                pv[j][1] = pp.y;
              } else {
                const float2 pp = *reinterpret_cast<const float2*>(vt);
                pv[j][0] = pp.x;
                pv[j][1] = pp.y;
              }
            }
#pragma unroll
            for (int v = 0; v < 2; v++) {
              Sc cc = p.c0;
              if constexpr (POT) cc += pv[j][v];
              Sc s = cc * row[R + v];
#pragma unroll
              for (int m = 1; m <= R; m++) {
                s = fma(p.cz[kMaxR - m], row[R + v - m], s);
                s = fma(p.cz[kMaxR + m], row[R + v + m], s);
              }
              acc[j][v][u] += s;
            }
          }
#pragma unroll
          for (int j = 0; j < VY; j++)
#pragma unroll
            for (int v = 0; v < 2; v++) {
              Sc s = Sc(0);
#pragma unroll
              for (int m = 1; m <= R; m++) {
                const Sc a = j - m >= 0 ? ctr[j - m][v] : up[m - j - 1][v];
                const Sc b = j + m < VY ? ctr[j + m][v] : dn[j + m - VY][v];
                s = fma(p.cy[kMaxR - m], a, s);
                s = fma(p.cy[kMaxR + m], b, s);
              }
              acc[j][v][u] += s;
              own[j][v] = ctr[j][v];
            }
        } else {
#pragma unroll
          for (int j = 0; j < VY; j++)
#pragma unroll
            for (int v = 0; v < 2; v++) own[j][v] = T[j * RS * 2 + col_off(v)];
        }

        // Axis 0: plane pl's own values into the sums of outputs pl-R..pl+R
        // (a zero plane past a zero boundary adds nothing).
        if (xs >= 0) {
#pragma unroll
          for (int j = 0; j < VY; j++)
#pragma unroll
            for (int v = 0; v < 2; v++)
#pragma unroll
              for (int m = 1; m <= R; m++) {
                acc[j][v][(u - m + Q) % Q] = fma(p.cx[kMaxR + m], own[j][v], acc[j][v][(u - m + Q) % Q]);
                acc[j][v][(u + m) % Q] = fma(p.cx[kMaxR - m], own[j][v], acc[j][v][(u + m) % Q]);
              }
        }

        // Output plane pl - R is complete.
        const int q = pl - R;
        const int qs = (u - R + Q) % Q;
        if (q >= x0 && q < x1) {
          char* dstp = outb_c + size_t(q) * plane_b;
#pragma unroll
          for (int j = 0; j < VY; j++) {
            Sc r0 = acc[j][0][qs], r1 = acc[j][1][qs];
            if constexpr (RHO) {
              const Sc* rt = reinterpret_cast<const Sc*>(rtiles + st * OWN) +
                             ((w * VY + j) * BZ + k) * 2 + c;
              const Sc s0 = rt[0], s1 = rt[BZ];  // columns 2k (even half), 2k + 1 (odd half)
              if constexpr (MODE == MODE_JACOBI) {
                r0 = p.wc * (s0 - r0);
                r1 = p.wc * (s1 - r1);
              } else {
                r0 = r0 - s0;
                r1 = r1 - s1;
              }
            }
            // Lane c = 0 holds the real parts of columns 2k, 2k+1, lane 1 the
            // imaginary parts: swap so lane 0 writes column 2k, lane 1 2k+1.
            const Sc give = c ? r0 : r1;
            const Sc got = __shfl_xor_sync(0xffffffffu, give, 1);
            V o;
            o.re = c ? got : r0;
            o.im = c ? r1 : got;
            if (ok[j][c]) {
              V* dst = reinterpret_cast<V*>(dstp + own_b[j]) + c;
              stcs(dst, o);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < VY; j++) {
          acc[j][0][qs] = Sc(0);
          acc[j][1][qs] = Sc(0);
        }
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace gfd
