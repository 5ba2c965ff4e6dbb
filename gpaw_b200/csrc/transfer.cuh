// transfer.cuh -- multigrid restriction and interpolation for sm_100a.
//
// The reference (c/bmgs/restrict.c, c/bmgs/interpolate.c, driven by
// c/transformers.c:54-123) fills a halo-padded copy of each band and then
// runs three transposing 1-D passes (axis 2, axis 1, axis 0) through scratch
// buffers: about four reads and four writes of the array.  Here one kernel
// does all three passes:
//   * a CTA owns a tile of output points in (axis 1, axis 2) and marches
//     along axis 0;
//   * each input plane (with its halo, mapped in-kernel: zero, periodic, or
//     periodic times the Bloch phase) is staged in shared memory, the axis-2
//     pass and then the axis-1 pass run there (the reference's pass order,
//     so the arithmetic matches term by term);
//   * the axis-0 pass reads a per-thread register queue of the last planes'
//     2-D results.
// HBM traffic is one read of the input and one write of the output.
//
// Weights: Lagrange weights for K = 2*nn taps (c/bmgs/restrict.c:37-57,
// c/bmgs/interpolate.c:46-59).
#pragma once

#include "common.cuh"
#include "internal.h"

namespace gfd {

template <int NN, class S> __device__ __forceinline__ S lagw(int m);
template <int NN, class S>
__device__ __forceinline__ S lagw(int m) {
  if (NN == 1) return S(0.5);
  if (NN == 2) return m == 0 ? S(0.5625) : S(-0.0625);
  if (NN == 3) return m == 0 ? S(0.58593750) : (m == 1 ? S(-0.09765625) : S(0.01171875));
  return m == 0 ? S(0.59814453125)
                : (m == 1 ? S(-0.11962890625) : (m == 2 ? S(0.02392578125) : S(-0.00244140625)));
}

// Restriction tap around a[0] with stride st (in elements of V):
// 0.5 * (a0 + w1 (a[+1] + a[-1]) + w2 (a[+3] + a[-3]) + ...)
template <int NN, class V, class Get>
__device__ __forceinline__ V rst_tap(Get get) {
  using S = typename vt<V>::S;
  V x = get(0);
#pragma unroll
  for (int k = 0; k < NN; k++) x = vadd(x, vmul(lagw<NN, S>(k), vadd(get(2 * k + 1), get(-(2 * k + 1)))));
  return vmul(S(0.5), x);
}

// Interpolated value between a[0] and a[1]:
// w0 (a[0] + a[1]) + w1 (a[-1] + a[2]) + ...
template <int NN, class V, class Get>
__device__ __forceinline__ V ip_tap(Get get) {
  using S = typename vt<V>::S;
  V x = vmul(lagw<NN, S>(0), vadd(get(0), get(1)));
#pragma unroll
  for (int m = 1; m < NN; m++) x = vadd(x, vmul(lagw<NN, S>(m), vadd(get(-m), get(1 + m))));
  return x;
}

template <class S>
struct TrParams {
  int ni0, ni1, ni2;   // input points per axis
  int no0, no1, no2;   // output points per axis
  int lo0, lo1, lo2;   // low-side padding of the input (pad[c][0])
  int sk0, sk1, sk2;   // interpolation: skip[c][0]
  int per0, per1, per2;
  int x_chunk, nxc;    // output planes per CTA along axis 0, chunk count
  long long band_in, band_out;
  Phases<S> P;
  // Restriction only: when seed != nullptr, also write seed = seed_scale *
  // out (same layout as out).  A weighted-Jacobi sweep from a zero guess
  // gives exactly (w / c0) rho, so a multigrid level's first sweep comes
  // out of the restriction that produces its rho.
  void* seed;
  S seed_scale;
  // Factor on the transferred value (1, or -1 for the negated transfers of
  // the band preconditioner; multiplying by -1 is exact).
  S out_scale;
};

// Transfer parameters of a transformer (host side).
template <class S>
void tr_params(const gfd_transformer* tr, const double* ph, void* seed, double seed_scale,
               double out_scale, TrParams<S>& p) {
  p = TrParams<S>{};
  p.ni0 = tr->nin[0]; p.ni1 = tr->nin[1]; p.ni2 = tr->nin[2];
  p.no0 = tr->nout[0]; p.no1 = tr->nout[1]; p.no2 = tr->nout[2];
  p.lo0 = tr->pad[0][0]; p.lo1 = tr->pad[1][0]; p.lo2 = tr->pad[2][0];
  p.sk0 = tr->skip[0][0]; p.sk1 = tr->skip[1][0]; p.sk2 = tr->skip[2][0];
  p.per0 = tr->per[0]; p.per1 = tr->per[1]; p.per2 = tr->per[2];
  p.band_in = (long long)tr->nin[0] * tr->nin[1] * tr->nin[2];
  p.band_out = (long long)tr->nout[0] * tr->nout[1] * tr->nout[2];
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 2; d++) {
      p.P.ph[c][d].re = ph ? S(ph[4 * c + 2 * d]) : S(1);
      p.P.ph[c][d].im = ph ? S(ph[4 * c + 2 * d + 1]) : S(0);
    }
  p.seed = seed;
  p.seed_scale = S(seed_scale);
  p.out_scale = S(out_scale);
}

// Pack an in-plane source offset and its wrap sides; -1 = zero point.
__device__ __forceinline__ int pack_src(int ys, int zs, int n2, int ysd, int zsd) {
  if (ys < 0 || zs < 0) return -1;
  return ((ys * n2 + zs) << 4) | ((ysd + 1) | ((zsd + 1) << 2));
}

template <class V, class S>
__device__ __forceinline__ V apply_phases(V v, int code, int xside, const Phases<S>& P) {
  if constexpr (vt<V>::NC == 2) {
    if (xside >= 0) v = phase_mul(phase_of(P, 0, xside), v);
    int ys = (code & 3) - 1, zs = ((code >> 2) & 3) - 1;
    if (ys >= 0) v = phase_mul(phase_of(P, 1, ys), v);
    if (zs >= 0) v = phase_mul(phase_of(P, 2, zs), v);
  }
  return v;
}

// Staged fine rows of the restriction kernel (RZ cells) are stored with
// their even positions first and their odd ones from HALF on.  HALF sits
// half a 128-byte segment past a segment start (E / 2 elements mod E), so
// the even and odd runs that one shared-memory wavefront writes land in
// different banks.
template <class V, int RZ>
constexpr int rst_half() {
  constexpr int E = 128 / int(sizeof(V));
  int h = (RZ + 1) / 2;
  while (h % E != E / 2) ++h;
  return h;
}
template <class V, int RZ>
constexpr int rst_pitch() {
  return rst_half<V, RZ>() + RZ / 2;
}

// Types up to 8 bytes: each thread restricts two neighbouring coarse
// columns at once, and a staged fine row is kept in four phases (position
// mod 4), phase q at q * QS + position / 4.  The 2nn + 1 taps of the pair
// (even positions) and its two centres (odd ones) are then consecutive
// words across lanes: 2nn + 3 loads per pair instead of 2 (2nn + 1).  QS is
// E / 4 past a 128-byte segment start (E / 4 elements mod E), so the four
// phase runs one wavefront writes use each bank at most twice.
template <class V, int RZ>
constexpr int rst_quad() {
  constexpr int E = 128 / int(sizeof(V));
  int q = (RZ + 3) / 4;
  while (q % E != E / 4) ++q;
  return q;
}
template <class V>
constexpr bool rst_pairs() {
  return sizeof(V) <= 8;
}
// Shared-memory row pitch of a staged fine row (elements).
template <class V, int RZ>
constexpr int rst_row_pitch() {
  if constexpr (rst_pairs<V>()) return 4 * rst_quad<V, RZ>();
  else return rst_pitch<V, RZ>();
}

template <class V>
struct alignas(2 * sizeof(V)) VPair {
  V a, b;
};

// ---------------------------------------------------------------------------
// Restriction: coarse index i on an axis takes the fine padded point
// (K-1) + 2i (c/bmgs/restrict.c:65-69), i.e. fine array index
// 2i + (2nn-1) - lo.
// ---------------------------------------------------------------------------
template <class V, int NN, int BZC, int TYC, int VYC>
__global__ void __launch_bounds__(BZC * TYC)
restrict_kernel(const V* __restrict__ in, V* __restrict__ out,
                const TrParams<typename vt<V>::S> p) {
  pdl_enter();
  using S = typename vt<V>::S;
  constexpr int NT = BZC * TYC, BYC = TYC * VYC;
  constexpr int W = 2 * NN - 1;           // wing of one restriction tap
  constexpr int RY = 2 * BYC - 1 + 2 * W;
  constexpr int RZ = 2 * BZC - 1 + 2 * W;
  constexpr int CELLS = RY * RZ;
  constexpr int CC = (CELLS + NT - 1) / NT;
  constexpr int QL = 2 * W + 1;           // fine planes feeding one coarse plane
  // Each staged fine row holds its even positions first, then its odd ones:
  // the axis-2 taps of neighbouring coarse points are then consecutive
  // words (a stride-2 read would hit every bank twice).
  constexpr bool PAIRS = rst_pairs<V>();
  constexpr int HALF = rst_half<V, RZ>(), QS = rst_quad<V, RZ>();
  constexpr int RZP = rst_row_pitch<V, RZ>(), STG = RY * RZP;
  static_assert(!PAIRS || BZC % 2 == 0, "coarse columns come in pairs");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* F = reinterpret_cast<V*>(smem_raw);          // [2][RY][RZP], rows in phases
  V* T = F + 2 * STG;                             // [2][RY][BZC]

  const int t = threadIdx.x, tz = t % BZC, ty = t / BZC;
  const int Z0 = blockIdx.x * BZC, Y0 = blockIdx.y * BYC;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int X0 = xc * p.x_chunk, X1 = min(p.no0, X0 + p.x_chunk);
  const long long plane_in = (long long)p.ni1 * p.ni2;
  const long long plane_out = (long long)p.no1 * p.no2;
  const V* inb = in + bnd * p.band_in;
  V* outb = out + bnd * p.band_out;
  const int fy0 = 2 * Y0 - p.lo1, fz0 = 2 * Z0 - p.lo2;

  int src[CC];
  int dpos[CC];  // stage position of cell t + i * NT
#pragma unroll
  for (int i = 0; i < CC; i++) {
    int c = t + i * NT;
    src[i] = -1;
    dpos[i] = 0;
    if (c < CELLS) {
      int sy = c / RZ, sz = c % RZ;
      if constexpr (PAIRS) dpos[i] = sy * RZP + (sz & 3) * QS + (sz >> 2);
      else dpos[i] = sy * RZP + ((sz & 1) ? HALF + (sz >> 1) : (sz >> 1));
      int ysd, zsd;
      int ys = wrap_axis(fy0 + sy, p.ni1, p.per1, ysd);
      int zs = wrap_axis(fz0 + sz, p.ni2, p.per2, zsd);
      src[i] = pack_src(ys, zs, p.ni2, ysd, zsd);
    }
  }

  const int fbeg = 2 * X0 + W - p.lo0 - W;
  const int fend = 2 * (X1 - 1) + W - p.lo0 + W + 1;

  V rv[CC];
  auto load = [&](int f) {
    int xside;
    int xs = (f < fend) ? wrap_axis(f, p.ni0, p.per0, xside) : -1;
#pragma unroll
    for (int i = 0; i < CC; i++) {
      V v = vzero<V>();
      if (xs >= 0 && src[i] >= 0) {
        v = ldro(inb + xs * plane_in + (src[i] >> 4));
        v = apply_phases<V, S>(v, src[i] & 15, xside, p.P);
      }
      rv[i] = v;
    }
  };

  V q[VYC][QL];
#pragma unroll
  for (int j = 0; j < VYC; j++)
#pragma unroll
    for (int k = 0; k < QL; k++) q[j][k] = vzero<V>();

  load(fbeg);
  for (int f = fbeg; f < fend; ++f) {
    V* Fb = F + (f & 1) * STG;
    V* Tb = T + (f & 1) * RY * BZC;
#pragma unroll
    for (int i = 0; i < CC; i++)
      if (t + i * NT < CELLS) Fb[dpos[i]] = rv[i];
    load(f + 1);
    __syncthreads();
    if constexpr (PAIRS) {
      // axis-2 pass, columns cz = 2m and 2m + 1 of every staged row: their
      // taps are fine positions 4m + 2j (j = 0 .. 2nn; j = 0 .. 2nn - 1 for
      // cz = 2m, 1 .. 2nn for 2m + 1), their centres 4m + W and 4m + W + 2.
      for (int c = t; c < RY * (BZC / 2); c += NT) {
        const int sy = c / (BZC / 2), m = c % (BZC / 2);
        const V* row = Fb + sy * RZP + m;
        V tap[2 * NN + 1];
#pragma unroll
        for (int j = 0; j <= 2 * NN; j++) tap[j] = row[((2 * j) & 3) * QS + (j >> 1)];
        const V c0 = row[(W & 3) * QS + (W >> 2)];
        const V c1 = row[((W + 2) & 3) * QS + ((W + 2) >> 2)];
        VPair<V> r;
        r.a = rst_tap<NN, V>([&](int o) { return o == 0 ? c0 : tap[(o + W) >> 1]; });
        r.b = rst_tap<NN, V>([&](int o) { return o == 0 ? c1 : tap[((o + W) >> 1) + 1]; });
        *reinterpret_cast<VPair<V>*>(Tb + sy * BZC + 2 * m) = r;
      }
    } else {
      // axis-2 pass: Tb[sy][cz] for every staged row; fine position
      // 2 cz + W + o sits at (W + o) & 1 ? HALF : 0, + cz + (W + o) / 2.
      for (int c = t; c < RY * BZC; c += NT) {
        const int sy = c / BZC, cz = c % BZC;
        const V* row = Fb + sy * RZP + cz;
        Tb[c] = rst_tap<NN, V>([&](int o) { return row[((W + o) & 1 ? HALF : 0) + ((W + o) >> 1)]; });
      }
    }
    __syncthreads();
    // axis-1 pass for this thread's coarse points, pushed into the queue
#pragma unroll
    for (int j = 0; j < VYC; j++) {
      const V* col = Tb + (2 * (ty + j * TYC) + W) * BZC + tz;
      V v = rst_tap<NN, V>([&](int o) { return col[o * BZC]; });
#pragma unroll
      for (int k = 0; k + 1 < QL; k++) q[j][k] = q[j][k + 1];
      q[j][QL - 1] = v;
    }
    // axis-0 pass: the queue centre is fine plane f - W
    const int fc = f - W;
    const int rel = fc - W + p.lo0;
    if (f - fbeg >= QL - 1 && (rel & 1) == 0) {
      const int X = rel >> 1;
      if (X >= X0 && X < X1) {
#pragma unroll
        for (int j = 0; j < VYC; j++) {
          const int y = Y0 + ty + j * TYC, z = Z0 + tz;
          if (y < p.no1 && z < p.no2) {
            V v = rst_tap<NN, V>([&](int o) { return q[j][W + o]; });
            if (p.out_scale != S(1)) v = vmul(p.out_scale, v);
            const long long o = X * plane_out + (long long)y * p.no2 + z;
            stcs(outb + o, v);
            if (p.seed) stcs(static_cast<V*>(p.seed) + (outb - out) + o, vmul(p.seed_scale, v));
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Interpolation: fine index f on an axis has g = f + skip[c][0]; g = 2i is a
// copy of coarse padded point (nn-1) + i, g = 2i + 1 the K-tap value between
// (nn-1) + i and (nn-1) + i + 1 (c/bmgs/interpolate.c:19-66).  Coarse array
// index of step i: c(i) = i + nn - 1 - lo.
// ---------------------------------------------------------------------------
// SUB: out = base - interpolated value (the multigrid correction
// phi -= interpolate(e), in place when base == out).
template <class V, int NN, int BZF, int TYF, int VYF, bool SUB>
__global__ void __launch_bounds__(BZF * TYF)
interp_kernel(const V* __restrict__ in, V* out, const V* base,
              const TrParams<typename vt<V>::S> p) {
  pdl_enter();
  using S = typename vt<V>::S;
  constexpr int NT = BZF * TYF, BYF = TYF * VYF;
  constexpr int CY = BYF / 2 + 2 * NN, CZ = BZF / 2 + 2 * NN;
  constexpr int CELLS = CY * CZ;
  constexpr int CC = (CELLS + NT - 1) / NT;
  constexpr int QL = 2 * NN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* C = reinterpret_cast<V*>(smem_raw);  // [2][CY][CZ]
  V* T = C + 2 * CELLS;                   // [2][CY][BZF]

  const int t = threadIdx.x, tz = t % BZF, ty = t / BZF;
  const int Z0 = blockIdx.x * BZF, Y0 = blockIdx.y * BYF;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int X0 = xc * p.x_chunk, X1 = min(p.no0, X0 + p.x_chunk);
  const long long plane_in = (long long)p.ni1 * p.ni2;
  const long long plane_out = (long long)p.no1 * p.no2;
  const V* inb = in + bnd * p.band_in;
  V* outb = out + bnd * p.band_out;
  const V* baseb = SUB ? base + bnd * p.band_out : nullptr;
  const int iy0 = (Y0 + p.sk1) >> 1, iz0 = (Z0 + p.sk2) >> 1;
  const int cy0 = iy0 - p.lo1, cz0 = iz0 - p.lo2;  // coarse origin of the tile

  int src[CC];
#pragma unroll
  for (int i = 0; i < CC; i++) {
    int c = t + i * NT;
    src[i] = -1;
    if (c < CELLS) {
      int sy = c / CZ, sz = c % CZ;
      int ysd, zsd;
      int ys = wrap_axis(cy0 + sy, p.ni1, p.per1, ysd);
      int zs = wrap_axis(cz0 + sz, p.ni2, p.per2, zsd);
      src[i] = pack_src(ys, zs, p.ni2, ysd, zsd);
    }
  }

  const int ia = (X0 + p.sk0) >> 1, ib = (X1 - 1 + p.sk0) >> 1;
  const int cbeg = ia - p.lo0;                    // c(ia) - (nn-1)
  const int cend = ib + NN - 1 - p.lo0 + NN + 1;  // one past c(ib) + nn

  V rv[CC];
  auto load = [&](int c) {
    int xside;
    int xs = (c < cend) ? wrap_axis(c, p.ni0, p.per0, xside) : -1;
#pragma unroll
    for (int i = 0; i < CC; i++) {
      V v = vzero<V>();
      if (xs >= 0 && src[i] >= 0) {
        v = ldro(inb + xs * plane_in + (src[i] >> 4));
        v = apply_phases<V, S>(v, src[i] & 15, xside, p.P);
      }
      rv[i] = v;
    }
  };

  V q[VYF][QL];
#pragma unroll
  for (int j = 0; j < VYF; j++)
#pragma unroll
    for (int k = 0; k < QL; k++) q[j][k] = vzero<V>();

  // One barrier per coarse plane: plane c + 1 is staged (into the other
  // buffer) while plane c's axis-2 results are being written, and both C
  // and T are double-buffered, so every read of a buffer is separated from
  // the next write into it by a barrier.
  load(cbeg);
#pragma unroll
  for (int i = 0; i < CC; i++)
    if (t + i * NT < CELLS) C[(cbeg & 1) * CELLS + t + i * NT] = rv[i];
  load(cbeg + 1);
  __syncthreads();
  for (int c = cbeg; c < cend; ++c) {
    const V* Cb = C + (c & 1) * CELLS;
    V* Tb = T + (c & 1) * CY * BZF;
    // axis-2 pass: every staged coarse row to this tile's fine columns, two
    // adjacent fine columns per thread (one even, one odd, whatever the
    // skip), so every lane does one copy and one K-tap value.
    static_assert(BZF % 2 == 0, "fine columns come in pairs");
    for (int e = t; e < CY * (BZF / 2); e += NT) {
      const int sy = e / (BZF / 2), fz = 2 * (e % (BZF / 2));
      const int g = Z0 + fz + p.sk2;
      const int odd0 = g & 1;  // the same for every pair of the tile
      const int ge = g + odd0, go = g + 1 - odd0;  // the pair's even and odd g
      const V* rowe = Cb + sy * CZ + ((ge >> 1) - iz0 + NN - 1);
      const V* rowo = Cb + sy * CZ + ((go >> 1) - iz0 + NN - 1);
      V* out = Tb + sy * BZF + fz;
      out[odd0] = rowe[0];
      out[1 - odd0] = ip_tap<NN, V>([&](int o) { return rowo[o]; });
    }
    if (c + 1 < cend) {
      V* Cn = C + ((c + 1) & 1) * CELLS;
#pragma unroll
      for (int i = 0; i < CC; i++)
        if (t + i * NT < CELLS) Cn[t + i * NT] = rv[i];
      load(c + 2);
    }
    __syncthreads();
    // axis-1 pass for this thread's fine points
#pragma unroll
    for (int j = 0; j < VYF; j++) {
      const int g = Y0 + ty + j * TYF + p.sk1;
      const int cl = (g >> 1) - iy0 + NN - 1;
      const V* col = Tb + cl * BZF + tz;
      V v = (g & 1) ? ip_tap<NN, V>([&](int o) { return col[o * BZF]; }) : col[0];
#pragma unroll
      for (int k = 0; k + 1 < QL; k++) q[j][k] = q[j][k + 1];
      q[j][QL - 1] = v;
    }
    // axis-0 pass: step i with c(i) + nn == c emits fine g = 2i and 2i + 1
    const int i = c - 2 * NN + 1 + p.lo0;
    if (c - cbeg >= QL - 1 && i >= ia && i <= ib) {
#pragma unroll
      for (int par = 0; par < 2; par++) {
        const int X = 2 * i + par - p.sk0;
        if (X < X0 || X >= X1) continue;
#pragma unroll
        for (int j = 0; j < VYF; j++) {
          const int y = Y0 + ty + j * TYF, z = Z0 + tz;
          if (y < p.no1 && z < p.no2) {
            V v = par ? ip_tap<NN, V>([&](int o) { return q[j][NN - 1 + o]; }) : q[j][NN - 1];
            const long long o = X * plane_out + (long long)y * p.no2 + z;
            if (p.out_scale != S(1)) v = vmul(p.out_scale, v);
            if constexpr (SUB) v = vsub(baseb[o], v);
            stcs(outb + o, v);
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Direct forms for small grids (coarse multigrid levels): one thread per
// output point, the three 1-D passes nested in registers in the reference's
// order (axis 2 innermost, then axis 1, then axis 0), neighbours read through
// the L1 cache.  The marching kernels above pay a memory round trip per plane,
// which dominates on grids of a few thousand points.
// ---------------------------------------------------------------------------
template <class LD, class V, class S>
__device__ __forceinline__ V tr_fetch(const V* base, int x, int y, int z, const TrParams<S>& p) {
  int sx, sy, sz;
  const int i = wrap_axis(x, p.ni0, p.per0, sx);
  const int j = wrap_axis(y, p.ni1, p.per1, sy);
  const int k = wrap_axis(z, p.ni2, p.per2, sz);
  if (i < 0 || j < 0 || k < 0) return vzero<V>();
  V v = LD::ld(base + ((long long)i * p.ni1 + j) * p.ni2 + k);
  if constexpr (vt<V>::NC == 2) {
    if (sx >= 0) v = phase_mul(phase_of(p.P, 0, sx), v);
    if (sy >= 0) v = phase_mul(phase_of(p.P, 1, sy), v);
    if (sz >= 0) v = phase_mul(phase_of(p.P, 2, sz), v);
  }
  return v;
}

// One restricted point at output coordinates (X, Y, Z) of a band (base:
// the band's input), times out_scale; LD is the load policy (common.cuh).
template <class V, int NN, class LD>
__device__ __forceinline__ V restrict_point_at(const V* __restrict__ base, int X, int Y, int Z,
                                               const TrParams<typename vt<V>::S>& p) {
  constexpr int W = 2 * NN - 1;
  // fine centre of each axis: 2i + (2nn-1) - lo
  const int fx = 2 * X + W - p.lo0, fy = 2 * Y + W - p.lo1, fz = 2 * Z + W - p.lo2;
  V v = rst_tap<NN, V>([&](int ox) {
    return rst_tap<NN, V>([&](int oy) {
      return rst_tap<NN, V>([&](int oz) { return tr_fetch<LD>(base, fx + ox, fy + oy, fz + oz, p); });
    });
  });
  if (p.out_scale != typename vt<V>::S(1)) v = vmul(p.out_scale, v);
  return v;
}

// The same at flat index g over all output bands.
template <class V, int NN, class LD>
__device__ __forceinline__ V restrict_point(const V* __restrict__ in,
                                            const TrParams<typename vt<V>::S>& p, long long g) {
  const long long plane_out = (long long)p.no1 * p.no2;
  const long long b = g / p.band_out;
  const long long rem = g - b * p.band_out;
  const int X = int(rem / plane_out);
  const int r1 = int(rem - X * plane_out);
  const int Y = r1 / p.no2, Z = r1 - Y * p.no2;
  return restrict_point_at<V, NN, LD>(in + b * p.band_in, X, Y, Z, p);
}

// One interpolated point at output coordinates (X, Y, Z), times out_scale
// (SUB: *bo, the base value at that point, minus it).
template <class V, int NN, bool SUB, class LD>
__device__ __forceinline__ V interp_point_at(const V* __restrict__ base, const V* bo, int X, int Y,
                                             int Z, const TrParams<typename vt<V>::S>& p) {
  // g = f + skip[c][0]; even g: coarse point c(i) = i + nn - 1 - lo, odd: between c(i), c(i)+1
  const int gx = X + p.sk0, gy = Y + p.sk1, gz = Z + p.sk2;
  const int cx = (gx >> 1) + NN - 1 - p.lo0, cy = (gy >> 1) + NN - 1 - p.lo1,
            cz = (gz >> 1) + NN - 1 - p.lo2;
  auto along = [&](int odd, auto get) -> V { return odd ? ip_tap<NN, V>(get) : get(0); };
  V v = along(gx & 1, [&](int ox) {
    return along(gy & 1, [&](int oy) {
      return along(gz & 1, [&](int oz) { return tr_fetch<LD>(base, cx + ox, cy + oy, cz + oz, p); });
    });
  });
  if (p.out_scale != typename vt<V>::S(1)) v = vmul(p.out_scale, v);
  // bo may be the output itself (in-place correction): a plain load.
  if constexpr (SUB) v = vsub(*bo, v);
  return v;
}

// The same at flat index g over all output bands.
template <class V, int NN, bool SUB, class LD>
__device__ __forceinline__ V interp_point(const V* __restrict__ in, const V* base_out,
                                          const TrParams<typename vt<V>::S>& p, long long g) {
  const long long plane_out = (long long)p.no1 * p.no2;
  const long long b = g / p.band_out;
  const long long rem = g - b * p.band_out;
  const int X = int(rem / plane_out);
  const int r1 = int(rem - X * plane_out);
  const int Y = r1 / p.no2, Z = r1 - Y * p.no2;
  return interp_point_at<V, NN, SUB, LD>(in + b * p.band_in, SUB ? base_out + g : nullptr, X, Y,
                                         Z, p);
}

template <class V, int NN>
__global__ void __launch_bounds__(256)
restrict_direct_kernel(const V* __restrict__ in, V* __restrict__ out,
                       const TrParams<typename vt<V>::S> p, long long total) {
  pdl_enter();
  for (long long g = blockIdx.x * 256LL + threadIdx.x; g < total; g += (long long)gridDim.x * 256) {
    const V v = restrict_point<V, NN, LoadRO>(in, p, g);
    out[g] = v;
    if (p.seed) static_cast<V*>(p.seed)[g] = vmul(p.seed_scale, v);
  }
}

template <class V, int NN, bool SUB>
__global__ void __launch_bounds__(256)
interp_direct_kernel(const V* __restrict__ in, V* out, const V* base_out,
                     const TrParams<typename vt<V>::S> p, long long total) {
  pdl_enter();
  for (long long g = blockIdx.x * 256LL + threadIdx.x; g < total; g += (long long)gridDim.x * 256)
    out[g] = interp_point<V, NN, SUB, LoadRO>(in, base_out, p, g);
}

}  // namespace gfd
