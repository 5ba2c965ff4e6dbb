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

enum { MODE_APPLY = 0, MODE_JACOBI = 1, MODE_RESIDUAL = 2 };

template <class S>
struct StarParams {
  int n0, n1, n2;
  int per0, per1, per2;
  int x_chunk;      // outputs along axis 0 per CTA
  int nxc;          // number of axis-0 chunks
  long long band;   // elements per band
  S c0;             // centre weight
  S cx[2 * kMaxR + 1];  // weight of offset k along axis 0 at index kMaxR + k
  S cy[2 * kMaxR + 1];
  S cz[2 * kMaxR + 1];
  S w;              // Jacobi weight
  Phases<S> P;
  double* partials; // MODE_RESIDUAL: one sum of r^2 per CTA (or nullptr)
};

template <class V>
__device__ __forceinline__ V load_mapped(const V* base, int off) {
  return off >= 0 ? ldro(base + off) : vzero<V>();
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

template <class V, int R, int BZ, int TY, int VY, int D, int MODE>
__global__ void __launch_bounds__(BZ * TY)
star_kernel(const V* __restrict__ in, V* __restrict__ out, const V* __restrict__ rho,
            const StarParams<typename vt<V>::S> p) {
  using S = typename vt<V>::S;
  constexpr int NT = BZ * TY;
  constexpr int BY = TY * VY;
  constexpr int SY = BY + 2 * R;
  constexpr int SZ = BZ + 2 * R;
  constexpr int HN = 2 * R * BZ + 2 * R * BY;  // halo cells of one plane
  constexpr int HC = (HN + NT - 1) / NT;       // halo cells per thread
  constexpr int Q = 2 * R + 1;

  __shared__ V tile[2][SY][SZ];
  __shared__ double red[NT / 32];

  const int t = threadIdx.x;
  const int tz = t % BZ, ty = t / BZ;
  const int z0 = blockIdx.x * BZ, y0 = blockIdx.y * BY;
  const int bnd = blockIdx.z / p.nxc, xc = blockIdx.z % p.nxc;
  const int x0 = xc * p.x_chunk;
  const int x1 = min(p.n0, x0 + p.x_chunk);
  const long long plane = (long long)p.n1 * p.n2;
  const V* inb = in + bnd * p.band;
  V* outb = out + bnd * p.band;
  const V* rhob = rho ? rho + bnd * p.band : nullptr;

  // Own points: rows y0 + ty + j*TY, column z0 + tz.  The in-plane source
  // offset is -1 for a zero boundary point; out-of-domain points of partial
  // tiles still need a (wrapped or zero) value in shared memory.
  int own_src[VY];
  int own_code[VY];  // wrap sides (y in bits 0-1, z in bits 2-3), 0xF = none
  bool own_in[VY];
  {
    int sz_side;
    int zs = wrap_axis(z0 + tz, p.n2, p.per2, sz_side);
#pragma unroll
    for (int j = 0; j < VY; j++) {
      int y = y0 + ty + j * TY;
      int sy_side;
      int ys = wrap_axis(y, p.n1, p.per1, sy_side);
      own_in[j] = (y < p.n1) && (z0 + tz < p.n2);
      own_src[j] = (ys >= 0 && zs >= 0) ? ys * p.n2 + zs : -1;
      own_code[j] = (sy_side + 1) | ((sz_side + 1) << 2);
    }
  }
  // Halo cells of this thread: y-halo rows first, then z-halo columns.
  int h_smem[HC];
  int h_src[HC];
  int h_code[HC];
#pragma unroll
  for (int i = 0; i < HC; i++) {
    int h = t + i * NT;
    h_smem[i] = -1;
    h_src[i] = -1;
    h_code[i] = 0;
    if (h < HN) {
      int sy, sz;
      if (h < 2 * R * BZ) {
        int r = h / BZ, c = h % BZ;
        sy = r < R ? r : BY + r;
        sz = R + c;
      } else {
        int hh = h - 2 * R * BZ;
        int r = hh / (2 * R), c = hh % (2 * R);
        sy = R + r;
        sz = c < R ? c : BZ + c;
      }
      int ysd, zsd;
      int ys = wrap_axis(y0 - R + sy, p.n1, p.per1, ysd);
      int zs = wrap_axis(z0 - R + sz, p.n2, p.per2, zsd);
      h_smem[i] = sy * SZ + sz;
      h_src[i] = (ys >= 0 && zs >= 0) ? ys * p.n2 + zs : -1;
      h_code[i] = (ysd + 1) | ((zsd + 1) << 2);
    }
  }

  auto with_phase = [&](V v, int code) -> V {
    if constexpr (vt<V>::NC == 2) {
      int ys = (code & 3) - 1, zs = ((code >> 2) & 3) - 1;
      if (ys >= 0) v = phase_mul(phase_of(p.P, 1, ys), v);
      if (zs >= 0) v = phase_mul(phase_of(p.P, 2, zs), v);
    }
    return v;
  };

  // Prefetch ring: own values and halo values of the next D planes.
  V rc[D][VY];
  V rh[D][HC];
  const int pbeg = x0 - R, pend = x1 + R;

  auto load_plane = [&](int pl, V (&cv)[VY], V (&hv)[HC]) {
    int xside;
    int xs = wrap_axis(pl, p.n0, p.per0, xside);
    if (xs < 0 || pl < pbeg || pl >= pend) {
#pragma unroll
      for (int j = 0; j < VY; j++) cv[j] = vzero<V>();
#pragma unroll
      for (int i = 0; i < HC; i++) hv[i] = vzero<V>();
      return;
    }
    const V* base = inb + xs * plane;
#pragma unroll
    for (int j = 0; j < VY; j++) cv[j] = load_mapped(base, own_src[j]);
    const bool need_halo = (pl >= x0 && pl < x1);
#pragma unroll
    for (int i = 0; i < HC; i++) hv[i] = need_halo ? load_mapped(base, h_src[i]) : vzero<V>();
  };

#pragma unroll
  for (int d = 0; d < D; d++) load_plane(pbeg + d, rc[d], rh[d]);

  V acc[VY][Q];
#pragma unroll
  for (int j = 0; j < VY; j++)
#pragma unroll
    for (int q = 0; q < Q; q++) acc[j][q] = vzero<V>();

  // Centre values of the last R+1 planes (Jacobi epilogue) and the next
  // output's source term.
  V hist[VY][R + 1];
  V rcur[VY];
#pragma unroll
  for (int j = 0; j < VY; j++) {
#pragma unroll
    for (int q = 0; q <= R; q++) hist[j][q] = vzero<V>();
    rcur[j] = vzero<V>();
  }
  double sumsq = 0.0;

  for (int pl = pbeg; pl < pend; ++pl) {
    V cv[VY], hv[HC];
#pragma unroll
    for (int j = 0; j < VY; j++) cv[j] = rc[0][j];
#pragma unroll
    for (int i = 0; i < HC; i++) hv[i] = rh[0][i];
#pragma unroll
    for (int d = 0; d + 1 < D; d++) {
#pragma unroll
      for (int j = 0; j < VY; j++) rc[d][j] = rc[d + 1][j];
#pragma unroll
      for (int i = 0; i < HC; i++) rh[d][i] = rh[d + 1][i];
    }
    load_plane(pl + D, rc[D - 1], rh[D - 1]);

    // Source term for output pl - R + 1 (used next step).
    V rnext[VY];
    if constexpr (MODE != MODE_APPLY) {
      const int qn = pl - R + 1;
#pragma unroll
      for (int j = 0; j < VY; j++)
        rnext[j] = (qn >= x0 && qn < x1 && own_in[j])
                       ? ldro(rhob + qn * plane + own_src[j])
                       : vzero<V>();
    }

    if (pl >= x0 && pl < x1) {
      V(*buf)[SZ] = tile[pl & 1];
#pragma unroll
      for (int j = 0; j < VY; j++) buf[R + ty + j * TY][R + tz] = with_phase(cv[j], own_code[j]);
#pragma unroll
      for (int i = 0; i < HC; i++)
        if (h_smem[i] >= 0) (&buf[0][0])[h_smem[i]] = with_phase(hv[i], h_code[i]);
      __syncthreads();
#pragma unroll
      for (int j = 0; j < VY; j++) {
        const int yy = R + ty + j * TY, zz = R + tz;
        V s = (MODE == MODE_JACOBI) ? vzero<V>() : vmul(p.c0, cv[j]);
#pragma unroll
        for (int k = 1; k <= R; k++) {
          madd(s, p.cy[kMaxR - k], buf[yy - k][zz]);
          madd(s, p.cy[kMaxR + k], buf[yy + k][zz]);
        }
#pragma unroll
        for (int k = 1; k <= R; k++) {
          madd(s, p.cz[kMaxR - k], buf[yy][zz - k]);
          madd(s, p.cz[kMaxR + k], buf[yy][zz + k]);
        }
        acc[j][R] = vadd(acc[j][R], s);
      }
    }

    // Contributions of this plane's own values along axis 0.
    {
      int xside;
      int xs = wrap_axis(pl, p.n0, p.per0, xside);
      if (xs >= 0) {
#pragma unroll
        for (int j = 0; j < VY; j++) {
          V v = cv[j];
          if constexpr (vt<V>::NC == 2) {
            if (xside >= 0) v = phase_mul(phase_of(p.P, 0, xside), v);
          }
#pragma unroll
          for (int k = 1; k <= R; k++) {
            madd(acc[j][R - k], p.cx[kMaxR + k], v);
            madd(acc[j][R + k], p.cx[kMaxR - k], v);
          }
        }
      }
    }

    if constexpr (MODE == MODE_JACOBI) {
#pragma unroll
      for (int j = 0; j < VY; j++) {
#pragma unroll
        for (int q = 0; q < R; q++) hist[j][q] = hist[j][q + 1];
        hist[j][R] = cv[j];
      }
    }

    const int q = pl - R;
    if (q >= x0 && q < x1) {
#pragma unroll
      for (int j = 0; j < VY; j++) {
        if (!own_in[j]) continue;
        V* dst = outb + q * plane + own_src[j];
        if constexpr (MODE == MODE_APPLY) {
          stcs(dst, acc[j][0]);
        } else if constexpr (MODE == MODE_JACOBI) {
          // b = (1 - w) b + w (src - x) / coefs[0]   (c/bmgs/relax.c:64)
          static_assert(vt<V>::NC == 1, "relaxation is real only");
          stcs(dst, (S(1) - p.w) * hist[j][0] + p.w * (rcur[j] - acc[j][0]) / p.c0);
        } else {
          V r = vsub(acc[j][0], rcur[j]);
          stcs(dst, r);
          if constexpr (vt<V>::NC == 1) sumsq += sq(r);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < VY; j++) {
#pragma unroll
      for (int qq = 0; qq + 1 < Q; qq++) acc[j][qq] = acc[j][qq + 1];
      acc[j][Q - 1] = vzero<V>();
      if constexpr (MODE != MODE_APPLY) rcur[j] = rnext[j];
    }
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
  Phases<S> P;
  double* partials;
};

template <class V, int BZ, int TY, int VY, int MODE>
__global__ void __launch_bounds__(BZ * TY)
general_kernel(const V* __restrict__ in, V* __restrict__ out, const V* __restrict__ rho,
               const GenParams<typename vt<V>::S> p, int mp) {
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
    int xs = wrap_axis(pl, p.n0, p.per0, xside);
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
            static_assert(vt<V>::NC == 1, "relaxation is real only");
            const V* sl = ring + ((q - (x0 - mp)) % NR) * CELLS;
            V ctr = sl[(mp + ty + j * TY) * SZ + (mp + tz)];
            *dst = (S(1) - p.w) * ctr + p.w * (src - s) / p.coefs[0];
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
template <class V>
__global__ void __launch_bounds__(256)
color_gs_kernel(V* __restrict__ phi, const V* __restrict__ rho, const V* __restrict__ frozen,
                const GenParams<typename vt<V>::S> p, int ncolor, int color) {
  using S = typename vt<V>::S;
  const long long n = (long long)p.n0 * p.n1 * p.n2;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    int i2 = int(g % p.n2);
    long long r = g / p.n2;
    int i1 = int(r % p.n1);
    int i0 = int(r / p.n1);
    if ((i0 + i1 + i2) % ncolor != color) continue;
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
    phi[g] = (rho[g] - s) * (S(1) / p.coefs[0]);
  }
}

}  // namespace gfd
