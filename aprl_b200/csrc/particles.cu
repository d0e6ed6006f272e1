// particles.cu -- per-particle kernels of the conservative-source step:
// the wide-shape weights, the orbit-averaged electric gather and the F3 x-z
// (or trilinear) magnetic gather, the Lapenta-Markidis push with prescribed
// lab magnets, charge-conserving deposition, particle-boundary events with
// CPML current carriers, the fixed-point residual, and stable compaction.
//
// One thread owns one particle; its gathers and weights run in the
// reference's visit order, so in FP64 (no FMA contraction) the per-particle
// arithmetic matches the reference, except that the quintic shape's four
// Gauss points of a cut piece are summed per node before the gather's read
// and the deposit's atomic.  Deposition accumulates with atomics into J; the
// summation order of J differs from the reference.
//
// The walkers are templated on the type F of J and of the weight
// arithmetic.  Positions, chord cuts and cell indices are always binary64,
// and so are the E and B arrays; the weights are evaluated in F from the
// cell-relative offsets, the field values are rounded to F as they are read
// and accumulated in F, and J is accumulated in F.  F = double is the FP64
// drop-in, F = float the FP32-mixed mode.
#include "common.cuh"
#include "particles.cuh"

namespace aprl_gpu {

// ---------------------------------------------------------------------------
// shapes (src/longitudinal_shape.h:15-117, src/transverse_source_shape.h:8-10)
template <class F>
__device__ __forceinline__ void node_weights(F f, F w[4]) {
  w[0] = F(0.25) * (F(1.) - f);
  w[1] = F(0.5) - F(0.25) * f;
  w[2] = F(0.25) + F(0.25) * f;
  w[3] = F(0.25) * f;
}

// binomialXZSegment (src/longitudinal_shape.h:61-94).
template <class G, class V>
__device__ __forceinline__ void binomial_xz_segment(const GridT<G>& g, const double s[3],
                                                    const double d[3], double first,
                                                    double last, V& visit) {
  using F = typename V::Weight;
  const F width = F(last - first);
  const double mid = (first + last) * 0.5;
  const double x = s[0] + mid * d[0], y = s[1] + mid * d[1], z = s[2] + mid * d[2];
  long long i = (long long)floor(x), j = (long long)floor(y);
  const long long k = (long long)floor(z);
  if (i == (long long)g.nx) --i;
  if (j == (long long)g.ny) --j;
  F wx[4], wz[4];
  node_weights(F(x - i), wx);
  node_weights(F(z - k), wz);
  const F wy[2] = {F(1.) - F(y - j), F(y - j)};
  const F edge[3] = {F(0.25), F(0.5), F(0.25)};
  const F slope[4] = {F(-0.25), F(-0.25), F(0.25), F(0.25)};
  const F sy[2] = {F(-1.), F(1.)};
  const F curvature = width * width / F(12.);
  const F xy = curvature * F(d[0]) * F(d[1]);
  const F xz = curvature * F(d[0]) * F(d[2]);
  const F yz = curvature * F(d[1]) * F(d[2]);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const F weight = width * (wy[b] * wz[c] + yz * sy[b] * slope[c]);
#pragma unroll
      for (int a = 0; a < 3; ++a) visit(0, i - 1 + a, j + b, k - 1 + c, weight * edge[a]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
      visit(1, i - 1 + a, j, k - 1 + c, width * (wx[a] * wz[c] + xz * slope[a] * slope[c]));
  }
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const F weight = width * (wx[a] * wy[b] + xy * slope[a] * sy[b]);
#pragma unroll
      for (int c = 0; c < 3; ++c) visit(2, i - 1 + a, j + b, k - 1 + c, weight * edge[c]);
    }
}

// Four-point Gauss quadrature of the quintic-compensated shape over one cut
// piece of the chord (the quintic branch of longitudinal_shape::weights).
template <class G, class V>
__device__ __forceinline__ void quintic_segment(const GridT<G>& g, const double x[3],
                                                const double v[3], double lower,
                                                double upper, double width, V& visit) {
  using F = typename V::Weight;
  const double q[4] = {-.8611363115940525752, -.3399810435848562648,
                       .3399810435848562648, .8611363115940525752};
  const double qw[4] = {.3478548451374538574, .6521451548625461426,
                        .6521451548625461426, .3478548451374538574};
  for (int t = 0; t < 4; ++t) {
    const double u = .5 * (upper + lower + width * q[t]), xx = x[0] + u * v[0],
                 yy = x[1] + u * v[1], zz = x[2] + u * v[2];
    const F factor = F(.5 * width * qw[t]);
    long long i = (long long)floor(xx), j = (long long)floor(yy);
    if (i == (long long)g.nx) --i;
    if (j == (long long)g.ny) --j;
    const F fx = F(xx - i), fy = F(yy - j);
    QuinticSplines<F> spline;
    quintic_splines(zz, spline);
    Basis<F> nodes, edge;
    quintic_compensate(spline.node, 5, spline.cell, nodes);
    quintic_compensate(spline.edge, 4, spline.cell, edge);
    for (int k = 0; k < nodes.count; ++k) {
      const F w = factor * nodes.v[k];
      if (w == F(0.)) continue;
      for (int b = 0; b < 2; ++b) visit(0, i, j + b, nodes.first + k, w * (b ? fy : F(1.) - fy));
      for (int a = 0; a < 2; ++a) visit(1, i + a, j, nodes.first + k, w * (a ? fx : F(1.) - fx));
    }
    for (int k = 0; k < edge.count; ++k) {
      const F w = factor * edge.v[k];
      if (w == F(0.)) continue;
      for (int b = 0; b < 2; ++b)
        for (int a = 0; a < 2; ++a)
          visit(2, i + a, j + b, edge.first + k,
                w * (a ? fx : F(1.) - fx) * (b ? fy : F(1.) - fy));
    }
  }
}

// quintic_segment for the deposit and the electric gather: every Gauss point
// of a cut piece lies in the same cell, so the 4 x 92 node visits fall on 92
// nodes; each node's four weights are summed first and visited once (a
// quarter of the atomics or S reads).  The weights are quintic_segment's;
// only their summation order changes.  The
// walk is node by node: a Gauss point's compensated value at a node is formed
// once (quintic_compensated_at, the same sums as quintic_compensate) and
// shared by the component's transverse corners, so a node keeps four live
// sums and the 12-node loop stays rolled.  A piece whose Gauss points
// straddle a cell (only possible through rounding at a cut) is visited point
// by point.
template <class G, class V>
__device__ __forceinline__ void quintic_segment_summed(const GridT<G>& g, const double x[3],
                                                       const double v[3], double lower,
                                                       double upper, double width, V& visit) {
  using F = typename V::Weight;
  const double q[4] = {-.8611363115940525752, -.3399810435848562648,
                       .3399810435848562648, .8611363115940525752};
  const double qw[4] = {.3478548451374538574, .6521451548625461426,
                        .6521451548625461426, .3478548451374538574};
  double zz[4];
  F factor[4], fx[4], fy[4];
  long long i = 0, j = 0, kz = 0;
  bool same = true;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const double u = .5 * (upper + lower + width * q[t]), xx = x[0] + u * v[0],
                 yy = x[1] + u * v[1];
    zz[t] = x[2] + u * v[2];
    factor[t] = F(.5 * width * qw[t]);
    long long it = (long long)floor(xx), jt = (long long)floor(yy);
    if (it == (long long)g.nx) --it;
    if (jt == (long long)g.ny) --jt;
    const long long kt = (long long)floor(zz[t]);
    fx[t] = F(xx - it);
    fy[t] = F(yy - jt);
    if (t == 0) {
      i = it;
      j = jt;
      kz = kt;
    } else if (it != i || jt != j || kt != kz) {
      same = false;
    }
  }
  if (!same) {
    quintic_segment(g, x, v, lower, upper, width, visit);
    return;
  }
  // Each Gauss point's spline recursion once.
  QuinticSplines<F> spline[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) quintic_splines(zz[t], spline[t]);
  const long long first = (long long)spline[0].cell - 5;
  // Jx at (i, j + c) and Jy at (i + c, j): node basis, 12 nodes.
#pragma unroll 1
  for (int k = 0; k < 12; ++k) {
    F acc[4] = {F(0.), F(0.), F(0.), F(0.)};
    bool hit = false;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const F w = factor[t] * quintic_compensated_at(spline[t].node, 5, k);
      if (w == F(0.)) continue;
      hit = true;
      acc[0] += w * (F(1.) - fy[t]);
      acc[1] += w * fy[t];
      acc[2] += w * (F(1.) - fx[t]);
      acc[3] += w * fx[t];
    }
    if (!hit) continue;
    visit(0, i, j, first + k, acc[0]);
    visit(0, i, j + 1, first + k, acc[1]);
    visit(1, i, j, first + k, acc[2]);
    visit(1, i + 1, j, first + k, acc[3]);
  }
  // Jz at (i + a, j + c): edge basis, 11 nodes.
#pragma unroll 1
  for (int k = 0; k < 11; ++k) {
    F acc[4] = {F(0.), F(0.), F(0.), F(0.)};
    bool hit = false;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const F w = factor[t] * quintic_compensated_at(spline[t].edge, 4, k);
      if (w == F(0.)) continue;
      hit = true;
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int a = 0; a < 2; ++a)
          acc[2 * c + a] += w * (a ? fx[t] : F(1.) - fx[t]) * (c ? fy[t] : F(1.) - fy[t]);
    }
    if (!hit) continue;
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int a = 0; a < 2; ++a) visit(2, i + a, j + c, first + k, acc[2 * c + a]);
  }
}

// longitudinal_shape::weights (src/longitudinal_shape.h:97-117) with
// smoothX = (shape == linear-binomial3).  Returns the segment count, or -1
// when the chord exceeds the 64-cut crossing budget.
// lattice_shape_weights takes the chord in lattice units: start
// x = (begin - origin)/h and extent v = (end - begin)/h per axis.
template <int S, class F, class V>
__device__ int lattice_shape_weights(const GridT<F>& g, const double x[3], const double v[3],
                                     V& visit);

template <int S, class F, class V>
__device__ __forceinline__ int shape_weights(const GridT<F>& g, const double begin[3],
                                             const double end[3], V& visit) {
  const double h[3] = {g.dx, g.dy, g.dz};
  double x[3], v[3];
  for (int a = 0; a < 3; ++a) {
    x[a] = (begin[a] - g.origin[a]) / h[a];
    v[a] = (end[a] - begin[a]) / h[a];
  }
  return lattice_shape_weights<S>(g, x, v, visit);
}

template <int S, class F, class V>
__device__ __forceinline__ int lattice_shape_weights(const GridT<F>& g, const double x[3],
                                                     const double v[3], V& visit) {
  // The cell-boundary cuts of the chord, ascending.  Along each axis the cuts
  // (j - x)/v of the crossed lattice planes j are already monotone, so a
  // three-way merge yields the sorted cut sequence of the reference (same
  // values, ties give zero-width pieces) without a cut array.
  double next[3];
  long long plane[3], left[3];
  int dir[3];
  long long total = 0;
  for (int a = 0; a < 3; ++a) {
    left[a] = 0;
    if (v[a] != 0.) {
      const double lo = fmin(x[a], x[a] + v[a]), hi = fmax(x[a], x[a] + v[a]);
      const long long first = (long long)floor(lo) + 1, last = (long long)ceil(hi) - 1;
      left[a] = last >= first ? last - first + 1 : 0;
      dir[a] = v[a] > 0. ? 1 : -1;
      plane[a] = v[a] > 0. ? first : last;
      if (left[a]) next[a] = (plane[a] - x[a]) / v[a];
    }
    total += left[a];
  }
  if (total > 62) return -1;  // more than 64 cuts with the chord ends
  int segments = 0;
  double lower = 0.;
  for (;;) {
    int axis = -1;
    for (int a = 0; a < 3; ++a)
      if (left[a] && (axis < 0 || next[a] < next[axis])) axis = a;
    double upper = 1.;
    if (axis >= 0) {
      upper = next[axis];
      plane[axis] += dir[axis];
      if (--left[axis]) next[axis] = (plane[axis] - x[axis]) / v[axis];
    }
    const double width = upper - lower;
    const double piece_lower = lower;
    lower = upper;
    if (width > 0.) {
      ++segments;
      if constexpr (S == 0) {
        if constexpr (V::kF3Segment)
          visit.f3_segment(g, x, v, piece_lower, upper);
        else
          binomial_xz_segment(g, x, v, piece_lower, upper, visit);
      } else {
        if constexpr (V::kQuinticSummed)
          quintic_segment_summed(g, x, v, piece_lower, upper, width, visit);
        else
          quintic_segment(g, x, v, piece_lower, upper, width, visit);
      }
    }
    if (axis < 0) break;
  }
  return segments;
}

// ---------------------------------------------------------------------------
// gathers (src/source_coupling.cpp:31-51, src/source_coupling_math.h:122-250)
struct OpenOrbit {
  double first, last;
  double begin[3], end[3];
  bool valid;
};

// clipOpenOrbit at one rank (src/source_coupling_math.h:234-250).
template <class F>
__device__ __forceinline__ bool clip_open_orbit(const GridT<F>& g, const double b[3],
                                                const double e[3], OpenOrbit& o) {
  const double ds[3] = {g.dx, g.dy, g.dz};
  const double size[3] = {(double)g.nx, (double)g.ny, (double)g.nz};
  o.first = 0.;
  o.last = 1.;
  o.valid = true;
  for (int a = 0; a < 3; ++a) {
    o.begin[a] = b[a];
    o.end[a] = e[a];
  }
  for (int a = 0; a < 3; ++a) {
    const double x = (b[a] - g.origin[a]) / ds[a], d = (e[a] - b[a]) / ds[a];
    if (!isfinite(x) || !isfinite(d)) return false;
    if (d == 0.) {
      if (x < 0. || x > size[a]) o.valid = false;
      continue;
    }
    {
      const double t = -x / d;
      if (d > 0.) o.first = fmax(o.first, t);
      else o.last = fmin(o.last, t);
    }
    {
      const double t = (size[a] - x) / d;
      if (d > 0.) o.last = fmin(o.last, t);
      else o.first = fmax(o.first, t);
    }
  }
  o.valid = o.valid && o.last >= o.first;
  if (o.valid)
    for (int a = 0; a < 3; ++a) {
      const double d = e[a] - b[a];
      if (o.first != 0.) o.begin[a] = b[a] + o.first * d;
      if (o.last != 1.) o.end[a] = b[a] + o.last * d;
    }
  return true;
}

// Orbit average of 1/2 (E_new + E^n) with the shape weights, read from the
// orbit sum S = E_new + E^n that orbit_sum_kernel forms once per trial
// (E_new = E* - dt/eps0 J for the residual, E* for the first-trial guess).
// Three component arrays passed by value, so that constant component
// indices keep the pointers in registers.
template <class W>
struct Ptr3 {
  const W* p[3];
};

// The cut pieces of a chord in lattice units, one at a time, in the order
// and with the cut values of shape_weights (longitudinal_shape::weights).
struct CutWalker {
  double x[3], v[3], next[3], lower;
  long long plane[3], left[3];
  int dir[3];
  bool done;
  // The chord's lattice coordinates; false beyond the 64-cut budget.
  __device__ bool init(const double begin[3], const double end[3], const double origin[3],
                       const double h[3]) {
    long long total = 0;
    for (int a = 0; a < 3; ++a) {
      x[a] = (begin[a] - origin[a]) / h[a];
      v[a] = (end[a] - begin[a]) / h[a];
      left[a] = 0;
      dir[a] = 1;
      plane[a] = 0;
      next[a] = 0.;
      if (v[a] != 0.) {
        const double lo = fmin(x[a], x[a] + v[a]), hi = fmax(x[a], x[a] + v[a]);
        const long long first = (long long)floor(lo) + 1, last = (long long)ceil(hi) - 1;
        left[a] = last >= first ? last - first + 1 : 0;
        dir[a] = v[a] > 0. ? 1 : -1;
        plane[a] = v[a] > 0. ? first : last;
        if (left[a]) next[a] = (plane[a] - x[a]) / v[a];
      }
      total += left[a];
    }
    lower = 0.;
    done = false;
    return total <= 62;
  }
  // The next piece of nonzero width, as shape_weights cuts the chord.
  __device__ bool advance(double& first, double& last) {
    while (!done) {
      int axis = -1;
      for (int a = 0; a < 3; ++a)
        if (left[a] && (axis < 0 || next[a] < next[axis])) axis = a;
      double upper = 1.;
      if (axis >= 0) {
        upper = next[axis];
        plane[axis] += dir[axis];
        if (--left[axis]) next[axis] = (plane[axis] - x[axis]) / v[axis];
      } else {
        done = true;
      }
      const double width = upper - lower;
      first = lower;
      last = upper;
      lower = upper;
      if (width > 0.) return true;
    }
    return false;
  }
};

template <class W, class F>
struct ElectricVisitor {
  static constexpr bool kF3Segment = true;
  // Quintic pieces arrive with each node's four Gauss-point weights summed:
  // the gather is linear in the weights, so this reads each S node once
  // instead of four times; the per-particle sum then differs from the
  // reference's point-by-point order in the last bits (binomial3 pieces keep
  // the reference's order exactly).
  static constexpr bool kQuinticSummed = true;
  using Weight = W;
  const GridT<F>* g;
  Ptr3<W> s;             // orbit sum S = E_new + E^n per E node (ring layout)
  W r[3];
  __device__ __forceinline__ void operator()(int d, long long i, long long j, long long k, W w) {
    const GridT<F>& G = *g;
    if (i < 0 || j < 0 || i >= e_nx(G, d) || j >= e_ny(G, d)) return;
    if (k < 0 || k >= e_nz(G, d)) return;
    r[d] += W(.5) * w * s.p[d][e_index(G, d, (int)i, (int)j, (int)k)];
  }

  // One accumulation .5*w*(E_new + E^n) at the ring offset n of a node.
  __device__ __forceinline__ W term(int d, size_t n, size_t, W w) const {
    return W(.5) * w * s.p[d][APRL_BOUNDED(g->status, n, e_count(*g, d), 24 + d)];
  }

  // binomialXZSegment specialised for the gather.  When the whole 4x2x4
  // stencil is inside every component and inside the current mask (true
  // for particles away from the PEC faces and the window ends), each stencil
  // row is addressed once and its nodes read back to back; otherwise the
  // generic visits run.  Per component the accumulation order is the
  // reference's (Ex: k, y, x; Ey: k, x; Ez: y, x, k).
  __device__ __forceinline__ void f3_segment(const GridT<F>& G, const double s[3],
                                             const double d[3], double first, double last) {
    const W width = W(last - first);
    const double mid = (first + last) * 0.5;
    const double x = s[0] + mid * d[0], y = s[1] + mid * d[1], z = s[2] + mid * d[2];
    long long i = (long long)floor(x), j = (long long)floor(y);
    const long long k = (long long)floor(z);
    if (i == (long long)G.nx) --i;
    if (j == (long long)G.ny) --j;
    if (!(i >= 2 && i <= G.nx - 3 && j >= 1 && j <= G.ny - 2 && k >= 2 && k <= G.nz - 3)) {
      binomial_xz_segment(G, s, d, first, last, *this);
      return;
    }
    W wx[4], wz[4];
    node_weights(W(x - i), wx);
    node_weights(W(z - k), wz);
    const W wy[2] = {W(1.) - W(y - j), W(y - j)};
    const W edge[3] = {W(0.25), W(0.5), W(0.25)};
    const W slope[4] = {W(-0.25), W(-0.25), W(0.25), W(0.25)};
    const W sy[2] = {W(-1.), W(1.)};
    const W curvature = width * width / W(12.);
    const W xy = curvature * W(d[0]) * W(d[1]);
    const W xz = curvature * W(d[0]) * W(d[2]);
    const W yz = curvature * W(d[1]) * W(d[2]);
    const int I = (int)i, J = (int)j, K = (int)k;
    // Ex (nx, ny+1, nz+1): nodes x I-1..I+1, y J..J+1, z K-1..K+2
    {
      const int nxc = G.nx, nyc = G.ny + 1, nzc = G.nz + 1;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const size_t plane = (size_t)ring(K - 1 + c, G.zb_e[0], nzc) * nyc;
        const size_t jplane = (size_t)(K - 1 + c) * nyc;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const W weight = width * (wy[b] * wz[c] + yz * sy[b] * slope[c]);
          const size_t n0 = (plane + J + b) * nxc + (I - 1);
          const size_t j0 = (jplane + J + b) * nxc + (I - 1);
#pragma unroll
          for (int a = 0; a < 3; ++a) r[0] += term(0, n0 + a, j0 + a, weight * edge[a]);
        }
      }
    }
    // Ey (nx+1, ny, nz+1): nodes x I-1..I+2, y J, z K-1..K+2
    {
      const int nxc = G.nx + 1, nyc = G.ny, nzc = G.nz + 1;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const size_t n0 = ((size_t)ring(K - 1 + c, G.zb_e[1], nzc) * nyc + J) * nxc + (I - 1);
        const size_t j0 = ((size_t)(K - 1 + c) * nyc + J) * nxc + (I - 1);
#pragma unroll
        for (int a = 0; a < 4; ++a)
          r[1] += term(1, n0 + a, j0 + a, width * (wx[a] * wz[c] + xz * slope[a] * slope[c]));
      }
    }
    // Ez (nx+1, ny+1, nz): nodes x I-1..I+2, y J..J+1, z K-1..K+1
    {
      const int nxc = G.nx + 1, nyc = G.ny + 1, nzc = G.nz;
      size_t plane[3], jplane[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        plane[c] = (size_t)ring(K - 1 + c, G.zb_e[2], nzc) * nyc;
        jplane[c] = (size_t)(K - 1 + c) * nyc;
      }
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const W weight = width * (wx[a] * wy[b] + xy * slope[a] * sy[b]);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            r[2] += term(2, (plane[c] + J + b) * nxc + (I - 1 + a),
                         (jplane[c] + J + b) * nxc + (I - 1 + a), weight * edge[c]);
        }
    }
  }
};

template <class W, class F>
__device__ __forceinline__ W open_b(const GridT<F>& g, const Ptr3<W>& bsrc, int a, long long i,
                                    long long j, long long k) {
  const long long nxc = b_nx(g, a), nyc = b_ny(g, a), nzc = b_nz(g, a);
  if (i < 0) i = 0;
  if (i > nxc - 1) i = nxc - 1;
  if (j < 0) j = 0;
  if (j > nyc - 1) j = nyc - 1;
  if (k < 0) k = 0;
  if (k >= nzc) k = nzc - 1;
  return bsrc.p[a][b_index(g, a, (int)i, (int)j, (int)k)];
}

// binomialXZMagneticSample (src/source_coupling_math.h:142-167).  Rows of
// the 4x2x4 stencil that lie inside the component are read without the
// open-face clamps; the clamped form runs otherwise.  Same order either way.
template <class W, class F>
__device__ __forceinline__ void binomial_xz_magnetic(const GridT<F>& g, const Ptr3<W>& bsrc,
                                                     const double p[3], double value[3]) {
  const double h[3] = {g.dx, g.dy, g.dz};
  // the point in lattice units, shared by the three components' staggerings
  double lattice[3];
  for (int d = 0; d < 3; ++d) lattice[d] = (p[d] - g.origin[d]) / h[d];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    long long cell[3];
    double fraction[3];
    for (int d = 0; d < 3; ++d) {
      const double pos = lattice[d] - (a == d ? 0. : 0.5);
      cell[d] = (long long)floor(pos);
      fraction[d] = pos - cell[d];
    }
    W wx[4], wz[4];
    node_weights(W(fraction[0]), wx);
    node_weights(W(fraction[2]), wz);
    const W wy[2] = {W(1. - fraction[1]), W(fraction[1])};
    const long long nxc = b_nx(g, a), nyc = b_ny(g, a), nzc = b_nz(g, a);
    W v = W(0.);
    if (cell[0] >= 1 && cell[0] + 2 <= nxc - 1 && cell[1] >= 0 && cell[1] + 1 <= nyc - 1 &&
        cell[2] >= 1 && cell[2] + 2 <= nzc - 1) {
      const W* base = bsrc.p[a];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const size_t plane = (size_t)ring((int)cell[2] - 1 + k, g.zb_b[a], (int)nzc) * nyc;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const size_t row = (plane + cell[1] + j) * nxc + (cell[0] - 1);
          W r = W(0.);
#pragma unroll
          for (int i = 0; i < 4; ++i)
            r += wx[i] * base[APRL_BOUNDED(g.status, row + i, b_count(g, a), 27 + a)];
          v += wz[k] * wy[j] * r;
        }
      }
    } else {
      for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 2; ++j) {
          W row = W(0.);
          for (int i = 0; i < 4; ++i)
            row += wx[i] * open_b(g, bsrc, a, cell[0] - 1 + i, cell[1] + j, cell[2] - 1 + k);
          v += wz[k] * wy[j] * row;
        }
    }
    value[a] = double(v);
  }
}

// magneticSample(bounds=false, halo, openFaces=true) (src/source_coupling_math.h:122-138).
template <class W, class F>
__device__ __forceinline__ void trilinear_magnetic(const GridT<F>& g, const Ptr3<W>& bsrc,
                                                   const double p[3], double value[3]) {
  const double ds[3] = {g.dx, g.dy, g.dz};
  int cell[2][3];
  double fraction[2][3];
  for (int half = 0; half < 2; ++half)
    for (int d = 0; d < 3; ++d) {
      const double x = (p[d] - g.origin[d]) / ds[d] - .5 * half;
      cell[half][d] = (int)floor(x);
      fraction[half][d] = x - cell[half][d];
    }
  for (int axis = 0; axis < 3; ++axis) {
    const int hx = axis == 0 ? 0 : 1, hy = axis == 1 ? 0 : 1, hz = axis == 2 ? 0 : 1;
    W v = W(0.);
    for (int k = 0; k < 2; ++k)
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
          const W x = W(i ? fraction[hx][0] : 1 - fraction[hx][0]),
                  y = W(j ? fraction[hy][1] : 1 - fraction[hy][1]),
                  z = W(k ? fraction[hz][2] : 1 - fraction[hz][2]);
          v += x * y * z *
               open_b(g, bsrc, axis, cell[hx][0] + i, cell[hy][1] + j, cell[hz][2] + k);
        }
    value[axis] = double(v);
  }
}

// Impl::electric(a, b, open=true) for wide shapes and Impl::magnetic
// (src/source_coupling.cpp:31-51) of one chord a -> b: both clip the chord
// with clipOpenOrbit, which is done once here; the electric error (crossing
// budget) skips the magnetic gather, as the reference's call order does.
template <int S, class W, class F>
__device__ __forceinline__ unsigned gather_fields(const GridT<F>& g, const double a[3],
                                                  const double b[3], const Ptr3<W>& orbit,
                                                  const Ptr3<W>& bsrc, double e_out[3],
                                                  double b_out[3]) {
  OpenOrbit path;
  if (!clip_open_orbit(g, a, b, path)) return kErrNonFinite;
  if (!path.valid) return kErrOrbitOutside;
  double middle[3];
  for (int d = 0; d < 3; ++d) middle[d] = (path.begin[d] + path.end[d]) * .5;
  const double fraction = path.last - path.first;
  ElectricVisitor<W, F> ev{&g, orbit, {W(0.), W(0.), W(0.)}};
  if (shape_weights<S>(g, path.begin, path.end, ev) < 0) return kErrCrossingBudget;
  for (int d = 0; d < 3; ++d) e_out[d] = double(ev.r[d]) * fraction;
  if constexpr (S == 0)
    binomial_xz_magnetic(g, bsrc, middle, b_out);
  else
    trilinear_magnetic(g, bsrc, middle, b_out);
  return kErrNone;
}

// ---------------------------------------------------------------------------
// deposition: Current::deposit at one rank (src/longitudinal_shape.h:175-187)
// Q: the deterministic mode's fixed-point sum (fixed_add into G.jq) instead
// of binary64 atomics into J.
template <class F, bool Q>
struct DepositVisitor {
  static constexpr bool kF3Segment = false;
  static constexpr bool kQuinticSummed = true;
  using Weight = F;
  const GridT<F>* g;
  F scale[3];
  bool smooth_x;
  unsigned error;
  __device__ __forceinline__ void operator()(int a, long long i, long long j, long long k, F w) {
    if (scale[a] == F(0.)) return;
    const GridT<F>& G = *g;
    if (i < 0 || i >= e_nx(G, a)) {
      if (!smooth_x) error = kErrSupportX;
      return;
    }
    if (j < 0 || j >= e_ny(G, a)) {
      error = kErrSupportY;
      return;
    }
    if (k < 0 || k >= e_nz(G, a)) return;
    const size_t at = j_index(G, a, (int)i, (int)j, (int)k);
    if constexpr (Q) {
      // Order-free integer sum, converted to J once per trial.
      if (!fixed_add(G.jq[a] + 2 * at, double(scale[a] * w), G.jq_scale)) error = kErrFixedRange;
    } else {
      atomicAdd(&G.j[a][at], scale[a] * w);
    }
  }
};

// ChargeConservingCurrentDepositor::depositSegment (src/eb_deposition.cpp:41-51,
// validatePosition 228-246).
template <class F>
__device__ __forceinline__ unsigned validate_segment(const GridT<F>& g, const double b[3],
                                                     const double e[3], double charge) {
  const double extent[3] = {(double)g.nx * g.dx, (double)g.ny * g.dy, (double)g.nz * g.dz};
  for (int a = 0; a < 3; ++a) {
    const double tol = 64.0 * kEpsilon * fmax(1.0, fmax(fabs(g.origin[a]), extent[a]));
    const double rb = b[a] - g.origin[a], re = e[a] - g.origin[a];
    if (!isfinite(b[a]) || rb < -tol || rb > extent[a] + tol) return kErrDepositOutside;
    if (!isfinite(e[a]) || re < -tol || re > extent[a] + tol) return kErrDepositOutside;
  }
  if (!isfinite(charge)) return kErrNonFinite;
  return kErrNone;
}

template <int S, bool Q, class F>
__device__ unsigned deposit_segment(const GridT<F>& g, const double b[3],
                                    const double e[3], double charge) {
  const unsigned invalid = validate_segment(g, b, e, charge);
  if (invalid) return invalid;
  DepositVisitor<F, Q> v;
  v.g = &g;
  v.smooth_x = S == 0;
  v.error = kErrNone;
  for (int a = 0; a < 3; ++a)
    v.scale[a] = F(charge * (e[a] - b[a]) / (g.dx * g.dy * g.dz * g.dt));
  if (shape_weights<S>(g, b, e, v) < 0) return kErrCrossingBudget;
  return v.error;
}

// ---------------------------------------------------------------------------
// push (src/source_coupling_math.h:272-293, src/source_coupling.cpp:90-104)

// source_coupling_math::momentum.  Returns 0 or an error code.
__device__ unsigned momentum(double u[3], const double e[3], const double mag[3],
                             double q, double m, double h, double g0) {
  const double before[3] = {u[0], u[1], u[2]};
  const double ks = q * h / (2 * m * kC);
  const double bs = q * h / (2 * m);
  double kick[3], b[3], a[3], axb[3];
  for (int i = 0; i < 3; ++i) {
    kick[i] = e[i] * ks;
    b[i] = mag[i] * bs;
  }
  for (int i = 0; i < 3; ++i) a[i] = before[i] + kick[i];
  axb[0] = a[1] * b[2] - a[2] * b[1];
  axb[1] = a[2] * b[0] - a[0] * b[2];
  axb[2] = a[0] * b[1] - a[1] * b[0];
  const double b2 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  const double ka = kick[0] * a[0] + kick[1] * a[1] + kick[2] * a[2];
  const double kb = kick[0] * b[0] + kick[1] * b[1] + kick[2] * b[2];
  const double ab = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  const double kcross = kick[0] * axb[0] + kick[1] * axb[1] + kick[2] * axb[2];
  const double first = (kick[0] * before[0] + kick[1] * before[1] + kick[2] * before[2]) / g0;
  const double kk = kick[0] * kick[0] + kick[1] * kick[1] + kick[2] * kick[2];
  double G = g0 + first + (kk + kcross / g0 - first * first) / g0;
  G = fmax(G, .5 * (g0 + 1.));
  int iteration = 0;
  for (; iteration < 12; ++iteration) {
    const double den = G * G + b2, numerator = G * G * ka + G * kcross + ab * kb;
    const double f = G * (G - g0) - numerator / den;
    const double derivative =
        2 * G - g0 - ((2 * G * ka + kcross) * den - 2 * G * numerator) / (den * den);
    const double correction = f / derivative;
    const double next = G - correction;
    if (!isfinite(next) || next < .5 * (g0 + 1.) - 1e-13) return kErrRootNonphysical;
    G = fmax(next, .5 * (g0 + 1.));
    if (fabs(correction) <= 8 * kEpsilon * fmax(1., G)) break;
  }
  if (iteration == 12) return kErrRootNoConvergence;
  const double den = G * G + b2;
  for (int k = 0; k < 3; ++k) u[k] = 2 * (G * G * a[k] + ab * b[k] + G * axb[k]) / den - before[k];
  return kErrNone;
}

// SIMagneticElement::fieldsLab, magnetic part (src/eb_sources.cpp:352-447).
__device__ void magnet_lab(const DMagnet& m, const double pos[3], double b[3]) {
  b[0] = b[1] = b[2] = 0.0;
  const double rel[3] = {pos[0] - m.center[0], pos[1] - m.center[1], pos[2] - m.center[2]};
  const double z = rel[2];
  if (m.type == 2) {
    if (z >= 0.0 && z <= m.length) {
      const double x = rel[0] * m.cos_angle + rel[1] * m.sin_angle;
      const double y = -rel[0] * m.sin_angle + rel[1] * m.cos_angle;
      const double bx = m.quadrupole_gradient * y, by = m.quadrupole_gradient * x;
      b[0] = bx * m.cos_angle - by * m.sin_angle;
      b[1] = bx * m.sin_angle + by * m.cos_angle;
    }
    return;
  }
  if (m.type == 1) {
    if (z >= 0.0 && z <= m.length) {
      b[0] = m.peak_field * m.cos_angle;
      b[1] = m.peak_field * m.sin_angle;
    }
    return;
  }
  const double k = m.wave_number;
  double ts = 0.0, ls = 0.0;
  if (z >= 0.0 && z <= m.length) {
    ts = sin(k * z);
    ls = cos(k * z);
  } else if (m.gaussian_fringe) {
    const double fc = z < 0.0 ? z : z - m.length;
    const double distance = fabs(fc);
    if (distance >= m.fringe_extent) return;
    const double q = distance / m.fringe_extent;
    const double q2 = q * q, q3 = q2 * q, q4 = q3 * q, q5 = q4 * q;
    const double taper = 1.0 - 10.0 * q3 + 15.0 * q4 - 6.0 * q5;
    const double taper_derivative = (-30.0 * q2 + 60.0 * q3 - 30.0 * q4) / m.fringe_extent;
    const double gaussian = exp(-0.5 * pow(k * distance, 2.0));
    ls = gaussian * taper;
    const double dbd = gaussian * (taper_derivative - k * k * distance * taper);
    ts = z < 0.0 ? dbd / k : -dbd / k;
  } else {
    return;
  }
  const double tc = rel[0] * m.cos_angle + rel[1] * m.sin_angle;
  const double tf = m.peak_field * cosh(k * tc) * ts;
  b[0] = tf * m.cos_angle;
  b[1] = tf * m.sin_angle;
  b[2] = m.peak_field * sinh(k * tc) * ls;
}

// SIFieldSourceSet::addPrescribedBox (src/eb_sources.cpp:537-582) with lab
// magnets only: box event -> lab event, sum of magnets, lab -> box fields.
template <class F>
__device__ void add_prescribed_box(const PushArgs<F>& a, const double pos[3], double t_box,
                                   double e[3], double b[3]) {
  if (a.n_magnets == 0) return;
  const DFrame& f = a.frame;
  const double z_shift = pos[2] - f.box_z_origin;
  const double pos_lab[3] = {pos[0], pos[1],
                             f.lab_z_origin + fma(f.gamma_beta * kC, t_box, f.gamma * z_shift)};
  double bl[3] = {0., 0., 0.};
  for (int n = 0; n < a.n_magnets; ++n) {
    double c[3];
    magnet_lab(a.magnets[n], pos_lab, c);
    for (int d = 0; d < 3; ++d) bl[d] += c[d];
  }
  // fieldsLabToBox with zero lab E (src/boostframe.cpp:262-273)
  const double el[3] = {0., 0., 0.};
  const double ebx[3] = {fma(-f.gamma_beta * kC, bl[1], f.gamma * el[0]),
                         fma(f.gamma_beta * kC, bl[0], f.gamma * el[1]), el[2]};
  const double bbx[3] = {fma(f.gamma_beta / kC, el[1], f.gamma * bl[0]),
                         fma(-f.gamma_beta / kC, el[0], f.gamma * bl[1]), bl[2]};
  for (int d = 0; d < 3; ++d) {
    e[d] += ebx[d];
    b[d] += bbx[d];
  }
}

// Adds the number of lanes with `flag` to *counter with one atomic per
// converged group of the warp.
__device__ __forceinline__ void count_lanes(unsigned long long* counter, bool flag) {
  const unsigned group = __activemask();
  const unsigned ballot = __ballot_sync(group, flag);
  if (ballot && (threadIdx.x & 31) == __ffs(group) - 1)
    atomicAdd(counter, (unsigned long long)__popc(ballot));
}

// ---------------------------------------------------------------------------
// particle boundaries (src/particle_boundary.cpp)
struct Hit {
  double position[3];
  double fraction;
  int face;
};

// ParticleCPMLRegion::firstEntry (src/particle_boundary.cpp:104-174).
__device__ unsigned cpml_first_entry(const DRegion& r, const double s[3], const double e[3],
                                     Hit& hit, bool& entered) {
  double best = INFINITY;
  int best_face = 0;
  entered = false;
  for (int axis = 0; axis < 3; ++axis) {
    if (!isfinite(s[axis]) || !isfinite(e[axis])) return kErrNonFinite;
    if (s[axis] < r.physical_lower[axis] - r.tolerance[axis] ||
        s[axis] > r.physical_upper[axis] + r.tolerance[axis])
      return kErrStartInCpml;
    if (r.cells[axis] == 0) continue;
    double candidate = 0.0;
    int face = 0;
    bool h = false;
    if (e[axis] < r.physical_lower[axis]) {
      candidate = (r.physical_lower[axis] - s[axis]) / (e[axis] - s[axis]);
      face = 2 * axis;
      h = true;
    } else if (e[axis] > r.physical_upper[axis]) {
      candidate = (r.physical_upper[axis] - s[axis]) / (e[axis] - s[axis]);
      face = 2 * axis + 1;
      h = true;
    }
    if (h && candidate < best) {
      best = candidate;
      best_face = face;
      entered = true;
    }
  }
  if (!entered) return kErrNone;
  const double ft = 64.0 * kEpsilon;
  if (!isfinite(best) || best < -ft || best > 1.0 + ft) return kErrHitLocate;
  hit.fraction = fmax(0.0, fmin(1.0, best));
  hit.face = best_face;
  for (int a = 0; a < 3; ++a) {
    hit.position[a] = s[a] + hit.fraction * (e[a] - s[a]);
    hit.position[a] = fmax(r.outer_lower[a], fmin(r.outer_upper[a], hit.position[a]));
  }
  const int normal = best_face / 2;
  hit.position[normal] = (best_face % 2) ? r.physical_upper[normal] : r.physical_lower[normal];
  return kErrNone;
}

// ParticleOpenBoundary::firstExit (src/particle_boundary.cpp:303-373).
__device__ unsigned outer_first_exit(const DRegion& r, const double s[3], const double e[3],
                                     Hit& hit, bool& escaped) {
  double best = INFINITY;
  int best_face = 0;
  escaped = false;
  for (int axis = 0; axis < 3; ++axis) {
    if (!isfinite(s[axis]) || !isfinite(e[axis])) return kErrNonFinite;
    if (s[axis] < r.global_lower[axis] - r.global_tolerance[axis] ||
        s[axis] > r.global_upper[axis] + r.global_tolerance[axis])
      return kErrStartOutside;
    double candidate = 0.0;
    int face = 0;
    bool h = false;
    if (e[axis] < r.global_lower[axis]) {
      candidate = (r.global_lower[axis] - s[axis]) / (e[axis] - s[axis]);
      face = 2 * axis;
      h = true;
    } else if (e[axis] > r.global_upper[axis]) {
      candidate = (r.global_upper[axis] - s[axis]) / (e[axis] - s[axis]);
      face = 2 * axis + 1;
      h = true;
    }
    if (h && candidate < best) {
      best = candidate;
      best_face = face;
      escaped = true;
    }
  }
  if (!escaped) return kErrNone;
  const double ft = 64.0 * kEpsilon;
  if (best < -ft || best > 1.0 + ft || !isfinite(best)) return kErrHitLocate;
  hit.fraction = fmax(0.0, fmin(1.0, best));
  hit.face = best_face;
  for (int a = 0; a < 3; ++a) {
    hit.position[a] = s[a] + hit.fraction * (e[a] - s[a]);
    hit.position[a] = fmax(r.global_lower[a], fmin(r.global_upper[a], hit.position[a]));
  }
  const int normal = best_face / 2;
  hit.position[normal] = (best_face % 2) ? r.global_upper[normal] : r.global_lower[normal];
  return kErrNone;
}

// ParticleCPMLRegion::conductivityRate / currentDampingFactor
// (src/particle_boundary.cpp:176-240).
__device__ double conductivity_rate(const DRegion& r, const double p[3]) {
  double rate = 0.0;
  for (int axis = 0; axis < 3; ++axis) {
    if (r.cells[axis] == 0) continue;
    double depth = 0.0;
    if (p[axis] < r.physical_lower[axis])
      depth = (r.physical_lower[axis] - p[axis]) / r.thickness[axis];
    else if (p[axis] > r.physical_upper[axis])
      depth = (p[axis] - r.physical_upper[axis]) / r.thickness[axis];
    depth = fmax(0.0, fmin(1.0, depth));
    rate += r.max_rate[axis] * pow(depth, r.order);
  }
  return rate;
}

__device__ double damping_factor(const DRegion& r, const double s[3], const double e[3],
                                 double duration) {
  if (duration == 0.0) return 1.0;
  const double abscissa = sqrt(3.0 / 5.0);
  const double node[3] = {0.5 * (1.0 - abscissa), 0.5, 0.5 * (1.0 + abscissa)};
  const double weight[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
  double average = 0.0;
  for (int k = 0; k < 3; ++k) {
    double p[3];
    for (int a = 0; a < 3; ++a) p[a] = s[a] + node[k] * (e[a] - s[a]);
    average += weight[k] * conductivity_rate(r, p);
  }
  const double exponent = -duration * average;
  return exponent < log(kDblMin) ? 0.0 : exp(exponent);
}

struct CarrierState {
  double pos[3], vel[3], q, w;
};

// processCarrierSegment at one rank (src/simulation.cpp:4310-4407).
// Returns an error code; *kept tells whether the carrier survives.
template <int S, bool Q, class F>
__device__ unsigned carrier_segment(const GridT<F>& g, const DRegion& r,
                                    CarrierState& c, const double seg_start[3],
                                    double seg_start_fraction, TrialCounters* counters,
                                    bool& kept) {
  const double cutoff = 64.0 * kEpsilon;
  kept = false;
  if (!(c.w >= 0.0) || !isfinite(c.w)) return kErrCarrierWeight;
  if (c.w <= cutoff) return kErrNone;
  Hit outer;
  bool exits = false;
  unsigned err = outer_first_exit(r, seg_start, c.pos, outer, exits);
  if (err) return err;
  double local_end = 1.0;
  double seg_end[3] = {c.pos[0], c.pos[1], c.pos[2]};
  if (exits) {
    local_end = outer.fraction;
    for (int a = 0; a < 3; ++a) seg_end[a] = outer.position[a];
  }
  const double global_end = seg_start_fraction + local_end * (1.0 - seg_start_fraction);
  const double duration = (global_end - seg_start_fraction) * g.dt;
  double midpoint[3];
  for (int a = 0; a < 3; ++a) midpoint[a] = 0.5 * (seg_start[a] + seg_end[a]);
  const double mid_damping = damping_factor(r, seg_start, midpoint, 0.5 * duration);
  const double end_damping = damping_factor(r, seg_start, seg_end, duration);
  const double deposited = c.w * mid_damping;
  const double end_weight = c.w * end_damping;
  err = deposit_segment<S, Q>(g, seg_start, seg_end, c.q * deposited);
  if (err) return err;
  if (exits) {
    atomicAdd(&counters->carrier_outer[outer.face], 1ull);
    atomicAdd(&counters->carrier_outer_charge[outer.face], c.q * end_weight);
    return kErrNone;
  }
  if (end_weight <= cutoff) return kErrNone;
  c.w = end_weight;
  for (int a = 0; a < 3; ++a) c.pos[a] = seg_end[a];
  kept = true;
  return kErrNone;
}

// ---------------------------------------------------------------------------
// Existing CPML carriers: ballistic step, damped deposit, outer exit
// (src/simulation.cpp:4531-4537).  Carriers deposit with the run's shape,
// like every ChargeConservingCurrentDepositor call.
template <class F, int S, bool Q>
__global__ void carrier_kernel(CarrierArgs<F> a) {
  if (trial_skipped(a.g)) return;
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.count) return;
  CarrierState c;
  c.pos[0] = a.in.px[n]; c.pos[1] = a.in.py[n]; c.pos[2] = a.in.pz[n];
  c.vel[0] = a.in.vx[n]; c.vel[1] = a.in.vy[n]; c.vel[2] = a.in.vz[n];
  c.q = a.in.q[n];
  c.w = a.in.w[n];
  const double start[3] = {c.pos[0], c.pos[1], c.pos[2]};
  for (int d = 0; d < 3; ++d) c.pos[d] += a.g.dt * c.vel[d];
  bool kept = false;
  const unsigned err = carrier_segment<S, Q>(a.g, a.region, c, start, 0.0, a.counters, kept);
  if (err) raise_error(a.status, err, (unsigned long long)n);
  count_lanes(&a.counters->carriers_kept, kept);
  a.keep[n] = kept ? 1 : 0;
  a.out.px[n] = c.pos[0]; a.out.py[n] = c.pos[1]; a.out.pz[n] = c.pos[2];
  a.out.vx[n] = c.vel[0]; a.out.vy[n] = c.vel[1]; a.out.vz[n] = c.vel[2];
  a.out.q[n] = c.q;
  a.out.w[n] = c.w;
  a.out.key[n] = a.in.key[n];
}

// ConservativeSourceCoupling::push of one slot (src/source_coupling.cpp:90-104):
// `substeps` Lapenta-Markidis substeps with the prescribed magnets, using the
// slot's gathered fields (the ballistic-guess gather of the first trial, or
// the previous residual's re-gather).
template <class F>
__device__ unsigned coupling_push(const PushArgs<F>& a, long long n, double pos[3], double u[3],
                                  double q, double m, double time, double dt, double used_e[3],
                                  double used_b[3], double& abs_work) {
  for (int d = 0; d < 3; ++d) {
    used_e[d] = a.next_e[3 * n + d];
    used_b[d] = a.next_b[3 * n + d];
  }
  abs_work = 0.0;
  const double h = dt / a.substeps;
  for (int s = 0; s < a.substeps; ++s) {
    const double before_pos[3] = {pos[0], pos[1], pos[2]};
    const double before_u[3] = {u[0], u[1], u[2]};
    const double g0 = gamma_u(u[0], u[1], u[2]);
    const double ps = .5 * h * kC / g0;
    const double point[3] = {pos[0] + ps * u[0], pos[1] + ps * u[1], pos[2] + ps * u[2]};
    double ee[3] = {0., 0., 0.}, bb[3] = {0., 0., 0.};
    add_prescribed_box(a, point, time + (s + .5) * h, ee, bb);
    double e[3], b[3];
    for (int d = 0; d < 3; ++d) {
      e[d] = used_e[d] + ee[d];
      b[d] = used_b[d] + bb[d];
    }
    const unsigned err = momentum(u, e, b, q, m, h, g0);
    if (err) return err;
    const double g1 = gamma_u(u[0], u[1], u[2]);
    const double xs = h * kC / (g0 + g1);
    for (int d = 0; d < 3; ++d) pos[d] += xs * (before_u[d] + u[d]);
    // |BorisWork::gridWork| of this substep (chargeWork, evaluated in
    // binary64 here; the reference keeps long double).
    double w = 0.0;
    for (int d = 0; d < 3; ++d) w += q * used_e[d] * (pos[d] - before_pos[d]);
    abs_work += fabs(w);
  }
  return kErrNone;
}

// Longitudinal-shape Current::deposit without the depositor's endpoint
// validation (src/longitudinal_shape.h:175-187): the upstream part of an
// admitted held particle and the frozen source support
// (src/source_coupling.cpp:73-78) deposit this way.
template <int S, bool Q, class F>
__device__ unsigned deposit_current(const GridT<F>& g, const double b[3],
                                    const double e[3], double charge) {
  DepositVisitor<F, Q> v;
  v.g = &g;
  v.smooth_x = S == 0;
  v.error = kErrNone;
  for (int a = 0; a < 3; ++a)
    v.scale[a] = F(charge * (e[a] - b[a]) / (g.dx * g.dy * g.dz * g.dt));
  if (shape_weights<S>(g, b, e, v) < 0) return kErrCrossingBudget;
  return v.error;
}

// Where the coupled push of one particle starts this step: prepareParticle
// with hold_transverse_until_activation (src/simulation.cpp:4919-5035).  An
// active particle is pushed from the step start over dt; a held particle
// advances along z at c*frozenBetaZ and, when its chord reaches the fixed lab
// activation plane, is released there and pushed over the rest of the step.
struct SlotPlan {
  double start[3];     // push start: the step start or the activation kink
  double time, dt;     // push time and duration
  double held_z;       // z after the held advance (held for the whole step)
  unsigned char seen;  // 0 no push, 1 push from the step start, 2 from the kink
  bool released;       // held at the step start, active at its end
  unsigned err;
};

template <class F>
__device__ __forceinline__ SlotPlan plan_slot(const GridT<F>& g, const DFrame& f, double plane,
                                              double t, const double start[3], bool frozen,
                                              double beta) {
  SlotPlan s;
  for (int d = 0; d < 3; ++d) s.start[d] = start[d];
  s.time = t;
  s.dt = g.dt;
  s.held_z = start[2];
  s.seen = 0;
  s.released = false;
  s.err = kErrNone;
  if (!frozen) {
    if (start[2] < g.origin[2]) s.err = kErrUpstream;
    else s.seen = 1;
    return s;
  }
  const double dt = g.dt;
  const double start_lab = lab_z_from_box_zt(f, start[2], t);
  s.held_z = start[2] + kC * dt * beta;
  const double end_lab = lab_z_from_box_zt(f, s.held_z, t + dt);
  if (!(end_lab >= plane)) return s;
  if (start[2] < g.origin[2]) {
    s.err = kErrEarlyRelease;
    return s;
  }
  const double crossing =
      start_lab >= plane ? 0.0 : fmax(0.0, fmin(1.0, (plane - start_lab) / (end_lab - start_lab)));
  s.start[2] = start[2] + kC * crossing * dt * beta;
  s.released = true;
  s.time = t + crossing * dt;
  s.dt = (1.0 - crossing) * dt;
  if (s.dt > 0.0) s.seen = 2;
  return s;
}

// First trial: the fields along each slot's ballistic guess chord
// (Impl::Slot::guess, src/source_coupling.cpp:92-95), gathered from E*
// before any current of the trial is deposited; the push reads them as the
// previous residual's fields.
template <class W, class F, int S>
__global__ void APRL_GATHER_BOUNDS guess_gather_kernel(PushArgs<F> a) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.count) return;
  const double start[3] = {a.p.x[n], a.p.y[n], a.p.z[n]};
  const bool frozen = a.p.frozen[n] != 0;
  const SlotPlan s = plan_slot(a.g, a.frame, a.activation_plane_lab_z, a.time, start, frozen,
                               frozen ? a.p.beta[n] : 0.0);
  if (s.err || !s.seen) return;  // the push reports the error
  const double u[3] = {a.p.ux[n], a.p.uy[n], a.p.uz[n]};
  const double gamma = gamma_u(u[0], u[1], u[2]);
  const double sc = s.dt * kC / gamma;
  const double guess[3] = {s.start[0] + sc * u[0], s.start[1] + sc * u[1],
                           s.start[2] + sc * u[2]};
  double ne[3], nb[3];
  const Ptr3<W> orbit{{static_cast<const W*>(a.orbit[0]), static_cast<const W*>(a.orbit[1]),
                       static_cast<const W*>(a.orbit[2])}};
  const Ptr3<W> bsrc{{static_cast<const W*>(a.bgather[0]), static_cast<const W*>(a.bgather[1]),
                      static_cast<const W*>(a.bgather[2])}};
  const unsigned err = gather_fields<S>(a.g, s.start, guess, orbit, bsrc, ne, nb);
  if (err) raise_error(a.status, err, (unsigned long long)n);
  double* next_e = const_cast<double*>(a.next_e);
  double* next_b = const_cast<double*>(a.next_b);
  for (int d = 0; d < 3; ++d) {
    next_e[3 * n + d] = ne[d];
    next_b[3 * n + d] = nb[d];
  }
}

// One fixed-point trial of one particle of the list: prepareParticle
// (src/simulation.cpp:4919-5035), then the deposit and boundary pass
// (src/simulation.cpp:5083-5368): upstream admission clip, the frozen part
// up to an activation kink (4684-4756) and processActiveSegment (4760-4917)
// with Simulation::firstMovingWindowEntry
// (src/simulation_moving_window.cpp:380-395).
template <class F, int S, bool Q>
__global__ void APRL_PUSH_BOUNDS push_deposit_kernel(PushArgs<F> a) {
  if (trial_skipped(a.g)) return;
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.count) return;
  const GridT<F>& g = a.g;
  const double t = a.time, dt = g.dt;
  double start[3] = {a.p.x[n], a.p.y[n], a.p.z[n]};
  double u[3] = {a.p.ux[n], a.p.uy[n], a.p.uz[n]};
  const double q = a.p.q[n], m = a.p.m[n];
  const bool frozen0 = a.p.frozen[n] != 0;
  const SlotPlan s = plan_slot(g, a.frame, a.activation_plane_lab_z, t, start, frozen0,
                               frozen0 ? a.p.beta[n] : 0.0);
  unsigned err = s.err;
  const bool frozen1 = frozen0 && !s.released;
  double pos[3] = {s.start[0], s.start[1], frozen1 ? s.held_z : s.start[2]};
  double used_e[3] = {0., 0., 0.}, used_b[3] = {0., 0., 0.};
  double abs_work = 0.0;
  if (!err && s.seen)
    err = coupling_push(a, n, pos, u, q, m, s.time, s.dt, used_e, used_b, abs_work);
  if (!err && s.released) atomicAdd(&a.counters->activations, 1ull);
  // An optional leading piece, then the main segment: the upstream part of
  // an admitted held particle (deposited without validation), or the frozen
  // part up to an activation kink (which may not cross a boundary).
  double seg_frac = 0.0;
  bool has_pre = false, pre_validate = false, has_main = true;
  double pre_end[3] = {pos[0], pos[1], pos[2]};
  double pre_start[3] = {start[0], start[1], start[2]};
  if (!err && start[2] < g.origin[2]) {
    if (!frozen0 || !frozen1) {
      err = kErrAdmission;
    } else if (pos[2] < g.origin[2]) {
      has_pre = true;
      has_main = false;
    } else {
      const double fraction = (g.origin[2] - start[2]) / (pos[2] - start[2]);
      if (!(fraction >= 0.0 && fraction <= 1.0) || !isfinite(fraction)) {
        err = kErrAdmission;
      } else {
        for (int d = 0; d < 3; ++d) pre_end[d] = start[d] + fraction * (pos[d] - start[d]);
        pre_end[2] = g.origin[2];
        has_pre = true;
        seg_frac = fraction;
        for (int d = 0; d < 3; ++d) start[d] = pre_end[d];
      }
    }
  } else if (!err && s.released && s.time > t && s.time < t + dt) {
    Hit hc, ho;
    bool enters = false, exits = false;
    err = cpml_first_entry(a.region, start, s.start, hc, enters);
    if (!err) err = outer_first_exit(a.region, start, s.start, ho, exits);
    if (!err && (enters || exits)) err = kErrHeldBoundary;
    for (int d = 0; d < 3; ++d) pre_end[d] = s.start[d];
    has_pre = true;
    pre_validate = true;
    for (int d = 0; d < 3; ++d) start[d] = s.start[d];
    seg_frac = (s.time - t) / dt;
  }
  unsigned char action = 0;
  bool deferred = false;
  Hit selected;
  for (int piece = has_pre ? 0 : 1; piece < (has_main ? 2 : 1) && !err; ++piece) {
    double b[3], e[3];
    bool validate = true;
    if (piece == 0) {
      for (int d = 0; d < 3; ++d) {
        b[d] = pre_start[d];
        e[d] = pre_end[d];
      }
      validate = pre_validate;
    } else {
      // firstMovingWindowEntry = CPML first entry + fixed-lab exit plane
      Hit cpml_hit, outer_hit;
      bool enters = false, exits = false;
      err = cpml_first_entry(a.region, start, pos, cpml_hit, enters);
      if (!err) {
        const double za = lab_z_from_box_zt(a.frame, start[2], t + seg_frac * dt) - a.exit_lab_z;
        const double zb = lab_z_from_box_zt(a.frame, pos[2], t + dt) - a.exit_lab_z;
        if (za >= 0.) err = kErrBeyondExit;
        else if (zb >= 0. && zb > za) {
          const double fraction = -za / (zb - za);
          if (!enters || fraction < cpml_hit.fraction) {
            for (int d = 0; d < 3; ++d) cpml_hit.position[d] = start[d] + fraction * (pos[d] - start[d]);
            cpml_hit.fraction = fraction;
            cpml_hit.face = 5;
            enters = true;
          }
        }
      }
      if (!err) err = outer_first_exit(a.region, start, pos, outer_hit, exits);
      if (err) break;
      if (enters && (!exits || cpml_hit.fraction <= outer_hit.fraction + 64.0 * kEpsilon)) {
        action = 1;
        selected = cpml_hit;
      } else if (exits) {
        action = 2;
        selected = outer_hit;
      }
      for (int d = 0; d < 3; ++d) {
        b[d] = start[d];
        e[d] = action ? selected.position[d] : pos[d];
      }
    }
    if constexpr (S == 0) {
      // The main chord of a linear-binomial3 particle is validated here and
      // deposited by chord_deposit_kernel, whose converged warps merge the
      // stencils of particles in the same cell before the reductions.
      if (piece == 1) {
        err = validate_segment(g, b, e, q);
        if (!err) {
          for (int d = 0; d < 3; ++d) {
            a.dep_b[d][n] = b[d];
            a.dep_e[d][n] = e[d];
          }
          deferred = true;
        }
        continue;
      }
    }
    err = validate ? deposit_segment<S, Q>(g, b, e, q) : deposit_current<S, Q>(g, b, e, q);
  }
  bool born_kept = false;
  CarrierState born;
  if (!err && has_main && action == 1) {
    if (selected.face == 5) {
      atomicAdd(&a.counters->exits, 1ull);
      atomicAdd(&a.counters->exit_charge, q);
    } else {
      atomicAdd(&a.counters->cpml[selected.face], 1ull);
      atomicAdd(&a.counters->cpml_charge[selected.face], q);
    }
    for (int d = 0; d < 3; ++d) born.pos[d] = pos[d];
    const double gamma = gamma_u(u[0], u[1], u[2]);
    const double sv = kC / gamma;
    for (int d = 0; d < 3; ++d) born.vel[d] = u[d] * sv;
    born.q = q;
    born.w = 1.0;
    const double global_end = seg_frac + selected.fraction * (1.0 - seg_frac);
    err = carrier_segment<S, Q>(g, a.region, born, selected.position, global_end, a.counters,
                          born_kept);
  } else if (!err && has_main && action == 2) {
    atomicAdd(&a.counters->direct[selected.face], 1ull);
    atomicAdd(&a.counters->direct_charge[selected.face], q);
  }
  if (err) raise_error(a.status, err, (unsigned long long)n);
  // Retained, held and newborn-carrier counts (one atomic per warp group).
  count_lanes(&a.counters->held, !err && action == 0 && frozen1);
  count_lanes(&a.counters->retained, action == 0);
  count_lanes(&a.counters->born_kept, born_kept);
  a.x1[n] = pos[0]; a.y1[n] = pos[1]; a.z1[n] = pos[2];
  a.ux1[n] = u[0]; a.uy1[n] = u[1]; a.uz1[n] = u[2];
  a.frozen1[n] = frozen1 ? 1 : 0;
  a.slot.seen[n] = s.seen;
  if (s.seen == 2) {
    a.slot.x0[n] = s.start[0];
    a.slot.y0[n] = s.start[1];
    a.slot.z0[n] = s.start[2];
    a.slot.dt[n] = s.dt;
  }
  for (int d = 0; d < 3; ++d) {
    a.used_e[3 * n + d] = used_e[d];
    a.used_b[3 * n + d] = used_b[d];
  }
  a.abs_grid_work[n] = abs_work;
  a.action[n] = action;
  if constexpr (S == 0) a.dep_mode[n] = deferred ? 1 : 0;
  a.born_keep[n] = born_kept ? 1 : 0;
  if (born_kept) {
    a.born.px[n] = born.pos[0]; a.born.py[n] = born.pos[1]; a.born.pz[n] = born.pos[2];
    a.born.vx[n] = born.vel[0]; a.born.vy[n] = born.vel[1]; a.born.vz[n] = born.vel[2];
    a.born.q[n] = born.q;
    a.born.w[n] = born.w;
    a.born.key[n] = a.key_base | (a.p.order[n] & 0xffffffffull);
  }
}

// ---------------------------------------------------------------------------
// The deposit of the main chords of linear-binomial3 particles
// (Current::deposit, src/longitudinal_shape.h:175-187, with the cut pieces of
// weights() and binomialXZSegment, :61-117), one thread per particle with the
// warp converged.  The warp walks the cut pieces of its lanes' chords in
// step: at each step every lane holds at most one piece, whose 4x2x4 node
// block is fixed by the piece's cell (i, j, k).  Particles are stored in cell
// order, so lanes holding pieces of the same cell sit side by side; such a
// run of lanes adds its 32 stencil weights (8 Jx, 16 Jy, 8 Jz products of
// the x, y and z factors; the edge smoothing [1/4, 1/2, 1/4] of Jx along x
// and of Jz along z is applied after the sum) with a segmented shuffle scan,
// and the run's last lane issues the 64 reductions for all of them.  A lone
// lane adds its own weights.  The weights are binomialXZSegment's; only the
// order of the floating-point additions into J differs from one reduction
// per particle and node.
// Inclusive sum of v over the lanes from `head` (the first lane of this
// lane's run) to this lane; `span` = the longest run in the warp.
__device__ __forceinline__ double run_sum(double v, int lane, int head, unsigned span) {
  for (unsigned d = 1; d < span; d <<= 1) {
    const double u = __shfl_up_sync(0xffffffffu, v, d);
    if (lane - (int)d >= head) v += u;
  }
  return v;
}

// The 4x2x4 node block of component `ax` around a piece in cell (i, j, k):
// nodes (i-1+x, j+b, k-1+c), with in-range masks per x, b and c.
struct ChordBlock {
  long long base, row, plane;
  unsigned xok, yok, zok;
  __device__ __forceinline__ bool in(int c, int b) const {
    return ((zok >> c) & 1u) && ((yok >> b) & 1u);
  }
  __device__ __forceinline__ size_t at(int c, int b, int x) const {
    return (size_t)(base + c * plane + b * row + x);
  }
};

// `levels`: z levels k-1 .. k-2+levels.
__device__ __forceinline__ ChordBlock chord_block(const DGrid& g, int ax, long long i,
                                                  long long j, long long k, int levels) {
  const long long nxc = e_nx(g, ax), nyc = e_ny(g, ax), nzc = e_nz(g, ax);
  ChordBlock s;
  s.row = nxc;
  s.plane = nxc * nyc;
  s.base = ((k - 1) * nyc + j) * nxc + (i - 1);
  s.xok = s.yok = s.zok = 0u;
#pragma unroll
  for (int x = 0; x < 4; ++x)
    if (i - 1 + x >= 0 && i - 1 + x < nxc) s.xok |= 1u << x;
#pragma unroll
  for (int b = 0; b < 2; ++b)
    if (j + b >= 0 && j + b < nyc) s.yok |= 1u << b;
#pragma unroll
  for (int c = 0; c < 5; ++c)
    if (c < levels && k - 1 + c >= 0 && k - 1 + c < nzc) s.zok |= 1u << c;
  return s;
}

template <bool Q>
__device__ __forceinline__ void chord_add(const DGrid& g, int a, size_t at, double v,
                                          unsigned& err) {
  if constexpr (Q) {
    if (!fixed_add(g.jq[a] + 2 * at, v, g.jq_scale)) err = kErrFixedRange;
  } else {
    atomicAdd(&g.j[a][at], v);
  }
}

// One cut piece's cell and binomialXZSegment factors.
struct PieceGeometry {
  long long i, j, k;
  double wx[4], wz[4], wy[2];
  double width, xy, xz, yz;
};

__device__ __forceinline__ void piece_geometry(const DGrid& g, const CutWalker& w, double first,
                                               double last, PieceGeometry& p) {
  p.width = last - first;
  const double mid = (first + last) * 0.5;
  const double px = w.x[0] + mid * w.v[0], py = w.x[1] + mid * w.v[1], pz = w.x[2] + mid * w.v[2];
  p.i = (long long)floor(px);
  p.j = (long long)floor(py);
  p.k = (long long)floor(pz);
  if (p.i == (long long)g.nx) --p.i;
  if (p.j == (long long)g.ny) --p.j;
  node_weights(px - p.i, p.wx);
  node_weights(pz - p.k, p.wz);
  p.wy[0] = 1. - (py - p.j);
  p.wy[1] = py - p.j;
  const double curvature = p.width * p.width / 12.;
  p.xy = curvature * w.v[0] * w.v[1];
  p.xz = curvature * w.v[0] * w.v[2];
  p.yz = curvature * w.v[1] * w.v[2];
}

__device__ __forceinline__ unsigned long long piece_key(long long i, long long j, long long k,
                                                        unsigned long long kind) {
  return (kind << 63) | ((unsigned long long)(k + 2) << 42) |
         ((unsigned long long)(j + 2) << 21) | (unsigned long long)(i + 2);
}

// Runs of neighbouring lanes holding the same key: this lane's run head,
// whether it is the run's last lane, and the longest run of the warp.
struct Runs {
  int head;
  bool last;
  unsigned span;
};

__device__ __forceinline__ Runs lane_runs(unsigned long long key, int lane) {
  const unsigned long long previous = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = lane == 0 || previous != key;
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  Runs r;
  r.head = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
  r.last = lane == 31 || ((heads >> (lane + 1)) & 1u) != 0u;
  r.span = __reduce_max_sync(0xffffffffu, (unsigned)(lane - r.head + 1));
  return r;
}

template <bool Q>
__global__ void APRL_CHORD_BOUNDS chord_deposit_kernel(ChordArgs a) {
  if (trial_skipped(a.g)) return;
  const DGrid& g = a.g;
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  bool alive = n < a.count && a.mode[n] != 0;
  unsigned err = kErrNone;
  double scale[3] = {0., 0., 0.};
  CutWalker w;
  w.done = true;
  if (alive) {
    double b[3], e[3];
    for (int d = 0; d < 3; ++d) {
      b[d] = a.b[d][n];
      e[d] = a.e[d][n];
    }
    const double q = a.q[n];
    for (int d = 0; d < 3; ++d) scale[d] = q * (e[d] - b[d]) / (g.dx * g.dy * g.dz * g.dt);
    const double h[3] = {g.dx, g.dy, g.dz};
    if (!w.init(b, e, g.origin, h)) {
      err = kErrCrossingBudget;
      alive = false;
    }
  }
  const double edge[3] = {0.25, 0.5, 0.25};
  const double slope[4] = {-0.25, -0.25, 0.25, 0.25};
  const double sy[2] = {-1., 1.};
  // ---- chords of exactly two pieces in z-neighbouring cells of one (i, j)
  // column (a chord crossing one z plane: nearly every chord of a beam that
  // moves about a cell per step along z).  Their stencils overlap, so the two
  // pieces are added per node of the union before the reductions: 82 nodes
  // instead of 2 x 64.
  double f0 = 0., l0 = 0., f1 = 0., l1 = 0.;
  bool pair = false;
  if (alive) {
    const bool two = w.advance(f0, l0) && w.advance(f1, l1);
    double fx, lx;
    if (two && !w.advance(fx, lx)) {
      PieceGeometry p0, p1;
      piece_geometry(g, w, f0, l0, p0);
      piece_geometry(g, w, f1, l1, p1);
      pair = p0.i == p1.i && p0.j == p1.j && (p1.k - p0.k == 1 || p0.k - p1.k == 1);
      if (pair && p1.k < p0.k) {  // lower piece first
        double t = f0; f0 = f1; f1 = t;
        t = l0; l0 = l1; l1 = t;
      }
    }
    if (!pair) {  // the general walk below starts over
      double b[3], e[3];
      for (int d = 0; d < 3; ++d) {
        b[d] = a.b[d][n];
        e[d] = a.e[d][n];
      }
      const double h[3] = {g.dx, g.dy, g.dz};
      w.init(b, e, g.origin, h);
    }
  }
  if (__any_sync(0xffffffffu, pair)) {
    PieceGeometry lo, up;
    unsigned long long key = ~0ull - (unsigned long long)lane;
    if (pair) {
      piece_geometry(g, w, f0, l0, lo);
      piece_geometry(g, w, f1, l1, up);
      key = piece_key(lo.i, lo.j, lo.k, 1);
    } else {
      lo = PieceGeometry{};
      up = PieceGeometry{};
    }
    const Runs runs = lane_runs(key, lane);
    const bool adds = pair && runs.last;
    const long long i = lo.i, j = lo.j, k = lo.k;
    // Node blocks of the union: z levels k-1 .. k+3 (Jx, Jy) and k-1 .. k+2 (Jz).
    const ChordBlock bx = chord_block(g, 0, i, j, k, 5), by = chord_block(g, 1, i, j, k, 5),
                     bz = chord_block(g, 2, i, j, k, 4);
    if (pair) {
      if (scale[0] != 0. && (bx.xok & 7u) && (bx.yok & 3u) != 3u) err = kErrSupportY;
      if (scale[1] != 0. && (by.xok & 15u) && !(by.yok & 1u)) err = kErrSupportY;
      if (scale[2] != 0. && (bz.xok & 15u) && (bz.yok & 3u) != 3u) err = kErrSupportY;
    }
    // Jx: level zz takes the lower piece's c = zz and the upper's c = zz - 1.
#pragma unroll
    for (int zz = 0; zz < 5; ++zz) {
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        double v = 0.;
        if (zz < 4) v += lo.width * (lo.wy[b] * lo.wz[zz] + lo.yz * sy[b] * slope[zz]);
        if (zz >= 1)
          v += up.width * (up.wy[b] * up.wz[zz - 1] + up.yz * sy[b] * slope[zz - 1]);
        const double total = run_sum(scale[0] * v, lane, runs.head, runs.span);
        if (adds && total != 0. && bx.in(zz, b))
#pragma unroll
          for (int x = 0; x < 3; ++x)
            if ((bx.xok >> x) & 1u) chord_add<Q>(g, 0, bx.at(zz, b, x), total * edge[x], err);
      }
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        double v = 0.;
        if (zz < 4) v += lo.width * (lo.wx[x] * lo.wz[zz] + lo.xz * slope[x] * slope[zz]);
        if (zz >= 1)
          v += up.width * (up.wx[x] * up.wz[zz - 1] + up.xz * slope[x] * slope[zz - 1]);
        const double total = run_sum(scale[1] * v, lane, runs.head, runs.span);
        if (adds && total != 0. && by.in(zz, 0) && ((by.xok >> x) & 1u))
          chord_add<Q>(g, 1, by.at(zz, 0, x), total, err);
      }
    }
    // Jz: each piece's weight is smoothed over three z nodes (its k-1, k,
    // k+1), so the lower piece covers levels 0..2 and the upper 1..3.
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const double vl = lo.width * (lo.wx[x] * lo.wy[b] + lo.xy * slope[x] * sy[b]);
        const double vu = up.width * (up.wx[x] * up.wy[b] + up.xy * slope[x] * sy[b]);
        const double tl = run_sum(scale[2] * vl, lane, runs.head, runs.span);
        const double tu = run_sum(scale[2] * vu, lane, runs.head, runs.span);
        if (adds && ((bz.xok >> x) & 1u) && ((bz.yok >> b) & 1u)) {
          const double level[4] = {tl * edge[0], tl * edge[1] + tu * edge[0],
                                   tl * edge[2] + tu * edge[1], tu * edge[2]};
#pragma unroll
          for (int zz = 0; zz < 4; ++zz)
            if (((bz.zok >> zz) & 1u) && level[zz] != 0.)
              chord_add<Q>(g, 2, bz.at(zz, b, x), level[zz], err);
        }
      }
  }
  if (pair) alive = false;
  // ---- every other chord, one piece per lane per round
  while (__any_sync(0xffffffffu, alive)) {
    double first = 0., last = 0.;
    const bool have = alive && w.advance(first, last);
    if (!have) alive = false;
    // A lane without a piece takes a key no other lane has and adds nothing.
    PieceGeometry p;
    unsigned long long key = ~0ull - (unsigned long long)lane;
    if (have) {
      piece_geometry(g, w, first, last, p);
      key = piece_key(p.i, p.j, p.k, 0);
    } else {
      p = PieceGeometry{};
    }
    const Runs runs = lane_runs(key, lane);
    const bool adds = have && runs.last;
    const long long i = p.i, j = p.j, k = p.k;
    // The three node blocks of the piece, with the visitor's support rules
    // for this lane: x outside is skipped (the F3 x-support may leave the
    // grid), y outside is an error when the lane carries current on that
    // axis, z outside is skipped.  The run's sums are added by its last lane.
    const ChordBlock bx = chord_block(g, 0, i, j, k, 4), by = chord_block(g, 1, i, j, k, 4),
                     bz = chord_block(g, 2, i, j, k, 4);
    if (have) {
      if (scale[0] != 0. && (bx.xok & 7u) && (bx.yok & 3u) != 3u) err = kErrSupportY;
      if (scale[1] != 0. && (by.xok & 15u) && !(by.yok & 1u)) err = kErrSupportY;
      if (scale[2] != 0. && (bz.xok & 15u) && (bz.yok & 3u) != 3u) err = kErrSupportY;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const double weight = p.width * (p.wy[b] * p.wz[c] + p.yz * sy[b] * slope[c]);
        const double total = run_sum(scale[0] * weight, lane, runs.head, runs.span);
        if (adds && total != 0. && bx.in(c, b))
#pragma unroll
          for (int x = 0; x < 3; ++x)
            if ((bx.xok >> x) & 1u) chord_add<Q>(g, 0, bx.at(c, b, x), total * edge[x], err);
      }
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const double weight = p.width * (p.wx[x] * p.wz[c] + p.xz * slope[x] * slope[c]);
        const double total = run_sum(scale[1] * weight, lane, runs.head, runs.span);
        if (adds && total != 0. && by.in(c, 0) && ((by.xok >> x) & 1u))
          chord_add<Q>(g, 1, by.at(c, 0, x), total, err);
      }
    }
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const double weight = p.width * (p.wx[x] * p.wy[b] + p.xy * slope[x] * sy[b]);
        const double total = run_sum(scale[2] * weight, lane, runs.head, runs.span);
        if (adds && total != 0. && ((bz.xok >> x) & 1u) && ((bz.yok >> b) & 1u))
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if ((bz.zok >> c) & 1u) chord_add<Q>(g, 2, bz.at(c, b, x), total * edge[c], err);
      }
  }
  if (err) raise_error(a.status, err, (unsigned long long)n);
}

// ---------------------------------------------------------------------------
// RelativisticBorisPusher::push (src/eb_particles.cpp:207-216): the Boris
// momentum update with the half electric kicks and the magnetic rotation
// (pushMomentum, :99-127), then the drift at the new proper velocity
// (pushPosition, :129-136), in the reference's operation order.
__device__ __forceinline__ void boris_push(double x[3], double u[3], const double e[3],
                                           const double b[3], double q, double m, double dt) {
  const double kick = q * dt / (2.0 * m * kC);
  double minus[3];
  for (int d = 0; d < 3; ++d) minus[d] = u[d] + kick * e[d];
  const double gamma_minus = gamma_u(minus[0], minus[1], minus[2]);
  const double rs = q * dt / (2.0 * m * gamma_minus);
  const double t[3] = {rs * b[0], rs * b[1], rs * b[2]};
  double prime[3] = {minus[1] * t[2] - minus[2] * t[1], minus[2] * t[0] - minus[0] * t[2],
                     minus[0] * t[1] - minus[1] * t[0]};
  for (int d = 0; d < 3; ++d) prime[d] += minus[d];
  const double norm2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  const double f = 2.0 / (1.0 + norm2);
  const double sv[3] = {t[0] * f, t[1] * f, t[2] * f};
  double plus[3] = {prime[1] * sv[2] - prime[2] * sv[1], prime[2] * sv[0] - prime[0] * sv[2],
                    prime[0] * sv[1] - prime[1] * sv[0]};
  for (int d = 0; d < 3; ++d) plus[d] += minus[d];
  for (int d = 0; d < 3; ++d) u[d] = plus[d] + kick * e[d];
  const double gamma = gamma_u(u[0], u[1], u[2]);
  const double drift = kC * dt / gamma;
  for (int d = 0; d < 3; ++d) x[d] += drift * u[d];
}

__global__ void boris_push_kernel(BorisArgs a) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.count) return;
  double x[3] = {a.x[n], a.y[n], a.z[n]}, u[3] = {a.ux[n], a.uy[n], a.uz[n]};
  const double e[3] = {a.e[3 * n], a.e[3 * n + 1], a.e[3 * n + 2]};
  const double b[3] = {a.b[3 * n], a.b[3 * n + 1], a.b[3 * n + 2]};
  boris_push(x, u, e, b, a.q[n], a.m[n], a.dt);
  a.x[n] = x[0]; a.y[n] = x[1]; a.z[n] = x[2];
  a.ux[n] = u[0]; a.uy[n] = u[1]; a.uz[n] = u[2];
}

// ---------------------------------------------------------------------------
// ConservativeSourceCoupling::localResidual (src/source_coupling.cpp:105-159):
// re-gather along the actual chord, then force = max, defect and scale =
// sums.  Block reduction with warp shuffles, one atomic per block.
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <class W, class F, int S>
__global__ void APRL_RESIDUAL_BOUNDS residual_kernel(ResidualArgs<F> a) {
  if (trial_skipped(a.g)) return;
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double force = 0.0, defect = 0.0, scale = 0.0;
  const unsigned char seen = n < a.count ? a.slot.seen[n] : 0;
  if (seen) {
    // Slot start: the step start, or the activation kink of a held
    // particle released during the step (seen == 2).
    double first[3], dt = a.g.dt;
    if (seen == 2) {
      first[0] = a.slot.x0[n]; first[1] = a.slot.y0[n]; first[2] = a.slot.z0[n];
      dt = a.slot.dt[n];
    } else {
      first[0] = a.p.x[n]; first[1] = a.p.y[n]; first[2] = a.p.z[n];
    }
    const double last[3] = {a.x1[n], a.y1[n], a.z1[n]};
    double ne[3], nb[3];
    const Ptr3<W> orbit{{static_cast<const W*>(a.orbit[0]),
                         static_cast<const W*>(a.orbit[1]),
                         static_cast<const W*>(a.orbit[2])}};
    const Ptr3<W> bsrc{{static_cast<const W*>(a.bgather[0]),
                        static_cast<const W*>(a.bgather[1]),
                        static_cast<const W*>(a.bgather[2])}};
    const unsigned err = gather_fields<S>(a.g, first, last, orbit, bsrc, ne, nb);
    if (err) {
      raise_error(a.status, err, (unsigned long long)n);
      for (int d = 0; d < 3; ++d) ne[d] = nb[d] = 0.0;
    }
    // The trial's reads, issued together before the first store (which may
    // alias them as far as the compiler knows).
    double used_e[3], used_b[3];
    for (int d = 0; d < 3; ++d) {
      used_e[d] = a.used_e[3 * n + d];
      used_b[d] = a.used_b[3 * n + d];
    }
    const double q = a.p.q[n], m = a.p.m[n], abs_work = a.abs_grid_work[n];
    double de[3], db[3];
    for (int d = 0; d < 3; ++d) {
      a.next_e[3 * n + d] = ne[d];
      a.next_b[3 * n + d] = nb[d];
      de[d] = ne[d] - used_e[d];
      db[d] = nb[d] - used_b[d];
    }
    force = fabs(q / m) * dt / kC *
            (sqrt(de[0] * de[0] + de[1] * de[1] + de[2] * de[2]) +
             kC * sqrt(db[0] * db[0] + db[1] * db[1] + db[2] * db[2]));
    double wd = 0.0, wn = 0.0;
    for (int d = 0; d < 3; ++d) {
      wd += q * de[d] * (last[d] - first[d]);
      wn += q * ne[d] * (last[d] - first[d]);
    }
    defect = fabs(wd);
    scale = abs_work + fabs(wn);
  }
  __shared__ unsigned s_calls[32];
  const unsigned calls = __popc(__ballot_sync(0xffffffffu, seen != 0));
  __shared__ double s_force[32], s_defect[32], s_scale[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  force = warp_max(force);
  defect = warp_sum(defect);
  scale = warp_sum(scale);
  if (lane == 0) {
    s_force[warp] = force;
    s_defect[warp] = defect;
    s_scale[warp] = scale;
    s_calls[warp] = calls;
  }
  __syncthreads();
  if (warp == 0) {
    const int warps = blockDim.x >> 5;
    force = lane < warps ? s_force[lane] : 0.0;
    defect = lane < warps ? s_defect[lane] : 0.0;
    scale = lane < warps ? s_scale[lane] : 0.0;
    unsigned block_calls = lane < warps ? s_calls[lane] : 0u;
    force = warp_max(force);
    defect = warp_sum(defect);
    scale = warp_sum(scale);
    for (int o = 16; o > 0; o >>= 1) block_calls += __shfl_xor_sync(0xffffffffu, block_calls, o);
    if (lane == 0) {
      atomicMax(&a.sums->force_bits, (unsigned long long)__double_as_longlong(force));
      if (block_calls) atomicAdd(&a.sums->calls, (unsigned long long)block_calls);
      a.partial[2 * blockIdx.x] = defect;
      a.partial[2 * blockIdx.x + 1] = scale;
    }
  }
  // The defect and scale sums in a fixed order: the last block to finish
  // adds the block partials (thread t takes blocks t, t + 128, ... in turn,
  // then a fixed shuffle tree), so the sums do not depend on which blocks
  // finished first.
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  defect = 0.0;
  scale = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    defect += __ldcg(&a.partial[2 * b]);
    scale += __ldcg(&a.partial[2 * b + 1]);
  }
  defect = warp_sum(defect);
  scale = warp_sum(scale);
  __syncthreads();
  if (lane == 0) {
    s_defect[warp] = defect;
    s_scale[warp] = scale;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double d = 0.0, c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      d += s_defect[w];
      c += s_scale[w];
    }
    a.sums->defect = d;
    a.sums->scale = c;
    *a.ticket = 0u;
  }
}

// ---------------------------------------------------------------------------
// Stable compaction: the retained list keeps the reference's push_back
// order (src/simulation.cpp:4916, 5581).
__global__ void flag_count_kernel(const unsigned char* flag, unsigned char want, long long n,
                                  unsigned* block_count) {
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  const bool f = i < n && flag[i] == want;
  const unsigned ballot = __ballot_sync(0xffffffffu, f);
  __shared__ unsigned warp_count[kScanBlock / 32];
  if ((threadIdx.x & 31) == 0) warp_count[threadIdx.x >> 5] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned s = 0;
    for (int w = 0; w < kScanBlock / 32; ++w) s += warp_count[w];
    block_count[blockIdx.x] = s;
  }
}

// Exclusive scan of the per-block counts by one block of 1024 threads.
__global__ void block_offset_scan_kernel(const unsigned* block_count, int blocks,
                                         unsigned* block_offset,
                                         unsigned long long* total) {
  __shared__ unsigned partial[1024];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < blocks; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned v = i < blocks ? block_count[i] : 0u;
    partial[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const unsigned add = threadIdx.x >= off ? partial[threadIdx.x - off] : 0u;
      __syncthreads();
      partial[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < blocks) block_offset[i] = (unsigned)(carry + partial[threadIdx.x] - v);
    __syncthreads();
    if (threadIdx.x == 1023) carry += partial[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__device__ __forceinline__ long long compact_slot(const unsigned char* flag, unsigned char want,
                                                  long long n, const unsigned* block_offset,
                                                  bool& selected) {
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  selected = i < n && flag[i] == want;
  const unsigned ballot = __ballot_sync(0xffffffffu, selected);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ unsigned warp_base[kScanBlock / 32];
  if (lane == 0) warp_base[warp] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned s = 0;
    for (int w = 0; w < kScanBlock / 32; ++w) {
      const unsigned c = warp_base[w];
      warp_base[w] = s;
      s += c;
    }
  }
  __syncthreads();
  return (long long)block_offset[blockIdx.x] + warp_base[warp] +
         __popc(ballot & ((1u << lane) - 1u));
}

__global__ void gather_particles_kernel(DParticles out, DParticles src, const double* x1,
                                        const double* y1, const double* z1,
                                        const double* ux1, const double* uy1,
                                        const double* uz1, const unsigned char* frozen1,
                                        const unsigned char* flag, unsigned char want,
                                        long long n, const unsigned* block_offset) {
  bool selected;
  const long long slot = compact_slot(flag, want, n, block_offset, selected);
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  if (!selected) return;
  // Every read before the first store (which may alias them as far as the
  // compiler knows), so the reads' latencies overlap.
  const double x = x1[i], y = y1[i], z = z1[i], ux = ux1[i], uy = uy1[i], uz = uz1[i];
  const double q = src.q[i], m = src.m[i], beta = src.beta[i];
  const unsigned long long id = src.id[i], order = src.order[i];
  const unsigned char frozen = frozen1[i];
  out.x[slot] = x; out.y[slot] = y; out.z[slot] = z;
  out.ux[slot] = ux; out.uy[slot] = uy; out.uz[slot] = uz;
  out.q[slot] = q;
  out.m[slot] = m;
  out.id[slot] = id;
  out.order[slot] = order;
  out.frozen[slot] = frozen;
  out.beta[slot] = beta;
}

__global__ void gather_carriers_kernel(DCarriers out, DCarriers src, const unsigned char* flag,
                                       unsigned char want, long long n,
                                       const unsigned* block_offset,
                                       unsigned long long base) {
  bool selected;
  const long long slot = compact_slot(flag, want, n, block_offset, selected) + (long long)base;
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  if (!selected) return;
  const double px = src.px[i], py = src.py[i], pz = src.pz[i];
  const double vx = src.vx[i], vy = src.vy[i], vz = src.vz[i];
  const double q = src.q[i], w = src.w[i];
  const unsigned long long key = src.key[i];
  out.px[slot] = px; out.py[slot] = py; out.pz[slot] = pz;
  out.vx[slot] = vx; out.vy[slot] = vy; out.vz[slot] = vz;
  out.q[slot] = q;
  out.w[slot] = w;
  out.key[slot] = key;
}

// ---------------------------------------------------------------------------
// Cell sort: particles of one cell become contiguous, in cell order (x
// fastest), so the 4x2x4 F3 stencils of a warp overlap in L1 instead of
// scattering over HBM.  A stable least-significant-digit radix sort of the
// cell index (8-bit digits): the order of particles within a cell is their
// previous storage order, so the permutation -- and every block reduction
// over the particle list -- is the same from run to run.
__global__ void sort_key_kernel(DParticles p, long long n, DGrid g, int tiles_x, int tiles_y,
                                unsigned* key, unsigned* index) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double lx = (p.x[i] - g.origin[0]) / g.dx;
  const double ly = (p.y[i] - g.origin[1]) / g.dy;
  const double lz = (p.z[i] - g.origin[2]) / g.dz;
  const int cx = (int)fmin(fmax(floor(lx), 0.0), (double)(g.nx - 1));
  const int cy = (int)fmin(fmax(floor(ly), 0.0), (double)(g.ny - 1));
  const int cz = (int)fmin(fmax(floor(lz), 0.0), (double)(g.nz - 1));
  key[i] = (unsigned)((((cz >> kTileShift) * tiles_y) + (cy >> kTileShift)) * tiles_x +
                      (cx >> kTileShift));
  index[i] = (unsigned)i;
}

// Digit counts of each block's kRadixTile keys: count[digit * blocks + block].
__global__ void __launch_bounds__(kRadixThreads) radix_count_kernel(const unsigned* key,
                                                                    long long n, int shift,
                                                                    unsigned* count) {
  __shared__ unsigned c[kRadixBins];
  c[threadIdx.x] = 0u;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixItems; ++r) {
    const long long i = base + r * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(&c[(key[i] >> shift) & (kRadixBins - 1)], 1u);
  }
  __syncthreads();
  count[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = c[threadIdx.x];
}

// Stable scatter of one digit pass.  offset[digit * blocks + block] is the
// exclusive scan of radix_count_kernel's counts in that digit-major order.
// A block walks its keys in index order, 256 at a time; within a round a
// key's rank among equal digits is its warp's lanes below it (match_any)
// plus the equal digits of the warps before it and of the earlier rounds.
__global__ void __launch_bounds__(kRadixThreads) radix_scatter_kernel(
    const unsigned* key_in, const unsigned* index_in, unsigned* key_out, unsigned* index_out,
    long long n, int shift, const unsigned* offset) {
  constexpr int kWarps = kRadixThreads / 32;
  __shared__ unsigned running[kRadixBins];
  __shared__ unsigned warp_count[kWarps][kRadixBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  running[threadIdx.x] = offset[(size_t)threadIdx.x * gridDim.x + blockIdx.x];
  const long long base = (long long)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixItems; ++r) {
    const long long i = base + r * kRadixThreads + threadIdx.x;
    const bool valid = i < n;
    const unsigned k = valid ? key_in[i] : 0u;
    const unsigned digit = valid ? (k >> shift) & (kRadixBins - 1) : kRadixBins;
    for (int w = 0; w < kWarps; ++w) warp_count[w][threadIdx.x] = 0u;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const unsigned rank = __popc(peers & below);
    if (valid && rank == 0) warp_count[warp][digit] = __popc(peers);
    __syncthreads();
    {  // per digit: exclusive prefix over the warps, then advance the running base
      unsigned at = running[threadIdx.x];
      for (int w = 0; w < kWarps; ++w) {
        const unsigned c = warp_count[w][threadIdx.x];
        warp_count[w][threadIdx.x] = at;
        at += c;
      }
      running[threadIdx.x] = at;
    }
    __syncthreads();
    if (valid) {
      const unsigned d = warp_count[warp][digit] + rank;
      key_out[d] = k;
      index_out[d] = index_in[i];
    }
    __syncthreads();
  }
}

// The storage permutation: out[d] = src[index[d]].
__global__ void permute_particles_kernel(DParticles out, DParticles src, long long n,
                                         const unsigned* index) {
  const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  const long long i = index[d];
  // Every read before the first store, as in gather_particles_kernel.
  const double x = src.x[i], y = src.y[i], z = src.z[i];
  const double ux = src.ux[i], uy = src.uy[i], uz = src.uz[i];
  const double q = src.q[i], m = src.m[i], beta = src.beta[i];
  const unsigned long long id = src.id[i], order = src.order[i];
  const unsigned char frozen = src.frozen[i];
  out.x[d] = x; out.y[d] = y; out.z[d] = z;
  out.ux[d] = ux; out.uy[d] = uy; out.uz[d] = uz;
  out.q[d] = q;
  out.m[d] = m;
  out.id[d] = id;
  out.order[d] = order;
  out.frozen[d] = frozen;
  out.beta[d] = beta;
}

// Exclusive scan of 1024-element chunks; chunk totals go to chunk_sum.
__global__ void chunk_scan_kernel(const unsigned* in, long long n, unsigned* out,
                                  unsigned* chunk_sum) {
  __shared__ unsigned part[1024];
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  const unsigned v = i < n ? in[i] : 0u;
  part[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const unsigned add = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  if (i < n) out[i] = part[threadIdx.x] - v;
  if (threadIdx.x == 1023) chunk_sum[blockIdx.x] = part[1023];
}

__global__ void chunk_add_kernel(unsigned* data, long long n, const unsigned* chunk_offset) {
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) data[i] += chunk_offset[blockIdx.x];
}

// PendingParticleQueue::admit (src/pending_particle_queue.cpp:163-186): the
// queue entries [begin, begin+count) join the end of the list with their
// held z advanced by `steps` separately rounded additions of
// (c*dt)*frozenBetaZ.
__global__ void admit_kernel(DParticles out, long long first_slot, DPending src,
                             long long begin, long long count, unsigned long long steps,
                             double held_distance_per_beta, unsigned long long first_order) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const long long k = begin + i, d = first_slot + i;
  const double beta = src.beta[k];
  out.x[d] = src.x[k];
  out.y[d] = src.y[k];
  out.z[d] = repeat_held_addition(src.z[k], held_distance_per_beta * beta, steps);
  out.ux[d] = src.ux[k]; out.uy[d] = src.uy[k]; out.uz[d] = src.uz[k];
  out.q[d] = src.q[k];
  out.m[d] = src.m[k];
  out.id[d] = src.id[k];
  out.order[d] = first_order + (unsigned long long)i;
  out.frozen[d] = 1;
  out.beta[d] = beta;
}

// Frozen source support of the queue entries due within the next steps
// (PendingParticleQueue::visitNear + depositFrozenSourceSupport,
// src/simulation.cpp:4170-4172, src/source_coupling.cpp:73-78): each
// deposits its held chord of this step without endpoint validation.
template <class F, int S, bool Q>
__global__ void frozen_support_kernel(SupportArgs<F> a) {
  if (trial_skipped(a.g)) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.count) return;
  const long long k = a.begin + i;
  const double beta = a.src.beta[k];
  const double increment = a.held_distance_per_beta * beta;
  const double start[3] = {a.src.x[k], a.src.y[k],
                           repeat_held_addition(a.src.z[k], increment, a.steps)};
  const double stop[3] = {start[0], start[1], start[2] + increment};
  const unsigned err = deposit_current<S, Q>(a.g, start, stop, a.src.q[k]);
  if (err) raise_error(a.status, err, (unsigned long long)k);
}

// finishMovingWindowStep carrier crop (src/simulation_moving_window.cpp:363-368).
__global__ void crop_flags_kernel(DCarriers c, long long n, double upper, double lower,
                                  unsigned char* keep, TrialCounters* counters,
                                  DeviceStatus* status) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double z = c.pz[i];
  unsigned char k = 1;
  if (z >= upper) {
    k = 0;
    atomicAdd(&counters->cropped, 1ull);
    atomicAdd(&counters->cropped_charge, c.q[i] * c.w[i]);
  } else if (z < lower) {
    raise_error(status, kErrFellBehind, (unsigned long long)i);
  }
  keep[i] = k;
}

// migrateWindowObjects' inlet guard (src/simulation_moving_window.cpp:355-358).
__global__ void inlet_check_kernel(const double* z, const unsigned char* frozen, long long n,
                                   double origin, DeviceStatus* status) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && z[i] < origin && !frozen[i])
    raise_error(status, kErrFellBehind, (unsigned long long)i);
}

__global__ void inlet_charge_kernel(InletMatchArgs a) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.np + a.pcount) return;
  double pos[3], q;
  long long where;
  if (n < a.np) {
    pos[0] = a.p.x[n];
    pos[1] = a.p.y[n];
    pos[2] = a.p.z[n];
    q = a.p.q[n];
    where = n;
  } else {
    const long long k = a.pbegin + (n - a.np);
    pos[0] = a.src.x[k];
    pos[1] = a.src.y[k];
    pos[2] = repeat_held_addition(a.src.z[k], a.held_distance_per_beta * a.src.beta[k], a.steps);
    q = a.src.q[k];
    where = k;
  }
  // longitudinal_shape::nodeWeight(z, 1, shape) (src/longitudinal_shape.h:25-56)
  const double z = (pos[2] - a.origin[2]) / a.dz;
  double wz = 0.;
  if (a.shape == 0) {
    const double cell = floor(z), f = z - cell;
    double v[4] = {0., 0., 0., 0.};
    const double c[3] = {.25, .5, .25};
    for (int k = -1; k <= 1; ++k) {
      v[k + 1] += c[k + 1] * (1. - f);
      v[k + 2] += c[k + 1] * f;
    }
    const long long first = (long long)cell - 1;
    if (1 >= first && 1 < first + 4) wz = v[1 - first];
  } else {
    Basis<double> b;
    quintic_basis<double>(z, false, b);
    if (1 >= b.first && 1 < b.first + b.count) wz = b.v[1 - b.first];
  }
  if (wz == 0.) return;
  const double x = (pos[0] - a.origin[0]) / a.dx, y = (pos[1] - a.origin[1]) / a.dy;
  if (!isfinite(x) || !isfinite(y) || !isfinite(z) || !isfinite(q)) {
    raise_error(a.status, kErrInletSource, (unsigned long long)where);
    return;
  }
  const bool binomial3 = a.shape == 0;
  if (y < 0. || y > (double)a.ny) return;
  if (binomial3 ? (x <= -2. || x >= (double)a.nx + 2.) : (x < 0. || x > (double)a.nx)) return;
  const long long ix = (long long)floor(x);
  const long long j = (long long)floor(y);
  const double fx = x - ix, fy = y - j, scale = q * (1. / (a.dx * a.dy * a.dz));
  double wx[4] = {1. - fx, fx, 0., 0.};
  if (binomial3) node_weights(fx, wx);
  const int n_x = binomial3 ? 4 : 2;
  const long long first = ix - (binomial3 ? 1 : 0);
  for (int b = 0; b < 2; ++b)
    for (int c = 0; c < n_x; ++c) {
      const long long i = first + c;
      if (i >= 0 && i <= a.nx && j + b <= a.ny) {
        const size_t at = (size_t)(j + b) * (a.nx + 1) + (size_t)i;
        const double v = scale * wx[c] * (b ? fy : 1. - fy) * wz;
        if (a.rho_pairs == nullptr)
          atomicAdd(&a.rho[at], v);
        else if (!fixed_add(a.rho_pairs + 2 * at, v, a.rho_scale))
          raise_error(a.status, kErrFixedRange, (unsigned long long)where);
      }
    }
}

__global__ void trial_clear_kernel(GridT<double> g, TrialCounters* counters, ResidualSums* sums,
                                   int clear_current) {
  if (trial_skipped(g)) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (int c = 0; c < 3 && clear_current; ++c) {
    const long long count = (long long)e_nx(g, c) * e_ny(g, c) * e_nz(g, c);
    if (clear_current == 2) {
      ulonglong2* pairs = reinterpret_cast<ulonglong2*>(g.jq[c]);
      for (long long n = first; n < count; n += stride) pairs[n] = make_ulonglong2(0ull, 0ull);
    } else {
      for (long long n = first; n < count; n += stride) g.j[c][n] = 0.;
    }
  }
  if (first == 0) {
    *counters = TrialCounters{};
    *sums = ResidualSums{};
  }
}

__global__ void current_convert_kernel(GridT<double> g, double unscale) {
  if (trial_skipped(g)) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (int c = 0; c < 3; ++c) {
    const long long count = (long long)e_nx(g, c) * e_ny(g, c) * e_nz(g, c);
    const ulonglong2* pairs = reinterpret_cast<const ulonglong2*>(g.jq[c]);
    for (long long n = first; n < count; n += stride) {
      const ulonglong2 v = pairs[n];
      g.j[c][n] = (v.x | v.y) ? fixed_value(v.x, v.y, unscale) : 0.;
    }
  }
}

__global__ void fixed_convert_kernel(const unsigned long long* pairs, double* out, long long n,
                                     double unscale) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long lo = pairs[2 * i], hi = pairs[2 * i + 1];
  out[i] = (lo | hi) ? fixed_value(lo, hi, unscale) : 0.;
}

__global__ void trial_verdict_kernel(const ResidualSums* sums, unsigned iterations,
                                     double force_tolerance, double work_tolerance, int* stop) {
  if (*stop) return;
  const double force = __longlong_as_double((long long)sums->force_bits);
  const double calls = (double)sums->calls;
  const double work =
      calls == 0. ? 0. : (sums->scale > 0. ? sums->defect / sums->scale : sums->defect);
  if (iterations >= (calls > 0. ? 2u : 1u) && force < force_tolerance && work < work_tolerance)
    *stop = (int)iterations;
}

// The grid and J are binary64 in every mode; the gathers are built with
// binary64 (FP64 drop-in) and binary32 (FP32-mixed) arithmetic.
// Each particle kernel is built once per shape (S = 0 linear-binomial3,
// 1 quintic-compensated), so a kernel carries the registers and local
// memory of its own shape's weights only.
#define APRL_SHAPE_KERNELS(S)                                                        \
  template __global__ void push_deposit_kernel<double, S, false>(PushArgs<double>);  \
  template __global__ void push_deposit_kernel<double, S, true>(PushArgs<double>);   \
  template __global__ void carrier_kernel<double, S, false>(CarrierArgs<double>);    \
  template __global__ void carrier_kernel<double, S, true>(CarrierArgs<double>);     \
  template __global__ void frozen_support_kernel<double, S, false>(SupportArgs<double>); \
  template __global__ void frozen_support_kernel<double, S, true>(SupportArgs<double>); \
  template __global__ void guess_gather_kernel<double, double, S>(PushArgs<double>); \
  template __global__ void guess_gather_kernel<float, double, S>(PushArgs<double>);  \
  template __global__ void residual_kernel<double, double, S>(ResidualArgs<double>); \
  template __global__ void residual_kernel<float, double, S>(ResidualArgs<double>);
APRL_SHAPE_KERNELS(0)
APRL_SHAPE_KERNELS(1)
template __global__ void chord_deposit_kernel<false>(ChordArgs);
template __global__ void chord_deposit_kernel<true>(ChordArgs);
#undef APRL_SHAPE_KERNELS

}  // namespace aprl_gpu
