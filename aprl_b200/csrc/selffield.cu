// selffield.cu -- kernels of the initial self-field solve (selffield.cuh).
#include "selffield.cuh"

namespace aprl_gpu {

namespace {

__device__ DD sf_block_sum(DD v, DD* shared) {
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  shared[t] = v;
  __syncthreads();
  for (int s = kSelfFieldThreads / 2; s > 0; s >>= 1) {
    if (t < s) shared[t] = dd_add(shared[t], shared[t + s]);
    __syncthreads();
  }
  const DD out = shared[0];
  __syncthreads();
  return out;
}

// positiveLightFrontComponent, properVelocityFromPositiveLightFront and
// heldLongitudinalBetaZ (src/boostframe.cpp:89-167).
__device__ __forceinline__ double sf_positive(double u0, double u1, double u2) {
  const double gamma = gamma_u(u0, u1, u2);
  const double tms = fma(u0, u0, fma(u1, u1, 1.0));
  if (u2 >= 0.0) return gamma + u2;
  return tms / (gamma - u2);
}
__device__ __forceinline__ double sf_longitudinal(double u0, double u1, double positive) {
  const double tms = fma(u0, u0, fma(u1, u1, 1.0));
  const double negative = tms / positive;
  return 0.5 * (positive - negative);
}
__device__ __forceinline__ double sf_held_beta_z(double u0, double u1, double u2,
                                                 double rapidity) {
  const double lab = sf_longitudinal(u0, u1, sf_positive(u0, u1, u2) * rapidity);
  const double box = sf_longitudinal(0.0, 0.0, sf_positive(0.0, 0.0, lab) / rapidity);
  return box / hypot(1.0, box);
}

__device__ __forceinline__ size_t sf_at(const SfLattice& L, int i, int j, int p) {
  return ((size_t)p * L.ly + j) * L.lx + i;
}

__device__ __forceinline__ bool sf_stopped(const SfArgs& a) { return a.state->done != 0; }

// The interior vertices of this block's tile: (i, j) and planes [p0, p1].
struct SfTile {
  int i, j, p0, p1;
  bool column;  // (i, j) is an interior column
};
__device__ __forceinline__ SfTile sf_tile(const SfArgs& a) {
  const SfLattice& L = a.L;
  SfTile t;
  t.i = blockIdx.x * kSfTileX + threadIdx.x;
  t.j = blockIdx.y * kSfTileY + threadIdx.y;
  t.column = t.i > L.lo[0] && t.i < L.hi[0] && t.j > L.lo[1] && t.j < L.hi[1];
  // planes p = k + 1 with k in (lo2, hi2)
  t.p0 = max(L.lo[2] + 2, 1 + (int)blockIdx.z * a.chunk);
  t.p1 = min(L.hi[2], (int)(blockIdx.z + 1) * a.chunk);
  return t;
}
__device__ __forceinline__ int sf_block_index() {
  return (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
}
__device__ __forceinline__ bool sf_first_thread() { return threadIdx.x == 0 && threadIdx.y == 0; }

// Called by every thread of a block after its first thread has stored the
// block's partial: true in the one block of the launch that arrives last,
// when every block's partial is in memory (each first thread fences its
// store before it counts itself).  That block resets the count for the next
// launch.  No block waits on another.
__device__ __forceinline__ bool sf_last_block(const SfArgs& a) {
  __shared__ int last;
  if (sf_first_thread()) {
    __threadfence();
    const unsigned blocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned before = atomicAdd(&a.state->arrivals, 1u);
    last = before == blocks - 1;
    if (last) a.state->arrivals = 0;
  }
  __syncthreads();
  return last != 0;
}

// The sum of the launch's per-block partials in a fixed order (thread t adds
// partials t, t + 128, ..., then the block tree), read through L2 since other
// blocks of this launch wrote them.
__device__ DD sf_partials_sum(const SfArgs& a, DD* shared) {
  const int blocks = (int)(gridDim.x * gridDim.y * gridDim.z);
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  const double* words = reinterpret_cast<const double*>(a.partial);
  DD s{0., 0.};
  for (int b = t; b < blocks; b += kSelfFieldThreads)
    s = dd_add(s, DD{__ldcg(words + 2 * b), __ldcg(words + 2 * b + 1)});
  return sf_block_sum(s, shared);
}

}  // namespace

// Host helpers.
double sf_ratio(DD a, DD b) { return dd_value(dd_div_dd(a, b)); }
long double sf_long(DD a) { return (long double)a.hi + (long double)a.lo; }

// Per-block partial moments of the particles: mass, mass * beta (x, y, z;
// or the held longitudinal beta_z), mass * position, mass * position^2,
// charge (meanVelocity and distributionResolution,
// src/eb_initial_field.cpp:629-741, and the total charge).
__global__ void __launch_bounds__(kSelfFieldThreads) sf_moments_kernel(SfParticles p, DD* partial) {
  __shared__ DD shared[kSelfFieldThreads];
  DD m[kMoments];
  for (int q = 0; q < kMoments; ++q) m[q] = DD{0., 0.};
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < p.n;
       n += (long long)gridDim.x * blockDim.x) {
    const double w = p.m[n];
    const double u0 = p.ux[n], u1 = p.uy[n], u2 = p.uz[n];
    m[0] = dd_add(m[0], DD{w, 0.});
    if (p.hold) {
      m[3] = dd_add(m[3], two_prod(w, sf_held_beta_z(u0, u1, u2, p.rapidity)));
    } else {
      const double gamma = gamma_u(u0, u1, u2);
      m[1] = dd_add(m[1], two_prod(w, u0 / gamma));
      m[2] = dd_add(m[2], two_prod(w, u1 / gamma));
      m[3] = dd_add(m[3], two_prod(w, u2 / gamma));
    }
    const double x[3] = {p.x[n], p.y[n], p.z[n]};
    for (int a = 0; a < 3; ++a) {
      const DD wx = two_prod(w, x[a]);
      m[4 + a] = dd_add(m[4 + a], wx);
      m[7 + a] = dd_add(m[7 + a], dd_mul(wx, x[a]));
    }
    m[10] = dd_add(m[10], DD{p.q[n], 0.});
  }
  for (int q = 0; q < kMoments; ++q) {
    const DD s = sf_block_sum(m[q], shared);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * kMoments + q] = s;
  }
}

// One block: the partials of `quantities` sums, in block order.
__global__ void __launch_bounds__(kSelfFieldThreads) sf_finish_kernel(const DD* partial, int blocks,
                                                                     int quantities, DD* out) {
  __shared__ DD shared[kSelfFieldThreads];
  for (int q = 0; q < quantities; ++q) {
    DD s{0., 0.};
    for (int b = threadIdx.x; b < blocks; b += kSelfFieldThreads)
      s = dd_add(s, partial[(size_t)b * quantities + q]);
    s = sf_block_sum(s, shared);
    if (threadIdx.x == 0) out[q] = s;
  }
}

// ChargeConservingCurrentDepositor::depositCharge (src/eb_deposition.cpp:168-193,
// validatePosition 228-246, normalize 250-262, containingCell 264-279) into a
// lattice lx nodes wide with the Maxwell grid's vertices at offset `pad`.
__global__ void sf_deposit_kernel(SfParticles p, DGrid g, double* rho, int lx, int ly, int pad,
                                  DeviceStatus* status) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.n) return;
  const double pos[3] = {p.x[n], p.y[n], p.z[n]};
  const double h[3] = {g.dx, g.dy, g.dz};
  const int cells[3] = {g.nx, g.ny, g.nz};
  const double extent[3] = {(double)g.nx * g.dx, (double)g.ny * g.dy, (double)g.nz * g.dz};
  int c[3];
  double f[3];
  for (int a = 0; a < 3; ++a) {
    const double relative = pos[a] - g.origin[a];
    const double tol = 64.0 * kEpsilon * fmax(1.0, fmax(fabs(g.origin[a]), extent[a]));
    if (!isfinite(pos[a]) || relative < -tol || relative > extent[a] + tol) {
      raise_error(status, kErrDepositOutside, (unsigned long long)n);
      return;
    }
    const double x = fmax(0.0, fmin((double)cells[a], (pos[a] - g.origin[a]) / h[a]));
    c[a] = x <= 0.0 ? 0 : (x >= (double)cells[a] ? cells[a] - 1 : (int)floor(x));
    f[a] = fmax(0.0, fmin(1.0, x - (double)c[a]));
  }
  const double inverse_volume = 1.0 / (g.dx * g.dy * g.dz);
  for (int cz = 0; cz < 2; ++cz)
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        const double sa = a ? f[0] : 1.0 - f[0];
        const double sb = b ? f[1] : 1.0 - f[1];
        const double sc = cz ? f[2] : 1.0 - f[2];
        atomicAdd(&rho[((size_t)(c[2] + cz) * ly + (c[1] + b + pad)) * lx + (c[0] + a + pad)],
                  p.q[n] * inverse_volume * sa * sb * sc);
      }
}

// BlockedCowanReference::depositQuintic (src/blocked_cowan_reference.cpp:
// 559-592): the shaped source with which the moving window prepares its
// reference (the mesh shape, src/simulation_moving_window.cpp:145-148).  Per
// particle x = (p - origin)/h; for linear-binomial3 the binomial3
// transverse x weights over nodes floor(x)-1 .. floor(x)+2
// (src/transverse_source_shape.h:8-10) and the binomial3 node basis in z,
// for quintic-compensated linear x weights and the quintic node basis; y is
// linear.  Each nonzero contribution ((q/(dx dy dz)) wx) wy wz must land on
// an interior node of L's zero-potential box, else the reference's
// "Reference charge support touches Dirichlet surface".  Binary64 atomics:
// the same terms as the reference's serial sum, in another order.
__global__ void sf_shaped_deposit_kernel(SfParticles p, DGrid g, double* rho, int lx, int ly,
                                         SfLattice L, int binomial, DeviceStatus* status) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.n) return;
  const double q = p.q[n];
  if (!isfinite(q)) {
    raise_error(status, kErrReferenceCharge, (unsigned long long)n);
    return;
  }
  const double x = (p.x[n] - g.origin[0]) / g.dx, y = (p.y[n] - g.origin[1]) / g.dy,
               z = (p.z[n] - g.origin[2]) / g.dz;
  if (!isfinite(z)) {
    raise_error(status, kErrReferenceSource, (unsigned long long)n);
    return;
  }
  if (!isfinite(x) || !isfinite(y)) {  // no node of such a support is interior
    raise_error(status, kErrReferenceSupport, (unsigned long long)n);
    return;
  }
  const double cx = floor(x), cy = floor(y);
  const long long ix = (long long)cx, iy = (long long)cy;
  const double fx = x - cx, fy = y - cy, scale = q / (g.dx * g.dy * g.dz);
  double wz[12];
  long long zfirst;
  int zcount;
  if (binomial) {
    // basis(z, false, LinearBinomial3) (src/longitudinal_shape.h:26-36)
    const double cell = floor(z), f = z - cell;
    const double c3[3] = {0.25, 0.5, 0.25};
    for (int t = 0; t < 4; ++t) wz[t] = 0.0;
    for (int s = 0; s < 3; ++s) {
      wz[s] += c3[s] * (1.0 - f);
      wz[s + 1] += c3[s] * f;
    }
    zfirst = (long long)cell - 1;
    zcount = 4;
  } else {
    Basis<double> b;
    quintic_basis<double>(z, false, b);
    for (int t = 0; t < 12; ++t) wz[t] = b.v[t];
    zfirst = b.first;
    zcount = b.count;
  }
  double wx[4] = {1.0 - fx, fx, 0.0, 0.0};
  if (binomial) {
    wx[0] = 0.25 * (1.0 - fx);
    wx[1] = 0.5 - 0.25 * fx;
    wx[2] = 0.25 + 0.25 * fx;
    wx[3] = 0.25 * fx;
  }
  const long long xfirst = ix - (binomial ? 1 : 0);
  const int xcount = binomial ? 4 : 2;
  for (int c = 0; c < zcount; ++c) {
    const long long k = zfirst + c;
    if (wz[c] == 0.0) continue;
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < xcount; ++i) {
        const double value = scale * wx[i] * (j ? fy : 1.0 - fy) * wz[c];
        if (value == 0.0) continue;
        const long long nx = xfirst + i, ny = iy + j;
        if (!(nx > L.lo[0] && nx < L.hi[0] && ny > L.lo[1] && ny < L.hi[1] && k > L.lo[2] &&
              k < L.hi[2])) {
          raise_error(status, kErrReferenceSupport, (unsigned long long)n);
          return;
        }
        atomicAdd(&rho[((size_t)k * ly + (size_t)ny) * lx + (size_t)nx], value);
      }
  }
}

// The Poisson source rho/eps0 at the interior vertices (into the residual
// and the first direction), with partial sums of the interior charge and of
// the source norm (src/eb_initial_field.cpp:991-1027).
__global__ void __launch_bounds__(kSelfFieldThreads) sf_source_kernel(SfArgs a, DD volume) {
  __shared__ DD shared[kSelfFieldThreads];
  const SfLattice& L = a.L;
  const SfTile t = sf_tile(a);
  DD charge{0., 0.}, source{0., 0.};
  if (t.column)
    for (int p = t.p0; p <= t.p1; ++p) {
      const double q = a.rho[((size_t)(p - 1) * L.ly + t.j) * L.lx + t.i];
      const double v = q / kEpsilon0;
      a.residual[sf_at(L, t.i, t.j, p)] = v;
      a.direction[sf_at(L, t.i, t.j, p)] = v;
      charge = dd_add(charge, dd_mul(volume, q));
      source = dd_add(source, two_prod(v, v));
    }
  charge = sf_block_sum(charge, shared);
  source = sf_block_sum(source, shared);
  if (sf_first_thread()) {
    a.partial[2 * sf_block_index()] = charge;
    a.partial[2 * sf_block_index() + 1] = source;
  }
}

// image = A direction at the interior vertices: the 7-point relativistic
// operator (applyNegativeLaplacian, src/eb_initial_field.cpp:210-236) or the
// 27-point Cowan one (applyNegativeCowanLaplacian, :318-342; its 27-term sum
// in the reference's order, each term a fused multiply-add, which halves the
// kernel's FP64 instructions and moves each sum by at most a rounding per
// term); partial sums of direction . image.
__global__ void __launch_bounds__(kSelfFieldThreads) sf_apply_kernel(SfArgs a) {
  __shared__ DD shared[kSelfFieldThreads];
  if (sf_stopped(a)) return;
  const SfLattice& L = a.L;
  const SfTile t = sf_tile(a);
  const int i = t.i, j = t.j;
  DD dot{0., 0.};
  if (t.column)
    for (int p = t.p0; p <= t.p1; ++p) {
      const double* d = a.direction;
      double value;
      if (a.cowan) {
        value = 0.0;
#pragma unroll
        for (int z = 0; z < 3; ++z)
#pragma unroll
          for (int y = 0; y < 3; ++y)
#pragma unroll
            for (int x = 0; x < 3; ++x)
              value = fma(a.stencil[(z * 3 + y) * 3 + x],
                          d[sf_at(L, i - 1 + x, j - 1 + y, p - 1 + z)], value);
      } else {
        value = a.diagonal * d[sf_at(L, i, j, p)] -
                a.cx * (d[sf_at(L, i - 1, j, p)] + d[sf_at(L, i + 1, j, p)]) -
                a.cy * (d[sf_at(L, i, j - 1, p)] + d[sf_at(L, i, j + 1, p)]) -
                a.cz * (d[sf_at(L, i, j, p - 1)] + d[sf_at(L, i, j, p + 1)]);
      }
      a.image[sf_at(L, i, j, p)] = value;
      dot = dd_add(dot, two_prod(d[sf_at(L, i, j, p)], value));
    }
  dot = sf_block_sum(dot, shared);
  if (sf_first_thread()) a.partial[sf_block_index()] = dot;
  if (!sf_last_block(a)) return;
  // The last block: alpha = |r|^2 / (d . A d), rounded once to binary64.
  const DD s = sf_partials_sum(a, shared);
  if (!sf_first_thread()) return;
  SfState& st = *a.state;
  st.denominator = s;
  if (!(s.hi > 0.) || !isfinite(s.hi)) {
    st.done = 2;
    return;
  }
  st.alpha = dd_value(dd_div_dd(st.rr, s));
}

// potential += alpha d, residual += (-alpha) A d at the interior vertices
// (updateInterior, src/eb_initial_field.cpp:405-421); partial sums of |r|^2.
__global__ void __launch_bounds__(kSelfFieldThreads) sf_update_kernel(SfArgs a) {
  __shared__ DD shared[kSelfFieldThreads];
  if (sf_stopped(a)) return;
  const SfLattice& L = a.L;
  const SfTile t = sf_tile(a);
  const double alpha = a.state->alpha;
  DD dot{0., 0.};
  if (t.column)
    for (int p = t.p0; p <= t.p1; ++p) {
      const size_t at = sf_at(L, t.i, t.j, p);
      a.potential[at] += alpha * a.direction[at];
      const double r = a.residual[at] + -alpha * a.image[at];
      a.residual[at] = r;
      dot = dd_add(dot, two_prod(r, r));
    }
  dot = sf_block_sum(dot, shared);
  if (sf_first_thread()) a.partial[sf_block_index()] = dot;
  if (!sf_last_block(a)) return;
  // The last block: the relative residual, the stopping test and beta
  // (src/eb_initial_field.cpp:1046-1064).
  const DD s = sf_partials_sum(a, shared);
  if (!sf_first_thread()) return;
  SfState& st = *a.state;
  st.next = s;
  st.iterations += 1;
  st.relative = dd_value(dd_sqrt(dd_div_dd(s, st.source)));
  if (st.relative <= a.tolerance) {
    st.rr = s;
    st.done = 1;
    return;
  }
  if (!(s.hi >= 0.) || !isfinite(s.hi)) {
    st.done = 3;
    return;
  }
  st.beta = dd_value(dd_div_dd(s, st.rr));
  st.rr = s;
}

// direction = r + beta direction at the interior vertices
// (combineDirection, src/eb_initial_field.cpp:423-438); the other vertices
// of the direction are zero from the start and stay zero.
__global__ void sf_direction_kernel(SfArgs a) {
  if (sf_stopped(a)) return;
  const SfLattice& L = a.L;
  const SfTile t = sf_tile(a);
  const double beta = a.state->beta;
  if (t.column)
    for (int p = t.p0; p <= t.p1; ++p) {
      const size_t at = sf_at(L, t.i, t.j, p);
      a.direction[at] = a.residual[at] + beta * a.direction[at];
    }
}

// The Cowan-smoothed potential of one axis minus the translation term, at
// the interior vertices, into `image` (cowanSmoothedPotential and
// fieldsFromCowanPotential, src/eb_initial_field.cpp:344-382, 503-517).
__global__ void sf_smooth_kernel(SfArgs a, int axis) {
  const SfLattice& L = a.L;
  const int ta = (axis + 1) % 3, tb = (axis + 2) % 3;
  const SfTile t = sf_tile(a);
  if (!t.column) return;
  for (int p = t.p0; p <= t.p1; ++p) {
    const int i = t.i, j = t.j;
    const double* phi = a.potential;
    double value = a.alpha[axis] * phi[sf_at(L, i, j, p)];
    for (int sign = -1; sign <= 1; sign += 2) {
      int pa[3] = {i, j, p}, pb[3] = {i, j, p};
      pa[ta] += sign;
      pb[tb] += sign;
      value += a.beta[ta] * phi[sf_at(L, pa[0], pa[1], pa[2])];
      value += a.beta[tb] * phi[sf_at(L, pb[0], pb[1], pb[2])];
    }
    for (int s = -1; s <= 1; s += 2)
      for (int u = -1; u <= 1; u += 2) {
        int pt[3] = {i, j, p};
        pt[ta] += s;
        pt[tb] += u;
        value += a.delta[axis] * phi[sf_at(L, pt[0], pt[1], pt[2])];
      }
    a.image[sf_at(L, i, j, p)] =
        value - (axis == 2 ? a.translation * phi[sf_at(L, i, j, p)] : 0.0);
  }
}

// ---- the open-transverse-wall reference ----------------------------------
// OpenTransverseTrace::at (src/open_transverse_trace.h:52-58): zero on the
// longitudinal end planes; a point with x on or outside a face in x reads
// that face's row (corners included), else the face in y.
__device__ __forceinline__ double open_at(const SfOpenSide& s, int i, int j, int k) {
  if (k <= 0 || k >= s.nz) return 0.0;
  const int tx = i <= 0 ? i + 1 : (i >= s.nx ? i - s.nx + 2 : -1);
  if (tx >= 0) return s.values[(long long)k * s.width + tx * (s.ny + 3) + j + 1];
  const int ty = j <= 0 ? j + 1 : j - s.ny + 2;
  return s.values[(long long)k * s.width + 4 * (s.ny + 3) + ty * (s.nx + 3) + i + 1];
}

// OpenTransverseTrace::Sources::potential (src/open_transverse_trace.h:25-34)
// at each target: a block per target, its threads over the sources, then a
// block sum (another summation order than the reference's loop).
__global__ void __launch_bounds__(256) sf_coulomb_kernel(const double* tx, const double* ty,
                                                         const double* tz, long long targets,
                                                         const double* sx, const double* sy,
                                                         const double* sz, const double* sq,
                                                         long long sources, double* out) {
  __shared__ double warp_sums[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long t = blockIdx.x; t < targets; t += gridDim.x) {
    const double x = tx[t], y = ty[t], z = tz[t];
    double sum = 0.0;
    for (long long s = threadIdx.x; s < sources; s += blockDim.x) {
      const double dx = x - sx[s], dy = y - sy[s], dz = z - sz[s];
      sum += sq[s] / sqrt(dx * dx + dy * dy + dz * dz);
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) warp_sums[warp] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      double total = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += warp_sums[w];
      out[t] = total;
    }
    __syncthreads();
  }
}

// BlockedCowanReference::liftOpenSides (src/blocked_cowan_reference.cpp:
// 694-706) on the compact interior array of the modal solve (x fastest,
// vertices lo+1 .. hi-1 with the transverse lo = 0): each node next to a
// face subtracts the sum of the elliptic stencil's weights times the face
// potentials it reaches, summed over dz, dy, dx as the reference does.
__global__ void sf_open_lift_kernel(SfArgs a, SfOpenSide side, double* rhs, int ix, int iy,
                                    int iz) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (long long)ix * iy * iz) return;
  const SfLattice& L = a.L;
  const int i = L.lo[0] + 1 + (int)(n % ix), j = L.lo[1] + 1 + (int)((n / ix) % iy),
            k = L.lo[2] + 1 + (int)(n / ((long long)ix * iy));
  if (!(i == 1 || i == side.nx - 1 || j == 1 || j == side.ny - 1)) return;
  double value = 0.0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int x = i + dx, y = j + dy;
        if (x == 0 || x == side.nx || y == 0 || y == side.ny)
          value += a.stencil[(dz + 1) * 9 + (dy + 1) * 3 + dx + 1] * open_at(side, x, y, k + dz);
      }
  rhs[n] -= value;
}

// The face node m of a plane: x faces first (j = 0 .. ny at i = 0, then at
// i = nx), then the y faces' inner nodes (i = 1 .. nx-1 at j = 0, then ny).
__device__ __forceinline__ void open_face_node(const SfOpenSide& s, int m, int& i, int& j) {
  if (m < 2 * (s.ny + 1)) {
    i = m < s.ny + 1 ? 0 : s.nx;
    j = m % (s.ny + 1);
  } else {
    m -= 2 * (s.ny + 1);
    j = m < s.nx - 1 ? 0 : s.ny;
    i = 1 + m % (s.nx - 1);
  }
}

// The face potentials of planes 1 .. nz-1 into the potential lattice
// (ensureField's phi fill, src/blocked_cowan_reference.cpp:872-877).
__global__ void sf_open_wall_fill_kernel(SfArgs a, SfOpenSide side) {
  const int per = 2 * (side.ny + 1) + 2 * (side.nx - 1);
  const long long count = (long long)per * (side.nz - 1);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int k = 1 + (int)(n / per);
    int i, j;
    open_face_node(side, (int)(n % per), i, j);
    a.potential[sf_at(a.L, i, j, k + 1)] = open_at(side, i, j, k);
  }
}

// smoothOnWall (src/blocked_cowan_reference.cpp:842-858) at the face nodes of
// planes 1 .. nz-1: the nine transverse-plane terms in the reference's order
// (a outer, b inner), the face table for every point on or outside a face,
// minus the translation term on the longitudinal axis.
__global__ void sf_open_wall_smooth_kernel(SfArgs a, SfOpenSide side, int axis) {
  const int ta = (axis + 1) % 3, tb = (axis + 2) % 3;
  const int per = 2 * (side.ny + 1) + 2 * (side.nx - 1);
  const long long count = (long long)per * (side.nz - 1);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int k = 1 + (int)(n / per);
    int i, j;
    open_face_node(side, (int)(n % per), i, j);
    double value = 0.0;
    for (int u = -1; u <= 1; ++u)
      for (int v = -1; v <= 1; ++v) {
        int d[3] = {0, 0, 0};
        d[ta] = u;
        d[tb] = v;
        const int x = i + d[0], y = j + d[1], z = k + d[2];
        const double p = (x <= 0 || y <= 0 || x >= side.nx || y >= side.ny)
                             ? open_at(side, x, y, z)
                             : a.potential[sf_at(a.L, x, y, z + 1)];
        const double w = u == 0 ? (v == 0 ? a.alpha[axis] : a.beta[tb])
                                : (v == 0 ? a.beta[ta] : a.delta[axis]);
        value += w * p;
      }
    a.image[sf_at(a.L, i, j, k + 1)] =
        value - (axis == 2 ? a.translation * open_at(side, i, j, k) : 0.0);
  }
}

// One E component from the potential (or its smoothed form) by a forward
// difference, E = -(coefficient * difference) / spacing
// (fieldsFromPotential and fieldsFromCowanPotential,
// src/eb_initial_field.cpp:427-449, 518-527), into the run's E.
__global__ void sf_electric_kernel(SfArgs a, int axis, double coefficient, int from_smoothed) {
  const DGrid& g = a.g;
  const SfLattice& L = a.L;
  const int nxc = e_nx(g, axis), nyc = e_ny(g, axis), nzc = e_nz(g, axis);
  const long long count = (long long)nxc * nyc * nzc;
  const double* s = from_smoothed ? a.image : a.potential;
  const double h = axis == 0 ? g.dx : (axis == 1 ? g.dy : g.dz);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % nxc);
    const int j = (int)((n / nxc) % nyc);
    const int k = (int)(n / ((long long)nxc * nyc));
    const double upper = s[sf_at(L, i + L.pad + (axis == 0), j + L.pad + (axis == 1),
                                 k + 1 + (axis == 2))];
    const double lower = s[sf_at(L, i + L.pad, j + L.pad, k + 1)];
    g.e_old[axis][e_index(g, axis, i, j, k)] = -coefficient * (upper - lower) / h;
  }
}

// B at the half step from E of the rigidly translating charge
// (src/eb_initial_field.cpp:451-484, 529-552).
__global__ void sf_magnetic_kernel(SfArgs a, double scale, double lower_w, double upper_w) {
  const DGrid& g = a.g;
  const long long per = (long long)(g.nx + 1) * (g.ny + 1) * g.nz;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < per;
       n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % (g.nx + 1));
    const int j = (int)((n / (g.nx + 1)) % (g.ny + 1));
    const int k = (int)(n / ((long long)(g.nx + 1) * (g.ny + 1)));
    if (j < g.ny)  // Bx (nx+1, ny, nz)
      g.b[0][b_index(g, 0, i, j, k)] =
          -scale * (lower_w * g.e_old[1][e_index(g, 1, i, j, k)] +
                    upper_w * g.e_old[1][e_index(g, 1, i, j, k + 1)]);
    if (i < g.nx)  // By (nx, ny+1, nz)
      g.b[1][b_index(g, 1, i, j, k)] =
          scale * (lower_w * g.e_old[0][e_index(g, 0, i, j, k)] +
                   upper_w * g.e_old[0][e_index(g, 0, i, j, k + 1)]);
  }
  const long long bz = (long long)g.nx * g.ny * (g.nz + 1);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < bz;
       n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nx);
    const int j = (int)((n / g.nx) % g.ny);
    const int k = (int)(n / ((long long)g.nx * g.ny));
    g.b[2][b_index(g, 2, i, j, k)] = 0.0;
  }
}

// clearComponentOutsidePhysical (src/eb_initial_field.cpp:564-607) for
// component 0..5 (Ex Ey Ez Bx By Bz).
__global__ void sf_clear_outside_kernel(SfArgs a, int component, int gx, int gy, int gz) {
  const DGrid& g = a.g;
  const bool electric = component < 3;
  const int axis = component % 3;
  const int n3[3] = {electric ? e_nx(g, axis) : b_nx(g, axis),
                     electric ? e_ny(g, axis) : b_ny(g, axis),
                     electric ? e_nz(g, axis) : b_nz(g, axis)};
  const int cells[3] = {g.nx, g.ny, g.nz};
  const int guard[3] = {gx, gy, gz};
  const long long count = (long long)n3[0] * n3[1] * n3[2];
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int c[3] = {(int)(n % n3[0]), (int)((n / n3[0]) % n3[1]),
                      (int)(n / ((long long)n3[0] * n3[1]))};
    bool inside = true;
    for (int d = 0; d < 3; ++d) {
      const bool vertex = electric ? d != axis : d == axis;
      inside = inside && c[d] >= guard[d] &&
               (vertex ? c[d] <= cells[d] - guard[d] : c[d] < cells[d] - guard[d]);
    }
    if (inside) continue;
    if (electric)
      g.e_old[axis][e_index(g, axis, c[0], c[1], c[2])] = 0.0;
    else
      g.b[axis][b_index(g, axis, c[0], c[1], c[2])] = 0.0;
  }
}

// validateGauss (src/eb_initial_field.cpp:743-806): partial sums of the
// squared Gauss error and source over the physical interior vertices, and
// their largest error.
__global__ void __launch_bounds__(kSelfFieldThreads)
sf_gauss_kernel(SfArgs a, const double* rho, int plo0, int phi0, int plo1, int phi1, int plo2,
                int phi2, unsigned long long* max_bits) {
  __shared__ DD shared[kSelfFieldThreads];
  const DGrid& g = a.g;
  const int vx = g.nx + 1, vy = g.ny + 1;
  const long long count = (long long)vx * vy * g.nz;
  DD res{0., 0.}, src{0., 0.};
  double worst = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % vx);
    const int j = (int)((n / vx) % vy);
    const int k = (int)(n / ((long long)vx * vy));
    if (!(k > plo2 && k < phi2 && j > plo1 && j < phi1 && i > plo0 && i < phi0)) continue;
    const double left_z = k > 0 ? g.e_old[2][e_index(g, 2, i, j, k - 1)] : 0.0;
    const double divergence =
        (g.e_old[0][e_index(g, 0, i, j, k)] - g.e_old[0][e_index(g, 0, i - 1, j, k)]) / g.dx +
        (g.e_old[1][e_index(g, 1, i, j, k)] - g.e_old[1][e_index(g, 1, i, j - 1, k)]) / g.dy +
        (g.e_old[2][e_index(g, 2, i, j, k)] - left_z) / g.dz;
    const double source = rho[((size_t)k * vy + j) * vx + i] / kEpsilon0;
    const double error = divergence - source;
    res = dd_add(res, two_prod(error, error));
    src = dd_add(src, two_prod(source, source));
    worst = fmax(worst, fabs(error));
  }
  res = sf_block_sum(res, shared);
  src = sf_block_sum(src, shared);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = res;
    a.partial[2 * blockIdx.x + 1] = src;
  }
  if (worst > 0.) atomicMax(max_bits, (unsigned long long)__double_as_longlong(worst));
}

// initialFieldEnergy (src/eb_initial_field.cpp:665-691): partial sums of
// the electric and magnetic energies over the cells; `volume` carries the
// factors 0.5 eps0 dV (hi, lo) and the magnetic factor 0.5 dV / mu0 is
// passed in a.stencil[0..1].
__global__ void __launch_bounds__(kSelfFieldThreads) sf_energy_kernel(SfArgs a, DD volume) {
  __shared__ DD shared[kSelfFieldThreads];
  const DGrid& g = a.g;
  const DD magnetic_factor{a.stencil[0], a.stencil[1]};
  const long long count = (long long)g.nx * g.ny * g.nz;
  DD we{0., 0.}, wm{0., 0.};
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nx);
    const int j = (int)((n / g.nx) % g.ny);
    const int k = (int)(n / ((long long)g.nx * g.ny));
    const double* ex = g.e_old[0];
    const double* ey = g.e_old[1];
    const double* ez = g.e_old[2];
    const double e0 = 0.25 * (((ex[e_index(g, 0, i, j, k)] + ex[e_index(g, 0, i, j + 1, k)]) +
                               ex[e_index(g, 0, i, j, k + 1)]) + ex[e_index(g, 0, i, j + 1, k + 1)]);
    const double e1 = 0.25 * (((ey[e_index(g, 1, i, j, k)] + ey[e_index(g, 1, i + 1, j, k)]) +
                               ey[e_index(g, 1, i, j, k + 1)]) + ey[e_index(g, 1, i + 1, j, k + 1)]);
    const double e2 = 0.25 * (((ez[e_index(g, 2, i, j, k)] + ez[e_index(g, 2, i + 1, j, k)]) +
                               ez[e_index(g, 2, i, j + 1, k)]) + ez[e_index(g, 2, i + 1, j + 1, k)]);
    const double m0 = 0.5 * (g.b[0][b_index(g, 0, i, j, k)] + g.b[0][b_index(g, 0, i + 1, j, k)]);
    const double m1 = 0.5 * (g.b[1][b_index(g, 1, i, j, k)] + g.b[1][b_index(g, 1, i, j + 1, k)]);
    const double m2 = 0.5 * (g.b[2][b_index(g, 2, i, j, k)] + g.b[2][b_index(g, 2, i, j, k + 1)]);
    const double en = (e0 * e0 + e1 * e1) + e2 * e2;
    const double bn = (m0 * m0 + m1 * m1) + m2 * m2;
    we = dd_add(we, dd_mul(volume, en));
    wm = dd_add(wm, dd_mul(magnetic_factor, bn));
  }
  we = sf_block_sum(we, shared);
  wm = sf_block_sum(wm, shared);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = we;
    a.partial[2 * blockIdx.x + 1] = wm;
  }
}

}  // namespace aprl_gpu

namespace aprl_gpu {

// ---------------------------------------------------------------------------
// The transverse-mode (modal) direct solve of the same discrete operator on
// the same Dirichlet box: the method of the reference's blocked Cowan
// reference (src/blocked_cowan_reference.h:59-130), which expands the
// potential in the sine modes of the transverse Dirichlet problem and solves
// one tridiagonal system along z per mode.  The 7-point and 27-point
// operators have constant coefficients and are even in x and in y, so the
// type-I sine transform along x and along y diagonalises them: mode (m, n)
// sees the z stencil lambda_c = sum over (dy, dx) of st[c][dy][dx] *
// C_x(dx) * C_y(dy), C(0) = 1, C(+-1) = cos(pi (m+1) / (N+1)).  Transforms
// are dense sums against a sine table (the interior is at most a few
// hundred nodes across), in binary64 with fused multiply-adds.
//
// Compact interior layout: index (k * Iy + j) * Ix + i.

__global__ void sf_modal_gather_kernel(SfArgs a, double* out, int ix, int iy, int iz) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (long long)ix * iy * iz) return;
  const int i = (int)(n % ix), j = (int)((n / ix) % iy), k = (int)(n / ((long long)ix * iy));
  const SfLattice& L = a.L;
  out[n] = a.residual[sf_at(L, L.lo[0] + 1 + i, L.lo[1] + 1 + j, L.lo[2] + 2 + k)];
}

__global__ void sf_modal_scatter_kernel(SfArgs a, const double* in, int ix, int iy, int iz) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (long long)ix * iy * iz) return;
  const int i = (int)(n % ix), j = (int)((n / ix) % iy), k = (int)(n / ((long long)ix * iy));
  const SfLattice& L = a.L;
  a.potential[sf_at(L, L.lo[0] + 1 + i, L.lo[1] + 1 + j, L.lo[2] + 2 + k)] = in[n];
}

// out = scale * S in along x (axis 0) or y (axis 1), S[m][t] = table[m * len + t].
__global__ void sf_modal_transform_kernel(const double* in, double* out, const double* table,
                                          int axis, int ix, int iy, int iz, double scale) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (long long)ix * iy * iz) return;
  const int i = (int)(n % ix), j = (int)((n / ix) % iy);
  const long long plane = n / ((long long)ix * iy) * ((long long)ix * iy);
  double v = 0.0;
  if (axis == 0) {
    const double* line = in + plane + (long long)j * ix;
    const double* row = table + (long long)i * ix;
    for (int t = 0; t < ix; ++t) v = fma(row[t], line[t], v);
  } else {
    const double* column = in + plane + i;
    const double* row = table + (long long)j * iy;
    for (int t = 0; t < iy; ++t) v = fma(row[t], column[(long long)t * ix], v);
  }
  out[n] = scale * v;
}

// One tridiagonal solve along z per transverse mode (Thomas elimination; the
// per-mode operator is symmetric positive definite).  `work` holds the
// eliminated super-diagonal.
__global__ void sf_modal_z_kernel(SfArgs a, double* data, double* work, const double* cos_x,
                                  const double* cos_y, int ix, int iy, int iz) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y * blockDim.y + threadIdx.y;
  if (m >= ix || n >= iy) return;
  double st[27];
  if (a.cowan) {
    for (int q = 0; q < 27; ++q) st[q] = a.stencil[q];
  } else {
    for (int q = 0; q < 27; ++q) st[q] = 0.0;
    st[13] = a.diagonal;
    st[12] = st[14] = -a.cx;
    st[10] = st[16] = -a.cy;
    st[4] = st[22] = -a.cz;
  }
  const double cx = cos_x[m], cy = cos_y[n];
  const double fx[3] = {cx, 1.0, cx}, fy[3] = {cy, 1.0, cy};
  double lambda[3];
  for (int c = 0; c < 3; ++c) {
    double v = 0.0;
    for (int y = 0; y < 3; ++y)
      for (int x = 0; x < 3; ++x) v = fma(st[(c * 3 + y) * 3 + x], fx[x] * fy[y], v);
    lambda[c] = v;
  }
  const long long step = (long long)ix * iy, base = (long long)n * ix + m;
  const double sub = lambda[0], diag = lambda[1], sup = lambda[2];
  double previous_c = 0.0, previous_d = 0.0;
  for (int k = 0; k < iz; ++k) {
    const double den = diag - sub * previous_c;
    const double ck = sup / den;
    const double dk = (data[base + k * step] - sub * previous_d) / den;
    work[base + k * step] = ck;
    data[base + k * step] = dk;
    previous_c = ck;
    previous_d = dk;
  }
  double next = 0.0;
  for (int k = iz - 1; k >= 0; --k) {
    next = data[base + k * step] - work[base + k * step] * next;
    data[base + k * step] = next;
  }
}

}  // namespace aprl_gpu
