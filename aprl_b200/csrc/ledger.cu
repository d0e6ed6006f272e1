// ledger.cu -- double-double reductions of the moving-window energy ledger.
#include "ledger.cuh"

namespace aprl_gpu {

constexpr double kElectronMass = 9.1093837139e-31;  // src/eb_field.cpp:18

namespace {

__device__ __forceinline__ double ex_at(const LedgerArgs& a, int i, int j, int k, bool sub) {
  if (sub && k == 0) return a.pre[0][(size_t)j * a.g.nx + i];
  return a.g.e_old[0][e_index(a.g, 0, i, j, k)];
}
__device__ __forceinline__ double ey_at(const LedgerArgs& a, int i, int j, int k, bool sub) {
  if (sub && k == 0) return a.pre[1][(size_t)j * (a.g.nx + 1) + i];
  return a.g.e_old[1][e_index(a.g, 1, i, j, k)];
}
__device__ __forceinline__ double ez_at(const LedgerArgs& a, int i, int j, int k) {
  return a.g.e_old[2][e_index(a.g, 2, i, j, k)];
}
__device__ __forceinline__ double b_at(const LedgerArgs& a, int c, int i, int j, int k) {
  return a.g.b[c][b_index(a.g, c, i, j, k)];
}

struct CellFields {
  double e[3], b[3];
};

// The cell's collocated E and B of fieldEnergyDensityCell and
// poyntingComponentCell (src/eb_field.cpp:715-781), same operation order.
__device__ __forceinline__ CellFields collocate(const LedgerArgs& a, int i, int j, int k,
                                                bool sub) {
  CellFields f;
  f.e[0] = 0.25 * (((ex_at(a, i, j, k, sub) + ex_at(a, i, j + 1, k, sub)) +
                    ex_at(a, i, j, k + 1, sub)) + ex_at(a, i, j + 1, k + 1, sub));
  f.e[1] = 0.25 * (((ey_at(a, i, j, k, sub) + ey_at(a, i + 1, j, k, sub)) +
                    ey_at(a, i, j, k + 1, sub)) + ey_at(a, i + 1, j, k + 1, sub));
  f.e[2] = 0.25 * (((ez_at(a, i, j, k) + ez_at(a, i + 1, j, k)) + ez_at(a, i, j + 1, k)) +
                   ez_at(a, i + 1, j + 1, k));
  f.b[0] = 0.5 * (b_at(a, 0, i, j, k) + b_at(a, 0, i + 1, j, k));
  f.b[1] = 0.5 * (b_at(a, 1, i, j, k) + b_at(a, 1, i, j + 1, k));
  f.b[2] = 0.5 * (b_at(a, 2, i, j, k) + b_at(a, 2, i, j, k + 1));
  return f;
}

__device__ __forceinline__ double energy_density(const CellFields& f) {
  const double en = (f.e[0] * f.e[0] + f.e[1] * f.e[1]) + f.e[2] * f.e[2];
  const double bn = (f.b[0] * f.b[0] + f.b[1] * f.b[1]) + f.b[2] * f.b[2];
  return 0.5 * (kEpsilon0 * en + bn / kMu0);
}

__device__ __forceinline__ double poynting(const CellFields& f, int axis) {
  const int p = axis == 0 ? 1 : axis == 1 ? 2 : 0;  // first transverse component
  const int q = axis == 0 ? 2 : axis == 1 ? 0 : 1;  // second
  return (f.e[p] * f.b[q] - f.e[q] * f.b[p]) / kMu0;
}

__device__ DD term_value(const LedgerArgs& a, const LedgerTerm& t, long long n) {
  const int w = a.i1 - a.i0, h = a.j1 - a.j0;
  const bool sub = t.substitute != 0;
  switch (t.kind) {
    case kLedgerPlane: {
      const int j = a.j0 + (int)(n / w), i = a.i0 + (int)(n % w);
      return dd_mul(a.volume, energy_density(collocate(a, i, j, t.index, sub)));
    }
    case kLedgerVolume: {
      const long long per = (long long)w * h;
      const int k = (int)(n / per);
      const long long r = n % per;
      const int j = a.j0 + (int)(r / w), i = a.i0 + (int)(r % w);
      return dd_mul(a.volume, energy_density(collocate(a, i, j, k, false)));
    }
    case kLedgerFaceX: {
      const int k = (int)(n / h), j = a.j0 + (int)(n % h);
      return dd_mul(a.area_yz, t.sign * poynting(collocate(a, t.index, j, k, sub), 0));
    }
    case kLedgerFaceY: {
      const int k = (int)(n / w), i = a.i0 + (int)(n % w);
      return dd_mul(a.area_xz, t.sign * poynting(collocate(a, i, t.index, k, sub), 1));
    }
    case kLedgerFaceZ: {
      const int j = a.j0 + (int)(n / w), i = a.i0 + (int)(n % w);
      return dd_mul(a.area_xy, t.sign * poynting(collocate(a, i, j, t.index, sub), 2));
    }
    default: {
      const double ux = a.ux[n], uy = a.uy[n], uz = a.uz[n], m = a.m[n];
      if (t.kind == kLedgerRepresented) return dd_div(DD{m, 0.}, kElectronMass);
      const DD rest = dd_mul(a.c2, m);
      const double gamma = gamma_u(ux, uy, uz);
      if (t.kind == kLedgerTotal) return dd_mul(rest, gamma);
      const double u2 = (ux * ux + uy * uy) + uz * uz;
      return dd_div(dd_mul(rest, u2), gamma + 1.0);
    }
  }
}

// Fixed-order tree over the block.
__device__ DD block_sum(DD v, DD* shared) {
  const int t = threadIdx.x;
  shared[t] = v;
  __syncthreads();
  for (int s = kLedgerThreads / 2; s > 0; s >>= 1) {
    if (t < s) shared[t] = dd_add(shared[t], shared[t + s]);
    __syncthreads();
  }
  const DD out = shared[0];
  __syncthreads();
  return out;
}

// The term table with constant indices only (a dynamically indexed kernel
// parameter would be copied to local memory).
__device__ __forceinline__ LedgerTerm select_term(const LedgerArgs& a, int q) {
  LedgerTerm t = a.q[0];
#pragma unroll
  for (int s = 1; s < kLedgerMaxTerms; ++s)
    if (s == q) t = a.q[s];
  return t;
}

}  // namespace

DD ledger_product(double a, double b) { return two_prod(a, b); }
DD ledger_product(DD a, double b) { return dd_mul(a, b); }

__global__ void __launch_bounds__(kLedgerThreads) ledger_partial_kernel(LedgerArgs a) {
  __shared__ DD shared[kLedgerThreads];
  const int b = blockIdx.x;
  int q = 0;
#pragma unroll
  for (int s = 1; s < kLedgerMaxTerms; ++s)
    if (s < a.nq && b >= a.q[s].first_block) q = s;
  const LedgerTerm t = select_term(a, q);
  DD sum{0., 0.};
  const long long stride = (long long)t.blocks * kLedgerThreads;
  for (long long n = (long long)(b - t.first_block) * kLedgerThreads + threadIdx.x; n < t.count;
       n += stride)
    sum = dd_add(sum, term_value(a, t, n));
  sum = block_sum(sum, shared);
  if (threadIdx.x == 0) a.partial[b] = sum;
}

// One block, one warp per quantity: each quantity's partials in index order
// (a fixed lane-strided sum and shuffle tree), then the ledger update of the
// phase (src/moving_window_fields.cpp:214-218, 281-288, 431-436, 500-514).
__global__ void __launch_bounds__(kLedgerFinishThreads) ledger_finish_kernel(LedgerArgs a) {
  __shared__ DD result[kLedgerMaxTerms];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  for (int q = warp; q < a.nq; q += kLedgerFinishThreads / 32) {
    const LedgerTerm t = select_term(a, q);
    DD sum{0., 0.};
    for (int n = lane; n < t.blocks; n += 32) sum = dd_add(sum, a.partial[t.first_block + n]);
    for (int offset = 16; offset > 0; offset >>= 1) {
      const DD other{__shfl_down_sync(0xffffffffu, sum.hi, offset),
                     __shfl_down_sync(0xffffffffu, sum.lo, offset)};
      sum = dd_add(sum, other);
    }
    if (lane == 0) result[q] = sum;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  DLedger& l = *a.ledger;
  switch (a.phase) {
    case kLedgerPhaseBegin:
      for (int f = 0; f < 6; ++f) l.start[f] = result[f];
      break;
    case kLedgerPhaseFinish: {
      // 0/1: plane 0 before/after the overwrite; 2-6/7-11: inlet-only face
      // power before/after; 12-17: end power; 18: plane nz-1.
      l.overwrite = dd_add(l.overwrite, dd_add(result[1], dd_neg(result[0])));
      ++l.overwrite_events;
      const DD half_dt{a.half_dt, 0.};
      for (int f = 0; f < 6; ++f) {
        const DD delta = f < 5 ? dd_add(result[7 + f], dd_neg(result[2 + f])) : DD{0., 0.};
        const DD sum = dd_add(dd_add(l.start[f], result[12 + f]), dd_neg(delta));
        l.outward[f] = dd_add(l.outward[f], dd_mul(sum, half_dt.hi));
      }
      ++l.flux_steps;
      l.removed = result[18];
      break;
    }
    case kLedgerPhaseShift:
      // 0: the inserted plane; 1-6: the boundary power of the shifted state,
      // which is the next step's start power.
      l.remap = dd_add(l.remap, dd_add(result[0], dd_neg(l.removed)));
      l.inserted = dd_add(l.inserted, result[0]);
      l.cropped = dd_add(l.cropped, l.removed);
      ++l.remap_steps;
      for (int f = 0; f < 6; ++f) l.start[f] = result[1 + f];
      break;
    default:
      for (int q = 0; q < a.nq && q < 10; ++q) l.snapshot[q] = result[q];
      break;
  }
}

// ---- discrete Gauss law ----------------------------------------------------
// Node charge density of one particle: the density whose change the
// run's current balances.  linear-binomial3 (the F3 density of
// verification/transverse_binomial_checks.cpp:12-66): F3 weights in x over
// nodes i-1..i+2, linear in y over j, j+1, the binomial3 smoothing of the
// linear z weights over k-1..k+2.  quintic-compensated: linear in x and y
// (nodes i, i+1 and j, j+1) and the quintic node basis in z
// (longitudinal_shape::nodeWeight, src/longitudinal_shape.h:48-56, nodes
// floor(z)-5 .. floor(z)+6), the density of quintic_segment's current (x and
// y edge currents with linear transverse weights, the edge basis along z).
__global__ void gauss_deposit_kernel(GaussArgs a) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.np) return;
  const DGrid& g = a.g;
  const double x = (a.x[n] - g.origin[0]) / g.dx;
  const double y = (a.y[n] - g.origin[1]) / g.dy;
  const double z = (a.z[n] - g.origin[2]) / g.dz;
  const double fi = floor(x), fj = floor(y), fk = floor(z);
  const int i = (int)fi, j = (int)fj, k = (int)fk;
  const double fx = x - fi, fy = y - fj, fz = z - fk;
  double wx[4], wz[12];
  int xfirst, xcount, zfirst, zcount;
  if (a.shape == 0) {
    wx[0] = 0.25 * (1.0 - fx);
    wx[1] = 0.5 - 0.25 * fx;
    wx[2] = 0.25 + 0.25 * fx;
    wx[3] = 0.25 * fx;
    xfirst = i - 1;
    xcount = 4;
    for (int t = 0; t < 4; ++t) wz[t] = 0.;
    const double bw[3] = {0.25, 0.5, 0.25};
    for (int s = 0; s < 3; ++s) {
      wz[s] += bw[s] * (1.0 - fz);
      wz[s + 1] += bw[s] * fz;
    }
    zfirst = k - 1;
    zcount = 4;
  } else {
    wx[0] = 1.0 - fx;
    wx[1] = fx;
    xfirst = i;
    xcount = 2;
    Basis<double> b;
    quintic_basis<double>(z, false, b);
    for (int t = 0; t < 12; ++t) wz[t] = b.v[t];
    zfirst = (int)b.first;
    zcount = b.count;
  }
  const double wy[2] = {1.0 - fy, fy};
  const double q = a.q[n] / (g.dx * g.dy * g.dz);
  const int nx = g.nx + 1, ny = g.ny + 1, nz = g.nz + 1;
  unsigned long long missed = 0;
  for (int t = 0; t < zcount; ++t) {
    const int kk = zfirst + t;
    for (int v = 0; v < 2; ++v) {
      const int jj = j + v;
      for (int u = 0; u < xcount; ++u) {
        const int ii = xfirst + u;
        if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) {
          ++missed;
          continue;
        }
        atomicAdd(&a.node[((size_t)kk * ny + jj) * nx + ii], q * wx[u] * wy[v] * wz[t]);
      }
    }
  }
  if (missed) atomicAdd(a.outside, missed);
}

__device__ __forceinline__ double e_or_zero(const DGrid& g, int c, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= e_nx(g, c) || j >= e_ny(g, c) || k >= e_nz(g, c))
    return 0.;
  return g.e_old[c][e_index(g, c, i, j, k)];
}

// G = eps0 div E - rho at each node (edges outside the grid count as zero),
// written over rho; sum of G^2 and max |G| over the interior nodes, sum of
// rho dV and max |rho| over all nodes.
__global__ void __launch_bounds__(kLedgerThreads) gauss_residual_kernel(GaussArgs a) {
  __shared__ DD shared[kLedgerThreads];
  const DGrid& g = a.g;
  const int nx = g.nx + 1, ny = g.ny + 1;
  const long long count = (long long)nx * ny * (g.nz + 1);
  DD g2{0., 0.}, charge{0., 0.};
  double gmax = 0., rmax = 0.;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % nx);
    const int j = (int)((n / nx) % ny);
    const int k = (int)(n / ((long long)nx * ny));
    const double rho = a.node[n];
    const double div = (e_or_zero(g, 0, i, j, k) - e_or_zero(g, 0, i - 1, j, k)) / g.dx +
                       (e_or_zero(g, 1, i, j, k) - e_or_zero(g, 1, i, j - 1, k)) / g.dy +
                       (e_or_zero(g, 2, i, j, k) - e_or_zero(g, 2, i, j, k - 1)) / g.dz;
    const double residual = kEpsilon0 * div - rho;
    a.node[n] = residual;
    charge = dd_add(charge, dd_mul(a.volume, rho));
    rmax = fmax(rmax, fabs(rho));
    if (i >= a.i0 && i < a.i1 && j >= a.j0 && j < a.j1 && k >= a.k0 && k < a.k1) {
      g2 = dd_add(g2, two_prod(residual, residual));
      gmax = fmax(gmax, fabs(residual));
    }
  }
  g2 = block_sum(g2, shared);
  charge = block_sum(charge, shared);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = g2;
    a.partial[2 * blockIdx.x + 1] = charge;
  }
  // Non-negative doubles order like their bit patterns.
  if (gmax > 0.) atomicMax(&a.max_bits[0], (unsigned long long)__double_as_longlong(gmax));
  if (rmax > 0.) atomicMax(&a.max_bits[1], (unsigned long long)__double_as_longlong(rmax));
}

__global__ void __launch_bounds__(kLedgerThreads) gauss_finish_kernel(GaussArgs a, int blocks) {
  __shared__ DD shared[kLedgerThreads];
  for (int q = 0; q < 2; ++q) {
    DD sum{0., 0.};
    for (int n = threadIdx.x; n < blocks; n += kLedgerThreads)
      sum = dd_add(sum, a.partial[2 * n + q]);
    sum = block_sum(sum, shared);
    if (threadIdx.x == 0) a.result[q] = sum;
  }
}

}  // namespace aprl_gpu
