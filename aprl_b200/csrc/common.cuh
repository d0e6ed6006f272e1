// common.cuh -- device-side views, constants and helpers shared by the field
// and particle kernels of the B200 PIC step.
//
// Memory layout in HBM (one run):
//   * Yee components in the reference's SoA layout, x fastest,
//     index (k*ny_c + j)*nx_c + i (src/eb_field.h:134-141), but E and B are
//     z RING BUFFERS: logical plane k lives at physical plane
//     (k + zbase_c) mod nz_c.  The moving-window shift
//     (src/moving_window_fields.cpp:439-518) then only decrements zbase and
//     rewrites the one inserted plane instead of moving the volume.
//   * Two E buffers: E^n ("old", read by the orbit-averaged gather) and
//     E* ("star", the zero-current preview with its boundary applied).  The
//     trial candidate E* - dt/eps0 J is never stored: every gather forms it
//     from E* and J, so a fixed-point trial touches the grid only through J.
//   * J is not ring-buffered: it is cleared before every trial.
//   * CPML convolution histories keep the reference's [slot][k][row] order
//     (src/eb_cpml.cpp:42-96) with the same z ring as their component.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace aprl_gpu {

constexpr double kC = 299792458.0;          // src/eb_field.cpp:15-19
constexpr double kEpsilon0 = 8.8541878128e-12;
constexpr double kMu0 = 1.25663706212e-6;
constexpr double kEpsilon = 2.220446049250313080847e-16;  // DBL_EPSILON
constexpr double kDblMin = 2.2250738585072013830903e-308;
constexpr double kPi = 3.14159265358979323846;

// Device error codes (first error wins; the host maps them to statuses).
enum DeviceError : unsigned {
  kErrNone = 0,
  kErrCrossingBudget = 1,     // weights(): more than 64 cuts
  kErrOrbitOutside = 2,       // clipOpenOrbit found no in-domain part
  kErrDepositOutside = 3,     // depositor endpoint outside the E/B domain
  kErrSupportX = 4,           // quintic transverse support outside x grid
  kErrSupportY = 5,           // transverse support outside y grid
  kErrRootNonphysical = 6,    // momentum(): nonphysical mean-gamma root
  kErrRootNoConvergence = 7,  // momentum(): 12 Newton steps exhausted
  kErrNonFinite = 8,          // non-finite particle coordinate
  kErrStartInCpml = 9,        // active particle starts in the CPML region
  kErrStartOutside = 10,      // trajectory starts outside the domain
  kErrBeyondExit = 11,        // active particle started beyond the exit
  kErrUpstream = 12,          // active particle upstream of the inlet
  kErrCarrierWeight = 13,     // invalid carrier weight
  kErrFellBehind = 14,        // particle/carrier behind the moving inlet
  kErrReferenceRange = 15,    // inlet reference query outside the table
  kErrHitLocate = 16,         // boundary hit fraction outside [0,1]
  kErrEarlyRelease = 17,      // held particle released before entering the window
  kErrAdmission = 18,         // invalid upstream admission of a held particle
  kErrHeldBoundary = 19,      // held segment crossed a particle boundary
  kErrInletSource = 20,       // non-finite charge-matched inlet source
  kErrInletField = 21,        // non-finite charge-matched inlet field
  kErrFixedRange = 22,        // deterministic deposit: contribution beyond the fixed-point range
  kErrBounds = 23,            // bounds-checked build: an index outside its array
  kErrSurfaceCurrent = 24,    // non-finite equivalent boundary current of the reference
  kErrReferenceSupport = 25,  // shaped reference source on or outside the zero-potential box
  kErrReferenceSource = 26,   // shaped reference source: non-finite longitudinal coordinate
  kErrReferenceCharge = 27,   // shaped reference source: non-finite charge
  kErrCount
};

struct DeviceStatus {
  unsigned code;
  unsigned long long where;  // particle or element index of the first error
};

__device__ __forceinline__ void raise_error(DeviceStatus* s, unsigned code,
                                            unsigned long long where) {
  if (atomicCAS(&s->code, 0u, code) == 0u) s->where = where;
}

// The bounds-checked build (-DAPRL_GPU_BOUNDS_CHECK, libaprl_b200_checked.so):
// every field, current, orbit-sum, CPML-history and inlet-plane index of the
// step's kernels is tested against its array before the access.  An index
// outside raises kErrBounds in the run's status word with `site` (which
// access) in the top 16 bits of the recorded element and the index below,
// and the access goes to element 0 instead: the kernel never touches memory
// outside its arrays and never traps.  In the normal build the checks
// compile to nothing.
#ifdef APRL_GPU_BOUNDS_CHECK
__device__ __forceinline__ size_t bounded(DeviceStatus* s, size_t index, size_t extent,
                                          unsigned site) {
  if (index < extent) return index;
  if (s) raise_error(s, kErrBounds, ((unsigned long long)site << 48) | (index & 0xffffffffffffull));
  return 0;
}
#define APRL_BOUNDED(status, index, extent, site) \
  ::aprl_gpu::bounded((status), (size_t)(index), (size_t)(extent), (site))
#else
#define APRL_BOUNDED(status, index, extent, site) ((size_t)(index))
#endif

// One magnet of SIFieldSourceSet (src/eb_sources.h:103-140).
struct DMagnet {
  int type;  // 0 undulator, 1 dipole, 2 quadrupole
  int gaussian_fringe;
  double center[3];
  double length, period, peak_field;
  double quadrupole_gradient, wave_number, fringe_extent;
  double cos_angle, sin_angle;
};

struct DFrame {  // BoostFrameTransform
  double gamma, beta, gamma_beta;
  double lab_time_origin, lab_z_origin, box_z_origin;
};

// Everything the kernels need about the grid; passed by value.  E and B are
// binary64 in every mode.  F is the type of the current J and of the
// particle-side weight arithmetic: double for the FP64 drop-in, float for
// the FP32-mixed mode.
template <class F>
struct GridT {
  int nx, ny, nz;
  double dx, dy, dz, dt;
  double origin[3];      // localOriginBox_ of the current window
  double* e_old[3];      // E^n  (ring)
  double* e_star[3];     // E*   (ring)
  double* b[3];          // B    (ring)
  F* j[3];               // J    (plain)
  int zb_e[3];           // ring bases of Ex Ey Ez
  int zb_b[3];           // ring bases of Bx By Bz
  F jcoef;               // (-1*dt)/eps0, applyCurrentSource(-1) scale
  // Deterministic mode: the deposit adds into these (lo, hi) word pairs
  // (fixed_add, scale jq_scale) instead of J, and a conversion pass writes J
  // from them once per trial.  Null in the default mode.
  unsigned long long* jq[3];
  double jq_scale;
  // Set for the kernels of a fixed-point trial issued ahead of the verdict
  // on the previous one: nonzero once an earlier trial of the step has
  // converged, and the trial's kernels then return at once.
  const int* stop;
  DeviceStatus* status;  // the run's status word (the bounds-checked build reports here)
};

// True when the trial this grid view belongs to was made unnecessary.
template <class F>
__device__ __forceinline__ bool trial_skipped(const GridT<F>& g) {
  return g.stop != nullptr && *g.stop != 0;
}
using DGrid = GridT<double>;

template <class F>
__device__ __forceinline__ int e_nx(const GridT<F>& g, int c) { return g.nx + (c != 0); }
template <class F>
__device__ __forceinline__ int e_ny(const GridT<F>& g, int c) { return g.ny + (c != 1); }
template <class F>
__device__ __forceinline__ int e_nz(const GridT<F>& g, int c) { return g.nz + (c != 2); }
template <class F>
__device__ __forceinline__ int b_nx(const GridT<F>& g, int c) { return g.nx + (c == 0); }
template <class F>
__device__ __forceinline__ int b_ny(const GridT<F>& g, int c) { return g.ny + (c == 1); }
template <class F>
__device__ __forceinline__ int b_nz(const GridT<F>& g, int c) { return g.nz + (c == 2); }

__device__ __forceinline__ int ring(int k, int base, int n) {
  int p = k + base;
  return p >= n ? p - n : p;
}

#ifdef APRL_GPU_BOUNDS_CHECK
// (i, j, k) inside an nx x ny x nz component, else kErrBounds and node 0.
__device__ __forceinline__ bool node_inside(DeviceStatus* s, int i, int j, int k, int nx, int ny,
                                            int nz, unsigned site) {
  if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) return true;
  if (s) raise_error(s, kErrBounds, ((unsigned long long)site << 48) |
                                        ((unsigned long long)(unsigned)k << 24) |
                                        (((unsigned long long)(unsigned)j & 0xfffull) << 12) |
                                        ((unsigned long long)(unsigned)i & 0xfffull));
  return false;
}
#define APRL_NODE_CHECK(g, i, j, k, nx, ny, nz, site) \
  if (!node_inside((g).status, (i), (j), (k), (nx), (ny), (nz), (site))) return 0
#else
#define APRL_NODE_CHECK(g, i, j, k, nx, ny, nz, site)
#endif

template <class F>
__device__ __forceinline__ size_t e_index(const GridT<F>& g, int c, int i, int j, int k) {
  const int nzc = e_nz(g, c);
  APRL_NODE_CHECK(g, i, j, k, e_nx(g, c), e_ny(g, c), nzc, 1 + c);
  return ((size_t)ring(k, g.zb_e[c], nzc) * e_ny(g, c) + j) * e_nx(g, c) + i;
}

template <class F>
__device__ __forceinline__ size_t b_index(const GridT<F>& g, int c, int i, int j, int k) {
  const int nzc = b_nz(g, c);
  APRL_NODE_CHECK(g, i, j, k, b_nx(g, c), b_ny(g, c), nzc, 4 + c);
  return ((size_t)ring(k, g.zb_b[c], nzc) * b_ny(g, c) + j) * b_nx(g, c) + i;
}

template <class F>
__device__ __forceinline__ size_t j_index(const GridT<F>& g, int c, int i, int j, int k) {
  APRL_NODE_CHECK(g, i, j, k, e_nx(g, c), e_ny(g, c), e_nz(g, c), 7 + c);
  return ((size_t)k * e_ny(g, c) + j) * e_nx(g, c) + i;
}

// Elements of E component c (also of J and of the orbit sum) and of B component c.
template <class F>
__device__ __forceinline__ size_t e_count(const GridT<F>& g, int c) {
  return (size_t)e_nx(g, c) * e_ny(g, c) * e_nz(g, c);
}
template <class F>
__device__ __forceinline__ size_t b_count(const GridT<F>& g, int c) {
  return (size_t)b_nx(g, c) * b_ny(g, c) * b_nz(g, c);
}

// applyCurrentSource's interior mask (src/source_coupling.cpp:87) at one rank.
template <class F>
__device__ __forceinline__ bool current_mask(const GridT<F>& g, int c, int i, int j, int k) {
  if (c == 0) return j > 0 && j < g.ny && k != 0 && k != g.nz;
  if (c == 1) return i > 0 && i < g.nx && k != 0 && k != g.nz;
  return i > 0 && i < g.nx && j > 0 && j < g.ny;
}

// Trial candidate E* - dt/eps0 J at a native node (applyCurrentSource(-1)).
template <class F>
__device__ __forceinline__ F e_candidate(const GridT<F>& g, int c, int i, int j, int k) {
  F v = F(g.e_star[c][e_index(g, c, i, j, k)]);
  if (current_mask(g, c, i, j, k)) {
    const F jc = g.j[c][j_index(g, c, i, j, k)];
    if (jc != F(0.)) v += g.jcoef * jc;
  }
  return v;
}

// ---------------------------------------------------------------------------
// Order-free summation of binary64 contributions (the deterministic mode).
// A contribution v becomes the integer n = round(v * scale), |n| < 2^62,
// split into lo = n mod 2^32 (0 <= lo < 2^32) and hi = floor(n / 2^32), and
// both parts are added with 64-bit integer reductions into a (lo, hi) word
// pair.  Integer addition is associative, so after any interleaving of the
// adds the pair holds the exact sum of the rounded contributions,
// hi * 2^32 + lo (hi two's complement), and so does every other run: the
// pair's value does not depend on the order of the adds.  lo stays below
// 2^64 for fewer than 2^32 adds and hi below 2^63 in magnitude for fewer
// than 2^33.  `scale` is a power of two chosen by the host so that the
// largest contribution a run can make maps below 2^62.
constexpr double kFixedLimit = 4611686018427387904.0;  // 2^62

// Returns false (and adds nothing) for a value outside the range.
__device__ __forceinline__ bool fixed_add(unsigned long long* pair, double v, double scale) {
  const double s = v * scale;
  if (!(fabs(s) < kFixedLimit)) return false;
  const long long n = __double2ll_rn(s);
  const unsigned long long lo = (unsigned long long)n & 0xffffffffull;
  const long long hi = n >> 32;
  if (lo) atomicAdd(&pair[0], lo);
  if (hi) atomicAdd(&pair[1], (unsigned long long)hi);
  return true;
}

// The pair's value hi * 2^32 + lo, rounded once to binary64 and multiplied
// by `unscale` (1/scale, a power of two, so that product is exact).
__device__ __forceinline__ double fixed_value(unsigned long long lo, unsigned long long hi_word,
                                              double unscale) {
  const long long hi = (long long)hi_word;
  // 128-bit two's complement (vh:vl) = hi * 2^32 + lo.
  const unsigned long long shifted = (unsigned long long)hi << 32;
  unsigned long long vl = shifted + lo;
  long long vh = (hi >> 32) + (vl < shifted ? 1 : 0);
  const bool negative = vh < 0;
  unsigned long long mh = (unsigned long long)vh, ml = vl;
  if (negative) {  // magnitude: two's complement negation of the 128-bit value
    ml = ~ml + 1ull;
    mh = ~mh + (ml == 0ull ? 1ull : 0ull);
  }
  double m;
  if (mh == 0ull) {
    m = __ull2double_rn(ml);
  } else {
    // The leading 64 bits, with every bit below them folded into bit 0 (a
    // sticky bit under the 11 bits the conversion drops), round once.
    const int lz = __clzll((long long)mh);
    unsigned long long top = lz ? (mh << lz) | (ml >> (64 - lz)) : mh;
    const unsigned long long rest = lz ? ml << lz : ml;
    top |= rest != 0ull ? 1ull : 0ull;
    m = ldexp(__ull2double_rn(top), 64 - lz);
  }
  return (negative ? -m : m) * unscale;
}

// ---------------------------------------------------------------------------
// The quintic-compensated node and edge bases, shared by the deposit, the
// gathers, the charge-matched inlet and the Gauss-law node density.
template <class F>
struct Basis {
  long long first;
  int count;
  F v[12];
};

// The seven compensation coefficients of the p = 5 spline
// (src/longitudinal_shape.h:48-54), each formed in binary64 and rounded once
// to the arithmetic type.
namespace quintic_detail {
constexpr double p = 5., a = p / 6., b = 3 * p / 40. + p * (p - 1) / 72.,
                 d = 5 * p / 112. + p * (p - 1) / 80. + p * (p - 1) * (p - 2) / 1296.;
constexpr double c[7] = {-d / 64.,
                         b / 16. + 3 * d / 32.,
                         -a / 4. - b / 4. - 15 * d / 64.,
                         1 + a / 2. + 3 * b / 8. + 5 * d / 16.,
                         -a / 4. - b / 4. - 15 * d / 64.,
                         b / 16. + 3 * d / 32.,
                         -d / 64.};
}  // namespace quintic_detail

static __constant__ double kQuinticC64[7] = {
    quintic_detail::c[0], quintic_detail::c[1], quintic_detail::c[2], quintic_detail::c[3],
    quintic_detail::c[4], quintic_detail::c[5], quintic_detail::c[6]};
static __constant__ float kQuinticC32[7] = {
    float(quintic_detail::c[0]), float(quintic_detail::c[1]), float(quintic_detail::c[2]),
    float(quintic_detail::c[3]), float(quintic_detail::c[4]), float(quintic_detail::c[5]),
    float(quintic_detail::c[6])};

template <class F>
__device__ __forceinline__ F quintic_coefficient(int k);
template <>
__device__ __forceinline__ double quintic_coefficient<double>(int k) {
  return kQuinticC64[k];
}
template <>
__device__ __forceinline__ float quintic_coefficient<float>(int k) {
  return kQuinticC32[k];
}

// basis(z, edge, QuinticCompensated) (src/longitudinal_shape.h:48-54): the
// cell in binary64, the B-spline and compensation arithmetic in F on the
// cell-relative offset.  The compensation of the degree-`degree` spline
// values n[0..degree]:
template <class F>
__device__ __forceinline__ void quintic_compensate(const F* n, unsigned degree, double cell,
                                                   Basis<F>& r) {
  r.first = (long long)cell - 5;
  r.count = degree + 7;
  for (int q = 0; q < 12; ++q) r.v[q] = F(0.);
  for (unsigned j = 0; j <= degree; ++j)
    for (unsigned k = 0; k < 7; ++k) r.v[j + k] += n[j] * quintic_coefficient<F>(k);
}

// Node q of quintic_compensate's result alone: the same products, summed in
// the same order (spline index j rising), so the value is bit for bit
// quintic_compensate's r.v[q].
template <class F>
__device__ __forceinline__ F quintic_compensated_at(const F* n, int degree, int q) {
  F v = F(0.);
#pragma unroll
  for (int j = 0; j <= 5; ++j)
    if (j <= degree && q - j >= 0 && q - j < 7) v += n[j] * quintic_coefficient<F>(q - j);
  return v;
}

// The B-spline recursion on f = z - floor(z) up to `degree`.
template <class F>
__device__ __forceinline__ void quintic_spline_level(F n[6], F f, unsigned j) {
  F saved = F(0.);
  for (unsigned k = 0; k < j; ++k) {
    const F t = n[k] / F(j);
    n[k] = saved + (F(k + 1) - f) * t;
    saved = (f + F(j) - F(k) - F(1)) * t;
  }
  n[j] = saved;
}

template <class F>
__device__ __forceinline__ void quintic_basis(double z, bool edge, Basis<F>& r) {
  const unsigned degree = edge ? 4 : 5;
  const double cell = floor(z);
  const F f = F(z - cell);
  F n[6] = {F(1.), F(0.), F(0.), F(0.), F(0.), F(0.)};
  for (unsigned j = 1; j <= degree; ++j) quintic_spline_level(n, f, j);
  quintic_compensate(n, degree, cell, r);
}

// Both spline sets of one point: the edge basis (degree 4) is the node
// basis's recursion (degree 5) stopped after its fourth level, so one pass
// yields the values quintic_basis computes for either.
template <class F>
struct QuinticSplines {
  double cell;
  F edge[5];
  F node[6];
};

template <class F>
__device__ __forceinline__ void quintic_splines(double z, QuinticSplines<F>& s) {
  s.cell = floor(z);
  const F f = F(z - s.cell);
  F n[6] = {F(1.), F(0.), F(0.), F(0.), F(0.), F(0.)};
#pragma unroll
  for (unsigned j = 1; j <= 4; ++j) quintic_spline_level(n, f, j);
#pragma unroll
  for (int q = 0; q < 5; ++q) s.edge[q] = n[q];
  quintic_spline_level(n, f, 5);
#pragma unroll
  for (int q = 0; q < 6; ++q) s.node[q] = n[q];
}

// BoostFrameTransform::gammaFromProperVelocity (src/boostframe.cpp:74-87).
__device__ __forceinline__ double gamma_u(double ux, double uy, double uz) {
  const double scale = fmax(1.0, fmax(fabs(ux), fmax(fabs(uy), fabs(uz))));
  const double inv = 1.0 / scale;
  const double a = ux * inv, b = uy * inv, c = uz * inv;
  return scale * sqrt(inv * inv + a * a + b * b + c * c);
}

// repeatHeldAddition (src/pending_particle_queue.cpp:38-88): `count`
// separately rounded binary64 additions, with runs of constant spacing
// skipped by integer ULP arithmetic.  Host and device share this code.
__host__ __device__ __forceinline__ unsigned long long held_bits(double v) {
#ifdef __CUDA_ARCH__
  return (unsigned long long)__double_as_longlong(v);
#else
  unsigned long long b;
  memcpy(&b, &v, 8);
  return b;
#endif
}
__host__ __device__ __forceinline__ double held_from_bits(unsigned long long b) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double v;
  memcpy(&v, &b, 8);
  return v;
#endif
}
__host__ __device__ __forceinline__ unsigned long long held_ordered(unsigned long long v) {
  return (v & 0x8000000000000000ull) ? ~v : v ^ 0x8000000000000000ull;
}
__host__ __device__ __forceinline__ double held_from_ordered(unsigned long long v) {
  return held_from_bits((v & 0x8000000000000000ull) ? v ^ 0x8000000000000000ull : ~v);
}
__host__ __device__ __forceinline__ bool held_same_spacing(unsigned long long a,
                                                           unsigned long long b) {
  const unsigned long long m = 0x8000000000000000ull | 0x7ff0000000000000ull;
  return (a & m) == (b & m);
}
__host__ __device__ __forceinline__ double held_repeat_positive(double x, double increment,
                                                                unsigned long long count) {
  while (count) {
    const double y = x + increment;
    if (!isfinite(y)) return y;
    if (count == 1 || y == x) return y;
    const double z = y + increment;
    const unsigned long long bx = held_bits(x), by = held_bits(y), bz = held_bits(z);
    if (isfinite(z) && held_same_spacing(bx, by) && held_same_spacing(by, bz)) {
      const unsigned long long ox = held_ordered(bx), oy = held_ordered(by), oz = held_ordered(bz);
      const unsigned long long stride = oy - ox;
      if (stride && oz - oy == stride) {
        const unsigned long long last_bits =
            (bx & 0x8000000000000000ull) ? bx & (0x8000000000000000ull | 0x7ff0000000000000ull)
                                         : bx | 0x000fffffffffffffull;
        const unsigned long long available = (held_ordered(last_bits) - ox) / stride;
        const unsigned long long safe = available ? available - 1 : 0;
        const unsigned long long jump = safe < count ? safe : count;
        if (jump) {
          x = held_from_ordered(ox + jump * stride);
          count -= jump;
          continue;
        }
      }
    }
    x = y;
    --count;
  }
  return x;
}
__host__ __device__ __forceinline__ double repeat_held_addition(double initial, double increment,
                                                                unsigned long long count) {
  if (!count) return initial;
  if (increment < 0.) {
    const double result = -held_repeat_positive(-initial, -increment, count);
    return result == 0. ? 0. : result;
  }
  return held_repeat_positive(initial, increment, count);
}

// labZFromBoxZT (src/boostframe.cpp:241-245).
__device__ __forceinline__ double lab_z_from_box_zt(const DFrame& f, double z, double t) {
  return f.lab_z_origin + fma(f.gamma_beta * kC, t, f.gamma * (z - f.box_z_origin));
}

}  // namespace aprl_gpu
