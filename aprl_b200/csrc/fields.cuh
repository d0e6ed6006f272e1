// fields.cuh -- argument blocks of the grid kernels (fields.cu).
#pragma once

#include "common.cuh"

namespace aprl_gpu {

// One CPML profile axis (makeProfile, src/eb_cpml.cpp:195-248) on device:
// per native index the coefficients and the history slot (-1 inactive).
struct CpmlAxis {
  const double* inverse_kappa_minus_one;
  const double* decay;
  const double* drive;
  const int* ordinal;
};

// One active convolution history in [slot][k][row] order.
struct CpmlHistory {
  double* data;
  int slots, layers, row;
};

// The prepared inlet reference sampled at one (k, step): the lerp weights of
// Simulation::movingWindowFieldValue (src/simulation_moving_window.cpp:
// 284-293) are the same for every (i, j), so the host evaluates them once.
struct InletTable {
  const double* table[6];
  int nxc[6], nyc[6];
  int lo[6], hi[6];
  double fraction;
};

__device__ __forceinline__ double inlet_value(const InletTable& t, int c, int i, int j) {
  const size_t plane = (size_t)t.nyc[c] * t.nxc[c];
  const size_t cell = (size_t)j * t.nxc[c] + i;
  const double lower = t.table[c][(size_t)t.lo[c] * plane + cell];
  return t.fraction == 0. ? lower
                          : (1. - t.fraction) * lower +
                                t.fraction * t.table[c][(size_t)t.hi[c] * plane + cell];
}

// Argument blocks.  E, B, the halo planes and the CPML histories are
// binary64 in every mode; the template parameter F is the type of J (the
// grid view GridT<F>), which only the commit reads.
template <class F>
struct CowanArgs {
  GridT<F> g;            // B (ring) is updated in place
  const double* e[3];    // E^n (ring)
  const double* lower[3];  // inlet lower halo planes
  double alpha[3], beta[3], delta_xy, delta_yz, delta_zx;
  CpmlAxis mx, my;       // magnetic profiles (half-integer positions)
  CpmlHistory h[4];      // magnetic histories 0 (Bx,y) 3 (By,x) 4 (Bz,x) 5 (Bz,y)
  int chunk;             // z planes marched by one block
};

template <class F>
struct PreviewArgs {
  GridT<F> g;            // e_old = E^n, e_star = E* (written)
  CpmlAxis ex_prof, ey_prof;  // electric profiles (integer positions)
  CpmlHistory h[4];      // electric histories 6 (Ex,y) 9 (Ey,x) 10 (Ez,x) 11 (Ez,y)
  InletTable inlet;      // reference(a, i, j, offset, step+1)
  double* pre_inlet[2];  // when set: Ex, Ey of plane 0 before the inlet overwrite
  // When set: the first trial's orbit sum S = E* + E^n (the current-free pass
  // of orbit_sum_kernel), written here from the values already in hand;
  // binary32 when orbit_float, else binary64.
  void* orbit[3];
  int orbit_float;
};

// ChargeMatchedInlet::complete (src/charge_matched_inlet.h:55-71): Ez of the
// inserted layer at the interior nodes from the discrete Gauss law.
struct InletCompleteArgs {
  DGrid g;                  // e_old = E after the shift
  const double* rho;        // (nx+1) x (ny+1) inlet-layer charge
  int cx, cy;
  DeviceStatus* status;
};
__global__ void inlet_complete_kernel(InletCompleteArgs a);

// Boundary::begin with centred normal matching (src/moving_window_fields.cpp:225-236):
// the lower Ez halo takes minus Ez's departure from the reference at k = 0.
struct InletHaloArgs {
  DGrid g;
  double* lower_ez;         // (nx+1) x (ny+1)
  InletTable inlet;         // reference(a, i, j, offset, step)
  int cx, cy;
};
__global__ void inlet_halo_kernel(InletHaloArgs a);

struct InletPlaneArgs {
  int nx, ny;
  double* out[3];
  InletTable inlet;      // reference(a, i, j, offset-1, step)
};

template <class F>
struct ShiftArgs {
  GridT<F> g;            // e_old = the committed E (ring, bases already moved)
  InletTable inlet;      // reference(a, i, j, offset, step) after the shift
  CpmlHistory h[8];      // magnetic 0,3,4,5 then electric 6,9,10,11
  int history_base[8];
};

template <class F>
struct DetectorArgs {
  GridT<F> g;            // e_old = committed E
  DFrame frame;
  double origin_xy[2];
  int vertex_lower, half_lower;
  double vertex_fraction, half_fraction;
  double* out;
};

// Cowan kernel geometry: 32x8 column tiles, each block marching up to
// kCowanChunk z planes (fewer on small grids, so that there are enough
// blocks); APRL_COWAN_MIN_BLOCKS resident blocks per SM bound its registers.
// Measured on the 128x128x512 dipole grid: 8 planes at 6 blocks per SM,
// 0.47 ms, against 0.50 (16 at 5), 0.49 (16 at 6), 0.56-0.58 (32) and 0.47
// (4 at 6): more, shorter marches hide the plane loads better than the two
// halo planes per chunk cost.
#ifndef APRL_COWAN_CHUNK
#define APRL_COWAN_CHUNK 8
#endif
#ifndef APRL_COWAN_MIN_BLOCKS
#define APRL_COWAN_MIN_BLOCKS 6
#endif
constexpr int kCowanTileX = 32, kCowanTileY = 8, kCowanChunk = APRL_COWAN_CHUNK;
template <class F> __global__ void cowan_magnetic_kernel(CowanArgs<F> a);
template <class F> __global__ void electric_preview_kernel(PreviewArgs<F> a);
template <class F> __global__ void electric_commit_kernel(GridT<F> g);
__global__ void inlet_lower_kernel(InletPlaneArgs a);
template <class F> __global__ void shift_insert_kernel(ShiftArgs<F> a);
template <class F> __global__ void detector_plane_kernel(DetectorArgs<F> a);
template <class W>
__global__ void orbit_sum_kernel(GridT<double> g, W* s0, W* s1, W* s2, int with_current);
struct BShadowArgs {
  const double* b[3];
  float* out[3];
  long long n[3];
};
__global__ void b_shadow_kernel(BShadowArgs a);

// The reference's equivalent surface current (TransverseReferenceCurrent).
struct SurfaceArgs {
  const unsigned* points;   // (i, j) per target point
  double* table;            // [reference plane][point]
  long long count, planes;
  const double *bx, *by;    // reference B tables (native layout), for the preparation
  int nx, ny;
  double dx, dy;
  DeviceStatus* status;
  GridT<double> g;          // J of the trial, for the addition
  long long offset;
  unsigned long long step;  // step + 1 of the trial
  double beta;
};
__global__ void surface_prepare_kernel(SurfaceArgs a);
__global__ void surface_add_kernel(SurfaceArgs a);

}  // namespace aprl_gpu
