// selffield.cuh -- the initial self-field solve on the device
// (EBGaussFieldInitializer, src/eb_initial_field.cpp:829-1095).
//
// Scalars (potential, residual, CG direction, operator image) live on the
// node lattice of the Poisson geometry, lx = nx+1+2 pad by ly = ny+1+2 pad
// nodes, with nz+2 planes: plane p holds node k = p-1 and planes 0 and nz+1
// are the zero Dirichlet ghosts (the single-rank ScalarSlab).  Only the
// interior vertices of the solve domain are ever written in the CG vectors.
// Every reduction (dot products, charge and velocity moments, the Gauss
// check, the field energies) is a double-double sum: per-block partials in
// a fixed order, then one finishing block, so results do not depend on
// scheduling and agree with the reference's long double sums to about an
// ulp.  The CG scalars alpha, beta and the relative residual are formed on
// the device from those sums, so iterations run back to back; the host
// reads the iteration state once per batch.
#pragma once

#include "common.cuh"
#include "ledger.cuh"

namespace aprl_gpu {

constexpr int kSelfFieldThreads = 128;
constexpr int kSelfFieldBlocks = 1184;  // eight blocks per SM
constexpr int kMoments = 11;            // mass, m beta[3], m x[3], m x^2[3], charge

struct SfLattice {
  int lx, ly, planes;           // Poisson node lattice, planes = nz + 2
  int pad;                      // transverse padding (0 or 2)
  int lo[3], hi[3];             // solve domain: interior i in (lo, hi), k = p-1 likewise
};

// CG state on the device.
struct SfState {
  DD rr, source, denominator, next;
  double alpha, beta, relative;
  unsigned long long iterations;
  int done;                     // 1 converged, 2 lost positive definiteness, 3 non-finite
  // Blocks of the running apply or update launch that have written their
  // partial; the last one to arrive forms alpha or beta and resets it to 0.
  unsigned int arrivals;
};

struct SfArgs {
  DGrid g;                      // e_old = the run's E (written), b = the run's B
  SfLattice L;
  double *potential, *residual, *direction, *image;
  double* rho;                  // lx x ly x (nz+1) charge (Poisson lattice)
  double dx, dy, dz;
  // 7-point operator
  double cx, cy, cz, diagonal;
  // 27-point Cowan operator and smoothing
  int cowan;
  double stencil[27];           // [z][y][x]
  double alpha[3], beta[3], delta[3];  // delta per axis: yz, zx, xy
  double translation;
  double tolerance;
  int chunk;                    // planes per block of the tiled CG kernels
  DD* partial;
  SfState* state;
};

// Tiled CG kernels: blocks of kSfTileX x kSfTileY threads over the lattice's
// (i, j) columns, each marching `chunk` planes; one partial per block.
constexpr int kSfTileX = 32, kSfTileY = 4;

struct SfParticles {
  const double *x, *y, *z, *ux, *uy, *uz, *q, *m;
  long long n;
  int hold;                     // mean beta_z from the held longitudinal velocity
  double rapidity;              // gamma + gamma*beta of the boost
};

__global__ void sf_moments_kernel(SfParticles p, DD* partial);
__global__ void sf_finish_kernel(const DD* partial, int blocks, int quantities, DD* out);
__global__ void sf_deposit_kernel(SfParticles p, DGrid g, double* rho, int lx, int ly, int pad,
                                  DeviceStatus* status);
// The moving window's shaped reference source (BlockedCowanReference::
// depositQuintic) into an unpadded lattice; binomial selects linear-binomial3.
__global__ void sf_shaped_deposit_kernel(SfParticles p, DGrid g, double* rho, int lx, int ly,
                                         SfLattice L, int binomial, DeviceStatus* status);
__global__ void sf_source_kernel(SfArgs a, DD volume);
// One CG iteration is three launches: apply (its last block forms alpha),
// update (its last block forms the relative residual, the stopping test and
// beta) and direction.
__global__ void sf_apply_kernel(SfArgs a);
__global__ void sf_update_kernel(SfArgs a);
__global__ void sf_direction_kernel(SfArgs a);
__global__ void sf_smooth_kernel(SfArgs a, int axis);
__global__ void sf_electric_kernel(SfArgs a, int axis, double coefficient, int from_smoothed);
__global__ void sf_magnetic_kernel(SfArgs a, double scale, double lower_w, double upper_w);
__global__ void sf_clear_outside_kernel(SfArgs a, int component, int gx, int gy, int gz);
__global__ void sf_gauss_kernel(SfArgs a, const double* rho, int plo0, int phi0, int plo1,
                                int phi1, int plo2, int phi2, unsigned long long* max_bits);
__global__ void sf_energy_kernel(SfArgs a, DD volume);
// The transverse-mode direct solve (interior box in a compact layout).
__global__ void sf_modal_gather_kernel(SfArgs a, double* out, int ix, int iy, int iz);
__global__ void sf_modal_scatter_kernel(SfArgs a, const double* in, int ix, int iy, int iz);
__global__ void sf_modal_transform_kernel(const double* in, double* out, const double* table,
                                          int axis, int ix, int iy, int iz, double scale);
__global__ void sf_modal_z_kernel(SfArgs a, double* data, double* work, const double* cos_x,
                                  const double* cos_y, int ix, int iy, int iz);

// The open-transverse-wall reference (src/open_transverse_trace.h:20-235):
// the wall table in OpenTransverseTrace's layout, width = 4 (nx+3+ny+3)
// values per plane: the faces x = -dx, 0, nx dx, (nx+1) dx (ny+3 values
// each, j = -1 .. ny+1), then the faces in y (nx+3 values each).
struct SfOpenSide {
  const double* values;
  int nx, ny, nz;
  long long width;
};
// Free-space potential sum_s q_s / |t - s| at each target (one block each).
__global__ void sf_coulomb_kernel(const double* tx, const double* ty, const double* tz,
                                  long long targets, const double* sx, const double* sy,
                                  const double* sz, const double* sq, long long sources,
                                  double* out);
// liftOpenSides: the compact modal right-hand side minus the stencil's wall terms.
__global__ void sf_open_lift_kernel(SfArgs a, SfOpenSide side, double* rhs, int ix, int iy,
                                    int iz);
// The wall potentials into the potential lattice (interior planes).
__global__ void sf_open_wall_fill_kernel(SfArgs a, SfOpenSide side);
// smoothOnWall: the Cowan smoothing of `axis` at the wall nodes into image.
__global__ void sf_open_wall_smooth_kernel(SfArgs a, SfOpenSide side, int axis);

// Host helpers: the double-double quotient and square root rounded to binary64.
double sf_ratio(DD a, DD b);
long double sf_long(DD a);

}  // namespace aprl_gpu
