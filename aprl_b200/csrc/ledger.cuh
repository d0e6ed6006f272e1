// ledger.cuh -- the moving-window energy ledger on the device.
//
// Every quantity of the ledger is a sum over cells of a face or plane of the
// physical region (outside the xy CPML), over the whole interior, or over
// the stored particles.  The reference accumulates them in long double
// (src/moving_window_fields.cpp:387-437, src/simulation.cpp:3308-3340,
// 3591-3604).  Here each term is formed in binary64 exactly as the reference
// forms it, scaled by the cell volume / face area in double-double, and
// summed in double-double (Knuth's TwoSum, Dekker's product through fma, the
// QD library's renormalisation and division by a double), so the rounded
// result agrees with the long double sum to the last bit or so, whatever the
// summation order.  Reduction: each block sums a strided share of one
// quantity's terms and writes a double-double partial; one finishing block
// sums the partials in index order (deterministic) and applies the step's
// update to the device-resident ledger, so stepping takes no host round trip.
#pragma once

#include "common.cuh"
#include "dd.cuh"

namespace aprl_gpu {

enum LedgerKind : int {
  kLedgerPlane = 0,      // planeEnergy(k)
  kLedgerVolume = 1,     // localInteriorFieldEnergy
  kLedgerFaceX = 2,      // x face at cell column `index`, planes [0, kmax)
  kLedgerFaceY = 3,      // y face at cell row `index`, planes [0, kmax)
  kLedgerFaceZ = 4,      // z face of plane `index`
  kLedgerKinetic = 5,    // sum m c^2 u^2 / (gamma + 1)
  kLedgerTotal = 6,      // sum m c^2 gamma
  kLedgerRepresented = 7 // sum m / m_e
};

enum LedgerPhase : int {
  kLedgerPhaseBegin = 0,     // Boundary::begin: start power of the step
  kLedgerPhaseFinish = 1,    // overwrite energy and power, end power, dropped plane
  kLedgerPhaseShift = 2,     // inserted plane and the next start power after the shift
  kLedgerPhaseSnapshot = 3   // interior energy, power now, particle sums
};

struct LedgerTerm {
  int kind;
  int index;
  int kmax;
  int substitute;   // Ex/Ey of plane 0 from the pre-overwrite copies
  double sign;      // -1 for the lower faces
  long long count;  // terms
  int first_block, blocks;
};

constexpr int kLedgerMaxTerms = 20;
constexpr int kLedgerThreads = 256;
constexpr int kLedgerFinishThreads = 32 * kLedgerMaxTerms;  // one warp per quantity

// Device-resident ledger state (one per run).
struct DLedger {
  DD overwrite, inserted, cropped, remap;
  DD outward[6];
  DD start[6];      // boundary power at the step's begin
  DD removed;       // energy of plane nz-1 before the shift
  unsigned long long overwrite_events, flux_steps, remap_steps;
  DD snapshot[10];  // interior energy, power[6], kinetic, total, represented
};

struct LedgerArgs {
  DGrid g;                 // e_old = the committed E
  const double* pre[2];    // Ex (nx x ny+1), Ey (nx+1 x ny) of plane 0 before the overwrite
  const double *ux, *uy, *uz, *m;
  int i0, i1, j0, j1;      // physical aperture (cells)
  int nq;
  LedgerTerm q[kLedgerMaxTerms];
  DD volume, area_yz, area_xz, area_xy, c2;
  double half_dt;
  int phase;
  DD* partial;
  DLedger* ledger;
};

// Discrete Gauss law: rho from the particles with the node density the
// linear-binomial3 current conserves (F3 in x, linear in y, binomial3 in z),
// then G = eps0 div E - rho at every node, reduced over the interior nodes.
struct GaussArgs {
  DGrid g;                         // e_old = the committed E
  const double *x, *y, *z, *q;     // particle box positions and charges
  long long np;
  int shape;                       // 0 linear-binomial3, 1 quintic-compensated
  double* node;                    // (nx+1)(ny+1)(nz+1), [k][j][i]: rho, then G in place
  int i0, i1, j0, j1, k0, k1;      // interior nodes [i0, i1) x [j0, j1) x [k0, k1)
  DD volume;
  DD* partial;                     // per residual block: sum G^2, sum rho dV
  unsigned long long* max_bits;    // max |G| (interior), max |rho|, as ordered bits
  unsigned long long* outside;     // node contributions that fell outside the grid
  DD* result;                      // sum G^2, sum rho dV
};

constexpr int kGaussBlocks = 1184;  // eight 256-thread blocks per SM

__global__ void gauss_deposit_kernel(GaussArgs a);
__global__ void gauss_residual_kernel(GaussArgs a);
__global__ void gauss_finish_kernel(GaussArgs a, int blocks);

__global__ void ledger_partial_kernel(LedgerArgs a);
__global__ void ledger_finish_kernel(LedgerArgs a);

// Host-side double-double helpers for the scale factors (exact products of
// two binary64 values, then one more factor).
DD ledger_product(double a, double b);
DD ledger_product(DD a, double b);

}  // namespace aprl_gpu
