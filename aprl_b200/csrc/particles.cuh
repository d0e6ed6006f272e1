// particles.cuh -- argument blocks of the particle kernels (particles.cu).
#pragma once

#include "common.cuh"

namespace aprl_gpu {

constexpr int kMaxMagnets = 4;

// ParticleCPMLRegion + ParticleOpenBoundary geometry of the current window
// (src/particle_boundary.cpp:56-85, 251-283), evaluated on the host.
struct DRegion {
  double outer_lower[3], outer_upper[3];
  double physical_lower[3], physical_upper[3], tolerance[3];
  double max_rate[3];     // maximumConductivityRate per axis
  double thickness[3];    // cells*spacing per axis (0 when no CPML)
  int cells[3];
  double global_lower[3], global_upper[3], global_tolerance[3];
  double order;           // polynomial order of the grading
};

// Particle SoA (RelativisticParticleSI without the diagnostics).  Storage
// is sorted by cell (x fastest) for gather/deposit locality; `order` keeps
// each particle's rank in the reference's list order, which the ABI
// restores on read-out.
struct DParticles {
  double *x, *y, *z, *ux, *uy, *uz, *q, *m;
  unsigned long long* id;
  unsigned long long* order;
  unsigned char* frozen;  // held lab-plane injection state
  double* beta;           // frozenBetaZ
};

constexpr int kTileShift = 0;  // sort granularity: single cells (2^0)

// CPML carriers.  `key` = (birth step + 1) << 32 | rank of the parent in
// the particle list, so sorting by key restores the reference's carrier
// order (survivors first, then newborns in particle order); storage order
// is free.
struct DCarriers {
  double *px, *py, *pz, *vx, *vy, *vz, *q, *w;
  unsigned long long* key;
};

// Per-trial counters of the boundary bookkeeping (src/simulation.cpp:
// 4841-4901, 4375-4383); cumulative counters live on the host.
struct TrialCounters {
  unsigned long long exits;
  double exit_charge;
  unsigned long long cpml[6];
  double cpml_charge[6];
  unsigned long long direct[6];
  double direct_charge[6];
  unsigned long long carrier_outer[6];
  double carrier_outer_charge[6];
  unsigned long long cropped;     // carriers beyond the window upper edge
  double cropped_charge;
  unsigned long long activations; // held particles crossing the activation plane
  unsigned long long held;        // held particles retained by the trial
  // Compaction sizes, so the commit needs no further host round trip.
  unsigned long long retained;    // particles with action 0
  unsigned long long born_kept;   // newborn carriers kept
  unsigned long long carriers_kept;  // existing carriers kept
};

struct ResidualSums {
  unsigned long long force_bits;  // max over particles (non-negative double bits)
  double defect;
  double scale;
  unsigned long long calls;       // pushed (seen) slots
};

// Per-slot record of one trial push (ConservativeSourceCoupling::Impl::Slot,
// src/source_coupling.cpp:19): where and when the push started and its dt
// (a held particle released mid-step is pushed from its activation kink for
// the remaining fraction of the step).
struct DSlots {
  double *x0, *y0, *z0;
  double* dt;
  unsigned char* seen;
};

// The argument blocks of the particle kernels are templated on the type F
// of J in the grid view (binary64 in both modes of this library).  Particle
// state, the push, the deposit and the boundary logic are binary64.
template <class F>
struct PushArgs {
  GridT<F> g;
  // What the gathers read, in their arithmetic type: the orbit sum
  // S = E_new + E^n per E node and B, both in the ring layout of E and B.
  const void* orbit[3];
  const void* bgather[3];
  DFrame frame;
  DRegion region;
  DMagnet magnets[kMaxMagnets];
  int n_magnets;
  int shape;
  int substeps;
  double time;           // box time at the start of the step
  double exit_lab_z;
  double activation_plane_lab_z;
  long long count;
  DParticles p;          // state at the start of the step (read only)
  double *x1, *y1, *z1, *ux1, *uy1, *uz1;  // state after the trial push
  unsigned char* frozen1;                  // held state after the trial
  DSlots slot;
  double* used_e;        // 3*count, written
  double* used_b;
  const double* next_e;  // 3*count, from the previous residual
  const double* next_b;
  double* abs_grid_work; // sum over substeps of |grid work|
  unsigned char* action; // 0 retain, 1 CPML/exit carrier, 2 outer exit
  DCarriers born;        // carrier created by a CPML entry (when kept)
  // linear-binomial3: the main chord, validated, for chord_deposit_kernel
  // (dep_mode 1; 0 when the particle deposits no main chord this trial)
  double* dep_b[3];
  double* dep_e[3];
  unsigned char* dep_mode;
  unsigned long long key_base;  // (step + 1) << 32 for newborn carrier keys
  unsigned char* born_keep;
  TrialCounters* counters;
  DeviceStatus* status;
};

template <class F>
struct CarrierArgs {
  GridT<F> g;
  DRegion region;
  int shape;
  long long count;
  DCarriers in;          // carriers at the start of the step
  DCarriers out;         // after this step's segment
  unsigned char* keep;
  TrialCounters* counters;
  DeviceStatus* status;
};

template <class F>
struct ResidualArgs {
  GridT<F> g;
  const void* orbit[3];     // as in PushArgs
  const void* bgather[3];
  int shape;
  long long count;
  DParticles p;
  DSlots slot;
  const double *x1, *y1, *z1;
  const double* used_e;
  const double* used_b;
  double* next_e;
  double* next_b;
  const double* abs_grid_work;
  ResidualSums* sums;
  // defect and scale per block; the last block to finish sums them in block
  // order (ticket counts the finished blocks and is left at zero).
  double* partial;
  unsigned* ticket;
  DeviceStatus* status;
};

// push_deposit_kernel leaves the main chords of linear-binomial3 particles
// to chord_deposit_kernel, in both current-summation modes.  On the dipole
// workload (1M particles, 128x128x512 cells) per trial: fused push and
// deposit 0.49 ms; push 0.13 ms + merged deposit 0.30 ms with binary64
// atomics; with the fixed-point sum, whose two integer reductions per
// contribution bound it, 1.13 ms fused against 0.14 + 0.65 ms.

// The deferred main chords of a linear-binomial3 trial.
struct ChordArgs {
  GridT<double> g;
  long long count;
  const unsigned char* mode;
  const double* b[3];
  const double* e[3];
  const double* q;
  DeviceStatus* status;
};

// Occupancy knobs of the hot particle kernels (blocks of 128 threads
// that must fit one SM; 0 leaves the register count to the compiler).
// Measured on the 128x128x512 dipole grid with 1M particles, with the
// kernels built per shape: push_deposit at 6 blocks (80 registers) beats 5,
// 7 and 8 on the binomial3, FP32-mixed and drift workloads and ties on
// quintic (binomial3 launch 0.133 -> 0.120 ms against 8 blocks, whose
// 64 registers spilled; with the main chords still deposited inside it, 8
// had been best); the residual and the guess gather at 6 blocks (80
// registers) beat 4, 5, 7 and 8 (dipole step 4.47 -> 4.44 ms, FP32-mixed
// 3.44 -> 3.35 ms, quintic 15.99 -> 15.62 ms).
#ifndef APRL_PUSH_MIN_BLOCKS
#define APRL_PUSH_MIN_BLOCKS 6
#endif
#ifndef APRL_RESIDUAL_MIN_BLOCKS
#define APRL_RESIDUAL_MIN_BLOCKS 6
#endif
#ifndef APRL_GATHER_MIN_BLOCKS
#define APRL_GATHER_MIN_BLOCKS 6
#endif
// chord_deposit is left to the compiler (96 registers, 5 blocks): at 6 or 8
// blocks it was unchanged; at 4 (118 registers) the dipole launch went
// 0.307 -> 0.302 ms but the drift one 0.048 -> 0.049 ms.
#ifndef APRL_CHORD_MIN_BLOCKS
#define APRL_CHORD_MIN_BLOCKS 0
#endif
#if APRL_CHORD_MIN_BLOCKS > 0
#define APRL_CHORD_BOUNDS __launch_bounds__(128, APRL_CHORD_MIN_BLOCKS)
#else
#define APRL_CHORD_BOUNDS __launch_bounds__(128)
#endif
#if APRL_GATHER_MIN_BLOCKS > 0
#define APRL_GATHER_BOUNDS __launch_bounds__(128, APRL_GATHER_MIN_BLOCKS)
#else
#define APRL_GATHER_BOUNDS
#endif
#if APRL_PUSH_MIN_BLOCKS > 0
#define APRL_PUSH_BOUNDS __launch_bounds__(128, APRL_PUSH_MIN_BLOCKS)
#else
#define APRL_PUSH_BOUNDS
#endif
#if APRL_RESIDUAL_MIN_BLOCKS > 0
#define APRL_RESIDUAL_BOUNDS __launch_bounds__(128, APRL_RESIDUAL_MIN_BLOCKS)
#else
#define APRL_RESIDUAL_BOUNDS
#endif

// W: arithmetic of the gathers (double, or float in the FP32-mixed mode).
// S: the particle shape, 0 linear-binomial3, 1 quintic-compensated.
template <class W, class F, int S> __global__ void guess_gather_kernel(PushArgs<F> a);
// Q: the deterministic mode's fixed-point current sum.
template <class F, int S, bool Q>
__global__ void APRL_PUSH_BOUNDS push_deposit_kernel(PushArgs<F> a);
template <class F, int S, bool Q> __global__ void carrier_kernel(CarrierArgs<F> a);
template <bool Q> __global__ void APRL_CHORD_BOUNDS chord_deposit_kernel(ChordArgs a);
template <class W, class F, int S>
__global__ void APRL_RESIDUAL_BOUNDS residual_kernel(ResidualArgs<F> a);

// RelativisticBorisPusher::push of `count` particles (SoA, in place) with
// per-particle E and B (3 values each).
struct BorisArgs {
  long long count;
  double *x, *y, *z, *ux, *uy, *uz;
  const double *q, *m, *e, *b;
  double dt;
};
__global__ void boris_push_kernel(BorisArgs a);

// Stable compaction helpers (warp ballot + block scan + block-offset scan).
constexpr int kScanBlock = 256;
__global__ void flag_count_kernel(const unsigned char* flag, unsigned char want,
                                  long long n, unsigned* block_count);
__global__ void block_offset_scan_kernel(const unsigned* block_count, int blocks,
                                         unsigned* block_offset,
                                         unsigned long long* total);
__global__ void gather_particles_kernel(DParticles out, DParticles src,
                                        const double* x1, const double* y1,
                                        const double* z1, const double* ux1,
                                        const double* uy1, const double* uz1,
                                        const unsigned char* frozen1,
                                        const unsigned char* flag, unsigned char want,
                                        long long n, const unsigned* block_offset);
__global__ void gather_carriers_kernel(DCarriers out, DCarriers src,
                                       const unsigned char* flag, unsigned char want,
                                       long long n, const unsigned* block_offset,
                                       unsigned long long base);
// Stable radix sort of the particle storage by cell (8-bit digits).
constexpr int kRadixBins = 256;
constexpr int kRadixThreads = 256;  // one thread per digit in the scatter's prefix
constexpr int kRadixItems = 8;
constexpr int kRadixTile = kRadixThreads * kRadixItems;
static_assert(kRadixThreads == kRadixBins, "radix_scatter_kernel: one thread per digit");
__global__ void sort_key_kernel(DParticles p, long long n, DGrid g, int tiles_x, int tiles_y,
                                unsigned* key, unsigned* index);
__global__ void radix_count_kernel(const unsigned* key, long long n, int shift, unsigned* count);
__global__ void radix_scatter_kernel(const unsigned* key_in, const unsigned* index_in,
                                     unsigned* key_out, unsigned* index_out, long long n,
                                     int shift, const unsigned* offset);
__global__ void permute_particles_kernel(DParticles out, DParticles src, long long n,
                                         const unsigned* index);
__global__ void chunk_scan_kernel(const unsigned* in, long long n, unsigned* out,
                                  unsigned* chunk_sum);
__global__ void chunk_add_kernel(unsigned* data, long long n, const unsigned* chunk_offset);
// Pending queue (PendingParticleQueue) on the device: particles sorted by
// their due step, initial state.
struct DPending {
  double *x, *y, *z, *ux, *uy, *uz, *q, *m, *beta;
  unsigned long long* id;
};
__global__ void admit_kernel(DParticles out, long long first_slot, DPending src,
                             long long begin, long long count, unsigned long long steps,
                             double held_distance_per_beta, unsigned long long first_order);
template <class F>
struct SupportArgs {
  GridT<F> g;
  int shape;
  DPending src;
  long long begin, count;
  unsigned long long steps;      // step - initial step
  double held_distance_per_beta; // c*dt
  DeviceStatus* status;
};
template <class F, int S, bool Q> __global__ void frozen_support_kernel(SupportArgs<F> a);
__global__ void crop_flags_kernel(DCarriers c, long long n, double upper,
                                  double lower, unsigned char* keep,
                                  TrialCounters* counters, DeviceStatus* status);
// finishMovingWindowStep's guard (src/simulation_moving_window.cpp:358-359):
// an active particle may not fall behind the inlet; held ones may.
__global__ void inlet_check_kernel(const double* z, const unsigned char* frozen, long long n,
                                   double origin, DeviceStatus* status);
// The inlet-layer charge of the charge-matched inlet (ChargeMatchedInlet::particle,
// src/charge_matched_inlet.h:31-53) from the stored particles and the
// pending entries [pbegin, pbegin + pcount) at their held positions of step
// `steps` after the queue's first.
struct InletMatchArgs {
  DParticles p;
  long long np;
  DPending src;
  long long pbegin, pcount;
  unsigned long long steps;
  double held_distance_per_beta;
  double origin[3];
  double dx, dy, dz;
  int nx, ny, shape;
  double* rho;                 // (nx+1) x (ny+1) node plane
  // Deterministic mode: the charge goes into these (lo, hi) word pairs
  // instead (fixed_add with rho_scale), converted by fixed_convert_kernel.
  unsigned long long* rho_pairs;
  double rho_scale;
  DeviceStatus* status;
};
__global__ void inlet_charge_kernel(InletMatchArgs a);

// A trial's start: J, the trial counters and the residual sums cleared
// (skipped with the trial).
// clear_current: 1 clears J; in the deterministic mode 2 clears the
// fixed-point pairs of J instead (J is then written by current_convert).
__global__ void trial_clear_kernel(GridT<double> g, TrialCounters* counters, ResidualSums* sums,
                                   int clear_current);
// Deterministic mode: J from its fixed-point pairs, every node.
__global__ void current_convert_kernel(GridT<double> g, double unscale);
// out[i] = value of pair i (fixed_value), for i < n.
__global__ void fixed_convert_kernel(const unsigned long long* pairs, double* out, long long n,
                                     double unscale);
// solveConservativeSourceStep's stopping rule (src/simulation_source_coupling.cpp:50)
// applied to trial `iterations`' residual sums: on convergence *stop = iterations.
__global__ void trial_verdict_kernel(const ResidualSums* sums, unsigned iterations,
                                     double force_tolerance, double work_tolerance, int* stop);

}  // namespace aprl_gpu
