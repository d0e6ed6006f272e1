// run.cu -- host runtime and C ABI of the B200 PIC step (include/aprl_gpu.h).
//
// An aprl_run owns all device state of one moving-window run and drives the
// kernels of fields.cu and particles.cu on its stream in the reference's
// step order (src/simulation.cpp:493-613,
// src/simulation_source_coupling.cpp:16-65): inlet halos and the Cowan B
// update, the zero-current E preview, fixed-point trials (carriers, push +
// deposit, residual) until force < 1e-13 and work < 1e-8 after at least two
// trials, the commit E^{n+1} = E* - dt/eps0 J with stable particle/carrier
// compaction, and the ring-buffer window shift.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/aprl_gpu.h"
#include "common.cuh"
#include "fields.cuh"
#include "ledger.cuh"
#include "particles.cuh"
#include "selffield.cuh"

using namespace aprl_gpu;

namespace {

thread_local std::string g_error;

aprl_status fail(aprl_status s, const char* format, ...) {
  char buffer[640];
  va_list args;
  va_start(args, format);
  vsnprintf(buffer, sizeof buffer, format, args);
  va_end(args);
  g_error = buffer;
  return s;
}

#define CUDA_TRY(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess)                                                      \
      return fail(APRL_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

enum Kernel : unsigned {
  kInletLower, kCowanMagnetic, kElectricPreview, kCarrier, kPushDeposit,
  kResidual, kElectricCommit, kFlagCount, kBlockScan, kGatherParticles,
  kGatherCarriers, kShiftInsert, kCropFlags, kInletCheck, kDetectorPlane,
  kSortKey, kChunkScan, kChunkAdd, kRadixScatter, kAdmit, kFrozenSupport,
  kGuessGather, kOrbitSum, kBShadow, kLedgerPartial, kLedgerFinish,
  kGaussDeposit, kGaussResidual, kGaussFinish, kTrialClear, kTrialVerdict,
  kSfMoments, kSfFinish, kSfDeposit, kSfSource, kSfApply, kSfUpdate,
  kSfDirection, kSfSmooth, kSfElectric, kSfMagnetic, kSfClear, kSfGauss, kSfEnergy,
  kInletHalo, kInletCharge, kInletComplete, kRadixCount, kPermuteParticles,
  kCurrentConvert, kFixedConvert, kChordDeposit, kSfModal, kSurfaceCurrent, kSfOpen, kKernelCount
};

const char* kKernelNames[kKernelCount] = {
  "inlet_lower", "cowan_magnetic", "electric_preview", "carrier",
  "push_deposit", "residual", "electric_commit", "flag_count",
  "block_offset_scan", "gather_particles", "gather_carriers",
  "shift_insert", "crop_flags", "inlet_check", "detector_plane",
  "sort_key", "chunk_scan", "chunk_add", "radix_scatter", "admit",
  "frozen_support", "guess_gather", "orbit_sum", "b_shadow", "ledger_partial",
  "ledger_finish", "gauss_deposit", "gauss_residual", "gauss_finish", "trial_clear",
  "trial_verdict", "sf_moments", "sf_finish", "sf_deposit", "sf_source", "sf_apply",
  "sf_update", "sf_direction", "sf_smooth", "sf_electric", "sf_magnetic",
  "sf_clear", "sf_gauss", "sf_energy", "inlet_halo", "inlet_charge", "inlet_complete",
  "radix_count", "permute_particles", "current_convert", "fixed_convert", "chord_deposit", "sf_modal", "surface_current", "sf_open"};

const char* device_error_text(unsigned code) {
  switch (code) {
    case kErrCrossingBudget: return "Quintic orbit exceeds crossing budget";
    case kErrOrbitOutside: return "Active coupling orbit has no in-domain portion";
    case kErrDepositOutside: return "Particle trajectory endpoint is outside the E/B domain";
    case kErrSupportX: return "Transverse current support outside x grid";
    case kErrSupportY: return "Transverse current support outside y grid";
    case kErrRootNonphysical: return "Nonphysical local mean-gamma root";
    case kErrRootNoConvergence: return "Local mean-gamma root did not converge";
    case kErrNonFinite: return "Particle trajectory contains a non-finite coordinate";
    case kErrStartInCpml: return "Active particle starts inside the non-physical CPML region";
    case kErrStartOutside: return "Particle trajectory starts outside the global E/B domain";
    case kErrBeyondExit: return "Active particle started beyond trusted moving-window exit";
    case kErrUpstream: return "An active particle is upstream of the moving window";
    case kErrCarrierWeight: return "Invalid CPML carrier current weight";
    case kErrFellBehind: return "Active particle fell behind moving inlet";
    case kErrReferenceRange: return "Moving reference query outside prepared native field";
    case kErrHitLocate: return "Cannot locate the first particle boundary crossing";
    case kErrEarlyRelease:
      return "A pending upstream held particle would release before a complete in-window step";
    case kErrAdmission:
      return "Moving-window upstream admission requires an unreleased held particle on rank zero";
    case kErrHeldBoundary:
      return "Held-transverse activation crossed a particle boundary during the frozen part of a field step";
    case kErrInletSource: return "Nonfinite charge-matched inlet source";
    case kErrInletField: return "Nonfinite charge-matched inlet field";
    case kErrFixedRange:
      return "Deposit contribution beyond the deterministic fixed-point range";
    case kErrSurfaceCurrent: return "Nonfinite equivalent boundary current";
    case kErrReferenceSupport: return "Reference charge support touches Dirichlet surface";
    case kErrReferenceSource: return "Nonfinite quintic reference source";
    case kErrReferenceCharge: return "Nonfinite quintic reference charge";
    case kErrBounds:
      return "Array index outside its array (bounds-checked build)";
  }
  return "unknown device error";
}

aprl_status device_error_status(unsigned code) {
  switch (code) {
    case kErrOrbitOutside: case kErrDepositOutside: case kErrSupportX:
    case kErrSupportY: case kErrStartInCpml: case kErrStartOutside:
    case kErrReferenceRange: case kErrBounds:
      return APRL_ERR_OUT_OF_RANGE;
    case kErrReferenceSupport: case kErrReferenceSource: case kErrReferenceCharge:
      return APRL_ERR_INVALID_ARGUMENT;
    default:
      return APRL_ERR_RUNTIME;
  }
}

// EBCowanCoefficients::forZDispersion (src/eb_field.cpp:33-73).
aprl_status cowan(double dx, double dy, double dz, double out[12]) {
  if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0) || !std::isfinite(dx) ||
      !std::isfinite(dy) || !std::isfinite(dz))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Cowan-z grid spacing must be positive and finite");
  const double tolerance = 64.0 * DBL_EPSILON * std::max(dx, std::max(dy, dz));
  if (dx + tolerance < dz || dy + tolerance < dz)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Cowan-z requires dz to be the smallest grid spacing");
  const double rx = (dz / dx) * (dz / dx), ry = (dz / dy) * (dz / dy), rz = 1.0;
  const double den = rx * ry + ry * rz + rz * rx;
  if (!(den > 0.0) || !std::isfinite(den))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid Cowan-z aspect ratios");
  const double pf = rx * ry * rz / den;
  double beta[3] = {rx * (1.0 - pf) / 8.0, ry * (1.0 - pf) / 8.0, rz * (1.0 - pf) / 8.0};
  const double dxy = rx * ry * (1.0 / 16.0 - rx * ry / (8.0 * den));
  const double dyz = ry * rz * (1.0 / 16.0 - ry * rz / (8.0 * den));
  const double dzx = rz * rx * (1.0 / 16.0 - rz * rx / (8.0 * den));
  out[0] = 1.0 - 2.0 * beta[1] - 2.0 * beta[2] - 4.0 * dyz;
  out[1] = 1.0 - 2.0 * beta[2] - 2.0 * beta[0] - 4.0 * dzx;
  out[2] = 1.0 - 2.0 * beta[0] - 2.0 * beta[1] - 4.0 * dxy;
  out[3] = beta[0]; out[4] = beta[1]; out[5] = beta[2];
  out[6] = dxy; out[7] = dyz; out[8] = dzx;
  out[9] = rx; out[10] = ry; out[11] = rz;
  return APRL_OK;
}

struct HostProfile {  // makeProfile result for one axis
  std::vector<double> ikm1, decay, drive;
  std::vector<int> ordinal;
  int active = 0;
};

// EBCPMLParameters::maximumConductivityRate (src/eb_cpml.cpp:277-294).
double maximum_rate(const aprl_run_config& g, int axis) {
  const uint64_t cells = axis == 0 ? g.cpml_cells_x : (axis == 1 ? g.cpml_cells_y : 0);
  if (cells == 0) return 0.0;
  const double spacing = axis == 0 ? g.dx : (axis == 1 ? g.dy : g.dz);
  const double thickness = static_cast<double>(cells) * spacing;
  return -(g.cpml_polynomial_order + 1.0) * kC * std::log(g.cpml_target_reflection) /
         (2.0 * thickness);
}

// makeProfile (src/eb_cpml.cpp:195-248) at one rank.
HostProfile make_profile(const aprl_run_config& g, int axis, bool electric) {
  HostProfile r;
  const size_t local = axis == 0 ? g.nx : g.ny;
  const size_t count = local + (electric ? 1 : 0);
  r.ikm1.assign(count, 0.0);
  r.decay.assign(count, 0.0);
  r.drive.assign(count, 0.0);
  r.ordinal.assign(count, -1);
  const size_t thickness_cells = axis == 0 ? g.cpml_cells_x : g.cpml_cells_y;
  if (thickness_cells == 0) return r;
  const double thickness = static_cast<double>(thickness_cells);
  const double sigma_max = maximum_rate(g, axis);
  for (size_t index = 0; index < count; ++index) {
    const double position = static_cast<double>(index) + (electric ? 0.0 : 0.5);
    double depth = 0.0;
    if (position < thickness) depth = (thickness - position) / thickness;
    const double upper_start = static_cast<double>(local - thickness_cells);
    if (position > upper_start) depth = std::max(depth, (position - upper_start) / thickness);
    if (!(depth > 0.0)) continue;
    depth = std::min(1.0, depth);
    const double graded = std::pow(depth, g.cpml_polynomial_order);
    const double sigma = sigma_max * graded;
    const double kappa = 1.0 + (g.cpml_kappa_max - 1.0) * graded;
    const double alpha = g.cpml_alpha_fraction * sigma_max * (1.0 - depth);
    r.ikm1[index] = 1.0 / kappa - 1.0;
    r.decay[index] = std::exp(-(sigma / kappa + alpha) * g.dt);
    const double den = sigma * kappa + alpha * kappa * kappa;
    r.drive[index] = den > 0.0 ? sigma * (r.decay[index] - 1.0) / den : 0.0;
    r.ordinal[index] = r.active++;
  }
  return r;
}

struct DeviceProfile {
  double *ikm1 = nullptr, *decay = nullptr, *drive = nullptr;
  int* ordinal = nullptr;
  int active = 0;
  CpmlAxis view() const { return CpmlAxis{ikm1, decay, drive, ordinal}; }
};

// One of the 8 active histories.  component: ABI index (0..5); derivative
// axis 0/1; the history's k ring follows its component's ring.
struct HistoryBuffer {
  double* data = nullptr;
  int slots = 0, layers = 0, row = 0;
  int component = 0;
  int abi_index = 0;
  size_t length() const { return (size_t)slots * layers * row; }
  CpmlHistory view() const { return CpmlHistory{data, slots, layers, row}; }
};

struct Timing {
  cudaEvent_t start, stop;
  unsigned kernel;
};

}  // namespace

// Fixed-point trials issued per step before the host reads any residual
// (the usual count at FP64; FP32-mixed runs usually stop after two).
constexpr unsigned kTrialSlots = 3;

// Steps between the cell sorts of the particle list (see do_commit).
constexpr uint64_t kSortInterval = 4;

// A launch of the autotuner's measurements, harvested after the next wait.
struct TunePending {
  int kernel;
  int candidate;
  cudaEvent_t start, stop;
};

struct aprl_run {
  aprl_run_config cfg{};
  std::string error;  // the message of this run's failure in aprl_runs_step
  int device = 0;
  int tune_choice[4] = {-1, -1, -1, -1};  // autotuner choices seen by this run
  std::vector<TunePending> tune_pending;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;   // device memory (device_pool of the run's device)
  void* pinned = nullptr;         // the page-locked block the h_* read-backs live in
  // The CPML carriers of a trial run on `side`, forked from `stream` after
  // the trial's clear and joined before the orbit sum that reads J, so their
  // short, latency-bound launch overlaps the particles' push.
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // Reference planes set with aprl_run_set_reference_planes cross PCIe on
  // `upload`, into a staging buffer, as soon as they are given; the run's
  // stream then copies them device to device into the table at the call's
  // place in its own order (after the slot's `staged` event), so the
  // transfer overlaps the work already queued.  Two slots per component
  // take turns; `drained` marks the stream's copy out of a slot, which the
  // next transfer into that slot waits for.
  struct Stage {
    double* data = nullptr;
    size_t bytes = 0;
    cudaEvent_t staged = nullptr, drained = nullptr;
    bool used = false;
  };
  cudaStream_t upload = nullptr;
  Stage staging[6][2];
  int staging_next[6] = {};
  double coeff[12]{};
  // E, B and J are binary64 in both modes (`fes`: J element size); the
  // FP32-mixed mode runs the gathers in binary32.
  bool fp32 = false;
  size_t fes = 8;
  double* e[2][3]{};
  int cur = 0;  // e[cur] = E^n (committed), e[1-cur] = E*
  double* b[3]{};
  void* jc[3]{};
  // J is known to be zero everywhere (set by a clear, kept by a trial that
  // deposits nothing): the next clear and the commit's pass over J are
  // skipped, which is most of a field-only step's work besides the field
  // updates.
  bool j_zero = true;
  // The preview of this step wrote the current-free orbit sum.
  bool orbit_from_preview = false;
  double* lower[3]{};
  // What the gathers read: the orbit sum S = E_new + E^n per E node (binary64,
  // or binary32 in the FP32-mixed mode) and, in that mode, a binary32 B.
  void* orbit[3]{};
  float* bshadow[3]{};
  int zb_e[3]{}, zb_b[3]{};
  double* ref[6]{};
  bool ref_set[6]{};
  double* inlet_rho = nullptr;  // charge-matched inlet: the inlet-layer charge plane
  DeviceProfile mprof[2], eprof[2];
  HistoryBuffer hist[8];  // ABI indices 0,3,4,5,6,9,10,11
  double max_rate[3]{};
  // particles
  size_t np = 0, pcap = 0;
  DParticles p{}, p_alt{};
  double *x1 = nullptr, *y1 = nullptr, *z1 = nullptr, *ux1 = nullptr, *uy1 = nullptr,
         *uz1 = nullptr;
  double *used_e = nullptr, *used_b = nullptr, *next_e = nullptr, *next_b = nullptr;
  double* abs_work = nullptr;
  // linear-binomial3: each particle's validated main chord of the trial,
  // deposited by chord_deposit_kernel after the push
  double* dep_b[3]{};
  double* dep_e[3]{};
  unsigned char* dep_mode = nullptr;
  unsigned char* action = nullptr;
  DCarriers born{};
  unsigned char* born_keep = nullptr;
  size_t nslot = 0;
  unsigned long long* slot_order = nullptr;  // p.order at the last preview
  unsigned long long next_order = 0;
  unsigned char* frozen1 = nullptr;           // held state after a trial
  DSlots slots{};                             // per-slot push start (kinks)
  // held lab-plane injection: PendingParticleQueue at one rank
  struct Queue {
    bool extracted = false;
    uint64_t initial_step = 0, last_step = 0, maximum_step = 0, next_due = 0;
    size_t n = 0, cursor = 0;
    std::vector<size_t> offsets;  // bucket b = due step - initial_step
    DPending d{};                 // entries in due order
  } queue;
  uint64_t admitted = 0;
  uint64_t held = 0;              // frozen particles in the list
  // cell sort scratch: keys and storage indices (two of each for the radix
  // passes), per-block digit counts and their chunk sums
  unsigned *sort_key[2]{}, *sort_index[2]{};
  unsigned *radix_count = nullptr, *chunk_sum = nullptr, *chunk_offset = nullptr;
  size_t ntiles = 0;
  int tiles[3]{};
  int sort_bits = 0;
  // Deterministic mode (aprl_run_config.deterministic): J's fixed-point
  // (lo, hi) pairs, the scale that maps the largest possible contribution
  // below 2^61 (a power of two), and the largest |charge| uploaded so far.
  bool deterministic = false;
  unsigned long long* jq[3]{};
  double jq_scale = 1.0;
  double max_abs_charge = 0.0;
  unsigned long long* inlet_rho_pairs = nullptr;
  // the reference's equivalent surface current: target points (i, j) and
  // curl_z(B_ref)/mu0 per reference plane and point
  unsigned* surface_points = nullptr;
  double* surface_table = nullptr;
  size_t surface_count = 0;
  bool surface_ready = false;
  // residual block partials (defect, scale) and the finished-block ticket
  double* res_partial = nullptr;
  unsigned* res_ticket = nullptr;
  size_t res_blocks = 0;
  // carriers
  size_t nc = 0, ccap = 0;
  DCarriers c{}, c_alt{}, c_out{};
  unsigned char* c_keep = nullptr;
  // reductions, counters, status, scan scratch
  TrialCounters* d_counters = nullptr;
  ResidualSums* d_sums = nullptr;
  DeviceStatus* d_status = nullptr;
  unsigned* scan_count = nullptr;
  unsigned* scan_offset = nullptr;
  unsigned long long* scan_total = nullptr;
  size_t scan_cap = 0;
  // pinned host mirrors
  ResidualSums* h_sums = nullptr;        // the slot of the last trial read
  ResidualSums* h_sums_slots = nullptr;  // one slot per trial issued ahead of a read
  TrialCounters* h_counters_slots = nullptr;
  int* d_stop = nullptr;                 // device verdict of the trials issued ahead
  int* h_stop = nullptr;
  DeviceStatus* h_status = nullptr;
  TrialCounters* h_counters = nullptr;
  unsigned long long* h_total = nullptr;
  TrialCounters cumulative{};
  // window state
  uint64_t step = 0;
  int64_t offset = 0;
  double time = 0.0;
  double origin[3]{};
  int stage = 0;
  bool step_open = false;  // aprl_run_step_begin without its aprl_run_step_end yet
  unsigned trials = 0;
  uint32_t last_iterations = 0, max_iterations = 0;
  uint64_t total_iterations = 0;
  double last_force = 0.0, last_work = 0.0;
  // detector scratch
  double* d_detector = nullptr;
  size_t detector_cap = 0;
  // energy ledger (ledger.cuh): device state, block partials, and Ex/Ey of
  // plane 0 before the inlet overwrite (written by the preview)
  bool ledger_on = false;
  bool ledger_start_ready = false;  // the last shift already took the start power
  DLedger* d_ledger = nullptr;
  DD* d_ledger_partial = nullptr;
  double* ledger_pre[2]{};
  // Gauss-law scratch: node array, then block partials, results and maxima
  double* gauss_node = nullptr;
  unsigned char* gauss_scratch = nullptr;
  // profiling
  bool profile = false;
  std::vector<Timing> pending;
  std::vector<cudaEvent_t> event_pool;
  double kernel_ms[kKernelCount]{};
  uint64_t kernel_launches[kKernelCount]{};
  uint64_t launches = 0;
};

namespace {

// Device memory of every run comes from one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the run's stream).  Memory a
// run frees goes back to the pool and the next run reuses it, so creating
// and destroying runs -- once per request in the scan server -- maps and
// unmaps no device memory: with cudaMalloc/cudaFree that took 0.4-1.5 s for
// some large runs and varied several-fold from call to call.  A block is
// reused only once its free has completed on the GPU or the allocating stream
// is already ordered after it (no opportunistic reuse).  Up to kPoolKeepBytes
// of freed memory stay in the pool; the driver releases the rest at the next
// synchronisation.
constexpr uint64_t kPoolKeepBytes = 16ull << 30;

cudaMemPool_t device_pool(int device) {
  static std::mutex lock;
  static std::vector<cudaMemPool_t> pools;
  std::lock_guard<std::mutex> hold(lock);
  if (device < 0) return nullptr;
  if ((size_t)device >= pools.size()) pools.resize(device + 1, nullptr);
  if (!pools[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = kPoolKeepBytes;
    int no = 0;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess ||
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &no) != cudaSuccess ||
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no) !=
            cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return nullptr;
    }
    pools[device] = pool;
  }
  return pools[device];
}

// The allocation is waited for on the run's stream, so the block is valid for
// every stream and for the synchronous copies that fill it (allocations are
// made outside the step loop, or on a stream that is idle anyway).
aprl_status device_alloc_bytes(aprl_run* r, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 8;
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, r->pool, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(APRL_ERR_CUDA, "device allocation of %zu bytes failed: %s", bytes,
                cudaGetErrorString(e));
  }
  return APRL_OK;
}

template <class T>
aprl_status device_alloc(aprl_run* r, T** p, size_t count) {
  void* v = nullptr;
  const aprl_status s = device_alloc_bytes(r, &v, (count ? count : 1) * sizeof(T));
  *p = static_cast<T*>(v);
  return s;
}

// Back to the pool in stream order (after the work queued on the run's stream).
void device_free(aprl_run* r, void* p) {
  if (p) cudaFreeAsync(p, r->stream);
}

// Every copy and fill of a run goes through the run's stream.  A plain
// cudaMemcpy or cudaMemset runs on the legacy default stream, which the
// run's (possibly non-blocking) stream does not wait for, and returns before
// a device-to-device copy or a fill is done; a stream-ordered free of the
// source right after it could then hand the block to another run while the
// copy still reads it.  A copy returns once it has completed, as its callers
// expect (host buffers are reused or read right after).
cudaError_t run_copy(aprl_run* r, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  return e;
}
cudaError_t run_fill(aprl_run* r, void* dst, int value, size_t bytes) {
  return cudaMemsetAsync(dst, value, bytes, r->stream);
}

// Page-locked 4 KiB blocks for the runs' small read-back areas, kept for
// reuse (cudaMallocHost/cudaFreeHost per run cost milliseconds each).
constexpr size_t kPinnedBlock = 4096;

static_assert(kTrialSlots * sizeof(ResidualSums) + sizeof(DeviceStatus) +
                      kTrialSlots * sizeof(TrialCounters) + sizeof(int) +
                      sizeof(unsigned long long) + 5 * 64 <= kPinnedBlock,
              "read-back areas exceed the pinned block");

std::mutex& pinned_lock() {
  static std::mutex lock;
  return lock;
}
std::vector<void*>& pinned_free() {
  static std::vector<void*> blocks;
  return blocks;
}

void* pinned_take() {
  {
    std::lock_guard<std::mutex> hold(pinned_lock());
    if (!pinned_free().empty()) {
      void* b = pinned_free().back();
      pinned_free().pop_back();
      return b;
    }
  }
  void* b = nullptr;
  if (cudaMallocHost(&b, kPinnedBlock) != cudaSuccess) return nullptr;
  return b;
}

void pinned_give(void* b) {
  if (!b) return;
  std::lock_guard<std::mutex> hold(pinned_lock());
  pinned_free().push_back(b);
}

size_t e_count(const aprl_run_config& g, int c) {
  return (size_t)(g.nx + (c != 0)) * (g.ny + (c != 1)) * (g.nz + (c != 2));
}
size_t b_count(const aprl_run_config& g, int c) {
  return (size_t)(g.nx + (c == 0)) * (g.ny + (c == 1)) * (g.nz + (c == 2));
}
void comp_shape(const aprl_run_config& g, unsigned a, size_t s[3]) {
  const bool electric = a < 3 || a >= 6;
  const unsigned axis = a % 3;
  const size_t cells[3] = {g.nx, g.ny, g.nz};
  for (unsigned d = 0; d < 3; ++d) s[d] = cells[d] + (electric ? (d != axis) : (d == axis));
}

// True when every value is finite.  A binary64 is non-finite exactly when its
// 11 exponent bits are all ones; adding one to that field then carries into
// bit 11.  The branch-free OR over a chunk vectorises with plain SSE2
// integer ops, so a host inlet plane is checked at memory speed rather than
// one compare-and-branch per value.
bool all_finite(const double* v, size_t n) {
  constexpr size_t kChunk = 4096;
  for (size_t lo = 0; lo < n; lo += kChunk) {
    const size_t hi = std::min(n, lo + kChunk);
    uint64_t bad = 0;
    for (size_t i = lo; i < hi; ++i) {
      uint64_t bits;
      std::memcpy(&bits, v + i, 8);
      bad |= (((bits >> 52) & 0x7ffu) + 1u) >> 11;
    }
    if (bad) return false;
  }
  return true;
}

cudaEvent_t take_event(aprl_run* r) {
  if (!r->event_pool.empty()) {
    cudaEvent_t e = r->event_pool.back();
    r->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

aprl_status drain_timings(aprl_run* r) {
  for (auto& t : r->pending) {
    CUDA_TRY(cudaEventSynchronize(t.stop));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, t.start, t.stop));
    r->kernel_ms[t.kernel] += ms;
    r->event_pool.push_back(t.start);
    r->event_pool.push_back(t.stop);
  }
  r->pending.clear();
  return APRL_OK;
}

// Launch on `stream` with optional stage timing.
template <class K, class... Args>
aprl_status launch_on(aprl_run* r, cudaStream_t stream, unsigned id, K kernel, dim3 grid,
                      dim3 block, Args... args) {
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return APRL_OK;
  Timing t{};
  if (r->profile) {
    t.start = take_event(r);
    t.stop = take_event(r);
    t.kernel = id;
    CUDA_TRY(cudaEventRecord(t.start, stream));
  }
  kernel<<<grid, block, 0, stream>>>(args...);
  CUDA_TRY(cudaGetLastError());
  if (r->profile) {
    CUDA_TRY(cudaEventRecord(t.stop, stream));
    r->pending.push_back(t);
  }
  ++r->kernel_launches[id];
  ++r->launches;
  return APRL_OK;
}

// Launch on the run's stream.
template <class K, class... Args>
aprl_status launch(aprl_run* r, unsigned id, K kernel, dim3 grid, dim3 block, Args... args) {
  return launch_on(r, r->stream, id, kernel, grid, block, args...);
}

#define TRY(expr)                    \
  do {                               \
    aprl_status s_ = (expr);         \
    if (s_ != APRL_OK) return s_;    \
  } while (0)

// ---- autotuner -------------------------------------------------------------
// The launch shapes of the grid kernels are chosen by measurement, per device
// and grid extent: the Cowan magnetic kernel's z planes per block and the
// thread-block shape of the preview, orbit-sum and commit kernels.  Every
// candidate computes each node exactly as the others do (one thread per node,
// or the same plane ring over a different split of z), so a choice changes
// timing only, never a bit of a result.  While a grid extent has no choice
// yet, the runs on it launch the candidates in turn -- each a real launch of
// the step, timed with CUDA events and read after the step's own wait -- and
// once every candidate has two samples the one with the smallest sample
// becomes the choice for every later launch of every run of that extent in
// the process.
enum TunedKernel { kTuneCowan = 0, kTunePreview, kTuneOrbit, kTuneCommit, kTuneCount };
constexpr int kTuneCandidates = 4;
constexpr int kTuneSamples = 2;
constexpr int kCowanChunks[kTuneCandidates] = {2, 4, 8, 16};
const dim3 kGridBlocks[kTuneCandidates] = {dim3(32, 4), dim3(32, 8), dim3(64, 2), dim3(64, 4)};

struct TuneKey {
  int device, kernel;
  uint64_t nx, ny, nz;
  bool operator<(const TuneKey& o) const {
    if (device != o.device) return device < o.device;
    if (kernel != o.kernel) return kernel < o.kernel;
    if (nx != o.nx) return nx < o.nx;
    if (ny != o.ny) return ny < o.ny;
    return nz < o.nz;
  }
};

struct TuneEntry {
  float best[kTuneCandidates] = {0.f, 0.f, 0.f, 0.f};
  int samples[kTuneCandidates] = {0, 0, 0, 0};
  int choice = -1;
};

std::mutex& tune_lock() {
  static std::mutex m;
  return m;
}
std::map<TuneKey, TuneEntry>& tune_table() {
  static std::map<TuneKey, TuneEntry> t;
  return t;
}

TuneKey tune_key(const aprl_run* r, int kernel) {
  return TuneKey{r->device, kernel, r->cfg.nx, r->cfg.ny, r->cfg.nz};
}

// The candidate for this launch of `kernel`; *timed is set when the launch
// is a measurement.
int tune_pick(aprl_run* r, int kernel, bool* timed) {
  *timed = false;
  if (r->tune_choice[kernel] >= 0) return r->tune_choice[kernel];
  std::lock_guard<std::mutex> lock(tune_lock());
  TuneEntry& e = tune_table()[tune_key(r, kernel)];
  if (e.choice >= 0) {
    r->tune_choice[kernel] = e.choice;
    return e.choice;
  }
  int pending[kTuneCandidates] = {0, 0, 0, 0};
  for (const auto& p : r->tune_pending)
    if (p.kernel == kernel) ++pending[p.candidate];
  int pick = 0;
  for (int c = 1; c < kTuneCandidates; ++c)
    if (e.samples[c] + pending[c] < e.samples[pick] + pending[pick]) pick = c;
  *timed = true;
  return pick;
}

// Reads the measurements whose launches have completed.
void tune_harvest(aprl_run* r) {
  if (r->tune_pending.empty()) return;
  std::vector<TunePending> still;
  std::lock_guard<std::mutex> lock(tune_lock());
  for (auto& p : r->tune_pending) {
    if (cudaEventQuery(p.stop) != cudaSuccess) {
      still.push_back(p);
      continue;
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
      TuneEntry& e = tune_table()[tune_key(r, p.kernel)];
      if (e.samples[p.candidate] == 0 || ms < e.best[p.candidate]) e.best[p.candidate] = ms;
      ++e.samples[p.candidate];
      if (e.choice < 0) {
        bool complete = true;
        int best = 0;
        for (int c = 0; c < kTuneCandidates; ++c) {
          complete = complete && e.samples[c] >= kTuneSamples;
          if (e.best[c] < e.best[best]) best = c;
        }
        if (complete) e.choice = best;
      }
    }
    r->event_pool.push_back(p.start);
    r->event_pool.push_back(p.stop);
  }
  (void)cudaGetLastError();  // a not-ready query leaves no error behind
  r->tune_pending.swap(still);
}

// A tuned launch: tune_begin picks the candidate (and starts a measurement
// when the choice is still open); the caller launches with that candidate's
// shape; tune_end closes the measurement.
struct TuneLaunch {
  int kernel = 0, candidate = 0;
  bool timed = false;
  cudaEvent_t start = nullptr, stop = nullptr;
};

aprl_status tune_begin(aprl_run* r, int kernel, TuneLaunch& t) {
  t.kernel = kernel;
  t.candidate = tune_pick(r, kernel, &t.timed);
  if (t.timed) {
    t.start = take_event(r);
    t.stop = take_event(r);
    CUDA_TRY(cudaEventRecord(t.start, r->stream));
  }
  return APRL_OK;
}

aprl_status tune_end(aprl_run* r, const TuneLaunch& t) {
  if (!t.timed) return APRL_OK;
  CUDA_TRY(cudaEventRecord(t.stop, r->stream));
  r->tune_pending.push_back(TunePending{t.kernel, t.candidate, t.start, t.stop});
  return APRL_OK;
}

// Device view of the grid in the run's field element type F.
template <class F>
GridT<F> make_grid(const aprl_run* r) {
  GridT<F> g{};
  g.nx = (int)r->cfg.nx;
  g.ny = (int)r->cfg.ny;
  g.nz = (int)r->cfg.nz;
  g.dx = r->cfg.dx;
  g.dy = r->cfg.dy;
  g.dz = r->cfg.dz;
  g.dt = r->cfg.dt;
  for (int a = 0; a < 3; ++a) {
    g.origin[a] = r->origin[a];
    g.e_old[a] = r->e[r->cur][a];
    g.e_star[a] = r->e[1 - r->cur][a];
    g.b[a] = r->b[a];
    g.j[a] = static_cast<F*>(r->jc[a]);
    g.zb_e[a] = r->zb_e[a];
    g.zb_b[a] = r->zb_b[a];
  }
  g.jcoef = F(-1. * r->cfg.dt / kEpsilon0);
  g.status = r->d_status;
  if (r->deterministic) {
    for (int a = 0; a < 3; ++a) g.jq[a] = r->jq[a];
    g.jq_scale = r->jq_scale;
  }
  return g;
}

// The fixed-point scale of the deterministic mode: a power of two 2^e with
// bound * 2^e < 2^61, where `bound` exceeds any single contribution the run
// can make.  A deposit visit adds q * (dx_a / dt) / (dx dy dz) * w with
// |dx_a / dt| <= c and |w| <= 2 (the quintic compensation's largest node
// weight is about 1.6), so bound = 4 max|q| c / (dx dy dz); the layer
// charge of the charge-matched inlet is at most max|q| / (dx dy dz).
double fixed_scale(double bound) {
  if (!(bound > 0.0) || !std::isfinite(bound)) return 1.0;
  int exponent = 0;
  std::frexp(bound, &exponent);  // bound < 2^exponent
  return std::ldexp(1.0, std::max(-1000, std::min(1000, 61 - exponent)));
}

void note_charges(aprl_run* r, const double* charge, size_t n) {
  double m = r->max_abs_charge;
  for (size_t i = 0; i < n; ++i) m = std::max(m, std::fabs(charge[i]));
  r->max_abs_charge = m;
  r->jq_scale = fixed_scale(4.0 * m * kC / (r->cfg.dx * r->cfg.dy * r->cfg.dz));
}

// Geometry only (no field pointers), for the particle sort.
DGrid make_geometry(const aprl_run* r) {
  DGrid g{};
  g.nx = (int)r->cfg.nx;
  g.ny = (int)r->cfg.ny;
  g.nz = (int)r->cfg.nz;
  g.dx = r->cfg.dx;
  g.dy = r->cfg.dy;
  g.dz = r->cfg.dz;
  g.dt = r->cfg.dt;
  for (int a = 0; a < 3; ++a) g.origin[a] = r->origin[a];
  return g;
}

// The detector arguments with the grid view of the run's field type.
template <class F>
DetectorArgs<F> retyped(const DetectorArgs<double>& d, const GridT<F>& g) {
  DetectorArgs<F> a{};
  a.g = g;
  a.frame = d.frame;
  a.origin_xy[0] = d.origin_xy[0];
  a.origin_xy[1] = d.origin_xy[1];
  a.vertex_lower = d.vertex_lower;
  a.half_lower = d.half_lower;
  a.vertex_fraction = d.vertex_fraction;
  a.half_fraction = d.half_fraction;
  a.out = d.out;
  return a;
}

DFrame make_frame(const aprl_run_config& c) {
  return DFrame{c.boost_gamma, c.boost_beta, c.boost_gamma_beta,
                c.lab_time_origin, c.lab_z_origin, c.box_z_origin};
}

// Simulation::movingWindowFieldValue's lerp weights for (k, step)
// (src/simulation_moving_window.cpp:284-293).
aprl_status inlet_table(const aprl_run* r, int64_t k, uint64_t step, InletTable& t) {
  const double z = static_cast<double>(k) - r->cfg.translation_beta * static_cast<double>(step);
  for (int a = 0; a < 6; ++a) {
    if (!r->ref_set[a])
      return fail(APRL_ERR_INVALID_ARGUMENT, "Missing moving-window inlet reference component %d", a);
    const size_t count = r->cfg.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0);
    if (!std::isfinite(z) || z < 0. || z > static_cast<double>(count - 1))
      return fail(APRL_ERR_OUT_OF_RANGE, "Moving reference query outside prepared native field");
    const size_t lo = static_cast<size_t>(std::floor(z));
    const size_t hi = std::min(lo + 1, count - 1);
    size_t s[3];
    comp_shape(r->cfg, a, s);
    t.table[a] = r->ref[a];
    t.nxc[a] = (int)s[0];
    t.nyc[a] = (int)s[1];
    t.lo[a] = (int)lo;
    t.hi[a] = (int)hi;
    t.fraction = z - static_cast<double>(lo);
  }
  return APRL_OK;
}

// ParticleCPMLRegion / ParticleOpenBoundary on the current window.
DRegion make_region(const aprl_run* r) {
  const aprl_run_config& g = r->cfg;
  DRegion d{};
  const double spacing[3] = {g.dx, g.dy, g.dz};
  const size_t cells[3] = {g.nx, g.ny, g.nz};
  const size_t pc[3] = {g.cpml_cells_x, g.cpml_cells_y, 0};
  for (int a = 0; a < 3; ++a) {
    d.outer_lower[a] = r->origin[a];
    d.outer_upper[a] = r->origin[a] + static_cast<double>(cells[a]) * spacing[a];
    d.physical_lower[a] = d.outer_lower[a] + static_cast<double>(pc[a]) * spacing[a];
    d.physical_upper[a] = d.outer_upper[a] - static_cast<double>(pc[a]) * spacing[a];
    d.tolerance[a] = 64.0 * DBL_EPSILON *
                     std::max(1.0, std::max(std::abs(d.outer_lower[a]), std::abs(d.outer_upper[a])));
    d.max_rate[a] = r->max_rate[a];
    d.thickness[a] = static_cast<double>(pc[a]) * spacing[a];
    d.cells[a] = (int)pc[a];
    d.global_lower[a] = r->origin[a];
    d.global_upper[a] = std::fma(static_cast<double>(cells[a]), spacing[a], r->origin[a]);
    d.global_tolerance[a] = 64.0 * DBL_EPSILON *
        std::max(1.0, std::max(std::abs(d.global_lower[a]), std::abs(d.global_upper[a])));
  }
  d.order = g.cpml_polynomial_order;
  return d;
}

aprl_status validate(const aprl_run_config& g) {
  if (g.nx < 2 || g.ny < 2 || g.nz < 2)
    return fail(APRL_ERR_INVALID_ARGUMENT, "E/B staggered grid needs at least two cells in every direction");
  if (g.nx > (1u << 20) || g.ny > (1u << 20) || g.nz > (1u << 24))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Grid extent exceeds the supported index range");
  if (!(g.dx > 0.0) || !(g.dy > 0.0) || !(g.dz > 0.0) || !(g.dt > 0.0) || !std::isfinite(g.dx) ||
      !std::isfinite(g.dy) || !std::isfinite(g.dz) || !std::isfinite(g.dt))
    return fail(APRL_ERR_INVALID_ARGUMENT, "E/B grid spacing and time step must be positive finite SI values");
  if (std::abs(kC * g.dt - g.dz) > 64 * DBL_EPSILON * g.dz)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Moving-window requires c*dt=dz");
  if (g.cpml_cells_x < 2 || g.cpml_cells_y < 2 || 2 * g.cpml_cells_x >= g.nx || 2 * g.cpml_cells_y >= g.ny)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Moving-window requires valid Cowan integer z slabs, xy-only CPML and an inlet reference");
  if (!(g.cpml_polynomial_order > 0.0) ||
      !(g.cpml_target_reflection > 0.0 && g.cpml_target_reflection < 1.0) ||
      !(g.cpml_kappa_max >= 1.0) || !(g.cpml_alpha_fraction >= 0.0))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid CPML grading parameters");
  if (g.precision != APRL_PRECISION_FP64 && g.precision != APRL_PRECISION_FP32_MIXED)
    return fail(APRL_ERR_INVALID_ARGUMENT, "precision must be APRL_PRECISION_FP64 or APRL_PRECISION_FP32_MIXED");
  if (g.shape != APRL_SHAPE_LINEAR_BINOMIAL3 && g.shape != APRL_SHAPE_QUINTIC_COMPENSATED)
    return fail(APRL_ERR_INVALID_ARGUMENT, "APRL 2.1 longitudinal_shape must be linear-binomial3 or quintic-compensated");
  if (g.substeps < 1 || g.max_trials < 1 || g.max_trials > 64)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid substep or trial count");
  if (!(g.boost_gamma >= 1.0) || !std::isfinite(g.boost_gamma))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Lorentz gamma must be finite and >= 1");
  if (g.n_magnets > APRL_MAX_MAGNETS)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Too many prescribed magnets");
  // ChargeMatchedInlet's constructor (src/charge_matched_inlet.h:21-27).
  if (g.inlet_charge_match &&
      (g.cpml_cells_x + 1 >= g.nx - g.cpml_cells_x || g.cpml_cells_y + 1 >= g.ny - g.cpml_cells_y))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Charge-matched inlet needs an interior physical aperture");
  return APRL_OK;
}

aprl_status ensure_scan(aprl_run* r, size_t n) {
  const size_t blocks = (n + kScanBlock - 1) / kScanBlock + 1;
  if (blocks <= r->scan_cap) return APRL_OK;
  device_free(r, r->scan_count);
  device_free(r, r->scan_offset);
  TRY(device_alloc(r, &r->scan_count, blocks));
  TRY(device_alloc(r, &r->scan_offset, blocks));
  r->scan_cap = blocks;
  return APRL_OK;
}

aprl_status alloc_particles(aprl_run* r, DParticles& p, size_t n) {
  TRY(device_alloc(r, &p.x, n)); TRY(device_alloc(r, &p.y, n)); TRY(device_alloc(r, &p.z, n));
  TRY(device_alloc(r, &p.ux, n)); TRY(device_alloc(r, &p.uy, n)); TRY(device_alloc(r, &p.uz, n));
  TRY(device_alloc(r, &p.q, n)); TRY(device_alloc(r, &p.m, n)); TRY(device_alloc(r, &p.id, n));
  TRY(device_alloc(r, &p.order, n));
  TRY(device_alloc(r, &p.frozen, n)); TRY(device_alloc(r, &p.beta, n));
  return APRL_OK;
}
void free_particles(aprl_run* r, DParticles& p) {
  device_free(r, p.x); device_free(r, p.y); device_free(r, p.z); device_free(r, p.ux); device_free(r, p.uy);
  device_free(r, p.uz); device_free(r, p.q); device_free(r, p.m); device_free(r, p.id); device_free(r, p.order);
  device_free(r, p.frozen); device_free(r, p.beta);
  p = DParticles{};
}
void free_pending(aprl_run* r, DPending& d) {
  device_free(r, d.x); device_free(r, d.y); device_free(r, d.z); device_free(r, d.ux); device_free(r, d.uy);
  device_free(r, d.uz); device_free(r, d.q); device_free(r, d.m); device_free(r, d.beta); device_free(r, d.id);
  d = DPending{};
}
aprl_status alloc_carriers(aprl_run* r, DCarriers& c, size_t n) {
  TRY(device_alloc(r, &c.px, n)); TRY(device_alloc(r, &c.py, n)); TRY(device_alloc(r, &c.pz, n));
  TRY(device_alloc(r, &c.vx, n)); TRY(device_alloc(r, &c.vy, n)); TRY(device_alloc(r, &c.vz, n));
  TRY(device_alloc(r, &c.q, n)); TRY(device_alloc(r, &c.w, n)); TRY(device_alloc(r, &c.key, n));
  return APRL_OK;
}
void free_carriers(aprl_run* r, DCarriers& c) {
  device_free(r, c.px); device_free(r, c.py); device_free(r, c.pz); device_free(r, c.vx); device_free(r, c.vy);
  device_free(r, c.vz); device_free(r, c.q); device_free(r, c.w); device_free(r, c.key);
  c = DCarriers{};
}

// Particle capacity: state (two copies for compaction), trial outputs,
// slots, newborn carriers.  Existing contents of p are preserved.
aprl_status reserve_particles(aprl_run* r, size_t n) {
  if (n <= r->pcap) return APRL_OK;
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  DParticles np{};
  TRY(alloc_particles(r, np, n));
  if (r->np) {
    CUDA_TRY(run_copy(r, np.x, r->p.x, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.y, r->p.y, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.z, r->p.z, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.ux, r->p.ux, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.uy, r->p.uy, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.uz, r->p.uz, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.q, r->p.q, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.m, r->p.m, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.id, r->p.id, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.order, r->p.order, r->np * 8, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.frozen, r->p.frozen, r->np, cudaMemcpyDeviceToDevice));
    CUDA_TRY(run_copy(r, np.beta, r->p.beta, r->np * 8, cudaMemcpyDeviceToDevice));
  }
  free_particles(r, r->p);
  free_particles(r, r->p_alt);
  r->p = np;
  TRY(alloc_particles(r, r->p_alt, n));
  double** trial[] = {&r->x1,       &r->y1,       &r->z1,       &r->ux1,      &r->uy1,
                      &r->uz1,      &r->abs_work, &r->slots.x0, &r->slots.y0, &r->slots.z0,
                      &r->slots.dt, &r->dep_b[0], &r->dep_b[1], &r->dep_b[2], &r->dep_e[0],
                      &r->dep_e[1], &r->dep_e[2]};
  for (double** t : trial) {
    device_free(r, *t);
    TRY(device_alloc(r, t, n));
  }
  double** slot[] = {&r->used_e, &r->used_b, &r->next_e, &r->next_b};
  for (double** t : slot) {
    device_free(r, *t);
    TRY(device_alloc(r, t, 3 * n));
  }
  device_free(r, r->action);
  device_free(r, r->born_keep);
  device_free(r, r->slot_order);
  for (int k = 0; k < 2; ++k) {
    device_free(r, r->sort_key[k]);
    device_free(r, r->sort_index[k]);
  }
  device_free(r, r->radix_count);
  device_free(r, r->chunk_sum);
  device_free(r, r->chunk_offset);
  device_free(r, r->res_partial);
  device_free(r, r->frozen1);
  device_free(r, r->slots.seen);
  TRY(device_alloc(r, &r->frozen1, n));
  TRY(device_alloc(r, &r->slots.seen, n));
  device_free(r, r->dep_mode);
  TRY(device_alloc(r, &r->action, n));
  TRY(device_alloc(r, &r->dep_mode, n));
  TRY(device_alloc(r, &r->born_keep, n));
  TRY(device_alloc(r, &r->slot_order, n));
  for (int k = 0; k < 2; ++k) {
    TRY(device_alloc(r, &r->sort_key[k], n));
    TRY(device_alloc(r, &r->sort_index[k], n));
  }
  {
    const size_t counts = (size_t)kRadixBins * ((n + kRadixTile - 1) / kRadixTile);
    TRY(device_alloc(r, &r->radix_count, counts));
    TRY(device_alloc(r, &r->chunk_sum, counts / 1024 + 1));
    TRY(device_alloc(r, &r->chunk_offset, counts / 1024 + 1));
  }
  r->res_blocks = (n + 127) / 128;
  TRY(device_alloc(r, &r->res_partial, 2 * r->res_blocks));
  free_carriers(r, r->born);
  TRY(alloc_carriers(r, r->born, n));
  r->pcap = n;
  return ensure_scan(r, n);
}

aprl_status copy_carriers(aprl_run* r, DCarriers& dst, const DCarriers& src, size_t n) {
  if (!n) return APRL_OK;
  const double* s[] = {src.px, src.py, src.pz, src.vx, src.vy, src.vz, src.q, src.w};
  double* d[] = {dst.px, dst.py, dst.pz, dst.vx, dst.vy, dst.vz, dst.q, dst.w};
  for (int k = 0; k < 8; ++k)
    CUDA_TRY(run_copy(r, d[k], s[k], n * 8, cudaMemcpyDeviceToDevice));
  CUDA_TRY(run_copy(r, dst.key, src.key, n * 8, cudaMemcpyDeviceToDevice));
  return APRL_OK;
}

// Carrier capacity.  The current list and the per-step outputs (c_out,
// c_keep) of the `nc` existing carriers survive a reallocation.
// The first reservation takes at least a sixteenth of the particle capacity
// (and 4096), so that the carriers a bunch sheds into the CPML over its
// first steps do not regrow the lists -- each regrowth is a stream sync plus
// 27 cudaMalloc/cudaFree calls inside a step.
aprl_status reserve_carriers(aprl_run* r, size_t n) {
  if (n <= r->ccap) return APRL_OK;
  n = std::max({n, 2 * r->ccap, std::max<size_t>(4096, r->pcap / 16)});
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  DCarriers nc{}, nout{};
  unsigned char* nkeep = nullptr;
  TRY(alloc_carriers(r, nc, n));
  TRY(alloc_carriers(r, nout, n));
  TRY(device_alloc(r, &nkeep, n));
  TRY(copy_carriers(r, nc, r->c, r->nc));
  TRY(copy_carriers(r, nout, r->c_out, r->nc));
  if (r->nc) CUDA_TRY(run_copy(r, nkeep, r->c_keep, r->nc, cudaMemcpyDeviceToDevice));
  free_carriers(r, r->c);
  free_carriers(r, r->c_alt);
  free_carriers(r, r->c_out);
  device_free(r, r->c_keep);
  r->c = nc;
  r->c_out = nout;
  r->c_keep = nkeep;
  TRY(alloc_carriers(r, r->c_alt, n));
  r->ccap = n;
  return ensure_scan(r, n);
}

// Rotate between logical (window) and physical (ring) plane order.
aprl_status copy_ring(aprl_run* r, double* device, const double* host_in, double* host_out,
                      size_t plane, size_t layers, int base, size_t slots = 1) {
  for (size_t s = 0; s < slots; ++s) {
    const size_t slot_offset = s * layers * plane;
    for (size_t k = 0; k < layers; ++k) {
      const size_t pk = (k + base) % layers;
      double* d = device + slot_offset + pk * plane;
      if (host_in)
        CUDA_TRY(cudaMemcpyAsync(d, host_in + slot_offset + k * plane, plane * 8,
                                 cudaMemcpyHostToDevice, r->stream));
      else
        CUDA_TRY(cudaMemcpyAsync(host_out + slot_offset + k * plane, d, plane * 8,
                                 cudaMemcpyDeviceToHost, r->stream));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

aprl_status check_device(aprl_run* r) {
  CUDA_TRY(cudaMemcpyAsync(r->h_status, r->d_status, sizeof(DeviceStatus),
                           cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  if (r->h_status->code)
    return fail(device_error_status(r->h_status->code), "%s (element %llu)",
                device_error_text(r->h_status->code), r->h_status->where);
  return APRL_OK;
}

dim3 grid3(const aprl_run_config& g, dim3 block) {
  return dim3((unsigned)((g.nx + 1 + block.x - 1) / block.x),
              (unsigned)((g.ny + 1 + block.y - 1) / block.y), (unsigned)(g.nz + 1));
}

unsigned blocks_for(size_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

void add_counters(TrialCounters& to, const TrialCounters& from) {
  to.exits += from.exits;
  to.exit_charge += from.exit_charge;
  for (int f = 0; f < 6; ++f) {
    to.cpml[f] += from.cpml[f];
    to.cpml_charge[f] += from.cpml_charge[f];
    to.direct[f] += from.direct[f];
    to.direct_charge[f] += from.direct_charge[f];
    to.carrier_outer[f] += from.carrier_outer[f];
    to.carrier_outer_charge[f] += from.carrier_outer_charge[f];
  }
  to.cropped += from.cropped;
  to.cropped_charge += from.cropped_charge;
  to.activations += from.activations;
}

// Block offsets of a stable compaction of `n` flagged elements (the kept
// count is known to the caller).
aprl_status compact_offsets(aprl_run* r, const unsigned char* flag, unsigned char want,
                            size_t n) {
  if (n == 0) return APRL_OK;
  TRY(ensure_scan(r, n));
  const unsigned blocks = blocks_for(n, kScanBlock);
  TRY(launch(r, kFlagCount, flag_count_kernel, dim3(blocks), dim3(kScanBlock), flag, want,
             (long long)n, r->scan_count));
  return launch(r, kBlockScan, block_offset_scan_kernel, dim3(1), dim3(1024),
                (const unsigned*)r->scan_count, (int)blocks, r->scan_offset, r->scan_total);
}

// Stable radix sort of the particle storage by cell index: the key pass,
// then per 8-bit digit the block digit counts, their exclusive scan in
// digit-major order (chunk scan, chunk-sum scan, chunk add) and the stable
// scatter of keys and storage indices; finally the particle arrays are
// permuted.  No atomic ticket decides an order, so the storage order after
// a sort is a function of the storage order before it.
aprl_status sort_particles(aprl_run* r) {
  if (r->np < 2 || r->sort_bits == 0) return APRL_OK;
  const long long n = (long long)r->np;
  const DGrid g = make_geometry(r);
  TRY(launch(r, kSortKey, sort_key_kernel, dim3(blocks_for(r->np, 256)), dim3(256), r->p, n, g,
             r->tiles[0], r->tiles[1], r->sort_key[0], r->sort_index[0]));
  const unsigned blocks = blocks_for(r->np, kRadixTile);
  const long long counts = (long long)kRadixBins * blocks;
  const unsigned chunks = blocks_for((size_t)counts, 1024);
  int from = 0;
  for (int shift = 0; shift < r->sort_bits; shift += 8) {
    TRY(launch(r, kRadixCount, radix_count_kernel, dim3(blocks), dim3(kRadixThreads),
               (const unsigned*)r->sort_key[from], n, shift, r->radix_count));
    TRY(launch(r, kChunkScan, chunk_scan_kernel, dim3(chunks), dim3(1024),
               (const unsigned*)r->radix_count, counts, r->radix_count, r->chunk_sum));
    TRY(launch(r, kBlockScan, block_offset_scan_kernel, dim3(1), dim3(1024),
               (const unsigned*)r->chunk_sum, (int)chunks, r->chunk_offset, r->scan_total));
    TRY(launch(r, kChunkAdd, chunk_add_kernel, dim3(chunks), dim3(1024), r->radix_count,
               counts, (const unsigned*)r->chunk_offset));
    TRY(launch(r, kRadixScatter, radix_scatter_kernel, dim3(blocks), dim3(kRadixThreads),
               (const unsigned*)r->sort_key[from], (const unsigned*)r->sort_index[from],
               r->sort_key[1 - from], r->sort_index[1 - from], n, shift,
               (const unsigned*)r->radix_count));
    from = 1 - from;
  }
  TRY(launch(r, kPermuteParticles, permute_particles_kernel, dim3(blocks_for(r->np, 256)),
             dim3(256), r->p_alt, r->p, n, (const unsigned*)r->sort_index[from]));
  std::swap(r->p, r->p_alt);
  return APRL_OK;
}

// ---- held lab-plane injection: PendingParticleQueue at one rank
// (src/pending_particle_queue.cpp).  The queue's bookkeeping lives on the
// host; its entries live on the device in due order, so one admission is
// one contiguous range.
double held_distance_per_beta(const aprl_run_config& c) { return kC * c.dt; }

// PendingParticleQueue::origin (src/pending_particle_queue.cpp:106-111).
double pending_origin(const aprl_run_config& c, uint64_t step) {
  const int64_t offset = c.initial_offset - static_cast<int64_t>(step);
  return std::fma(static_cast<double>(offset), c.dz, c.reference_origin[2]);
}

// participates (src/pending_particle_queue.cpp:113-117): the held chord of
// `step` ends at or beyond that step's inlet.
bool participates(const aprl_run* r, double z, double beta, uint64_t step) {
  const double end = repeat_held_addition(z, held_distance_per_beta(r->cfg) * beta,
                                          step - r->queue.initial_step + 1);
  return end >= pending_origin(r->cfg, step);
}

// firstDue (src/pending_particle_queue.cpp:119-126): extended-precision
// estimate, confirmed or replaced by bisection over participates.
uint64_t first_due(const aprl_run* r, double z, double beta) {
  const auto& q = r->queue;
  const double increment = held_distance_per_beta(r->cfg) * beta;
  const long double distance = static_cast<long double>(pending_origin(r->cfg, q.initial_step)) -
                               static_cast<long double>(z) - static_cast<long double>(increment);
  const long double estimate = std::ceil(
      distance / (static_cast<long double>(r->cfg.dz) + static_cast<long double>(increment)));
  const uint64_t sentinel = q.maximum_step + 1;
  const long double steps_left = static_cast<long double>(q.maximum_step - q.initial_step);
  const uint64_t guess =
      estimate > steps_left
          ? sentinel
          : q.initial_step + static_cast<uint64_t>(estimate > 1.L ? estimate : 1.L);
  if (guess <= q.maximum_step && participates(r, z, beta, guess) &&
      !participates(r, z, beta, guess - 1))
    return guess;
  if (guess == sentinel && !participates(r, z, beta, q.maximum_step)) return sentinel;
  uint64_t lower = q.initial_step + 1, upper = sentinel;
  while (lower < upper) {
    const uint64_t middle = lower + (upper - lower) / 2;
    if (participates(r, z, beta, middle)) upper = middle;
    else lower = middle + 1;
  }
  return lower;
}

void advance_next_due(aprl_run::Queue& q) {
  while (q.next_due <= q.maximum_step && q.offsets[q.next_due - q.initial_step + 1] <= q.cursor)
    ++q.next_due;
}

// PendingParticleQueue::admit (src/pending_particle_queue.cpp:163-186),
// called by admitMovingWindowParticles at the start of the step
// (src/simulation.cpp:513).
aprl_status admit_pending(aprl_run* r) {
  auto& q = r->queue;
  if (!q.extracted) return APRL_OK;
  const uint64_t step = r->step;
  if (step < q.last_step || step > q.maximum_step || step > q.next_due)
    return fail(APRL_ERR_RUNTIME, "Pending admission skipped an event or exceeds its horizon");
  q.last_step = step;
  const size_t end = q.offsets[step - q.initial_step + 1];
  const size_t k = end - q.cursor;
  if (k) {
    TRY(reserve_particles(r, r->np + k));
    TRY(launch(r, kAdmit, admit_kernel, dim3(blocks_for(k, 256)), dim3(256), r->p,
               (long long)r->np, q.d, (long long)q.cursor, (long long)k,
               (unsigned long long)(step - q.initial_step), held_distance_per_beta(r->cfg),
               (unsigned long long)r->next_order));
    r->np += k;
    r->next_order += k;
    q.cursor = end;
    r->admitted += k;
    r->held += k;
  }
  advance_next_due(q);
  return APRL_OK;
}

// ---- energy ledger (ledger.cuh) -------------------------------------------
constexpr int kLedgerMaxBlocks = 592;  // four blocks per SM

aprl_status ensure_ledger(aprl_run* r) {
  if (r->d_ledger) return APRL_OK;
  const aprl_run_config& c = r->cfg;
  TRY(device_alloc(r, &r->d_ledger, 1));
  TRY(device_alloc(r, &r->d_ledger_partial, (size_t)kLedgerMaxTerms * kLedgerMaxBlocks));
  TRY(device_alloc(r, &r->ledger_pre[0], (size_t)c.nx * (c.ny + 1)));
  TRY(device_alloc(r, &r->ledger_pre[1], (size_t)(c.nx + 1) * c.ny));
  CUDA_TRY(cudaMemsetAsync(r->d_ledger, 0, sizeof(DLedger), r->stream));
  return APRL_OK;
}

LedgerArgs ledger_args(const aprl_run* r, int phase) {
  const aprl_run_config& c = r->cfg;
  LedgerArgs a{};
  a.g = make_grid<double>(r);
  a.pre[0] = r->ledger_pre[0];
  a.pre[1] = r->ledger_pre[1];
  a.ux = r->p.ux;
  a.uy = r->p.uy;
  a.uz = r->p.uz;
  a.m = r->p.m;
  a.i0 = (int)c.cpml_cells_x;
  a.i1 = (int)(c.nx - c.cpml_cells_x);
  a.j0 = (int)c.cpml_cells_y;
  a.j1 = (int)(c.ny - c.cpml_cells_y);
  a.volume = ledger_product(ledger_product(c.dx, c.dy), c.dz);
  a.area_yz = ledger_product(c.dy, c.dz);
  a.area_xz = ledger_product(c.dx, c.dz);
  a.area_xy = ledger_product(c.dx, c.dy);
  a.c2 = ledger_product(kC, kC);
  a.half_dt = 0.5 * c.dt;
  a.phase = phase;
  a.partial = r->d_ledger_partial;
  a.ledger = r->d_ledger;
  return a;
}

void ledger_term(LedgerArgs& a, int kind, int index, int kmax, bool substitute, double sign,
                 long long count) {
  LedgerTerm& t = a.q[a.nq++];
  t.kind = kind;
  t.index = index;
  t.kmax = kmax;
  t.substitute = substitute ? 1 : 0;
  t.sign = sign;
  t.count = count;
}

void ledger_plane(LedgerArgs& a, int k, bool substitute) {
  ledger_term(a, kLedgerPlane, k, 1, substitute, 1., (long long)(a.i1 - a.i0) * (a.j1 - a.j0));
}

// boundaryPower's faces x-, x+, y-, y+, z- and (unless inlet_only) z+.
void ledger_faces(LedgerArgs& a, int nz, bool inlet_only, bool substitute) {
  const long long w = a.i1 - a.i0, h = a.j1 - a.j0;
  const int kmax = inlet_only ? 1 : nz;
  ledger_term(a, kLedgerFaceX, a.i0, kmax, substitute, -1., h * kmax);
  ledger_term(a, kLedgerFaceX, a.i1 - 1, kmax, substitute, 1., h * kmax);
  ledger_term(a, kLedgerFaceY, a.j0, kmax, substitute, -1., w * kmax);
  ledger_term(a, kLedgerFaceY, a.j1 - 1, kmax, substitute, 1., w * kmax);
  ledger_term(a, kLedgerFaceZ, 0, 1, substitute, -1., w * h);
  if (!inlet_only) ledger_term(a, kLedgerFaceZ, nz - 1, 1, substitute, 1., w * h);
}

aprl_status ledger_launch(aprl_run* r, LedgerArgs& a) {
  int blocks = 0;
  for (int q = 0; q < a.nq; ++q) {
    LedgerTerm& t = a.q[q];
    const long long per_block = (long long)kLedgerThreads * 4;
    const long long want = (t.count + per_block - 1) / per_block;
    t.blocks = (int)std::min<long long>(std::max<long long>(want, 1), kLedgerMaxBlocks);
    t.first_block = blocks;
    blocks += t.blocks;
  }
  TRY(launch(r, kLedgerPartial, ledger_partial_kernel, dim3(blocks), dim3(kLedgerThreads), a));
  return launch(r, kLedgerFinish, ledger_finish_kernel, dim3(1), dim3(kLedgerFinishThreads), a);
}

// Boundary::begin (src/moving_window_fields.cpp:214-218): the step's start power.
aprl_status ledger_begin(aprl_run* r) {
  LedgerArgs a = ledger_args(r, kLedgerPhaseBegin);
  ledger_faces(a, (int)r->cfg.nz, false, false);
  return ledger_launch(r, a);
}

// After the commit: the measured inlet overwrite (src/moving_window_fields.cpp:265-290),
// finishEnergyLedgerStep (:425-437) and the plane the shift drops (:446-450).
aprl_status ledger_finish(aprl_run* r) {
  LedgerArgs a = ledger_args(r, kLedgerPhaseFinish);
  const int nz = (int)r->cfg.nz;
  ledger_plane(a, 0, true);
  ledger_plane(a, 0, false);
  ledger_faces(a, nz, true, true);
  ledger_faces(a, nz, true, false);
  ledger_faces(a, nz, false, false);
  ledger_plane(a, nz - 1, false);
  return ledger_launch(r, a);
}

// After the shift: the inserted plane (src/moving_window_fields.cpp:500-515)
// and the boundary power of the shifted fields, which the next begin would
// measure on the same fields.
aprl_status ledger_shift(aprl_run* r) {
  LedgerArgs a = ledger_args(r, kLedgerPhaseShift);
  ledger_plane(a, 0, false);
  ledger_faces(a, (int)r->cfg.nz, false, false);
  TRY(ledger_launch(r, a));
  r->ledger_start_ready = true;
  return APRL_OK;
}

aprl_status ledger_snapshot(aprl_run* r) {
  LedgerArgs a = ledger_args(r, kLedgerPhaseSnapshot);
  const int nz = (int)r->cfg.nz;
  ledger_term(a, kLedgerVolume, 0, nz, false, 1.,
              (long long)(a.i1 - a.i0) * (a.j1 - a.j0) * nz);
  ledger_faces(a, nz, false, false);
  ledger_term(a, kLedgerKinetic, 0, 0, false, 1., (long long)r->np);
  ledger_term(a, kLedgerTotal, 0, 0, false, 1., (long long)r->np);
  ledger_term(a, kLedgerRepresented, 0, 0, false, 1., (long long)r->np);
  return ledger_launch(r, a);
}

template <class F>
aprl_status advance_magnetic_t(aprl_run* r) {
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Moving-window beginStep phase/origin mismatch");
  TRY(admit_pending(r));
  if (r->ledger_on && !r->ledger_start_ready) TRY(ledger_begin(r));
  r->ledger_start_ready = false;
  const aprl_run_config& c = r->cfg;
  if (!r->j_zero)
    for (int a = 0; a < 3; ++a)
      CUDA_TRY(cudaMemsetAsync(r->jc[a], 0, e_count(c, a) * sizeof(F), r->stream));
  r->j_zero = true;
  InletPlaneArgs ia{};
  ia.nx = (int)c.nx;
  ia.ny = (int)c.ny;
  for (int a = 0; a < 3; ++a) ia.out[a] = r->lower[a];
  TRY(inlet_table(r, r->offset - 1, r->step, ia.inlet));
  TRY(launch(r, kInletLower, inlet_lower_kernel,
             dim3(blocks_for(c.nx + 1, 32), blocks_for(c.ny + 1, 8), 3), dim3(32, 8), ia));
  if (c.inlet_charge_match) {
    InletHaloArgs ha{};
    ha.g = make_grid<double>(r);
    ha.lower_ez = r->lower[2];
    ha.cx = (int)c.cpml_cells_x;
    ha.cy = (int)c.cpml_cells_y;
    TRY(inlet_table(r, r->offset, r->step, ha.inlet));
    TRY(launch(r, kInletHalo, inlet_halo_kernel,
               dim3(blocks_for(c.nx + 1, 32), blocks_for(c.ny + 1, 8)), dim3(32, 8), ha));
  }
  CowanArgs<F> ca{};
  ca.g = make_grid<F>(r);
  for (int a = 0; a < 3; ++a) {
    ca.e[a] = r->e[r->cur][a];
    ca.lower[a] = r->lower[a];
    ca.alpha[a] = r->coeff[a];
    ca.beta[a] = r->coeff[3 + a];
  }
  ca.delta_xy = r->coeff[6];
  ca.delta_yz = r->coeff[7];
  ca.delta_zx = r->coeff[8];
  ca.mx = r->mprof[0].view();
  ca.my = r->mprof[1].view();
  for (int h = 0; h < 4; ++h) ca.h[h] = r->hist[h].view();
  // Column tiles marching z chunks (fields.cuh: kCowanTileX/Y, kCowanChunk):
  // at most kCowanChunk planes per block, fewer when that leaves fewer than
  // about four blocks per SM.
  const dim3 cblock(kCowanTileX, kCowanTileY);
  const unsigned columns = blocks_for(c.nx + 1, kCowanTileX) * blocks_for(c.ny + 1, kCowanTileY);
  (void)columns;
  const size_t planes = c.nz + 1;
  TuneLaunch tl;
  TRY(tune_begin(r, kTuneCowan, tl));
  ca.chunk = (int)std::min<size_t>(kCowanChunks[tl.candidate], planes);
  const dim3 cgrid(blocks_for(c.nx + 1, kCowanTileX), blocks_for(c.ny + 1, kCowanTileY),
                   blocks_for(planes, ca.chunk));
  TRY(launch(r, kCowanMagnetic, cowan_magnetic_kernel<F>, cgrid, cblock, ca));
  TRY(tune_end(r, tl));
  r->stage = 1;
  return APRL_OK;
}

aprl_status do_advance_magnetic(aprl_run* r) {
  return advance_magnetic_t<double>(r);
}

template <class F>
aprl_status preview_electric_t(aprl_run* r) {
  if (r->stage != 1) return fail(APRL_ERR_RUNTIME, "Moving-window electric phase mismatch");
  const aprl_run_config& c = r->cfg;
  PreviewArgs<F> pa{};
  pa.g = make_grid<F>(r);
  pa.ex_prof = r->eprof[0].view();
  pa.ey_prof = r->eprof[1].view();
  for (int h = 0; h < 4; ++h) pa.h[h] = r->hist[4 + h].view();
  for (int a = 0; a < 2; ++a) pa.pre_inlet[a] = r->ledger_on ? r->ledger_pre[a] : nullptr;
  // With particles to gather, the first trial's current-free orbit sum is
  // written by the preview itself (E* and E^n are in its registers there).
  r->orbit_from_preview = r->np != 0;
  for (int a = 0; a < 3; ++a) pa.orbit[a] = r->orbit_from_preview ? r->orbit[a] : nullptr;
  pa.orbit_float = r->fp32 ? 1 : 0;
  TRY(inlet_table(r, r->offset, r->step + 1, pa.inlet));
  TuneLaunch tl;
  TRY(tune_begin(r, kTunePreview, tl));
  const dim3 block = kGridBlocks[tl.candidate];
  TRY(launch(r, kElectricPreview, electric_preview_kernel<F>, grid3(c, block), block, pa));
  TRY(tune_end(r, tl));
  if (r->fp32 && r->np) {  // B is final for the step: its binary32 copy for the gathers
    BShadowArgs sa{};
    size_t most = 0;
    for (int a = 0; a < 3; ++a) {
      sa.b[a] = r->b[a];
      sa.out[a] = r->bshadow[a];
      sa.n[a] = (long long)b_count(c, a);
      most = std::max(most, b_count(c, a));
    }
    TRY(launch(r, kBShadow, b_shadow_kernel, dim3(blocks_for(most, 256), 3), dim3(256), sa));
  }
  if (r->np)
    CUDA_TRY(cudaMemcpyAsync(r->slot_order, r->p.order, r->np * 8, cudaMemcpyDeviceToDevice,
                             r->stream));
  r->nslot = r->np;
  r->trials = 0;
  r->stage = 2;
  return APRL_OK;
}

aprl_status do_preview_electric(aprl_run* r) {
  return preview_electric_t<double>(r);
}

// TransverseReferenceCurrent (src/transverse_reference_current.cpp:19-28,
// 46-63, 104-118): the target points of the physical region's transverse
// faces in the reference's order, curl_z(B_ref)/mu0 at each for every
// reference plane (prepared on the device from the reference tables when
// first needed), and each trial Jz += the plane lerp at
// offset + k - beta (step + 1) for every window plane k.
aprl_status surface_current_prepare(aprl_run* r) {
  if (r->surface_ready) return APRL_OK;
  const aprl_run_config& c = r->cfg;
  if (!c.cpml_cells_x || !c.cpml_cells_y)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Reference surface current requires transverse-only CPML");
  if (!r->ref_set[3] || !r->ref_set[4])
    return fail(APRL_ERR_INVALID_ARGUMENT, "Missing moving-window inlet reference component");
  const size_t x0 = c.cpml_cells_x, x1 = c.nx - c.cpml_cells_x;
  const size_t y0 = c.cpml_cells_y, y1 = c.ny - c.cpml_cells_y;
  std::vector<unsigned> points;
  for (size_t i = x0; i <= x1; ++i) {
    points.push_back((unsigned)i); points.push_back((unsigned)y0);
    points.push_back((unsigned)i); points.push_back((unsigned)y1);
  }
  for (size_t j = y0 + 1; j < y1; ++j) {
    points.push_back((unsigned)x0); points.push_back((unsigned)j);
    points.push_back((unsigned)x1); points.push_back((unsigned)j);
  }
  const size_t count = points.size() / 2;
  device_free(r, r->surface_points);
  device_free(r, r->surface_table);
  r->surface_points = nullptr;
  r->surface_table = nullptr;
  TRY(device_alloc(r, &r->surface_points, points.size()));
  TRY(device_alloc(r, &r->surface_table, count * std::max<uint64_t>(1, c.reference_nz)));
  CUDA_TRY(run_copy(r, r->surface_points, points.data(), points.size() * sizeof(unsigned),
                    cudaMemcpyHostToDevice));
  SurfaceArgs a{};
  a.points = r->surface_points;
  a.table = r->surface_table;
  a.count = (long long)count;
  a.planes = (long long)c.reference_nz;
  a.bx = r->ref[3];
  a.by = r->ref[4];
  a.nx = (int)c.nx;
  a.ny = (int)c.ny;
  a.dx = c.dx;
  a.dy = c.dy;
  a.status = r->d_status;
  TRY(launch(r, kSurfaceCurrent, surface_prepare_kernel,
             dim3(blocks_for(count * c.reference_nz, 256)), dim3(256), a));
  TRY(check_device(r));
  r->surface_count = count;
  r->surface_ready = true;
  return APRL_OK;
}

aprl_status surface_current_add(aprl_run* r, const GridT<double>& g) {
  TRY(surface_current_prepare(r));
  const aprl_run_config& c = r->cfg;
  // The reference's range check (src/transverse_reference_current.cpp:109-110),
  // for the first and last window planes (z grows with k).
  const double step = static_cast<double>(r->step + 1);
  const double z0 = static_cast<double>(r->offset) - c.translation_beta * step;
  const double z1 = static_cast<double>(r->offset + (int64_t)c.nz - 1) - c.translation_beta * step;
  if (!std::isfinite(z0) || z0 < 0. || z1 > static_cast<double>(c.reference_nz) - 1.)
    return fail(APRL_ERR_OUT_OF_RANGE, "Reference surface-current query outside domain");
  SurfaceArgs a{};
  a.points = r->surface_points;
  a.table = r->surface_table;
  a.count = (long long)r->surface_count;
  a.planes = (long long)c.reference_nz;
  a.offset = r->offset;
  a.step = r->step + 1;
  a.beta = c.translation_beta;
  a.g = g;
  return launch(r, kSurfaceCurrent, surface_add_kernel,
                dim3(blocks_for(r->surface_count * c.nz, 256)), dim3(256), a);
}

// One coupling trial; W is the arithmetic of the gathers.
template <class W>
aprl_status trial_enqueue_t(aprl_run* r, int slot, bool ahead) {
  using F = double;
  if (r->stage != 2 && r->stage != 3)
    return fail(APRL_ERR_RUNTIME, "Coupling trial requires a previewed electric field");
  const aprl_run_config& c = r->cfg;
  GridT<F> g = make_grid<F>(r);
  if (ahead) g.stop = r->d_stop;
  // Frozen source support of the entries due within min(8, horizon) steps.
  size_t frozen_end = 0;
  if (r->queue.extracted) {
    const auto& q = r->queue;
    const uint64_t room = q.maximum_step - r->step;
    const uint64_t until = r->step + std::min<uint64_t>(8, room);
    frozen_end = q.offsets[until - q.initial_step + 1];
  }
  const bool deposits = r->np || r->nc || (r->queue.extracted && frozen_end > r->queue.cursor);
  size_t most = 0;
  for (int a = 0; a < 3; ++a) most = std::max(most, e_count(c, a));
  const unsigned grid_blocks = std::min<unsigned>(blocks_for(most, 256), 148 * 8);
  // Deterministic mode: the deposits of the trial go into J's fixed-point
  // pairs, and J is written from them once they are all done.
  const bool convert = r->deterministic && deposits;
  {
    // The counters and sums always; J unless it is known to be zero (its
    // pairs instead when the conversion will write J).
    const int clear_current = convert ? 2 : (r->j_zero ? 0 : 1);
    const unsigned blocks = clear_current ? grid_blocks : 1u;
    TRY(launch(r, kTrialClear, trial_clear_kernel, dim3(blocks), dim3(256), g, r->d_counters,
               r->d_sums, clear_current));
  }
  const bool surface = c.reference_surface_current != 0;
  r->j_zero = !deposits && !surface;
  // J complete for the trial: the fixed-point pairs converted (deterministic
  // mode), then the reference's equivalent surface current added.
  bool converted = false;
  auto convert_current = [&]() -> aprl_status {
    if (converted) return APRL_OK;
    converted = true;
    if (convert)
      TRY(launch(r, kCurrentConvert, current_convert_kernel, dim3(grid_blocks), dim3(256), g,
                 1.0 / r->jq_scale));
    if (surface) TRY(surface_current_add(r, g));
    return APRL_OK;
  };
  const DRegion region = make_region(r);
  // Each particle kernel is built per shape: 0 linear-binomial3, else quintic.
  const bool binomial = c.shape == 0;
  if (r->queue.extracted) {
    const auto& q = r->queue;
    const size_t end = frozen_end;
    if (end > q.cursor) {
      SupportArgs<F> sa{};
      sa.g = g;
      sa.shape = c.shape;
      sa.src = q.d;
      sa.begin = (long long)q.cursor;
      sa.count = (long long)(end - q.cursor);
      sa.steps = r->step - q.initial_step;
      sa.held_distance_per_beta = held_distance_per_beta(c);
      sa.status = r->d_status;
      TRY(launch(r, kFrozenSupport,
                 r->deterministic
                     ? (binomial ? frozen_support_kernel<F, 0, true> : frozen_support_kernel<F, 1, true>)
                     : (binomial ? frozen_support_kernel<F, 0, false> : frozen_support_kernel<F, 1, false>),
                 dim3(blocks_for(end - q.cursor, 128)),
                 dim3(128), sa));
    }
  }
  // Carriers share only J, the counters and the status word with the
  // particle kernels, all through atomics, so they run beside them.
  bool joined = true;
  if (r->nc) {
    CarrierArgs<F> ca{};
    ca.g = g;
    ca.region = region;
    ca.shape = c.shape;
    ca.count = (long long)r->nc;
    ca.in = r->c;
    ca.out = r->c_out;
    ca.keep = r->c_keep;
    ca.counters = r->d_counters;
    ca.status = r->d_status;
    CUDA_TRY(cudaEventRecord(r->fork, r->stream));
    CUDA_TRY(cudaStreamWaitEvent(r->side, r->fork, 0));
    TRY(launch_on(r, r->side, kCarrier,
                  r->deterministic
                      ? (binomial ? carrier_kernel<F, 0, true> : carrier_kernel<F, 1, true>)
                      : (binomial ? carrier_kernel<F, 0, false> : carrier_kernel<F, 1, false>),
                  dim3(blocks_for(r->nc, 128)),
                  dim3(128), ca));
    CUDA_TRY(cudaEventRecord(r->join, r->side));
    joined = false;
  }
  auto join_carriers = [&]() -> aprl_status {
    if (!joined) CUDA_TRY(cudaStreamWaitEvent(r->stream, r->join, 0));
    joined = true;
    return APRL_OK;
  };
  if (r->np) {
    PushArgs<F> pa{};
    pa.g = g;
    pa.frame = make_frame(c);
    pa.region = region;
    pa.n_magnets = (int)c.n_magnets;
    for (uint32_t m = 0; m < c.n_magnets; ++m) {
      const aprl_magnet& s = c.magnets[m];
      DMagnet& d = pa.magnets[m];
      d.type = s.type == APRL_MAGNET_PLANAR_UNDULATOR ? 0 : (s.type == APRL_MAGNET_UNIFORM_DIPOLE ? 1 : 2);
      d.gaussian_fringe = s.gaussian_fringe;
      for (int a = 0; a < 3; ++a) d.center[a] = s.center[a];
      d.length = s.length;
      d.period = s.period;
      d.peak_field = s.peak_field;
      d.quadrupole_gradient = s.quadrupole_gradient;
      d.wave_number = s.wave_number;
      d.fringe_extent = s.fringe_extent;
      d.cos_angle = s.cos_angle;
      d.sin_angle = s.sin_angle;
    }
    pa.shape = c.shape;
    pa.substeps = (int)c.substeps;
    pa.time = r->time;
    pa.exit_lab_z = c.exit_lab_z;
    pa.activation_plane_lab_z = c.activation_plane_lab_z;
    pa.count = (long long)r->np;
    pa.p = r->p;
    pa.x1 = r->x1; pa.y1 = r->y1; pa.z1 = r->z1;
    pa.ux1 = r->ux1; pa.uy1 = r->uy1; pa.uz1 = r->uz1;
    pa.frozen1 = r->frozen1;
    pa.slot = r->slots;
    pa.used_e = r->used_e;
    pa.used_b = r->used_b;
    pa.next_e = r->next_e;
    pa.next_b = r->next_b;
    pa.abs_grid_work = r->abs_work;
    pa.action = r->action;
    pa.born = r->born;
    pa.born_keep = r->born_keep;
    for (int d = 0; d < 3; ++d) {
      pa.dep_b[d] = r->dep_b[d];
      pa.dep_e[d] = r->dep_e[d];
    }
    pa.dep_mode = r->dep_mode;
    pa.key_base = (unsigned long long)(r->step + 1) << 32;
    pa.counters = r->d_counters;
    pa.status = r->d_status;
    W* orbit[3] = {static_cast<W*>(r->orbit[0]), static_cast<W*>(r->orbit[1]),
                   static_cast<W*>(r->orbit[2])};
    for (int a = 0; a < 3; ++a) {
      pa.orbit[a] = orbit[a];
      pa.bgather[a] = r->fp32 ? static_cast<const void*>(r->bshadow[a])
                              : static_cast<const void*>(r->b[a]);
    }
    const dim3 oblock(32, 4);
    if (r->trials == 0) {
      if (!r->orbit_from_preview)
        TRY(launch(r, kOrbitSum, orbit_sum_kernel<W>, grid3(c, oblock), oblock, g, orbit[0],
                   orbit[1], orbit[2], 0));
      TRY(launch(r, kGuessGather,
                 binomial ? guess_gather_kernel<W, F, 0> : guess_gather_kernel<W, F, 1>,
                 dim3(blocks_for(r->np, 128)),
                 dim3(128), pa));
    }
    TRY(launch(r, kPushDeposit,
               r->deterministic
                   ? (binomial ? push_deposit_kernel<F, 0, true> : push_deposit_kernel<F, 1, true>)
                   : (binomial ? push_deposit_kernel<F, 0, false> : push_deposit_kernel<F, 1, false>),
               dim3(blocks_for(r->np, 128)), dim3(128),
               pa));
    if (binomial) {
      ChordArgs da{};
      da.g = g;
      da.count = (long long)r->np;
      da.mode = r->dep_mode;
      for (int d = 0; d < 3; ++d) {
        da.b[d] = r->dep_b[d];
        da.e[d] = r->dep_e[d];
      }
      da.q = r->p.q;
      da.status = r->d_status;
      TRY(launch(r, kChordDeposit,
                 r->deterministic ? chord_deposit_kernel<true> : chord_deposit_kernel<false>,
                 dim3(blocks_for(r->np, 128)), dim3(128), da));
    }
    TRY(join_carriers());
    TRY(convert_current());
    {
      // Measured only in a step's first trial: a trial issued ahead may be
      // skipped (its kernels return at once), which would time nothing.
      TuneLaunch tl;
      if (r->trials == 0) {
        TRY(tune_begin(r, kTuneOrbit, tl));
      } else {
        tl.candidate = std::max(0, r->tune_choice[kTuneOrbit]);
      }
      const dim3 sblock = kGridBlocks[tl.candidate];
      TRY(launch(r, kOrbitSum, orbit_sum_kernel<W>, grid3(c, sblock), sblock, g, orbit[0],
                 orbit[1], orbit[2], 1));
      TRY(tune_end(r, tl));
    }
    ResidualArgs<F> ra{};
    ra.g = g;
    for (int a = 0; a < 3; ++a) {
      ra.orbit[a] = pa.orbit[a];
      ra.bgather[a] = pa.bgather[a];
    }
    ra.shape = c.shape;
    ra.count = (long long)r->np;
    ra.p = r->p;
    ra.slot = r->slots;
    ra.x1 = r->x1; ra.y1 = r->y1; ra.z1 = r->z1;
    ra.used_e = r->used_e;
    ra.used_b = r->used_b;
    ra.next_e = r->next_e;
    ra.next_b = r->next_b;
    ra.abs_grid_work = r->abs_work;
    ra.sums = r->d_sums;
    ra.partial = r->res_partial;
    ra.ticket = r->res_ticket;
    ra.status = r->d_status;
    TRY(launch(r, kResidual, binomial ? residual_kernel<W, F, 0> : residual_kernel<W, F, 1>,
               dim3(blocks_for(r->np, 128)), dim3(128), ra));
  }
  TRY(join_carriers());
  TRY(convert_current());
  if (ahead)
    TRY(launch(r, kTrialVerdict, trial_verdict_kernel, dim3(1), dim3(1),
               (const ResidualSums*)r->d_sums, r->trials + 1, c.force_tolerance,
               c.work_tolerance, r->d_stop));
  CUDA_TRY(cudaMemcpyAsync(&r->h_sums_slots[slot], r->d_sums, sizeof(ResidualSums),
                           cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaMemcpyAsync(&r->h_counters_slots[slot], r->d_counters, sizeof(TrialCounters),
                           cudaMemcpyDeviceToHost, r->stream));
  ++r->trials;
  r->stage = 3;
  return APRL_OK;
}

// The residual of the trial copied to `slot` (after the stream has reached
// it); the slot becomes the run's current trial counters.
void trial_read(aprl_run* r, int slot, double residual[4]) {
  r->h_sums = &r->h_sums_slots[slot];
  r->h_counters = &r->h_counters_slots[slot];
  double force;
  const unsigned long long bits = r->h_sums->force_bits;
  std::memcpy(&force, &bits, sizeof force);
  residual[0] = force;
  residual[1] = r->h_sums->defect;
  residual[2] = r->h_sums->scale;
  residual[3] = static_cast<double>(r->h_sums->calls);
}

aprl_status enqueue_trial(aprl_run* r, int slot, bool ahead) {
  return r->fp32 ? trial_enqueue_t<float>(r, slot, ahead) : trial_enqueue_t<double>(r, slot, ahead);
}

// solveConservativeSourceStep's stopping rule (src/simulation_source_coupling.cpp:50).
bool trial_converged(const aprl_run_config& c, unsigned iterations, const double res[4],
                     double& force, double& work) {
  force = res[0];
  work = res[3] == 0. ? 0. : (res[2] > 0. ? res[1] / res[2] : res[1]);
  return iterations >= (res[3] > 0. ? 2u : 1u) && force < c.force_tolerance &&
         work < c.work_tolerance;
}

aprl_status do_trial(aprl_run* r, double residual[4]) {
  TRY(enqueue_trial(r, 0, false));
  TRY(check_device(r));
  trial_read(r, 0, residual);
  return APRL_OK;
}

aprl_status do_commit(aprl_run* r) {
  if (r->stage != 3) return fail(APRL_ERR_RUNTIME, "Commit requires a completed coupling trial");
  const aprl_run_config& c = r->cfg;
  // E^{n+1} = E* - dt/eps0 J, in place where J is nonzero: nothing to do
  // when J is known to be zero.
  if (!r->j_zero) {
    TuneLaunch tl;
    TRY(tune_begin(r, kTuneCommit, tl));
    const dim3 block = kGridBlocks[tl.candidate];
    TRY(launch(r, kElectricCommit, electric_commit_kernel<double>, grid3(c, block), block,
               make_grid<double>(r)));
    TRY(tune_end(r, tl));
  }
  r->cur = 1 - r->cur;
  // The counters of the converged trial (read back with its residual) give
  // every compaction size: no host round trip in the commit.
  const TrialCounters& tc = *r->h_counters;
  const unsigned long long kept_old = r->nc ? tc.carriers_kept : 0;
  const unsigned long long kept_born = r->np ? tc.born_kept : 0;
  // Carriers: surviving old carriers, then carriers born this step, in
  // particle order (retainedCarriers, src/simulation.cpp:4401-4405).
  TRY(reserve_carriers(r, kept_old + kept_born));
  if (r->nc) {
    TRY(compact_offsets(r, r->c_keep, 1, r->nc));
    TRY(launch(r, kGatherCarriers, gather_carriers_kernel, dim3(blocks_for(r->nc, kScanBlock)),
               dim3(kScanBlock), r->c_alt, r->c_out, (const unsigned char*)r->c_keep,
               (unsigned char)1, (long long)r->nc, (const unsigned*)r->scan_offset, 0ull));
  }
  if (r->np && kept_born) {
    TRY(compact_offsets(r, r->born_keep, 1, r->np));
    TRY(launch(r, kGatherCarriers, gather_carriers_kernel, dim3(blocks_for(r->np, kScanBlock)),
               dim3(kScanBlock), r->c_alt, r->born, (const unsigned char*)r->born_keep,
               (unsigned char)1, (long long)r->np, (const unsigned*)r->scan_offset,
               (unsigned long long)kept_old));
  }
  std::swap(r->c, r->c_alt);
  r->nc = kept_old + kept_born;
  // Particles: the retained list in order (src/simulation.cpp:4916, 5581).
  if (r->np) {
    const unsigned long long kept = tc.retained;
    TRY(compact_offsets(r, r->action, 0, r->np));
    TRY(launch(r, kGatherParticles, gather_particles_kernel, dim3(blocks_for(r->np, kScanBlock)),
               dim3(kScanBlock), r->p_alt, r->p, (const double*)r->x1, (const double*)r->y1,
               (const double*)r->z1, (const double*)r->ux1, (const double*)r->uy1,
               (const double*)r->uz1, (const unsigned char*)r->frozen1,
               (const unsigned char*)r->action, (unsigned char)0, (long long)r->np,
               (const unsigned*)r->scan_offset));
    std::swap(r->p, r->p_alt);
    r->np = kept;
    // Particles move about one cell per step, so the cell order survives a
    // few steps: re-sorting every kSortInterval steps kept push_deposit and
    // the residual at their sorted speed on the dipole and drift workloads
    // (1M particles: step 4.24 -> 4.14 ms against sorting every step; never
    // sorting, 8.4 ms).  Storage order changes no integer result; it changes
    // J only to roundoff through the order of the FP64 atomics, and not at
    // all in the deterministic mode, whose fixed-point sum is order-free.
    if (r->step % kSortInterval == 0) TRY(sort_particles(r));
  }
  add_counters(r->cumulative, tc);
  r->held = tc.held;
  r->stage = 4;
  return APRL_OK;
}

// MovingWindowFields::shift plane insertion on the ring (field type F).
template <class F>
aprl_status shift_insert_t(aprl_run* r) {
  const aprl_run_config& c = r->cfg;
  ShiftArgs<F> sa{};
  sa.g = make_grid<F>(r);
  TRY(inlet_table(r, r->offset, r->step, sa.inlet));
  for (int h = 0; h < 8; ++h) {
    sa.h[h] = r->hist[h].view();
    const int comp = r->hist[h].component;
    sa.history_base[h] = comp < 3 ? r->zb_e[comp] : r->zb_b[comp - 3];
  }
  int max_row = (int)std::max(c.nx, c.ny) + 1, max_slots = 1;
  for (int h = 0; h < 8; ++h) max_slots = std::max(max_slots, r->hist[h].slots);
  const int ydim = std::max(max_slots, (int)c.ny + 1);
  return launch(r, kShiftInsert, shift_insert_kernel<F>,
                dim3(blocks_for(max_row, 32), blocks_for(ydim, 8), 14), dim3(32, 8), sa);
}

// Simulation::completeMovingInletLayer (src/simulation_moving_window.cpp:312-318):
// the inlet-layer charge of the stored particles and of the pending entries
// due within 8 steps (visitNear), then Ez of the inserted layer.
aprl_status inlet_charge_match(aprl_run* r) {
  const aprl_run_config& c = r->cfg;
  InletMatchArgs m{};
  m.p = r->p;
  m.np = (long long)r->np;
  m.src = r->queue.d;
  const auto& q = r->queue;
  if (q.extracted) {
    if (r->step < q.initial_step || r->step > q.maximum_step)
      return fail(APRL_ERR_RUNTIME, "Invalid pending support view");
    const uint64_t room = q.maximum_step - r->step;
    const uint64_t until = r->step + std::min<uint64_t>(8, room);
    const size_t end = q.offsets[until - q.initial_step + 1];
    if (end > q.cursor) {
      m.pbegin = (long long)q.cursor;
      m.pcount = (long long)(end - q.cursor);
    }
    m.steps = r->step - q.initial_step;
  }
  m.held_distance_per_beta = held_distance_per_beta(c);
  m.origin[0] = c.reference_origin[0];
  m.origin[1] = c.reference_origin[1];
  m.origin[2] = std::fma(static_cast<double>(r->offset), c.dz, c.reference_origin[2]);
  m.dx = c.dx;
  m.dy = c.dy;
  m.dz = c.dz;
  m.nx = (int)c.nx;
  m.ny = (int)c.ny;
  m.shape = c.shape;
  m.rho = r->inlet_rho;
  m.status = r->d_status;
  const size_t nodes = (size_t)(c.nx + 1) * (c.ny + 1);
  if (r->deterministic) {
    m.rho_pairs = r->inlet_rho_pairs;
    m.rho_scale = fixed_scale(4.0 * r->max_abs_charge / (c.dx * c.dy * c.dz));
    CUDA_TRY(cudaMemsetAsync(r->inlet_rho_pairs, 0, 2 * nodes * sizeof(unsigned long long),
                             r->stream));
  } else {
    CUDA_TRY(cudaMemsetAsync(r->inlet_rho, 0, nodes * sizeof(double), r->stream));
  }
  TRY(launch(r, kInletCharge, inlet_charge_kernel, dim3(blocks_for(m.np + m.pcount, 128)),
             dim3(128), m));
  if (r->deterministic)
    TRY(launch(r, kFixedConvert, fixed_convert_kernel, dim3(blocks_for(nodes, 256)), dim3(256),
               (const unsigned long long*)r->inlet_rho_pairs, r->inlet_rho, (long long)nodes,
               1.0 / m.rho_scale));
  InletCompleteArgs ca{};
  ca.g = make_grid<double>(r);
  ca.rho = r->inlet_rho;
  ca.cx = (int)c.cpml_cells_x;
  ca.cy = (int)c.cpml_cells_y;
  ca.status = r->d_status;
  return launch(r, kInletComplete, inlet_complete_kernel,
                dim3(blocks_for(c.nx + 1, 32), blocks_for(c.ny + 1, 8)), dim3(32, 8), ca);
}

// `defer_check`: leave the device status to the next read (the stepping loop
// reads it with the next trial's residual and once at its end).
aprl_status do_shift(aprl_run* r, bool defer_check = false) {
  if (r->stage != 4)
    return fail(APRL_ERR_RUNTIME, "Moving-window requires one left shift after each complete step");
  if (r->ledger_on) TRY(ledger_finish(r));
  const aprl_run_config& c = r->cfg;
  r->time += c.dt;
  r->step += 1;
  r->offset = c.initial_offset - static_cast<int64_t>(r->step);
  for (int a = 0; a < 3; ++a) {
    const int nze = (int)(c.nz + (a != 2)), nzb = (int)(c.nz + (a == 2));
    r->zb_e[a] = (r->zb_e[a] + nze - 1) % nze;
    r->zb_b[a] = (r->zb_b[a] + nzb - 1) % nzb;
  }
  TRY(shift_insert_t<double>(r));
  if (c.inlet_charge_match) TRY(inlet_charge_match(r));
  if (r->ledger_on) TRY(ledger_shift(r));
  r->origin[2] = std::fma(static_cast<double>(r->offset), c.dz, c.reference_origin[2]);
  if (r->np)
    TRY(launch(r, kInletCheck, inlet_check_kernel, dim3(blocks_for(r->np, 256)), dim3(256),
               (const double*)r->p.z, (const unsigned char*)r->p.frozen, (long long)r->np,
               r->origin[2], r->d_status));
  if (r->nc) {
    // Crop flags and counts in one round trip (with the device status).
    const double upper = std::fma(static_cast<double>(c.nz), c.dz, r->origin[2]);
    CUDA_TRY(cudaMemsetAsync(r->d_counters, 0, sizeof(TrialCounters), r->stream));
    TRY(launch(r, kCropFlags, crop_flags_kernel, dim3(blocks_for(r->nc, 256)), dim3(256), r->c,
               (long long)r->nc, upper, r->origin[2], r->c_keep, r->d_counters, r->d_status));
    CUDA_TRY(cudaMemcpyAsync(r->h_counters, r->d_counters, sizeof(TrialCounters),
                             cudaMemcpyDeviceToHost, r->stream));
    TRY(check_device(r));
    const unsigned long long kept = r->nc - r->h_counters->cropped;
    TRY(compact_offsets(r, r->c_keep, 1, r->nc));
    TRY(launch(r, kGatherCarriers, gather_carriers_kernel, dim3(blocks_for(r->nc, kScanBlock)),
               dim3(kScanBlock), r->c_alt, r->c, (const unsigned char*)r->c_keep,
               (unsigned char)1, (long long)r->nc, (const unsigned*)r->scan_offset, 0ull));
    std::swap(r->c, r->c_alt);
    r->nc = kept;
    r->cumulative.cropped += r->h_counters->cropped;
    r->cumulative.cropped_charge += r->h_counters->cropped_charge;
  } else if (!defer_check) {
    TRY(check_device(r));
  }
  r->stage = 0;
  return APRL_OK;
}

HistoryBuffer* find_history(aprl_run* r, unsigned index) {
  for (auto& h : r->hist)
    if ((unsigned)h.abi_index == index) return &h;
  return nullptr;
}

}  // namespace

// The calling thread's error message, for the other host files of the
// library (the scan server).
namespace aprl_gpu {
// The message of a run's failure in aprl_runs_step (the scan server).
const char* run_error(const aprl_run* r) { return r->error.c_str(); }

aprl_status report_error(aprl_status status, const char* message) {
  g_error = message;
  return status;
}
}  // namespace aprl_gpu

// ===========================================================================
extern "C" {

const char* aprl_last_error(void) { return g_error.c_str(); }
int aprl_abi_version(void) { return APRL_GPU_ABI_VERSION; }

const char* aprl_kernel_name(unsigned kernel) {
  return kernel < kKernelCount ? kKernelNames[kernel] : "";
}

aprl_status aprl_cowan_coefficients(double dx, double dy, double dz, double out[12]) {
  return cowan(dx, dy, dz, out);
}

aprl_status aprl_magnet_prepare(aprl_magnet* m) {
  if (!m) return fail(APRL_ERR_INVALID_ARGUMENT, "null magnet");
  if (!std::isfinite(m->center[0]) || !std::isfinite(m->center[1]) || !std::isfinite(m->center[2]) ||
      !(m->length >= 0.0) || !std::isfinite(m->length) || !std::isfinite(m->peak_field) ||
      !std::isfinite(m->polarization_angle))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid SI magnetic element");
  if (m->type == APRL_MAGNET_PLANAR_UNDULATOR && (!(m->period > 0.0) || !std::isfinite(m->period)))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Undulator period must be positive");
  if (m->type == APRL_MAGNET_PLANAR_UNDULATOR && m->gaussian_fringe &&
      (!(m->fringe_relative_cutoff > 0.0) || !(m->fringe_relative_cutoff < 1.0)))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Undulator fringe_relative_cutoff must be in (0,1)");
  if (m->type == APRL_MAGNET_UNIFORM_DIPOLE && !(m->length > 0.0))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Dipole length must be positive");
  if (m->type == APRL_MAGNET_QUADRUPOLE && (!(m->length > 0.0) || !std::isfinite(m->quadrupole_gradient)))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Quadrupole length/gradient is invalid");
  m->wave_number = m->type == APRL_MAGNET_PLANAR_UNDULATOR ? 2.0 * kPi / m->period : 0.0;
  m->fringe_extent = m->type == APRL_MAGNET_PLANAR_UNDULATOR && m->gaussian_fringe
                         ? std::sqrt(-2.0 * std::log(m->fringe_relative_cutoff)) / m->wave_number
                         : 0.0;
  m->cos_angle = std::cos(m->polarization_angle);
  m->sin_angle = std::sin(m->polarization_angle);
  return APRL_OK;
}

aprl_status aprl_boris_push(size_t count, double* x, double* y, double* z, double* ux, double* uy,
                            double* uz, const double* charge, const double* mass,
                            const double* electric, const double* magnetic, double dt) {
  if (count && (!x || !y || !z || !ux || !uy || !uz || !charge || !mass || !electric || !magnetic))
    return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  // pushMomentum's parameter check (src/eb_particles.cpp:104-107).
  if (!(dt > 0.0) || !std::isfinite(dt))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid SI particle pusher parameters");
  for (size_t i = 0; i < count; ++i)
    if (!(mass[i] > 0.0) || !std::isfinite(mass[i]) || !std::isfinite(charge[i]))
      return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid SI particle pusher parameters");
  if (!count) return APRL_OK;
  cudaStream_t stream = nullptr;
  CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  double* d = nullptr;
  const size_t words = 14 * count;  // x y z ux uy uz q m, E and B (3 each)
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&d), words * sizeof(double), stream);
  if (e != cudaSuccess) {
    cudaStreamDestroy(stream);
    return fail(APRL_ERR_CUDA, "cudaMallocAsync: %s", cudaGetErrorString(e));
  }
  double* in[8] = {x, y, z, ux, uy, uz, const_cast<double*>(charge), const_cast<double*>(mass)};
  for (int k = 0; k < 8 && e == cudaSuccess; ++k)
    e = cudaMemcpyAsync(d + k * count, in[k], count * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d + 8 * count, electric, 3 * count * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d + 11 * count, magnetic, 3 * count * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) {
    BorisArgs a{};
    a.count = (long long)count;
    a.x = d; a.y = d + count; a.z = d + 2 * count;
    a.ux = d + 3 * count; a.uy = d + 4 * count; a.uz = d + 5 * count;
    a.q = d + 6 * count; a.m = d + 7 * count; a.e = d + 8 * count; a.b = d + 11 * count;
    a.dt = dt;
    boris_push_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(a);
    e = cudaGetLastError();
  }
  for (int k = 0; k < 6 && e == cudaSuccess; ++k)
    e = cudaMemcpyAsync(in[k], d + k * count, count * 8, cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(d, stream);
  const cudaError_t s2 = cudaStreamSynchronize(stream);
  cudaStreamDestroy(stream);
  if (e == cudaSuccess) e = s2;
  if (e != cudaSuccess) return fail(APRL_ERR_CUDA, "Boris push: %s", cudaGetErrorString(e));
  return APRL_OK;
}

aprl_status aprl_run_create(const aprl_run_config* config, void* stream, aprl_run** out) {
  if (!config || !out) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  TRY(validate(*config));
  aprl_run* r = new (std::nothrow) aprl_run();
  if (!r) return fail(APRL_ERR_RUNTIME, "out of host memory");
  r->cfg = *config;
  r->stream = static_cast<cudaStream_t>(stream);
  aprl_status s = cowan(config->dx, config->dy, config->dz, r->coeff);
  auto cleanup = [&](aprl_status st) {
    aprl_run_destroy(r);
    return st;
  };
  if (s != APRL_OK) return cleanup(s);
  {
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess || !(r->pool = device_pool(device)))
      return cleanup(fail(APRL_ERR_CUDA, "no stream-ordered memory pool on this device"));
    r->device = device;
  }
  const aprl_run_config& c = *config;
  r->fp32 = c.precision == APRL_PRECISION_FP32_MIXED;
  r->fes = sizeof(double);
  const size_t fes = r->fes;
  for (int a = 0; a < 3; ++a) {
    for (int k = 0; k < 2; ++k) {
      if ((s = device_alloc(r, &r->e[k][a], e_count(c, a))) != APRL_OK) return cleanup(s);
      cudaMemsetAsync(r->e[k][a], 0, e_count(c, a) * 8, r->stream);
    }
    if ((s = device_alloc(r, &r->b[a], b_count(c, a))) != APRL_OK) return cleanup(s);
    cudaMemsetAsync(r->b[a], 0, b_count(c, a) * 8, r->stream);
    if ((s = device_alloc_bytes(r, &r->jc[a], e_count(c, a) * fes)) != APRL_OK) return cleanup(s);
    cudaMemsetAsync(r->jc[a], 0, e_count(c, a) * fes, r->stream);
    const size_t plane = (size_t)(c.nx + (a != 0)) * (c.ny + (a != 1));
    if ((s = device_alloc(r, &r->lower[a], plane)) != APRL_OK) return cleanup(s);
    const size_t gather_bytes = r->fp32 ? sizeof(float) : sizeof(double);
    if ((s = device_alloc_bytes(r, &r->orbit[a], e_count(c, a) * gather_bytes)) != APRL_OK)
      return cleanup(s);
    if (r->fp32 && (s = device_alloc(r, &r->bshadow[a], b_count(c, a))) != APRL_OK)
      return cleanup(s);
    r->max_rate[a] = maximum_rate(c, a);
  }
  // CPML profiles (x, y) for magnetic (half-integer) and electric nodes.
  for (int axis = 0; axis < 2; ++axis) {
    for (int electric = 0; electric < 2; ++electric) {
      const HostProfile hp = make_profile(c, axis, electric != 0);
      DeviceProfile& dp = electric ? r->eprof[axis] : r->mprof[axis];
      const size_t n = hp.ikm1.size();
      if ((s = device_alloc(r, &dp.ikm1, n)) != APRL_OK) return cleanup(s);
      if ((s = device_alloc(r, &dp.decay, n)) != APRL_OK) return cleanup(s);
      if ((s = device_alloc(r, &dp.drive, n)) != APRL_OK) return cleanup(s);
      if ((s = device_alloc(r, &dp.ordinal, n)) != APRL_OK) return cleanup(s);
      run_copy(r, dp.ikm1, hp.ikm1.data(), n * 8, cudaMemcpyHostToDevice);
      run_copy(r, dp.decay, hp.decay.data(), n * 8, cudaMemcpyHostToDevice);
      run_copy(r, dp.drive, hp.drive.data(), n * 8, cudaMemcpyHostToDevice);
      run_copy(r, dp.ordinal, hp.ordinal.data(), n * sizeof(int), cudaMemcpyHostToDevice);
      dp.active = hp.active;
    }
  }
  // Active histories: ABI index, component (ABI), derivative axis.
  const int defs[8][3] = {{0, 3, 1}, {3, 4, 0}, {4, 5, 0}, {5, 5, 1},
                          {6, 0, 1}, {9, 1, 0}, {10, 2, 0}, {11, 2, 1}};
  for (int h = 0; h < 8; ++h) {
    HistoryBuffer& hb = r->hist[h];
    hb.abi_index = defs[h][0];
    hb.component = defs[h][1];
    const int der = defs[h][2];
    size_t sh[3];
    comp_shape(c, (unsigned)hb.component, sh);
    const DeviceProfile& prof = hb.component < 3 ? r->eprof[der] : r->mprof[der];
    hb.slots = prof.active;
    hb.layers = (int)sh[2];
    hb.row = (int)(der == 0 ? sh[1] : sh[0]);
    if ((s = device_alloc(r, &hb.data, hb.length())) != APRL_OK) return cleanup(s);
    cudaMemsetAsync(hb.data, 0, std::max<size_t>(1, hb.length()) * 8, r->stream);
  }
  for (int a = 0; a < 3; ++a) {
    const uint64_t cells = a == 0 ? c.nx : (a == 1 ? c.ny : c.nz);
    r->tiles[a] = (int)((cells + (1u << kTileShift) - 1) >> kTileShift);
  }
  r->ntiles = (size_t)r->tiles[0] * r->tiles[1] * r->tiles[2];
  while (r->sort_bits < 32 && ((size_t)1 << r->sort_bits) < r->ntiles) ++r->sort_bits;
  if ((s = device_alloc(r, &r->res_ticket, 1)) != APRL_OK) return cleanup(s);
  cudaMemsetAsync(r->res_ticket, 0, sizeof(unsigned), r->stream);
  r->deterministic = c.deterministic != 0;
  if (r->deterministic) {
    for (int a = 0; a < 3; ++a) {
      if ((s = device_alloc(r, &r->jq[a], 2 * e_count(c, a))) != APRL_OK) return cleanup(s);
      cudaMemsetAsync(r->jq[a], 0, 2 * e_count(c, a) * sizeof(unsigned long long), r->stream);
    }
    if (c.inlet_charge_match &&
        (s = device_alloc(r, &r->inlet_rho_pairs, 2 * (size_t)(c.nx + 1) * (c.ny + 1))) != APRL_OK)
      return cleanup(s);
  }
  if ((s = device_alloc(r, &r->d_counters, 1)) != APRL_OK) return cleanup(s);
  if ((s = device_alloc(r, &r->d_sums, 1)) != APRL_OK) return cleanup(s);
  if ((s = device_alloc(r, &r->d_status, 1)) != APRL_OK) return cleanup(s);
  if ((s = device_alloc(r, &r->scan_total, 1)) != APRL_OK) return cleanup(s);
  cudaMemsetAsync(r->d_status, 0, sizeof(DeviceStatus), r->stream);
  if ((s = device_alloc(r, &r->d_stop, 1)) != APRL_OK) return cleanup(s);
  if (c.inlet_charge_match &&
      (s = device_alloc(r, &r->inlet_rho, (size_t)(c.nx + 1) * (c.ny + 1))) != APRL_OK)
    return cleanup(s);
  // The read-back areas, 64-byte aligned inside one reused page-locked block.
  if (!(r->pinned = pinned_take()))
    return cleanup(fail(APRL_ERR_CUDA, "cudaMallocHost failed"));
  {
    char* at = static_cast<char*>(r->pinned);
    auto carve = [&](size_t bytes) {
      char* p = at;
      at += (bytes + 63) / 64 * 64;
      return static_cast<void*>(p);
    };
    r->h_sums_slots = static_cast<ResidualSums*>(carve(kTrialSlots * sizeof(ResidualSums)));
    r->h_status = static_cast<DeviceStatus*>(carve(sizeof(DeviceStatus)));
    r->h_counters_slots = static_cast<TrialCounters*>(carve(kTrialSlots * sizeof(TrialCounters)));
    r->h_stop = static_cast<int*>(carve(sizeof(int)));
    r->h_total = static_cast<unsigned long long*>(carve(sizeof(unsigned long long)));
    std::memset(r->pinned, 0, kPinnedBlock);
  }
  if (cudaStreamCreateWithFlags(&r->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&r->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&r->join, cudaEventDisableTiming) != cudaSuccess)
    return cleanup(fail(APRL_ERR_CUDA, "side stream creation failed"));
  if (cudaStreamCreateWithFlags(&r->upload, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(APRL_ERR_CUDA, "upload stream creation failed"));
  for (auto& component : r->staging)
    for (auto& st : component)
      if (cudaEventCreateWithFlags(&st.staged, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&st.drained, cudaEventDisableTiming) != cudaSuccess)
        return cleanup(fail(APRL_ERR_CUDA, "upload event creation failed"));
  r->h_sums = r->h_sums_slots;
  r->h_counters = r->h_counters_slots;
  r->offset = c.initial_offset;
  r->origin[0] = c.reference_origin[0];
  r->origin[1] = c.reference_origin[1];
  r->origin[2] = std::fma(static_cast<double>(c.initial_offset), c.dz, c.reference_origin[2]);
  if (cudaStreamSynchronize(r->stream) != cudaSuccess)
    return cleanup(fail(APRL_ERR_CUDA, "stream synchronise failed at creation"));
  *out = r;
  return APRL_OK;
}

aprl_status aprl_run_destroy(aprl_run* r) {
  if (!r) return APRL_OK;
  if (r->stream) cudaStreamSynchronize(r->stream); else cudaDeviceSynchronize();
  if (r->side) {
    cudaStreamSynchronize(r->side);
    cudaStreamDestroy(r->side);
  }
  if (r->fork) cudaEventDestroy(r->fork);
  if (r->join) cudaEventDestroy(r->join);
  if (r->upload) {
    cudaStreamSynchronize(r->upload);
    cudaStreamDestroy(r->upload);
  }
  for (auto& component : r->staging)
    for (auto& st : component) {
      if (st.staged) cudaEventDestroy(st.staged);
      if (st.drained) cudaEventDestroy(st.drained);
      device_free(r, st.data);
    }
  for (auto& t : r->pending) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  for (auto& p : r->tune_pending) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  for (auto e : r->event_pool) cudaEventDestroy(e);
  for (int a = 0; a < 3; ++a) {
    device_free(r, r->e[0][a]); device_free(r, r->e[1][a]); device_free(r, r->b[a]); device_free(r, r->jc[a]);
    device_free(r, r->lower[a]);
    device_free(r, r->orbit[a]);
    device_free(r, r->bshadow[a]);
  }
  for (int a = 0; a < 6; ++a) device_free(r, r->ref[a]);
  for (int a = 0; a < 2; ++a) {
    for (DeviceProfile* dp : {&r->mprof[a], &r->eprof[a]}) {
      device_free(r, dp->ikm1); device_free(r, dp->decay); device_free(r, dp->drive); device_free(r, dp->ordinal);
    }
  }
  for (auto& h : r->hist) device_free(r, h.data);
  free_particles(r, r->p);
  free_particles(r, r->p_alt);
  double* singles[] = {r->x1,       r->y1,       r->z1,       r->ux1,        r->uy1,
                       r->uz1,      r->used_e,   r->used_b,   r->next_e,     r->next_b,
                       r->abs_work, r->slots.x0, r->slots.y0, r->slots.z0,   r->slots.dt,
                       r->d_detector, r->dep_b[0], r->dep_b[1], r->dep_b[2], r->dep_e[0],
                       r->dep_e[1], r->dep_e[2]};
  for (double* d : singles) device_free(r, d);
  device_free(r, r->slots.seen);
  device_free(r, r->frozen1);
  free_pending(r, r->queue.d);
  device_free(r, r->action);
  device_free(r, r->dep_mode);
  device_free(r, r->born_keep);
  device_free(r, r->slot_order);
  for (int k = 0; k < 2; ++k) {
    device_free(r, r->sort_key[k]);
    device_free(r, r->sort_index[k]);
  }
  device_free(r, r->radix_count);
  device_free(r, r->chunk_sum);
  device_free(r, r->chunk_offset);
  device_free(r, r->res_partial);
  device_free(r, r->res_ticket);
  device_free(r, r->surface_points);
  device_free(r, r->surface_table);
  for (int a = 0; a < 3; ++a) device_free(r, r->jq[a]);
  device_free(r, r->inlet_rho_pairs);
  free_carriers(r, r->born);
  free_carriers(r, r->c);
  free_carriers(r, r->c_alt);
  free_carriers(r, r->c_out);
  device_free(r, r->c_keep);
  device_free(r, r->gauss_node);
  device_free(r, r->gauss_scratch);
  device_free(r, r->d_ledger);
  device_free(r, r->d_ledger_partial);
  device_free(r, r->ledger_pre[0]);
  device_free(r, r->ledger_pre[1]);
  device_free(r, r->d_counters);
  device_free(r, r->d_sums);
  device_free(r, r->d_status);
  device_free(r, r->scan_count);
  device_free(r, r->scan_offset);
  device_free(r, r->scan_total);
  r->h_sums_slots = nullptr;
  r->h_stop = nullptr;
  device_free(r, r->d_stop);
  device_free(r, r->inlet_rho);
  r->h_status = nullptr;
  r->h_counters_slots = nullptr;
  r->h_total = nullptr;
  pinned_give(r->pinned);
  delete r;
  return APRL_OK;
}

aprl_status aprl_run_set_reference(aprl_run* r, unsigned a, const double* host, size_t count) {
  if (!r || a >= 6) return fail(APRL_ERR_OUT_OF_RANGE, "Moving-window component");
  size_t s[3];
  comp_shape(r->cfg, a, s);
  const size_t n = s[0] * s[1] * (r->cfg.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0));
  if (count != n) return fail(APRL_ERR_INVALID_ARGUMENT, "Reference component size mismatch");
  if (host && !all_finite(host, n)) return fail(APRL_ERR_RUNTIME, "Non-finite moving-window inlet");
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  device_free(r, r->ref[a]);
  r->ref[a] = nullptr;
  TRY(device_alloc(r, &r->ref[a], n));
  if (host)
    CUDA_TRY(run_copy(r, r->ref[a], host, n * 8, cudaMemcpyHostToDevice));
  else
    CUDA_TRY(run_fill(r, r->ref[a], 0, n * 8));
  r->ref_set[a] = true;
  if (a == 3 || a == 4) r->surface_ready = false;  // prepared again from the new table
  return APRL_OK;
}

aprl_status aprl_run_set_reference_planes(aprl_run* r, unsigned a, uint64_t first, uint64_t planes,
                                          const double* host) {
  if (!r || a >= 6) return fail(APRL_ERR_OUT_OF_RANGE, "Moving-window component");
  if (!r->ref_set[a]) return fail(APRL_ERR_INVALID_ARGUMENT, "Reference component not allocated");
  size_t s[3];
  comp_shape(r->cfg, a, s);
  const uint64_t layers = r->cfg.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0);
  if (!host || first > layers || planes > layers - first)
    return fail(APRL_ERR_OUT_OF_RANGE, "Reference planes outside the prepared native field");
  const size_t plane = s[0] * s[1];
  if (!all_finite(host, planes * plane))
    return fail(APRL_ERR_RUNTIME, "Non-finite moving-window inlet");
  const size_t bytes = planes * plane * 8;
  if (bytes) {
    aprl_run::Stage& st = r->staging[a][r->staging_next[a]];
    if (st.bytes < bytes) {
      // The old block's last reader is the stream's copy out of it, which
      // the stream-ordered free follows.  The new block is allocated in the
      // upload stream's order, without a wait: the transfer into it follows
      // on that stream, and the run's stream reads it only after `staged`.
      device_free(r, st.data);
      st.data = nullptr;
      st.bytes = 0;
      st.used = false;
      void* block = nullptr;
      const cudaError_t e = cudaMallocFromPoolAsync(&block, bytes, r->pool, r->upload);
      if (e != cudaSuccess)
        return fail(APRL_ERR_CUDA, "device allocation of %zu bytes failed: %s", bytes,
                    cudaGetErrorString(e));
      st.data = static_cast<double*>(block);
      st.bytes = bytes;
    }
    r->staging_next[a] ^= 1;
    if (st.used) CUDA_TRY(cudaStreamWaitEvent(r->upload, st.drained, 0));
    CUDA_TRY(cudaMemcpyAsync(st.data, host, bytes, cudaMemcpyHostToDevice, r->upload));
    CUDA_TRY(cudaEventRecord(st.staged, r->upload));
    CUDA_TRY(cudaStreamWaitEvent(r->stream, st.staged, 0));
    CUDA_TRY(cudaMemcpyAsync(r->ref[a] + first * plane, st.data, bytes,
                             cudaMemcpyDeviceToDevice, r->stream));
    CUDA_TRY(cudaEventRecord(st.drained, r->stream));
    st.used = true;
  }
  if (a == 3 || a == 4) r->surface_ready = false;
  return APRL_OK;
}

aprl_status aprl_run_field_shape(const aprl_run* r, unsigned a, uint64_t shape[3]) {
  if (!r || a >= 9) return fail(APRL_ERR_OUT_OF_RANGE, "Field component");
  size_t s[3];
  comp_shape(r->cfg, a, s);
  for (int d = 0; d < 3; ++d) shape[d] = s[d];
  return APRL_OK;
}

static aprl_status field_io(aprl_run* r, unsigned a, const double* in, double* out, size_t count) {
  if (!r || a >= 9) return fail(APRL_ERR_OUT_OF_RANGE, "Field component");
  size_t s[3];
  comp_shape(r->cfg, a, s);
  if (count != s[0] * s[1] * s[2] || (!in && !out))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Field component size mismatch");
  if (r->stage != 0 && r->stage != 4 && in)
    return fail(APRL_ERR_RUNTIME, "Fields can only be replaced between steps");
  const size_t plane = s[0] * s[1];
  if (a >= 6) {
    if (in) r->j_zero = false;
    return copy_ring(r, static_cast<double*>(r->jc[a - 6]), in, out, plane, s[2], 0);
  }
  if (a < 3) return copy_ring(r, r->e[r->cur][a], in, out, plane, s[2], r->zb_e[a]);
  return copy_ring(r, r->b[a - 3], in, out, plane, s[2], r->zb_b[a - 3]);
}

aprl_status aprl_run_set_field(aprl_run* r, unsigned a, const double* host, size_t count) {
  if (r && a < 6) r->ledger_start_ready = false;  // the next begin measures the new fields
  return field_io(r, a, host, nullptr, count);
}

aprl_status aprl_run_get_field(aprl_run* r, unsigned a, double* host, size_t count) {
  return field_io(r, a, nullptr, host, count);
}

aprl_status aprl_run_history_length(const aprl_run* r, unsigned index, uint64_t* length) {
  if (!r || index >= 12) return fail(APRL_ERR_OUT_OF_RANGE, "CPML checkpoint history index is out of range");
  HistoryBuffer* h = find_history(const_cast<aprl_run*>(r), index);
  *length = h ? h->length() : 0;
  return APRL_OK;
}

static aprl_status history_io(aprl_run* r, unsigned index, const double* in, double* out, size_t count) {
  if (!r || index >= 12) return fail(APRL_ERR_OUT_OF_RANGE, "CPML checkpoint history index is out of range");
  HistoryBuffer* h = find_history(r, index);
  const size_t length = h ? h->length() : 0;
  if (count != length) return fail(APRL_ERR_INVALID_ARGUMENT, "CPML history size mismatch");
  if (!length) return APRL_OK;
  const int comp = h->component;
  const int base = comp < 3 ? r->zb_e[comp] : r->zb_b[comp - 3];
  return copy_ring(r, h->data, in, out, (size_t)h->row, (size_t)h->layers, base,
                   (size_t)h->slots);
}

aprl_status aprl_run_set_history(aprl_run* r, unsigned index, const double* host, size_t count) {
  return history_io(r, index, host, nullptr, count);
}

aprl_status aprl_run_get_history(aprl_run* r, unsigned index, double* host, size_t count) {
  return history_io(r, index, nullptr, host, count);
}

aprl_status aprl_run_set_particles(aprl_run* r, size_t n, const double* x, const double* y,
                                   const double* z, const double* ux, const double* uy,
                                   const double* uz, const double* q, const double* m,
                                   const uint64_t* id, int reset_carriers) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Particles can only be replaced between steps");
  if (n && (!x || !y || !z || !ux || !uy || !uz || !q || !m || !id))
    return fail(APRL_ERR_INVALID_ARGUMENT, "null particle array");
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(z[i]) ||
        !std::isfinite(ux[i]) || !std::isfinite(uy[i]) || !std::isfinite(uz[i]) ||
        !std::isfinite(q[i]) || !(m[i] > 0.0))
      return fail(APRL_ERR_INVALID_ARGUMENT, "Particle %zu has a non-finite state or nonpositive mass", i);
  TRY(reserve_particles(r, n));
  TRY(reserve_carriers(r, 1));
  note_charges(r, q, n);
  r->np = 0;
  const double* src[] = {x, y, z, ux, uy, uz, q, m};
  double* dst[] = {r->p.x, r->p.y, r->p.z, r->p.ux, r->p.uy, r->p.uz, r->p.q, r->p.m};
  for (int k = 0; k < 8; ++k)
    CUDA_TRY(run_copy(r, dst[k], src[k], n * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(run_copy(r, r->p.id, id, n * 8, cudaMemcpyHostToDevice));
  std::vector<unsigned long long> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  if (n) CUDA_TRY(run_copy(r, r->p.order, order.data(), n * 8, cudaMemcpyHostToDevice));
  if (n) {
    CUDA_TRY(run_fill(r, r->p.frozen, 0, n));
    CUDA_TRY(run_fill(r, r->p.beta, 0, n * 8));
  }
  r->next_order = n;
  r->np = n;
  r->held = 0;
  if (reset_carriers) r->nc = 0;
  TRY(sort_particles(r));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

aprl_status aprl_run_particle_count(const aprl_run* r, size_t* count) {
  if (!r || !count) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *count = r->np;
  return APRL_OK;
}

// Storage is tile-sorted; read-out restores the reference's list order.
static aprl_status storage_permutation(aprl_run* r, const unsigned long long* device_order,
                                       size_t n, std::vector<size_t>& perm) {
  std::vector<unsigned long long> order(n);
  if (n) CUDA_TRY(run_copy(r, order.data(), device_order, n * 8, cudaMemcpyDeviceToHost));
  perm.resize(n);
  for (size_t i = 0; i < n; ++i) perm[i] = i;
  std::sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return order[a] < order[b]; });
  return APRL_OK;
}

aprl_status aprl_run_get_particles(aprl_run* r, size_t capacity, double* x, double* y, double* z,
                                   double* ux, double* uy, double* uz, double* q, double* m,
                                   uint64_t* id, size_t* count) {
  if (!r || !count) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (capacity < r->np) return fail(APRL_ERR_INVALID_ARGUMENT, "Particle buffer too small");
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  const size_t n = r->np;
  std::vector<size_t> perm;
  TRY(storage_permutation(r, r->p.order, n, perm));
  std::vector<double> t(n);
  double* dst[] = {x, y, z, ux, uy, uz, q, m};
  const double* src[] = {r->p.x, r->p.y, r->p.z, r->p.ux, r->p.uy, r->p.uz, r->p.q, r->p.m};
  for (int k = 0; k < 8; ++k) {
    if (!dst[k] || !n) continue;
    CUDA_TRY(run_copy(r, t.data(), src[k], n * 8, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) dst[k][i] = t[perm[i]];
  }
  if (id && n) {
    std::vector<uint64_t> ids(n);
    CUDA_TRY(run_copy(r, ids.data(), r->p.id, n * 8, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) id[i] = ids[perm[i]];
  }
  *count = n;
  return APRL_OK;
}

aprl_status aprl_run_set_held(aprl_run* r, size_t n, const uint8_t* frozen, const double* beta) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Held state can only be set between steps");
  if (n != r->np) return fail(APRL_ERR_INVALID_ARGUMENT, "Held state must cover the particle list");
  if (n && (!frozen || !beta)) return fail(APRL_ERR_INVALID_ARGUMENT, "null held array");
  auto& q = r->queue;
  if (q.extracted) return fail(APRL_ERR_RUNTIME, "Pending queue can only be initialized once");
  const aprl_run_config& c = r->cfg;
  q.initial_step = r->step;
  q.last_step = r->step;
  q.maximum_step = c.maximum_step;
  q.next_due = r->step;
  if (!(c.dz > 0.) || q.initial_step > q.maximum_step)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid pending-window geometry/horizon");
  // The list in reference order.
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  std::vector<size_t> perm;
  TRY(storage_permutation(r, r->p.order, n, perm));
  std::vector<double> v[8];
  const double* dsrc[] = {r->p.x, r->p.y, r->p.z, r->p.ux, r->p.uy, r->p.uz, r->p.q, r->p.m};
  for (int k = 0; k < 8; ++k) {
    std::vector<double> t(n);
    if (n) CUDA_TRY(run_copy(r, t.data(), dsrc[k], n * 8, cudaMemcpyDeviceToHost));
    v[k].resize(n);
    for (size_t i = 0; i < n; ++i) v[k][i] = t[perm[i]];
  }
  std::vector<unsigned long long> ids(n), id(n);
  if (n) CUDA_TRY(run_copy(r, ids.data(), r->p.id, n * 8, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; ++i) id[i] = ids[perm[i]];
  // PendingParticleQueue::extract (src/pending_particle_queue.cpp:128-154).
  const size_t buckets = static_cast<size_t>(q.maximum_step - q.initial_step + 2);
  q.offsets.assign(buckets + 1, 0);
  const double inlet = pending_origin(c, q.initial_step);
  std::vector<size_t> kept, queued, due;
  for (size_t i = 0; i < n; ++i) {
    const double z = v[2][i];
    if (frozen[i] && z < inlet && beta[i] >= 0. && !participates(r, z, beta[i], q.initial_step)) {
      const uint64_t event = first_due(r, z, beta[i]);
      due.push_back(static_cast<size_t>(event - q.initial_step));
      ++q.offsets[event - q.initial_step + 1];
      queued.push_back(i);
    } else {
      kept.push_back(i);
    }
  }
  for (size_t b = 1; b < buckets + 1; ++b) q.offsets[b] += q.offsets[b - 1];
  std::vector<size_t> slot(queued.size());
  {
    std::vector<size_t> insertion(q.offsets);
    for (size_t j = 0; j < queued.size(); ++j) slot[insertion[due[j]]++] = j;
  }
  // Queue entries on the device, in due order.
  free_pending(r, q.d);
  const size_t nq = queued.size();
  q.n = nq;
  q.cursor = 0;
  if (nq) {
    double** qd[] = {&q.d.x, &q.d.y, &q.d.z, &q.d.ux, &q.d.uy, &q.d.uz, &q.d.q, &q.d.m};
    std::vector<double> t(nq);
    for (int k = 0; k < 8; ++k) {
      TRY(device_alloc(r, qd[k], nq));
      for (size_t s = 0; s < nq; ++s) t[s] = v[k][queued[slot[s]]];
      CUDA_TRY(run_copy(r, *qd[k], t.data(), nq * 8, cudaMemcpyHostToDevice));
    }
    TRY(device_alloc(r, &q.d.beta, nq));
    for (size_t s = 0; s < nq; ++s) t[s] = beta[queued[slot[s]]];
    CUDA_TRY(run_copy(r, q.d.beta, t.data(), nq * 8, cudaMemcpyHostToDevice));
    std::vector<unsigned long long> qi(nq);
    for (size_t s = 0; s < nq; ++s) qi[s] = id[queued[slot[s]]];
    TRY(device_alloc(r, &q.d.id, nq));
    CUDA_TRY(run_copy(r, q.d.id, qi.data(), nq * 8, cudaMemcpyHostToDevice));
  }
  // The retained list, in order, with its held state.
  const size_t nk = kept.size();
  if (nk) {
    double* pd[] = {r->p.x, r->p.y, r->p.z, r->p.ux, r->p.uy, r->p.uz, r->p.q, r->p.m};
    std::vector<double> t(nk);
    for (int k = 0; k < 8; ++k) {
      for (size_t s = 0; s < nk; ++s) t[s] = v[k][kept[s]];
      CUDA_TRY(run_copy(r, pd[k], t.data(), nk * 8, cudaMemcpyHostToDevice));
    }
    for (size_t s = 0; s < nk; ++s) t[s] = beta[kept[s]];
    CUDA_TRY(run_copy(r, r->p.beta, t.data(), nk * 8, cudaMemcpyHostToDevice));
    std::vector<unsigned long long> ki(nk), ko(nk);
    std::vector<unsigned char> kf(nk);
    uint64_t held = 0;
    for (size_t s = 0; s < nk; ++s) {
      ki[s] = id[kept[s]];
      ko[s] = s;
      kf[s] = frozen[kept[s]] ? 1 : 0;
      held += kf[s];
    }
    CUDA_TRY(run_copy(r, r->p.id, ki.data(), nk * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(run_copy(r, r->p.order, ko.data(), nk * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(run_copy(r, r->p.frozen, kf.data(), nk, cudaMemcpyHostToDevice));
    r->held = held;
  } else {
    r->held = 0;
  }
  r->np = nk;
  r->next_order = nk;
  q.extracted = true;
  advance_next_due(q);
  TRY(sort_particles(r));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

aprl_status aprl_run_get_held(aprl_run* r, size_t capacity, uint8_t* frozen, double* beta,
                              size_t* count) {
  if (!r || !count) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (capacity < r->np) return fail(APRL_ERR_INVALID_ARGUMENT, "Particle buffer too small");
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  const size_t n = r->np;
  std::vector<size_t> perm;
  TRY(storage_permutation(r, r->p.order, n, perm));
  if (frozen && n) {
    std::vector<unsigned char> f(n);
    CUDA_TRY(run_copy(r, f.data(), r->p.frozen, n, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) frozen[i] = f[perm[i]];
  }
  if (beta && n) {
    std::vector<double> b(n);
    CUDA_TRY(run_copy(r, b.data(), r->p.beta, n * 8, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) beta[i] = b[perm[i]];
  }
  *count = n;
  return APRL_OK;
}

aprl_status aprl_run_carrier_count(const aprl_run* r, size_t* count) {
  if (!r || !count) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *count = r->nc;
  return APRL_OK;
}

aprl_status aprl_run_get_carriers(aprl_run* r, size_t capacity, double* pos, double* vel,
                                  double* q, double* w, size_t* count) {
  if (!r || !count) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (capacity < r->nc) return fail(APRL_ERR_INVALID_ARGUMENT, "Carrier buffer too small");
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  const size_t n = r->nc;
  std::vector<size_t> perm;
  TRY(storage_permutation(r, r->c.key, n, perm));
  std::vector<double> t(n);
  const double* comps[] = {r->c.px, r->c.py, r->c.pz, r->c.vx, r->c.vy, r->c.vz};
  for (int k = 0; k < 6; ++k) {
    double* dst = k < 3 ? pos : vel;
    if (!dst || !n) continue;
    CUDA_TRY(run_copy(r, t.data(), comps[k], n * 8, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) dst[3 * i + (k % 3)] = t[perm[i]];
  }
  double* scalars[] = {q, w};
  const double* ssrc[] = {r->c.q, r->c.w};
  for (int k = 0; k < 2; ++k) {
    if (!scalars[k] || !n) continue;
    CUDA_TRY(run_copy(r, t.data(), ssrc[k], n * 8, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) scalars[k][i] = t[perm[i]];
  }
  *count = n;
  return APRL_OK;
}

aprl_status aprl_run_set_carriers(aprl_run* r, size_t n, const double* pos, const double* vel,
                                  const double* q, const double* w) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Carriers can only be replaced between steps");
  if (n && (!pos || !vel || !q || !w)) return fail(APRL_ERR_INVALID_ARGUMENT, "null carrier array");
  TRY(reserve_carriers(r, n));
  note_charges(r, q, n);
  std::vector<double> t(n);
  double* comps[] = {r->c.px, r->c.py, r->c.pz, r->c.vx, r->c.vy, r->c.vz};
  for (int k = 0; k < 6; ++k) {
    const double* src = k < 3 ? pos : vel;
    for (size_t i = 0; i < n; ++i) t[i] = src[3 * i + (k % 3)];
    if (n) CUDA_TRY(run_copy(r, comps[k], t.data(), n * 8, cudaMemcpyHostToDevice));
  }
  if (n) CUDA_TRY(run_copy(r, r->c.q, q, n * 8, cudaMemcpyHostToDevice));
  if (n) CUDA_TRY(run_copy(r, r->c.w, w, n * 8, cudaMemcpyHostToDevice));
  std::vector<unsigned long long> keys(n);
  for (size_t i = 0; i < n; ++i) keys[i] = i;
  if (n) CUDA_TRY(run_copy(r, r->c.key, keys.data(), n * 8, cudaMemcpyHostToDevice));
  r->nc = n;
  return APRL_OK;
}

// The seams and whole-step calls refuse to run inside a step opened with
// aprl_run_step_begin: its trials are in flight and step_finish reads them.
static aprl_status no_open_step(const aprl_run* r) {
  if (r->step_open)
    return fail(APRL_ERR_RUNTIME,
                "A step begun with aprl_run_step_begin is open; end it with aprl_run_step_end");
  return APRL_OK;
}

aprl_status aprl_run_advance_magnetic(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(no_open_step(r));
  TRY(do_advance_magnetic(r));
  return check_device(r);
}

aprl_status aprl_run_preview_electric(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(no_open_step(r));
  TRY(do_preview_electric(r));
  return check_device(r);
}

aprl_status aprl_run_coupling_trial(aprl_run* r, double residual[4]) {
  if (!r || !residual) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  TRY(no_open_step(r));
  return do_trial(r, residual);
}

aprl_status aprl_run_commit_electric(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(no_open_step(r));
  TRY(do_commit(r));
  return check_device(r);
}

aprl_status aprl_run_shift(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(no_open_step(r));
  return do_shift(r);
}

}  // extern "C"

namespace {

// A coupled step in two halves, so that several runs can be stepped in lock
// step with one host wait per run and step: step_enqueue queues the begin,
// the magnetic update, the preview and the fixed-point trials issued ahead
// (each followed by a device verdict) and the read-back of their residuals,
// and returns without waiting; step_finish waits for that read-back, applies
// the stopping rule (running further trials one at a time if none of those
// converged), then queues the commit and the shift.
unsigned trials_ahead(const aprl_run* r) {
  // three at FP64, where steps take three; two in the FP32-mixed mode,
  // whose looser tolerances stop at the minimum two
  return std::min<unsigned>(r->fp32 ? 2u : kTrialSlots, r->cfg.max_trials);
}

aprl_status step_enqueue(aprl_run* r) {
  TRY(do_advance_magnetic(r));
  TRY(do_preview_electric(r));
  // The first trials are issued without waiting: after each one a device
  // verdict applies the stopping rule, and the kernels of the trials after
  // a converged one return at once.  One round trip then reads them all.
  const unsigned ahead = trials_ahead(r);
  CUDA_TRY(cudaMemsetAsync(r->d_stop, 0, sizeof(int), r->stream));
  for (unsigned t = 0; t < ahead; ++t) TRY(enqueue_trial(r, (int)t, true));
  CUDA_TRY(cudaMemcpyAsync(r->h_stop, r->d_stop, sizeof(int), cudaMemcpyDeviceToHost,
                           r->stream));
  return APRL_OK;
}

aprl_status step_finish(aprl_run* r) {
  bool converged = false;
  unsigned iterations = 0;
  double force = 0.0, work = 0.0;
  const unsigned ahead = trials_ahead(r);
  TRY(check_device(r));
  tune_harvest(r);
  unsigned t = 0;
  // forceHistory / workHistory of the reference's failure message.
  std::vector<double> history;
  while (!converged && t < ahead) {
    double res[4];
    trial_read(r, (int)t, res);
    iterations = ++t;
    converged = trial_converged(r->cfg, iterations, res, force, work);
    history.push_back(force);
    history.push_back(work);
  }
  if ((converged ? (int)iterations : 0) != *r->h_stop)
    return fail(APRL_ERR_RUNTIME, "Device and host verdicts on the coupling trials differ");
  for (; !converged && t < r->cfg.max_trials; ++t) {
    double res[4];
    TRY(do_trial(r, res));
    iterations = t + 1;
    converged = trial_converged(r->cfg, iterations, res, force, work);
    history.push_back(force);
    history.push_back(work);
  }
  if (!converged) {
    // The reference's message (src/simulation_source_coupling.cpp:54):
    // the last residual, the trial count and every trial's force/work.
    std::string text;
    char item[64];
    std::snprintf(item, sizeof item, "%g", force);
    text = "Conservative source coupling failed at step " + std::to_string(r->step + 1) +
           ": force=" + item;
    std::snprintf(item, sizeof item, "%g", work);
    text += std::string(" work=") + item + " iterations=" + std::to_string(iterations) +
            " history(force/work)=";
    for (size_t h = 0; h + 1 < history.size(); h += 2) {
      std::snprintf(item, sizeof item, " %g/%g", history[h], history[h + 1]);
      text += item;
    }
    g_error = text;
    return APRL_ERR_NOT_CONVERGED;
  }
  r->last_iterations = iterations;
  r->max_iterations = std::max(r->max_iterations, iterations);
  r->total_iterations += iterations;
  r->last_force = force;
  r->last_work = work;
  TRY(do_commit(r));
  return do_shift(r, true);
}

}  // namespace

extern "C" {

aprl_status aprl_run_step(aprl_run* r, uint32_t steps) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(no_open_step(r));
  for (uint32_t n = 0; n < steps; ++n) {
    TRY(step_enqueue(r));
    TRY(step_finish(r));
  }
  return check_device(r);
}

aprl_status aprl_run_step_begin(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(no_open_step(r));
  TRY(step_enqueue(r));
  r->step_open = true;
  return APRL_OK;
}

aprl_status aprl_run_step_end(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  if (!r->step_open)
    return fail(APRL_ERR_RUNTIME, "No step begun with aprl_run_step_begin is open");
  r->step_open = false;
  TRY(step_finish(r));
  return check_device(r);
}

aprl_status aprl_runs_step(aprl_run* const* runs, size_t count, uint32_t steps,
                           aprl_status* statuses) {
  if (count && !runs) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  for (size_t i = 0; i < count; ++i) {
    if (!runs[i]) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
    TRY(no_open_step(runs[i]));
  }
  std::vector<aprl_status> status(count, APRL_OK);
  std::string first_error;
  auto note = [&](size_t i, aprl_status st) {
    if (st != APRL_OK && status[i] == APRL_OK) {
      status[i] = st;
      runs[i]->error = g_error;
      if (first_error.empty()) first_error = g_error;
    }
  };
  for (uint32_t n = 0; n < steps; ++n) {
    // Every run's step is queued before the first wait, so the GPU works
    // through the runs' kernels (on their own streams) while the host waits
    // for the first read-back.
    for (size_t i = 0; i < count; ++i)
      if (status[i] == APRL_OK) note(i, step_enqueue(runs[i]));
    for (size_t i = 0; i < count; ++i)
      if (status[i] == APRL_OK) note(i, step_finish(runs[i]));
  }
  for (size_t i = 0; i < count; ++i)
    if (status[i] == APRL_OK) note(i, check_device(runs[i]));
  aprl_status worst = APRL_OK;
  for (size_t i = 0; i < count; ++i) {
    if (statuses) statuses[i] = status[i];
    if (worst == APRL_OK) worst = status[i];
  }
  if (worst != APRL_OK) g_error = first_error;
  return worst;
}

aprl_status aprl_run_tuning(const aprl_run* r, aprl_tuning* out) {
  if (!r || !out) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  std::memset(out, 0, sizeof *out);
  std::lock_guard<std::mutex> lock(tune_lock());
  for (int k = 0; k < kTuneCount; ++k) {
    const auto it = tune_table().find(tune_key(r, k));
    int choice = 0;
    if (it != tune_table().end()) {
      const TuneEntry& e = it->second;
      for (int c = 0; c < kTuneCandidates; ++c) out->candidate_ms[k][c] = e.best[c];
      if (e.choice >= 0) {
        out->decided |= 1 << k;
        choice = e.choice;
      }
    }
    if (k == kTuneCowan) {
      out->cowan_planes_per_block = (uint32_t)kCowanChunks[choice];
    } else {
      uint32_t* b = k == kTunePreview ? out->preview_block
                                      : (k == kTuneOrbit ? out->orbit_block : out->commit_block);
      b[0] = kGridBlocks[choice].x;
      b[1] = kGridBlocks[choice].y;
    }
  }
  return APRL_OK;
}

aprl_status aprl_run_get_stats(const aprl_run* r, aprl_step_stats* st) {
  if (!r || !st) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  std::memset(st, 0, sizeof *st);
  st->step = r->step;
  st->iterations = r->last_iterations;
  st->max_iterations = r->max_iterations;
  st->total_iterations = r->total_iterations;
  st->force = r->last_force;
  st->work = r->last_work;
  st->particles = r->np;
  st->carriers = r->nc;
  st->exits = r->cumulative.exits;
  st->exit_charge = r->cumulative.exit_charge;
  for (int f = 0; f < 6; ++f) {
    st->cpml_entries[f] = r->cumulative.cpml[f];
    st->cpml_entry_charge[f] = r->cumulative.cpml_charge[f];
    st->carrier_outer[f] = r->cumulative.carrier_outer[f];
    st->carrier_outer_charge[f] = r->cumulative.carrier_outer_charge[f];
  }
  st->cropped_carriers = r->cumulative.cropped;
  st->cropped_charge = r->cumulative.cropped_charge;
  st->window_offset = r->offset;
  st->origin_z = r->origin[2];
  st->time_box = r->time;
  st->device_error = r->h_status ? r->h_status->code : 0;
  st->pending = r->queue.extracted ? r->queue.n - r->queue.cursor : 0;
  st->admitted = r->admitted;
  st->activations = r->cumulative.activations;
  st->held = r->held;
  return APRL_OK;
}

aprl_status aprl_run_reset_iteration_stats(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  r->max_iterations = 0;
  r->total_iterations = 0;
  return APRL_OK;
}

aprl_status aprl_run_get_slot_fields(aprl_run* r, size_t capacity, double* used_e, double* used_b,
                                     double* next_e, double* next_b, size_t* count) {
  if (!r || !count) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *count = r->nslot;
  if (!used_e && !used_b && !next_e && !next_b) return APRL_OK;
  if (capacity < r->nslot) return fail(APRL_ERR_INVALID_ARGUMENT, "Slot buffer too small");
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  const size_t n = r->nslot;
  std::vector<size_t> perm;
  TRY(storage_permutation(r, r->slot_order, n, perm));
  std::vector<double> t(3 * n);
  double* dst[] = {used_e, used_b, next_e, next_b};
  const double* src[] = {r->used_e, r->used_b, r->next_e, r->next_b};
  for (int k = 0; k < 4; ++k) {
    if (!dst[k] || !n) continue;
    CUDA_TRY(run_copy(r, t.data(), src[k], 3 * n * 8, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) dst[k][3 * i + d] = t[3 * perm[i] + d];
  }
  return APRL_OK;
}

// The detector plane's kernel and its copy to `out`, in stream order; `wait`
// returns only once the copy has landed.
static aprl_status sample_plane(aprl_run* r, double plane_lab_z, double* out, size_t count,
                                int* inside, bool wait) {
  if (!r || !out || !inside) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  const aprl_run_config& c = r->cfg;
  if (count != 6 * c.nx * c.ny) return fail(APRL_ERR_INVALID_ARGUMENT, "Detector buffer size mismatch");
  // boxZFromLabZAndBoxT (src/boostframe.cpp:231-235) and ownerRank
  // (src/simulation.cpp:4068-4085).
  const double box_z = c.box_z_origin + (plane_lab_z - c.lab_z_origin) / c.boost_gamma -
                       c.boost_beta * kC * r->time;
  const double coordinate = (box_z - r->origin[2]) / c.dz;
  const double tolerance = 64.0 * DBL_EPSILON * std::max(1.0, std::abs(coordinate));
  if (!(box_z < r->origin[2]) && coordinate > static_cast<double>(c.nz) + tolerance) {
    *inside = 0;
    return APRL_OK;
  }
  *inside = 1;
  auto axis = [](double lattice, size_t size, int* lower, double* fraction) {
    if (lattice <= 0.0) { *lower = 0; *fraction = 0.0; }
    else if (lattice >= static_cast<double>(size - 1)) { *lower = (int)size - 2; *fraction = 1.0; }
    else { *lower = (int)std::floor(lattice); *fraction = lattice - static_cast<double>(*lower); }
  };
  DetectorArgs<double> da{};
  da.frame = make_frame(c);
  da.origin_xy[0] = c.reference_origin[0];
  da.origin_xy[1] = c.reference_origin[1];
  axis(coordinate, c.nz + 1, &da.vertex_lower, &da.vertex_fraction);
  axis(coordinate - 0.5, c.nz, &da.half_lower, &da.half_fraction);
  if (r->detector_cap < count) {
    device_free(r, r->d_detector);
    TRY(device_alloc(r, &r->d_detector, count));
    r->detector_cap = count;
  }
  da.out = r->d_detector;
  const dim3 grid(blocks_for(c.nx, 32), blocks_for(c.ny, 8)), block(32, 8);
  TRY(launch(r, kDetectorPlane, detector_plane_kernel<double>, grid, block,
             retyped<double>(da, make_grid<double>(r))));
  CUDA_TRY(cudaMemcpyAsync(out, r->d_detector, count * 8, cudaMemcpyDeviceToHost, r->stream));
  if (wait) CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

aprl_status aprl_run_sample_field_plane(aprl_run* r, double plane_lab_z, double* out, size_t count,
                                        int* inside) {
  return sample_plane(r, plane_lab_z, out, count, inside, true);
}

aprl_status aprl_run_sample_field_plane_async(aprl_run* r, double plane_lab_z, double* out,
                                              size_t count, int* inside) {
  return sample_plane(r, plane_lab_z, out, count, inside, false);
}

aprl_status aprl_run_enable_energy_ledger(aprl_run* r, int enabled) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  if (r->step != 0 || r->stage != 0)
    return fail(APRL_ERR_RUNTIME,
                "Moving-window energy ledger must be configured before the first step");
  if (enabled) TRY(ensure_ledger(r));
  r->ledger_on = enabled != 0;
  return APRL_OK;
}

aprl_status aprl_run_energy_ledger(aprl_run* r, aprl_energy_ledger* out) {
  if (!r || !out) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Energy ledger read inside a step");
  TRY(ensure_ledger(r));
  TRY(ledger_snapshot(r));
  DLedger h{};
  CUDA_TRY(cudaMemcpyAsync(&h, r->d_ledger, sizeof h, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  TRY(check_device(r));
  const auto v = [](const DD& d) { return d.hi + d.lo; };
  std::memset(out, 0, sizeof *out);
  out->inlet_overwrite_energy = v(h.overwrite);
  out->inserted_energy = v(h.inserted);
  out->cropped_energy = v(h.cropped);
  out->remap_energy = v(h.remap);
  for (int f = 0; f < 6; ++f) out->outward_energy[f] = v(h.outward[f]);
  out->overwrite_events = h.overwrite_events;
  out->flux_steps = h.flux_steps;
  out->remap_steps = h.remap_steps;
  out->field_energy_interior = v(h.snapshot[0]);
  for (int f = 0; f < 6; ++f) out->boundary_power[f] = v(h.snapshot[1 + f]);
  out->particle_kinetic = v(h.snapshot[7]);
  out->particle_total = v(h.snapshot[8]);
  out->represented_electrons = v(h.snapshot[9]);
  out->particles = r->np;
  return APRL_OK;
}

aprl_status aprl_run_gauss_law(aprl_run* r, aprl_gauss_law* out, double* residual,
                               size_t count) {
  if (!r || !out) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (r->stage != 0 && r->stage != 4)
    return fail(APRL_ERR_RUNTIME, "Gauss-law reduction inside a step");
  const aprl_run_config& c = r->cfg;
  const size_t nodes = (size_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  if (residual && count != nodes)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Gauss-law residual size mismatch");
  const size_t partial_bytes = sizeof(DD) * 2 * kGaussBlocks;
  const size_t result_bytes = sizeof(DD) * 2;
  const size_t scratch_bytes = partial_bytes + result_bytes + 3 * sizeof(unsigned long long);
  if (!r->gauss_node) {
    TRY(device_alloc(r, &r->gauss_node, nodes));
    TRY(device_alloc(r, &r->gauss_scratch, scratch_bytes));
  }
  GaussArgs a{};
  a.g = make_grid<double>(r);
  a.x = r->p.x;
  a.y = r->p.y;
  a.z = r->p.z;
  a.q = r->p.q;
  a.np = (long long)r->np;
  a.node = r->gauss_node;
  a.shape = c.shape == APRL_SHAPE_LINEAR_BINOMIAL3 ? 0 : 1;
  a.i0 = (int)c.cpml_cells_x + 1;
  a.i1 = (int)(c.nx - c.cpml_cells_x);
  a.j0 = (int)c.cpml_cells_y + 1;
  a.j1 = (int)(c.ny - c.cpml_cells_y);
  a.k0 = 1;
  a.k1 = (int)c.nz;
  a.volume = ledger_product(ledger_product(c.dx, c.dy), c.dz);
  a.partial = reinterpret_cast<DD*>(r->gauss_scratch);
  a.result = reinterpret_cast<DD*>(r->gauss_scratch + partial_bytes);
  a.max_bits = reinterpret_cast<unsigned long long*>(r->gauss_scratch + partial_bytes + result_bytes);
  a.outside = a.max_bits + 2;
  CUDA_TRY(cudaMemsetAsync(r->gauss_node, 0, nodes * sizeof(double), r->stream));
  CUDA_TRY(cudaMemsetAsync(a.max_bits, 0, 3 * sizeof(unsigned long long), r->stream));
  if (r->np)
    TRY(launch(r, kGaussDeposit, gauss_deposit_kernel, dim3(blocks_for(r->np, 256)), dim3(256), a));
  const int blocks = (int)std::min<size_t>(kGaussBlocks, blocks_for(nodes, kLedgerThreads));
  TRY(launch(r, kGaussResidual, gauss_residual_kernel, dim3(blocks), dim3(kLedgerThreads), a));
  TRY(launch(r, kGaussFinish, gauss_finish_kernel, dim3(1), dim3(kLedgerThreads), a, blocks));
  DD sums[2];
  unsigned long long bits[3];
  CUDA_TRY(cudaMemcpyAsync(sums, a.result, sizeof sums, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaMemcpyAsync(bits, a.max_bits, sizeof bits, cudaMemcpyDeviceToHost, r->stream));
  if (residual)
    CUDA_TRY(cudaMemcpyAsync(residual, r->gauss_node, nodes * sizeof(double),
                             cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  TRY(check_device(r));
  const auto as_double = [](unsigned long long b) {
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
  };
  const uint64_t interior = (uint64_t)std::max(0, a.i1 - a.i0) * std::max(0, a.j1 - a.j0) *
                            std::max(0, a.k1 - a.k0);
  std::memset(out, 0, sizeof *out);
  out->max_residual = as_double(bits[0]);
  out->rms_residual = interior ? std::sqrt((sums[0].hi + sums[0].lo) / (double)interior) : 0.;
  out->max_charge_density = as_double(bits[1]);
  out->total_charge = sums[1].hi + sums[1].lo;
  out->interior_nodes = interior;
  out->outside = bits[2];
  return APRL_OK;
}

namespace {

// Device buffers of one initial-field solve, released on every exit.
struct SfBuffers {
  aprl_run* r;
  double *slab[4] = {}, *rho = nullptr;
  DD *partial = nullptr, *out = nullptr;
  SfState* state = nullptr;
  unsigned long long* max_bits = nullptr;
  double* side = nullptr;  // the open-transverse-wall table
  ~SfBuffers() {
    for (double* p : slab) device_free(r, p);
    device_free(r, rho);
    device_free(r, side);
    device_free(r, partial);
    device_free(r, out);
    device_free(r, state);
    device_free(r, max_bits);
  }
};

aprl_status sf_read(aprl_run* r, const DD* device, DD* host, int count) {
  CUDA_TRY(cudaMemcpyAsync(host, device, count * sizeof(DD), cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

// The free-space potential of the open-wall sources at a batch of targets
// (coordinates relative to the grid origin, z stretched), on the GPU.
struct OpenSources {
  aprl_run* r;
  long long count = 0;
  double* device = nullptr;  // x, y, z, q, each `count` long
  ~OpenSources() { device_free(r, device); }

  aprl_status potential(const std::vector<double>& tx, const std::vector<double>& ty,
                        const std::vector<double>& tz, std::vector<double>& out) {
    const size_t n = tx.size();
    out.assign(n, 0.0);
    if (n == 0) return APRL_OK;
    double* t = nullptr;
    TRY(device_alloc(r, &t, 4 * n));
    aprl_status s = APRL_OK;
    if (run_copy(r, t, tx.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        run_copy(r, t + n, ty.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        run_copy(r, t + 2 * n, tz.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      s = fail(APRL_ERR_CUDA, "cudaMemcpyAsync failed");
    if (s == APRL_OK)
      s = launch(r, kSfOpen, sf_coulomb_kernel, dim3((unsigned)std::min<size_t>(n, 1u << 20)),
                 dim3(256), (const double*)t, (const double*)(t + n),
                 (const double*)(t + 2 * n), (long long)n, (const double*)device,
                 (const double*)(device + count), (const double*)(device + 2 * count),
                 (const double*)(device + 3 * count), count, t + 3 * n);
    if (s == APRL_OK &&
        (run_copy(r, out.data(), t + 3 * n, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
         cudaStreamSynchronize(r->stream) != cudaSuccess))
      s = fail(APRL_ERR_CUDA, "open-wall potential read-back failed");
    device_free(r, t);
    return s;
  }
};

// OpenTransverseTrace's 8-point Lagrange interpolation of a coarse table
// (src/open_transverse_trace.h:214-232), weights formed as the reference does.
struct OpenInterpolation {
  int first = 0;
  double w[8] = {};
  double eval(const double* v, int stride) const {
    double sum = 0.;
    for (int j = 0; j < 8; ++j) sum += w[j] * v[(first + j) * stride];
    return sum;
  }
};

std::vector<OpenInterpolation> open_weights(int count, int stride, int coarse) {
  std::vector<OpenInterpolation> out(count);
  for (int i = 0; i < count; ++i) {
    const double x = double(i) / stride + 3.;
    OpenInterpolation& s = out[i];
    s.first = std::max(0, std::min(coarse - 8, int(x) - 3));
    for (int j = 0; j < 8; ++j) {
      double v = 1.;
      for (int l = 0; l < 8; ++l)
        if (l != j) v *= (x - (s.first + l)) / (j - l);
      s.w[j] = v;
    }
  }
  return out;
}

// The open-transverse-wall table (OpenTransverseTrace::build,
// src/open_transverse_trace.h:65-190) of the charge in `rho` (an unpadded
// (nx+1) x (ny+1) x (nz+1) vertex lattice, charge per volume), with the
// sources of BlockedCowanReference::openSources (src/blocked_cowan_reference.cpp:
// 662-681): every nonzero interior vertex, at (i dx, j dy, k dz gamma) with
// charge rho gamma dx dy dz / (4 pi eps0), gamma = 1/sqrt(1 - translation).
// For each of the eight faces (x = -dx, 0, nx dx, (nx+1) dx, then in y) the
// potential is sampled on a coarse grid, interpolated to the native nodes,
// compared with direct sums at 99 points, and evaluated directly at every
// native node where the interpolation misses by more than 2e-7.  The
// potential sums run on the GPU; the rest is the reference's host logic.
aprl_status open_wall_trace(aprl_run* r, const aprl_run_config& c, const double* rho_device,
                            double translation, const uint64_t guards[3],
                            std::vector<double>& values) {
  const int nx = (int)c.nx, ny = (int)c.ny, nz = (int)c.nz;
  const size_t lx = c.nx + 1, ly = c.ny + 1;
  std::vector<double> rho(lx * ly * (c.nz + 1));
  CUDA_TRY(run_copy(r, rho.data(), rho_device, rho.size() * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  const double gamma = 1. / std::sqrt(1. - translation);
  const double scale = gamma * c.dx * c.dy * c.dz / (4. * std::acos(-1.) * kEpsilon0);
  std::vector<double> sx, sy, sz, sq;
  for (int k = 1; k < nz; ++k)
    for (int j = 1; j < ny; ++j)
      for (int i = 1; i < nx; ++i) {
        const double density = rho[((size_t)k * ly + j) * lx + i];
        if (density == 0.) continue;
        if (i <= (int)guards[0] || i >= nx - (int)guards[0] || j <= (int)guards[1] ||
            j >= ny - (int)guards[1])
          return fail(APRL_ERR_RUNTIME, "Open reference charge overlaps original deposition guard");
        sx.push_back(i * c.dx);
        sy.push_back(j * c.dy);
        sz.push_back(k * c.dz * gamma);
        sq.push_back(density * scale);
      }
  const size_t width = 4 * ((size_t)nx + 3 + ny + 3);
  values.assign(width * (c.nz + 1), 0.);
  if (sq.empty()) return APRL_OK;
  if (!(gamma > 0.) || !std::isfinite(gamma))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid open trace gamma");
  for (size_t s = 0; s < sq.size(); ++s)
    if (!std::isfinite(sx[s]) || !std::isfinite(sy[s]) || !std::isfinite(sz[s]) ||
        !std::isfinite(sq[s]))
      return fail(APRL_ERR_INVALID_ARGUMENT, "Nonfinite open trace source");
  OpenSources src{r};
  src.count = (long long)sq.size();
  TRY(device_alloc(r, &src.device, 4 * sq.size()));
  const std::vector<double>* columns[4] = {&sx, &sy, &sz, &sq};
  for (int a = 0; a < 4; ++a)
    CUDA_TRY(run_copy(r, src.device + a * sq.size(), columns[a]->data(), sq.size() * 8,
                      cudaMemcpyHostToDevice));
  const double hz = c.dz * gamma;
  std::vector<double> tx, ty, tz, coarse, rows, exact, native;
  for (int tile = 0; tile < 8; ++tile) {
    const bool fixed_x = tile < 4;
    const int t = tile % 4;
    const int n = fixed_x ? nx : ny, ns = fixed_x ? ny : nx;
    const double hf = fixed_x ? c.dx : c.dy, hs = fixed_x ? c.dy : c.dx;
    const double fixed = (t < 2 ? t - 1 : n + t - 2) * hf;
    const std::vector<double>& coords = fixed_x ? sx : sy;
    const auto extremes = std::minmax_element(coords.begin(), coords.end());
    const double dist = t < 2 ? *extremes.first - fixed : fixed - *extremes.second;
    if (!(dist > 0.))
      return fail(APRL_ERR_INVALID_ARGUMENT, "Beam support must be inside each open outer face");
    // about 13 samples per closest-source distance, or every native node
    const int ds = std::max(1, static_cast<int>(std::min(0.075 * dist / hs, (ns + 2) / 7.)));
    const int dz = std::max(1, static_cast<int>(std::min(0.075 * dist / hz, nz / 7.)));
    const int cs = (ns + 2 + ds - 1) / ds + 8, cz = (nz + dz - 1) / dz + 8;
    const auto place = [&](double tangent, double z) {
      tx.push_back(fixed_x ? fixed : tangent);
      ty.push_back(fixed_x ? tangent : fixed);
      tz.push_back(z);
    };
    tx.clear(), ty.clear(), tz.clear();
    for (int k = 0; k < cz; ++k)
      for (int p = 0; p < cs; ++p) place(((p - 3) * ds - 1) * hs, (k - 3) * dz * hz);
    TRY(src.potential(tx, ty, tz, coarse));
    const size_t offset = fixed_x ? (size_t)t * (ny + 3) : 4 * ((size_t)ny + 3) + (size_t)t * (nx + 3);
    const auto sp = open_weights(ns + 3, ds, cs), zp = open_weights(nz + 1, dz, cz);
    rows.assign((size_t)(ns + 3) * cz, 0.);
    for (int k = 0; k < cz; ++k)
      for (int p = 0; p < ns + 3; ++p) rows[(size_t)k * (ns + 3) + p] = sp[p].eval(&coarse[(size_t)k * cs], 1);
    for (int k = 1; k < nz; ++k)
      for (int p = 0; p < ns + 3; ++p)
        values[(size_t)k * width + offset + p] = zp[k].eval(&rows[p], ns + 3);
    // direct checks away from the interpolation nodes, near sources too
    const auto zlimits = std::minmax_element(sz.begin(), sz.end());
    const std::vector<double>& other = fixed_x ? sy : sx;
    const auto slimits = std::minmax_element(other.begin(), other.end());
    const auto check_index = [&](int a, int b, int& k, int& p) {
      const double znear = (*zlimits.first + *zlimits.second) * 0.5 / hz;
      const double snear = (*slimits.first + *slimits.second) * 0.5 / hs;
      k = a < 7 ? int(znear + (a - 3) * dist / (3. * hz) + 0.4 * dz) : int((a - 6.4) * nz / 4.2);
      p = b < 5 ? int(snear + (b - 2) * dist / (3. * hs) + 0.35 * ds) + 1
                : int((b - 4.6) * (ns + 2) / 3.6);
      k = std::max(1, std::min(nz - 1, k));
      p = std::max(0, std::min(ns + 2, p));
    };
    tx.clear(), ty.clear(), tz.clear();
    for (int index = 0; index < 99; ++index) {
      int k, p;
      check_index(index / 9, index % 9, k, p);
      place((p - 1) * hs, k * hz);
    }
    TRY(src.potential(tx, ty, tz, exact));
    double tile_error = 0.;
    for (int a = 0; a < 11; ++a)
      for (int b = 0; b < 9; ++b) {
        int k, p;
        check_index(a, b, k, p);
        const double want = exact[a * 9 + b], got = values[(size_t)k * width + offset + p];
        if (!std::isfinite(want) || !std::isfinite(got))
          return fail(APRL_ERR_RUNTIME, "Nonfinite open wall trace");
        if (want != 0.)
          tile_error = std::max(tile_error, std::abs((got - want) / want));
        else if (got != 0.)
          tile_error = std::numeric_limits<double>::infinity();
      }
    if (tile_error > 2.e-7) {
      tx.clear(), ty.clear(), tz.clear();
      for (int k = 1; k < nz; ++k)
        for (int p = 0; p < ns + 3; ++p) place((p - 1) * hs, k * hz);
      TRY(src.potential(tx, ty, tz, native));
      for (int k = 1; k < nz; ++k)
        for (int p = 0; p < ns + 3; ++p)
          values[(size_t)k * width + offset + p] = native[(size_t)(k - 1) * (ns + 3) + p];
    }
  }
  return APRL_OK;
}

}  // namespace

aprl_status aprl_run_initialize_self_field(aprl_run* r, const aprl_self_field_config* cfg,
                                           aprl_self_field_report* rep) {
  if (!r || !cfg || !rep) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "The initial self-field is set between steps");
  std::memset(rep, 0, sizeof *rep);
  const aprl_run_config& c = r->cfg;
  if (!(cfg->relative_tolerance > 0.0) || !(cfg->relative_tolerance < 1.0) ||
      !std::isfinite(cfg->relative_tolerance) || cfg->maximum_iterations == 0)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid initial Gauss-field convergence controls");
  if (!(cfg->maximum_mean_transverse_beta >= 0.0) || !(cfg->maximum_mean_transverse_beta < 1.0) ||
      !std::isfinite(cfg->maximum_mean_transverse_beta))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid initial self-field maximum mean transverse beta");
  if (cfg->model < 0 || cfg->model > 2)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Unknown initial self-field model");
  const bool include = cfg->include_transverse_cpml_particles != 0;
  if (include && (cfg->guard_cells[0] < 2 || cfg->guard_cells[1] < 2))
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "Transverse CPML-source initialization requires at least two physical guard "
                "cells in x and y");
  if (cfg->source_shape != APRL_SOURCE_SHAPE_CIC &&
      cfg->source_shape != APRL_SOURCE_SHAPE_RUN_SHAPE)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Unknown initial self-field source shape");
  const bool shaped = cfg->source_shape == APRL_SOURCE_SHAPE_RUN_SHAPE;
  if (shaped && include)
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "The shaped reference source has no transverse CPML-source padding");
  // The open-transverse-wall reference (BlockedCowanReference::configure,
  // src/blocked_cowan_reference.cpp:314-329): its solve reaches the outer
  // transverse faces, where the wall table holds the potential.
  const bool open = cfg->open_transverse != 0;
  if (open && (cfg->guard_cells[2] != 0 || cfg->guard_cells[0] == 0 || cfg->guard_cells[1] == 0))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Open transverse reference requires only transverse CPML");
  if (open && (cfg->solver != APRL_SELF_FIELD_SOLVER_MODAL ||
               cfg->model != APRL_SELF_FIELD_COWAN_RELATIVISTIC_POISSON || include))
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "The open transverse reference is the Cowan relativistic-Poisson modal solve "
                "without transverse CPML-source padding");
  const bool cowan = cfg->model == APRL_SELF_FIELD_COWAN_RELATIVISTIC_POISSON;
  const bool relativistic = cfg->model == APRL_SELF_FIELD_RELATIVISTIC_POISSON || cowan;
  const int pad = include ? 2 : 0;
  const uint64_t cells[3] = {c.nx, c.ny, c.nz};
  const uint64_t pcells[3] = {c.nx + 2 * pad, c.ny + 2 * pad, c.nz};
  SfLattice L{};
  int physical_lo[3], physical_hi[3];
  for (int a = 0; a < 3; ++a) {
    if (2 * cfg->guard_cells[a] + 2 >= cells[a])
      return fail(APRL_ERR_INVALID_ARGUMENT,
                  "Initial static-field guard leaves fewer than two physical cells");
    physical_lo[a] = (int)cfg->guard_cells[a];
    physical_hi[a] = (int)(cells[a] - cfg->guard_cells[a]);
    L.lo[a] = (include || open) && a < 2 ? 0 : (int)cfg->guard_cells[a];
    L.hi[a] = (int)(pcells[a] - L.lo[a]);
  }
  L.lx = (int)pcells[0] + 1;
  L.ly = (int)pcells[1] + 1;
  L.planes = (int)c.nz + 2;
  L.pad = pad;
  const size_t slab = (size_t)L.lx * L.ly * L.planes;
  const size_t rho_count = (size_t)L.lx * L.ly * (c.nz + 1);

  // clearFields (src/eb_field.cpp:265-269)
  for (int a = 0; a < 3; ++a) {
    CUDA_TRY(cudaMemsetAsync(r->e[r->cur][a], 0, e_count(c, a) * sizeof(double), r->stream));
    CUDA_TRY(cudaMemsetAsync(r->b[a], 0, b_count(c, a) * sizeof(double), r->stream));
  }
  r->ledger_start_ready = false;

  // Tiled CG grid: (i, j) column tiles, z split into chunks for about two
  // blocks per SM's worth of blocks.
  const unsigned gx = blocks_for((size_t)L.lx, kSfTileX), gy = blocks_for((size_t)L.ly, kSfTileY);
  const unsigned gz = (unsigned)std::max<size_t>(
      1, std::min<size_t>(c.nz, (2 * kSelfFieldBlocks + gx * gy - 1) / (gx * gy)));
  const dim3 tile_grid(gx, gy, gz), tile_block(kSfTileX, kSfTileY);
  const int tblocks = (int)(gx * gy * gz);
  SfBuffers buf{r};
  for (int q = 0; q < 4; ++q) TRY(device_alloc(r, &buf.slab[q], slab));
  TRY(device_alloc(r, &buf.rho, rho_count));
  TRY(device_alloc(r, &buf.partial,
                   std::max<size_t>((size_t)kSelfFieldBlocks * kMoments, 2 * (size_t)tblocks)));
  TRY(device_alloc(r, &buf.out, 16));
  TRY(device_alloc(r, &buf.state, 1));
  TRY(device_alloc(r, &buf.max_bits, 1));
  for (int q = 0; q < 4; ++q)
    CUDA_TRY(cudaMemsetAsync(buf.slab[q], 0, slab * sizeof(double), r->stream));
  CUDA_TRY(cudaMemsetAsync(buf.rho, 0, rho_count * sizeof(double), r->stream));

  // meanVelocity and distributionResolution moments (src/eb_initial_field.cpp:629-741)
  SfParticles P{r->p.x, r->p.y, r->p.z, r->p.ux, r->p.uy, r->p.uz, r->p.q, r->p.m,
                (long long)r->np, cfg->hold_transverse_until_activation != 0,
                c.boost_gamma + c.boost_gamma_beta};
  const int pblocks = (int)std::max<size_t>(1, std::min<size_t>(kSelfFieldBlocks,
                                                                 blocks_for(r->np, kSelfFieldThreads)));
  DD moments[kMoments] = {};
  if (r->np) {
    TRY(launch(r, kSfMoments, sf_moments_kernel, dim3(pblocks), dim3(kSelfFieldThreads), P,
               buf.partial));
    TRY(launch(r, kSfFinish, sf_finish_kernel, dim3(1), dim3(kSelfFieldThreads),
               (const DD*)buf.partial, pblocks, kMoments, buf.out));
    TRY(sf_read(r, buf.out, moments, kMoments));
  }
  const long double m0 = sf_long(moments[0]);
  if (!(m0 > 0.0L))
    return fail(APRL_ERR_RUNTIME,
                "Initial relativistic-Poisson field requires positive represented mass");
  const double beta_x = (double)(sf_long(moments[1]) / m0);
  const double beta_y = (double)(sf_long(moments[2]) / m0);
  const double beta_z = (double)(sf_long(moments[3]) / m0);
  const double beta_t = std::hypot(beta_x, beta_y);
  if (!std::isfinite(beta_z) || !std::isfinite(beta_t) || beta_t >= 1.0 || std::fabs(beta_z) >= 1.0)
    return fail(APRL_ERR_RUNTIME, "Initial particle mean velocity is not a finite subluminal vector");
  if (relativistic && beta_t > cfg->maximum_mean_transverse_beta)
    return fail(APRL_ERR_RUNTIME,
                "%s mean beta_box_transverse=%.12g exceeds "
                "initial_self_field.maximum_mean_transverse_beta=%.12g",
                cowan ? "cowan-relativistic-poisson" : "relativistic-poisson", beta_t,
                cfg->maximum_mean_transverse_beta);
  const double applied = relativistic ? beta_z : 0.0;
  const double longitudinal = std::fma(-applied, applied, 1.0);
  if (!cowan && !(longitudinal > 64.0 * DBL_EPSILON))
    return fail(APRL_ERR_RUNTIME,
                "Initial relativistic-Poisson operator is ill-conditioned because the bunch "
                "remains too relativistic in the simulation frame");

  SfArgs A{};
  A.g = make_grid<double>(r);
  A.L = L;
  A.potential = buf.slab[0];
  A.residual = buf.slab[1];
  A.direction = buf.slab[2];
  A.image = buf.slab[3];
  A.rho = buf.rho;
  A.dx = c.dx;
  A.dy = c.dy;
  A.dz = c.dz;
  A.cx = 1.0 / (c.dx * c.dx);
  A.cy = 1.0 / (c.dy * c.dy);
  A.cz = longitudinal / (c.dz * c.dz);
  A.diagonal = 2.0 * (A.cx + A.cy + A.cz);
  A.cowan = cowan ? 1 : 0;
  A.tolerance = cfg->relative_tolerance;
  A.chunk = (int)((c.nz + gz - 1) / gz);
  A.partial = buf.partial;
  A.state = buf.state;
  for (int a = 0; a < 3; ++a) {
    A.alpha[a] = r->coeff[a];
    A.beta[a] = r->coeff[3 + a];
  }
  A.delta[0] = r->coeff[7];  // deltaYZ
  A.delta[1] = r->coeff[8];  // deltaZX
  A.delta[2] = r->coeff[6];  // deltaXY
  if (cowan) {
    // CowanPoissonOperator (src/eb_initial_field.cpp:246-316)
    const double velocity = applied * kC;
    A.translation = velocity * velocity * kEpsilon0 * kMu0;
    const double spacing[3] = {c.dx, c.dy, c.dz};
    double st[3][3][3] = {};
    for (int axis = 0; axis < 3; ++axis) {
      const int ta = (axis + 1) % 3, tb = (axis + 2) % 3;
      const double delta = A.delta[axis];
      double minimum = INFINITY;
      for (int a = -1; a <= 1; a += 2)
        for (int b = -1; b <= 1; b += 2)
          minimum = std::min(minimum, A.alpha[axis] + 2.0 * A.beta[ta] * a +
                                          2.0 * A.beta[tb] * b + 4.0 * delta * a * b);
      if (axis == 2) minimum -= A.translation;
      if (!(minimum > 64.0 * DBL_EPSILON))
        return fail(APRL_ERR_RUNTIME,
                    "Initial Cowan-Poisson operator fails the sufficient positive-definiteness "
                    "bound on axis %d: minimum smoothing symbol%s=%.12g; choose boost_gamma "
                    "closer to the bunch mean gamma or a grid aspect ratio with positive Cowan "
                    "symbols",
                    axis, axis == 2 ? " minus v^2*epsilon0*mu0" : "", minimum);
      const double inverse2 = 1.0 / (spacing[axis] * spacing[axis]);
      for (int a = -1; a <= 1; ++a)
        for (int b = -1; b <= 1; ++b) {
          const double weight =
              a == 0 ? (b == 0 ? A.alpha[axis] : A.beta[tb]) : (b == 0 ? A.beta[ta] : delta);
          int pt[3] = {1, 1, 1};
          pt[ta] += a;
          pt[tb] += b;
          st[pt[2]][pt[1]][pt[0]] += 2.0 * weight * inverse2;
          --pt[axis];
          st[pt[2]][pt[1]][pt[0]] -= weight * inverse2;
          pt[axis] += 2;
          st[pt[2]][pt[1]][pt[0]] -= weight * inverse2;
        }
    }
    const double tz = A.translation / (c.dz * c.dz);
    st[1][1][1] -= 2.0 * tz;
    st[0][1][1] += tz;
    st[2][1][1] += tz;
    std::memcpy(A.stencil, st, sizeof st);
  }
  rep->mean_beta_z = beta_z;
  rep->mean_beta_transverse = beta_t;
  rep->transverse_poisson_padding_cells = pad;
  for (int a = 0; a < 3; ++a) rep->static_field_guard_cells[a] = L.lo[a];
  {
    // distributionResolution (src/eb_initial_field.cpp:693-741)
    const double spacing[3] = {c.dx, c.dy, c.dz};
    const double origin[3] = {r->origin[0] - (double)pad * c.dx, r->origin[1] - (double)pad * c.dy,
                              r->origin[2]};
    for (int a = 0; a < 3; ++a) {
      const long double mean = sf_long(moments[4 + a]) / m0;
      const long double variance = std::max(0.0L, sf_long(moments[7 + a]) / m0 - mean * mean);
      const double rms = (double)std::sqrt(variance);
      rep->rms_position_cells[a] = rms / spacing[a];
      if (rms > 0.0) {
        const double lower = origin[a] + (double)L.lo[a] * spacing[a];
        const double upper = origin[a] + (double)L.hi[a] * spacing[a];
        rep->centre_padding_rms[a] = std::min((double)mean - lower, upper - (double)mean) / rms;
      }
    }
  }
  rep->temporary_bytes = 4 * slab * sizeof(double) +
                         (size_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1) * sizeof(double) +
                         (pad ? rho_count * sizeof(double) : 0);

  // The CIC charge (or the shaped reference source) and the Poisson source
  // (src/eb_initial_field.cpp:979-1027)
  const DGrid g = make_grid<double>(r);
  const int binomial = c.shape == APRL_SHAPE_LINEAR_BINOMIAL3;
  if (shaped)
    TRY(launch(r, kSfDeposit, sf_shaped_deposit_kernel, dim3(blocks_for(r->np, 256)), dim3(256),
               P, g, buf.rho, L.lx, L.ly, L, binomial, r->d_status));
  else
    TRY(launch(r, kSfDeposit, sf_deposit_kernel, dim3(blocks_for(r->np, 256)), dim3(256), P, g,
               buf.rho, L.lx, L.ly, pad, r->d_status));
  const DD vertex_volume = ledger_product(ledger_product(c.dx, c.dy), c.dz);
  TRY(launch(r, kSfSource, sf_source_kernel, tile_grid, tile_block, A, vertex_volume));
  TRY(launch(r, kSfFinish, sf_finish_kernel, dim3(1), dim3(kSelfFieldThreads),
             (const DD*)buf.partial, tblocks, 2, buf.out));
  DD sums[2];
  TRY(sf_read(r, buf.out, sums, 2));
  TRY(check_device(r));
  const long double total = sf_long(moments[10]);
  rep->total_charge = (double)total;
  const long double interior = sf_long(sums[0]);
  if (std::fabs((interior - total) / total) > 1.0e-12L)
    return fail(APRL_ERR_RUNTIME,
                "Initial CIC charge cloud touches the static zero-potential boundary; move every "
                "particle at least one complete cell inside the CPML entrance or enlarge the "
                "physical mesh padding");
  if (!(sums[1].hi > 0.0) || !std::isfinite(sums[1].hi))
    return fail(APRL_ERR_RUNTIME, "Initial particle charge produced an invalid Poisson source norm");
  SfOpenSide side{nullptr, (int)c.nx, (int)c.ny, (int)c.nz,
                  4 * ((long long)c.nx + 3 + (long long)c.ny + 3)};
  if (open) {
    std::vector<double> values;
    TRY(open_wall_trace(r, c, buf.rho, A.translation, cfg->guard_cells, values));
    TRY(device_alloc(r, &buf.side, values.size()));
    CUDA_TRY(run_copy(r, buf.side, values.data(), values.size() * 8, cudaMemcpyHostToDevice));
    side.values = buf.side;
  }

  SfState state{};
  if (cfg->solver == APRL_SELF_FIELD_SOLVER_MODAL) {
    // The transverse-mode direct solve on the same box (sf_modal_*): the
    // source b = rho/eps0 (in the residual slab) into a compact interior
    // array, sine transforms along x and y, one tridiagonal solve along z per
    // mode, the inverse transforms, and the potential back into the lattice.
    const int ix = L.hi[0] - L.lo[0] - 1, iy = L.hi[1] - L.lo[1] - 1, iz = L.hi[2] - L.lo[2] - 1;
    if (ix < 1 || iy < 1 || iz < 1)
      return fail(APRL_ERR_INVALID_ARGUMENT, "Initial field solve domain has no interior");
    const size_t count = (size_t)ix * iy * iz;
    std::vector<double> table_x((size_t)ix * ix), table_y((size_t)iy * iy), cos_x(ix), cos_y(iy);
    for (int m = 0; m < ix; ++m) {
      cos_x[m] = std::cos(kPi * (m + 1) / (ix + 1));
      for (int t = 0; t < ix; ++t)
        table_x[(size_t)m * ix + t] = std::sin(kPi * (double)((long long)(m + 1) * (t + 1) % (2 * (ix + 1))) / (ix + 1));
    }
    for (int m = 0; m < iy; ++m) {
      cos_y[m] = std::cos(kPi * (m + 1) / (iy + 1));
      for (int t = 0; t < iy; ++t)
        table_y[(size_t)m * iy + t] = std::sin(kPi * (double)((long long)(m + 1) * (t + 1) % (2 * (iy + 1))) / (iy + 1));
    }
    double* tables = nullptr;
    const size_t table_words = table_x.size() + table_y.size() + ix + iy;
    TRY(device_alloc(r, &tables, table_words));
    double* tx = tables;
    double* ty = tx + table_x.size();
    double* cx = ty + table_y.size();
    double* cy = cx + ix;
    CUDA_TRY(run_copy(r, tx, table_x.data(), table_x.size() * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(run_copy(r, ty, table_y.data(), table_y.size() * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(run_copy(r, cx, cos_x.data(), ix * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(run_copy(r, cy, cos_y.data(), iy * 8, cudaMemcpyHostToDevice));
    double* w0 = A.direction;  // compact arrays: the two free CG slabs and
    double* w1 = A.image;      // the residual slab (after the gather)
    double* work = A.residual;
    const unsigned blocks = blocks_for(count, 256);
    TRY(launch(r, kSfModal, sf_modal_gather_kernel, dim3(blocks), dim3(256), A, w0, ix, iy, iz));
    if (open)
      TRY(launch(r, kSfOpen, sf_open_lift_kernel, dim3(blocks), dim3(256), A, side, w0, ix, iy,
                 iz));
    TRY(launch(r, kSfModal, sf_modal_transform_kernel, dim3(blocks), dim3(256),
               (const double*)w0, w1, (const double*)tx, 0, ix, iy, iz, 1.0));
    TRY(launch(r, kSfModal, sf_modal_transform_kernel, dim3(blocks), dim3(256),
               (const double*)w1, w0, (const double*)ty, 1, ix, iy, iz, 1.0));
    TRY(launch(r, kSfModal, sf_modal_z_kernel, dim3(blocks_for(ix, 32), blocks_for(iy, 4)),
               dim3(32, 4), A, w0, work, (const double*)cx, (const double*)cy, ix, iy, iz));
    TRY(launch(r, kSfModal, sf_modal_transform_kernel, dim3(blocks), dim3(256),
               (const double*)w0, w1, (const double*)ty, 1, ix, iy, iz, 2.0 / (iy + 1)));
    TRY(launch(r, kSfModal, sf_modal_transform_kernel, dim3(blocks), dim3(256),
               (const double*)w1, w0, (const double*)tx, 0, ix, iy, iz, 2.0 / (ix + 1)));
    TRY(launch(r, kSfModal, sf_modal_scatter_kernel, dim3(blocks), dim3(256), A,
               (const double*)w0, ix, iy, iz));
    if (open)
      TRY(launch(r, kSfOpen, sf_open_wall_fill_kernel, dim3(64), dim3(256), A, side));
    device_free(r, tables);
    state.done = 1;
    rep->iterations = 0;
  } else {
  // Conjugate gradients, in batches of iterations between host reads.
  state.rr = sums[1];
  state.source = sums[1];
  CUDA_TRY(cudaMemcpyAsync(buf.state, &state, sizeof state, cudaMemcpyHostToDevice, r->stream));
  uint64_t issued = 0;
  while (issued < cfg->maximum_iterations) {
    const uint64_t batch = std::min<uint64_t>(32, cfg->maximum_iterations - issued);
    for (uint64_t it = 0; it < batch; ++it) {
      // alpha and beta are formed by the last block of apply and of update.
      TRY(launch(r, kSfApply, sf_apply_kernel, tile_grid, tile_block, A));
      TRY(launch(r, kSfUpdate, sf_update_kernel, tile_grid, tile_block, A));
      TRY(launch(r, kSfDirection, sf_direction_kernel, tile_grid, tile_block, A));
    }
    issued += batch;
    CUDA_TRY(cudaMemcpyAsync(&state, buf.state, sizeof state, cudaMemcpyDeviceToHost, r->stream));
    CUDA_TRY(cudaStreamSynchronize(r->stream));
    if (state.done) break;
  }
  rep->iterations = state.iterations;
  }
  if (state.done == 2) return fail(APRL_ERR_RUNTIME, "Initial Gauss-field CG lost positive definiteness");
  if (state.done == 3)
    return fail(APRL_ERR_RUNTIME, "Initial Gauss-field CG produced a non-finite residual");
  if (state.done != 1 || (cfg->solver != APRL_SELF_FIELD_SOLVER_MODAL &&
                          state.relative > cfg->relative_tolerance))
    return fail(APRL_ERR_RUNTIME,
                "Initial Gauss-field solve did not converge; increase "
                "initial_self_field.maximum_iterations, relax its relative_tolerance, or reduce "
                "the grid aspect ratio");

  // E and B from the potential (src/eb_initial_field.cpp:427-553)
  const int fblocks = (int)std::min<size_t>(kSelfFieldBlocks * 2, blocks_for(slab, 256));
  if (cowan) {
    for (int axis = 0; axis < 3; ++axis) {
      CUDA_TRY(cudaMemsetAsync(A.image, 0, slab * sizeof(double), r->stream));
      TRY(launch(r, kSfSmooth, sf_smooth_kernel, tile_grid, tile_block, A, axis));
      if (open)
        TRY(launch(r, kSfOpen, sf_open_wall_smooth_kernel, dim3(64), dim3(256), A, side, axis));
      TRY(launch(r, kSfElectric, sf_electric_kernel, dim3(fblocks), dim3(256), A, axis, 1.0, 1));
    }
  } else {
    TRY(launch(r, kSfElectric, sf_electric_kernel, dim3(fblocks), dim3(256), A, 0, 1.0, 0));
    TRY(launch(r, kSfElectric, sf_electric_kernel, dim3(fblocks), dim3(256), A, 1, 1.0, 0));
    TRY(launch(r, kSfElectric, sf_electric_kernel, dim3(fblocks), dim3(256), A, 2, longitudinal,
               0));
  }
  const double scale = cowan ? applied * kC * kEpsilon0 * kMu0 : applied / kC;
  const double upper_w = 0.5 + 0.5 * applied * kC * c.dt / c.dz;
  const double lower_w = 1.0 - upper_w;
  if (upper_w < 0.0 || upper_w > 1.0)
    return fail(APRL_ERR_RUNTIME, "Initial B half-step shift exceeds one longitudinal cell");
  TRY(launch(r, kSfMagnetic, sf_magnetic_kernel, dim3(fblocks), dim3(256), A, scale, lower_w,
             upper_w));
  if (include)
    for (int comp = 0; comp < 6; ++comp)
      TRY(launch(r, kSfClear, sf_clear_outside_kernel, dim3(fblocks), dim3(256), A, comp,
                 (int)cfg->guard_cells[0], (int)cfg->guard_cells[1], (int)cfg->guard_cells[2]));

  // validateGauss on the unpadded charge the potential was solved for
  // (src/eb_initial_field.cpp:1083-1091): CIC, or the shaped reference source
  // (whose lattice has no padding)
  const int vx = (int)c.nx + 1, vy = (int)c.ny + 1;
  CUDA_TRY(cudaMemsetAsync(buf.rho, 0, (size_t)vx * vy * (c.nz + 1) * sizeof(double), r->stream));
  CUDA_TRY(cudaMemsetAsync(buf.max_bits, 0, sizeof(unsigned long long), r->stream));
  if (shaped)
    TRY(launch(r, kSfDeposit, sf_shaped_deposit_kernel, dim3(blocks_for(r->np, 256)), dim3(256),
               P, g, buf.rho, vx, vy, L, binomial, r->d_status));
  else
    TRY(launch(r, kSfDeposit, sf_deposit_kernel, dim3(blocks_for(r->np, 256)), dim3(256), P, g,
               buf.rho, vx, vy, 0, r->d_status));
  const int gblocks = (int)std::min<size_t>(kSelfFieldBlocks,
                                            blocks_for((size_t)vx * vy * c.nz, kSelfFieldThreads));
  TRY(launch(r, kSfGauss, sf_gauss_kernel, dim3(gblocks), dim3(kSelfFieldThreads), A,
             (const double*)buf.rho, physical_lo[0], physical_hi[0], physical_lo[1],
             physical_hi[1], physical_lo[2], physical_hi[2], buf.max_bits));
  TRY(launch(r, kSfFinish, sf_finish_kernel, dim3(1), dim3(kSelfFieldThreads),
             (const DD*)buf.partial, gblocks, 2, buf.out));
  TRY(sf_read(r, buf.out, sums, 2));
  TRY(check_device(r));
  unsigned long long worst_bits = 0;
  CUDA_TRY(run_copy(r, &worst_bits, buf.max_bits, sizeof worst_bits, cudaMemcpyDeviceToHost));
  double worst;
  std::memcpy(&worst, &worst_bits, sizeof worst);
  const long double res2 = sf_long(sums[0]), src2 = sf_long(sums[1]);
  rep->relative_residual = src2 > 0.0L ? (double)std::sqrt(res2 / src2) : 0.0;
  rep->maximum_gauss_residual = worst;
  if (rep->relative_residual > 4.0 * cfg->relative_tolerance)
    return fail(APRL_ERR_RUNTIME, "Initial E field failed the post-solve discrete Gauss check");

  // initialFieldEnergy (src/eb_initial_field.cpp:665-691)
  const DD electric_factor = ledger_product(vertex_volume, 0.5 * kEpsilon0);
  const DD magnetic_factor = dd_div(ledger_product(vertex_volume, 0.5), kMu0);
  A.stencil[0] = magnetic_factor.hi;
  A.stencil[1] = magnetic_factor.lo;
  const int eblocks = (int)std::min<size_t>(kSelfFieldBlocks,
                                            blocks_for((size_t)c.nx * c.ny * c.nz, kSelfFieldThreads));
  TRY(launch(r, kSfEnergy, sf_energy_kernel, dim3(eblocks), dim3(kSelfFieldThreads), A,
             electric_factor));
  TRY(launch(r, kSfFinish, sf_finish_kernel, dim3(1), dim3(kSelfFieldThreads),
             (const DD*)buf.partial, eblocks, 2, buf.out));
  TRY(sf_read(r, buf.out, sums, 2));
  rep->initial_electric_energy = (double)sf_long(sums[0]);
  rep->initial_magnetic_energy = (double)sf_long(sums[1]);
  return APRL_OK;
}

aprl_status aprl_run_get_reference(aprl_run* r, unsigned a, double* host, size_t count) {
  if (!r || a >= 6 || !host) return fail(APRL_ERR_OUT_OF_RANGE, "Moving-window component");
  size_t s[3];
  comp_shape(r->cfg, a, s);
  const size_t n = s[0] * s[1] * (r->cfg.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0));
  if (count != n) return fail(APRL_ERR_INVALID_ARGUMENT, "Reference component size mismatch");
  if (!r->ref_set[a]) return fail(APRL_ERR_RUNTIME, "Moving-window reference component is not set");
  CUDA_TRY(cudaMemcpyAsync(host, r->ref[a], n * 8, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

aprl_status aprl_run_prepare_reference(aprl_run* r, size_t n, const double* x, const double* y,
                                       const double* z, const double* ux, const double* uy,
                                       const double* uz, const double* q, const double* m,
                                       const aprl_self_field_config* config,
                                       aprl_self_field_report* report) {
  if (!r || !config || !report) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  if (r->stage != 0 || r->step != 0)
    return fail(APRL_ERR_RUNTIME, "The inlet reference is prepared before the first step");
  // The reference grid as a run of its own: reference_nz cells from the
  // reference origin.
  aprl_run_config tc = r->cfg;
  tc.nz = r->cfg.reference_nz;
  tc.initial_offset = 0;
  aprl_run* t = nullptr;
  TRY(aprl_run_create(&tc, r->stream, &t));
  std::vector<uint64_t> ids(n);
  for (size_t i = 0; i < n; ++i) ids[i] = i;
  aprl_status s = aprl_run_set_particles(t, n, x, y, z, ux, uy, uz, q, m, ids.data(), 1);
  if (s == APRL_OK) s = aprl_run_initialize_self_field(t, config, report);
  for (int a = 0; s == APRL_OK && a < 6; ++a) {
    const size_t count = a < 3 ? e_count(tc, a) : b_count(tc, a - 3);
    const double* from = a < 3 ? t->e[t->cur][a] : t->b[a - 3];
    if (cudaStreamSynchronize(r->stream) != cudaSuccess) {
      s = fail(APRL_ERR_CUDA, "cudaStreamSynchronize failed");
      break;
    }
    device_free(r, r->ref[a]);
    r->ref[a] = nullptr;
    s = device_alloc(r, &r->ref[a], count);
    if (s != APRL_OK) break;
    // A fresh run's rings start at base 0: its fields are in native order.
    const cudaError_t e =
        cudaMemcpyAsync(r->ref[a], from, count * 8, cudaMemcpyDeviceToDevice, r->stream);
    if (e != cudaSuccess) {
      s = fail(APRL_ERR_CUDA, "cudaMemcpyAsync: %s", cudaGetErrorString(e));
      break;
    }
    r->ref_set[a] = true;
  }
  r->surface_ready = false;
  if (s == APRL_OK && cudaStreamSynchronize(r->stream) != cudaSuccess)
    s = fail(APRL_ERR_CUDA, "cudaStreamSynchronize failed");
  aprl_run_destroy(t);
  return s;
}

aprl_status aprl_run_synchronize(aprl_run* r) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

aprl_status aprl_run_profile_enable(aprl_run* r, int enabled) {
  if (!r) return fail(APRL_ERR_INVALID_ARGUMENT, "null run");
  TRY(drain_timings(r));
  r->profile = enabled != 0;
  for (unsigned k = 0; k < kKernelCount; ++k) {
    r->kernel_ms[k] = 0.0;
    r->kernel_launches[k] = 0;
  }
  return APRL_OK;
}

aprl_status aprl_run_profile_read(aprl_run* r, double* ms, uint64_t* launches, unsigned capacity,
                                  unsigned* kernels) {
  if (!r || !kernels) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  TRY(drain_timings(r));
  *kernels = kKernelCount;
  for (unsigned k = 0; k < kKernelCount && k < capacity; ++k) {
    if (ms) ms[k] = r->kernel_ms[k];
    if (launches) launches[k] = r->kernel_launches[k];
  }
  return APRL_OK;
}

aprl_status aprl_run_launch_count(const aprl_run* r, uint64_t* launches) {
  if (!r || !launches) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *launches = r->launches;
  return APRL_OK;
}

}  // extern "C"

// ===========================================================================
// Detector plane without device allocation.
//
// The plane is staged in this fixed array instead of the run's lazily
// allocated detector buffer.  In host code `g_plane_scratch` names a host-side
// stand-in, not device memory, so the kernel receives the address that
// cudaGetSymbolAddress reports for the current device.
static __device__ __align__(256) double g_plane_scratch[APRL_NOALLOC_PLANE_MAX_VALUES];

namespace {

constexpr int kPlaneScratchDevices = 64;
std::atomic<double*> g_plane_scratch_address[kPlaneScratchDevices];

// Device address of g_plane_scratch on the current device; looked up once
// per device, with that device current.
aprl_status plane_scratch(double** out) {
  int device = 0;
  CUDA_TRY(cudaGetDevice(&device));
  if (device < 0 || device >= kPlaneScratchDevices)
    return fail(APRL_ERR_UNSUPPORTED, "Device ordinal %d is beyond the %d devices of the fixed detector scratch",
                device, kPlaneScratchDevices);
  double* ptr = g_plane_scratch_address[device].load(std::memory_order_acquire);
  if (!ptr) {
    CUDA_TRY(cudaGetSymbolAddress((void**)&ptr, g_plane_scratch));
    g_plane_scratch_address[device].store(ptr, std::memory_order_release);
  }
  *out = ptr;
  return APRL_OK;
}

}  // namespace

extern "C" {

aprl_status aprl_run_sample_field_plane_noalloc(aprl_run* r, double plane_lab_z, double* out,
                                                size_t count, int* inside) {
  if (!r || !out || !inside) return fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  const aprl_run_config& c = r->cfg;
  if (count != 6 * c.nx * c.ny) return fail(APRL_ERR_INVALID_ARGUMENT, "Detector buffer size mismatch");
  if (count > APRL_NOALLOC_PLANE_MAX_VALUES)
    return fail(APRL_ERR_OUT_OF_RANGE,
                "Detector plane of %zu values exceeds the fixed %u-value scratch of "
                "aprl_run_sample_field_plane_noalloc; use aprl_run_sample_field_plane",
                count, APRL_NOALLOC_PLANE_MAX_VALUES);
  double* scratch = nullptr;
  TRY(plane_scratch(&scratch));
  // boxZFromLabZAndBoxT (src/boostframe.cpp:231-235) and the window test,
  // as in aprl_run_sample_field_plane.
  const double box_z = c.box_z_origin + (plane_lab_z - c.lab_z_origin) / c.boost_gamma -
                       c.boost_beta * kC * r->time;
  const double coordinate = (box_z - r->origin[2]) / c.dz;
  const double tolerance = 64.0 * DBL_EPSILON * std::max(1.0, std::abs(coordinate));
  if (!(box_z < r->origin[2]) && coordinate > static_cast<double>(c.nz) + tolerance) {
    *inside = 0;
    return APRL_OK;
  }
  *inside = 1;
  auto axis = [](double lattice, size_t size, int* lower, double* fraction) {
    if (lattice <= 0.0) { *lower = 0; *fraction = 0.0; }
    else if (lattice >= static_cast<double>(size - 1)) { *lower = (int)size - 2; *fraction = 1.0; }
    else { *lower = (int)std::floor(lattice); *fraction = lattice - static_cast<double>(*lower); }
  };
  DetectorArgs<double> da{};
  da.frame = make_frame(c);
  da.origin_xy[0] = c.reference_origin[0];
  da.origin_xy[1] = c.reference_origin[1];
  axis(coordinate, c.nz + 1, &da.vertex_lower, &da.vertex_fraction);
  axis(coordinate - 0.5, c.nz, &da.half_lower, &da.half_fraction);
  da.out = scratch;
  // The run's launch helper: with profiling on it times the kernel with CUDA
  // events (host-side objects, not device memory), like every other launch.
  const dim3 grid(blocks_for(c.nx, 32), blocks_for(c.ny, 8)), block(32, 8);
  TRY(launch(r, kDetectorPlane, detector_plane_kernel<double>, grid, block,
             retyped<double>(da, make_grid<double>(r))));
  CUDA_TRY(cudaMemcpyAsync(out, scratch, count * 8, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return APRL_OK;
}

}  // extern "C"
