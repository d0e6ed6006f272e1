/*
 * aprl_gpu.h -- C ABI of the B200 (sm_100a) implementation of APRL's
 * per-timestep particle-in-cell loop: Cowan-z E/B update, CFS-CPML, the
 * conservative-source (Lapenta-Markidis) gather/push with its implicit
 * fixed-point trials, wide-shape charge-conserving deposition, CPML current
 * carriers and the moving-window shift.
 *
 * The reference has no FFI layer: its seams are C++ classes called directly
 * by Simulation.  Each entry point below names the reference interface it
 * replaces (paths are relative to the APRL source tree).  Plain pointers and
 * sizes only; no C++ or torch types cross this boundary.
 *
 * Conventions
 *   - Every entry point returns an aprl_status.  On failure a message is kept
 *     in thread-local storage and returned by aprl_last_error(); the reference
 *     throws std::invalid_argument / std::out_of_range / std::runtime_error in
 *     the same situations (APRL_ERR_INVALID_ARGUMENT / _OUT_OF_RANGE /
 *     _RUNTIME).  Device-side failures never trap: kernels raise a flag that
 *     the host reads after the step.
 *   - Field arrays use the reference's Yee layout: component extents
 *     Ex(nx,ny+1,nz+1) Ey(nx+1,ny,nz+1) Ez(nx+1,ny+1,nz) Bx(nx+1,ny,nz)
 *     By(nx,ny+1,nz) Bz(nx,ny,nz+1), J collocated with E, x fastest:
 *     index (k*ny_c + j)*nx_c + i (src/eb_field.h:134-141, eb_field.cpp:217-225).
 *   - SI units throughout, as in the reference E/B core (src/eb_field.h:16-23).
 *   - A handle is not reentrant: one host thread drives one aprl_run.
 */
#ifndef APRL_GPU_H
#define APRL_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define APRL_GPU_ABI_VERSION 3

typedef enum {
  APRL_OK = 0,
  APRL_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  APRL_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range (particle/stencil outside the grid) */
  APRL_ERR_RUNTIME = 3,          /* std::runtime_error (non-finite, crossing budget) */
  APRL_ERR_NOT_CONVERGED = 4,    /* coupling fixed point exhausted its trials */
  APRL_ERR_CUDA = 5,             /* CUDA runtime failure */
  APRL_ERR_UNSUPPORTED = 6       /* valid in the reference, not built here */
} aprl_status;

/* mesh.longitudinal_shape (src/config.cpp:1097-1112).  linear-binomial3
 * implies transverseXBinomial3 (the F3 x-z product) in the production code. */
typedef enum {
  APRL_SHAPE_LINEAR_BINOMIAL3 = 0,
  APRL_SHAPE_QUINTIC_COMPENSATED = 1
} aprl_shape;

/* Arithmetic of a run.  FP64 is the drop-in: every stage in binary64 with
 * the reference's operation order.  FP32_MIXED runs the field gathers in
 * binary32: the shape weights (from binary64 cell-relative offsets), the
 * orbit-averaged E and the B the gathers read (binary32 copies made once per
 * trial / step) and their accumulation.  E, B, J, the CPML histories and
 * every field update, the deposit, particle positions and momenta, the
 * Lapenta-Markidis push, the boundary events, the window bookkeeping and the
 * residual reductions stay binary64, so the rounding of the mode perturbs
 * particle forces only, never the fields' own history.  The reference is
 * binary64 only; this mode has no counterpart there. */
typedef enum {
  APRL_PRECISION_FP64 = 0,
  APRL_PRECISION_FP32_MIXED = 1
} aprl_precision;

/* SIMagnetType (src/eb_sources.h:97-102). */
typedef enum {
  APRL_MAGNET_PLANAR_UNDULATOR = 0,
  APRL_MAGNET_UNIFORM_DIPOLE = 1,
  APRL_MAGNET_QUADRUPOLE = 2
} aprl_magnet_type;

/* SIMagneticElement (src/eb_sources.h:103-140).  The derived constants
 * (wave number, fringe extent, cos/sin of the polarisation angle) are filled
 * by aprl_magnet_prepare, the counterpart of SIMagneticElement::prepare. */
typedef struct {
  int32_t type;                  /* aprl_magnet_type */
  int32_t gaussian_fringe;       /* planar undulator only */
  double center[3];              /* m; center[2] is the entrance */
  double length;                 /* m */
  double period;                 /* m, planar undulator */
  double peak_field;             /* T */
  double polarization_angle;     /* rad from +x */
  double fringe_relative_cutoff; /* raw Gaussian at the compact edge */
  double quadrupole_gradient;    /* T/m */
  /* derived by aprl_magnet_prepare */
  double wave_number;
  double fringe_extent;
  double cos_angle;
  double sin_angle;
} aprl_magnet;

#define APRL_MAX_MAGNETS 4

/* Everything a single-GPU run needs.  Mirrors EBGridGeometry (solver fixed to
 * CowanZ), EBCPMLParameters (z CPML must be 0 under the moving window,
 * src/config.cpp:2064-2071), BoostFrameTransform, the moving-window state of
 * Simulation and the coupling tolerances of solveConservativeSourceStep. */
typedef struct {
  /* EBGridGeometry (src/eb_field.h:54-70); requires c*dt = dz */
  uint64_t nx, ny, nz;
  double dx, dy, dz, dt;
  /* EBCPMLParameters (src/eb_cpml.h:12-24) for x and y */
  uint64_t cpml_cells_x, cpml_cells_y;
  double cpml_polynomial_order;   /* 3 */
  double cpml_target_reflection;  /* 1e-8 */
  double cpml_kappa_max;          /* 8 */
  double cpml_alpha_fraction;     /* 0 */
  /* particle coupling */
  int32_t shape;                  /* aprl_shape */
  uint32_t substeps;              /* particleSubsteps_ (src/simulation.cpp:2623-2685) */
  uint32_t max_trials;            /* 64 (src/simulation_source_coupling.cpp:40) */
  uint32_t precision;             /* aprl_precision */
  double force_tolerance;         /* 1e-13 (src/simulation_source_coupling.cpp:50) */
  double work_tolerance;          /* 1e-8 */
  /* BoostFrameTransform (src/boostframe.h:8-17) */
  double boost_gamma, boost_beta, boost_gamma_beta;
  double lab_time_origin, lab_z_origin, box_z_origin;
  /* moving window (src/simulation_moving_window.cpp:53-117, 275-379) */
  double reference_origin[3];     /* box-frame origin of the prepared reference */
  int64_t initial_offset;         /* window start cell in reference native z */
  uint64_t reference_nz;          /* prepared reference cells in z */
  double translation_beta;        /* inlet lerp speed, in cells per step */
  double exit_lab_z;              /* fixed-lab particle exit plane */
  /* held lab-plane injection (src/config.cpp:2072-2076): held particles move
   * along z at c*frozenBetaZ until they cross this fixed lab plane */
  double activation_plane_lab_z;
  uint64_t maximum_step;          /* pending-queue horizon (PendingWindowGeometry) */
  /* prescribed lab magnets (SIFieldSourceSet::addPrescribedLabMagnet) */
  uint32_t n_magnets;
  /* mesh.moving_window.inlet_charge_match (src/config.cpp:711, 1152-1153;
   * off by default): complete Ez of each inserted inlet layer from the
   * discrete Gauss law of the incoming charge (ChargeMatchedInlet,
   * src/charge_matched_inlet.h:17-72) and extend its departure from the
   * reference oddly across the inlet for the Cowan magnetic update
   * (src/moving_window_fields.cpp:225-236). */
  uint32_t inlet_charge_match;
  aprl_magnet magnets[APRL_MAX_MAGNETS];
  /* Bit-reproducible mode (no counterpart in the reference, whose deposit is
   * serial and therefore repeatable).  0: the current J is summed with FP64
   * atomics, whose order -- and so the last bits of J -- varies from run to
   * run.  1: every deposit contribution is rounded once to a 128-bit fixed
   * point (a power-of-two quantum below 2^-61 of the run's largest possible
   * single contribution, 4*max|q|*c/(dx*dy*dz)) and summed as integers, which is exact and
   * order-free, then converted to binary64 once per trial; the charge-matched
   * inlet's layer charge is summed the same way.  Two runs of the same
   * requests then give identical bits on the same GPU, and J is closer to
   * the exact sum than either the FP64 atomics or the reference's serial
   * binary64 sum.  The particle sort, the compactions and the residual sums
   * are deterministic in both modes.  Costs a second L2 reduction per
   * contribution and one grid pass per trial. */
  uint32_t deterministic;
  /* mesh.moving_window.reference_surface_current (src/config.cpp:1150; off
   * by default; transverse-only CPML): the prescribed equivalent surface
   * current of the inlet reference (TransverseReferenceCurrent,
   * src/transverse_reference_current.h:12-28).  At the points of the
   * physical region's four transverse faces, Jz += curl_z(B_ref)/mu0 of the
   * reference planes lerped to the step (weights as the inlet lerp), after
   * every fixed-point trial's deposit, so it is in every trial's candidate
   * field and in the commit (src/simulation_source_coupling.cpp:44,
   * src/simulation.cpp:548-561).  Outgoing perturbations keep the plain
   * Maxwell/CPML update. */
  uint32_t reference_surface_current;
} aprl_run_config;

/* Per-step results of the coupled step (SourceCoupling log row,
 * src/source_coupling.cpp:189, plus the particle boundary counters of
 * Simulation, src/simulation.cpp:4841-4901). */
typedef struct {
  uint64_t step;                 /* completed steps */
  uint32_t iterations;           /* fixed-point trials of the last step */
  uint32_t max_iterations;       /* over all steps since the last reset */
  uint64_t total_iterations;     /* sum over steps since the last reset */
  double force;                  /* last converged self-force defect */
  double work;                   /* last relative work defect */
  uint64_t particles;            /* active particles after the step */
  uint64_t carriers;             /* CPML carriers after the step */
  uint64_t exits;                /* cumulative moving-window exits */
  double exit_charge;
  uint64_t cpml_entries[6];      /* cumulative CPML entries by face */
  double cpml_entry_charge[6];
  uint64_t carrier_outer[6];     /* carriers leaving through outer faces */
  double carrier_outer_charge[6];
  uint64_t cropped_carriers;     /* carriers beyond the window upper edge */
  double cropped_charge;
  int64_t window_offset;         /* current window offset (reference cells) */
  double origin_z;               /* current box-frame window origin z */
  double time_box;               /* box time after the last step */
  uint32_t device_error;         /* first device error code seen (0 = none) */
  uint32_t reserved;
  uint64_t pending;              /* held particles still upstream in the queue */
  uint64_t admitted;             /* cumulative PendingParticleQueue::admit count */
  uint64_t activations;          /* cumulative activation-plane crossings */
  uint64_t held;                 /* held (frozen) particles in the list */
} aprl_step_stats;

typedef struct aprl_run aprl_run;

/* ---------------------------------------------------------------------- */
const char* aprl_last_error(void);
int aprl_abi_version(void);

/* SIMagneticElement::prepare (src/eb_sources.cpp:313-350). */
aprl_status aprl_magnet_prepare(aprl_magnet* magnet);

/* Cowan-z smoothing coefficients, EBCowanCoefficients::forZDispersion
 * (src/eb_field.cpp:33-73).  out: alpha[3], beta[3], deltaXY, deltaYZ,
 * deltaZX, ratio[3] (12 doubles). */
aprl_status aprl_cowan_coefficients(double dx, double dy, double dz,
                                    double out[12]);

/* RelativisticBorisPusher::push (src/eb_particles.cpp:207-216): for each of
 * `count` particles, pushMomentum (:99-127: half electric kick, magnetic
 * rotation at the kicked gamma, half kick) with its own E and B
 * (electric/magnetic: 3*count values, box frame, SI), then pushPosition
 * (:129-136: drift over dt at the new proper velocity).  Positions and
 * proper velocities are updated in place (host arrays; the work runs on the
 * current device).  The reference checks the parameters the same way
 * ("Invalid SI particle pusher parameters", std::invalid_argument).  The
 * moving-window coupled step does not use it: held particles drift at
 * c*frozenBetaZ and active ones take the Lapenta-Markidis push. */
aprl_status aprl_boris_push(size_t count, double* x, double* y, double* z,
                            double* ux, double* uy, double* uz,
                            const double* charge, const double* mass,
                            const double* electric, const double* magnetic,
                            double dt);

/* EBFieldGrid(EBGridGeometry) + EBConvolutionalPML + MovingWindowFields +
 * ConservativeSourceCoupling construction (src/eb_field.cpp:211-229,
 * src/eb_cpml.cpp:296-372, src/moving_window_fields.cpp:327-360,
 * src/source_coupling.cpp:62-68).  `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  Allocates all device state of the run.
 *
 * Device memory: every run draws from one stream-ordered memory pool per
 * device owned by the library (cudaMallocFromPoolAsync on the run's stream).
 * aprl_run_destroy returns the run's memory to that pool, and later runs
 * reuse it without mapping new memory; up to 16 GiB of freed memory stays
 * in the pool for the life of the process (the rest is released to the
 * driver), so that memory is not available to other allocators in the
 * process, such as a framework's caching allocator, while it is held. */
aprl_status aprl_run_create(const aprl_run_config* config, void* stream,
                            aprl_run** out);
aprl_status aprl_run_destroy(aprl_run* run);

/* The prepared inlet reference (MovingWindowReference, src/moving_window_fields.h:15-20,
 * served by Simulation::movingWindowFieldValue, src/simulation_moving_window.cpp:280-294).
 * `component` 0..5 = Ex,Ey,Ez,Bx,By,Bz in the native layout of a grid with
 * (nx, ny, reference_nz) cells.  Copied to the device once. */
aprl_status aprl_run_set_reference(aprl_run* run, unsigned component,
                                   const double* host, size_t count);
/* Streaming form of the same supply, the counterpart of the reference's
 * bounded block reader (src/blocked_cowan_reference.h:59-98): when
 * aprl_run_set_reference was given host == NULL the table is allocated
 * zero-filled, and this call overwrites `planes` native z planes starting at
 * `first_plane` of one component (host holds planes*nx_c*ny_c doubles).
 * The planes take effect at this call's place in the run's stream order:
 * work queued before it reads the old values, work queued after it the new.
 * Their host-to-device transfer starts at once on a copy stream of the run,
 * beside the work already queued (for instance between aprl_run_step_begin
 * and aprl_run_step_end), into a staging buffer from which the run's stream
 * copies them.  From page-locked memory the call returns before the
 * transfer ends: keep `host` unchanged until the run's stream has passed
 * this call. */
aprl_status aprl_run_set_reference_planes(aprl_run* run, unsigned component,
                                          uint64_t first_plane, uint64_t planes,
                                          const double* host);

/* EBFieldGrid component accessors (src/eb_field.h:211-229).  component
 * 0..8 = Ex,Ey,Ez,Bx,By,Bz,Jx,Jy,Jz, logical (window) indexing. */
aprl_status aprl_run_set_field(aprl_run* run, unsigned component,
                               const double* host, size_t count);
aprl_status aprl_run_get_field(aprl_run* run, unsigned component,
                               double* host, size_t count);
/* Yee component extents {nx_c, ny_c, nz_c}. */
aprl_status aprl_run_field_shape(const aprl_run* run, unsigned component,
                                 uint64_t shape[3]);

/* EBConvolutionalPML::checkpointHistory (src/eb_cpml.cpp:568-596): index
 * 0..11, magnetic then electric, pairs (0,1),(0,2),(1,2),(1,0),(2,0),(2,1),
 * in the reference's [slot][k][row] order.  Histories of inactive
 * (z-derivative) terms have length 0. */
aprl_status aprl_run_history_length(const aprl_run* run, unsigned index,
                                    uint64_t* length);
aprl_status aprl_run_set_history(aprl_run* run, unsigned index,
                                 const double* host, size_t count);
aprl_status aprl_run_get_history(aprl_run* run, unsigned index,
                                 double* host, size_t count);

/* Active particles: RelativisticParticleSI (src/eb_particles.h:12-25) as SoA.
 * position in m (box frame), proper velocity u = gamma v / c, charge and
 * mass of the macro-particle (weight already applied), id.  Replaces the
 * particle list, and resets the carrier list when reset_carriers != 0. */
aprl_status aprl_run_set_particles(aprl_run* run, size_t count,
                                   const double* x, const double* y,
                                   const double* z, const double* ux,
                                   const double* uy, const double* uz,
                                   const double* charge, const double* mass,
                                   const uint64_t* id, int reset_carriers);
aprl_status aprl_run_particle_count(const aprl_run* run, size_t* count);
/* Held lab-plane injection state of the current list: frozen flag and held
 * speed frozenBetaZ per particle (src/eb_particles.h:21-22), followed by
 * PendingParticleQueue::extract (src/pending_particle_queue.cpp:128-154):
 * held particles upstream of the inlet that do not take part in the first
 * step leave the list for the queue, in their order; the rest stay. */
aprl_status aprl_run_set_held(aprl_run* run, size_t count, const uint8_t* frozen,
                              const double* frozen_beta_z);
/* Frozen flags and held speeds of the current list (reference order). */
aprl_status aprl_run_get_held(aprl_run* run, size_t capacity, uint8_t* frozen,
                              double* frozen_beta_z, size_t* count);
aprl_status aprl_run_get_particles(aprl_run* run, size_t capacity,
                                   double* x, double* y, double* z,
                                   double* ux, double* uy, double* uz,
                                   double* charge, double* mass,
                                   uint64_t* id, size_t* count);
/* ParticleCPMLCarrier (src/particle_boundary.h:76-84): position, velocity
 * (m/s), charge, currentWeight. */
aprl_status aprl_run_carrier_count(const aprl_run* run, size_t* count);
aprl_status aprl_run_get_carriers(aprl_run* run, size_t capacity,
                                  double* position /* 3*count */,
                                  double* velocity /* 3*count */,
                                  double* charge, double* weight,
                                  size_t* count);
aprl_status aprl_run_set_carriers(aprl_run* run, size_t count,
                                  const double* position,
                                  const double* velocity,
                                  const double* charge, const double* weight);

/* ---- per-operator seams (one step = begin, magnetic, preview, trials,
 *      commit, shift; aprl_run_step runs them all) ---------------------- */

/* MovingWindowFields::beginStep + physicalElectricHalos + EBFieldGrid::
 * advanceMagnetic(halo) with the CPML afterMagneticUpdate
 * (src/simulation.cpp:518-524, src/moving_window_fields.cpp:192-227,
 * src/eb_field.cpp:488-558, src/eb_cpml.cpp:406-468). */
aprl_status aprl_run_advance_magnetic(aprl_run* run);
/* previewElectricBoundary(true) + advanceElectric() with J = 0 + the
 * boundary preview (src/simulation_source_coupling.cpp:18-24,
 * src/eb_field.cpp:582-627, src/moving_window_fields.cpp:168-186). */
aprl_status aprl_run_preview_electric(aprl_run* run);
/* One fixed-point trial: clearCurrent, restore, carrier advance, push +
 * deposit of every active particle, and localResidual
 * (src/simulation_source_coupling.cpp:43-48, src/simulation.cpp:4167-5368,
 * src/source_coupling.cpp:90-159).  residual = {force, defect, scale, calls}. */
aprl_status aprl_run_coupling_trial(aprl_run* run, double residual[4]);
/* Replay + commitConservativeElectric: adopt the last trial's particle and
 * carrier states and E^{n+1} = E* - dt/eps0 J
 * (src/simulation_source_coupling.cpp:56-65). */
aprl_status aprl_run_commit_electric(aprl_run* run);
/* finishMovingWindowStep (src/simulation_moving_window.cpp:341-379):
 * MovingWindowFields::shift (src/moving_window_fields.cpp:439-518) as a
 * z ring-buffer rotation, origin update, carrier crop. */
aprl_status aprl_run_shift(aprl_run* run);

/* Whole steps: Simulation::solve's loop body for one rank with the moving
 * window and conservative-source coupling (src/simulation.cpp:493-613). */
aprl_status aprl_run_step(aprl_run* run, uint32_t steps);

/* One aprl_run_step in two halves (no counterpart in the reference), so that
 * the host can work while the step runs.  aprl_run_step_begin queues the
 * step's magnetic update, preview and the fixed-point trials issued ahead on
 * the run's stream and returns without waiting.  aprl_run_step_end waits for
 * their residuals, runs any further trials the stopping rule asks for, and
 * queues the commit and the shift; the result is exactly aprl_run_step's.
 * Between the two, reference planes may be uploaded
 * (aprl_run_set_reference_planes: stream-ordered after the trials, so the
 * step's commit and shift already see them) and host-side queries made; the
 * seam calls and the whole-step calls are refused until the step ends. */
aprl_status aprl_run_step_begin(aprl_run* run);
aprl_status aprl_run_step_end(aprl_run* run);

/* `steps` coupled steps of `count` independent runs in lock step (no
 * counterpart in the reference, which steps one Simulation per job): each
 * step of every run is queued -- begin, magnetic update, preview and the
 * fixed-point trials issued ahead -- before the host waits for any of them,
 * then each run's residuals are read, its stopping rule applied and its
 * commit and shift queued.  The runs' kernels overlap on their own streams
 * (give each run its own stream at aprl_run_create) and the host waits once
 * per run and step instead of stalling the GPU between runs.  Each run's
 * result is exactly what aprl_run_step gives it.  A run that fails stops
 * there (its status in statuses[i], which may be NULL) while the others go
 * on; the return value is the first failure's status, with its message. */
aprl_status aprl_runs_step(aprl_run* const* runs, size_t count, uint32_t steps,
                           aprl_status* statuses);

aprl_status aprl_run_get_stats(const aprl_run* run, aprl_step_stats* stats);

/* The autotuner's launch shapes for the run's grid extent (no counterpart in
 * the reference).  The grid kernels' launch shapes -- the Cowan magnetic
 * kernel's z planes per block (2, 4, 8, 16) and the thread blocks of the
 * preview, orbit-sum and commit kernels (32x4, 32x8, 64x2, 64x4) -- are
 * chosen per device and grid extent by timing each candidate twice on the
 * first steps of the runs of that extent (real launches of those steps, with
 * CUDA events); every candidate gives the same bits, so tuning changes no
 * result.  Kernels in order: Cowan magnetic, preview, orbit sum, commit. */
typedef struct {
  int32_t decided;                    /* bit k: kernel k's shape is chosen */
  uint32_t cowan_planes_per_block;    /* the choice, or the first candidate */
  uint32_t preview_block[2], orbit_block[2], commit_block[2];
  float candidate_ms[4][4];           /* smallest sample per kernel and candidate (0: none) */
} aprl_tuning;

aprl_status aprl_run_tuning(const aprl_run* run, aprl_tuning* out);
aprl_status aprl_run_reset_iteration_stats(aprl_run* run);

/* Gathered fields of the particles after the last trial: usedE/usedB of the
 * last push and nextE/nextB of the last residual (Slot,
 * src/source_coupling.cpp:19), 3*count doubles each; any pointer may be NULL,
 * and with all four NULL the call only stores the slot count. */
aprl_status aprl_run_get_slot_fields(aprl_run* run, size_t capacity,
                                     double* used_e, double* used_b,
                                     double* next_e, double* next_b,
                                     size_t* count);

/* Detector field plane at a fixed lab z: LabDetectorManager::sampleFieldPlanes
 * + samplePlane (src/lab_detectors.cpp:2426-2490, 2836-2905) without the HDF5
 * writer and without background subtraction.  The plane's box z at the
 * current box time is boxZFromLabZAndBoxT; each pixel (i,j) at the cell
 * centre is interpolated per Yee component (src/lab_detectors.cpp:39-99) and
 * transformed with fieldsBoxToLab.  out: 6*nx*ny doubles, pixel (i,j) ->
 * out[6*(j*nx+i) + {Ex,Ey,Ez,Bx,By,Bz}] (lab frame).  *inside is 0 (and out
 * untouched) when the plane lies outside the window. */
aprl_status aprl_run_sample_field_plane(aprl_run* run, double plane_lab_z,
                                        double* out, size_t count,
                                        int* inside);

/* aprl_run_sample_field_plane without the wait: the plane's kernel and its
 * copy into `out` are queued on the run's stream and the call returns at
 * once (*inside is set before it returns).  The values are in `out` once the
 * stream has passed the copy: after aprl_run_synchronize, or after any later
 * call on the run that waits for its stream -- aprl_run_step does, at each
 * step's coupling-trial read-back.  So a stepping loop can read step n's plane
 * while step n+1 runs.  `out` must stay valid, and unread, until then; it
 * should be page-locked host memory (cudaHostAlloc), or the copy is staged
 * and the call waits for it.  The reference writes each plane synchronously
 * (src/lab_detectors.cpp:2426-2490); this call has no counterpart there. */
aprl_status aprl_run_sample_field_plane_async(aprl_run* run, double plane_lab_z,
                                              double* out, size_t count,
                                              int* inside);

/* Largest plane (count = 6*nx*ny values) that
 * aprl_run_sample_field_plane_noalloc accepts: 6*256*256 doubles, i.e. a
 * fixed 3 MiB device array that every GPU which loads this library keeps
 * until the process exits. */
#define APRL_NOALLOC_PLANE_MAX_VALUES 393216u

/* The detector plane of aprl_run_sample_field_plane (same arguments, same
 * values, same *inside rule), for callers that cannot allocate device memory
 * in the middle of a run.  There is no counterpart of this call in the
 * reference.  Such callers are, for example, a host framework whose caching
 * allocator has already reserved the free device memory, so that a direct
 * cudaMalloc may fail even though the framework holds unused blocks, or a
 * stepping loop that must not take the device-wide synchronisation which
 * cudaFree brings.  aprl_run_sample_field_plane stages the plane in a device
 * buffer that the run allocates on first use; this call stages it in a fixed
 * array built into the library and calls no cudaMalloc or cudaFree.
 *   - count above APRL_NOALLOC_PLANE_MAX_VALUES is rejected with
 *     APRL_ERR_OUT_OF_RANGE; use aprl_run_sample_field_plane there.
 *   - The first call on each device looks up the array's device address, with
 *     that device current.  Make that first call before any stream capture.
 *   - Every call on a device uses the same array.  The call waits for its copy
 *     to the host before it returns, but calls that overlap on the GPU (from
 *     several host threads or runs at once) race for the array.
 *   - The kernel writes every value of the plane, so nothing left over from
 *     an earlier call needs clearing. */
aprl_status aprl_run_sample_field_plane_noalloc(aprl_run* run, double plane_lab_z,
                                                double* out, size_t count,
                                                int* inside);

/* Energy ledger of the moving window (MovingWindowFieldEnergyLedger,
 * src/moving_window_fields.h:37-57, with its measurements at
 * src/moving_window_fields.cpp:206-218, 265-290, 387-437, 444-516) and the
 * field and particle energy sums of the EnergyLedgerRecord
 * (src/energy_ledger.h:17-57, src/simulation.cpp:3308-3340, 3591-3626).
 * The reference sums in long double; every sum here is reduced on the GPU in
 * double-double (compensated binary64) arithmetic, in a fixed order, and
 * rounded to binary64 once.  Energies in joules and powers in watts, box
 * frame; faces in the order x-, x+, y-, y+, z-, z+. */
typedef struct {
  /* Cumulative over the steps taken while the ledger was enabled. */
  double inlet_overwrite_energy;  /* inletOverwriteEnergyJ */
  double inserted_energy;         /* insertedEnergyJ */
  double cropped_energy;          /* croppedEnergyJ */
  double remap_energy;            /* remapEnergyJ */
  double outward_energy[6];       /* outwardEnergyFace: trapezoid of the face powers */
  uint64_t overwrite_events;
  uint64_t flux_steps;
  uint64_t remap_steps;
  /* The current state (at the call). */
  double field_energy_interior;   /* localInteriorFieldEnergy: cells outside the xy CPML */
  double boundary_power[6];       /* boundaryPower: outward Poynting power per face */
  double particle_kinetic;        /* sum m c^2 u^2 / (gamma + 1) over stored particles */
  double particle_total;          /* sum m c^2 gamma */
  double represented_electrons;   /* sum m / m_e */
  uint64_t particles;             /* stored macroparticles (held ones included) */
} aprl_energy_ledger;

/* MovingWindowFields::enableEnergyLedger (src/moving_window_fields.cpp:541-545):
 * configure before the first step.  Disabled by default; when enabled, every
 * step adds a handful of plane and face reductions (no host round trip). */
aprl_status aprl_run_enable_energy_ledger(aprl_run* run, int enabled);

/* The ledger's cumulative terms and the reductions of the current state.
 * Valid between steps (no stage in progress).  Waits for the run's stream. */
aprl_status aprl_run_energy_ledger(aprl_run* run, aprl_energy_ledger* out);

/* InitialSelfFieldModel (src/config.h:141-146). */
typedef enum {
  APRL_SELF_FIELD_RELATIVISTIC_POISSON = 0,
  APRL_SELF_FIELD_ELECTROSTATIC_POISSON = 1,
  APRL_SELF_FIELD_COWAN_RELATIVISTIC_POISSON = 2
} aprl_self_field_model;

/* The arguments of EBGaussFieldInitializer::initialize
 * (src/eb_initial_field.h:52-68) beyond the grid and the particles. */
/* How the potential is solved.  CG: conjugate gradients, as
 * EBGaussFieldInitializer (src/eb_initial_field.cpp:829-1095).  MODAL: a
 * direct solve of the same discrete operator on the same Dirichlet box by
 * transverse sine modes and one tridiagonal system along z per mode, the
 * method of the blocked Cowan reference (src/blocked_cowan_reference.h:59-130,
 * whose own check holds it to the CG initializer, verification/
 * blocked_cowan_reference_checks.cpp:61-130); relative_tolerance and
 * maximum_iterations are then unused and iterations is reported as 0. */
typedef enum {
  APRL_SELF_FIELD_SOLVER_CG = 0,
  APRL_SELF_FIELD_SOLVER_MODAL = 1
} aprl_self_field_solver;

/* The charge the potential is solved for.  CIC: the cloud-in-cell charge of
 * EBGaussFieldInitializer (ChargeConservingCurrentDepositor::depositCharge,
 * src/eb_deposition.cpp:168-193).  RUN_SHAPE: the shaped source with which
 * the moving window prepares its inlet reference
 * (BlockedCowanReference::depositQuintic, src/blocked_cowan_reference.cpp:
 * 559-592, selected by the mesh shape at src/simulation_moving_window.cpp:
 * 145-148 and src/config.cpp:1084-1112): for linear-binomial3 the
 * binomial3 transverse weights in x (src/transverse_source_shape.h:8-10),
 * linear in y and the binomial3 node basis in z; for quintic-compensated
 * linear in x and y and the quintic node basis in z.  Its support must lie
 * inside the zero-potential box ("Reference charge support touches Dirichlet
 * surface") and it has no transverse CPML-source padding
 * (include_transverse_cpml_particles must be 0). */
typedef enum {
  APRL_SOURCE_SHAPE_CIC = 0,
  APRL_SOURCE_SHAPE_RUN_SHAPE = 1
} aprl_source_shape;

typedef struct {
  int32_t model;                      /* aprl_self_field_model */
  int32_t include_transverse_cpml_particles;
  int32_t hold_transverse_until_activation;  /* mean beta_z from the held longitudinal velocity */
  int32_t solver;                     /* aprl_self_field_solver */
  double relative_tolerance;          /* CG stop: |r| <= tol |b| */
  double maximum_mean_transverse_beta;
  uint64_t maximum_iterations;
  uint64_t guard_cells[3];            /* staticFieldGuardCells: the CPML cells per axis */
  int32_t source_shape;               /* aprl_source_shape */
  /* Nonzero: the open-transverse-wall reference (BlockedCowanReference with
   * openTransverse, src/blocked_cowan_reference.cpp:662-701, src/
   * open_transverse_trace.h:20-190; mesh.moving_window.open_transverse_reference).
   * The potential extends through the transverse CPML to the outer faces,
   * where it takes the free-space Coulomb potential of the deposited charge
   * (sampled coarsely and interpolated, checked against direct sums, direct
   * everywhere where the check fails), lifted into the solve and used by
   * the field reconstruction at the faces.  guard_cells must be the CPML
   * cells in x and y and 0 in z, the solver MODAL, and
   * include_transverse_cpml_particles 0. */
  int32_t open_transverse;
} aprl_self_field_config;

/* EBGaussInitializationReport (src/eb_initial_field.h:17-34). */
typedef struct {
  uint64_t iterations;
  double relative_residual;           /* post-solve discrete Gauss check */
  double maximum_gauss_residual;
  double total_charge;
  double mean_beta_z;
  double mean_beta_transverse;
  double initial_electric_energy;
  double initial_magnetic_energy;
  double rms_position_cells[3];
  double centre_padding_rms[3];
  uint64_t static_field_guard_cells[3];
  uint64_t transverse_poisson_padding_cells;
  uint64_t temporary_bytes;
} aprl_self_field_report;

/* EBGaussFieldInitializer::initialize (src/eb_initial_field.cpp:829-1095)
 * at one rank, on the GPU, with the run's stored particles as the source:
 * the CIC charge, a matrix-free conjugate-gradient solve of the
 * relativistic (7-point) or Cowan (27-point) Poisson operator with zero
 * potential on the guard surface, E from the potential, B = beta x E / c
 * shifted to the half step, and the discrete Gauss check.  Replaces E and
 * B of the run (J and the CPML histories are untouched); call it before
 * the first step.  The CG dot products are double-double reductions on the
 * device; the host reads the iteration state once per batch of iterations.
 * The reference's own errors (charge touching the zero-potential surface,
 * loss of positive definiteness, no convergence, ...) return
 * APRL_ERR_RUNTIME / APRL_ERR_INVALID_ARGUMENT with its message. */
aprl_status aprl_run_initialize_self_field(aprl_run* run, const aprl_self_field_config* config,
                                           aprl_self_field_report* report);

/* The inlet reference of a moving window prepared on the GPU from a bunch
 * (the role of BlockedCowanReference, src/blocked_cowan_reference.h:59-130,
 * and its fill of MovingWindowReference): the Cowan initial self-field
 * (aprl_run_initialize_self_field with `config`) of the given particles on
 * the reference grid (nx, ny, reference_nz cells from reference_origin),
 * whose E and B become the run's six reference tables.  With
 * config->source_shape = APRL_SOURCE_SHAPE_RUN_SHAPE the charge is the
 * shaped source the moving window uses for its reference (the run's own
 * shape, BlockedCowanReference::depositQuintic), with
 * config->solver = APRL_SELF_FIELD_SOLVER_MODAL the blocked reference's
 * sine-mode and tridiagonal solve; CIC and CG are the initializer's.  The
 * reference's own check holds its blocked solve to the initializer to the
 * CG tolerance (verification/blocked_cowan_reference_checks.cpp:61-130).
 * Particles in box coordinates at box time 0; ids are not needed.
 * Allocates a temporary run of the reference grid's size for the solve.
 * Before the first step. */
aprl_status aprl_run_prepare_reference(aprl_run* run, size_t count, const double* x,
                                       const double* y, const double* z, const double* ux,
                                       const double* uy, const double* uz,
                                       const double* charge, const double* mass,
                                       const aprl_self_field_config* config,
                                       aprl_self_field_report* report);

/* Read back one reference table (the layout of aprl_run_set_reference). */
aprl_status aprl_run_get_reference(aprl_run* run, unsigned component, double* host,
                                   size_t count);

/* Discrete Gauss law of the current state, reduced on the GPU.  The node
 * charge density is the one the run's current conserves, times q/(dx dy dz)
 * per particle: for linear-binomial3, F3 node weights in x over nodes
 * i-1..i+2, linear weights in y over j, j+1 and the binomial3-smoothed
 * linear weights in z over k-1..k+2 (the F3 density of
 * verification/transverse_binomial_checks.cpp:12-66); for
 * quintic-compensated, linear weights in x and y and the quintic node basis
 * in z over floor(z)-5..floor(z)+6 (longitudinal_shape::nodeWeight,
 * src/longitudinal_shape.h:48-56).  At every node
 * G = eps0 div E - rho, div E from the Yee edges around the node (edges
 * outside the grid count as zero).  The reference audits the same law
 * through the charge continuity of its deposit
 * (ChargeConservingCurrentDepositor::maxContinuityResidual,
 * src/eb_deposition.cpp:195-226); with a charge-conserving current and the
 * plain Yee curl of the Ampere update, G at interior nodes does not change
 * in a step except by roundoff. */
typedef struct {
  double max_residual;        /* max |G| over the interior nodes (C/m^3) */
  double rms_residual;        /* root mean square of G over the same nodes */
  double max_charge_density;  /* max |rho| over all nodes */
  double total_charge;        /* sum of rho dV over all nodes (C), double-double */
  uint64_t interior_nodes;    /* nodes i in [cx+1, nx-cx-1], j in [cy+1, ny-cy-1], k in [1, nz-1] */
  uint64_t outside;           /* particle node contributions that fell outside the grid */
} aprl_gauss_law;

/* Between steps, or after the commit and before the shift.  `residual` (may be NULL): (nx+1)*(ny+1)*(nz+1) doubles,
 * G at node (i, j, k) at [(k*(ny+1) + j)*(nx+1) + i].  The density is
 * summed with FP64 atomics, so G varies in the last bits from call to call. */
aprl_status aprl_run_gauss_law(aprl_run* run, aprl_gauss_law* out, double* residual,
                               size_t count);

/* Synchronise the run's stream. */
aprl_status aprl_run_synchronize(aprl_run* run);

/* Stage timers (the GPU counterpart of APRL_PROFILE_INTERVAL stages,
 * src/simulation.cpp:5748-5825): CUDA events around every kernel launch on
 * the run's stream.  aprl_run_profile_read returns, per kernel id, the summed
 * milliseconds and launch count since enable; names via aprl_kernel_name. */
aprl_status aprl_run_profile_enable(aprl_run* run, int enabled);
aprl_status aprl_run_profile_read(aprl_run* run, double* milliseconds,
                                  uint64_t* launches, unsigned capacity,
                                  unsigned* kernels);
const char* aprl_kernel_name(unsigned kernel);
/* Number of kernels this library launched on the run since creation. */
aprl_status aprl_run_launch_count(const aprl_run* run, uint64_t* launches);

/* ---------------------------------------------------------------------------
 * Parameter-scan server.  The reference runs one simulation per MPI job; it
 * has no counterpart of this.  A scan keeps independent runs (each an
 * aprl_run) resident on one GPU and overlaps them: every request waits in a
 * FIFO queue until a slot (a worker thread with its own CUDA stream) is free
 * and its estimated device footprint fits the scan's memory budget next to
 * the runs already on the device; requests that arrive while others run are
 * admitted as slots and memory free up.  Each run's result is the result
 * the same request gives alone, up to the order of the J atomics. */
typedef struct aprl_scan aprl_scan;

typedef struct {
  uint64_t device_budget_bytes;   /* device memory the scan's runs may hold at
                                     once; 0 = 90% of the free memory at create */
  uint32_t max_slots;             /* worker threads (1..256) */
  /* Runs each worker steps in lock step with aprl_runs_step (0 or 1: one run
   * per worker, stepped alone).  A worker admits queued requests into its
   * group at every step boundary while the group has room and the budget
   * allows, and a finished run leaves the group at once, so a request that
   * arrives while others run joins them at the next step. */
  uint32_t runs_per_slot;
} aprl_scan_config;

/* One run.  Every pointer is the caller's and must stay valid until the
 * request has finished (aprl_scan_wait returned it done). */
typedef struct {
  aprl_run_config config;
  uint64_t steps;                 /* coupled steps to run */
  size_t particles;
  const double *x, *y, *z, *ux, *uy, *uz, *charge, *mass;
  const uint64_t* id;
  const uint8_t* frozen;          /* optional held state (NULL: all active) */
  const double* frozen_beta_z;
  const double* reference[6];     /* inlet reference table per component;
                                     NULL: the zero (vacuum) inlet */
  double detector_lab_z;          /* lab plane sampled after the last step */
  double* detector;               /* out: 6*nx*ny doubles, or NULL */
} aprl_scan_request;

enum { APRL_SCAN_QUEUED = 0, APRL_SCAN_RUNNING = 1, APRL_SCAN_DONE = 2 };

typedef struct {
  int32_t state;                  /* APRL_SCAN_* */
  int32_t status;                 /* aprl_status of the finished run */
  int32_t detector_inside;        /* the detector plane was inside the window */
  int32_t slot;                   /* worker slot that ran it */
  uint64_t footprint_bytes;       /* device memory reserved for it */
  double queued_ms;               /* submit -> admission */
  double run_ms;                  /* admission -> finish */
  double total_ms;                /* submit -> finish (latency) */
  double submit_s, start_s, finish_s;  /* steady-clock seconds since create */
  aprl_step_stats stats;          /* of the finished run */
  char message[256];              /* aprl_last_error of a failed run */
} aprl_scan_result;

/* Estimated device bytes of one run: fields, histories, the inlet table,
 * particle and carrier storage. */
aprl_status aprl_scan_footprint(const aprl_run_config* config, size_t particles,
                                uint64_t* bytes);
/* Creates the scan on the current device and starts its worker threads. */
aprl_status aprl_scan_create(const aprl_scan_config* config, aprl_scan** out);
/* Queues a request; a request larger than the whole budget is refused. */
aprl_status aprl_scan_submit(aprl_scan* scan, const aprl_scan_request* request,
                             uint64_t* ticket);
/* Waits up to timeout_seconds (0: poll) for the request; *result holds its
 * state and, once done, its outcome.  Returns APRL_OK whether or not it
 * finished; a finished request is forgotten after it has been returned. */
aprl_status aprl_scan_wait(aprl_scan* scan, uint64_t ticket, double timeout_seconds,
                           aprl_scan_result* result);
/* Finishes the queued and running requests, then stops the workers. */
aprl_status aprl_scan_destroy(aprl_scan* scan);

#ifdef __cplusplus
}
#endif

#endif /* APRL_GPU_H */
