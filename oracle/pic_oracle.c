/*
 * pic_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY, never part of the
 * product path) for APRL 2.1's one-rank step with the moving window and the
 * conservative-source coupling.
 *
 * A serial plain-C restatement of the reference algorithm.  Every function
 * names the reference lines it follows (paths relative to the APRL tree).
 * Arithmetic keeps the reference's operation order and compiles without
 * floating-point contraction (-ffp-contract=off), so field updates agree
 * bit for bit with the reference's own translation units; the reference's
 * long double work sums are kept as long double.  Exceptions of the
 * reference become status codes with the same message text.
 */
#include "pic_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- SI constants (src/eb_field.cpp:13-20) ---------------------------- */
#define SI_C 299792458.0
#define SI_EPSILON0 8.8541878128e-12
#define SI_MU0 1.25663706212e-6
#define SI_E 1.602176634e-19
#define SI_ME 9.1093837139e-31
#define K_PI 3.14159265358979323846
#define K_TWO_PI (2.0 * K_PI)

static __thread char g_error[4096];

static aprl_status fail(aprl_status status, const char* format, ...) {
  va_list args;
  va_start(args, format);
  vsnprintf(g_error, sizeof g_error, format, args);
  va_end(args);
  return status;
}

const char* oracle_last_error(void) { return g_error; }

/* ---- storage ---------------------------------------------------------- */
typedef struct {
  size_t nx, ny, nz;
  double* v;
} comp_t;

static inline size_t cidx(const comp_t* c, size_t i, size_t j, size_t k) {
  return (k * c->ny + j) * c->nx + i;
}
#define AT(c, i, j, k) ((c)->v[cidx((c), (i), (j), (k))])

typedef struct {
  double inverse_kappa_minus_one, decay, drive;
  int active;
} cpml_point;

typedef struct {
  unsigned axis;
  size_t count;
  cpml_point* point;
  size_t* active;  /* activeIndices */
  size_t nactive;
} cpml_profile;

typedef struct {
  unsigned axis;
  size_t dims[3];
  size_t* base;  /* baseByAxisIndex, SIZE_MAX = inactive */
  double* history;
  size_t length;
} cpml_term;

typedef struct {
  double pos[3], u[3];
  double q, m;
  uint64_t id;
  int frozen;      /* RelativisticParticleSI::frozen */
  double beta;     /* RelativisticParticleSI::frozenBetaZ */
} particle_t;

/* PendingParticleQueue (src/pending_particle_queue.h:24-76) at one rank. */
typedef struct {
  particle_t* p;        /* pending_: initial states, extraction order */
  size_t n;
  size_t* order;        /* order_: indices sorted by due step (stable) */
  size_t* offsets;      /* offsets_: buckets + 1 prefix counts */
  size_t buckets;
  size_t cursor;
  uint64_t next_due, last_step, initial_step, maximum_step;
  int extracted;
} pending_t;

typedef struct {
  double pos[3], vel[3];
  double q, w;
} carrier_t;

typedef struct {
  particle_t first, last;
  double guess[3], used_e[3], used_b[3], next_e[3], next_b[3];
  int seen, initialized, replayed, next_ready;
  double time, dt;
  long double abs_grid_work; /* sum over substeps of |BorisWork::gridWork| */
} slot_t;

typedef struct {
  unsigned axis;
  size_t index;
  double value;
} preview_delta_t;

/* The equivalent surface current of the reference (TransverseReferenceCurrent):
 * target points and their prepared values per reference plane. */
typedef struct {
  size_t count;
  size_t* i;
  size_t* j;
  double* table; /* [reference plane][point] */
  int ready;
} surface_current_t;

struct oracle_run {
  aprl_run_config cfg;
  surface_current_t surface;
  double alpha[3], beta[3], delta_xy, delta_yz, delta_zx;
  comp_t f[9];    /* Ex Ey Ez Bx By Bz Jx Jy Jz */
  comp_t old[3];  /* ConservativeSourceCoupling::Impl::old */
  cpml_profile mprof[3], eprof[3];
  cpml_term mterm[3][3], eterm[3][3];
  int has_mterm[3][3], has_eterm[3][3];
  double max_rate[3]; /* ParticleCPMLRegion maximumRate_ */
  double* lower[3];
  double* upper[3];
  preview_delta_t* delta;
  size_t ndelta, delta_cap;
  int preview_present;
  comp_t ref[6];
  int ref_set[6];
  /* window / time state */
  uint64_t step;
  int64_t offset;
  double time;
  double origin[3]; /* globalOriginBox_ == localOriginBox_ at one rank */
  /* particles and carriers */
  particle_t* p;
  size_t np, pcap;
  carrier_t* c;
  size_t nc, ccap;
  slot_t* slot;
  size_t nslot;
  /* step-trial scratch */
  particle_t* retained;
  size_t nretained, rcap;
  carrier_t* rcarrier;
  size_t nrcarrier, rccap;
  /* counters */
  uint64_t exits;
  double exit_charge;
  uint64_t cpml_entries[6];
  double cpml_entry_charge[6];
  uint64_t direct_outer[6];
  double direct_outer_charge[6];
  uint64_t carrier_outer[6];
  double carrier_outer_charge[6];
  uint64_t cropped_carriers;
  double cropped_charge;
  uint32_t last_iterations, max_iterations;
  uint64_t total_iterations;
  double last_force, last_work;
  int replay;
  int stage; /* 0 idle, 1 magnetic done, 2 preview done, 3 trial done */
  uint32_t trials_this_step;
  pending_t pending;
  uint64_t admitted, activations;
  /* saved state of the step (solveConservativeSourceStep restore()) */
  particle_t* saved_p;
  size_t saved_np;
  carrier_t* saved_c;
  size_t saved_nc;
  uint64_t saved_exits, saved_activations;
  double saved_exit_charge;
  uint64_t saved_counts[3][6];
  double saved_charges[3][6];
  /* MovingWindowFieldEnergyLedger (src/moving_window_fields.h:37-57) and the
   * Boundary's per-step flux state (src/moving_window_fields.cpp:158-161). */
  int ledger;
  long double start_power[6], overwrite_power_delta[6];
  long double overwrite_energy, inserted_energy, cropped_energy, remap_energy;
  long double outward_energy[6];
  uint64_t overwrite_events, flux_steps, remap_steps;
};

static aprl_status pending_extract(oracle_run* r);
static aprl_status pending_admit(oracle_run* r);

static void* xrealloc(void* p, size_t bytes) {
  void* q = realloc(p, bytes ? bytes : 1);
  if (!q) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return q;
}

/* ---- Cowan coefficients: EBCowanCoefficients::forZDispersion
 *      (src/eb_field.cpp:33-73) ----------------------------------------- */
aprl_status oracle_cowan_coefficients(double dx, double dy, double dz,
                                      double out[12]) {
  if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0) || !isfinite(dx) ||
      !isfinite(dy) || !isfinite(dz))
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "Cowan-z grid spacing must be positive and finite");
  const double tolerance =
      64.0 * DBL_EPSILON * fmax(dx, fmax(dy, dz));
  if (dx + tolerance < dz || dy + tolerance < dz)
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "Cowan-z requires dz to be the smallest grid spacing");
  double ratio[3];
  ratio[0] = (dz / dx) * (dz / dx);
  ratio[1] = (dz / dy) * (dz / dy);
  ratio[2] = 1.0;
  const double rx = ratio[0], ry = ratio[1], rz = ratio[2];
  const double denominator = rx * ry + ry * rz + rz * rx;
  if (!(denominator > 0.0) || !isfinite(denominator))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid Cowan-z aspect ratios");
  const double product_fraction = rx * ry * rz / denominator;
  double beta[3], alpha[3];
  beta[0] = rx * (1.0 - product_fraction) / 8.0;
  beta[1] = ry * (1.0 - product_fraction) / 8.0;
  beta[2] = rz * (1.0 - product_fraction) / 8.0;
  const double delta_xy = rx * ry * (1.0 / 16.0 - rx * ry / (8.0 * denominator));
  const double delta_yz = ry * rz * (1.0 / 16.0 - ry * rz / (8.0 * denominator));
  const double delta_zx = rz * rx * (1.0 / 16.0 - rz * rx / (8.0 * denominator));
  alpha[0] = 1.0 - 2.0 * beta[1] - 2.0 * beta[2] - 4.0 * delta_yz;
  alpha[1] = 1.0 - 2.0 * beta[2] - 2.0 * beta[0] - 4.0 * delta_zx;
  alpha[2] = 1.0 - 2.0 * beta[0] - 2.0 * beta[1] - 4.0 * delta_xy;
  out[0] = alpha[0]; out[1] = alpha[1]; out[2] = alpha[2];
  out[3] = beta[0]; out[4] = beta[1]; out[5] = beta[2];
  out[6] = delta_xy; out[7] = delta_yz; out[8] = delta_zx;
  out[9] = ratio[0]; out[10] = ratio[1]; out[11] = ratio[2];
  return APRL_OK;
}

/* ---- SIMagneticElement::prepare (src/eb_sources.cpp:313-350) ----------- */
aprl_status oracle_magnet_prepare(aprl_magnet* m) {
  if (!isfinite(m->center[0]) || !isfinite(m->center[1]) ||
      !isfinite(m->center[2]) || !(m->length >= 0.0) || !isfinite(m->length) ||
      !isfinite(m->peak_field) || !isfinite(m->polarization_angle))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid SI magnetic element");
  if (m->type == APRL_MAGNET_PLANAR_UNDULATOR &&
      (!(m->period > 0.0) || !isfinite(m->period)))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Undulator period must be positive");
  if (m->type == APRL_MAGNET_PLANAR_UNDULATOR && m->gaussian_fringe &&
      (!(m->fringe_relative_cutoff > 0.0) ||
       !(m->fringe_relative_cutoff < 1.0) || !isfinite(m->fringe_relative_cutoff)))
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "Undulator fringe_relative_cutoff must be in (0,1)");
  if (m->type == APRL_MAGNET_UNIFORM_DIPOLE && !(m->length > 0.0))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Dipole length must be positive");
  if (m->type == APRL_MAGNET_QUADRUPOLE &&
      (!(m->length > 0.0) || !isfinite(m->quadrupole_gradient)))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Quadrupole length/gradient is invalid");
  m->wave_number = m->type == APRL_MAGNET_PLANAR_UNDULATOR ? K_TWO_PI / m->period : 0.0;
  m->fringe_extent = m->type == APRL_MAGNET_PLANAR_UNDULATOR && m->gaussian_fringe
      ? sqrt(-2.0 * log(m->fringe_relative_cutoff)) / m->wave_number
      : 0.0;
  m->cos_angle = cos(m->polarization_angle);
  m->sin_angle = sin(m->polarization_angle);
  return APRL_OK;
}

/* SIMagneticElement::fieldsLab (src/eb_sources.cpp:352-447), magnetic only;
 * internal end ramps and undulator phase are not modelled (zero defaults). */
static void magnet_fields_lab(const aprl_magnet* m, const double pos[3],
                              double b[3]) {
  b[0] = b[1] = b[2] = 0.0;
  double rel[3] = {pos[0] - m->center[0], pos[1] - m->center[1],
                   pos[2] - m->center[2]};
  const double z = rel[2];
  if (m->type == APRL_MAGNET_QUADRUPOLE) {
    if (z >= 0.0 && z <= m->length) {
      const double x = rel[0] * m->cos_angle + rel[1] * m->sin_angle;
      const double y = -rel[0] * m->sin_angle + rel[1] * m->cos_angle;
      const double bx = m->quadrupole_gradient * y;
      const double by = m->quadrupole_gradient * x;
      b[0] = bx * m->cos_angle - by * m->sin_angle;
      b[1] = bx * m->sin_angle + by * m->cos_angle;
    }
    return;
  }
  if (m->type == APRL_MAGNET_UNIFORM_DIPOLE) {
    if (z >= 0.0 && z <= m->length) {
      b[0] = m->peak_field * m->cos_angle;
      b[1] = m->peak_field * m->sin_angle;
    }
    return;
  }
  double transverse_shape = 0.0, longitudinal_shape = 0.0;
  const double k = m->wave_number;
  if (z >= 0.0 && z <= m->length) {
    transverse_shape = sin(k * z);
    longitudinal_shape = cos(k * z);
  } else if (m->gaussian_fringe) {
    const double fringe_coordinate = z < 0.0 ? z : z - m->length;
    const double distance = fabs(fringe_coordinate);
    if (distance >= m->fringe_extent) return;
    const double q = distance / m->fringe_extent;
    const double q2 = q * q, q3 = q2 * q, q4 = q3 * q, q5 = q4 * q;
    const double taper = 1.0 - 10.0 * q3 + 15.0 * q4 - 6.0 * q5;
    const double taper_derivative =
        (-30.0 * q2 + 60.0 * q3 - 30.0 * q4) / m->fringe_extent;
    const double gaussian = exp(-0.5 * pow(k * distance, 2.0));
    longitudinal_shape = gaussian * taper;
    const double derivative_by_distance =
        gaussian * (taper_derivative - k * k * distance * taper);
    transverse_shape = z < 0.0 ? derivative_by_distance / k
                               : -derivative_by_distance / k;
  } else {
    return;
  }
  const double tc = rel[0] * m->cos_angle + rel[1] * m->sin_angle;
  const double transverse_field = m->peak_field * cosh(k * tc) * transverse_shape;
  b[0] = transverse_field * m->cos_angle;
  b[1] = transverse_field * m->sin_angle;
  b[2] = m->peak_field * sinh(k * tc) * longitudinal_shape;
}

/* BoostFrameTransform::boxToLab (src/boostframe.cpp:221-229). */
static void box_to_lab(const aprl_run_config* g, double t_box, double z_box,
                       double* t_lab, double* z_lab) {
  const double z_shift = z_box - g->box_z_origin;
  *z_lab = g->lab_z_origin + fma(g->boost_gamma_beta * SI_C, t_box,
                                 g->boost_gamma * z_shift);
  *t_lab = g->lab_time_origin + fma(g->boost_gamma_beta / SI_C, z_shift,
                                    g->boost_gamma * t_box);
}

/* BoostFrameTransform::labZFromBoxZT (src/boostframe.cpp:241-245). */
static double lab_z_from_box_zt(const aprl_run_config* g, double z_box,
                                double t_box) {
  return g->lab_z_origin +
         fma(g->boost_gamma_beta * SI_C, t_box, g->boost_gamma * (z_box - g->box_z_origin));
}

/* BoostFrameTransform::boxZFromLabZAndBoxT (src/boostframe.cpp:231-235). */
static double box_z_from_lab_z_and_box_t(const aprl_run_config* g, double z_lab,
                                         double t_box) {
  return g->box_z_origin + (z_lab - g->lab_z_origin) / g->boost_gamma -
         g->boost_beta * SI_C * t_box;
}

/* fieldsLabToBox / fieldsBoxToLab (src/boostframe.cpp:262-285). */
static void fields_lab_to_box(const aprl_run_config* g, const double el[3],
                              const double bl[3], double eb[3], double bb[3]) {
  const double gb = g->boost_gamma_beta, ga = g->boost_gamma;
  eb[0] = fma(-gb * SI_C, bl[1], ga * el[0]);
  eb[1] = fma(gb * SI_C, bl[0], ga * el[1]);
  eb[2] = el[2];
  bb[0] = fma(gb / SI_C, el[1], ga * bl[0]);
  bb[1] = fma(-gb / SI_C, el[0], ga * bl[1]);
  bb[2] = bl[2];
}

static void fields_box_to_lab(const aprl_run_config* g, const double eb[3],
                              const double bb[3], double el[3], double bl[3]) {
  const double gb = g->boost_gamma_beta, ga = g->boost_gamma;
  el[0] = fma(gb * SI_C, bb[1], ga * eb[0]);
  el[1] = fma(-gb * SI_C, bb[0], ga * eb[1]);
  el[2] = eb[2];
  bl[0] = fma(-gb / SI_C, eb[1], ga * bb[0]);
  bl[1] = fma(gb / SI_C, eb[0], ga * bb[1]);
  bl[2] = bb[2];
}

/* SIFieldSourceSet::addPrescribedBox -> transformSampleToBox
 * (src/eb_sources.cpp:537-582): lab magnets only. */
static void add_prescribed_box(const aprl_run_config* g, const double pos[3],
                               double t_box, double e[3], double b[3]) {
  if (g->n_magnets == 0) return;
  double pos_lab[3] = {pos[0], pos[1], pos[2]};
  double t_lab = 0.0;
  box_to_lab(g, t_box, pos[2], &t_lab, &pos_lab[2]);
  double el[3] = {0.0, 0.0, 0.0}, bl[3] = {0.0, 0.0, 0.0};
  for (uint32_t n = 0; n < g->n_magnets; ++n) {
    double contribution[3];
    magnet_fields_lab(&g->magnets[n], pos_lab, contribution);
    for (int a = 0; a < 3; ++a) bl[a] += contribution[a];
  }
  double ebx[3], bbx[3];
  fields_lab_to_box(g, el, bl, ebx, bbx);
  for (int a = 0; a < 3; ++a) {
    e[a] += ebx[a];
    b[a] += bbx[a];
  }
}

aprl_status oracle_prescribed_box(const aprl_run_config* config,
                                  const double position[3], double time,
                                  double e[3], double b[3]) {
  e[0] = e[1] = e[2] = b[0] = b[1] = b[2] = 0.0;
  add_prescribed_box(config, position, time, e, b);
  return APRL_OK;
}

/* BoostFrameTransform::gammaFromProperVelocity (src/boostframe.cpp:74-87). */
static double gamma_u(const double u[3]) {
  const double scale = fmax(1.0, fmax(fabs(u[0]), fmax(fabs(u[1]), fabs(u[2]))));
  const double inverse_scale = 1.0 / scale;
  const double ux = u[0] * inverse_scale, uy = u[1] * inverse_scale,
               uz = u[2] * inverse_scale;
  return scale * sqrt(inverse_scale * inverse_scale + ux * ux + uy * uy + uz * uz);
}

double oracle_gamma(const double u[3]) { return gamma_u(u); }

static inline double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

static inline void cross3(const double l[3], const double r[3], double o[3]) {
  o[0] = l[1] * r[2] - l[2] * r[1];
  o[1] = l[2] * r[0] - l[0] * r[2];
  o[2] = l[0] * r[1] - l[1] * r[0];
}

/* RelativisticBorisPusher::push (src/eb_particles.cpp:99-139, 207-216):
 * pushMomentum then pushPosition, per particle, in place. */
aprl_status oracle_boris_push(size_t count, double* x, double* y, double* z, double* ux,
                              double* uy, double* uz, const double* charge, const double* mass,
                              const double* electric, const double* magnetic, double dt) {
  if (!(dt > 0.0) || !isfinite(dt))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid SI particle pusher parameters");
  for (size_t n = 0; n < count; ++n) {
    const double q = charge[n], m = mass[n];
    if (!(m > 0.0) || !isfinite(m) || !isfinite(q))
      return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid SI particle pusher parameters");
    const double* e = electric + 3 * n;
    const double* b = magnetic + 3 * n;
    double u[3] = {ux[n], uy[n], uz[n]};
    const double kick = q * dt / (2.0 * m * SI_C);
    double minus[3], t[3], prime[3], sv[3], plus[3];
    for (int d = 0; d < 3; ++d) minus[d] = u[d] + kick * e[d];
    const double rs = q * dt / (2.0 * m * gamma_u(minus));
    for (int d = 0; d < 3; ++d) t[d] = rs * b[d];
    cross3(minus, t, prime);
    for (int d = 0; d < 3; ++d) prime[d] += minus[d];
    const double f = 2.0 / (1.0 + (t[0] * t[0] + t[1] * t[1] + t[2] * t[2]));
    for (int d = 0; d < 3; ++d) sv[d] = t[d] * f;
    cross3(prime, sv, plus);
    for (int d = 0; d < 3; ++d) plus[d] += minus[d];
    for (int d = 0; d < 3; ++d) u[d] = plus[d] + kick * e[d];
    const double drift = SI_C * dt / gamma_u(u);
    x[n] += drift * u[0];
    y[n] += drift * u[1];
    z[n] += drift * u[2];
    ux[n] = u[0];
    uy[n] = u[1];
    uz[n] = u[2];
  }
  return APRL_OK;
}

/* source_coupling_math::momentum: Lapenta-Markidis mean-gamma Newton solve
 * (src/source_coupling_math.h:272-293).  Returns iterations+1, or -1 for a
 * nonphysical root, -2 for no convergence. */
int oracle_momentum(double u[3], const double e[3], const double magnetic[3],
                    double q, double m, double h, double known_gamma) {
  const double before[3] = {u[0], u[1], u[2]};
  const double g0 = known_gamma > 0.0 ? known_gamma : gamma_u(before);
  const double ks = q * h / (2 * m * SI_C);
  const double bs = q * h / (2 * m);
  double kick[3], b[3], a[3], axb[3];
  for (int i = 0; i < 3; ++i) {
    kick[i] = e[i] * ks;
    b[i] = magnetic[i] * bs;
  }
  for (int i = 0; i < 3; ++i) a[i] = before[i] + kick[i];
  cross3(a, b, axb);
  const double b2 = dot3(b, b), ka = dot3(kick, a), kb = dot3(kick, b),
               ab = dot3(a, b), kcross = dot3(kick, axb);
  const double first = dot3(kick, before) / g0;
  double G = g0 + first + (dot3(kick, kick) + kcross / g0 - first * first) / g0;
  G = fmax(G, .5 * (g0 + 1.));
  unsigned iteration = 0;
  for (; iteration < 12; ++iteration) {
    const double den = G * G + b2, numerator = G * G * ka + G * kcross + ab * kb;
    const double f = G * (G - g0) - numerator / den;
    const double derivative =
        2 * G - g0 - ((2 * G * ka + kcross) * den - 2 * G * numerator) / (den * den);
    const double correction = f / derivative;
    const double next = G - correction;
    if (!isfinite(next) || next < .5 * (g0 + 1.) - 1e-13) return -1;
    G = fmax(next, .5 * (g0 + 1.));
    if (fabs(correction) <= 8 * DBL_EPSILON * fmax(1., G)) break;
  }
  if (iteration == 12) return -2;
  const double den = G * G + b2;
  for (int k = 0; k < 3; ++k)
    u[k] = 2 * (G * G * a[k] + ab * b[k] + G * axb[k]) / den - before[k];
  return (int)iteration + 1;
}

/* source_coupling_math::chargeWork (src/source_coupling_math.h:24-26). */
static long double charge_work(double q, const double e[3], const double x[3],
                               const double y[3]) {
  long double s = 0;
  for (int a = 0; a < 3; ++a)
    s += (long double)q * e[a] * ((long double)y[a] - x[a]);
  return s;
}

/* ---- longitudinal shapes (src/longitudinal_shape.h:15-117,
 *      src/transverse_source_shape.h:8-10) ------------------------------ */
typedef struct {
  long long first;
  unsigned count;
  double v[12];
} basis_t;

static void node_weights(double f, double w[4]) {
  w[0] = 0.25 * (1. - f);
  w[1] = 0.5 - 0.25 * f;
  w[2] = 0.25 + 0.25 * f;
  w[3] = 0.25 * f;
}

/* basis() for the two production shapes (src/longitudinal_shape.h:25-55). */
static basis_t shape_basis(double z, int edge, int shape) {
  basis_t r;
  if (shape == APRL_SHAPE_LINEAR_BINOMIAL3) {
    const double cell = floor(z), f = z - cell;
    const double c[3] = {.25, .5, .25};
    r.first = (long long)cell - 1;
    r.count = edge ? 3 : 4;
    for (int n = 0; n < 12; ++n) r.v[n] = 0.;
    for (int k = -1; k <= 1; ++k) {
      const double w = c[k + 1];
      if (edge)
        r.v[k + 1] += w;
      else {
        r.v[k + 1] += w * (1. - f);
        r.v[k + 2] += w * f;
      }
    }
    return r;
  }
  const unsigned degree = edge ? 4 : 5;
  const double cell = floor(z), f = z - cell;
  double n[6] = {1., 0., 0., 0., 0., 0.};
  for (unsigned j = 1; j <= degree; ++j) {
    double saved = 0.;
    for (unsigned k = 0; k < j; ++k) {
      const double t = n[k] / j;
      n[k] = saved + (k + 1 - f) * t;
      saved = (f + j - k - 1) * t;
    }
    n[j] = saved;
  }
  const double p = 5., a = p / 6., b = 3 * p / 40. + p * (p - 1) / 72.,
               d = 5 * p / 112. + p * (p - 1) / 80. + p * (p - 1) * (p - 2) / 1296.;
  const double c[7] = {-d / 64., b / 16. + 3 * d / 32., -a / 4. - b / 4. - 15 * d / 64.,
                       1 + a / 2. + 3 * b / 8. + 5 * d / 16.,
                       -a / 4. - b / 4. - 15 * d / 64., b / 16. + 3 * d / 32., -d / 64.};
  r.first = (long long)cell - 5;
  r.count = degree + 7;
  for (int q = 0; q < 12; ++q) r.v[q] = 0.;
  for (unsigned j = 0; j <= degree; ++j)
    for (unsigned k = 0; k < 7; ++k) r.v[j + k] += n[j] * c[k];
  return r;
}

/* Visitor interface of longitudinal_shape::weights. */
typedef struct visitor visitor_t;
struct visitor {
  void (*visit)(visitor_t*, unsigned axis, long long i, long long j,
                long long k, double w);
};

/* binomialXZSegment (src/longitudinal_shape.h:61-94). */
static void binomial_xz_segment(const aprl_run_config* g, const double start[3],
                                const double delta[3], double first,
                                double last, visitor_t* visit) {
  const double width = last - first;
  const double mid = (first + last) * 0.5;
  const double x = start[0] + mid * delta[0], y = start[1] + mid * delta[1],
               z = start[2] + mid * delta[2];
  long long i = (long long)floor(x), j = (long long)floor(y);
  const long long k = (long long)floor(z);
  if (i == (long long)g->nx) --i;
  if (j == (long long)g->ny) --j;
  double wx[4], wz[4];
  node_weights(x - i, wx);
  node_weights(z - k, wz);
  const double wy[2] = {1. - (y - j), y - j};
  const double edge[3] = {0.25, 0.5, 0.25};
  const double slope[4] = {-0.25, -0.25, 0.25, 0.25};
  const double sy[2] = {-1., 1.};
  const double curvature = width * width / 12.;
  const double xy = curvature * delta[0] * delta[1];
  const double xz = curvature * delta[0] * delta[2];
  const double yz = curvature * delta[1] * delta[2];
  for (unsigned c = 0; c < 4; ++c) {
    for (unsigned b = 0; b < 2; ++b) {
      const double weight = width * (wy[b] * wz[c] + yz * sy[b] * slope[c]);
      for (unsigned a = 0; a < 3; ++a)
        visit->visit(visit, 0, i - 1 + a, j + b, k - 1 + c, weight * edge[a]);
    }
    for (unsigned a = 0; a < 4; ++a)
      visit->visit(visit, 1, i - 1 + a, j, k - 1 + c,
                   width * (wx[a] * wz[c] + xz * slope[a] * slope[c]));
  }
  for (unsigned b = 0; b < 2; ++b)
    for (unsigned a = 0; a < 4; ++a) {
      const double weight = width * (wx[a] * wy[b] + xy * slope[a] * sy[b]);
      for (unsigned c = 0; c < 3; ++c)
        visit->visit(visit, 2, i - 1 + a, j + b, k - 1 + c, weight * edge[c]);
    }
}

static int cmp_double(const void* a, const void* b) {
  const double x = *(const double*)a, y = *(const double*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* longitudinal_shape::weights (src/longitudinal_shape.h:97-117), with
 * smoothX = (shape == linear-binomial3) as in production
 * (src/config.cpp:1097-1112).  Returns segments, or -1 on crossing budget. */
static int shape_weights(const aprl_run_config* g, const double origin[3],
                         const double begin[3], const double end[3],
                         visitor_t* visit) {
  const double h[3] = {g->dx, g->dy, g->dz};
  double x[3], v[3], cuts[64];
  unsigned count = 2;
  cuts[0] = 0.;
  cuts[1] = 1.;
  for (unsigned a = 0; a < 3; ++a) {
    x[a] = (begin[a] - origin[a]) / h[a];
    v[a] = (end[a] - begin[a]) / h[a];
    if (v[a] != 0.)
      for (long long j = (long long)floor(fmin(x[a], x[a] + v[a])) + 1;
           j < fmax(x[a], x[a] + v[a]); ++j) {
        if (count == 64) return -1;
        cuts[count++] = (j - x[a]) / v[a];
      }
  }
  qsort(cuts, count, sizeof(double), cmp_double);
  const double q[4] = {-.8611363115940525752, -.3399810435848562648,
                       .3399810435848562648, .8611363115940525752};
  const double qw[4] = {.3478548451374538574, .6521451548625461426,
                        .6521451548625461426, .3478548451374538574};
  int segments = 0;
  for (unsigned s = 1; s < count; ++s) {
    const double width = cuts[s] - cuts[s - 1];
    if (width <= 0.) continue;
    ++segments;
    if (g->shape == APRL_SHAPE_LINEAR_BINOMIAL3) {
      binomial_xz_segment(g, x, v, cuts[s - 1], cuts[s], visit);
      continue;
    }
    for (unsigned t = 0; t < 4; ++t) {
      const double node = q[t], weight = qw[t];
      const double u = .5 * (cuts[s] + cuts[s - 1] + width * node),
                   factor = .5 * width * weight, xx = x[0] + u * v[0],
                   yy = x[1] + u * v[1], zz = x[2] + u * v[2];
      long long i = (long long)floor(xx), j = (long long)floor(yy);
      if (i == (long long)g->nx) --i;
      if (j == (long long)g->ny) --j;
      const double fx = xx - i, fy = yy - j;
      const basis_t nodes = shape_basis(zz, 0, g->shape),
                    edge = shape_basis(zz, 1, g->shape);
      for (unsigned k = 0; k < nodes.count; ++k) {
        const double w = factor * nodes.v[k];
        if (w == 0.) continue;
        for (unsigned b = 0; b < 2; ++b)
          visit->visit(visit, 0, i, j + b, nodes.first + k, w * (b ? fy : 1. - fy));
        for (unsigned a = 0; a < 2; ++a)
          visit->visit(visit, 1, i + a, j, nodes.first + k, w * (a ? fx : 1. - fx));
      }
      for (unsigned k = 0; k < edge.count; ++k) {
        const double w = factor * edge.v[k];
        if (w == 0.) continue;
        for (unsigned b = 0; b < 2; ++b)
          for (unsigned a = 0; a < 2; ++a)
            visit->visit(visit, 2, i + a, j + b, edge.first + k,
                         w * (a ? fx : 1. - fx) * (b ? fy : 1. - fy));
      }
    }
  }
  return segments;
}

typedef struct {
  visitor_t base;
  int32_t* axis;
  int64_t* index;
  double* weight;
  long count, capacity;
} record_visitor;

static void record_visit(visitor_t* v, unsigned axis, long long i, long long j,
                         long long k, double w) {
  record_visitor* r = (record_visitor*)v;
  if (r->count < r->capacity) {
    r->axis[r->count] = (int32_t)axis;
    r->index[3 * r->count] = i;
    r->index[3 * r->count + 1] = j;
    r->index[3 * r->count + 2] = k;
    r->weight[r->count] = w;
  }
  ++r->count;
}

long oracle_shape_weights(const aprl_run_config* config, const double origin[3],
                          const double begin[3], const double end[3],
                          int32_t* axis, int64_t* index, double* weight,
                          long capacity) {
  record_visitor r;
  r.base.visit = record_visit;
  r.axis = axis;
  r.index = index;
  r.weight = weight;
  r.count = 0;
  r.capacity = capacity;
  if (shape_weights(config, origin, begin, end, &r.base) < 0) {
    fail(APRL_ERR_RUNTIME, "Quintic orbit exceeds crossing budget");
    return -1;
  }
  return r.count;
}

/* ---- run construction -------------------------------------------------- */
static void comp_shape(const aprl_run_config* g, unsigned a, size_t s[3]) {
  /* moving_window_fields.cpp shape(): electric and current components are
   * node-centred off their own axis, magnetic ones on it. */
  const int electric = a < 3 || a >= 6;
  const unsigned axis = a % 3;
  const size_t cells[3] = {g->nx, g->ny, g->nz};
  for (unsigned d = 0; d < 3; ++d)
    s[d] = cells[d] + (electric ? (d != axis) : (d == axis));
}

static void comp_alloc(comp_t* c, const size_t s[3]) {
  c->nx = s[0];
  c->ny = s[1];
  c->nz = s[2];
  c->v = (double*)calloc((s[0] * s[1] * s[2]) ? s[0] * s[1] * s[2] : 1, sizeof(double));
}

/* EBCPMLParameters::maximumConductivityRate (src/eb_cpml.cpp:277-294). */
static double maximum_rate(const aprl_run_config* g, unsigned axis) {
  const size_t cells = axis == 0 ? g->cpml_cells_x : (axis == 1 ? g->cpml_cells_y : 0);
  if (cells == 0) return 0.0;
  const double spacing = axis == 0 ? g->dx : (axis == 1 ? g->dy : g->dz);
  const double thickness = (double)cells * spacing;
  return -(g->cpml_polynomial_order + 1.0) * SI_C *
         log(g->cpml_target_reflection) / (2.0 * thickness);
}

/* makeProfile (src/eb_cpml.cpp:195-248) at one rank (z offset 0). */
static void make_profile(const aprl_run_config* g, unsigned axis, int electric,
                         cpml_profile* r) {
  r->axis = axis;
  const size_t local_cells = axis == 0 ? g->nx : (axis == 1 ? g->ny : g->nz);
  const size_t count = local_cells + (electric ? 1 : 0);
  r->count = count;
  r->point = (cpml_point*)calloc(count, sizeof(cpml_point));
  r->active = (size_t*)calloc(count, sizeof(size_t));
  r->nactive = 0;
  const size_t thickness_cells =
      axis == 0 ? g->cpml_cells_x : (axis == 1 ? g->cpml_cells_y : 0);
  if (thickness_cells == 0) return;
  const double thickness = (double)thickness_cells;
  const double sigma_rate_maximum = maximum_rate(g, axis);
  for (size_t local = 0; local < count; ++local) {
    const double position = (double)local + (electric ? 0.0 : 0.5);
    double depth = 0.0;
    if (position < thickness) depth = (thickness - position) / thickness;
    const double upper_start = (double)(local_cells - thickness_cells);
    if (position > upper_start) depth = fmax(depth, (position - upper_start) / thickness);
    if (!(depth > 0.0)) continue;
    depth = fmin(1.0, depth);
    const double graded = pow(depth, g->cpml_polynomial_order);
    const double sigma_rate = sigma_rate_maximum * graded;
    const double kappa = 1.0 + (g->cpml_kappa_max - 1.0) * graded;
    const double alpha_rate = g->cpml_alpha_fraction * sigma_rate_maximum * (1.0 - depth);
    cpml_point* c = &r->point[local];
    c->inverse_kappa_minus_one = 1.0 / kappa - 1.0;
    c->decay = exp(-(sigma_rate / kappa + alpha_rate) * g->dt);
    const double denominator = sigma_rate * kappa + alpha_rate * kappa * kappa;
    c->drive = denominator > 0.0 ? sigma_rate * (c->decay - 1.0) / denominator : 0.0;
    c->active = 1;
    r->active[r->nactive++] = local;
  }
}

/* CPMLMemoryTerm (src/eb_cpml.cpp:42-96). */
static void make_term(unsigned derivative, const size_t shape[3],
                      const cpml_profile* profile, cpml_term* t) {
  t->axis = derivative;
  for (int d = 0; d < 3; ++d) t->dims[d] = shape[d];
  t->base = (size_t*)malloc(sizeof(size_t) * (shape[derivative] ? shape[derivative] : 1));
  for (size_t n = 0; n < shape[derivative]; ++n) t->base[n] = SIZE_MAX;
  const size_t cross = derivative == 0 ? shape[1] * shape[2]
                       : (derivative == 1 ? shape[0] * shape[2] : shape[0] * shape[1]);
  t->length = profile->nactive * cross;
  t->history = (double*)calloc(t->length ? t->length : 1, sizeof(double));
  for (size_t o = 0; o < profile->nactive; ++o) t->base[profile->active[o]] = o * cross;
}

static inline double* term_value(cpml_term* t, size_t i, size_t j, size_t k) {
  const size_t axis_index = t->axis == 0 ? i : (t->axis == 1 ? j : k);
  const size_t base = t->base[axis_index];
  const size_t cross = t->axis == 0 ? k * t->dims[1] + j
                       : (t->axis == 1 ? k * t->dims[0] + i : j * t->dims[0] + i);
  return &t->history[base + cross];
}

static aprl_status validate_config(const aprl_run_config* g) {
  if (g->nx < 2 || g->ny < 2 || g->nz < 2)
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "E/B staggered grid needs at least two cells in every direction");
  if (!(g->dx > 0.0) || !(g->dy > 0.0) || !(g->dz > 0.0) || !(g->dt > 0.0) ||
      !isfinite(g->dx) || !isfinite(g->dy) || !isfinite(g->dz) || !isfinite(g->dt))
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "E/B grid spacing and time step must be positive finite SI values");
  if (fabs(SI_C * g->dt - g->dz) > 64 * DBL_EPSILON * g->dz)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Moving-window requires c*dt=dz");
  if (g->cpml_cells_x < 2 || g->cpml_cells_y < 2 || 2 * g->cpml_cells_x >= g->nx ||
      2 * g->cpml_cells_y >= g->ny)
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "Moving-window requires valid Cowan integer z slabs, xy-only CPML and an inlet reference");
  if (!(g->cpml_polynomial_order > 0.0) ||
      !(g->cpml_target_reflection > 0.0 && g->cpml_target_reflection < 1.0) ||
      !(g->cpml_kappa_max >= 1.0) || !(g->cpml_alpha_fraction >= 0.0))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid CPML grading parameters");
  if (g->shape != APRL_SHAPE_LINEAR_BINOMIAL3 && g->shape != APRL_SHAPE_QUINTIC_COMPENSATED)
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "APRL 2.1 longitudinal_shape must be linear-binomial3 or quintic-compensated");
  /* ChargeMatchedInlet's constructor (src/charge_matched_inlet.h:21-27). */
  if (g->inlet_charge_match &&
      (g->cpml_cells_x + 1 >= g->nx - g->cpml_cells_x || g->cpml_cells_y + 1 >= g->ny - g->cpml_cells_y))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Charge-matched inlet needs an interior physical aperture");
  if (g->substeps < 1 || g->max_trials < 1 || g->max_trials > 64)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid substep or trial count");
  if (!(g->boost_gamma >= 1.0) || !isfinite(g->boost_gamma))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Lorentz gamma must be finite and >= 1");
  if (g->n_magnets > APRL_MAX_MAGNETS)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Too many prescribed magnets");
  return APRL_OK;
}

aprl_status oracle_run_create(const aprl_run_config* config, oracle_run** out) {
  aprl_status s = validate_config(config);
  if (s != APRL_OK) return s;
  if (config->precision != APRL_PRECISION_FP64)
    return fail(APRL_ERR_INVALID_ARGUMENT, "The oracle computes in binary64 only");
  oracle_run* r = (oracle_run*)calloc(1, sizeof(oracle_run));
  r->cfg = *config;
  double co[12];
  s = oracle_cowan_coefficients(config->dx, config->dy, config->dz, co);
  if (s != APRL_OK) {
    free(r);
    return s;
  }
  for (int a = 0; a < 3; ++a) {
    r->alpha[a] = co[a];
    r->beta[a] = co[3 + a];
  }
  r->delta_xy = co[6];
  r->delta_yz = co[7];
  r->delta_zx = co[8];
  for (unsigned a = 0; a < 9; ++a) {
    size_t sh[3];
    comp_shape(config, a, sh);
    comp_alloc(&r->f[a], sh);
    if (a < 3) comp_alloc(&r->old[a], sh);
    if (a < 6) {
      size_t rs[3] = {sh[0], sh[1], config->reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0)};
      r->ref[a].nx = rs[0];
      r->ref[a].ny = rs[1];
      r->ref[a].nz = rs[2];
      r->ref[a].v = NULL;
    }
  }
  for (unsigned axis = 0; axis < 3; ++axis) {
    make_profile(config, axis, 0, &r->mprof[axis]);
    make_profile(config, axis, 1, &r->eprof[axis]);
    r->max_rate[axis] = maximum_rate(config, axis);
  }
  const unsigned pairs[6][2] = {{0, 1}, {0, 2}, {1, 2}, {1, 0}, {2, 0}, {2, 1}};
  for (unsigned pair = 0; pair < 6; ++pair) {
    const unsigned comp = pairs[pair][0], der = pairs[pair][1];
    size_t sh[3];
    comp_shape(config, 3 + comp, sh);
    make_term(der, sh, &r->mprof[der], &r->mterm[comp][der]);
    r->has_mterm[comp][der] = 1;
    comp_shape(config, comp, sh);
    make_term(der, sh, &r->eprof[der], &r->eterm[comp][der]);
    r->has_eterm[comp][der] = 1;
  }
  for (unsigned a = 0; a < 3; ++a) {
    const size_t n = r->f[a].nx * r->f[a].ny;
    r->lower[a] = (double*)calloc(n, sizeof(double));
    r->upper[a] = (double*)calloc(n, sizeof(double));
  }
  r->offset = config->initial_offset;
  r->origin[0] = config->reference_origin[0];
  r->origin[1] = config->reference_origin[1];
  r->origin[2] = fma((double)config->initial_offset, config->dz, config->reference_origin[2]);
  *out = r;
  return APRL_OK;
}

aprl_status oracle_run_destroy(oracle_run* r) {
  if (!r) return APRL_OK;
  free(r->surface.i);
  free(r->surface.j);
  free(r->surface.table);
  for (int a = 0; a < 9; ++a) free(r->f[a].v);
  for (int a = 0; a < 3; ++a) {
    free(r->old[a].v);
    free(r->lower[a]);
    free(r->upper[a]);
  }
  for (int a = 0; a < 6; ++a) free(r->ref[a].v);
  for (int a = 0; a < 3; ++a) {
    free(r->mprof[a].point); free(r->mprof[a].active);
    free(r->eprof[a].point); free(r->eprof[a].active);
    for (int d = 0; d < 3; ++d) {
      if (r->has_mterm[a][d]) { free(r->mterm[a][d].base); free(r->mterm[a][d].history); }
      if (r->has_eterm[a][d]) { free(r->eterm[a][d].base); free(r->eterm[a][d].history); }
    }
  }
  free(r->pending.p); free(r->pending.order); free(r->pending.offsets);
  free(r->delta); free(r->p); free(r->c); free(r->slot); free(r->retained);
  free(r->rcarrier); free(r->saved_p); free(r->saved_c);
  free(r);
  return APRL_OK;
}

aprl_status oracle_run_set_reference(oracle_run* r, unsigned a, const double* host,
                                     size_t count) {
  if (a >= 6) return fail(APRL_ERR_OUT_OF_RANGE, "Moving-window component");
  const size_t n = r->ref[a].nx * r->ref[a].ny * r->ref[a].nz;
  if (count != n) return fail(APRL_ERR_INVALID_ARGUMENT, "Reference component size mismatch");
  free(r->ref[a].v);
  r->ref[a].v = (double*)calloc(n ? n : 1, sizeof(double));
  if (host) memcpy(r->ref[a].v, host, n * sizeof(double)); /* NULL: the zero inlet */
  r->ref_set[a] = 1;
  if (a == 3 || a == 4) { /* the surface current is prepared from Bx, By again */
    free(r->surface.i);
    free(r->surface.j);
    free(r->surface.table);
    memset(&r->surface, 0, sizeof r->surface);
  }
  return APRL_OK;
}

aprl_status oracle_run_field_shape(const oracle_run* r, unsigned a, uint64_t s[3]) {
  if (a >= 9) return fail(APRL_ERR_OUT_OF_RANGE, "Field component");
  s[0] = r->f[a].nx;
  s[1] = r->f[a].ny;
  s[2] = r->f[a].nz;
  return APRL_OK;
}

aprl_status oracle_run_set_field(oracle_run* r, unsigned a, const double* host, size_t count) {
  if (a >= 9) return fail(APRL_ERR_OUT_OF_RANGE, "Field component");
  const size_t n = r->f[a].nx * r->f[a].ny * r->f[a].nz;
  if (count != n) return fail(APRL_ERR_INVALID_ARGUMENT, "Field component size mismatch");
  memcpy(r->f[a].v, host, n * sizeof(double));
  return APRL_OK;
}

aprl_status oracle_run_get_field(oracle_run* r, unsigned a, double* host, size_t count) {
  if (a >= 9) return fail(APRL_ERR_OUT_OF_RANGE, "Field component");
  const size_t n = r->f[a].nx * r->f[a].ny * r->f[a].nz;
  if (count != n) return fail(APRL_ERR_INVALID_ARGUMENT, "Field component size mismatch");
  memcpy(host, r->f[a].v, n * sizeof(double));
  return APRL_OK;
}

static cpml_term* history_term(oracle_run* r, unsigned index) {
  const unsigned pairs[6][2] = {{0, 1}, {0, 2}, {1, 2}, {1, 0}, {2, 0}, {2, 1}};
  const unsigned comp = pairs[index % 6][0], der = pairs[index % 6][1];
  return index < 6 ? &r->mterm[comp][der] : &r->eterm[comp][der];
}

aprl_status oracle_run_history_length(const oracle_run* r, unsigned index, uint64_t* length) {
  if (index >= 12) return fail(APRL_ERR_OUT_OF_RANGE, "CPML checkpoint history index is out of range");
  *length = history_term((oracle_run*)r, index)->length;
  return APRL_OK;
}

aprl_status oracle_run_set_history(oracle_run* r, unsigned index, const double* host, size_t count) {
  if (index >= 12) return fail(APRL_ERR_OUT_OF_RANGE, "CPML checkpoint history index is out of range");
  cpml_term* t = history_term(r, index);
  if (count != t->length) return fail(APRL_ERR_INVALID_ARGUMENT, "CPML history size mismatch");
  memcpy(t->history, host, count * sizeof(double));
  return APRL_OK;
}

aprl_status oracle_run_get_history(oracle_run* r, unsigned index, double* host, size_t count) {
  if (index >= 12) return fail(APRL_ERR_OUT_OF_RANGE, "CPML checkpoint history index is out of range");
  cpml_term* t = history_term(r, index);
  if (count != t->length) return fail(APRL_ERR_INVALID_ARGUMENT, "CPML history size mismatch");
  memcpy(host, t->history, count * sizeof(double));
  return APRL_OK;
}

aprl_status oracle_run_set_particles(oracle_run* r, size_t n, const double* x, const double* y,
                                     const double* z, const double* ux, const double* uy,
                                     const double* uz, const double* q, const double* m,
                                     const uint64_t* id, int reset_carriers) {
  if (n > r->pcap) {
    r->pcap = n;
    r->p = (particle_t*)xrealloc(r->p, n * sizeof(particle_t));
  }
  for (size_t i = 0; i < n; ++i) {
    particle_t* p = &r->p[i];
    p->pos[0] = x[i]; p->pos[1] = y[i]; p->pos[2] = z[i];
    p->u[0] = ux[i]; p->u[1] = uy[i]; p->u[2] = uz[i];
    p->q = q[i]; p->m = m[i]; p->id = id[i];
    p->frozen = 0; p->beta = 0.0;
  }
  r->np = n;
  if (reset_carriers) r->nc = 0;
  return APRL_OK;
}

aprl_status oracle_run_set_held(oracle_run* r, size_t n, const uint8_t* frozen,
                                const double* beta) {
  if (n != r->np) return fail(APRL_ERR_INVALID_ARGUMENT, "Held state must cover the particle list");
  for (size_t i = 0; i < n; ++i) {
    r->p[i].frozen = frozen[i] ? 1 : 0;
    r->p[i].beta = beta[i];
  }
  return pending_extract(r);
}

aprl_status oracle_run_get_held(oracle_run* r, size_t capacity, uint8_t* frozen, double* beta,
                                size_t* count) {
  if (capacity < r->np) return fail(APRL_ERR_INVALID_ARGUMENT, "Particle buffer too small");
  for (size_t i = 0; i < r->np; ++i) {
    if (frozen) frozen[i] = (uint8_t)r->p[i].frozen;
    if (beta) beta[i] = r->p[i].beta;
  }
  *count = r->np;
  return APRL_OK;
}

aprl_status oracle_run_particle_count(const oracle_run* r, size_t* count) {
  *count = r->np;
  return APRL_OK;
}

aprl_status oracle_run_get_particles(oracle_run* r, size_t capacity, double* x, double* y,
                                     double* z, double* ux, double* uy, double* uz,
                                     double* q, double* m, uint64_t* id, size_t* count) {
  if (capacity < r->np) return fail(APRL_ERR_INVALID_ARGUMENT, "Particle buffer too small");
  for (size_t i = 0; i < r->np; ++i) {
    const particle_t* p = &r->p[i];
    if (x) x[i] = p->pos[0];
    if (y) y[i] = p->pos[1];
    if (z) z[i] = p->pos[2];
    if (ux) ux[i] = p->u[0];
    if (uy) uy[i] = p->u[1];
    if (uz) uz[i] = p->u[2];
    if (q) q[i] = p->q;
    if (m) m[i] = p->m;
    if (id) id[i] = p->id;
  }
  *count = r->np;
  return APRL_OK;
}

aprl_status oracle_run_carrier_count(const oracle_run* r, size_t* count) {
  *count = r->nc;
  return APRL_OK;
}

aprl_status oracle_run_get_carriers(oracle_run* r, size_t capacity, double* pos, double* vel,
                                    double* q, double* w, size_t* count) {
  if (capacity < r->nc) return fail(APRL_ERR_INVALID_ARGUMENT, "Carrier buffer too small");
  for (size_t i = 0; i < r->nc; ++i) {
    for (int a = 0; a < 3; ++a) {
      if (pos) pos[3 * i + a] = r->c[i].pos[a];
      if (vel) vel[3 * i + a] = r->c[i].vel[a];
    }
    if (q) q[i] = r->c[i].q;
    if (w) w[i] = r->c[i].w;
  }
  *count = r->nc;
  return APRL_OK;
}

aprl_status oracle_run_set_carriers(oracle_run* r, size_t n, const double* pos,
                                    const double* vel, const double* q, const double* w) {
  if (n > r->ccap) {
    r->ccap = n;
    r->c = (carrier_t*)xrealloc(r->c, n * sizeof(carrier_t));
  }
  for (size_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      r->c[i].pos[a] = pos[3 * i + a];
      r->c[i].vel[a] = vel[3 * i + a];
    }
    r->c[i].q = q[i];
    r->c[i].w = w[i];
  }
  r->nc = n;
  return APRL_OK;
}

/* ---- moving-window reference lookup: Simulation::movingWindowFieldValue
 *      (src/simulation_moving_window.cpp:280-294) ------------------------ */
static aprl_status reference_value(oracle_run* r, unsigned a, size_t i, size_t j,
                                   long long k, uint64_t step, double* out) {
  if (!r->ref_set[a]) return fail(APRL_ERR_INVALID_ARGUMENT, "Missing moving-window inlet reference");
  const double z = (double)k - r->cfg.translation_beta * (double)step;
  const size_t count = r->cfg.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0);
  if (a >= 6 || !isfinite(z) || z < 0. || z > (double)(count - 1))
    return fail(APRL_ERR_OUT_OF_RANGE, "Moving reference query outside prepared native field");
  const size_t lo = (size_t)floor(z), hi = lo + 1 < count - 1 ? lo + 1 : count - 1;
  const double f = z - (double)lo;
  const comp_t* c = &r->ref[a];
  const double lower = c->v[(lo * c->ny + j) * c->nx + i];
  double v = f == 0. ? lower : (1. - f) * lower + f * c->v[(hi * c->ny + j) * c->nx + i];
  if (!isfinite(v)) return fail(APRL_ERR_RUNTIME, "Non-finite moving-window inlet");
  *out = v;
  return APRL_OK;
}

/* ---- Cowan-z Faraday (src/eb_field.cpp:350-558) ------------------------ */
/* electricValue with the moving window's halo planes (both present at one
 * rank: lower = inlet reference, upper = zero plane). */
static double electric_value(const oracle_run* r, unsigned comp, long long i,
                             long long j, long long k) {
  const comp_t* c = &r->f[comp];
  long long coord[3] = {i, j, k};
  const long long size[3] = {(long long)c->nx, (long long)c->ny, (long long)c->nz};
  double sign = 1.0;
  for (unsigned axis = 0; axis < 2; ++axis) {
    if (coord[axis] < 0) {
      if (comp == axis)
        coord[axis] = 0;
      else {
        coord[axis] = -coord[axis];
        sign = -sign;
      }
    } else if (coord[axis] >= size[axis]) {
      if (comp == axis)
        coord[axis] = size[axis] - 1;
      else {
        coord[axis] = 2 * (size[axis] - 1) - coord[axis];
        sign = -sign;
      }
    }
  }
  if (coord[2] < 0 || coord[2] >= size[2]) {
    const double* plane = coord[2] < 0 ? r->lower[comp] : r->upper[comp];
    return sign * plane[(size_t)coord[1] * c->nx + (size_t)coord[0]];
  }
  return sign * AT(c, (size_t)coord[0], (size_t)coord[1], (size_t)coord[2]);
}

/* smoothedElectric (src/eb_field.cpp:419-486); one path, same order. */
static double smoothed_electric(const oracle_run* r, unsigned comp,
                                unsigned derivative, long long i, long long j,
                                long long k) {
  const unsigned ta = (derivative + 1) % 3, tb = (derivative + 2) % 3;
  const double delta = derivative == 0 ? r->delta_yz
                       : (derivative == 1 ? r->delta_zx : r->delta_xy);
  long long base[3] = {i, j, k};
  double result = r->alpha[derivative] * electric_value(r, comp, i, j, k);
  for (int direction = -1; direction <= 1; direction += 2) {
    long long pa[3] = {base[0], base[1], base[2]};
    long long pb[3] = {base[0], base[1], base[2]};
    pa[ta] += direction;
    pb[tb] += direction;
    result += r->beta[ta] * electric_value(r, comp, pa[0], pa[1], pa[2]);
    result += r->beta[tb] * electric_value(r, comp, pb[0], pb[1], pb[2]);
  }
  for (int da = -1; da <= 1; da += 2)
    for (int db = -1; db <= 1; db += 2) {
      long long p[3] = {base[0], base[1], base[2]};
      p[ta] += da;
      p[tb] += db;
      result += delta * electric_value(r, comp, p[0], p[1], p[2]);
    }
  return result;
}

/* advanceMagneticCowan (src/eb_field.cpp:488-558). */
static void advance_magnetic_cowan(oracle_run* r) {
  const aprl_run_config* g = &r->cfg;
  const double dtdx = g->dt / g->dx, dtdy = g->dt / g->dy, dtdz = g->dt / g->dz;
  comp_t* bx = &r->f[3];
  comp_t* by = &r->f[4];
  comp_t* bz = &r->f[5];
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = 0; j < g->ny; ++j)
      for (size_t i = 0; i <= g->nx; ++i) {
        const double dEzDy = smoothed_electric(r, 2, 1, i, j + 1, k) -
                             smoothed_electric(r, 2, 1, i, j, k);
        const double dEyDz = smoothed_electric(r, 1, 2, i, j, k + 1) -
                             smoothed_electric(r, 1, 2, i, j, k);
        AT(bx, i, j, k) -= dtdy * dEzDy - dtdz * dEyDz;
      }
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = 0; j <= g->ny; ++j) {
      double previous = smoothed_electric(r, 2, 0, 0, j, k);
      for (size_t i = 0; i < g->nx; ++i) {
        const double dExDz = smoothed_electric(r, 0, 2, i, j, k + 1) -
                             smoothed_electric(r, 0, 2, i, j, k);
        const double next = smoothed_electric(r, 2, 0, i + 1, j, k);
        const double dEzDx = next - previous;
        AT(by, i, j, k) -= dtdz * dExDz - dtdx * dEzDx;
        previous = next;
      }
    }
  for (size_t k = 0; k <= g->nz; ++k)
    for (size_t j = 0; j < g->ny; ++j) {
      double previous = smoothed_electric(r, 1, 0, 0, j, k);
      for (size_t i = 0; i < g->nx; ++i) {
        const double next = smoothed_electric(r, 1, 0, i + 1, j, k);
        const double dEyDx = next - previous;
        const double dExDy = smoothed_electric(r, 0, 1, i, j + 1, k) -
                             smoothed_electric(r, 0, 1, i, j, k);
        AT(bz, i, j, k) -= dtdx * dEyDx - dtdy * dExDy;
        previous = next;
      }
    }
}

/* forActivePoints order (src/eb_cpml.cpp:140-193), serial. */
typedef void (*point_op)(oracle_run*, void*, size_t, size_t, size_t);
static void for_active_points(oracle_run* r, const cpml_profile* profile,
                              const size_t begin[3], const size_t end[3],
                              point_op op, void* ctx) {
  if (profile->axis == 0) {
    for (size_t k = begin[2]; k < end[2]; ++k)
      for (size_t j = begin[1]; j < end[1]; ++j)
        for (size_t o = 0; o < profile->nactive; ++o) {
          const size_t i = profile->active[o];
          if (i >= begin[0] && i < end[0]) op(r, ctx, i, j, k);
        }
  } else if (profile->axis == 1) {
    for (size_t k = begin[2]; k < end[2]; ++k)
      for (size_t o = 0; o < profile->nactive; ++o) {
        const size_t j = profile->active[o];
        if (j < begin[1] || j >= end[1]) continue;
        for (size_t i = begin[0]; i < end[0]; ++i) op(r, ctx, i, j, k);
      }
  } else {
    for (size_t o = 0; o < profile->nactive; ++o)
      for (size_t j = begin[1]; j < end[1]; ++j) {
        const size_t k = profile->active[o];
        if (k < begin[2] || k >= end[2]) continue;
        for (size_t i = begin[0]; i < end[0]; ++i) op(r, ctx, i, j, k);
      }
  }
}

typedef struct {
  unsigned target, source, derivative;
  double sign, scale;
  cpml_term* term;
  const cpml_profile* profile;
} correct_ctx;

static void magnetic_correct_point(oracle_run* r, void* vctx, size_t i, size_t j, size_t k) {
  correct_ctx* c = (correct_ctx*)vctx;
  long long plus[3] = {(long long)i, (long long)j, (long long)k};
  ++plus[c->derivative];
  const double difference =
      smoothed_electric(r, c->source, c->derivative, plus[0], plus[1], plus[2]) -
      smoothed_electric(r, c->source, c->derivative, i, j, k);
  double* history = term_value(c->term, i, j, k);
  const cpml_point* coefficient =
      &c->profile->point[c->derivative == 0 ? i : (c->derivative == 1 ? j : k)];
  *history = coefficient->decay * *history + coefficient->drive * difference;
  const double correction = coefficient->inverse_kappa_minus_one * difference + *history;
  AT(&r->f[3 + c->target], i, j, k) += c->sign * c->scale * correction;
}

/* EBConvolutionalPML::afterMagneticUpdate (src/eb_cpml.cpp:406-468). */
static void cpml_after_magnetic(oracle_run* r) {
  const aprl_run_config* g = &r->cfg;
  const double scale[3] = {g->dt / g->dx, g->dt / g->dy, g->dt / g->dz};
  const int terms[6][3] = {{0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {1, 2, 0}, {2, 1, 0}, {2, 0, 1}};
  const double signs[6] = {-1.0, 1.0, -1.0, 1.0, -1.0, 1.0};
  for (int t = 0; t < 6; ++t) {
    const unsigned target = terms[t][0], source = terms[t][1], der = terms[t][2];
    const cpml_profile* profile = &r->mprof[der];
    if (profile->nactive == 0) continue;
    correct_ctx c = {target, source, der, signs[t], scale[der], &r->mterm[target][der], profile};
    const comp_t* tc = &r->f[3 + target];
    const size_t begin[3] = {0, 0, 0}, end[3] = {tc->nx, tc->ny, tc->nz};
    for_active_points(r, profile, begin, end, magnetic_correct_point, &c);
  }
}

static void electric_correct_point(oracle_run* r, void* vctx, size_t i, size_t j, size_t k) {
  correct_ctx* c = (correct_ctx*)vctx;
  const comp_t* s = &r->f[3 + c->source];
  const double difference =
      c->derivative == 0 ? AT(s, i, j, k) - AT(s, i - 1, j, k)
      : (c->derivative == 1 ? AT(s, i, j, k) - AT(s, i, j - 1, k)
                            : AT(s, i, j, k) - AT(s, i, j, k - 1));
  double* history = term_value(c->term, i, j, k);
  const cpml_point* coefficient =
      &c->profile->point[c->derivative == 0 ? i : (c->derivative == 1 ? j : k)];
  *history = coefficient->decay * *history + coefficient->drive * difference;
  const double correction = coefficient->inverse_kappa_minus_one * difference + *history;
  AT(&r->f[c->target], i, j, k) += c->sign * c->scale * correction;
}

/* PerfectElectricConductorBoundary::afterElectricUpdate with both z faces
 * non-physical (src/eb_field.cpp:151-209). */
static void pec_termination(oracle_run* r) {
  const aprl_run_config* g = &r->cfg;
  comp_t* ex = &r->f[0];
  comp_t* ey = &r->f[1];
  comp_t* ez = &r->f[2];
  for (size_t k = 0; k <= g->nz; ++k)
    for (size_t i = 0; i < g->nx; ++i) {
      AT(ex, i, 0, k) = 0.0;
      AT(ex, i, g->ny, k) = 0.0;
    }
  for (size_t k = 0; k <= g->nz; ++k)
    for (size_t j = 0; j < g->ny; ++j) {
      AT(ey, 0, j, k) = 0.0;
      AT(ey, g->nx, j, k) = 0.0;
    }
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = 0; j <= g->ny; ++j) {
      AT(ez, 0, j, k) = 0.0;
      AT(ez, g->nx, j, k) = 0.0;
    }
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t i = 0; i <= g->nx; ++i) {
      AT(ez, i, 0, k) = 0.0;
      AT(ez, i, g->ny, k) = 0.0;
    }
}

/* EBConvolutionalPML::afterElectricUpdate (src/eb_cpml.cpp:470-539) with
 * lowerZPhysical = upperZPhysical = false (moving-window Boundary). */
static void cpml_after_electric(oracle_run* r) {
  const aprl_run_config* g = &r->cfg;
  const double curl_scale = g->dt / (SI_MU0 * SI_EPSILON0);
  const double scale[3] = {curl_scale / g->dx, curl_scale / g->dy, curl_scale / g->dz};
  const int terms[6][3] = {{0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {1, 2, 0}, {2, 1, 0}, {2, 0, 1}};
  const double signs[6] = {1.0, -1.0, 1.0, -1.0, 1.0, -1.0};
  for (int t = 0; t < 6; ++t) {
    const unsigned target = terms[t][0], source = terms[t][1], der = terms[t][2];
    const cpml_profile* profile = &r->eprof[der];
    if (profile->nactive == 0) continue;
    correct_ctx c = {target, source, der, signs[t], scale[der], &r->eterm[target][der], profile};
    const comp_t* tc = &r->f[target];
    size_t begin[3] = {0, 0, 0}, end[3] = {tc->nx, tc->ny, tc->nz};
    if (target == 0) {
      begin[1] = 1; end[1] = g->ny;
      begin[2] = 0; end[2] = g->nz + 1;
    } else if (target == 1) {
      begin[0] = 1; end[0] = g->nx;
      begin[2] = 0; end[2] = g->nz + 1;
    } else {
      begin[0] = 1; end[0] = g->nx;
      begin[1] = 1; end[1] = g->ny;
    }
    for_active_points(r, profile, begin, end, electric_correct_point, &c);
  }
  pec_termination(r);
}

/* advanceElectric curl + current part (src/eb_field.cpp:582-627). */
static void advance_electric_curl(oracle_run* r) {
  const aprl_run_config* g = &r->cfg;
  const double curl_scale = g->dt / (SI_MU0 * SI_EPSILON0);
  const double current_scale = g->dt / SI_EPSILON0;
  const double cx = curl_scale / g->dx, cy = curl_scale / g->dy, cz = curl_scale / g->dz;
  comp_t *ex = &r->f[0], *ey = &r->f[1], *ez = &r->f[2];
  comp_t *bx = &r->f[3], *by = &r->f[4], *bz = &r->f[5];
  comp_t *jx = &r->f[6], *jy = &r->f[7], *jz = &r->f[8];
  for (size_t k = 1; k < g->nz; ++k)
    for (size_t j = 1; j < g->ny; ++j)
      for (size_t i = 0; i < g->nx; ++i)
        AT(ex, i, j, k) += cy * (AT(bz, i, j, k) - AT(bz, i, j - 1, k)) -
                           cz * (AT(by, i, j, k) - AT(by, i, j, k - 1)) -
                           current_scale * AT(jx, i, j, k);
  for (size_t k = 1; k < g->nz; ++k)
    for (size_t j = 0; j < g->ny; ++j)
      for (size_t i = 1; i < g->nx; ++i)
        AT(ey, i, j, k) += cz * (AT(bx, i, j, k) - AT(bx, i, j, k - 1)) -
                           cx * (AT(bz, i, j, k) - AT(bz, i - 1, j, k)) -
                           current_scale * AT(jy, i, j, k);
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = 1; j < g->ny; ++j)
      for (size_t i = 1; i < g->nx; ++i)
        AT(ez, i, j, k) += cx * (AT(by, i, j, k) - AT(by, i - 1, j, k)) -
                           cy * (AT(bx, i, j, k) - AT(bx, i, j - 1, k)) -
                           current_scale * AT(jz, i, j, k);
}

/* Boundary::afterElectricUpdate inlet overwrite (src/moving_window_fields.cpp:278-282). */
static aprl_status inlet_overwrite(oracle_run* r) {
  for (unsigned a = 0; a < 2; ++a) {
    comp_t* c = &r->f[a];
    for (size_t j = 0; j < c->ny; ++j)
      for (size_t i = 0; i < c->nx; ++i) {
        double v;
        aprl_status s = reference_value(r, a, i, j, r->offset, r->step + 1, &v);
        if (s != APRL_OK) return s;
        AT(c, i, j, 0) = v;
      }
  }
  return APRL_OK;
}

/* ---- energy ledger ------------------------------------------------------ */
/* EBFieldGrid::fieldEnergyDensityCell (src/eb_field.cpp:715-738): the cell's
 * collocated E (four-node averages) and B (two-node averages), binary64. */
static double energy_density_cell(const oracle_run* r, size_t i, size_t j, size_t k) {
  const comp_t *ex = &r->f[0], *ey = &r->f[1], *ez = &r->f[2];
  const comp_t *bx = &r->f[3], *by = &r->f[4], *bz = &r->f[5];
  const double e0 = 0.25 * (AT(ex, i, j, k) + AT(ex, i, j + 1, k) + AT(ex, i, j, k + 1) +
                            AT(ex, i, j + 1, k + 1));
  const double e1 = 0.25 * (AT(ey, i, j, k) + AT(ey, i + 1, j, k) + AT(ey, i, j, k + 1) +
                            AT(ey, i + 1, j, k + 1));
  const double e2 = 0.25 * (AT(ez, i, j, k) + AT(ez, i + 1, j, k) + AT(ez, i, j + 1, k) +
                            AT(ez, i + 1, j + 1, k));
  const double b0 = 0.5 * (AT(bx, i, j, k) + AT(bx, i + 1, j, k));
  const double b1 = 0.5 * (AT(by, i, j, k) + AT(by, i, j + 1, k));
  const double b2 = 0.5 * (AT(bz, i, j, k) + AT(bz, i, j, k + 1));
  const double en = e0 * e0 + e1 * e1 + e2 * e2;
  const double bn = b0 * b0 + b1 * b1 + b2 * b2;
  return 0.5 * (SI_EPSILON0 * en + bn / SI_MU0);
}

/* EBFieldGrid::poyntingComponentCell (src/eb_field.cpp:740-781). */
static double poynting_cell(const oracle_run* r, size_t i, size_t j, size_t k, unsigned axis) {
  const comp_t *ex = &r->f[0], *ey = &r->f[1], *ez = &r->f[2];
  const comp_t *bx = &r->f[3], *by = &r->f[4], *bz = &r->f[5];
  const double cx = 0.25 * (AT(ex, i, j, k) + AT(ex, i, j + 1, k) + AT(ex, i, j, k + 1) +
                            AT(ex, i, j + 1, k + 1));
  const double cy = 0.25 * (AT(ey, i, j, k) + AT(ey, i + 1, j, k) + AT(ey, i, j, k + 1) +
                            AT(ey, i + 1, j, k + 1));
  const double cz = 0.25 * (AT(ez, i, j, k) + AT(ez, i + 1, j, k) + AT(ez, i, j + 1, k) +
                            AT(ez, i + 1, j + 1, k));
  const double mx = 0.5 * (AT(bx, i, j, k) + AT(bx, i + 1, j, k));
  const double my = 0.5 * (AT(by, i, j, k) + AT(by, i, j + 1, k));
  const double mz = 0.5 * (AT(bz, i, j, k) + AT(bz, i, j, k + 1));
  double ea, eb, ma, mb;
  if (axis == 0) {
    ea = cy; eb = cz; ma = my; mb = mz;
  } else if (axis == 1) {
    ea = cz; eb = cx; ma = mz; mb = mx;
  } else {
    ea = cx; eb = cy; ma = mx; mb = my;
  }
  double s = ea * mb - eb * ma;
  s /= SI_MU0;
  return s;
}

/* planeEnergy (src/moving_window_fields.cpp:387-397): cells of plane k
 * outside the xy CPML, long double accumulation. */
static long double plane_energy(const oracle_run* r, size_t k) {
  const aprl_run_config* g = &r->cfg;
  const long double volume = (long double)g->dx * (long double)g->dy * (long double)g->dz;
  long double value = 0.;
  for (size_t j = g->cpml_cells_y; j < g->ny - g->cpml_cells_y; ++j)
    for (size_t i = g->cpml_cells_x; i < g->nx - g->cpml_cells_x; ++i)
      value += (long double)energy_density_cell(r, i, j, k) * volume;
  return value;
}

/* boundaryPower (src/moving_window_fields.cpp:399-423) at one rank (both z
 * faces local); `inlet_only` restricts it to plane 0 and drops face z+. */
static void boundary_power(const oracle_run* r, int inlet_only, long double power[6]) {
  const aprl_run_config* g = &r->cfg;
  const size_t i0 = g->cpml_cells_x, i1 = g->nx - i0;
  const size_t j0 = g->cpml_cells_y, j1 = g->ny - j0;
  const long double yz = (long double)g->dy * g->dz;
  const long double xz = (long double)g->dx * g->dz;
  const long double xy = (long double)g->dx * g->dy;
  for (int f = 0; f < 6; ++f) power[f] = 0.;
  for (size_t k = 0; k < (inlet_only ? 1 : g->nz); ++k) {
    for (size_t j = j0; j < j1; ++j) {
      power[0] -= (long double)poynting_cell(r, i0, j, k, 0) * yz;
      power[1] += (long double)poynting_cell(r, i1 - 1, j, k, 0) * yz;
    }
    for (size_t i = i0; i < i1; ++i) {
      power[2] -= (long double)poynting_cell(r, i, j0, k, 1) * xz;
      power[3] += (long double)poynting_cell(r, i, j1 - 1, k, 1) * xz;
    }
  }
  for (size_t j = j0; j < j1; ++j)
    for (size_t i = i0; i < i1; ++i) {
      power[4] -= (long double)poynting_cell(r, i, j, 0, 2) * xy;
      if (!inlet_only) power[5] += (long double)poynting_cell(r, i, j, g->nz - 1, 2) * xy;
    }
}

aprl_status oracle_run_enable_energy_ledger(oracle_run* r, int enabled) {
  if (r->step != 0 || r->stage != 0)
    return fail(APRL_ERR_RUNTIME,
                "Moving-window energy ledger must be configured before the first step");
  r->ledger = enabled != 0;
  return APRL_OK;
}

/* The ledger terms plus Simulation::localInteriorFieldEnergy
 * (src/simulation.cpp:3308-3340) and the particle energy sums of the ledger
 * record (src/simulation.cpp:3591-3604) at the current state. */
aprl_status oracle_run_energy_ledger(oracle_run* r, aprl_energy_ledger* out) {
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Energy ledger read inside a step");
  const aprl_run_config* g = &r->cfg;
  memset(out, 0, sizeof *out);
  out->inlet_overwrite_energy = (double)r->overwrite_energy;
  out->inserted_energy = (double)r->inserted_energy;
  out->cropped_energy = (double)r->cropped_energy;
  out->remap_energy = (double)r->remap_energy;
  for (int f = 0; f < 6; ++f) out->outward_energy[f] = (double)r->outward_energy[f];
  out->overwrite_events = r->overwrite_events;
  out->flux_steps = r->flux_steps;
  out->remap_steps = r->remap_steps;
  const long double volume = (long double)g->dx * (long double)g->dy * (long double)g->dz;
  long double energy = 0.;
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = g->cpml_cells_y; j < g->ny - g->cpml_cells_y; ++j)
      for (size_t i = g->cpml_cells_x; i < g->nx - g->cpml_cells_x; ++i)
        energy += (long double)energy_density_cell(r, i, j, k) * volume;
  out->field_energy_interior = (double)energy;
  long double power[6];
  boundary_power(r, 0, power);
  for (int f = 0; f < 6; ++f) out->boundary_power[f] = (double)power[f];
  long double kinetic = 0., total = 0., represented = 0.;
  for (size_t n = 0; n < r->np; ++n) {
    const particle_t* p = &r->p[n];
    const double gamma = gamma_u(p->u);
    const long double mass = (long double)p->m;
    const long double c = (long double)SI_C;
    const long double rest = mass * c * c;
    const long double u2 = (long double)(p->u[0] * p->u[0] + p->u[1] * p->u[1] +
                                         p->u[2] * p->u[2]);
    kinetic += rest * u2 / (long double)(gamma + 1.0);
    total += rest * (long double)gamma;
    represented += mass / (long double)SI_ME;
  }
  out->particle_kinetic = (double)kinetic;
  out->particle_total = (double)total;
  out->represented_electrons = (double)represented;
  out->particles = r->np;
  return APRL_OK;
}

/* ---- step stages -------------------------------------------------------- */
/* clearCurrent (src/eb_field.cpp:271-295). */
static void clear_current(oracle_run* r) {
  for (int a = 6; a < 9; ++a)
    memset(r->f[a].v, 0, r->f[a].nx * r->f[a].ny * r->f[a].nz * sizeof(double));
}

aprl_status oracle_run_advance_magnetic(oracle_run* r) {
  if (r->stage != 0) return fail(APRL_ERR_RUNTIME, "Moving-window beginStep phase/origin mismatch");
  /* admitMovingWindowParticles (src/simulation.cpp:513). */
  aprl_status admitted = pending_admit(r);
  if (admitted != APRL_OK) return admitted;
  /* Simulation::solve (src/simulation.cpp:518-524): clearCurrent, then
   * Boundary::begin (src/moving_window_fields.cpp:192-216) fills the lower
   * halo planes from the reference at (offset-1, step); the upper planes are
   * the zero vectors of the last rank. */
  clear_current(r);
  /* Boundary::begin's flux start (src/moving_window_fields.cpp:214-218). */
  if (r->ledger) {
    boundary_power(r, 0, r->start_power);
    for (int f = 0; f < 6; ++f) r->overwrite_power_delta[f] = 0.;
  }
  for (unsigned a = 0; a < 3; ++a) {
    const comp_t* c = &r->f[a];
    for (size_t j = 0; j < c->ny; ++j)
      for (size_t i = 0; i < c->nx; ++i) {
        double v;
        aprl_status s = reference_value(r, a, i, j, r->offset - 1, r->step, &v);
        if (s != APRL_OK) return s;
        r->lower[a][j * c->nx + i] = v;
      }
  }
  /* With the charge-matched inlet, Ez's departure from the reference at the
   * inlet is extended oddly across it (src/moving_window_fields.cpp:225-236). */
  if (r->cfg.inlet_charge_match) {
    const comp_t* ez = &r->f[2];
    for (size_t j = r->cfg.cpml_cells_y + 1; j < r->cfg.ny - r->cfg.cpml_cells_y; ++j)
      for (size_t i = r->cfg.cpml_cells_x + 1; i < r->cfg.nx - r->cfg.cpml_cells_x; ++i) {
        double v;
        aprl_status s = reference_value(r, 2, i, j, r->offset, r->step, &v);
        if (s != APRL_OK) return s;
        r->lower[2][j * ez->nx + i] -= AT(ez, i, j, 0) - v;
      }
  }
  advance_magnetic_cowan(r);
  cpml_after_magnetic(r);
  r->stage = 1;
  return APRL_OK;
}

static int in_preview_region(const oracle_run* r, unsigned a, size_t i, size_t j, size_t k) {
  const comp_t* v = &r->f[a];
  const size_t c0 = r->cfg.cpml_cells_x, c1 = r->cfg.cpml_cells_y;
  return i <= c0 + 2 || i + c0 + 3 >= v->nx || j <= c1 + 2 || j + c1 + 3 >= v->ny ||
         (a < 2 && k == 0);
}

aprl_status oracle_run_preview_electric(oracle_run* r) {
  if (r->stage != 1) return fail(APRL_ERR_RUNTIME, "Moving-window electric phase mismatch");
  /* ConservativeSourceCoupling::begin (src/source_coupling.cpp:71): snapshot
   * E^n and reset the per-particle slots. */
  for (int a = 0; a < 3; ++a)
    memcpy(r->old[a].v, r->f[a].v, r->f[a].nx * r->f[a].ny * r->f[a].nz * sizeof(double));
  if (r->np > r->nslot) r->slot = (slot_t*)xrealloc(r->slot, r->np * sizeof(slot_t));
  r->nslot = r->np;
  memset(r->slot, 0, r->nslot * sizeof(slot_t));
  /* advanceElectric with J = 0 and the reversible boundary preview
   * (src/simulation_source_coupling.cpp:20-24, src/moving_window_fields.cpp:168-186). */
  advance_electric_curl(r);
  r->ndelta = 0;
  for (unsigned a = 0; a < 3; ++a) {
    const comp_t* v = &r->f[a];
    for (size_t k = 0; k < v->nz; ++k)
      for (size_t j = 0; j < v->ny; ++j)
        for (size_t i = 0; i < v->nx; ++i)
          if (in_preview_region(r, a, i, j, k)) {
            if (r->ndelta == r->delta_cap) {
              r->delta_cap = r->delta_cap ? 2 * r->delta_cap : 4096;
              r->delta = (preview_delta_t*)xrealloc(r->delta, r->delta_cap * sizeof(preview_delta_t));
            }
            r->delta[r->ndelta].axis = a;
            r->delta[r->ndelta].index = cidx(v, i, j, k);
            r->delta[r->ndelta].value = AT(v, i, j, k);
            ++r->ndelta;
          }
  }
  double* saved[6];
  for (unsigned h = 6; h < 12; ++h) {
    cpml_term* t = history_term(r, h);
    saved[h - 6] = (double*)malloc((t->length ? t->length : 1) * sizeof(double));
    memcpy(saved[h - 6], t->history, t->length * sizeof(double));
  }
  cpml_after_electric(r);
  aprl_status s = inlet_overwrite(r);
  for (size_t n = 0; n < r->ndelta; ++n)
    r->delta[n].value = r->f[r->delta[n].axis].v[r->delta[n].index] - r->delta[n].value;
  for (unsigned h = 6; h < 12; ++h) {
    cpml_term* t = history_term(r, h);
    memcpy(t->history, saved[h - 6], t->length * sizeof(double));
    free(saved[h - 6]);
  }
  if (s != APRL_OK) return s;
  r->preview_present = 1;
  /* solveConservativeSourceStep saves the particle/carrier/counter state for
   * the transactional trials (src/simulation_source_coupling.cpp:26-35). */
  r->saved_p = (particle_t*)xrealloc(r->saved_p, (r->np ? r->np : 1) * sizeof(particle_t));
  memcpy(r->saved_p, r->p, r->np * sizeof(particle_t));
  r->saved_np = r->np;
  r->saved_c = (carrier_t*)xrealloc(r->saved_c, (r->nc ? r->nc : 1) * sizeof(carrier_t));
  memcpy(r->saved_c, r->c, r->nc * sizeof(carrier_t));
  r->saved_nc = r->nc;
  r->saved_exits = r->exits;
  r->saved_activations = r->activations;
  r->saved_exit_charge = r->exit_charge;
  memcpy(r->saved_counts[0], r->cpml_entries, sizeof r->cpml_entries);
  memcpy(r->saved_counts[1], r->direct_outer, sizeof r->direct_outer);
  memcpy(r->saved_counts[2], r->carrier_outer, sizeof r->carrier_outer);
  memcpy(r->saved_charges[0], r->cpml_entry_charge, sizeof r->cpml_entry_charge);
  memcpy(r->saved_charges[1], r->direct_outer_charge, sizeof r->direct_outer_charge);
  memcpy(r->saved_charges[2], r->carrier_outer_charge, sizeof r->carrier_outer_charge);
  r->trials_this_step = 0;
  r->stage = 2;
  return APRL_OK;
}

/* ConservativeSourceCoupling::applyCurrentSource (src/source_coupling.cpp:84-89). */
static void apply_current_source(oracle_run* r, double sign) {
  const aprl_run_config* g = &r->cfg;
  for (unsigned a = 0; a < 3; ++a) {
    comp_t* e = &r->f[a];
    const comp_t* jc = &r->f[6 + a];
    for (size_t k = 0; k < e->nz; ++k)
      for (size_t y = 0; y < e->ny; ++y)
        for (size_t x = 0; x < e->nx; ++x) {
          const int applied =
              a == 0 ? (y > 0 && y < g->ny && k != 0 && k != g->nz)
              : (a == 1 ? (x > 0 && x < g->nx && k != 0 && k != g->nz)
                        : (x > 0 && x < g->nx && y > 0 && y < g->ny));
          if (applied) {
            const size_t n = (k * e->ny + y) * e->nx + x;
            if (jc->v[n] != 0.) e->v[n] += sign * g->dt / SI_EPSILON0 * jc->v[n];
          }
        }
  }
}

static void restore_state(oracle_run* r) {
  if (r->saved_np > r->pcap) {
    r->pcap = r->saved_np;
    r->p = (particle_t*)xrealloc(r->p, r->pcap * sizeof(particle_t));
  }
  memcpy(r->p, r->saved_p, r->saved_np * sizeof(particle_t));
  r->np = r->saved_np;
  if (r->saved_nc > r->ccap) {
    r->ccap = r->saved_nc;
    r->c = (carrier_t*)xrealloc(r->c, r->ccap * sizeof(carrier_t));
  }
  memcpy(r->c, r->saved_c, r->saved_nc * sizeof(carrier_t));
  r->nc = r->saved_nc;
  r->exits = r->saved_exits;
  r->activations = r->saved_activations;
  r->exit_charge = r->saved_exit_charge;
  memcpy(r->cpml_entries, r->saved_counts[0], sizeof r->cpml_entries);
  memcpy(r->direct_outer, r->saved_counts[1], sizeof r->direct_outer);
  memcpy(r->carrier_outer, r->saved_counts[2], sizeof r->carrier_outer);
  memcpy(r->cpml_entry_charge, r->saved_charges[0], sizeof r->cpml_entry_charge);
  memcpy(r->direct_outer_charge, r->saved_charges[1], sizeof r->direct_outer_charge);
  memcpy(r->carrier_outer_charge, r->saved_charges[2], sizeof r->carrier_outer_charge);
}

/* ---- gathers (src/source_coupling.cpp:31-51, source_coupling_math.h) ---- */
typedef struct {
  double first, last;
  double begin[3], end[3];
  int valid;
} open_orbit;

/* clipOpenOrbit at one rank (src/source_coupling_math.h:234-250). */
static aprl_status clip_open_orbit(const oracle_run* r, const double begin[3],
                                   const double end[3], open_orbit* o) {
  const aprl_run_config* g = &r->cfg;
  const double ds[3] = {g->dx, g->dy, g->dz};
  const size_t size[3] = {g->nx, g->ny, g->nz};
  o->first = 0.;
  o->last = 1.;
  o->valid = 1;
  for (int a = 0; a < 3; ++a) {
    o->begin[a] = begin[a];
    o->end[a] = end[a];
  }
  for (int a = 0; a < 3; ++a) {
    const double x = (begin[a] - r->origin[a]) / ds[a], d = (end[a] - begin[a]) / ds[a];
    if (!isfinite(x) || !isfinite(d)) return fail(APRL_ERR_RUNTIME, "Nonfinite open coupling orbit");
    if (d == 0.) {
      if (x < 0. || x > (double)size[a]) o->valid = 0;
      continue;
    }
    {
      const double t = -x / d;
      if (d > 0.) o->first = fmax(o->first, t);
      else o->last = fmin(o->last, t);
    }
    {
      const double t = ((double)size[a] - x) / d;
      if (d > 0.) o->last = fmin(o->last, t);
      else o->first = fmax(o->first, t);
    }
  }
  o->valid = o->valid && o->last >= o->first;
  if (o->valid)
    for (int a = 0; a < 3; ++a) {
      const double d = end[a] - begin[a];
      if (o->first != 0.) o->begin[a] = begin[a] + o->first * d;
      if (o->last != 1.) o->end[a] = begin[a] + o->last * d;
    }
  return APRL_OK;
}

typedef struct {
  visitor_t base;
  const oracle_run* r;
  double result[3];
} electric_visitor;

static void electric_visit(visitor_t* v, unsigned d, long long i, long long j,
                           long long k, double w) {
  electric_visitor* ev = (electric_visitor*)v;
  const comp_t* c = &ev->r->f[d];
  if (i < 0 || j < 0 || i >= (long long)c->nx || j >= (long long)c->ny) return;
  if (k < 0 || k >= (long long)c->nz) return; /* no native halo at one rank */
  const size_t n = cidx(c, (size_t)i, (size_t)j, (size_t)k);
  ev->result[d] += .5 * w * (c->v[n] + ev->r->old[d].v[n]);
}

/* Impl::electric(a,b,open=true) for wide shapes (src/source_coupling.cpp:31-39). */
static aprl_status gather_electric(const oracle_run* r, const double a[3],
                                   const double b[3], double out[3]) {
  open_orbit path;
  aprl_status s = clip_open_orbit(r, a, b, &path);
  if (s != APRL_OK) return s;
  if (!path.valid) return fail(APRL_ERR_OUT_OF_RANGE, "Quintic active orbit outside domain");
  electric_visitor ev;
  ev.base.visit = electric_visit;
  ev.r = r;
  ev.result[0] = ev.result[1] = ev.result[2] = 0.0;
  if (shape_weights(&r->cfg, r->origin, path.begin, path.end, &ev.base) < 0)
    return fail(APRL_ERR_RUNTIME, "Quintic orbit exceeds crossing budget");
  const double fraction = path.last - path.first;
  for (int d = 0; d < 3; ++d) out[d] = ev.result[d] * fraction;
  return APRL_OK;
}

/* NativeHalo::openMagneticValue at one rank (src/source_coupling_math.h:113-119). */
static double open_magnetic_value(const comp_t* v, long long i, long long j, long long k) {
  if (i < 0) i = 0;
  if (i > (long long)v->nx - 1) i = (long long)v->nx - 1;
  if (j < 0) j = 0;
  if (j > (long long)v->ny - 1) j = (long long)v->ny - 1;
  if (k < 0) k = 0;
  if (k >= (long long)v->nz) k = (long long)v->nz - 1;
  return v->v[cidx(v, (size_t)i, (size_t)j, (size_t)k)];
}

/* binomialXZMagneticSample (src/source_coupling_math.h:142-167). */
static void binomial_xz_magnetic(const oracle_run* r, const double point[3], double value[3]) {
  const aprl_run_config* g = &r->cfg;
  const double h[3] = {g->dx, g->dy, g->dz};
  for (unsigned a = 0; a < 3; ++a) {
    long long cell[3];
    double fraction[3];
    for (unsigned d = 0; d < 3; ++d) {
      const double pos = (point[d] - r->origin[d]) / h[d] - (a == d ? 0. : 0.5);
      cell[d] = (long long)floor(pos);
      fraction[d] = pos - cell[d];
    }
    double wx[4], wz[4];
    node_weights(fraction[0], wx);
    node_weights(fraction[2], wz);
    const double wy[2] = {1. - fraction[1], fraction[1]};
    value[a] = 0.;
    const comp_t* f = &r->f[3 + a];
    for (unsigned k = 0; k < 4; ++k)
      for (unsigned j = 0; j < 2; ++j) {
        double row = 0.;
        for (unsigned i = 0; i < 4; ++i)
          row += wx[i] * open_magnetic_value(f, cell[0] - 1 + i, cell[1] + j, cell[2] - 1 + k);
        value[a] += wz[k] * wy[j] * row;
      }
  }
}

/* magneticSample(bounds=false, halo, openFaces=true) (src/source_coupling_math.h:122-138). */
static void trilinear_magnetic(const oracle_run* r, const double position[3], double value[3]) {
  const aprl_run_config* g = &r->cfg;
  const double ds[3] = {g->dx, g->dy, g->dz};
  int cell[2][3];
  double fraction[2][3];
  for (unsigned half = 0; half < 2; ++half)
    for (unsigned d = 0; d < 3; ++d) {
      const double x = (position[d] - r->origin[d]) / ds[d] - .5 * half;
      cell[half][d] = (int)floor(x);
      fraction[half][d] = x - cell[half][d];
    }
  for (unsigned axis = 0; axis < 3; ++axis) {
    const unsigned hx = axis == 0 ? 0 : 1, hy = axis == 1 ? 0 : 1, hz = axis == 2 ? 0 : 1;
    value[axis] = 0.;
    const comp_t* f = &r->f[3 + axis];
    for (unsigned k = 0; k < 2; ++k)
      for (unsigned j = 0; j < 2; ++j)
        for (unsigned i = 0; i < 2; ++i) {
          const double x = i ? fraction[hx][0] : 1 - fraction[hx][0],
                       y = j ? fraction[hy][1] : 1 - fraction[hy][1],
                       z = k ? fraction[hz][2] : 1 - fraction[hz][2];
          const double b = open_magnetic_value(f, cell[hx][0] + (int)i, cell[hy][1] + (int)j,
                                               cell[hz][2] + (int)k);
          value[axis] += x * y * z * b;
        }
  }
}

/* Impl::magnetic (src/source_coupling.cpp:40-51): F3 x-z tensor at the
 * clipped-chord midpoint for binomial3, trilinear for quintic. */
static aprl_status gather_magnetic(const oracle_run* r, const double a[3],
                                   const double b[3], double out[3]) {
  open_orbit path;
  aprl_status s = clip_open_orbit(r, a, b, &path);
  if (s != APRL_OK) return s;
  if (!path.valid)
    return fail(APRL_ERR_OUT_OF_RANGE,
                r->cfg.shape == APRL_SHAPE_LINEAR_BINOMIAL3
                    ? "Notch magnetic orbit outside domain"
                    : "Active coupling magnetic orbit has no in-domain portion");
  double middle[3];
  for (int d = 0; d < 3; ++d) middle[d] = (path.begin[d] + path.end[d]) * .5;
  if (r->cfg.shape == APRL_SHAPE_LINEAR_BINOMIAL3)
    binomial_xz_magnetic(r, middle, out);
  else
    trilinear_magnetic(r, middle, out);
  return APRL_OK;
}

/* ---- deposition: longitudinal_shape::Current::deposit at one rank
 *      (src/longitudinal_shape.h:175-187) -------------------------------- */
typedef struct {
  visitor_t base;
  oracle_run* r;
  double scale[3];
  int error;
} deposit_visitor;

static void deposit_visit(visitor_t* v, unsigned a, long long i, long long j,
                          long long k, double w) {
  deposit_visitor* dv = (deposit_visitor*)v;
  if (dv->scale[a] == 0.) return;
  comp_t* c = &dv->r->f[6 + a];
  if (i < 0 || i >= (long long)c->nx) {
    if (dv->r->cfg.shape == APRL_SHAPE_LINEAR_BINOMIAL3) return;
    dv->error = 1;
    return;
  }
  if (j < 0 || j >= (long long)c->ny) {
    dv->error = 2;
    return;
  }
  const double value = dv->scale[a] * w;
  if (k >= 0 && k < (long long)c->nz) AT(c, (size_t)i, (size_t)j, (size_t)k) += value;
}

/* longitudinal_shape::Current::deposit without the depositor's endpoint
 * validation: ConservativeSourceCoupling::depositFrozenSourceSupport
 * (src/source_coupling.cpp:73-78) deposits held sources this way. */
static aprl_status deposit_current(oracle_run* r, const double begin[3], const double end[3],
                                   double charge) {
  const aprl_run_config* g = &r->cfg;
  deposit_visitor dv;
  dv.base.visit = deposit_visit;
  dv.r = r;
  dv.error = 0;
  for (int a = 0; a < 3; ++a)
    dv.scale[a] = charge * (end[a] - begin[a]) / (g->dx * g->dy * g->dz * g->dt);
  if (shape_weights(g, r->origin, begin, end, &dv.base) < 0)
    return fail(APRL_ERR_RUNTIME, "Quintic orbit exceeds crossing budget");
  if (dv.error == 1) return fail(APRL_ERR_OUT_OF_RANGE, "Transverse current support outside x grid");
  if (dv.error == 2) return fail(APRL_ERR_OUT_OF_RANGE, "Transverse current support outside y grid");
  return APRL_OK;
}

/* ChargeConservingCurrentDepositor::depositSegment -> Current::deposit. */
static aprl_status deposit_segment(oracle_run* r, const double begin[3],
                                   const double end[3], double charge) {
  const aprl_run_config* g = &r->cfg;
  /* validatePosition (src/eb_deposition.cpp:228-250). */
  const double extent[3] = {(double)g->nx * g->dx, (double)g->ny * g->dy, (double)g->nz * g->dz};
  const double* pts[2] = {begin, end};
  for (int n = 0; n < 2; ++n)
    for (int a = 0; a < 3; ++a) {
      const double rel = pts[n][a] - r->origin[a];
      const double tol = 64.0 * DBL_EPSILON * fmax(1.0, fmax(fabs(r->origin[a]), extent[a]));
      if (!isfinite(pts[n][a]) || rel < -tol || rel > extent[a] + tol)
        return fail(APRL_ERR_OUT_OF_RANGE, "Particle trajectory endpoint is outside the E/B domain");
    }
  if (!isfinite(charge)) return fail(APRL_ERR_INVALID_ARGUMENT, "Deposited particle charge must be finite");
  deposit_visitor dv;
  dv.base.visit = deposit_visit;
  dv.r = r;
  dv.error = 0;
  for (int a = 0; a < 3; ++a)
    dv.scale[a] = charge * (end[a] - begin[a]) / (g->dx * g->dy * g->dz * g->dt);
  if (shape_weights(g, r->origin, begin, end, &dv.base) < 0)
    return fail(APRL_ERR_RUNTIME, "Quintic orbit exceeds crossing budget");
  if (dv.error == 1) return fail(APRL_ERR_OUT_OF_RANGE, "Transverse current support outside x grid");
  if (dv.error == 2) return fail(APRL_ERR_OUT_OF_RANGE, "Transverse current support outside y grid");
  return APRL_OK;
}

/* ---- particle boundaries (src/particle_boundary.cpp) -------------------- */
typedef struct {
  double position[3];
  double fraction;
  int face;
} boundary_hit;

static double coordinate_tolerance(double lower, double upper) {
  return 64.0 * DBL_EPSILON * fmax(1.0, fmax(fabs(lower), fabs(upper)));
}

typedef struct {
  double outer_lower[3], outer_upper[3], physical_lower[3], physical_upper[3], tolerance[3];
} cpml_region;

/* ParticleCPMLRegion constructor (src/particle_boundary.cpp:56-85) on the
 * global window geometry and origin. */
static void make_cpml_region(const oracle_run* r, cpml_region* c) {
  const aprl_run_config* g = &r->cfg;
  const double spacing[3] = {g->dx, g->dy, g->dz};
  const size_t cells[3] = {g->nx, g->ny, g->nz};
  const size_t pc[3] = {g->cpml_cells_x, g->cpml_cells_y, 0};
  for (int a = 0; a < 3; ++a) {
    c->outer_lower[a] = r->origin[a];
    c->outer_upper[a] = r->origin[a] + (double)cells[a] * spacing[a];
    c->physical_lower[a] = c->outer_lower[a] + (double)pc[a] * spacing[a];
    c->physical_upper[a] = c->outer_upper[a] - (double)pc[a] * spacing[a];
    c->tolerance[a] = coordinate_tolerance(c->outer_lower[a], c->outer_upper[a]);
  }
}

/* ParticleCPMLRegion::firstEntry (src/particle_boundary.cpp:104-174). */
static aprl_status cpml_first_entry(const oracle_run* r, const cpml_region* c,
                                    const double start[3], const double end[3],
                                    boundary_hit* hit, int* entered_out) {
  const size_t pc[3] = {r->cfg.cpml_cells_x, r->cfg.cpml_cells_y, 0};
  double best = INFINITY;
  int best_face = 0, entered = 0;
  for (int axis = 0; axis < 3; ++axis) {
    if (!isfinite(start[axis]) || !isfinite(end[axis]))
      return fail(APRL_ERR_RUNTIME, "Particle CPML trajectory contains a non-finite coordinate");
    if (start[axis] < c->physical_lower[axis] - c->tolerance[axis] ||
        start[axis] > c->physical_upper[axis] + c->tolerance[axis])
      return fail(APRL_ERR_OUT_OF_RANGE, "Active particle starts inside the non-physical CPML region");
    if (pc[axis] == 0) continue;
    double candidate = 0.0;
    int face = 0, hit_axis = 0;
    if (end[axis] < c->physical_lower[axis]) {
      candidate = (c->physical_lower[axis] - start[axis]) / (end[axis] - start[axis]);
      face = 2 * axis;
      hit_axis = 1;
    } else if (end[axis] > c->physical_upper[axis]) {
      candidate = (c->physical_upper[axis] - start[axis]) / (end[axis] - start[axis]);
      face = 2 * axis + 1;
      hit_axis = 1;
    }
    if (hit_axis && candidate < best) {
      best = candidate;
      best_face = face;
      entered = 1;
    }
  }
  *entered_out = entered;
  if (!entered) return APRL_OK;
  const double ft = 64.0 * DBL_EPSILON;
  if (!isfinite(best) || best < -ft || best > 1.0 + ft)
    return fail(APRL_ERR_RUNTIME, "Cannot locate the first particle entry into CPML");
  hit->fraction = fmax(0.0, fmin(1.0, best));
  hit->face = best_face;
  for (int a = 0; a < 3; ++a) {
    hit->position[a] = start[a] + hit->fraction * (end[a] - start[a]);
    hit->position[a] = fmax(c->outer_lower[a], fmin(c->outer_upper[a], hit->position[a]));
  }
  const int normal = best_face / 2;
  hit->position[normal] = (best_face % 2) != 0 ? c->physical_upper[normal] : c->physical_lower[normal];
  return APRL_OK;
}

/* ParticleCPMLRegion::conductivityRate / currentDampingFactor
 * (src/particle_boundary.cpp:176-240). */
static double conductivity_rate(const oracle_run* r, const cpml_region* c, const double pos[3]) {
  const aprl_run_config* g = &r->cfg;
  const double spacing[3] = {g->dx, g->dy, g->dz};
  const size_t pc[3] = {g->cpml_cells_x, g->cpml_cells_y, 0};
  double rate = 0.0;
  for (int axis = 0; axis < 3; ++axis) {
    if (pc[axis] == 0) continue;
    const double thickness = (double)pc[axis] * spacing[axis];
    double depth = 0.0;
    if (pos[axis] < c->physical_lower[axis])
      depth = (c->physical_lower[axis] - pos[axis]) / thickness;
    else if (pos[axis] > c->physical_upper[axis])
      depth = (pos[axis] - c->physical_upper[axis]) / thickness;
    depth = fmax(0.0, fmin(1.0, depth));
    rate += r->max_rate[axis] * pow(depth, g->cpml_polynomial_order);
  }
  return rate;
}

static double current_damping_factor(const oracle_run* r, const cpml_region* c,
                                     const double start[3], const double end[3],
                                     double duration) {
  if (duration == 0.0) return 1.0;
  const double abscissa = sqrt(3.0 / 5.0);
  const double node[3] = {0.5 * (1.0 - abscissa), 0.5, 0.5 * (1.0 + abscissa)};
  const double weight[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
  double average = 0.0;
  for (int s = 0; s < 3; ++s) {
    double pos[3];
    for (int a = 0; a < 3; ++a) pos[a] = start[a] + node[s] * (end[a] - start[a]);
    average += weight[s] * conductivity_rate(r, c, pos);
  }
  const double exponent = -duration * average;
  return exponent < log(DBL_MIN) ? 0.0 : exp(exponent);
}

/* ParticleOpenBoundary::firstExit (src/particle_boundary.cpp:303-373) on
 * the global window. */
static aprl_status outer_first_exit(const oracle_run* r, const double start[3],
                                    const double end[3], boundary_hit* hit, int* out) {
  const aprl_run_config* g = &r->cfg;
  const double spacing[3] = {g->dx, g->dy, g->dz};
  const size_t cells[3] = {g->nx, g->ny, g->nz};
  double lo[3], hi[3], tol[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = r->origin[a];
    hi[a] = fma((double)cells[a], spacing[a], r->origin[a]);
    tol[a] = coordinate_tolerance(lo[a], hi[a]);
  }
  double best = INFINITY;
  int best_face = 0, escaped = 0;
  for (int axis = 0; axis < 3; ++axis) {
    if (!isfinite(start[axis]) || !isfinite(end[axis]))
      return fail(APRL_ERR_RUNTIME, "Particle trajectory contains a non-finite coordinate");
    if (start[axis] < lo[axis] - tol[axis] || start[axis] > hi[axis] + tol[axis])
      return fail(APRL_ERR_OUT_OF_RANGE, "Particle trajectory starts outside the global E/B domain");
    double candidate = 0.0;
    int face = 0, e = 0;
    if (end[axis] < lo[axis]) {
      candidate = (lo[axis] - start[axis]) / (end[axis] - start[axis]);
      face = 2 * axis;
      e = 1;
    } else if (end[axis] > hi[axis]) {
      candidate = (hi[axis] - start[axis]) / (end[axis] - start[axis]);
      face = 2 * axis + 1;
      e = 1;
    }
    if (e && candidate < best) {
      best = candidate;
      best_face = face;
      escaped = 1;
    }
  }
  *out = escaped;
  if (!escaped) return APRL_OK;
  const double ft = 64.0 * DBL_EPSILON;
  if (best < -ft || best > 1.0 + ft || !isfinite(best))
    return fail(APRL_ERR_RUNTIME, "Cannot locate the first particle-domain exit");
  hit->fraction = fmax(0.0, fmin(1.0, best));
  hit->face = best_face;
  for (int a = 0; a < 3; ++a) {
    hit->position[a] = start[a] + hit->fraction * (end[a] - start[a]);
    hit->position[a] = fmax(lo[a], fmin(hi[a], hit->position[a]));
  }
  const int normal = best_face / 2;
  hit->position[normal] = (best_face % 2) ? hi[normal] : lo[normal];
  return APRL_OK;
}

/* Simulation::firstMovingWindowEntry (src/simulation_moving_window.cpp:380-395). */
static aprl_status moving_window_entry(const oracle_run* r, const cpml_region* c,
                                       const double start[3], const double end[3],
                                       double start_fraction, boundary_hit* hit, int* present) {
  aprl_status s = cpml_first_entry(r, c, start, end, hit, present);
  if (s != APRL_OK) return s;
  const double a = lab_z_from_box_zt(&r->cfg, start[2], r->time + start_fraction * r->cfg.dt) -
                   r->cfg.exit_lab_z;
  const double b = lab_z_from_box_zt(&r->cfg, end[2], r->time + r->cfg.dt) - r->cfg.exit_lab_z;
  if (a >= 0.) return fail(APRL_ERR_RUNTIME, "Active particle started beyond trusted moving-window exit");
  if (b >= 0. && b > a) {
    const double fraction = -a / (b - a);
    if (!*present || fraction < hit->fraction) {
      for (int d = 0; d < 3; ++d) hit->position[d] = start[d] + fraction * (end[d] - start[d]);
      hit->fraction = fraction;
      hit->face = 5;
      *present = 1;
    }
  }
  return APRL_OK;
}

/* ---- the particle part of one trial ------------------------------------ */
static void push_retained(oracle_run* r, const particle_t* p) {
  if (r->nretained == r->rcap) {
    r->rcap = r->rcap ? 2 * r->rcap : 1024;
    r->retained = (particle_t*)xrealloc(r->retained, r->rcap * sizeof(particle_t));
  }
  r->retained[r->nretained++] = *p;
}

static void push_rcarrier(oracle_run* r, const carrier_t* c) {
  if (r->nrcarrier == r->rccap) {
    r->rccap = r->rccap ? 2 * r->rccap : 256;
    r->rcarrier = (carrier_t*)xrealloc(r->rcarrier, r->rccap * sizeof(carrier_t));
  }
  r->rcarrier[r->nrcarrier++] = *c;
}

/* processCarrierSegment at one rank (src/simulation.cpp:4310-4407). */
static aprl_status process_carrier_segment(oracle_run* r, const cpml_region* reg,
                                           carrier_t carrier, const double seg_start[3],
                                           double seg_start_fraction) {
  const double cutoff = 64.0 * DBL_EPSILON;
  if (!(seg_start_fraction >= 0.0 && seg_start_fraction <= 1.0) || !isfinite(seg_start_fraction))
    return fail(APRL_ERR_RUNTIME, "Invalid CPML-carrier segment time fraction");
  if (!(carrier.w >= 0.0) || !isfinite(carrier.w))
    return fail(APRL_ERR_RUNTIME, "Invalid CPML carrier current weight");
  if (carrier.w <= cutoff) return APRL_OK;
  boundary_hit outer;
  int exits = 0;
  aprl_status s = outer_first_exit(r, seg_start, carrier.pos, &outer, &exits);
  if (s != APRL_OK) return s;
  double local_end = 1.0;
  double seg_end[3] = {carrier.pos[0], carrier.pos[1], carrier.pos[2]};
  int remove = 0;
  if (exits) {
    local_end = outer.fraction;
    for (int a = 0; a < 3; ++a) seg_end[a] = outer.position[a];
    remove = 1;
  }
  const double global_end = seg_start_fraction + local_end * (1.0 - seg_start_fraction);
  const double duration = (global_end - seg_start_fraction) * r->cfg.dt;
  double midpoint[3];
  for (int a = 0; a < 3; ++a) midpoint[a] = 0.5 * (seg_start[a] + seg_end[a]);
  const double mid_damping = current_damping_factor(r, reg, seg_start, midpoint, 0.5 * duration);
  const double end_damping = current_damping_factor(r, reg, seg_start, seg_end, duration);
  const double deposited = carrier.w * mid_damping;
  const double end_weight = carrier.w * end_damping;
  s = deposit_segment(r, seg_start, seg_end, carrier.q * deposited);
  if (s != APRL_OK) return s;
  if (remove) {
    ++r->carrier_outer[outer.face];
    r->carrier_outer_charge[outer.face] += carrier.q * end_weight;
    return APRL_OK;
  }
  if (end_weight <= cutoff) return APRL_OK;
  carrier.w = end_weight;
  for (int a = 0; a < 3; ++a) carrier.pos[a] = seg_end[a];
  push_rcarrier(r, &carrier);
  return APRL_OK;
}

/* ConservativeSourceCoupling::push (src/source_coupling.cpp:90-104) for a
 * push of `dt` starting at box time `time`. */
static aprl_status coupling_push(oracle_run* r, particle_t* p, slot_t* q, double time,
                                 double dt) {
  const aprl_run_config* g = &r->cfg;
  const unsigned steps = g->substeps;
  if (r->replay) {
    if (!q->seen || q->time != time || q->dt != dt)
      return fail(APRL_ERR_RUNTIME, "Missing converged particle replay");
    for (int a = 0; a < 3; ++a)
      if (q->first.pos[a] != p->pos[a] || q->first.u[a] != p->u[a])
        return fail(APRL_ERR_RUNTIME, "Release state changed during coupled replay");
    q->replayed = 1;
    *p = q->last;
    return APRL_OK;
  }
  if (!q->initialized) {
    for (int a = 0; a < 3; ++a) q->guess[a] = p->pos[a];
    const double gamma = gamma_u(p->u);
    const double s = dt * SI_C / gamma;
    for (int a = 0; a < 3; ++a) q->guess[a] += s * p->u[a];
    q->initialized = 1;
  }
  q->first = *p;
  q->time = time;
  q->dt = dt;
  q->seen = 1;
  if (q->next_ready) {
    for (int a = 0; a < 3; ++a) {
      q->used_e[a] = q->next_e[a];
      q->used_b[a] = q->next_b[a];
    }
  } else {
    aprl_status s = gather_electric(r, p->pos, q->guess, q->used_e);
    if (s != APRL_OK) return s;
    s = gather_magnetic(r, p->pos, q->guess, q->used_b);
    if (s != APRL_OK) return s;
  }
  q->abs_grid_work = 0;
  const double h = dt / steps;
  for (unsigned n = 0; n < steps; ++n) {
    const particle_t before = *p;
    const double g0 = gamma_u(p->u);
    double point[3];
    const double ps = .5 * h * SI_C / g0;
    for (int a = 0; a < 3; ++a) point[a] = p->pos[a] + ps * p->u[a];
    double ee[3] = {0., 0., 0.}, bb[3] = {0., 0., 0.};
    add_prescribed_box(g, point, time + (n + .5) * h, ee, bb);
    double e[3], b[3];
    for (int a = 0; a < 3; ++a) {
      e[a] = q->used_e[a] + ee[a];
      b[a] = q->used_b[a] + bb[a];
    }
    const int it = oracle_momentum(p->u, e, b, p->q, p->m, h, g0);
    if (it == -1) return fail(APRL_ERR_RUNTIME, "Nonphysical local mean-gamma root");
    if (it == -2) return fail(APRL_ERR_RUNTIME, "Local mean-gamma root did not converge");
    const double g1 = gamma_u(p->u);
    double mean[3];
    for (int a = 0; a < 3; ++a) mean[a] = before.u[a] + p->u[a];
    const double xs = h * SI_C / (g0 + g1);
    for (int a = 0; a < 3; ++a) p->pos[a] += xs * mean[a];
    const long double grid_work = charge_work(p->q, q->used_e, before.pos, p->pos);
    q->abs_grid_work += fabsl(grid_work);
  }
  q->last = *p;
  for (int a = 0; a < 3; ++a) q->guess[a] = p->pos[a];
  return APRL_OK;
}

/* ---- held lab-plane injection (src/pending_particle_queue.cpp,
 *      src/simulation.cpp:4919-5035, 5083-5160) --------------------------- */
static uint64_t dbits(double v) { uint64_t b; memcpy(&b, &v, 8); return b; }
static double dfrom(uint64_t b) { double v; memcpy(&v, &b, 8); return v; }
static uint64_t ordered_bits(uint64_t v) {
  return (v & 0x8000000000000000ull) ? ~v : v ^ 0x8000000000000000ull;
}
static double from_ordered(uint64_t v) {
  return dfrom((v & 0x8000000000000000ull) ? v ^ 0x8000000000000000ull : ~v);
}
static int same_spacing(uint64_t a, uint64_t b) {
  const uint64_t m = 0x8000000000000000ull | 0x7ff0000000000000ull;
  return (a & m) == (b & m);
}

/* repeatPositive (src/pending_particle_queue.cpp:38-71): `count` separately
 * rounded additions, skipping constant-spacing runs with integer ULP steps. */
static double repeat_positive(double x, double increment, size_t count, int* overflow) {
  while (count) {
    const double y = x + increment;
    if (!isfinite(y)) { *overflow = 1; return y; }
    if (count == 1 || y == x) return y;
    const double z = y + increment;
    const uint64_t bx = dbits(x), by = dbits(y), bz = dbits(z);
    if (isfinite(z) && same_spacing(bx, by) && same_spacing(by, bz)) {
      const uint64_t ox = ordered_bits(bx), oy = ordered_bits(by), oz = ordered_bits(bz);
      const uint64_t stride = oy - ox;
      if (stride && oz - oy == stride) {
        const uint64_t last_bits = (bx & 0x8000000000000000ull)
                                       ? bx & (0x8000000000000000ull | 0x7ff0000000000000ull)
                                       : bx | 0x000fffffffffffffull;
        const uint64_t available = (ordered_bits(last_bits) - ox) / stride;
        const uint64_t safe = available ? available - 1 : 0;
        const size_t jump = (size_t)(safe < count ? safe : count);
        if (jump) {
          x = from_ordered(ox + (uint64_t)jump * stride);
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

/* repeatHeldAddition (src/pending_particle_queue.cpp:73-88). */
static double repeat_held_addition(double initial, double increment, size_t count) {
  int overflow = 0;
  if (!count) return initial;
  if (increment < 0.) {
    const double result = -repeat_positive(-initial, -increment, count, &overflow);
    return result == 0. ? 0. : result;
  }
  return repeat_positive(initial, increment, count, &overflow);
}

static double held_increment(const oracle_run* r, const particle_t* p) {
  return SI_C * r->cfg.dt * p->beta;  /* heldDistancePerBeta * frozenBetaZ */
}

/* PendingParticleQueue::origin (src/pending_particle_queue.cpp:106-111). */
static double pending_origin(const oracle_run* r, uint64_t step) {
  const int64_t offset = r->cfg.initial_offset - (int64_t)step;
  return fma((double)offset, r->cfg.dz, r->cfg.reference_origin[2]);
}

/* participates (src/pending_particle_queue.cpp:113-117). */
static int participates(const oracle_run* r, const particle_t* p, uint64_t step) {
  const double end = repeat_held_addition(p->pos[2], held_increment(r, p),
                                          step - r->pending.initial_step + 1);
  return end >= pending_origin(r, step);
}

/* firstDue (src/pending_particle_queue.cpp:119-126). */
static uint64_t first_due(const oracle_run* r, const particle_t* p) {
  const pending_t* q = &r->pending;
  const double increment = held_increment(r, p);
  const long double distance = (long double)pending_origin(r, q->initial_step) -
                               (long double)p->pos[2] - (long double)increment;
  const long double estimate = ceill(distance / ((long double)r->cfg.dz + (long double)increment));
  const uint64_t sentinel = q->maximum_step + 1;
  const long double steps_left = (long double)(q->maximum_step - q->initial_step);
  const uint64_t guess = estimate > steps_left
                             ? sentinel
                             : q->initial_step + (uint64_t)(estimate > 1.L ? estimate : 1.L);
  if (guess <= q->maximum_step && participates(r, p, guess) && !participates(r, p, guess - 1))
    return guess;
  if (guess == sentinel && !participates(r, p, q->maximum_step)) return sentinel;
  uint64_t lower = q->initial_step + 1, upper = sentinel;
  while (lower < upper) {
    const uint64_t middle = lower + (upper - lower) / 2;
    if (participates(r, p, middle)) upper = middle;
    else lower = middle + 1;
  }
  return lower;
}

static void advance_next_due(pending_t* q) {
  while (q->next_due <= q->maximum_step &&
         q->offsets[q->next_due - q->initial_step + 1] <= q->cursor)
    ++q->next_due;
}

/* PendingParticleQueue::extract (src/pending_particle_queue.cpp:128-154). */
static aprl_status pending_extract(oracle_run* r) {
  pending_t* q = &r->pending;
  if (q->extracted) return fail(APRL_ERR_RUNTIME, "Pending queue can only be initialized once");
  q->initial_step = r->step;
  q->last_step = r->step;
  q->maximum_step = r->cfg.maximum_step;
  q->next_due = r->step;
  if (!(r->cfg.dz > 0.) || q->initial_step > q->maximum_step)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid pending-window geometry/horizon");
  q->buckets = (size_t)(q->maximum_step - q->initial_step + 2);
  q->offsets = (size_t*)calloc(q->buckets + 1, sizeof(size_t));
  q->p = (particle_t*)malloc((r->np ? r->np : 1) * sizeof(particle_t));
  size_t* due = (size_t*)malloc((r->np ? r->np : 1) * sizeof(size_t));
  const double inlet = pending_origin(r, q->initial_step);
  size_t retained = 0;
  q->n = 0;
  for (size_t i = 0; i < r->np; ++i) {
    const particle_t particle = r->p[i];
    if (particle.frozen && particle.pos[2] < inlet && particle.beta >= 0. &&
        !participates(r, &particle, q->initial_step)) {
      const uint64_t event = first_due(r, &particle);
      due[q->n] = (size_t)(event - q->initial_step);
      ++q->offsets[event - q->initial_step + 1];
      q->p[q->n++] = particle;
    } else {
      r->p[retained++] = particle;
    }
  }
  r->np = retained;
  for (size_t i = 1; i < q->buckets + 1; ++i) q->offsets[i] += q->offsets[i - 1];
  q->order = (size_t*)malloc((q->n ? q->n : 1) * sizeof(size_t));
  size_t* insertion = (size_t*)malloc((q->buckets + 1) * sizeof(size_t));
  memcpy(insertion, q->offsets, (q->buckets + 1) * sizeof(size_t));
  for (size_t i = 0; i < q->n; ++i) q->order[insertion[due[i]]++] = i;
  free(insertion);
  free(due);
  q->extracted = 1;
  advance_next_due(q);
  return APRL_OK;
}

/* PendingParticleQueue::admit (src/pending_particle_queue.cpp:163-186). */
static aprl_status pending_admit(oracle_run* r) {
  pending_t* q = &r->pending;
  if (!q->extracted) return APRL_OK;
  const uint64_t step = r->step;
  if (step < q->last_step || step > q->maximum_step || step > q->next_due)
    return fail(APRL_ERR_RUNTIME, "Pending admission skipped an event or exceeds its horizon");
  q->last_step = step;
  const size_t end = q->offsets[step - q->initial_step + 1];
  const size_t need = r->np + (end - q->cursor);
  if (need > r->pcap) {
    r->pcap = need;
    r->p = (particle_t*)xrealloc(r->p, r->pcap * sizeof(particle_t));
  }
  while (q->cursor < end) {
    particle_t particle = q->p[q->order[q->cursor]];
    particle.pos[2] = repeat_held_addition(particle.pos[2], held_increment(r, &particle),
                                           step - q->initial_step);
    r->p[r->np++] = particle;
    ++q->cursor;
    ++r->admitted;
  }
  advance_next_due(q);
  return APRL_OK;
}

/* ChargeMatchedInlet::particle (src/charge_matched_inlet.h:31-53): one
 * particle's share of the inlet-layer charge at node plane 1, with the wide
 * longitudinal node weight of the run's shape and, for linear-binomial3, the
 * transverse three-point x weights. */
static aprl_status charge_match_particle(const oracle_run* r, const double origin[3],
                                         const particle_t* p, double* rho) {
  const aprl_run_config* g = &r->cfg;
  const int binomial3 = g->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
  const double z = (p->pos[2] - origin[2]) / g->dz;
  const basis_t bz = shape_basis(z, 0, g->shape);
  const double wz = 1 < bz.first || 1 >= bz.first + (long long)bz.count ? 0. : bz.v[1 - bz.first];
  if (wz == 0.) return APRL_OK;
  const double x = (p->pos[0] - origin[0]) / g->dx, y = (p->pos[1] - origin[1]) / g->dy;
  if (!isfinite(x) || !isfinite(y) || !isfinite(z) || !isfinite(p->q))
    return fail(APRL_ERR_RUNTIME, "Nonfinite charge-matched inlet source");
  if (y < 0. || y > (double)g->ny) return APRL_OK;
  if (binomial3 ? (x <= -2. || x >= (double)g->nx + 2.) : (x < 0. || x > (double)g->nx))
    return APRL_OK;
  const long long ix = (long long)floor(x);
  const size_t j = (size_t)floor(y);
  const double fx = x - ix, fy = y - j, scale = p->q * (1. / (g->dx * g->dy * g->dz));
  double wx[4] = {1. - fx, fx, 0., 0.};
  if (binomial3) node_weights(fx, wx);
  const unsigned n_x = binomial3 ? 4 : 2;
  const long long first = ix - (binomial3 ? 1 : 0);
  for (unsigned b = 0; b < 2; ++b)
    for (unsigned a = 0; a < n_x; ++a) {
      const long long i = first + a;
      if (i >= 0 && i <= (long long)g->nx && j + b <= g->ny)
        rho[(j + b) * (g->nx + 1) + (size_t)i] += scale * wx[a] * (b ? fy : 1. - fy) * wz;
    }
  return APRL_OK;
}

/* Simulation::completeMovingInletLayer (src/simulation_moving_window.cpp:312-318)
 * with ChargeMatchedInlet::complete (src/charge_matched_inlet.h:55-71): the
 * stored particles and the pending ones due within 8 steps (visitNear), then
 * Ez of the inserted layer from the discrete Gauss law, in long double. */
static aprl_status inlet_charge_match(oracle_run* r) {
  const aprl_run_config* g = &r->cfg;
  const double origin[3] = {g->reference_origin[0], g->reference_origin[1],
                            fma((double)r->offset, g->dz, g->reference_origin[2])};
  double* rho = (double*)calloc((g->nx + 1) * (g->ny + 1), sizeof(double));
  aprl_status s = APRL_OK;
  for (size_t n = 0; n < r->np && s == APRL_OK; ++n)
    s = charge_match_particle(r, origin, &r->p[n], rho);
  const pending_t* q = &r->pending;
  if (s == APRL_OK && q->extracted) {
    const uint64_t step = r->step, room = q->maximum_step - step;
    const uint64_t until = step + (8 < room ? 8 : room);
    const size_t end = q->offsets[until - q->initial_step + 1];
    for (size_t n = q->cursor; n < end && s == APRL_OK; ++n) {
      particle_t p = q->p[q->order[n]];
      p.pos[2] = repeat_held_addition(p.pos[2], held_increment(r, &p), step - q->initial_step);
      s = charge_match_particle(r, origin, &p, rho);
    }
  }
  if (s != APRL_OK) {
    free(rho);
    return s;
  }
  comp_t *ex = &r->f[0], *ey = &r->f[1], *ez = &r->f[2];
  for (size_t j = g->cpml_cells_y + 1; j < g->ny - g->cpml_cells_y; ++j)
    for (size_t i = g->cpml_cells_x + 1; i < g->nx - g->cpml_cells_x; ++i) {
      const long double divxy = ((long double)AT(ex, i, j, 1) - AT(ex, i - 1, j, 1)) / g->dx +
                                ((long double)AT(ey, i, j, 1) - AT(ey, i, j - 1, 1)) / g->dy;
      const long double q_node = rho[j * (g->nx + 1) + i], retained = AT(ez, i, j, 1);
      const double value = (double)(retained + g->dz * (divxy - q_node / SI_EPSILON0));
      if (!isfinite(value)) {
        free(rho);
        return fail(APRL_ERR_RUNTIME, "Nonfinite charge-matched inlet field");
      }
      AT(ez, i, j, 0) = value;
    }
  free(rho);
  return APRL_OK;
}

/* Frozen source support of the pending particles due within 8 steps
 * (visitNear + depositFrozenSourceSupport, src/simulation.cpp:4170-4172). */
static aprl_status pending_support(oracle_run* r) {
  const pending_t* q = &r->pending;
  if (!q->extracted) return APRL_OK;
  const uint64_t step = r->step;
  const uint64_t room = q->maximum_step - step;
  const uint64_t until = step + (8 < room ? 8 : room);
  const size_t end = q->offsets[until - q->initial_step + 1];
  for (size_t n = q->cursor; n < end; ++n) {
    particle_t p = q->p[q->order[n]];
    p.pos[2] = repeat_held_addition(p.pos[2], held_increment(r, &p), step - q->initial_step);
    double stop[3] = {p.pos[0], p.pos[1], p.pos[2]};
    stop[2] += SI_C * r->cfg.dt * p.beta;
    aprl_status s = deposit_current(r, p.pos, stop, p.q);
    if (s != APRL_OK) return s;
  }
  return APRL_OK;
}

/* processActiveSegment at one rank (src/simulation.cpp:4555-4917), with the
 * held-activation kink (src/simulation.cpp:4684-4756); `cached` holds the
 * diagnostic boundary hits when the segment has no kink. */
typedef struct {
  boundary_hit cpml_hit, outer_hit;
  int enters, exits;
} segment_hits;

static aprl_status process_active_segment(oracle_run* r, const cpml_region* reg,
                                          particle_t particle, double seg_start[3],
                                          double seg_start_fraction, const double* kink,
                                          double kink_fraction, const segment_hits* cached) {
  const double crossing_tolerance = 64.0 * DBL_EPSILON;
  aprl_status s;
  if (kink) {
    boundary_hit ch, oh;
    int e1 = 0, e2 = 0;
    s = cpml_first_entry(r, reg, seg_start, kink, &ch, &e1);
    if (s != APRL_OK) return s;
    s = outer_first_exit(r, seg_start, kink, &oh, &e2);
    if (s != APRL_OK) return s;
    if (e1 || e2)
      return fail(APRL_ERR_RUNTIME,
                  "Held-transverse activation crossed a particle boundary during the frozen part of a field step");
    s = deposit_segment(r, seg_start, kink, particle.q);
    if (s != APRL_OK) return s;
    for (int a = 0; a < 3; ++a) seg_start[a] = kink[a];
    seg_start_fraction = kink_fraction;
  }
  segment_hits computed;
  if (!cached) {
    s = moving_window_entry(r, reg, seg_start, particle.pos, seg_start_fraction,
                            &computed.cpml_hit, &computed.enters);
    if (s != APRL_OK) return s;
    s = outer_first_exit(r, seg_start, particle.pos, &computed.outer_hit, &computed.exits);
    if (s != APRL_OK) return s;
    cached = &computed;
  }
  int action = 0;
  double local_end = 1.0, seg_end[3] = {particle.pos[0], particle.pos[1], particle.pos[2]};
  boundary_hit selected;
  if (cached->enters &&
      (!cached->exits || cached->cpml_hit.fraction <= cached->outer_hit.fraction + crossing_tolerance)) {
    action = 1;
    selected = cached->cpml_hit;
  } else if (cached->exits) {
    action = 2;
    selected = cached->outer_hit;
  }
  if (action) {
    local_end = selected.fraction;
    for (int a = 0; a < 3; ++a) seg_end[a] = selected.position[a];
  }
  s = deposit_segment(r, seg_start, seg_end, particle.q);
  if (s != APRL_OK) return s;
  const double global_end = seg_start_fraction + local_end * (1.0 - seg_start_fraction);
  if (action == 1) {
    if (selected.face == 5) {
      ++r->exits;
      r->exit_charge += particle.q;
    } else {
      ++r->cpml_entries[selected.face];
      r->cpml_entry_charge[selected.face] += particle.q;
    }
    carrier_t c;
    for (int a = 0; a < 3; ++a) c.pos[a] = particle.pos[a];
    const double gamma = gamma_u(particle.u);
    for (int a = 0; a < 3; ++a) c.vel[a] = particle.u[a] * (SI_C / gamma);
    c.q = particle.q;
    c.w = 1.0;
    return process_carrier_segment(r, reg, c, selected.position, global_end);
  }
  if (action == 2) {
    ++r->direct_outer[selected.face];
    r->direct_outer_charge[selected.face] += particle.q;
    return APRL_OK;
  }
  push_retained(r, &particle);
  return APRL_OK;
}

/* pushDepositAndMigrate at one rank (src/simulation.cpp:4167-5368): frozen
 * source support of the pending queue, CPML carriers, then every particle:
 * prepareParticle (held advance, activation crossing, coupled push) and the
 * serial deposit / boundary pass in list order. */
static aprl_status push_deposit(oracle_run* r) {
  cpml_region reg;
  make_cpml_region(r, &reg);
  r->nretained = 0;
  r->nrcarrier = 0;
  aprl_status s = pending_support(r);
  if (s != APRL_OK) return s;
  for (size_t n = 0; n < r->nc; ++n) {
    carrier_t c = r->c[n];
    const double start[3] = {c.pos[0], c.pos[1], c.pos[2]};
    for (int a = 0; a < 3; ++a) c.pos[a] += r->cfg.dt * c.vel[a];
    s = process_carrier_segment(r, &reg, c, start, 0.0);
    if (s != APRL_OK) return s;
  }
  const double t = r->time, dt = r->cfg.dt;
  for (size_t n = 0; n < r->np; ++n) {
    const particle_t original = r->p[n];
    particle_t particle = original;
    double start[3] = {original.pos[0], original.pos[1], original.pos[2]};
    if (start[2] < r->origin[2] && !particle.frozen)
      return fail(APRL_ERR_RUNTIME,
                  "An active particle is upstream of the moving window; the inlet guard did not contain its release event");
    /* prepareParticle (src/simulation.cpp:4919-5035), holdTransverse. */
    particle_t active_start = particle;
    double active_start_time = t;
    int has_active = !particle.frozen;
    if (particle.frozen) {
      const double beta_held = particle.beta;
      const double start_lab_z = lab_z_from_box_zt(&r->cfg, start[2], t);
      particle.pos[2] += SI_C * dt * beta_held;
      const double end_lab_z = lab_z_from_box_zt(&r->cfg, particle.pos[2], t + dt);
      if (end_lab_z >= r->cfg.activation_plane_lab_z) {
        if (start[2] < r->origin[2])
          return fail(APRL_ERR_RUNTIME,
                      "A pending upstream held particle would release before a complete in-window step");
        const double plane = r->cfg.activation_plane_lab_z;
        const double crossing = start_lab_z >= plane
                                    ? 0.0
                                    : fmax(0.0, fmin(1.0, (plane - start_lab_z) / (end_lab_z - start_lab_z)));
        for (int a = 0; a < 3; ++a) particle.pos[a] = start[a];
        particle.pos[2] += SI_C * crossing * dt * beta_held;
        particle.frozen = 0;
        has_active = 1;
        active_start = particle;
        active_start_time = t + crossing * dt;
        const double remaining = (1.0 - crossing) * dt;
        if (remaining > 0.0) {
          s = coupling_push(r, &particle, &r->slot[n], active_start_time, remaining);
          if (s != APRL_OK) return s;
        }
      }
    } else {
      s = coupling_push(r, &particle, &r->slot[n], t, dt);
      if (s != APRL_OK) return s;
    }
    if (original.frozen && has_active) ++r->activations;
    /* deposit and boundary pass (src/simulation.cpp:5083-5368) */
    double seg_start_fraction = 0.0;
    if (start[2] < r->origin[2]) {
      if (!original.frozen || !particle.frozen || has_active)
        return fail(APRL_ERR_RUNTIME,
                    "Moving-window upstream admission requires an unreleased held particle on rank zero");
      if (particle.pos[2] < r->origin[2]) {
        s = deposit_current(r, start, particle.pos, particle.q);
        if (s != APRL_OK) return s;
        push_retained(r, &particle);
        continue;
      }
      const double fraction = (r->origin[2] - start[2]) / (particle.pos[2] - start[2]);
      if (!(fraction >= 0.0 && fraction <= 1.0) || !isfinite(fraction))
        return fail(APRL_ERR_RUNTIME, "Invalid moving-window admission fraction");
      double clipped[3];
      for (int a = 0; a < 3; ++a) clipped[a] = start[a] + fraction * (particle.pos[a] - start[a]);
      clipped[2] = r->origin[2];
      seg_start_fraction = fraction;
      s = deposit_current(r, original.pos, clipped, particle.q);
      if (s != APRL_OK) return s;
      for (int a = 0; a < 3; ++a) start[a] = clipped[a];
    }
    const int has_kink = original.frozen && has_active && active_start_time > t &&
                         active_start_time < t + dt;
    const double kink_fraction = (active_start_time - t) / dt;
    if (has_kink) {
      s = process_active_segment(r, &reg, particle, start, seg_start_fraction,
                                 active_start.pos, kink_fraction, NULL);
    } else {
      segment_hits hits;
      s = moving_window_entry(r, &reg, start, particle.pos, seg_start_fraction,
                              &hits.cpml_hit, &hits.enters);
      if (s != APRL_OK) return s;
      s = outer_first_exit(r, start, particle.pos, &hits.outer_hit, &hits.exits);
      if (s != APRL_OK) return s;
      s = process_active_segment(r, &reg, particle, start, seg_start_fraction, NULL, 0.0, &hits);
    }
    if (s != APRL_OK) return s;
  }
  /* particles_ <- retained, pmlCarriers_ <- retainedCarriers. */
  if (r->nretained > r->pcap) {
    r->pcap = r->nretained;
    r->p = (particle_t*)xrealloc(r->p, r->pcap * sizeof(particle_t));
  }
  memcpy(r->p, r->retained, r->nretained * sizeof(particle_t));
  r->np = r->nretained;
  if (r->nrcarrier > r->ccap) {
    r->ccap = r->nrcarrier;
    r->c = (carrier_t*)xrealloc(r->c, r->ccap * sizeof(carrier_t));
  }
  memcpy(r->c, r->rcarrier, r->nrcarrier * sizeof(carrier_t));
  r->nc = r->nrcarrier;
  return APRL_OK;
}

/* ConservativeSourceCoupling::localResidual (src/source_coupling.cpp:105-159). */
static aprl_status local_residual(oracle_run* r, double out[4]) {
  double force = 0., defect = 0., scale = 0., calls = 0.;
  for (size_t n = 0; n < r->nslot; ++n) {
    slot_t* q = &r->slot[n];
    if (!q->seen) continue;
    calls += 1;
    aprl_status s = gather_electric(r, q->first.pos, q->last.pos, q->next_e);
    if (s != APRL_OK) return s;
    s = gather_magnetic(r, q->first.pos, q->last.pos, q->next_b);
    if (s != APRL_OK) return s;
    q->next_ready = 1;
    double de[3], db[3];
    for (int a = 0; a < 3; ++a) {
      de[a] = q->next_e[a] - q->used_e[a];
      db[a] = q->next_b[a] - q->used_b[a];
    }
    force = fmax(force, fabs(q->first.q / q->first.m) * q->dt / SI_C *
                            (sqrt(dot3(de, de)) + SI_C * sqrt(dot3(db, db))));
    defect += fabsl(charge_work(q->first.q, de, q->first.pos, q->last.pos));
    scale += q->abs_grid_work;
    scale += fabsl(charge_work(q->first.q, q->next_e, q->first.pos, q->last.pos));
  }
  out[0] = force;
  out[1] = defect;
  out[2] = scale;
  out[3] = calls;
  return APRL_OK;
}

/* TransverseReferenceCurrent at one rank: the target points of points()
 * (src/transverse_reference_current.cpp:19-28) in the same order, the
 * prepared value curl_z(B_ref)/mu0 per reference plane (prepare, :46-63)
 * and, each trial, Jz += the plane lerp at offset + k - beta*(step+1)
 * (apply, :104-118). */
static aprl_status surface_prepare(oracle_run* r) {
  surface_current_t* s = &r->surface;
  if (s->ready) return APRL_OK;
  const aprl_run_config* g = &r->cfg;
  if (!g->cpml_cells_x || !g->cpml_cells_y)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Reference surface current requires transverse-only CPML");
  if (!r->ref_set[3] || !r->ref_set[4])
    return fail(APRL_ERR_INVALID_ARGUMENT, "Missing moving-window inlet reference component");
  const size_t x0 = g->cpml_cells_x, x1 = g->nx - g->cpml_cells_x;
  const size_t y0 = g->cpml_cells_y, y1 = g->ny - g->cpml_cells_y;
  const size_t count = 2 * (x1 - x0 + 1) + 2 * (y1 - y0 - 1);
  s->i = (size_t*)malloc(count * sizeof(size_t));
  s->j = (size_t*)malloc(count * sizeof(size_t));
  const size_t planes = g->reference_nz;
  s->table = (double*)malloc((planes ? planes : 1) * count * sizeof(double));
  size_t p = 0;
  for (size_t i = x0; i <= x1; ++i) {
    s->i[p] = i; s->j[p] = y0; ++p;
    s->i[p] = i; s->j[p] = y1; ++p;
  }
  for (size_t j = y0 + 1; j < y1; ++j) {
    s->i[p] = x0; s->j[p] = j; ++p;
    s->i[p] = x1; s->j[p] = j; ++p;
  }
  s->count = count;
  const comp_t* bx = &r->ref[3];
  const comp_t* by = &r->ref[4];
  for (size_t k = 0; k < planes; ++k)
    for (size_t q = 0; q < count; ++q) {
      const size_t i = s->i[q], j = s->j[q];
      const double v = ((AT(by, i, j, k) - AT(by, i - 1, j, k)) / g->dx -
                        (AT(bx, i, j, k) - AT(bx, i, j - 1, k)) / g->dy) / SI_MU0;
      if (!isfinite(v)) return fail(APRL_ERR_RUNTIME, "Nonfinite equivalent boundary current");
      s->table[k * count + q] = v;
    }
  s->ready = 1;
  return APRL_OK;
}

static aprl_status surface_apply(oracle_run* r) {
  if (!r->cfg.reference_surface_current) return APRL_OK;
  aprl_status st = surface_prepare(r);
  if (st != APRL_OK) return st;
  surface_current_t* s = &r->surface;
  const size_t planes = r->cfg.reference_nz;
  comp_t* jz = &r->f[8];
  for (size_t k = 0; k < r->cfg.nz; ++k) {
    const double z = (double)r->offset + (double)k - r->cfg.translation_beta * (double)(r->step + 1);
    if (!isfinite(z) || z < 0. || z > (double)planes - 1.)
      return fail(APRL_ERR_OUT_OF_RANGE, "Reference surface-current query outside domain");
    const size_t lo = (size_t)floor(z);
    const size_t hi = lo + 1 < planes ? lo + 1 : planes - 1;
    const double fraction = z - (double)lo;
    const double* a = s->table + lo * s->count;
    const double* b = s->table + hi * s->count;
    for (size_t q = 0; q < s->count; ++q) {
      const double value = fraction == 0. ? a[q] : (1. - fraction) * a[q] + fraction * b[q];
      AT(jz, s->i[q], s->j[q], k) += value;
    }
  }
  return APRL_OK;
}

aprl_status oracle_run_coupling_trial(oracle_run* r, double residual[4]) {
  if (r->stage != 2 && r->stage != 3)
    return fail(APRL_ERR_RUNTIME, "Coupling trial requires a previewed electric field");
  /* Loop body of solveConservativeSourceStep (src/simulation_source_coupling.cpp:43-48). */
  if (r->trials_this_step) apply_current_source(r, 1.);
  clear_current(r);
  restore_state(r);
  for (size_t n = 0; n < r->nslot; ++n) r->slot[n].seen = 0; /* beginTrial */
  r->replay = 0;
  aprl_status s = push_deposit(r);
  if (s != APRL_OK) return s;
  s = surface_apply(r);
  if (s != APRL_OK) return s;
  apply_current_source(r, -1.);
  s = local_residual(r, residual);
  if (s != APRL_OK) return s;
  ++r->trials_this_step;
  r->stage = 3;
  return APRL_OK;
}

aprl_status oracle_run_commit_electric(oracle_run* r) {
  if (r->stage != 3) return fail(APRL_ERR_RUNTIME, "Commit requires a completed coupling trial");
  /* Remove the trial current, replay against E^n, then commit
   * (src/simulation_source_coupling.cpp:58-65). */
  apply_current_source(r, 1.);
  clear_current(r);
  restore_state(r);
  for (int a = 0; a < 3; ++a) {
    double* t = r->f[a].v;
    r->f[a].v = r->old[a].v;
    r->old[a].v = t;
  }
  r->replay = 1;
  aprl_status s = push_deposit(r);
  r->replay = 0;
  if (s != APRL_OK) return s;
  /* applyMovingTransverseReferenceCurrent before the commit (src/simulation.cpp:548-549). */
  s = surface_apply(r);
  if (s != APRL_OK) return s;
  for (int a = 0; a < 3; ++a) {
    double* t = r->f[a].v;
    r->f[a].v = r->old[a].v;
    r->old[a].v = t;
  }
  if (!r->preview_present) return fail(APRL_ERR_RUNTIME, "Missing electric boundary preview");
  for (size_t n = 0; n < r->ndelta; ++n)
    r->f[r->delta[n].axis].v[r->delta[n].index] -= r->delta[n].value;
  r->preview_present = 0;
  apply_current_source(r, -1.);
  cpml_after_electric(r);
  /* The measured inlet overwrite (src/moving_window_fields.cpp:265-290). */
  long double energy_before = 0., power_before[6], power_after[6];
  if (r->ledger) {
    energy_before = plane_energy(r, 0);
    boundary_power(r, 1, power_before);
  }
  s = inlet_overwrite(r);
  if (s != APRL_OK) return s;
  if (r->ledger) {
    r->overwrite_energy += plane_energy(r, 0) - energy_before;
    boundary_power(r, 1, power_after);
    for (int f = 0; f < 6; ++f) r->overwrite_power_delta[f] = power_after[f] - power_before[f];
    ++r->overwrite_events;
  }
  r->stage = 4;
  return APRL_OK;
}

aprl_status oracle_run_shift(oracle_run* r) {
  if (r->stage != 4) return fail(APRL_ERR_RUNTIME, "Moving-window requires one left shift after each complete step");
  const aprl_run_config* g = &r->cfg;
  /* finishEnergyLedgerStep (src/moving_window_fields.cpp:425-437), then the
   * energy of the plane the shift drops (src/moving_window_fields.cpp:446-450). */
  long double removed = 0.;
  if (r->ledger) {
    long double end_power[6];
    boundary_power(r, 0, end_power);
    const long double half_dt = .5L * (long double)g->dt;
    for (int f = 0; f < 6; ++f)
      r->outward_energy[f] += half_dt * (r->start_power[f] + end_power[f] -
                                         r->overwrite_power_delta[f]);
    ++r->flux_steps;
    removed = plane_energy(r, g->nz - 1);
  }
  r->time += g->dt;
  r->step += 1;
  r->offset = g->initial_offset - (int64_t)r->step;
  /* MovingWindowFields::Impl::shift (src/moving_window_fields.cpp:439-518). */
  for (unsigned a = 0; a < 6; ++a) {
    comp_t* c = &r->f[a];
    const size_t plane = c->nx * c->ny;
    double* fresh = (double*)malloc(plane * sizeof(double));
    for (size_t j = 0; j < c->ny; ++j)
      for (size_t i = 0; i < c->nx; ++i) {
        aprl_status s = reference_value(r, a, i, j, r->offset, r->step, &fresh[j * c->nx + i]);
        if (s != APRL_OK) {
          free(fresh);
          return s;
        }
      }
    memmove(c->v + plane, c->v, (c->nz - 1) * plane * sizeof(double));
    memcpy(c->v, fresh, plane * sizeof(double));
    free(fresh);
  }
  clear_current(r);
  for (unsigned h = 0; h < 12; ++h) {
    cpml_term* t = history_term(r, h);
    if (t->length == 0) continue;
    const size_t layers = t->dims[2];
    const size_t row = t->dims[t->axis == 0 ? 1 : 0];
    const size_t slots = t->length / (layers * row);
    for (size_t slot = 0; slot < slots; ++slot) {
      double* base = t->history + slot * layers * row;
      memmove(base + row, base, (layers - 1) * row * sizeof(double));
      memset(base, 0, row * sizeof(double));
    }
  }
  if (g->inlet_charge_match) {
    aprl_status s = inlet_charge_match(r);
    if (s != APRL_OK) return s;
  }
  /* Remap energy of the shift at one rank (src/moving_window_fields.cpp:500-515). */
  if (r->ledger) {
    const long double inserted = plane_energy(r, 0);
    r->remap_energy += inserted - removed;
    r->inserted_energy += inserted;
    r->cropped_energy += removed;
    ++r->remap_steps;
  }
  /* finishMovingWindowStep particle part (src/simulation_moving_window.cpp:352-371). */
  r->origin[2] = fma((double)r->offset, g->dz, g->reference_origin[2]);
  for (size_t n = 0; n < r->np; ++n)
    if (r->p[n].pos[2] < r->origin[2] && !r->p[n].frozen)
      return fail(APRL_ERR_RUNTIME, "Active particle fell behind moving inlet");
  const double upper = fma((double)g->nz, g->dz, r->origin[2]);
  size_t kept = 0;
  for (size_t n = 0; n < r->nc; ++n) {
    const carrier_t* c = &r->c[n];
    if (c->pos[2] >= upper) {
      ++r->cropped_carriers;
      r->cropped_charge += c->q * c->w;
    } else if (c->pos[2] < r->origin[2]) {
      return fail(APRL_ERR_RUNTIME, "Current carrier fell behind moving inlet");
    } else {
      r->c[kept++] = *c;
    }
  }
  r->nc = kept;
  r->stage = 0;
  return APRL_OK;
}

/* Simulation::solve loop body (src/simulation.cpp:493-613) with
 * solveConservativeSourceStep (src/simulation_source_coupling.cpp:16-60). */
aprl_status oracle_run_step(oracle_run* r, uint32_t steps) {
  for (uint32_t n = 0; n < steps; ++n) {
    aprl_status s = oracle_run_advance_magnetic(r);
    if (s != APRL_OK) return s;
    s = oracle_run_preview_electric(r);
    if (s != APRL_OK) return s;
    int converged = 0;
    unsigned iterations = 0;
    double force = 0., work = 0.;
    double history[2 * 64];
    for (unsigned t = 0; t < r->cfg.max_trials; ++t) {
      double res[4];
      s = oracle_run_coupling_trial(r, res);
      if (s != APRL_OK) return s;
      force = res[0];
      work = res[3] == 0. ? 0. : (res[2] > 0. ? res[1] / res[2] : res[1]);
      iterations = t + 1;
      if (t < 64) {
        history[2 * t] = force;
        history[2 * t + 1] = work;
      }
      if (iterations >= (res[3] > 0. ? 2u : 1u) && force < r->cfg.force_tolerance &&
          work < r->cfg.work_tolerance) {
        converged = 1;
        break;
      }
    }
    if (!converged) {
      /* The message of src/simulation_source_coupling.cpp:54, with the
       * per-trial force/work history. */
      int at = snprintf(g_error, sizeof g_error,
                        "Conservative source coupling failed at step %llu: force=%g work=%g "
                        "iterations=%u history(force/work)=",
                        (unsigned long long)(r->step + 1), force, work, iterations);
      for (unsigned t = 0; t < iterations && t < 64 && at > 0 && at < (int)sizeof g_error; ++t)
        at += snprintf(g_error + at, sizeof g_error - (size_t)at, " %g/%g", history[2 * t],
                       history[2 * t + 1]);
      return APRL_ERR_NOT_CONVERGED;
    }
    r->last_iterations = iterations;
    if (iterations > r->max_iterations) r->max_iterations = iterations;
    r->total_iterations += iterations;
    r->last_force = force;
    r->last_work = work;
    s = oracle_run_commit_electric(r);
    if (s != APRL_OK) return s;
    s = oracle_run_shift(r);
    if (s != APRL_OK) return s;
  }
  return APRL_OK;
}

aprl_status oracle_run_get_stats(const oracle_run* r, aprl_step_stats* st) {
  memset(st, 0, sizeof *st);
  st->step = r->step;
  st->iterations = r->last_iterations;
  st->max_iterations = r->max_iterations;
  st->total_iterations = r->total_iterations;
  st->force = r->last_force;
  st->work = r->last_work;
  st->particles = r->np;
  st->carriers = r->nc;
  st->exits = r->exits;
  st->exit_charge = r->exit_charge;
  for (int f = 0; f < 6; ++f) {
    st->cpml_entries[f] = r->cpml_entries[f];
    st->cpml_entry_charge[f] = r->cpml_entry_charge[f];
    st->carrier_outer[f] = r->carrier_outer[f];
    st->carrier_outer_charge[f] = r->carrier_outer_charge[f];
  }
  st->cropped_carriers = r->cropped_carriers;
  st->cropped_charge = r->cropped_charge;
  st->window_offset = r->offset;
  st->origin_z = r->origin[2];
  st->time_box = r->time;
  st->pending = r->pending.extracted ? r->pending.n - r->pending.cursor : 0;
  st->admitted = r->admitted;
  st->activations = r->activations;
  for (size_t i = 0; i < r->np; ++i) st->held += r->p[i].frozen ? 1 : 0;
  return APRL_OK;
}

aprl_status oracle_run_get_slot_fields(oracle_run* r, size_t capacity, double* used_e,
                                       double* used_b, double* next_e, double* next_b,
                                       size_t* count) {
  *count = r->nslot;
  if (!used_e && !used_b && !next_e && !next_b) return APRL_OK;
  if (capacity < r->nslot) return fail(APRL_ERR_INVALID_ARGUMENT, "Slot buffer too small");
  for (size_t n = 0; n < r->nslot; ++n)
    for (int a = 0; a < 3; ++a) {
      if (used_e) used_e[3 * n + a] = r->slot[n].used_e[a];
      if (used_b) used_b[3 * n + a] = r->slot[n].used_b[a];
      if (next_e) next_e[3 * n + a] = r->slot[n].next_e[a];
      if (next_b) next_b[3 * n + a] = r->slot[n].next_b[a];
    }
  *count = r->nslot;
  return APRL_OK;
}

/* ---- detector field plane (src/lab_detectors.cpp:39-99, 2426-2490,
 *      2836-2905) ----------------------------------------------------------- */
typedef struct {
  size_t lower;
  double fraction;
} interp_axis;

static interp_axis interpolation_axis(double lattice, size_t size) {
  interp_axis r;
  if (lattice <= 0.0) {
    r.lower = 0;
    r.fraction = 0.0;
  } else if (lattice >= (double)(size - 1)) {
    r.lower = size - 2;
    r.fraction = 1.0;
  } else {
    r.lower = (size_t)floor(lattice);
    r.fraction = lattice - (double)r.lower;
  }
  return r;
}

static double sample_detector_component(const comp_t* c, double lx, double ly,
                                        const interp_axis* z) {
  const interp_axis x = interpolation_axis(lx, c->nx), y = interpolation_axis(ly, c->ny);
  double value = 0.0;
  for (unsigned cz = 0; cz < 2; ++cz) {
    const double wz = cz ? z->fraction : 1.0 - z->fraction;
    if (wz == 0.0) continue;
    const size_t k = z->lower + cz;
    for (unsigned b = 0; b < 2; ++b)
      for (unsigned a = 0; a < 2; ++a) {
        const double wx = a ? x.fraction : 1.0 - x.fraction;
        const double wy = b ? y.fraction : 1.0 - y.fraction;
        value += wx * wy * wz * AT(c, x.lower + a, y.lower + b, k);
      }
  }
  return value;
}

aprl_status oracle_run_sample_field_plane(oracle_run* r, double plane_lab_z, double* out,
                                          size_t count, int* inside) {
  const aprl_run_config* g = &r->cfg;
  if (count != 6 * g->nx * g->ny) return fail(APRL_ERR_INVALID_ARGUMENT, "Detector buffer size mismatch");
  const double box_z = box_z_from_lab_z_and_box_t(g, plane_lab_z, r->time);
  const double coordinate = (box_z - r->origin[2]) / g->dz;
  /* ownerRank (src/simulation.cpp:4068-4085): upstream of the window maps
   * to rank 0; beyond the upper face nothing samples. */
  const double tolerance = 64.0 * DBL_EPSILON * fmax(1.0, fabs(coordinate));
  if (!(box_z < r->origin[2]) && coordinate > (double)g->nz + tolerance) {
    *inside = 0;
    return APRL_OK;
  }
  *inside = 1;
  const interp_axis vertex_z = interpolation_axis(coordinate, g->nz + 1);
  const interp_axis half_z = interpolation_axis(coordinate - 0.5, g->nz);
  for (size_t j = 0; j < g->ny; ++j) {
    const double py = g->reference_origin[1] + ((double)j + 0.5) * g->dy;
    const double y = (py - g->reference_origin[1]) / g->dy;
    for (size_t i = 0; i < g->nx; ++i) {
      const double px = g->reference_origin[0] + ((double)i + 0.5) * g->dx;
      const double x = (px - g->reference_origin[0]) / g->dx;
      double eb[3], bb[3], el[3], bl[3];
      eb[0] = sample_detector_component(&r->f[0], x - 0.5, y, &vertex_z);
      eb[1] = sample_detector_component(&r->f[1], x, y - 0.5, &vertex_z);
      eb[2] = sample_detector_component(&r->f[2], x, y, &half_z);
      bb[0] = sample_detector_component(&r->f[3], x, y - 0.5, &half_z);
      bb[1] = sample_detector_component(&r->f[4], x - 0.5, y, &half_z);
      bb[2] = sample_detector_component(&r->f[5], x - 0.5, y - 0.5, &vertex_z);
      fields_box_to_lab(g, eb, bb, el, bl);
      double* o = out + 6 * (j * g->nx + i);
      for (int a = 0; a < 3; ++a) {
        o[a] = el[a];
        o[3 + a] = bl[a];
      }
    }
  }
  return APRL_OK;
}

/* ---- initial self-field ------------------------------------------------- */
/* EBGaussFieldInitializer::initialize (src/eb_initial_field.cpp:829-1095)
 * at one rank, restated with its long double reductions and loop orders.
 * Scalars live on the node lattice of the Poisson geometry (nx+1+2 pad,
 * ny+1+2 pad) with nz+2 planes: plane p holds node k = p-1, planes 0 and
 * nz+1 are the zero ghosts of a single rank (ScalarSlab,
 * src/eb_initial_field.cpp:30-82). */
typedef struct {
  size_t nx, ny, planes;
  double* v;
} slab_t;

#define SAT(s, i, j, p) ((s)->v[((size_t)(p) * (s)->ny + (j)) * (s)->nx + (i)])

typedef struct {
  size_t lower[3], upper[3];
} sdomain_t;

static int sf_interior(size_t i, size_t j, size_t k, const sdomain_t* d) {
  return i > d->lower[0] && i < d->upper[0] && j > d->lower[1] && j < d->upper[1] &&
         k > d->lower[2] && k < d->upper[2];
}

/* positiveLightFrontComponent / properVelocityFromPositiveLightFront /
 * heldLongitudinalBetaZ (src/boostframe.cpp:89-167). */
static double sf_positive(const double u[3]) {
  const double gamma = gamma_u(u);
  const double tms = fma(u[0], u[0], fma(u[1], u[1], 1.0));
  if (u[2] >= 0.0) return gamma + u[2];
  return tms / (gamma - u[2]);
}
static void sf_from_positive(const double in[3], double positive, double out[3]) {
  const double tms = fma(in[0], in[0], fma(in[1], in[1], 1.0));
  const double negative = tms / positive;
  out[0] = in[0];
  out[1] = in[1];
  out[2] = 0.5 * (positive - negative);
}
static double sf_held_beta_z(const aprl_run_config* g, const double u[3]) {
  const double rapidity = g->boost_gamma + g->boost_gamma_beta;
  double lab[3], lon[3] = {0.0, 0.0, 0.0}, box[3];
  sf_from_positive(u, sf_positive(u) * rapidity, lab);
  lon[2] = lab[2];
  sf_from_positive(lon, sf_positive(lon) / rapidity, box);
  return box[2] / hypot(1.0, box[2]);
}

/* ChargeConservingCurrentDepositor::depositCharge (src/eb_deposition.cpp:168-193)
 * into an (nx+1, ny+1, nz+1) vertex array embedded at offset `pad` of a
 * lattice `lx` x `ly` wide. */
static aprl_status sf_deposit(const oracle_run* r, double* rho, size_t lx, size_t ly, size_t pad) {
  const aprl_run_config* g = &r->cfg;
  const double extent[3] = {(double)g->nx * g->dx, (double)g->ny * g->dy, (double)g->nz * g->dz};
  const double h[3] = {g->dx, g->dy, g->dz};
  const size_t cells[3] = {g->nx, g->ny, g->nz};
  const double inverse_volume = 1.0 / (g->dx * g->dy * g->dz);
  for (size_t n = 0; n < r->np; ++n) {
    const particle_t* p = &r->p[n];
    size_t c[3];
    double f[3];
    for (int a = 0; a < 3; ++a) {
      const double relative = p->pos[a] - r->origin[a];
      const double tol = 64.0 * DBL_EPSILON * fmax(1.0, fmax(fabs(r->origin[a]), extent[a]));
      if (!isfinite(p->pos[a]) || relative < -tol || relative > extent[a] + tol)
        return fail(APRL_ERR_OUT_OF_RANGE, "Particle trajectory endpoint is outside the E/B domain");
      const double x = fmax(0.0, fmin((double)cells[a], (p->pos[a] - r->origin[a]) / h[a]));
      if (x <= 0.0) c[a] = 0;
      else if (x >= (double)cells[a]) c[a] = cells[a] - 1;
      else c[a] = (size_t)floor(x);
      f[a] = fmax(0.0, fmin(1.0, x - (double)c[a]));
    }
    for (unsigned cz = 0; cz < 2; ++cz)
      for (unsigned b = 0; b < 2; ++b)
        for (unsigned a = 0; a < 2; ++a) {
          const double sa = a ? f[0] : 1.0 - f[0];
          const double sb = b ? f[1] : 1.0 - f[1];
          const double sc = cz ? f[2] : 1.0 - f[2];
          rho[((c[2] + cz) * ly + (c[1] + b + pad)) * lx + (c[0] + a + pad)] +=
              p->q * inverse_volume * sa * sb * sc;
        }
  }
  return APRL_OK;
}

/* The moving window's shaped reference source, BlockedCowanReference::
 * depositQuintic (src/blocked_cowan_reference.cpp:559-592): per particle
 * x = (p - origin)/h, the transverse x weights (src/transverse_source_shape.h:
 * 8-10, nodes floor(x)-1 .. floor(x)+2) for linear-binomial3 or linear ones,
 * linear y weights and the run shape's node basis in z; each nonzero
 * contribution q/(dx dy dz) wx wy wz must land on an interior node of the
 * zero-potential box `d`.  The reference adds a node's contributions in the
 * order of its z-block source buckets, this restatement in particle order:
 * the same terms, summed in another order. */
static aprl_status sf_shaped_deposit(const oracle_run* r, double* rho, size_t lx, size_t ly,
                                     const sdomain_t* d) {
  const aprl_run_config* g = &r->cfg;
  const int binomial = g->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
  for (size_t n = 0; n < r->np; ++n) {
    const particle_t* p = &r->p[n];
    if (!isfinite(p->q)) return fail(APRL_ERR_INVALID_ARGUMENT, "Nonfinite quintic reference charge");
    const double x = (p->pos[0] - r->origin[0]) / g->dx, y = (p->pos[1] - r->origin[1]) / g->dy,
                 z = (p->pos[2] - r->origin[2]) / g->dz;
    if (!isfinite(z)) return fail(APRL_ERR_INVALID_ARGUMENT, "Nonfinite quintic reference source");
    const long long ix = (long long)floor(x), iy = (long long)floor(y);
    const double fx = x - ix, fy = y - iy, scale = p->q / (g->dx * g->dy * g->dz);
    const basis_t weights = shape_basis(z, 0, g->shape);
    double wx[4] = {1. - fx, fx, 0., 0.};
    if (binomial) node_weights(fx, wx);
    const long long first_x = ix - (binomial ? 1 : 0);
    const unsigned count_x = binomial ? 4 : 2;
    for (unsigned c = 0; c < weights.count; ++c) {
      const long long k = weights.first + c;
      if (weights.v[c] == 0.) continue;
      for (unsigned j = 0; j < 2; ++j)
        for (unsigned i = 0; i < count_x; ++i) {
          const double value = scale * wx[i] * (j ? fy : 1. - fy) * weights.v[c];
          if (value == 0.) continue;
          const long long node_x = first_x + i, node_y = iy + j;
          if (k < 0 || node_x < 0 || node_y < 0 ||
              !sf_interior((size_t)node_x, (size_t)node_y, (size_t)k, d))
            return fail(APRL_ERR_INVALID_ARGUMENT,
                        "Reference charge support touches Dirichlet surface");
          rho[((size_t)k * ly + (size_t)node_y) * lx + (size_t)node_x] += value;
        }
    }
  }
  return APRL_OK;
}

static long double sf_dot(const slab_t* a, const slab_t* b, const sdomain_t* d, size_t nz) {
  long double local = 0.0L;
  for (size_t p = 1; p <= nz; ++p) {
    const size_t k = p - 1;
    if (k <= d->lower[2] || k >= d->upper[2]) continue;
    for (size_t j = d->lower[1] + 1; j < d->upper[1]; ++j)
      for (size_t i = d->lower[0] + 1; i < d->upper[0]; ++i)
        local += (long double)SAT(a, i, j, p) * (long double)SAT(b, i, j, p);
  }
  return local;
}

/* The CowanPoissonOperator stencil (src/eb_initial_field.cpp:246-316). */
static aprl_status sf_cowan_stencil(const oracle_run* r, double beta_z, double* translation,
                                    double stencil[3][3][3]) {
  const aprl_run_config* g = &r->cfg;
  const double velocity = beta_z * SI_C;
  *translation = velocity * velocity * SI_EPSILON0 * SI_MU0;
  const double spacing[3] = {g->dx, g->dy, g->dz};
  const double deltas[3] = {r->delta_yz, r->delta_zx, r->delta_xy};
  memset(stencil, 0, 27 * sizeof(double));
  for (unsigned axis = 0; axis < 3; ++axis) {
    const unsigned ta = (axis + 1) % 3, tb = (axis + 2) % 3;
    const double delta = deltas[axis];
    double minimum = INFINITY;
    for (int a = -1; a <= 1; a += 2)
      for (int b = -1; b <= 1; b += 2)
        minimum = fmin(minimum, r->alpha[axis] + 2.0 * r->beta[ta] * a + 2.0 * r->beta[tb] * b +
                                    4.0 * delta * a * b);
    if (axis == 2) minimum -= *translation;
    if (!(minimum > 64.0 * DBL_EPSILON))
      return fail(APRL_ERR_RUNTIME,
                  "Initial Cowan-Poisson operator fails the sufficient positive-definiteness "
                  "bound on axis %u: minimum smoothing symbol%s=%.12g; choose boost_gamma "
                  "closer to the bunch mean gamma or a grid aspect ratio with positive Cowan "
                  "symbols",
                  axis, axis == 2 ? " minus v^2*epsilon0*mu0" : "", minimum);
    const double inverse2 = 1.0 / (spacing[axis] * spacing[axis]);
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b) {
        const double weight =
            a == 0 ? (b == 0 ? r->alpha[axis] : r->beta[tb]) : (b == 0 ? r->beta[ta] : delta);
        int pt[3] = {1, 1, 1};
        pt[ta] += a;
        pt[tb] += b;
        stencil[pt[2]][pt[1]][pt[0]] += 2.0 * weight * inverse2;
        --pt[axis];
        stencil[pt[2]][pt[1]][pt[0]] -= weight * inverse2;
        pt[axis] += 2;
        stencil[pt[2]][pt[1]][pt[0]] -= weight * inverse2;
      }
  }
  const double tz = *translation / (g->dz * g->dz);
  stencil[1][1][1] -= 2.0 * tz;
  stencil[0][1][1] += tz;
  stencil[2][1][1] += tz;
  return APRL_OK;
}

/* cowanSmoothedPotential (src/eb_initial_field.cpp:344-382). */
static double sf_smoothed(const oracle_run* r, const slab_t* phi, unsigned axis, size_t i,
                          size_t j, size_t p) {
  const unsigned ta = (axis + 1) % 3, tb = (axis + 2) % 3;
  const double deltas[3] = {r->delta_yz, r->delta_zx, r->delta_xy};
  double value = r->alpha[axis] * SAT(phi, i, j, p);
  for (int sign = -1; sign <= 1; sign += 2) {
    size_t a[3] = {i, j, p}, b[3] = {i, j, p};
    if (sign < 0) {
      --a[ta];
      --b[tb];
    } else {
      ++a[ta];
      ++b[tb];
    }
    value += r->beta[ta] * SAT(phi, a[0], a[1], a[2]);
    value += r->beta[tb] * SAT(phi, b[0], b[1], b[2]);
  }
  for (int a = -1; a <= 1; a += 2)
    for (int b = -1; b <= 1; b += 2) {
      size_t pt[3] = {i, j, p};
      if (a < 0) --pt[ta]; else ++pt[ta];
      if (b < 0) --pt[tb]; else ++pt[tb];
      value += deltas[axis] * SAT(phi, pt[0], pt[1], pt[2]);
    }
  return value;
}

static void sf_free(slab_t* s, int n) {
  for (int q = 0; q < n; ++q) free(s[q].v);
}

aprl_status oracle_run_initialize_self_field(oracle_run* r, const aprl_self_field_config* cfg,
                                             aprl_self_field_report* rep) {
  const aprl_run_config* g = &r->cfg;
  memset(rep, 0, sizeof *rep);
  if (!(cfg->relative_tolerance > 0.0) || !(cfg->relative_tolerance < 1.0) ||
      !isfinite(cfg->relative_tolerance) || cfg->maximum_iterations == 0)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid initial Gauss-field convergence controls");
  if (!(cfg->maximum_mean_transverse_beta >= 0.0) || !(cfg->maximum_mean_transverse_beta < 1.0) ||
      !isfinite(cfg->maximum_mean_transverse_beta))
    return fail(APRL_ERR_INVALID_ARGUMENT, "Invalid initial self-field maximum mean transverse beta");
  if (cfg->model < 0 || cfg->model > 2)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Unknown initial self-field model");
  const int include = cfg->include_transverse_cpml_particles != 0;
  if (include && (cfg->guard_cells[0] < 2 || cfg->guard_cells[1] < 2))
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "Transverse CPML-source initialization requires at least two physical guard "
                "cells in x and y");
  if (cfg->source_shape != APRL_SOURCE_SHAPE_CIC && cfg->source_shape != APRL_SOURCE_SHAPE_RUN_SHAPE)
    return fail(APRL_ERR_INVALID_ARGUMENT, "Unknown initial self-field source shape");
  const int shaped = cfg->source_shape == APRL_SOURCE_SHAPE_RUN_SHAPE;
  if (shaped && include)
    return fail(APRL_ERR_INVALID_ARGUMENT,
                "The shaped reference source has no transverse CPML-source padding");
  const int cowan = cfg->model == APRL_SELF_FIELD_COWAN_RELATIVISTIC_POISSON;
  const int relativistic = cfg->model == APRL_SELF_FIELD_RELATIVISTIC_POISSON || cowan;
  const size_t pad = include ? 2 : 0;
  const size_t pnx = g->nx + 2 * pad, pny = g->ny + 2 * pad;
  const size_t cells[3] = {g->nx, g->ny, g->nz};
  const size_t pcells[3] = {pnx, pny, g->nz};
  sdomain_t domain, physical;
  for (int a = 0; a < 3; ++a) {
    if (2 * cfg->guard_cells[a] + 2 >= cells[a])
      return fail(APRL_ERR_INVALID_ARGUMENT,
                  "Initial static-field guard leaves fewer than two physical cells");
    physical.lower[a] = cfg->guard_cells[a];
    physical.upper[a] = cells[a] - cfg->guard_cells[a];
    domain.lower[a] = include && a < 2 ? 0 : cfg->guard_cells[a];
    domain.upper[a] = pcells[a] - domain.lower[a];
  }
  for (int a = 0; a < 6; ++a)
    memset(r->f[a].v, 0, r->f[a].nx * r->f[a].ny * r->f[a].nz * sizeof(double));

  /* meanVelocity (src/eb_initial_field.cpp:629-663) */
  long double mv[4] = {0.L, 0.L, 0.L, 0.L};
  for (size_t n = 0; n < r->np; ++n) {
    const particle_t* p = &r->p[n];
    const double gamma = gamma_u(p->u);
    const long double w = (long double)p->m;
    mv[0] += w;
    if (cfg->hold_transverse_until_activation)
      mv[3] += w * (long double)sf_held_beta_z(g, p->u);
    else
      for (int a = 0; a < 3; ++a) mv[a + 1] += w * (long double)(p->u[a] / gamma);
  }
  if (!(mv[0] > 0.0L))
    return fail(APRL_ERR_RUNTIME, "Initial relativistic-Poisson field requires positive represented mass");
  const double bx = (double)(mv[1] / mv[0]), by = (double)(mv[2] / mv[0]);
  const double beta_z = (double)(mv[3] / mv[0]);
  const double beta_t = hypot(bx, by);
  if (!isfinite(beta_z) || !isfinite(beta_t) || beta_t >= 1.0 || fabs(beta_z) >= 1.0)
    return fail(APRL_ERR_RUNTIME, "Initial particle mean velocity is not a finite subluminal vector");
  if (relativistic && beta_t > cfg->maximum_mean_transverse_beta)
    return fail(APRL_ERR_RUNTIME,
                "%s mean beta_box_transverse=%.12g exceeds "
                "initial_self_field.maximum_mean_transverse_beta=%.12g",
                cowan ? "cowan-relativistic-poisson" : "relativistic-poisson", beta_t,
                cfg->maximum_mean_transverse_beta);
  const double applied = relativistic ? beta_z : 0.0;
  const double longitudinal = fma(-applied, applied, 1.0);
  if (!cowan && !(longitudinal > 64.0 * DBL_EPSILON))
    return fail(APRL_ERR_RUNTIME,
                "Initial relativistic-Poisson operator is ill-conditioned because the bunch "
                "remains too relativistic in the simulation frame");
  double translation = 0.0, stencil[3][3][3];
  if (cowan) {
    aprl_status s = sf_cowan_stencil(r, applied, &translation, stencil);
    if (s != APRL_OK) return s;
  }
  rep->mean_beta_z = beta_z;
  rep->mean_beta_transverse = beta_t;
  rep->transverse_poisson_padding_cells = pad;
  for (int a = 0; a < 3; ++a) rep->static_field_guard_cells[a] = domain.lower[a];

  /* distributionResolution (src/eb_initial_field.cpp:693-741) */
  {
    long double m[7] = {0.L, 0.L, 0.L, 0.L, 0.L, 0.L, 0.L};
    for (size_t n = 0; n < r->np; ++n) {
      const long double w = (long double)r->p[n].m;
      m[0] += w;
      for (int a = 0; a < 3; ++a) {
        const long double x = (long double)r->p[n].pos[a];
        m[a + 1] += w * x;
        m[a + 4] += w * x * x;
      }
    }
    const double spacing[3] = {g->dx, g->dy, g->dz};
    const double origin[3] = {r->origin[0] - (double)pad * g->dx,
                              r->origin[1] - (double)pad * g->dy, r->origin[2]};
    for (int a = 0; a < 3; ++a) {
      const long double mean = m[a + 1] / m[0];
      long double variance = m[a + 4] / m[0] - mean * mean;
      if (variance < 0.0L) variance = 0.0L;
      const double rms = (double)sqrtl(variance);
      rep->rms_position_cells[a] = rms / spacing[a];
      if (rms > 0.0) {
        const double lower = origin[a] + (double)domain.lower[a] * spacing[a];
        const double upper = origin[a] + (double)domain.upper[a] * spacing[a];
        rep->centre_padding_rms[a] = fmin((double)mean - lower, upper - (double)mean) / rms;
      }
    }
  }
  slab_t s[4];
  const size_t planes = g->nz + 2, lx = pnx + 1, ly = pny + 1;
  for (int q = 0; q < 4; ++q) {
    s[q].nx = lx;
    s[q].ny = ly;
    s[q].planes = planes;
    s[q].v = (double*)calloc(lx * ly * planes, sizeof(double));
  }
  slab_t *potential = &s[0], *residual = &s[1], *direction = &s[2], *image = &s[3];
  rep->temporary_bytes = 4 * lx * ly * planes * sizeof(double) +
                         (g->nx + 1) * (g->ny + 1) * (g->nz + 1) * sizeof(double) +
                         (pad ? lx * ly * (g->nz + 1) * sizeof(double) : 0);
  double* rho = (double*)calloc(lx * ly * (g->nz + 1), sizeof(double));
  aprl_status st = shaped ? sf_shaped_deposit(r, rho, lx, ly, &domain)
                          : sf_deposit(r, rho, lx, ly, pad);
  if (st != APRL_OK) {
    free(rho);
    sf_free(s, 4);
    return st;
  }
  long double total = 0.L;
  for (size_t n = 0; n < r->np; ++n) total += (long double)r->p[n].q;
  rep->total_charge = (double)total;
  long double interior = 0.L;
  const long double vertex_volume = (long double)g->dx * (long double)g->dy * (long double)g->dz;
  for (size_t p = 1; p <= g->nz; ++p)
    for (size_t j = 0; j <= pny; ++j)
      for (size_t i = 0; i <= pnx; ++i)
        if (sf_interior(i, j, p - 1, &domain)) {
          const double q = rho[((p - 1) * ly + j) * lx + i];
          SAT(residual, i, j, p) = q / SI_EPSILON0;
          interior += (long double)q * vertex_volume;
        }
  free(rho);
  if (fabsl((interior - total) / total) > 1.0e-12L) {
    sf_free(s, 4);
    return fail(APRL_ERR_RUNTIME,
                "Initial CIC charge cloud touches the static zero-potential boundary; move every "
                "particle at least one complete cell inside the CPML entrance or enlarge the "
                "physical mesh padding");
  }
  memcpy(direction->v, residual->v, lx * ly * planes * sizeof(double));
  const long double source2 = sf_dot(residual, residual, &domain, g->nz);
  if (!(source2 > 0.0L) || !isfinite((double)source2)) {
    sf_free(s, 4);
    return fail(APRL_ERR_RUNTIME, "Initial particle charge produced an invalid Poisson source norm");
  }
  long double r2 = source2;
  const double cx = 1.0 / (g->dx * g->dx), cy = 1.0 / (g->dy * g->dy);
  const double cz = longitudinal / (g->dz * g->dz);
  const double diagonal = 2.0 * (cx + cy + cz);
  double relative = 0.0;
  for (uint64_t it = 0; it < cfg->maximum_iterations; ++it) {
    memset(image->v, 0, lx * ly * planes * sizeof(double));
    for (size_t p = 1; p <= g->nz; ++p) {
      const size_t k = p - 1;
      if (k <= domain.lower[2] || k >= domain.upper[2]) continue;
      for (size_t j = domain.lower[1] + 1; j < domain.upper[1]; ++j)
        for (size_t i = domain.lower[0] + 1; i < domain.upper[0]; ++i) {
          if (cowan) {
            double value = 0.0;
            for (size_t z = 0; z < 3; ++z)
              for (size_t y = 0; y < 3; ++y)
                for (size_t x = 0; x < 3; ++x)
                  value += stencil[z][y][x] * SAT(direction, i - 1 + x, j - 1 + y, p - 1 + z);
            SAT(image, i, j, p) = value;
          } else {
            SAT(image, i, j, p) =
                diagonal * SAT(direction, i, j, p) -
                cx * (SAT(direction, i - 1, j, p) + SAT(direction, i + 1, j, p)) -
                cy * (SAT(direction, i, j - 1, p) + SAT(direction, i, j + 1, p)) -
                cz * (SAT(direction, i, j, p - 1) + SAT(direction, i, j, p + 1));
          }
        }
    }
    const long double denominator = sf_dot(direction, image, &domain, g->nz);
    if (!(denominator > 0.0L) || !isfinite((double)denominator)) {
      sf_free(s, 4);
      return fail(APRL_ERR_RUNTIME, "Initial Gauss-field CG lost positive definiteness");
    }
    const double alpha = (double)(r2 / denominator);
    for (size_t p = 1; p <= g->nz; ++p) {
      const size_t k = p - 1;
      if (k <= domain.lower[2] || k >= domain.upper[2]) continue;
      for (size_t j = domain.lower[1] + 1; j < domain.upper[1]; ++j)
        for (size_t i = domain.lower[0] + 1; i < domain.upper[0]; ++i) {
          SAT(potential, i, j, p) += alpha * SAT(direction, i, j, p);
          SAT(residual, i, j, p) += -alpha * SAT(image, i, j, p);
        }
    }
    const long double next = sf_dot(residual, residual, &domain, g->nz);
    rep->iterations = it + 1;
    relative = (double)sqrtl(next / source2);
    if (relative <= cfg->relative_tolerance) {
      r2 = next;
      break;
    }
    if (!(next >= 0.0L) || !isfinite((double)next)) {
      sf_free(s, 4);
      return fail(APRL_ERR_RUNTIME, "Initial Gauss-field CG produced a non-finite residual");
    }
    const double beta = (double)(next / r2);
    for (size_t p = 1; p <= g->nz; ++p)
      for (size_t j = 0; j <= pny; ++j)
        for (size_t i = 0; i <= pnx; ++i)
          SAT(direction, i, j, p) = sf_interior(i, j, p - 1, &domain)
                                        ? SAT(residual, i, j, p) + beta * SAT(direction, i, j, p)
                                        : 0.0;
    r2 = next;
  }
  if (relative > cfg->relative_tolerance) {
    sf_free(s, 4);
    return fail(APRL_ERR_RUNTIME,
                "Initial Gauss-field solve did not converge; increase "
                "initial_self_field.maximum_iterations, relax its relative_tolerance, or reduce "
                "the grid aspect ratio");
  }
  comp_t *ex = &r->f[0], *ey = &r->f[1], *ez = &r->f[2];
  comp_t *bxc = &r->f[3], *byc = &r->f[4], *bzc = &r->f[5];
  if (cowan) {
    /* fieldsFromCowanPotential (src/eb_initial_field.cpp:487-553) */
    const double spacing[3] = {g->dx, g->dy, g->dz};
    for (unsigned axis = 0; axis < 3; ++axis) {
      memset(image->v, 0, lx * ly * planes * sizeof(double));
      for (size_t p = 1; p <= g->nz; ++p) {
        const size_t k = p - 1;
        if (k <= domain.lower[2] || k >= domain.upper[2]) continue;
        for (size_t j = domain.lower[1] + 1; j < domain.upper[1]; ++j)
          for (size_t i = domain.lower[0] + 1; i < domain.upper[0]; ++i)
            SAT(image, i, j, p) = sf_smoothed(r, potential, axis, i, j, p) -
                                  (axis == 2 ? translation * SAT(potential, i, j, p) : 0.0);
      }
      comp_t* c = &r->f[axis];
      for (size_t k = 0; k < c->nz; ++k)
        for (size_t j = 0; j < c->ny; ++j)
          for (size_t i = 0; i < c->nx; ++i)
            AT(c, i, j, k) = -(SAT(image, i + pad + (axis == 0), j + pad + (axis == 1),
                                   k + 1 + (axis == 2)) -
                               SAT(image, i + pad, j + pad, k + 1)) /
                             spacing[axis];
    }
  } else {
    /* fieldsFromPotential (src/eb_initial_field.cpp:427-485) */
    for (size_t k = 0; k <= g->nz; ++k)
      for (size_t j = 0; j <= g->ny; ++j)
        for (size_t i = 0; i < g->nx; ++i)
          AT(ex, i, j, k) = -(SAT(potential, i + pad + 1, j + pad, k + 1) -
                              SAT(potential, i + pad, j + pad, k + 1)) / g->dx;
    for (size_t k = 0; k <= g->nz; ++k)
      for (size_t j = 0; j < g->ny; ++j)
        for (size_t i = 0; i <= g->nx; ++i)
          AT(ey, i, j, k) = -(SAT(potential, i + pad, j + pad + 1, k + 1) -
                              SAT(potential, i + pad, j + pad, k + 1)) / g->dy;
    for (size_t k = 0; k < g->nz; ++k)
      for (size_t j = 0; j <= g->ny; ++j)
        for (size_t i = 0; i <= g->nx; ++i)
          AT(ez, i, j, k) = -longitudinal * (SAT(potential, i + pad, j + pad, k + 2) -
                                             SAT(potential, i + pad, j + pad, k + 1)) / g->dz;
  }
  sf_free(s, 4);
  const double scale = cowan ? applied * SI_C * SI_EPSILON0 * SI_MU0 : applied / SI_C;
  const double upper_w = 0.5 + 0.5 * applied * SI_C * g->dt / g->dz;
  const double lower_w = 1.0 - upper_w;
  if (upper_w < 0.0 || upper_w > 1.0)
    return fail(APRL_ERR_RUNTIME, "Initial B half-step shift exceeds one longitudinal cell");
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = 0; j < g->ny; ++j)
      for (size_t i = 0; i <= g->nx; ++i)
        AT(bxc, i, j, k) = -scale * (lower_w * AT(ey, i, j, k) + upper_w * AT(ey, i, j, k + 1));
  for (size_t k = 0; k < g->nz; ++k)
    for (size_t j = 0; j <= g->ny; ++j)
      for (size_t i = 0; i < g->nx; ++i)
        AT(byc, i, j, k) = scale * (lower_w * AT(ex, i, j, k) + upper_w * AT(ex, i, j, k + 1));
  memset(bzc->v, 0, bzc->nx * bzc->ny * bzc->nz * sizeof(double));
  if (include) {
    /* clearCpmlFields (src/eb_initial_field.cpp:564-626) */
    for (unsigned a = 0; a < 6; ++a) {
      comp_t* c = &r->f[a];
      const int electric = a < 3;
      const unsigned axis_c = a % 3;
      for (size_t k = 0; k < c->nz; ++k)
        for (size_t j = 0; j < c->ny; ++j)
          for (size_t i = 0; i < c->nx; ++i) {
            const size_t coord[3] = {i, j, k};
            int inside = 1;
            for (unsigned d = 0; d < 3; ++d) {
              const int vertex = electric ? d != axis_c : d == axis_c;
              const size_t gd = cfg->guard_cells[d];
              inside = inside && coord[d] >= gd &&
                       (vertex ? coord[d] <= cells[d] - gd : coord[d] < cells[d] - gd);
            }
            if (!inside) AT(c, i, j, k) = 0.0;
          }
    }
  }
  /* validateGauss (src/eb_initial_field.cpp:743-806) on the unpadded charge
   * the potential was solved for (CIC, or the shaped reference source) */
  {
    const size_t vx = g->nx + 1, vy = g->ny + 1;
    double* vrho = (double*)calloc(vx * vy * (g->nz + 1), sizeof(double));
    st = shaped ? sf_shaped_deposit(r, vrho, vx, vy, &physical) : sf_deposit(r, vrho, vx, vy, 0);
    if (st != APRL_OK) {
      free(vrho);
      return st;
    }
    long double res2 = 0.L, src2 = 0.L;
    double maximum = 0.0;
    for (size_t k = 0; k < g->nz; ++k) {
      if (k <= physical.lower[2] || k >= physical.upper[2]) continue;
      for (size_t j = physical.lower[1] + 1; j < physical.upper[1]; ++j)
        for (size_t i = physical.lower[0] + 1; i < physical.upper[0]; ++i) {
          const double left_z = k > 0 ? AT(ez, i, j, k - 1) : 0.0;
          const double divergence = (AT(ex, i, j, k) - AT(ex, i - 1, j, k)) / g->dx +
                                    (AT(ey, i, j, k) - AT(ey, i, j - 1, k)) / g->dy +
                                    (AT(ez, i, j, k) - left_z) / g->dz;
          const double source = vrho[(k * vy + j) * vx + i] / SI_EPSILON0;
          const double error = divergence - source;
          res2 += (long double)error * error;
          src2 += (long double)source * source;
          maximum = fmax(maximum, fabs(error));
        }
    }
    free(vrho);
    rep->relative_residual = src2 > 0.0L ? (double)sqrtl(res2 / src2) : 0.0;
    rep->maximum_gauss_residual = maximum;
    if (rep->relative_residual > 4.0 * cfg->relative_tolerance)
      return fail(APRL_ERR_RUNTIME, "Initial E field failed the post-solve discrete Gauss check");
  }
  /* initialFieldEnergy (src/eb_initial_field.cpp:665-691) */
  {
    long double we = 0.L, wm = 0.L;
    const long double volume = (long double)g->dx * (long double)g->dy * (long double)g->dz;
    for (size_t k = 0; k < g->nz; ++k)
      for (size_t j = 0; j < g->ny; ++j)
        for (size_t i = 0; i < g->nx; ++i) {
          const double e0 = 0.25 * (AT(ex, i, j, k) + AT(ex, i, j + 1, k) + AT(ex, i, j, k + 1) +
                                    AT(ex, i, j + 1, k + 1));
          const double e1 = 0.25 * (AT(ey, i, j, k) + AT(ey, i + 1, j, k) + AT(ey, i, j, k + 1) +
                                    AT(ey, i + 1, j, k + 1));
          const double e2 = 0.25 * (AT(ez, i, j, k) + AT(ez, i + 1, j, k) + AT(ez, i, j + 1, k) +
                                    AT(ez, i + 1, j + 1, k));
          const double m0 = 0.5 * (AT(bxc, i, j, k) + AT(bxc, i + 1, j, k));
          const double m1 = 0.5 * (AT(byc, i, j, k) + AT(byc, i, j + 1, k));
          const double m2 = 0.5 * (AT(bzc, i, j, k) + AT(bzc, i, j, k + 1));
          const double en = e0 * e0 + e1 * e1 + e2 * e2;
          const double bn = m0 * m0 + m1 * m1 + m2 * m2;
          we += 0.5L * (long double)SI_EPSILON0 * (long double)en * volume;
          wm += 0.5L / (long double)SI_MU0 * (long double)bn * volume;
        }
    rep->initial_electric_energy = (double)we;
    rep->initial_magnetic_energy = (double)wm;
  }
  return APRL_OK;
}
