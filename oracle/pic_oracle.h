/*
 * pic_oracle.h -- CPU oracle for the APRL per-timestep PIC loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a serial plain-C restatement of the
 * reference's one-rank, moving-window, conservative-source step, used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker.  The product (aprl_b200) never links, loads or calls it.
 *
 * The entry points mirror include/aprl_gpu.h one for one, with the prefix
 * oracle_ and an oracle_run handle, so a test drives both sides through the
 * same sequence of calls and compares the results.
 */
#ifndef APRL_PIC_ORACLE_H
#define APRL_PIC_ORACLE_H

#include "../include/aprl_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_run oracle_run;

const char* oracle_last_error(void);
aprl_status oracle_magnet_prepare(aprl_magnet* magnet);
aprl_status oracle_cowan_coefficients(double dx, double dy, double dz,
                                      double out[12]);

aprl_status oracle_run_create(const aprl_run_config* config, oracle_run** out);
aprl_status oracle_run_destroy(oracle_run* run);
aprl_status oracle_run_set_reference(oracle_run* run, unsigned component,
                                     const double* host, size_t count);
aprl_status oracle_run_set_field(oracle_run* run, unsigned component,
                                 const double* host, size_t count);
aprl_status oracle_run_get_field(oracle_run* run, unsigned component,
                                 double* host, size_t count);
aprl_status oracle_run_field_shape(const oracle_run* run, unsigned component,
                                   uint64_t shape[3]);
aprl_status oracle_run_history_length(const oracle_run* run, unsigned index,
                                      uint64_t* length);
aprl_status oracle_run_set_history(oracle_run* run, unsigned index,
                                   const double* host, size_t count);
aprl_status oracle_run_get_history(oracle_run* run, unsigned index,
                                   double* host, size_t count);
aprl_status oracle_run_set_particles(oracle_run* run, size_t count,
                                     const double* x, const double* y,
                                     const double* z, const double* ux,
                                     const double* uy, const double* uz,
                                     const double* charge, const double* mass,
                                     const uint64_t* id, int reset_carriers);
aprl_status oracle_run_particle_count(const oracle_run* run, size_t* count);
aprl_status oracle_run_set_held(oracle_run* run, size_t count, const uint8_t* frozen,
                                const double* frozen_beta_z);
aprl_status oracle_run_get_held(oracle_run* run, size_t capacity, uint8_t* frozen,
                                double* frozen_beta_z, size_t* count);
aprl_status oracle_run_get_particles(oracle_run* run, size_t capacity,
                                     double* x, double* y, double* z,
                                     double* ux, double* uy, double* uz,
                                     double* charge, double* mass,
                                     uint64_t* id, size_t* count);
aprl_status oracle_run_carrier_count(const oracle_run* run, size_t* count);
aprl_status oracle_run_get_carriers(oracle_run* run, size_t capacity,
                                    double* position, double* velocity,
                                    double* charge, double* weight,
                                    size_t* count);
aprl_status oracle_run_set_carriers(oracle_run* run, size_t count,
                                    const double* position,
                                    const double* velocity,
                                    const double* charge,
                                    const double* weight);
aprl_status oracle_run_advance_magnetic(oracle_run* run);
aprl_status oracle_run_preview_electric(oracle_run* run);
aprl_status oracle_run_coupling_trial(oracle_run* run, double residual[4]);
aprl_status oracle_run_commit_electric(oracle_run* run);
aprl_status oracle_run_shift(oracle_run* run);
aprl_status oracle_run_step(oracle_run* run, uint32_t steps);
aprl_status oracle_run_enable_energy_ledger(oracle_run* run, int enabled);
aprl_status oracle_run_energy_ledger(oracle_run* run, aprl_energy_ledger* out);
aprl_status oracle_run_initialize_self_field(oracle_run* run, const aprl_self_field_config* config,
                                             aprl_self_field_report* report);
aprl_status oracle_run_get_stats(const oracle_run* run, aprl_step_stats* stats);
aprl_status oracle_run_get_slot_fields(oracle_run* run, size_t capacity,
                                       double* used_e, double* used_b,
                                       double* next_e, double* next_b,
                                       size_t* count);
aprl_status oracle_run_sample_field_plane(oracle_run* run, double plane_lab_z,
                                          double* out, size_t count,
                                          int* inside);

/* Kernel-level checks used by the known-answer tests. */
/* longitudinal_shape::weights visits for one chord: writes up to capacity
 * (axis, i, j, k, w) records; returns the number of visits or -1. */
long oracle_shape_weights(const aprl_run_config* config, const double origin[3],
                          const double begin[3], const double end[3],
                          int32_t* axis, int64_t* index /* 3*capacity */,
                          double* weight, long capacity);
/* source_coupling_math::momentum (src/source_coupling_math.h:272-293). */
int oracle_momentum(double u[3], const double e[3], const double b[3],
                    double q, double m, double h, double known_gamma);
/* BoostFrameTransform::gammaFromProperVelocity. */
double oracle_gamma(const double u[3]);
/* RelativisticBorisPusher::push per particle (src/eb_particles.cpp:207-216). */
aprl_status oracle_boris_push(size_t count, double* x, double* y, double* z, double* ux,
                              double* uy, double* uz, const double* charge, const double* mass,
                              const double* electric, const double* magnetic, double dt);
/* Prescribed lab magnets seen in the box frame at (position, time). */
aprl_status oracle_prescribed_box(const aprl_run_config* config,
                                  const double position[3], double time,
                                  double e[3], double b[3]);

#ifdef __cplusplus
}
#endif
#endif
