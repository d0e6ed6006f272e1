// aprl_gpu.hpp -- C++ host interface over the C ABI of include/aprl_gpu.h,
// shaped like the reference's own seams so that APRL's Simulation can hand
// its per-step PIC loop to the GPU with the same names, argument meanings
// and error behaviour:
//
//   aprl::gpu::PicRun::advanceMagnetic()      EBZSlabHaloExchange::advanceMagnetic
//                                             with the moving-window halos
//                                             (src/simulation.cpp:518-524)
//   aprl::gpu::PicRun::previewElectric()      previewElectricBoundary + advanceElectric
//                                             (src/simulation_source_coupling.cpp:20-24)
//   aprl::gpu::PicRun::couplingTrial()        one fixed-point trial + localResidual
//                                             (src/simulation_source_coupling.cpp:43-48)
//   aprl::gpu::PicRun::commitConservativeElectric()
//                                             replay + commit (src/simulation_source_coupling.cpp:56-65)
//   aprl::gpu::PicRun::finishMovingWindowStep()
//                                             (src/simulation_moving_window.cpp:341-379)
//   aprl::gpu::PicRun::solveStep()            one Simulation::solve loop body
//
// Failures throw std::invalid_argument, std::out_of_range or
// std::runtime_error with the library's message, as the reference does.
// Header only; link against aprl_b200/libaprl_b200.so.
#ifndef APRL_GPU_HPP
#define APRL_GPU_HPP

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "aprl_gpu.h"

namespace aprl {
namespace gpu {

inline void check(aprl_status status) {
  if (status == APRL_OK) return;
  const std::string message = aprl_last_error();
  switch (status) {
    case APRL_ERR_INVALID_ARGUMENT: throw std::invalid_argument(message);
    case APRL_ERR_OUT_OF_RANGE: throw std::out_of_range(message);
    default: throw std::runtime_error(message);
  }
}

// Ex Ey Ez Bx By Bz Jx Jy Jz, as YeeComponent accessors of EBFieldGrid.
enum class Component : unsigned { Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz };

struct ParticleArrays {  // RelativisticParticleSI as structure of arrays
  std::vector<double> x, y, z, ux, uy, uz, charge, mass;
  std::vector<std::uint64_t> id;
  std::size_t size() const { return id.size(); }
};

class PicRun {
 public:
  explicit PicRun(const aprl_run_config& config, void* stream = nullptr) {
    check(aprl_run_create(&config, stream, &run_));
  }
  ~PicRun() { aprl_run_destroy(run_); }
  PicRun(const PicRun&) = delete;
  PicRun& operator=(const PicRun&) = delete;

  aprl_run* handle() { return run_; }

  // MovingWindowReference supply (src/moving_window_fields.h:15-20).
  void setReference(unsigned component, const std::vector<double>& values) {
    check(aprl_run_set_reference(run_, component, values.data(), values.size()));
  }

  std::array<std::uint64_t, 3> shape(Component c) const {
    std::array<std::uint64_t, 3> s{};
    check(aprl_run_field_shape(run_, static_cast<unsigned>(c), s.data()));
    return s;
  }
  void setField(Component c, const std::vector<double>& values) {
    check(aprl_run_set_field(run_, static_cast<unsigned>(c), values.data(), values.size()));
  }
  std::vector<double> field(Component c) {
    const auto s = shape(c);
    std::vector<double> out(s[0] * s[1] * s[2]);
    check(aprl_run_get_field(run_, static_cast<unsigned>(c), out.data(), out.size()));
    return out;
  }

  void setParticles(const ParticleArrays& p, bool resetCarriers = true) {
    check(aprl_run_set_particles(run_, p.size(), p.x.data(), p.y.data(), p.z.data(),
                                 p.ux.data(), p.uy.data(), p.uz.data(), p.charge.data(),
                                 p.mass.data(), p.id.data(), resetCarriers ? 1 : 0));
  }
  ParticleArrays particles() {
    std::size_t n = 0;
    check(aprl_run_particle_count(run_, &n));
    ParticleArrays p;
    for (auto* v : {&p.x, &p.y, &p.z, &p.ux, &p.uy, &p.uz, &p.charge, &p.mass}) v->resize(n);
    p.id.resize(n);
    check(aprl_run_get_particles(run_, n, p.x.data(), p.y.data(), p.z.data(), p.ux.data(),
                                 p.uy.data(), p.uz.data(), p.charge.data(), p.mass.data(),
                                 p.id.data(), &n));
    return p;
  }

  // The seams of one step, in the reference's order.
  void advanceMagnetic() { check(aprl_run_advance_magnetic(run_)); }
  void previewElectric() { check(aprl_run_preview_electric(run_)); }
  // {force, defect, scale, calls} of ConservativeSourceCoupling::localResidual.
  std::array<double, 4> couplingTrial() {
    std::array<double, 4> r{};
    check(aprl_run_coupling_trial(run_, r.data()));
    return r;
  }
  void commitConservativeElectric() { check(aprl_run_commit_electric(run_)); }
  void finishMovingWindowStep() { check(aprl_run_shift(run_)); }

  // Simulation::solve loop body with solveConservativeSourceStep's stopping
  // rule (>= 2 trials when work > 0, force < 1e-13, work < 1e-8).
  void solveStep(std::uint32_t steps = 1) { check(aprl_run_step(run_, steps)); }

  aprl_step_stats stats() const {
    aprl_step_stats s{};
    check(aprl_run_get_stats(run_, &s));
    return s;
  }

  // EBGaussFieldInitializer::initialize on the run's particles (before the
  // first step).
  aprl_self_field_report initializeSelfField(const aprl_self_field_config& config) {
    aprl_self_field_report report{};
    check(aprl_run_initialize_self_field(run_, &config, &report));
    return report;
  }

  // The inlet reference from the Cowan self-field of a bunch on the
  // reference grid (before the first step).
  aprl_self_field_report prepareReference(const ParticleArrays& p,
                                          const aprl_self_field_config& config) {
    aprl_self_field_report report{};
    check(aprl_run_prepare_reference(run_, p.x.size(), p.x.data(), p.y.data(), p.z.data(),
                                     p.ux.data(), p.uy.data(), p.uz.data(), p.charge.data(),
                                     p.mass.data(), &config, &report));
    return report;
  }

  // MovingWindowFields::enableEnergyLedger / energyLedger plus the ledger
  // record's interior field energy and particle energy sums.
  void enableEnergyLedger(bool enabled = true) {
    check(aprl_run_enable_energy_ledger(run_, enabled ? 1 : 0));
  }
  aprl_energy_ledger energyLedger() {
    aprl_energy_ledger l{};
    check(aprl_run_energy_ledger(run_, &l));
    return l;
  }

  // LabDetectorManager::samplePlane on a fixed lab plane (lab-frame E, B).
  bool sampleFieldPlane(double labZ, std::vector<double>& out) {
    const auto ex = shape(Component::Bz);
    out.resize(6 * ex[0] * ex[1]);
    int inside = 0;
    check(aprl_run_sample_field_plane(run_, labZ, out.data(), out.size(), &inside));
    return inside != 0;
  }

 private:
  aprl_run* run_ = nullptr;
};

}  // namespace gpu
}  // namespace aprl

#endif
