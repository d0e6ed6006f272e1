// A C++ host program in the shape of APRL's Simulation step loop, driving
// the B200 library only through include/aprl_gpu.hpp (the C ABI).  Used by
// tests/test_cpp_host.py: compiled on any host, run where a GPU exists.
#include <cmath>
#include <cstdio>
#include <vector>

#include "aprl_gpu.hpp"

int main() {
  aprl_run_config c{};
  c.nx = 16; c.ny = 16; c.nz = 32;
  c.dx = 5e-6; c.dy = 5e-6; c.dz = 2e-6; c.dt = c.dz / 299792458.0;
  c.cpml_cells_x = c.cpml_cells_y = 3;
  c.cpml_polynomial_order = 3.0; c.cpml_target_reflection = 1e-8;
  c.cpml_kappa_max = 8.0; c.cpml_alpha_fraction = 0.0;
  c.shape = APRL_SHAPE_LINEAR_BINOMIAL3; c.substeps = 1; c.max_trials = 64;
  c.force_tolerance = 1e-13; c.work_tolerance = 1e-8;
  c.boost_gamma = 10.0;
  c.boost_gamma_beta = std::sqrt(9.0) * std::sqrt(11.0);
  c.boost_beta = c.boost_gamma_beta / c.boost_gamma;
  c.initial_offset = 12; c.reference_nz = 14; c.translation_beta = 1.0;
  c.reference_origin[0] = -8 * c.dx; c.reference_origin[1] = -8 * c.dy;
  c.reference_origin[2] = -12 * c.dz;
  c.exit_lab_z = c.boost_gamma * 20 * c.dz;
  try {
    aprl::gpu::PicRun run(c);
    for (unsigned a = 0; a < 6; ++a) {
      const std::size_t n = (c.nx + (a < 3 ? (a != 0) : (a == 3))) *
                            (c.ny + (a < 3 ? (a != 1) : (a == 4))) *
                            (c.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0));
      run.setReference(a, std::vector<double>(n, 0.0));
    }
    aprl::gpu::ParticleArrays p;
    for (int n = 0; n < 64; ++n) {
      p.x.push_back((n % 8 - 3.5) * 1e-6);
      p.y.push_back((n / 8 - 3.5) * 1e-6);
      p.z.push_back((10 + 0.1 * n) * c.dz);
      p.ux.push_back(0.0); p.uy.push_back(0.0); p.uz.push_back(98.0);
      p.charge.push_back(-1.6e-19 * 1e4); p.mass.push_back(9.1e-31 * 1e4);
      p.id.push_back(n + 1);
    }
    run.setParticles(p);
    run.enableEnergyLedger();
    run.solveStep(2);
    const aprl_step_stats s = run.stats();
    const aprl_energy_ledger l = run.energyLedger();
    std::printf("steps=%llu particles=%llu trials=%u ledger_steps=%llu kinetic=%g\n",
                (unsigned long long)s.step, (unsigned long long)s.particles, s.iterations,
                (unsigned long long)l.flux_steps, l.particle_kinetic);
    if (l.flux_steps != 2 || !(l.particle_kinetic > 0.0)) return 3;
    // A bad argument must surface as the reference's exception type.
    try {
      run.setField(aprl::gpu::Component::Ex, std::vector<double>(3, 0.0));
      return 2;
    } catch (const std::invalid_argument&) {
    }
    return s.step == 2 ? 0 : 1;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
