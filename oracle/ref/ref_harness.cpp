// ref_harness.cpp -- drives the reference's OWN hot-path classes, compiled
// from the APRL sources by oracle/build_oracle.py into oracle/_ref/.
// TEST INFRASTRUCTURE ONLY: it pins the plain-C oracle (oracle/pic_oracle.c)
// to the reference arithmetic and times the reference CPU path for the
// benchmark's CPU-baseline leg.  The product never loads it.
//
// The numerical operators are the reference's: EBFieldGrid (Cowan-z),
// EBConvolutionalPML through MovingWindowFields' boundary, the moving-window
// shift, ConservativeSourceCoupling (gather, Lapenta-Markidis push,
// residual, E +/- J), ChargeConservingCurrentDepositor with
// longitudinal_shape::Current, ParticleCPMLRegion, ParticleOpenBoundary,
// BoostFrameTransform and SIFieldSourceSet.  Only the one-rank driver of
// Simulation (src/simulation.cpp:493-613, 4167-5605,
// src/simulation_source_coupling.cpp:16-65,
// src/simulation_moving_window.cpp:280-379), which lives in translation
// units that need HDF5/yaml/FFTW, is restated here for active particles and
// CPML carriers.  The exported functions mirror include/aprl_gpu.h with the
// prefix ref_.
#include <mpi.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <unistd.h>

#include <fstream>

#include "aprl_gpu.h"
#include "boostframe.h"
#include "charge_matched_inlet.h"
#include "compute_threads.h"
#include "eb_cpml.h"
#include "eb_deposition.h"
#include "eb_field.h"
#include "eb_initial_field.h"
#include "eb_particles.h"
#include "eb_sources.h"
#include "longitudinal_shape.h"
#include "moving_window_fields.h"
#include "particle_boundary.h"
#include "pending_particle_queue.h"
#include "source_coupling.h"
#include "source_coupling_math.h"
#include "blocked_cowan_reference.h"
#include "transverse_reference_current.h"

using namespace aprl;
typedef FieldVector<Double> Vec;

namespace {
thread_local std::string g_error;

aprl_status failWith(aprl_status s, const std::string& m) {
  g_error = m;
  return s;
}

template <class F>
aprl_status guarded(F f) {
  try {
    f();
    return APRL_OK;
  } catch (const std::invalid_argument& e) {
    return failWith(APRL_ERR_INVALID_ARGUMENT, e.what());
  } catch (const std::out_of_range& e) {
    return failWith(APRL_ERR_OUT_OF_RANGE, e.what());
  } catch (const std::exception& e) {
    return failWith(APRL_ERR_RUNTIME, e.what());
  }
}
}  // namespace

struct ref_run {
  aprl_run_config cfg;
  // The reference's own TransverseReferenceCurrent over a file the harness
  // prepared from the supplied reference tables.
  std::unique_ptr<aprl::TransverseReferenceCurrent> surface;
  std::string surfaceFile;
  EBGridGeometry geometry;
  EBCPMLParameters cpml;
  std::unique_ptr<EBFieldGrid> fields;
  std::unique_ptr<MovingWindowFields> window;
  std::unique_ptr<ConservativeSourceCoupling> coupling;
  BoostFrameTransform frame;
  SIFieldSourceSet sources;
  std::vector<double> reference[6];
  std::size_t referenceShape[6][3];
  std::vector<RelativisticParticleSI> particles, savedParticles;
  std::vector<ParticleCPMLCarrier> carriers, savedCarriers;
  std::size_t step = 0;
  std::ptrdiff_t offset = 0;
  double time = 0.;
  Vec origin;
  unsigned long long exits = 0, savedExits = 0;
  double exitCharge = 0., savedExitCharge = 0.;
  unsigned long long counts[3][6] = {}, savedCounts[3][6] = {};
  double charges[3][6] = {}, savedCharges[3][6] = {};
  unsigned long long croppedCarriers = 0;
  double croppedCharge = 0.;
  unsigned lastIterations = 0, maxIterations = 0;
  unsigned long long totalIterations = 0;
  double lastForce = 0., lastWork = 0.;
  unsigned trials = 0;
  int stage = 0;
  std::string directory;
  std::unique_ptr<PendingParticleQueue> pending;
  unsigned long long admitted = 0, activations = 0, savedActivations = 0;
  bool ledger = false;
  std::unique_ptr<ChargeMatchedInlet> inlet;
};

namespace {
// Simulation::movingWindowFieldValue (src/simulation_moving_window.cpp:280-294)
// over the supplied in-memory reference table.
Double referenceValue(void* context, unsigned a, std::size_t i, std::size_t j,
                      std::ptrdiff_t k, std::size_t step) {
  const ref_run& r = *static_cast<ref_run*>(context);
  const double z = static_cast<double>(k) - r.cfg.translation_beta * step;
  const std::size_t count = r.cfg.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0);
  if (a >= 6 || !std::isfinite(z) || z < 0. || z > count - 1)
    throw std::out_of_range("Moving reference query outside prepared native field");
  const auto lo = static_cast<std::size_t>(std::floor(z)), hi = std::min(lo + 1, count - 1);
  const auto& s = r.referenceShape[a];
  const double f = z - lo, lower = r.reference[a].at((lo * s[1] + j) * s[0] + i);
  return f == 0. ? lower : (1. - f) * lower + f * r.reference[a].at((hi * s[1] + j) * s[0] + i);
}

// Simulation::completeMovingInletLayer (src/simulation_moving_window.cpp:312-323)
// without its ledger file: the charge-matched Ez of the inserted inlet layer.
void completeInletLayer(void* context, EBFieldGrid& f, std::size_t step, std::ptrdiff_t offset) {
  ref_run& r = *static_cast<ref_run*>(context);
  Vec origin(0.);
  origin[0] = r.cfg.reference_origin[0];
  origin[1] = r.cfg.reference_origin[1];
  origin[2] = std::fma(static_cast<double>(offset), f.geometry().dz, r.cfg.reference_origin[2]);
  r.inlet->begin(origin);
  for (const auto& p : r.particles) r.inlet->particle(p);
  if (r.pending) {
    const auto visit = [&](const RelativisticParticleSI& p) { r.inlet->particle(p); };
    r.pending->visitNear(step, 8, visit);
  }
  r.inlet->complete(f, false);
}

YeeComponent& component(EBFieldGrid& f, unsigned a) {
  switch (a) {
    case 0: return f.ex(); case 1: return f.ey(); case 2: return f.ez();
    case 3: return f.bx(); case 4: return f.by(); case 5: return f.bz();
    case 6: return f.jx(); case 7: return f.jy(); default: return f.jz();
  }
}

void save(ref_run& r) {
  r.savedActivations = r.activations;
  r.savedParticles = r.particles;
  r.savedCarriers = r.carriers;
  r.savedExits = r.exits;
  r.savedExitCharge = r.exitCharge;
  std::memcpy(r.savedCounts, r.counts, sizeof r.counts);
  std::memcpy(r.savedCharges, r.charges, sizeof r.charges);
}

void restore(ref_run& r) {
  r.activations = r.savedActivations;
  r.particles = r.savedParticles;
  r.carriers = r.savedCarriers;
  r.exits = r.savedExits;
  r.exitCharge = r.savedExitCharge;
  std::memcpy(r.counts, r.savedCounts, sizeof r.counts);
  std::memcpy(r.charges, r.savedCharges, sizeof r.charges);
}

// Simulation::firstMovingWindowEntry (src/simulation_moving_window.cpp:380-395).
bool firstMovingWindowEntry(const ref_run& r, const ParticleCPMLRegion& cpml,
                            const Vec& start, const Vec& end, Double startFraction,
                            ParticleBoundaryHit& hit) {
  bool present = cpml.firstEntry(start, end, hit);
  const double a = r.frame.labZFromBoxZT(start[2], r.time + startFraction * r.cfg.dt) - r.cfg.exit_lab_z;
  const double b = r.frame.labZFromBoxZT(end[2], r.time + r.cfg.dt) - r.cfg.exit_lab_z;
  if (a >= 0.) throw std::runtime_error("Active particle started beyond trusted moving-window exit");
  if (b >= 0. && b > a) {
    const double fraction = -a / (b - a);
    if (!present || fraction < hit.fraction) {
      for (unsigned d = 0; d < 3; ++d) hit.position[d] = start[d] + fraction * (end[d] - start[d]);
      hit.fraction = fraction;
      hit.face = ParticleBoundaryFace::UpperZ;
      present = true;
    }
  }
  return present;
}

// pushDepositAndMigrate for one rank, active particles and CPML carriers
// (src/simulation.cpp:4167-5368; processCarrierSegment 4310-4407,
// processActiveSegment 4555-4917).
void pushDepositAndMigrate(ref_run& r) {
  ChargeConservingCurrentDepositor depositor(*r.fields, r.origin, r.coupling->longitudinalCurrent());
  ParticleCPMLRegion cpml(r.geometry, r.origin, r.cpml);
  ParticleOpenBoundary boundary(r.geometry, r.origin, r.geometry, r.origin, 0);
  const Double crossingTolerance = 64.0 * std::numeric_limits<Double>::epsilon();
  const Double carrierCutoff = 64.0 * std::numeric_limits<Double>::epsilon();
  std::vector<RelativisticParticleSI> retained;
  std::vector<ParticleCPMLCarrier> retainedCarriers;
  retained.reserve(r.particles.size());
  const auto processCarrierSegment = [&](ParticleCPMLCarrier carrier, const Vec& segmentStart,
                                         Double segmentStartFraction) {
    if (!(carrier.currentWeight >= 0.0) || !std::isfinite(carrier.currentWeight))
      throw std::runtime_error("Invalid CPML carrier current weight");
    if (carrier.currentWeight <= carrierCutoff) return;
    ParticleBoundaryHit outerHit;
    const bool exitsOuter = boundary.firstExit(segmentStart, carrier.position, outerHit);
    Double localEndFraction = 1.0;
    Vec segmentEnd(carrier.position);
    bool remove = false;
    if (exitsOuter) {
      localEndFraction = outerHit.fraction;
      segmentEnd = outerHit.position;
      remove = true;
    }
    const Double globalEndFraction = segmentStartFraction + localEndFraction * (1.0 - segmentStartFraction);
    const Double duration = (globalEndFraction - segmentStartFraction) * r.cfg.dt;
    Vec midpoint(0.0);
    for (unsigned a = 0; a < 3; ++a) midpoint[a] = 0.5 * (segmentStart[a] + segmentEnd[a]);
    const Double midpointDamping = cpml.currentDampingFactor(segmentStart, midpoint, 0.5 * duration);
    const Double endDamping = cpml.currentDampingFactor(segmentStart, segmentEnd, duration);
    const Double depositedWeight = carrier.currentWeight * midpointDamping;
    const Double endWeight = carrier.currentWeight * endDamping;
    depositor.depositSegment(segmentStart, segmentEnd, carrier.charge * depositedWeight);
    if (remove) {
      const std::size_t face = static_cast<std::size_t>(outerHit.face);
      ++r.counts[2][face];
      r.charges[2][face] += carrier.charge * endWeight;
      return;
    }
    if (endWeight <= carrierCutoff) return;
    carrier.currentWeight = endWeight;
    carrier.position = segmentEnd;
    retainedCarriers.push_back(carrier);
  };
  if (r.pending)
    r.pending->visitNear(r.step, 8, [&](const RelativisticParticleSI& p) {
      auto end = p.position;
      end[2] += SI::c * r.cfg.dt * p.frozenBetaZ;
      r.coupling->depositFrozenSourceSupport(p.position, end, p.charge, false);
    });
  for (std::size_t n = 0; n < r.carriers.size(); ++n) {
    ParticleCPMLCarrier carrier = r.carriers[n];
    const Vec start(carrier.position);
    carrier.position.pmv(r.cfg.dt, carrier.velocity);
    processCarrierSegment(carrier, start, 0.0);
  }
  struct Hits {
    ParticleBoundaryHit cpmlHit, outerHit;
    bool entersCpml = false, exitsOuter = false;
  };
  // processActiveSegment (src/simulation.cpp:4555-4917) at one rank.
  const auto processActiveSegment = [&](RelativisticParticleSI particle, Vec segmentStart,
                                        Double segmentStartFraction, const Vec* kink,
                                        Double kinkFraction, const Hits* cached) {
    if (kink) {
      ParticleBoundaryHit cpmlHit, outerHit;
      const bool entersCpml = cpml.firstEntry(segmentStart, *kink, cpmlHit);
      const bool exitsOuter = boundary.firstExit(segmentStart, *kink, outerHit);
      if (entersCpml || exitsOuter)
        throw std::runtime_error("Held-transverse activation crossed a particle boundary during the frozen part of a field step");
      depositor.depositSegment(segmentStart, *kink, particle.charge);
      segmentStart = *kink;
      segmentStartFraction = kinkFraction;
    }
    Hits computed;
    if (!cached) {
      computed.entersCpml = firstMovingWindowEntry(r, cpml, segmentStart, particle.position,
                                                   segmentStartFraction, computed.cpmlHit);
      computed.exitsOuter = boundary.firstExit(segmentStart, particle.position, computed.outerHit);
      cached = &computed;
    }
    int action = 0;
    Double localEndFraction = 1.0;
    Vec segmentEnd(particle.position);
    ParticleBoundaryHit selected;
    if (cached->entersCpml &&
        (!cached->exitsOuter ||
         cached->cpmlHit.fraction <= cached->outerHit.fraction + crossingTolerance)) {
      action = 1;
      localEndFraction = cached->cpmlHit.fraction;
      segmentEnd = cached->cpmlHit.position;
      selected = cached->cpmlHit;
    } else if (cached->exitsOuter) {
      action = 2;
      localEndFraction = cached->outerHit.fraction;
      segmentEnd = cached->outerHit.position;
      selected = cached->outerHit;
    }
    depositor.depositSegment(segmentStart, segmentEnd, particle.charge);
    const Double globalEndFraction = segmentStartFraction + localEndFraction * (1.0 - segmentStartFraction);
    if (action == 1) {
      const std::size_t face = static_cast<std::size_t>(selected.face);
      if (selected.face == ParticleBoundaryFace::UpperZ) {
        ++r.exits;
        r.exitCharge += particle.charge;
      } else {
        ++r.counts[0][face];
        r.charges[0][face] += particle.charge;
      }
      ParticleCPMLCarrier carrier;
      carrier.position = particle.position;
      const Double gamma = BoostFrameTransform::gammaFromProperVelocity(particle.properVelocity);
      carrier.velocity = particle.properVelocity;
      carrier.velocity *= SI::c / gamma;
      carrier.charge = particle.charge;
      carrier.currentWeight = 1.0;
      processCarrierSegment(carrier, selected.position, globalEndFraction);
    } else if (action == 2) {
      const std::size_t face = static_cast<std::size_t>(selected.face);
      ++r.counts[1][face];
      r.charges[1][face] += particle.charge;
    } else {
      retained.push_back(particle);
    }
  };
  const Double dt = r.cfg.dt, t = r.time;
  for (std::size_t n = 0; n < r.particles.size(); ++n) {
    const RelativisticParticleSI original = r.particles[n];
    RelativisticParticleSI particle = original;
    Vec start(particle.position);
    if (start[2] < r.origin[2] && !particle.frozen)
      throw std::runtime_error("An active particle is upstream of the moving window; the inlet guard did not contain its release event");
    // prepareParticle (src/simulation.cpp:4919-5035) with holdTransverse.
    RelativisticParticleSI activeStart = particle;
    Double activeStartTime = t;
    bool hasActiveSegment = !particle.frozen;
    if (particle.frozen) {
      const Double betaHeld = particle.frozenBetaZ;
      const Double startLabZ = r.frame.labZFromBoxZT(start[2], t);
      particle.position[2] += SI::c * dt * betaHeld;
      const Double endLabZ = r.frame.labZFromBoxZT(particle.position[2], t + dt);
      if (endLabZ >= r.cfg.activation_plane_lab_z) {
        if (start[2] < r.origin[2])
          throw std::runtime_error("A pending upstream held particle would release before a complete in-window step");
        const Double plane = r.cfg.activation_plane_lab_z;
        const Double crossingFraction = startLabZ >= plane ? 0.0 :
          std::max(0.0, std::min(1.0, (plane - startLabZ) / (endLabZ - startLabZ)));
        particle.position = start;
        particle.position[2] += SI::c * crossingFraction * dt * betaHeld;
        particle.frozen = false;
        hasActiveSegment = true;
        activeStart = particle;
        activeStartTime = t + crossingFraction * dt;
        const Double remaining = (1.0 - crossingFraction) * dt;
        if (remaining > 0.0)
          r.coupling->push(particle, r.sources, r.frame, activeStartTime, remaining,
                           r.cfg.substeps, 0, 0, 0);
      }
    } else {
      r.coupling->push(particle, r.sources, r.frame, t, dt, r.cfg.substeps, 0, 0, 0);
    }
    if (original.frozen && hasActiveSegment) ++r.activations;
    Double segmentStartFraction = 0.0;
    if (start[2] < r.origin[2]) {
      if (!original.frozen || !particle.frozen || hasActiveSegment)
        throw std::runtime_error("Moving-window upstream admission requires an unreleased held particle on rank zero");
      if (particle.position[2] < r.origin[2]) {
        r.coupling->depositFrozenSourceSupport(start, particle.position, particle.charge, false);
        retained.push_back(particle);
        continue;
      }
      const Double fraction = (r.origin[2] - start[2]) / (particle.position[2] - start[2]);
      if (!(fraction >= 0.0 && fraction <= 1.0) || !std::isfinite(fraction))
        throw std::runtime_error("Invalid moving-window admission fraction");
      for (unsigned axis = 0; axis < 3; ++axis)
        start[axis] += fraction * (particle.position[axis] - start[axis]);
      start[2] = r.origin[2];
      segmentStartFraction = fraction;
      r.coupling->depositFrozenSourceSupport(original.position, start, particle.charge, false);
    }
    const bool hasActivationKink = original.frozen && hasActiveSegment &&
                                   activeStartTime > t && activeStartTime < t + dt;
    const Double activationKinkFraction = (activeStartTime - t) / dt;
    if (hasActivationKink) {
      processActiveSegment(particle, start, segmentStartFraction, &activeStart.position,
                           activationKinkFraction, nullptr);
    } else {
      Hits hits;
      hits.entersCpml = firstMovingWindowEntry(r, cpml, start, particle.position,
                                               segmentStartFraction, hits.cpmlHit);
      hits.exitsOuter = boundary.firstExit(start, particle.position, hits.outerHit);
      processActiveSegment(particle, start, segmentStartFraction, nullptr, 0.0, &hits);
    }
  }
  r.particles.swap(retained);
  r.carriers.swap(retainedCarriers);
}
}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

aprl_status ref_run_create(const aprl_run_config* config, ref_run** out) {
  auto run = std::unique_ptr<ref_run>(new ref_run());
  ref_run& r = *run;
  r.cfg = *config;
  return guarded([&] {
    r.geometry = EBGridGeometry(config->nx, config->ny, config->nz, config->dx, config->dy,
                                config->dz, config->dt, EBMaxwellSolver::CowanZ);
    r.cpml.cells[0] = config->cpml_cells_x;
    r.cpml.cells[1] = config->cpml_cells_y;
    r.cpml.cells[2] = 0;
    r.cpml.polynomialOrder = config->cpml_polynomial_order;
    r.cpml.targetReflection = config->cpml_target_reflection;
    r.cpml.kappaMax = config->cpml_kappa_max;
    r.cpml.alphaFraction = config->cpml_alpha_fraction;
    r.fields.reset(new EBFieldGrid(r.geometry));
    for (unsigned a = 0; a < 6; ++a) {
      const YeeComponent& c = component(*r.fields, a);
      r.referenceShape[a][0] = c.nx();
      r.referenceShape[a][1] = c.ny();
      r.referenceShape[a][2] = config->reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0);
    }
    MovingWindowReference reference;
    reference.context = &r;
    reference.value = &referenceValue;
    r.window.reset(new MovingWindowFields(r.geometry, config->nz, 0, MPI_COMM_WORLD, r.cpml, reference));
    r.window->installBoundary(*r.fields);
    if (config->inlet_charge_match) {
      // Simulation::initializeMovingWindow (src/simulation_moving_window.cpp:300-303)
      const bool binomial3 = config->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
      r.inlet.reset(new ChargeMatchedInlet(r.geometry, config->cpml_cells_x, config->cpml_cells_y,
                                           !binomial3, false, binomial3, binomial3));
      r.window->setNewLayerCompletion(&completeInletLayer, &r, true);
    }
    char pattern[] = "/tmp/aprl_ref_XXXXXX";
    const char* dir = mkdtemp(pattern);
    if (!dir) throw std::runtime_error("Cannot create coupling log directory");
    r.directory = dir;
    const bool binomial = config->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
    r.coupling.reset(new ConservativeSourceCoupling(MPI_COMM_WORLD, r.directory, !binomial, false,
                                                    binomial, false, false, binomial));
    r.frame.setOriginsFromGamma(config->boost_gamma, SI::c, config->lab_time_origin,
                                config->lab_z_origin, config->box_z_origin);
    for (unsigned m = 0; m < config->n_magnets; ++m) {
      const aprl_magnet& g = config->magnets[m];
      SIMagneticElement e;
      e.type = g.type == APRL_MAGNET_PLANAR_UNDULATOR ? SIMagnetType::PlanarUndulator
               : (g.type == APRL_MAGNET_UNIFORM_DIPOLE ? SIMagnetType::UniformDipole
                                                       : SIMagnetType::Quadrupole);
      for (unsigned a = 0; a < 3; ++a) e.center[a] = g.center[a];
      e.length = g.length;
      e.period = g.period;
      e.peakMagneticField = g.peak_field;
      e.polarizationAngle = g.polarization_angle;
      e.gaussianFringe = g.gaussian_fringe != 0;
      e.fringeRelativeCutoff = g.fringe_relative_cutoff;
      e.quadrupoleGradient = g.quadrupole_gradient;
      e.prepare();
      r.sources.addPrescribedLabMagnet(e);
    }
    r.offset = config->initial_offset;
    r.origin[0] = config->reference_origin[0];
    r.origin[1] = config->reference_origin[1];
    r.origin[2] = std::fma(static_cast<double>(config->initial_offset), config->dz,
                           config->reference_origin[2]);
    *out = run.release();
  });
}

aprl_status ref_run_destroy(ref_run* r) {
  if (r) {
    if (!r->surfaceFile.empty()) ::unlink(r->surfaceFile.c_str());
    const std::string dir = r->directory;
    delete r;
    if (!dir.empty()) {
      std::string command = "rm -rf '" + dir + "'";
      if (std::system(command.c_str()) != 0) return failWith(APRL_ERR_RUNTIME, "cannot remove log directory");
    }
  }
  return APRL_OK;
}

aprl_status ref_set_threads(unsigned threads) {
  return guarded([&] { configureComputeThreads(MPI_THREAD_FUNNELED, static_cast<int>(threads)); });
}

aprl_status ref_run_set_reference(ref_run* r, unsigned a, const double* host, size_t count) {
  if (a >= 6) return failWith(APRL_ERR_OUT_OF_RANGE, "Moving-window component");
  const auto& s = r->referenceShape[a];
  if (count != s[0] * s[1] * s[2]) return failWith(APRL_ERR_INVALID_ARGUMENT, "Reference component size mismatch");
  if (host) r->reference[a].assign(host, host + count);
  else r->reference[a].assign(count, 0.0);  // the zero inlet
  return APRL_OK;
}

aprl_status ref_run_set_field(ref_run* r, unsigned a, const double* host, size_t count) {
  if (a >= 9) return failWith(APRL_ERR_OUT_OF_RANGE, "Field component");
  YeeComponent& c = component(*r->fields, a);
  if (count != c.size()) return failWith(APRL_ERR_INVALID_ARGUMENT, "Field component size mismatch");
  std::copy(host, host + count, c.data());
  return APRL_OK;
}

aprl_status ref_run_get_field(ref_run* r, unsigned a, double* host, size_t count) {
  if (a >= 9) return failWith(APRL_ERR_OUT_OF_RANGE, "Field component");
  YeeComponent& c = component(*r->fields, a);
  if (count != c.size()) return failWith(APRL_ERR_INVALID_ARGUMENT, "Field component size mismatch");
  std::copy(c.data(), c.data() + count, host);
  return APRL_OK;
}

aprl_status ref_run_history_length(ref_run* r, unsigned index, uint64_t* length) {
  return guarded([&] {
    EBConvolutionalPML& p = dynamic_cast<EBConvolutionalPML&>(r->fields->boundary());
    *length = p.checkpointHistory(index).size();
  });
}

aprl_status ref_run_set_history(ref_run* r, unsigned index, const double* host, size_t count) {
  return guarded([&] {
    EBConvolutionalPML& p = dynamic_cast<EBConvolutionalPML&>(r->fields->boundary());
    std::vector<Double>& h = p.checkpointHistory(index);
    if (h.size() != count) throw std::invalid_argument("CPML history size mismatch");
    std::copy(host, host + count, h.begin());
  });
}

aprl_status ref_run_get_history(ref_run* r, unsigned index, double* host, size_t count) {
  return guarded([&] {
    EBConvolutionalPML& p = dynamic_cast<EBConvolutionalPML&>(r->fields->boundary());
    const std::vector<Double>& h = p.checkpointHistory(index);
    if (h.size() != count) throw std::invalid_argument("CPML history size mismatch");
    std::copy(h.begin(), h.end(), host);
  });
}

aprl_status ref_run_set_particles(ref_run* r, size_t n, const double* x, const double* y,
                                  const double* z, const double* ux, const double* uy,
                                  const double* uz, const double* q, const double* m,
                                  const uint64_t* id, int resetCarriers) {
  r->particles.assign(n, RelativisticParticleSI());
  for (size_t i = 0; i < n; ++i) {
    RelativisticParticleSI& p = r->particles[i];
    p.position[0] = x[i]; p.position[1] = y[i]; p.position[2] = z[i];
    p.properVelocity[0] = ux[i]; p.properVelocity[1] = uy[i]; p.properVelocity[2] = uz[i];
    p.charge = q[i]; p.mass = m[i]; p.weight = 1.0; p.id = id[i]; p.sourceId = id[i];
    p.frozen = false; p.frozenBetaZ = 0.0;
  }
  if (resetCarriers) r->carriers.clear();
  return APRL_OK;
}

aprl_status ref_run_set_held(ref_run* r, size_t n, const uint8_t* frozen, const double* beta) {
  return guarded([&] {
    if (n != r->particles.size()) throw std::invalid_argument("Held state must cover the particle list");
    for (size_t i = 0; i < n; ++i) {
      r->particles[i].frozen = frozen[i] != 0;
      r->particles[i].frozenBetaZ = beta[i];
    }
    PendingWindowGeometry geometry;
    geometry.referenceOriginZ = r->cfg.reference_origin[2];
    geometry.initialOffset = r->cfg.initial_offset;
    geometry.dz = r->cfg.dz;
    geometry.heldDistancePerBeta = SI::c * r->cfg.dt;
    geometry.maximumStep = r->cfg.maximum_step;
    r->pending.reset(new PendingParticleQueue(geometry, r->step));
    r->pending->extract(r->particles);
  });
}

aprl_status ref_run_get_held(ref_run* r, size_t capacity, uint8_t* frozen, double* beta,
                             size_t* count) {
  if (capacity < r->particles.size()) return failWith(APRL_ERR_INVALID_ARGUMENT, "Particle buffer too small");
  for (size_t i = 0; i < r->particles.size(); ++i) {
    if (frozen) frozen[i] = r->particles[i].frozen ? 1 : 0;
    if (beta) beta[i] = r->particles[i].frozenBetaZ;
  }
  *count = r->particles.size();
  return APRL_OK;
}

aprl_status ref_run_particle_count(ref_run* r, size_t* count) {
  *count = r->particles.size();
  return APRL_OK;
}

aprl_status ref_run_get_particles(ref_run* r, size_t capacity, double* x, double* y, double* z,
                                  double* ux, double* uy, double* uz, double* q, double* m,
                                  uint64_t* id, size_t* count) {
  if (capacity < r->particles.size()) return failWith(APRL_ERR_INVALID_ARGUMENT, "Particle buffer too small");
  for (size_t i = 0; i < r->particles.size(); ++i) {
    const RelativisticParticleSI& p = r->particles[i];
    if (x) x[i] = p.position[0];
    if (y) y[i] = p.position[1];
    if (z) z[i] = p.position[2];
    if (ux) ux[i] = p.properVelocity[0];
    if (uy) uy[i] = p.properVelocity[1];
    if (uz) uz[i] = p.properVelocity[2];
    if (q) q[i] = p.charge;
    if (m) m[i] = p.mass;
    if (id) id[i] = p.id;
  }
  *count = r->particles.size();
  return APRL_OK;
}

aprl_status ref_run_carrier_count(ref_run* r, size_t* count) {
  *count = r->carriers.size();
  return APRL_OK;
}

aprl_status ref_run_get_carriers(ref_run* r, size_t capacity, double* pos, double* vel,
                                 double* q, double* w, size_t* count) {
  if (capacity < r->carriers.size()) return failWith(APRL_ERR_INVALID_ARGUMENT, "Carrier buffer too small");
  for (size_t i = 0; i < r->carriers.size(); ++i) {
    const ParticleCPMLCarrier& c = r->carriers[i];
    for (unsigned a = 0; a < 3; ++a) {
      if (pos) pos[3 * i + a] = c.position[a];
      if (vel) vel[3 * i + a] = c.velocity[a];
    }
    if (q) q[i] = c.charge;
    if (w) w[i] = c.currentWeight;
  }
  *count = r->carriers.size();
  return APRL_OK;
}

aprl_status ref_run_set_carriers(ref_run* r, size_t n, const double* pos, const double* vel,
                                 const double* q, const double* w) {
  r->carriers.assign(n, ParticleCPMLCarrier());
  for (size_t i = 0; i < n; ++i) {
    for (unsigned a = 0; a < 3; ++a) {
      r->carriers[i].position[a] = pos[3 * i + a];
      r->carriers[i].velocity[a] = vel[3 * i + a];
    }
    r->carriers[i].charge = q[i];
    r->carriers[i].currentWeight = w[i];
  }
  return APRL_OK;
}

aprl_status ref_run_advance_magnetic(ref_run* r) {
  return guarded([&] {
    if (r->stage != 0) throw std::logic_error("Moving-window beginStep phase/origin mismatch");
    if (r->pending) r->admitted += r->pending->admit(r->step, r->particles);
    r->fields->clearCurrent();
    r->window->beginStep(*r->fields, r->step, r->offset);
    const EBElectricHaloView halo = r->window->physicalElectricHalos(*r->fields, r->step);
    r->fields->advanceMagnetic(halo);
    r->stage = 1;
  });
}

aprl_status ref_run_preview_electric(ref_run* r) {
  return guarded([&] {
    if (r->stage != 1) throw std::logic_error("Moving-window electric phase mismatch");
    r->coupling->begin(*r->fields, r->origin, r->particles, r->cfg.cpml_cells_x, r->cfg.cpml_cells_y);
    r->window->previewElectricBoundary(true);
    r->fields->advanceElectric();
    r->window->previewElectricBoundary(false);
    save(*r);
    r->trials = 0;
    r->stage = 2;
  });
}

// TransverseReferenceCurrent::prepare's values (src/transverse_reference_current.cpp:
// 19-27, 46-63) from in-memory Bx and By tables of a reference grid of
// nz planes: curl_z(B_ref)/mu0 at the points() targets of every plane, plane
// by plane.  prepare_surface writes them in the reference's file format;
// ref_surface_current_pin holds them to the reference's own prepare.
std::vector<double> surface_values(const aprl_run_config& c, std::size_t nz,
                                   const std::vector<double>& bx, const std::size_t sx[3],
                                   const std::vector<double>& by, const std::size_t sy[3],
                                   std::size_t& count) {
  const std::size_t gx = c.cpml_cells_x, gy = c.cpml_cells_y;
  const std::size_t x0 = gx, x1 = c.nx - gx, y0 = gy, y1 = c.ny - gy;
  std::vector<std::pair<std::size_t, std::size_t>> target;
  for (std::size_t i = x0; i <= x1; ++i) {
    target.push_back({i, y0});
    target.push_back({i, y1});
  }
  for (std::size_t j = y0 + 1; j < y1; ++j) {
    target.push_back({x0, j});
    target.push_back({x1, j});
  }
  count = target.size();
  std::vector<double> values(nz * count);
  for (std::size_t k = 0; k < nz; ++k)
    for (std::size_t p = 0; p < count; ++p) {
      const std::size_t i = target[p].first, j = target[p].second;
      const double dby = by.at((k * sy[1] + j) * sy[0] + i) - by.at((k * sy[1] + j) * sy[0] + i - 1);
      const double dbx = bx.at((k * sx[1] + j) * sx[0] + i) - bx.at((k * sx[1] + j - 1) * sx[0] + i);
      values[k * count + p] = (dby / c.dx - dbx / c.dy) / SI::mu0;
      if (!std::isfinite(values[k * count + p]))
        throw std::runtime_error("Nonfinite equivalent boundary current");
    }
  return values;
}

// The file of TransverseReferenceCurrent::prepare (header, the values, the
// completion marker) written from the run's reference tables; then the
// reference's class opens it.
void prepare_surface(ref_run& r) {
  if (r.surface) return;
  const aprl_run_config& c = r.cfg;
  const std::size_t gx = c.cpml_cells_x, gy = c.cpml_cells_y;
  std::size_t count = 0;
  const std::vector<double> values = surface_values(c, c.reference_nz, r.reference[3],
                                                    r.referenceShape[3], r.reference[4],
                                                    r.referenceShape[4], count);
  struct Header {
    std::uint64_t tag, version, nx, ny, nz, gx, gy, count;
    double dx, dy, dz, dt, beta;
  };
  const bool binomial3 = c.shape == APRL_SHAPE_LINEAR_BINOMIAL3;
  const Header h{0x4150524c53555246ULL, binomial3 ? 2ULL : 1ULL, c.nx, c.ny, c.reference_nz,
                 gx, gy, count, c.dx, c.dy, c.dz, c.dt, 0.0};
  char name[] = "/tmp/aprl-surface-XXXXXX";
  const int fd = ::mkstemp(name);
  if (fd < 0) throw std::runtime_error("Cannot create reference surface-current file");
  bool ok = ::write(fd, &h, sizeof h) == (ssize_t)sizeof h;
  const ssize_t bytes = (ssize_t)(values.size() * sizeof(double));
  ok = ok && ::write(fd, values.data(), values.size() * sizeof(double)) == bytes;
  const std::uint64_t complete = 0x434f4d504c455445ULL;
  ok = ok && ::write(fd, &complete, sizeof complete) == (ssize_t)sizeof complete;
  ::close(fd);
  if (!ok) {
    ::unlink(name);
    throw std::runtime_error("Cannot write reference surface current");
  }
  r.surfaceFile = name;
  const EBGridGeometry g(c.nx, c.ny, c.reference_nz, c.dx, c.dy, c.dz, c.dt,
                         EBMaxwellSolver::CowanZ);
  const std::size_t guards[3] = {gx, gy, 0};
  r.surface.reset(new aprl::TransverseReferenceCurrent(name, g, guards, 0.0, "", binomial3));
}

void apply_surface(ref_run& r) {
  if (!r.cfg.reference_surface_current) return;
  prepare_surface(r);
  r.surface->apply(*r.fields, r.offset, r.step, r.cfg.translation_beta, false);
}

void finish_surface(ref_run& r) {
  if (r.cfg.reference_surface_current && r.surface) r.surface->finish(*r.fields);
}

aprl_status ref_run_coupling_trial(ref_run* r, double residual[4]) {
  return guarded([&] {
    if (r->stage != 2 && r->stage != 3) throw std::logic_error("Coupling trial requires a previewed electric field");
    if (r->trials) r->coupling->applyCurrentSource(1.);
    r->fields->clearCurrent();
    restore(*r);
    r->coupling->beginTrial();
    r->coupling->exchangeCandidate();
    pushDepositAndMigrate(*r);
    r->coupling->completeCurrent();
    // src/simulation_source_coupling.cpp:44
    apply_surface(*r);
    finish_surface(*r);
    r->coupling->applyCurrentSource(-1.);
    r->coupling->exchangeCandidate();
    const auto res = r->coupling->localResidual();
    for (int i = 0; i < 4; ++i) residual[i] = res[i];
    ++r->trials;
    r->stage = 3;
  });
}

aprl_status ref_run_commit_electric(ref_run* r) {
  return guarded([&] {
    if (r->stage != 3) throw std::logic_error("Commit requires a completed coupling trial");
    r->coupling->applyCurrentSource(1.);
    r->fields->clearCurrent();
    restore(*r);
    r->coupling->swapElectric();
    r->coupling->setReplay(true);
    pushDepositAndMigrate(*r);
    r->coupling->completeCurrent();
    r->coupling->setReplay(false);
    r->coupling->finish(r->step + 1, r->lastIterations, r->lastForce, r->lastWork);
    // applyMovingTransverseReferenceCurrent before the commit, finish after
    // (src/simulation.cpp:548-549, 560-561)
    apply_surface(*r);
    r->coupling->swapElectric();
    r->window->undoPreviewElectricBoundary(*r->fields);
    r->coupling->applyCurrentSource(-1.);
    r->window->commitPreparedElectricBoundary(*r->fields);
    finish_surface(*r);
    r->stage = 4;
  });
}

aprl_status ref_run_shift(ref_run* r) {
  return guarded([&] {
    if (r->stage != 4) throw std::logic_error("Moving-window requires one left shift after each complete step");
    // Simulation calls this after the electric step, before the shift
    // (src/simulation.cpp:3490-3493).
    if (r->ledger) r->window->finishEnergyLedgerStep(*r->fields);
    r->time += r->cfg.dt;
    ++r->step;
    r->offset = r->cfg.initial_offset - static_cast<std::ptrdiff_t>(r->step);
    r->window->shift(*r->fields, r->step, r->offset);
    r->origin[2] = std::fma(static_cast<double>(r->offset), r->cfg.dz, r->cfg.reference_origin[2]);
    for (const auto& p : r->particles)
      if (p.position[2] < r->origin[2] && !p.frozen)
        throw std::runtime_error("Active particle fell behind moving inlet");
    const double upper = std::fma(static_cast<double>(r->cfg.nz), r->cfg.dz, r->origin[2]);
    std::size_t kept = 0;
    for (const auto& c : r->carriers) {
      if (c.position[2] >= upper) {
        ++r->croppedCarriers;
        r->croppedCharge += c.charge * c.currentWeight;
      } else if (c.position[2] < r->origin[2]) {
        throw std::runtime_error("Current carrier fell behind moving inlet");
      } else {
        r->carriers[kept++] = c;
      }
    }
    r->carriers.resize(kept);
    r->stage = 0;
  });
}

aprl_status ref_run_step(ref_run* r, uint32_t steps) {
  for (uint32_t n = 0; n < steps; ++n) {
    aprl_status s = ref_run_advance_magnetic(r);
    if (s != APRL_OK) return s;
    s = ref_run_preview_electric(r);
    if (s != APRL_OK) return s;
    bool converged = false;
    unsigned iterations = 0;
    double force = 0., work = 0.;
    for (unsigned t = 0; t < r->cfg.max_trials; ++t) {
      double res[4];
      s = ref_run_coupling_trial(r, res);
      if (s != APRL_OK) return s;
      force = res[0];
      work = res[3] == 0. ? 0. : (res[2] > 0. ? res[1] / res[2] : res[1]);
      iterations = t + 1;
      if (iterations >= (res[3] > 0. ? 2u : 1u) && force < r->cfg.force_tolerance &&
          work < r->cfg.work_tolerance) {
        converged = true;
        break;
      }
    }
    if (!converged) return failWith(APRL_ERR_NOT_CONVERGED, "Conservative source coupling failed");
    r->lastIterations = iterations;
    r->maxIterations = std::max(r->maxIterations, iterations);
    r->totalIterations += iterations;
    r->lastForce = force;
    r->lastWork = work;
    s = ref_run_commit_electric(r);
    if (s != APRL_OK) return s;
    s = ref_run_shift(r);
    if (s != APRL_OK) return s;
  }
  return APRL_OK;
}

aprl_status ref_run_get_stats(ref_run* r, aprl_step_stats* st) {
  std::memset(st, 0, sizeof *st);
  st->step = r->step;
  st->iterations = r->lastIterations;
  st->max_iterations = r->maxIterations;
  st->total_iterations = r->totalIterations;
  st->force = r->lastForce;
  st->work = r->lastWork;
  st->particles = r->particles.size();
  st->carriers = r->carriers.size();
  st->exits = r->exits;
  st->exit_charge = r->exitCharge;
  for (int f = 0; f < 6; ++f) {
    st->cpml_entries[f] = r->counts[0][f];
    st->cpml_entry_charge[f] = r->charges[0][f];
    st->carrier_outer[f] = r->counts[2][f];
    st->carrier_outer_charge[f] = r->charges[2][f];
  }
  st->cropped_carriers = r->croppedCarriers;
  st->cropped_charge = r->croppedCharge;
  st->window_offset = r->offset;
  st->origin_z = r->origin[2];
  st->time_box = r->time;
  st->pending = r->pending ? r->pending->size() : 0;
  st->admitted = r->admitted;
  st->activations = r->activations;
  for (const auto& p : r->particles) st->held += p.frozen ? 1 : 0;
  return APRL_OK;
}

// Direct operator probes on the reference's own kernels.
long ref_shape_weights(const aprl_run_config* config, const double origin[3], const double begin[3],
                       const double end[3], int32_t* axis, int64_t* index, double* weight,
                       long capacity) {
  try {
    EBGridGeometry g(config->nx, config->ny, config->nz, config->dx, config->dy, config->dz,
                     config->dt, EBMaxwellSolver::CowanZ);
    Vec o, b, e;
    for (unsigned a = 0; a < 3; ++a) { o[a] = origin[a]; b[a] = begin[a]; e[a] = end[a]; }
    long count = 0;
    const bool binomial = config->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
    longitudinal_shape::weights(g, o, b, e, [&](unsigned d, long long i, long long j, long long k, double w) {
      if (count < capacity) {
        axis[count] = static_cast<int32_t>(d);
        index[3 * count] = i; index[3 * count + 1] = j; index[3 * count + 2] = k;
        weight[count] = w;
      }
      ++count;
    }, binomial ? longitudinal_shape::Shape::LinearBinomial3 : longitudinal_shape::Shape::QuinticCompensated, binomial);
    return count;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

int ref_momentum(double u[3], const double e[3], const double b[3], double q, double m, double h,
                 double knownGamma) {
  try {
    Vec uu, ee, bb;
    for (unsigned a = 0; a < 3; ++a) { uu[a] = u[a]; ee[a] = e[a]; bb[a] = b[a]; }
    const unsigned it = source_coupling_math::momentum(uu, ee, bb, q, m, h, knownGamma);
    for (unsigned a = 0; a < 3; ++a) u[a] = uu[a];
    return static_cast<int>(it);
  } catch (const std::exception& ex) {
    g_error = ex.what();
    return -1;
  }
}

// The reference's own RelativisticBorisPusher::push, particle by particle.
aprl_status ref_boris_push(size_t count, double* x, double* y, double* z, double* ux, double* uy,
                           double* uz, const double* charge, const double* mass,
                           const double* electric, const double* magnetic, double dt) {
  try {
    for (size_t n = 0; n < count; ++n) {
      aprl::RelativisticParticleSI p;
      p.position[0] = x[n]; p.position[1] = y[n]; p.position[2] = z[n];
      p.properVelocity[0] = ux[n]; p.properVelocity[1] = uy[n]; p.properVelocity[2] = uz[n];
      p.charge = charge[n];
      p.mass = mass[n];
      Vec e, b;
      for (unsigned a = 0; a < 3; ++a) {
        e[a] = electric[3 * n + a];
        b[a] = magnetic[3 * n + a];
      }
      aprl::RelativisticBorisPusher::push(p, e, b, dt);
      x[n] = p.position[0]; y[n] = p.position[1]; z[n] = p.position[2];
      ux[n] = p.properVelocity[0]; uy[n] = p.properVelocity[1]; uz[n] = p.properVelocity[2];
    }
    return APRL_OK;
  } catch (const std::invalid_argument& ex) {
    g_error = ex.what();
    return APRL_ERR_INVALID_ARGUMENT;
  } catch (const std::exception& ex) {
    g_error = ex.what();
    return APRL_ERR_RUNTIME;
  }
}

double ref_gamma(const double u[3]) {
  Vec uu;
  for (unsigned a = 0; a < 3; ++a) uu[a] = u[a];
  return BoostFrameTransform::gammaFromProperVelocity(uu);
}

aprl_status ref_prescribed_box(ref_run* r, const double position[3], double time, double e[3],
                               double b[3]) {
  return guarded([&] {
    Vec p, ee(0.), bb(0.);
    for (unsigned a = 0; a < 3; ++a) p[a] = position[a];
    r->sources.addPrescribedBox(p, time, r->frame, ee, bb);
    for (unsigned a = 0; a < 3; ++a) { e[a] = ee[a]; b[a] = bb[a]; }
  });
}

aprl_status ref_cowan_coefficients(double dx, double dy, double dz, double out[12]) {
  return guarded([&] {
    const EBCowanCoefficients c = EBCowanCoefficients::forZDispersion(dx, dy, dz);
    for (int a = 0; a < 3; ++a) { out[a] = c.alpha[a]; out[3 + a] = c.beta[a]; out[9 + a] = c.ratio[a]; }
    out[6] = c.deltaXY; out[7] = c.deltaYZ; out[8] = c.deltaZX;
  });
}

aprl_status ref_run_enable_energy_ledger(ref_run* r, int enabled) {
  return guarded([&] {
    r->window->enableEnergyLedger(enabled != 0);
    r->ledger = enabled != 0;
  });
}

// MovingWindowFields::energyLedger plus the field and particle sums of
// Simulation's ledger record at one rank: localInteriorFieldEnergy
// (src/simulation.cpp:3308-3340), boundaryPower's loops
// (src/moving_window_fields.cpp:399-423) and the particle loop
// (src/simulation.cpp:3591-3604), over the reference's own cell operators.
aprl_status ref_run_energy_ledger(ref_run* r, aprl_energy_ledger* out) {
  return guarded([&] {
    std::memset(out, 0, sizeof *out);
    const MovingWindowFieldEnergyLedger& l = r->window->energyLedger();
    out->inlet_overwrite_energy = static_cast<double>(l.inletOverwriteEnergyJ);
    out->inserted_energy = static_cast<double>(l.insertedEnergyJ);
    out->cropped_energy = static_cast<double>(l.croppedEnergyJ);
    out->remap_energy = static_cast<double>(l.remapEnergyJ);
    for (int f = 0; f < 6; ++f) out->outward_energy[f] = static_cast<double>(l.outwardEnergyFace[f]);
    out->overwrite_events = l.overwriteEvents;
    out->flux_steps = l.fluxSteps;
    out->remap_steps = l.remapSteps;
    const EBGridGeometry& g = r->geometry;
    const std::size_t i0 = r->cfg.cpml_cells_x, i1 = g.nx - i0;
    const std::size_t j0 = r->cfg.cpml_cells_y, j1 = g.ny - j0;
    const long double volume = static_cast<long double>(g.dx) *
                               static_cast<long double>(g.dy) * static_cast<long double>(g.dz);
    long double energy = 0.L;
    for (std::size_t k = 0; k < g.nz; ++k)
      for (std::size_t j = j0; j < j1; ++j)
        for (std::size_t i = i0; i < i1; ++i)
          energy += static_cast<long double>(r->fields->fieldEnergyDensityCell(i, j, k)) * volume;
    out->field_energy_interior = static_cast<double>(energy);
    long double power[6] = {};
    const long double yz = static_cast<long double>(g.dy) * g.dz;
    const long double xz = static_cast<long double>(g.dx) * g.dz;
    const long double xy = static_cast<long double>(g.dx) * g.dy;
    for (std::size_t k = 0; k < g.nz; ++k) {
      for (std::size_t j = j0; j < j1; ++j) {
        power[0] -= static_cast<long double>(r->fields->poyntingComponentCell(i0, j, k, 0)) * yz;
        power[1] += static_cast<long double>(r->fields->poyntingComponentCell(i1 - 1, j, k, 0)) * yz;
      }
      for (std::size_t i = i0; i < i1; ++i) {
        power[2] -= static_cast<long double>(r->fields->poyntingComponentCell(i, j0, k, 1)) * xz;
        power[3] += static_cast<long double>(r->fields->poyntingComponentCell(i, j1 - 1, k, 1)) * xz;
      }
    }
    for (std::size_t j = j0; j < j1; ++j)
      for (std::size_t i = i0; i < i1; ++i) {
        power[4] -= static_cast<long double>(r->fields->poyntingComponentCell(i, j, 0, 2)) * xy;
        power[5] += static_cast<long double>(r->fields->poyntingComponentCell(i, j, g.nz - 1, 2)) * xy;
      }
    for (int f = 0; f < 6; ++f) out->boundary_power[f] = static_cast<double>(power[f]);
    long double kinetic = 0.L, total = 0.L, represented = 0.L;
    for (const auto& p : r->particles) {
      const Double gammaBox = BoostFrameTransform::gammaFromProperVelocity(p.properVelocity);
      const long double mass = static_cast<long double>(p.mass);
      const long double c = static_cast<long double>(SI::c);
      const long double rest = mass * c * c;
      const long double u2 = static_cast<long double>(p.properVelocity.norm2());
      kinetic += rest * u2 / static_cast<long double>(gammaBox + 1.0);
      total += rest * static_cast<long double>(gammaBox);
      represented += mass / static_cast<long double>(SI::electronMass);
    }
    out->particle_kinetic = static_cast<double>(kinetic);
    out->particle_total = static_cast<double>(total);
    out->represented_electrons = static_cast<double>(represented);
    out->particles = r->particles.size();
  });
}

// EBGaussFieldInitializer::initialize at one rank on the run's particles.
// The reference's own BlockedCowanReference (src/blocked_cowan_reference.h:
// 59-130), built here over the FFTW stand-in of fftw_shim/, on a reference
// grid of config->nx x ny x reference_nz cells from reference_origin: its
// charge deposit, transverse-mode solve and native E/B, read back with
// field() into the six tables (x fastest, the layout of
// aprl_run_set_reference).  shape 0 deposits CIC; shape 1 the run's own
// shape as the moving window prepares its reference
// (src/simulation_moving_window.cpp:145-148 with src/config.cpp:1084-1112):
// linear-binomial3 in z with the binomial3 transverse x weights, or the
// quintic-compensated node basis in z.  open: the open-transverse-wall
// variant (openTransverse; guards must then be the CPML cells in x and y and
// 0 in z).  `directory` must not exist: the reference creates it, and its
// files are removed afterwards.  report: source charge, deposited charge,
// minimum Thomas pivot, minimum mode eigenvalue, and for the open variant
// the wall table's largest checked interpolation error and its fallback
// tiles.
aprl_status ref_blocked_reference(const aprl_run_config* config, size_t n, const double* x,
                                  const double* y, const double* z, const double* charge,
                                  double beta, const uint64_t guards[3], uint64_t block_layers,
                                  int shape, int open, const char* directory,
                                  double* const tables[6], double report[6]) {
  return guarded([&] {
    const EBGridGeometry g(config->nx, config->ny, config->reference_nz, config->dx, config->dy,
                           config->dz, config->dt, EBMaxwellSolver::CowanZ);
    Vec origin;
    for (unsigned a = 0; a < 3; ++a) origin[a] = config->reference_origin[a];
    std::vector<RelativisticParticleSI> particles(n);
    for (size_t i = 0; i < n; ++i) {
      particles[i].position[0] = x[i];
      particles[i].position[1] = y[i];
      particles[i].position[2] = z[i];
      particles[i].charge = charge[i];
      particles[i].id = i;
    }
    const bool shaped = shape != 0;
    const bool binomial = config->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
    const std::size_t guard[3] = {guards[0], guards[1], guards[2]};
    const std::string dir(directory);
    {
      verification::BlockedCowanReference ref(
          g, origin, particles, beta, guard, block_layers, dir, MPI_COMM_SELF,
          shaped && !binomial, false, shaped && binomial, shaped && binomial, open != 0);
      const std::size_t nx[6] = {g.nx, g.nx + 1, g.nx + 1, g.nx + 1, g.nx, g.nx};
      const std::size_t ny[6] = {g.ny + 1, g.ny, g.ny + 1, g.ny, g.ny + 1, g.ny};
      const std::size_t nz[6] = {g.nz + 1, g.nz + 1, g.nz, g.nz, g.nz, g.nz + 1};
      for (unsigned c = 0; c < 6; ++c)
        for (std::size_t k = 0; k < nz[c]; ++k)
          for (std::size_t j = 0; j < ny[c]; ++j)
            for (std::size_t i = 0; i < nx[c]; ++i)
              tables[c][(k * ny[c] + j) * nx[c] + i] = ref.field(c, i, j, k);
      const auto& rep = ref.report();
      report[0] = rep.sourceCharge;
      report[1] = rep.depositedCharge;
      report[2] = rep.minimumPivot;
      report[3] = rep.minimumModeEigenvalue;
      report[4] = rep.openTraceMaxRelativeError;
      report[5] = (double)rep.openTraceFallbackTiles;
    }
    for (const char* name :
         {"/rho.bin", "/checkpoints.bin", "/phi.bin", "/metadata.txt", "/side-potential.bin"})
      (void)::unlink((dir + name).c_str());
    (void)::rmdir(dir.c_str());
  });
}

// The reference's own TransverseReferenceCurrent::prepare
// (src/transverse_reference_current.cpp:46-63) over its own
// BlockedCowanReference of the bunch (shaped source, guards = the CPML
// cells, as src/simulation_moving_window.cpp:145-157 prepares both), and the
// values surface_values forms from that reference's Bx and By tables, each
// `count` points per plane over reference_nz planes.
aprl_status ref_surface_current_pin(const aprl_run_config* config, size_t n, const double* x,
                                    const double* y, const double* z, const double* charge,
                                    double beta, uint64_t block_layers, const char* directory,
                                    double* from_reference, double* from_tables,
                                    size_t capacity, size_t* count) {
  return guarded([&] {
    const EBGridGeometry g(config->nx, config->ny, config->reference_nz, config->dx, config->dy,
                           config->dz, config->dt, EBMaxwellSolver::CowanZ);
    Vec origin;
    for (unsigned a = 0; a < 3; ++a) origin[a] = config->reference_origin[a];
    std::vector<RelativisticParticleSI> particles(n);
    for (size_t i = 0; i < n; ++i) {
      particles[i].position[0] = x[i];
      particles[i].position[1] = y[i];
      particles[i].position[2] = z[i];
      particles[i].charge = charge[i];
      particles[i].id = i;
    }
    const bool binomial = config->shape == APRL_SHAPE_LINEAR_BINOMIAL3;
    const std::size_t guard[3] = {config->cpml_cells_x, config->cpml_cells_y, 0};
    const std::string dir(directory), file = dir + "/transverse-current.bin";
    {
      verification::BlockedCowanReference ref(g, origin, particles, beta, guard, block_layers,
                                               dir, MPI_COMM_SELF, !binomial, false, binomial,
                                               binomial, false);
      TransverseReferenceCurrent::prepare(file, ref, g, guard, beta, binomial);
      std::vector<double> bx, by;
      const std::size_t sx[3] = {g.nx + 1, g.ny, g.nz}, sy[3] = {g.nx, g.ny + 1, g.nz};
      bx.resize(sx[0] * sx[1] * sx[2]);
      by.resize(sy[0] * sy[1] * sy[2]);
      for (std::size_t k = 0; k < g.nz; ++k)
        for (std::size_t j = 0; j < g.ny + 1; ++j)
          for (std::size_t i = 0; i < g.nx + 1; ++i) {
            if (j < g.ny) bx[(k * sx[1] + j) * sx[0] + i] = ref.field(3, i, j, k);
            if (i < g.nx) by[(k * sy[1] + j) * sy[0] + i] = ref.field(4, i, j, k);
          }
      std::size_t points = 0;
      const std::vector<double> mine = surface_values(*config, g.nz, bx, sx, by, sy, points);
      *count = points;
      if (mine.size() > capacity) throw std::invalid_argument("surface-current capacity too small");
      std::copy(mine.begin(), mine.end(), from_tables);
      // the reference's file: header (8 words + 5 doubles), values, marker
      std::ifstream in(file, std::ios::binary);
      in.seekg(13 * 8);
      in.read(reinterpret_cast<char*>(from_reference), (std::streamsize)(mine.size() * 8));
      if (!in) throw std::runtime_error("Cannot read the reference's surface-current file");
    }
    for (const char* name : {"/transverse-current.bin", "/rho.bin", "/checkpoints.bin",
                             "/phi.bin", "/metadata.txt"})
      (void)::unlink((dir + name).c_str());
    (void)::rmdir(dir.c_str());
  });
}

aprl_status ref_run_initialize_self_field(ref_run* r, const aprl_self_field_config* c,
                                          aprl_self_field_report* out) {
  return guarded([&] {
    std::memset(out, 0, sizeof *out);
    const InitialSelfFieldModel model =
        c->model == APRL_SELF_FIELD_COWAN_RELATIVISTIC_POISSON
            ? InitialSelfFieldModel::CowanRelativisticPoisson
            : (c->model == APRL_SELF_FIELD_ELECTROSTATIC_POISSON
                   ? InitialSelfFieldModel::ElectrostaticPoisson
                   : InitialSelfFieldModel::RelativisticPoisson);
    const std::size_t guard[3] = {c->guard_cells[0], c->guard_cells[1], c->guard_cells[2]};
    const EBGaussInitializationReport rep = EBGaussFieldInitializer::initialize(
        *r->fields, r->geometry, 0, r->origin, r->particles, model,
        c->maximum_mean_transverse_beta, guard, c->relative_tolerance, c->maximum_iterations,
        MPI_COMM_WORLD, c->include_transverse_cpml_particles != 0,
        c->hold_transverse_until_activation != 0, &r->frame);
    out->iterations = rep.iterations;
    out->relative_residual = rep.relativeResidual;
    out->maximum_gauss_residual = rep.maximumGaussResidual;
    out->total_charge = rep.totalCharge;
    out->mean_beta_z = rep.meanBetaZ;
    out->mean_beta_transverse = rep.meanBetaTransverse;
    out->initial_electric_energy = rep.initialElectricEnergy;
    out->initial_magnetic_energy = rep.initialMagneticEnergy;
    for (int a = 0; a < 3; ++a) {
      out->rms_position_cells[a] = rep.rmsPositionCells[a];
      out->centre_padding_rms[a] = rep.centrePaddingRms[a];
      out->static_field_guard_cells[a] = rep.staticFieldGuardCells[a];
    }
    out->transverse_poisson_padding_cells = rep.transversePoissonPaddingCells;
    out->temporary_bytes = rep.temporaryBytes;
  });
}

}  // extern "C"
