// scan.cu -- parameter-scan server: independent runs kept resident on one
// GPU and overlapped on separate streams.
//
// Requests wait in one FIFO queue.  A worker thread (a slot, with its own
// CUDA stream) takes the head request as soon as the head's estimated device
// footprint fits the budget next to the runs already admitted, builds an
// aprl_run on its stream, steps it, samples the detector plane, frees the
// run and returns the memory.  Requests that arrive while others are on the
// GPU are admitted as slots and memory free up, so their kernels overlap.
// The head of the queue is never overtaken, so a large request cannot be
// starved by smaller ones behind it.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/aprl_gpu.h"

namespace aprl_gpu {
aprl_status report_error(aprl_status status, const char* message);
const char* run_error(const aprl_run* r);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  uint64_t ticket = 0;
  aprl_scan_request request{};
  uint64_t footprint = 0;
  int state = APRL_SCAN_QUEUED;
  aprl_scan_result result{};
  Clock::time_point submitted, started, finished;
};

aprl_status scan_fail(aprl_status s, const char* message) {
  return aprl_gpu::report_error(s, message);
}

size_t component_count(const aprl_run_config& c, int a, bool electric) {
  const uint64_t n[3] = {c.nx, c.ny, c.nz};
  size_t count = 1;
  for (int d = 0; d < 3; ++d) count *= (size_t)(n[d] + (electric ? (d != a) : (d == a)));
  return count;
}

// Device bytes of one run, following aprl_run_create and the particle and
// carrier capacities a step uses.
uint64_t footprint(const aprl_run_config& c, size_t particles) {
  const size_t fes = c.precision == APRL_PRECISION_FP32_MIXED ? 4 : 8;
  uint64_t bytes = 0;
  for (int a = 0; a < 3; ++a) {
    bytes += 3 * component_count(c, a, true) * fes;   // E^n, E*, J
    bytes += component_count(c, a, false) * fes;      // B
    bytes += (c.nx + 1) * (c.ny + 1) * fes;           // inlet halo plane
  }
  // CPML histories: at most 2*cells slots of one plane row per layer, 8 terms.
  const uint64_t cells = std::max(c.cpml_cells_x, c.cpml_cells_y);
  bytes += 8 * 2 * cells * (std::max(c.nx, c.ny) + 1) * (c.nz + 1) * fes;
  // Inlet reference table (binary64), six components.
  for (int a = 0; a < 6; ++a) {
    const bool electric = a < 3;
    const int axis = a % 3;
    const size_t plane = (size_t)(c.nx + (electric ? axis != 0 : axis == 0)) *
                         (c.ny + (electric ? axis != 1 : axis == 1));
    bytes += plane * (c.reference_nz + 1) * 8;
  }
  // Particles (two state copies, trial outputs, slots, newborn carriers,
  // sort scratch) and a carrier allowance of a quarter of the particles (at
  // least the 4096 carriers a run reserves up front).
  bytes += (uint64_t)particles * 480 +
           (std::max<uint64_t>(particles / 4, 4096) + 1024) * 3 * 80;
  // Cell sort and scan scratch, reductions.
  bytes += (uint64_t)c.nx * c.ny * c.nz * 8 + (32ull << 20);
  return bytes;
}

double seconds_since(Clock::time_point origin, Clock::time_point t) {
  return std::chrono::duration<double>(t - origin).count();
}

}  // namespace

struct aprl_scan {
  int device = 0;
  uint64_t budget = 0;
  uint64_t in_use = 0;
  bool stopping = false;
  uint64_t next_ticket = 1;
  Clock::time_point origin = Clock::now();
  std::mutex mutex;
  std::condition_variable changed;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<uint64_t, std::shared_ptr<Job>> jobs;
  std::vector<std::thread> workers;

  uint32_t runs_per_slot = 1;

  void work(int slot);
  aprl_run* start_job(Job& job, int slot, cudaStream_t stream);
  void end_job(Job& job, aprl_run* run, aprl_status s);
};

// A request's run: created on `stream`, inlet tables and particles set.
// Returns nullptr (with the failure in the job's result) when that fails.
aprl_run* aprl_scan::start_job(Job& job, int slot, cudaStream_t stream) {
  const aprl_scan_request& q = job.request;
  job.result.slot = slot;
  aprl_run* run = nullptr;
  aprl_status s = aprl_run_create(&q.config, stream, &run);
  for (unsigned a = 0; a < 6 && s == APRL_OK; ++a) {
    const bool electric = a < 3;
    const int axis = (int)(a % 3);
    const size_t count = (size_t)(q.config.nx + (electric ? axis != 0 : axis == 0)) *
                         (q.config.ny + (electric ? axis != 1 : axis == 1)) *
                         (q.config.reference_nz + ((a == 0 || a == 1 || a == 5) ? 1 : 0));
    s = aprl_run_set_reference(run, a, q.reference[a], count);  // NULL: zero inlet
  }
  if (s == APRL_OK)
    s = aprl_run_set_particles(run, q.particles, q.x, q.y, q.z, q.ux, q.uy, q.uz, q.charge,
                               q.mass, q.id, 1);
  if (s == APRL_OK && q.frozen)
    s = aprl_run_set_held(run, q.particles, q.frozen, q.frozen_beta_z);
  if (s != APRL_OK) {
    end_job(job, run, s);
    return nullptr;
  }
  return run;
}

// The detector plane and statistics of a finished run (or its failure),
// then the run is destroyed.
void aprl_scan::end_job(Job& job, aprl_run* run, aprl_status s) {
  const aprl_scan_request& q = job.request;
  aprl_scan_result& res = job.result;
  int inside = 0;
  if (s == APRL_OK && q.detector)
    s = aprl_run_sample_field_plane(run, q.detector_lab_z, q.detector,
                                    (size_t)(6 * q.config.nx * q.config.ny), &inside);
  if (run) aprl_run_get_stats(run, &res.stats);
  res.status = s;
  res.detector_inside = inside;
  if (s != APRL_OK) std::snprintf(res.message, sizeof res.message, "%s", aprl_last_error());
  if (run) aprl_run_destroy(run);
}

// A worker steps a group of up to runs_per_slot runs in lock step.  At every
// step boundary it admits queue heads that fit the budget into free places
// of the group (FIFO, the head never overtaken) and retires the runs that
// have taken their steps, so requests join and leave a running group.
void aprl_scan::work(int slot) {
  cudaSetDevice(device);
  const size_t capacity = std::max<uint32_t>(1u, runs_per_slot);
  std::vector<cudaStream_t> streams(capacity, nullptr);
  for (auto& st : streams) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  struct Active {
    std::shared_ptr<Job> job;
    aprl_run* run;
    size_t place;
    uint64_t done;
  };
  std::vector<Active> group;
  std::vector<bool> busy(capacity, false);
  auto retire = [&](Active& a, aprl_status s) {
    end_job(*a.job, a.run, s);
    busy[a.place] = false;
    {
      std::lock_guard<std::mutex> lock(mutex);
      a.job->finished = Clock::now();
      a.job->state = APRL_SCAN_DONE;
      in_use -= a.job->footprint;
    }
    changed.notify_all();
  };
  for (;;) {
    std::vector<std::shared_ptr<Job>> admitted;
    {
      std::unique_lock<std::mutex> lock(mutex);
      if (group.empty())
        changed.wait(lock, [&] {
          return (!queue.empty() && in_use + queue.front()->footprint <= budget) ||
                 (stopping && queue.empty());
        });
      if (group.empty() && queue.empty()) break;
      while (group.size() + admitted.size() < capacity && !queue.empty() &&
             in_use + queue.front()->footprint <= budget) {
        auto job = queue.front();
        queue.pop_front();
        in_use += job->footprint;
        job->state = APRL_SCAN_RUNNING;
        job->started = Clock::now();
        admitted.push_back(job);
      }
    }
    if (!admitted.empty()) changed.notify_all();
    for (auto& job : admitted) {
      size_t place = 0;
      while (busy[place]) ++place;
      busy[place] = true;
      Active a{job, nullptr, place, 0};
      a.run = start_job(*job, slot, streams[place]);
      if (!a.run) {
        busy[place] = false;
        std::lock_guard<std::mutex> lock(mutex);
        job->finished = Clock::now();
        job->state = APRL_SCAN_DONE;
        in_use -= job->footprint;
        continue;
      }
      if (job->request.steps == 0) {
        retire(a, APRL_OK);
        continue;
      }
      group.push_back(a);
    }
    if (group.empty()) {
      changed.notify_all();
      continue;
    }
    std::vector<aprl_run*> runs(group.size());
    std::vector<aprl_status> status(group.size(), APRL_OK);
    for (size_t i = 0; i < group.size(); ++i) runs[i] = group[i].run;
    aprl_runs_step(runs.data(), runs.size(), 1, status.data());
    std::vector<Active> next;
    for (size_t i = 0; i < group.size(); ++i) {
      Active& a = group[i];
      if (status[i] != APRL_OK) {
        aprl_gpu::report_error(status[i], aprl_gpu::run_error(a.run));
        retire(a, status[i]);
      } else if (++a.done >= a.job->request.steps) {
        retire(a, APRL_OK);
      } else {
        next.push_back(a);
      }
    }
    group.swap(next);
  }
  for (auto& st : streams)
    if (st) cudaStreamDestroy(st);
}

extern "C" {

aprl_status aprl_scan_footprint(const aprl_run_config* config, size_t particles,
                                uint64_t* bytes) {
  if (!config || !bytes) return scan_fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = footprint(*config, particles);
  return APRL_OK;
}

aprl_status aprl_scan_create(const aprl_scan_config* config, aprl_scan** out) {
  if (!config || !out) return scan_fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (config->max_slots < 1 || config->max_slots > 256)
    return scan_fail(APRL_ERR_INVALID_ARGUMENT, "A scan needs 1..256 slots");
  aprl_scan* scan = new (std::nothrow) aprl_scan();
  if (!scan) return scan_fail(APRL_ERR_RUNTIME, "out of host memory");
  if (cudaGetDevice(&scan->device) != cudaSuccess) {
    delete scan;
    return scan_fail(APRL_ERR_CUDA, "No current CUDA device for the scan");
  }
  scan->budget = config->device_budget_bytes;
  scan->runs_per_slot = std::max<uint32_t>(1u, config->runs_per_slot);
  if (scan->budget == 0) {
    size_t free_bytes = 0, total = 0;
    if (cudaMemGetInfo(&free_bytes, &total) != cudaSuccess) {
      delete scan;
      return scan_fail(APRL_ERR_CUDA, "cudaMemGetInfo failed");
    }
    scan->budget = (uint64_t)(0.9 * (double)free_bytes);
  }
  for (uint32_t s = 0; s < config->max_slots; ++s)
    scan->workers.emplace_back([scan, s] { scan->work((int)s); });
  *out = scan;
  return APRL_OK;
}

aprl_status aprl_scan_submit(aprl_scan* scan, const aprl_scan_request* request,
                             uint64_t* ticket) {
  if (!scan || !request || !ticket) return scan_fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  const uint64_t bytes = footprint(request->config, request->particles);
  auto job = std::make_shared<Job>();
  job->request = *request;
  job->footprint = bytes;
  job->result.footprint_bytes = bytes;
  {
    std::lock_guard<std::mutex> lock(scan->mutex);
    if (scan->stopping) return scan_fail(APRL_ERR_RUNTIME, "The scan is shutting down");
    if (bytes > scan->budget) {
      char message[160];
      std::snprintf(message, sizeof message,
                    "Run footprint of %llu bytes exceeds the scan's device budget of %llu bytes",
                    (unsigned long long)bytes, (unsigned long long)scan->budget);
      return scan_fail(APRL_ERR_OUT_OF_RANGE, message);
    }
    job->ticket = scan->next_ticket++;
    job->submitted = Clock::now();
    scan->queue.push_back(job);
    scan->jobs[job->ticket] = job;
    *ticket = job->ticket;
  }
  scan->changed.notify_all();
  return APRL_OK;
}

aprl_status aprl_scan_wait(aprl_scan* scan, uint64_t ticket, double timeout_seconds,
                           aprl_scan_result* result) {
  if (!scan || !result) return scan_fail(APRL_ERR_INVALID_ARGUMENT, "null argument");
  std::unique_lock<std::mutex> lock(scan->mutex);
  auto it = scan->jobs.find(ticket);
  if (it == scan->jobs.end()) return scan_fail(APRL_ERR_INVALID_ARGUMENT, "Unknown scan ticket");
  std::shared_ptr<Job> job = it->second;
  const auto deadline =
      Clock::now() + std::chrono::duration_cast<Clock::duration>(
                         std::chrono::duration<double>(std::max(0.0, timeout_seconds)));
  scan->changed.wait_until(lock, deadline, [&] { return job->state == APRL_SCAN_DONE; });
  *result = job->result;
  result->state = job->state;
  result->submit_s = seconds_since(scan->origin, job->submitted);
  if (job->state != APRL_SCAN_QUEUED) {
    result->start_s = seconds_since(scan->origin, job->started);
    result->queued_ms = 1e3 * (result->start_s - result->submit_s);
  }
  if (job->state == APRL_SCAN_DONE) {
    result->finish_s = seconds_since(scan->origin, job->finished);
    result->run_ms = 1e3 * (result->finish_s - result->start_s);
    result->total_ms = 1e3 * (result->finish_s - result->submit_s);
    scan->jobs.erase(it);
  }
  return APRL_OK;
}

aprl_status aprl_scan_destroy(aprl_scan* scan) {
  if (!scan) return APRL_OK;
  {
    std::lock_guard<std::mutex> lock(scan->mutex);
    scan->stopping = true;
  }
  scan->changed.notify_all();
  for (auto& t : scan->workers) t.join();
  delete scan;
  return APRL_OK;
}

}  // extern "C"
