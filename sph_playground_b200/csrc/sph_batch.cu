// Batches of independent instances (include/sph_abi.h, "batches of
// instances").  When every instance can take device-resident steps, the
// batch steps as one device loop (sph::batch_graph_run: a CUDA graph whose
// while node iterates one if node per instance, each holding that
// instance's captured step, with per-instance clocks and error words on the
// device); otherwise one host worker per instance runs that instance's time
// loop on its own stream, so that the kernels and host round trips of the
// instances overlap on the device.
//
// The reference runs such sweeps one Context after another (the experiment
// runners, e.g. runner/000_anisopaper_v1_gls_kxx.py, through
// CleanRun / ContinueRun, core.py:152-156); every instance here computes
// exactly what sph_step / sph_run_to compute for it alone.
#include <algorithm>
#include <condition_variable>
#include <limits>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "sph_abi.h"
#include "sph_internal.h"

struct sph_batch {
  std::vector<sph_handle*> h;
  std::vector<int> status;
  std::vector<std::string> msg;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_go, cv_done;
  std::function<int(sph_handle*)> job;  // the current call's work for one instance
  long long generation = 0;             // bumped per call
  int pending = 0;
  bool quit = false;
  sph::BatchGraph* bg = nullptr;  // the device loop, built on first use

  // the device loop over all instances; *used = false when it does not apply
  int device_loop(double tfinish, bool use_state, long long limit, bool* used) {
    // start the instances that have not run yet on the host workers, side
    // by side (the start-up iterate of main.f90 runs on the host path, with
    // its round trips); an instance that fails there is reported below
    constexpr int kStateTfinish = 11;  // the state slot of tfinish (const.f90 ec_tfinish)
    if (!use_state)
      for (auto* x : h) sph_set_param(x, kStateTfinish, tfinish);
    run([](sph_handle* x) { return sph::start_for_device_loop(x); });
    std::vector<int> st0 = status;
    std::vector<std::string> msg0 = msg;
    std::fill(status.begin(), status.end(), 0);
    std::fill(msg.begin(), msg.end(), std::string());
    int rc = sph::batch_graph_run(&bg, h.data(), int(h.size()), tfinish, use_state, limit, status,
                                  msg, used);
    for (size_t i = 0; i < h.size(); ++i)
      if (st0[i] && !status[i]) {
        status[i] = st0[i];
        msg[i] = msg0[i];
      }
    if (rc || !*used) return rc;
    for (size_t i = 0; i < h.size(); ++i)
      if (status[i]) return sph::sph_fail(status[i], "instance " + std::to_string(i) + ": " + msg[i]);
    return SPH_OK;
  }

  void worker(int i) {
    cudaSetDevice(sph::handle_device(h[i]));
    long long seen = 0;
    for (;;) {
      std::function<int(sph_handle*)> fn;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_go.wait(lk, [&] { return quit || generation != seen; });
        if (quit) return;
        seen = generation;
        fn = job;
      }
      const int rc = fn(h[i]);
      std::string m = rc ? std::string(sph_last_error()) : std::string();
      {
        std::lock_guard<std::mutex> lk(mu);
        status[i] = rc;
        msg[i] = m;
        if (--pending == 0) cv_done.notify_all();
      }
    }
  }

  int run(std::function<int(sph_handle*)> fn) {
    {
      std::unique_lock<std::mutex> lk(mu);
      job = std::move(fn);
      pending = int(h.size());
      ++generation;
    }
    cv_go.notify_all();
    std::unique_lock<std::mutex> lk(mu);
    cv_done.wait(lk, [&] { return pending == 0; });
    for (size_t i = 0; i < h.size(); ++i)
      if (status[i]) return sph::sph_fail(status[i], "instance " + std::to_string(i) + ": " + msg[i]);
    return SPH_OK;
  }
};

extern "C" {

int sph_batch_create(int n_inst, sph_handle* const* handles, sph_batch** out) {
  if (!out || !handles || n_inst <= 0) return sph::sph_fail(SPH_ERR_ARG, "bad batch arguments");
  for (int i = 0; i < n_inst; ++i) {
    if (!handles[i]) return sph::sph_fail(SPH_ERR_ARG, "null handle in batch");
    for (int j = 0; j < i; ++j)
      if (handles[j] == handles[i]) return sph::sph_fail(SPH_ERR_ARG, "handle twice in batch");
  }
  auto* b = new sph_batch();
  b->h.assign(handles, handles + n_inst);
  b->status.assign(n_inst, 0);
  b->msg.assign(n_inst, std::string());
  try {
    for (int i = 0; i < n_inst; ++i) b->workers.emplace_back(&sph_batch::worker, b, i);
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(b->mu);
      b->quit = true;
    }
    b->cv_go.notify_all();
    for (auto& t : b->workers) t.join();
    delete b;
    return sph::sph_fail(SPH_ERR_OOM, "could not start the batch workers");
  }
  *out = b;
  return SPH_OK;
}

int sph_batch_step(sph_batch* b, int nsteps) {
  if (!b || nsteps < 0) return sph::sph_fail(SPH_ERR_ARG, "bad argument");
  bool used = false;
  int rc = b->device_loop(0.0, true, nsteps, &used);
  if (used || rc) return rc;
  return b->run([nsteps](sph_handle* h) { return sph_step(h, nsteps); });
}

int sph_batch_run_to(sph_batch* b, double tfinish) {
  if (!b) return sph::sph_fail(SPH_ERR_ARG, "null batch");
  bool used = false;
  int rc = b->device_loop(tfinish, false, std::numeric_limits<long long>::max(), &used);
  if (used || rc) return rc;
  return b->run([tfinish](sph_handle* h) { return sph_run_to(h, tfinish); });
}

int sph_batch_status(sph_batch* b, int* status, int n) {
  if (!b || !status) return sph::sph_fail(SPH_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(b->mu);
  for (int i = 0; i < n && i < int(b->status.size()); ++i) status[i] = b->status[i];
  return SPH_OK;
}

void sph_batch_destroy(sph_batch* b) {
  if (!b) return;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->quit = true;
  }
  b->cv_go.notify_all();
  for (auto& t : b->workers) t.join();
  sph::batch_graph_destroy(b->bg);
  delete b;
}

}  // extern "C"
