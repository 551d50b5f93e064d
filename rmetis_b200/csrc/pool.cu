// Worker pool: concurrent partitions on one device (the attempts of one call,
// the graphs of a batch, asynchronous requests).
#include <atomic>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "engine.h"

namespace rmb {

size_t footprint_bytes(int64_t n, int64_t m, int k, int ncon) {
  // Input (xadj, adjncy, adjwgt, vwgt), the coarse hierarchy (about 1.5x the
  // input), refinement scratch per level (mover records, candidates, flags)
  // and the grow trials on the coarsest graph; rounded up generously.
  const int64_t input = 4 * (n + 1) + 8 * m + 4 * n * ncon;
  const int64_t hierarchy = input * 3 / 2 + 16 * n;
  // (+ the parallel admission's per-mover target, rank, slot and sums)
  const int64_t refine = 88 * n + 12 * n + 8 * n * ncon + 8 * m + 24 * (int64_t)k * ncon;
  const int64_t grow = 32 * (16 * std::max<int64_t>(20 * (int64_t)k, 20) * 4);
  return (size_t)(input + hierarchy + refine + grow + ((int64_t)64 << 20));
}

size_t arena_cap_bytes() {
  static const size_t cap = [] {
    const char* e = std::getenv("RMETIS_B200_ARENA_CAP");
    return e ? (size_t)std::strtoull(e, nullptr, 10) : (size_t)0;
  }();
  return cap;
}

bool arena_cap_reserve(int device, long long delta) {
  static std::atomic<long long> used[64];
  if (device < 0 || device >= 64) return false;
  const long long now = used[device].fetch_add(delta) + delta;
  if (delta > 0 && now > (long long)arena_cap_bytes()) {
    used[device].fetch_sub(delta);
    return false;
  }
  return true;
}

WorkerPool::WorkerPool(int device, int nworkers, size_t budget_bytes)
    : device_(device), budget_(budget_bytes), worker_epoch_(nworkers, 0) {
  for (int i = 0; i < nworkers; ++i) threads_.emplace_back([this, i] { worker_main(i); });
}

WorkerPool::~WorkerPool() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  for (auto& t : threads_)
    if (t.joinable()) t.join();
}

void WorkerPool::set_budget(size_t b) {
  {
    std::lock_guard<std::mutex> lk(mu_);
    budget_ = b;
  }
  cv_.notify_all();
}

std::future<int> WorkerPool::submit(size_t footprint, std::function<int(Engine&)> fn) {
  auto job = std::make_unique<Job>();
  job->footprint = footprint;
  job->fn = std::move(fn);
  std::future<int> f = job->prom.get_future();
  {
    std::lock_guard<std::mutex> lk(mu_);
    queue_.push_back(std::move(job));
  }
  cv_.notify_all();
  return f;
}

void WorkerPool::worker_main(int idx) {
  cudaSetDevice(device_);
  std::unique_ptr<Engine> engine;
  try {
    engine = std::make_unique<Engine>(/*is_worker=*/true);
  } catch (...) {
    engine.reset();  // every job this thread takes then fails with METIS_ERROR
  }
  auto free_workspace = [&] {
    if (!engine) return;
    cudaStreamSynchronize(engine->stream());
    engine->arena().release();
  };
  unsigned my_epoch = 0;
  for (;;) {
    std::unique_ptr<Job> job;
    bool trim = false;
    {
      std::unique_lock<std::mutex> lk(mu_);
      // Admission in submission order: the head starts when its footprint
      // fits next to the running jobs, or when nothing runs (a retried job
      // only then, and only once every worker has freed its workspace).
      cv_.wait(lk, [&] {
        if (stop_ || my_epoch != trim_epoch_) return true;
        if (queue_.empty()) return false;
        const Job& h = *queue_.front();
        if (h.alone) {
          if (running_ != 0) return false;
          for (unsigned e : worker_epoch_)
            if (e != trim_epoch_) return false;
          return true;
        }
        return running_ == 0 || in_use_ + h.footprint <= budget_;
      });
      if (stop_) return;
      if (my_epoch != trim_epoch_) {
        my_epoch = trim_epoch_;
        trim = true;
      } else {
        job = std::move(queue_.front());
        queue_.pop_front();
        in_use_ += job->footprint;
        ++running_;
      }
    }
    if (trim) {
      free_workspace();
      {
        std::lock_guard<std::mutex> lk(mu_);
        worker_epoch_[idx] = my_epoch;
      }
      cv_.notify_all();
      continue;
    }
    int rc = -4;
    if (engine) {
      try {
        rc = job->fn(*engine);
      } catch (const Error& e) {
        rc = e.code;
      } catch (const std::bad_alloc&) {
        rc = -3;
      } catch (...) {
        rc = -4;
      }
      // A failed job must not leave its workspace half used.
      engine->arena().rewind();
    }
    bool retry = false;
    {
      std::lock_guard<std::mutex> lk(mu_);
      in_use_ -= job->footprint;
      --running_;
      if (rc == -3 && !job->alone && engine) {
        // Out of device memory next to other jobs: every worker frees its
        // workspace, and this job runs again with nothing beside it.
        retry = true;
        ++trim_epoch_;
        my_epoch = trim_epoch_;
      }
    }
    if (retry) {
      free_workspace();
      if (std::getenv("RMETIS_B200_VERBOSE"))
        std::fprintf(stderr, "rmetis_b200: a job ran out of device memory beside others; retrying it alone\n");
      std::lock_guard<std::mutex> lk(mu_);
      worker_epoch_[idx] = my_epoch;
      job->alone = true;
      queue_.push_front(std::move(job));
    }
    cv_.notify_all();
    if (!retry) job->prom.set_value(rc);
  }
}

WorkerPool& pool_for_device(int device) {
  static std::mutex m;
  static std::vector<WorkerPool*> pools;
  std::lock_guard<std::mutex> lk(m);
  if ((int)pools.size() <= device) pools.resize(device + 1, nullptr);
  if (!pools[device]) {
    int n = 8;
    if (const char* e = std::getenv("RMETIS_B200_WORKERS")) n = std::max(1, std::atoi(e));
    size_t budget = (size_t)150 << 30;
    if (const char* e = std::getenv("RMETIS_B200_POOL_BYTES")) budget = (size_t)std::strtoull(e, nullptr, 10);
    pools[device] = new WorkerPool(device, n, budget);  // lives until process exit
  }
  return *pools[device];
}

}  // namespace rmb
