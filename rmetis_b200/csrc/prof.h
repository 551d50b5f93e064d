// Per-launch device timing with CUDA events (off unless enabled). Used by the
// benchmark to measure the dominant kernel's average launch duration on the
// stream it runs on.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

namespace rmb {

enum ProfId {
  kProfGain = 0,      // k_gain: gain table of one refinement pass
  kProfDecide,        // k_decide / k_decide_seq
  kProfPropose,       // k_match_propose
  kProfContract,      // k_contract_thread
  kProfCut,           // k_cut
  kProfGrow,          // k_grow
  kProfLevel,         // k_refine_level: all passes of a small level in one launch
  kProfTail,          // k_coarsen_tail: the remaining coarsening levels of a small graph
  kProfAdmit,         // k_admit_pick + k_admit: one cut pass decided by parallel admission
  kProfCount
};

struct ProfTotals {
  long long launches[kProfCount];
  double ms[kProfCount];
  double bytes[kProfCount];
};

class Profiler {
 public:
  bool on = false;
  int begin(int id, cudaStream_t st);
  void end(int handle, cudaStream_t st, double bytes);
  // Sets the algorithmic bytes of a recorded launch after the fact (for
  // launches whose size is only known on the device when they are queued).
  void set_bytes(int handle, double bytes) {
    std::lock_guard<std::mutex> lk(mu_);
    if (handle >= 0 && handle < (int)recs_.size()) recs_[handle].bytes = bytes;
  }
  // Synchronises on the recorded events and adds them to the totals.
  void collect();
  void reset();
  ProfTotals totals{};

 private:
  struct Rec {
    int id;
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<Rec> recs_;
  std::mutex mu_;  // worker threads record launches concurrently
  std::vector<cudaEvent_t> pool_;
  cudaEvent_t get();
};

Profiler& profiler();

}  // namespace rmb
