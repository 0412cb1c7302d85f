// Batched path: many independent matrices as one block-diagonal structure (swc_batch.cu).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "swc_engine.h"

namespace swc {

// Relaxation parameters of a supernode partition (meaning as in supernode_partition).
struct PartitionParams {
  int nrelax[3];
  double zrelax[3];
  int max_width;
};

struct BatchState {
  int nmat = 0, N = 0;
  std::vector<int64_t> col_off;     // first column of each matrix in the block-diagonal order
  std::vector<int> cp, ri;          // block-diagonal lower CSC
  uint64_t key = 0;                 // structure hash (autotuner cache key)
  int partition = 0;                // chosen candidates
  Tuning plan;
  int64_t *d_seg = nullptr;         // device copy of col_off
  ~BatchState();
  bool set(int nmat, const int *n, const int *c, const int *r, std::string &err);
  bool analyze(Engine &eng, int partition, const Tuning &t, std::string &err);
  // Times every candidate on the device values (factor of the whole batch, mean of reps
  // runs after one warm-up) and leaves the engine analysed with the best one.
  bool autotune(Engine &eng, const double *d_values, int mode, const char *cache_path, int reps,
                int *choice, double *best_ms, std::string &err);
};

// Execution-plan candidates of the autotuner (also selectable with swc_set_plan).
Tuning plan_candidate(int k);
int num_plans();

}  // namespace swc
