// Definition of the opaque handle of the C ABI (shared by the C-ABI translation units).
#pragma once
#include <memory>
#include <string>

#include "swc_batch.h"
#include "swc_engine.h"

namespace swc {
// Sets the message returned by swc_last_error() on this thread.
void set_last_error(const std::string &msg);
}  // namespace swc

struct swc_handle {
  std::unique_ptr<swc::Engine> eng;
  int device = 0;
  bool analyzed = false;
  bool factored = false;
  int plan = 0;                             // execution-plan candidate (swc_set_plan)
  std::unique_ptr<swc::BatchState> batch;   // set by swc_batch_analyze
};
