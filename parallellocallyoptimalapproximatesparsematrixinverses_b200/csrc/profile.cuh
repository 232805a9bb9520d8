#pragma once
// Opt-in, event-based accounting of the library's kernel classes.  When
// enabled (spai_profile_enable), every profiled launch site records a CUDA
// event pair on its own stream plus the algorithmic bytes the launch must
// move; spai_profile_read sums elapsed times and bytes per class.  Disabled,
// a scope costs one branch.

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace spai {
namespace prof {

bool Enabled();
void SetEnabled(bool on);
void Reset();
// Adds algorithmic bytes to a class after the fact (for a launch whose output
// size is only known once it has run).
void AddBytes(const char* name, double bytes);
// Totals for one class: elapsed milliseconds, launches, algorithmic bytes.
bool Read(const std::string& name, double* ms, int64_t* count, double* bytes);

class Scope {
 public:
  Scope(cudaStream_t stream, const char* name, double bytes);
  ~Scope();
  Scope(const Scope&) = delete;
  Scope& operator=(const Scope&) = delete;

 private:
  cudaStream_t stream_;
  const char* name_;
  double bytes_;
  cudaEvent_t start_ = nullptr;
  bool active_ = false;
};

}  // namespace prof
}  // namespace spai
