// Optional per-launch timing of the library's own kernels with CUDA events on
// the launching stream.  Off by default; maxi_profile_enable(1) turns it on,
// maxi_profile_read() waits for the recorded events and returns the summed
// device time and launch count per kernel kind.
#pragma once

#include <cuda_runtime.h>

namespace maxi {

bool profiling_enabled();
void profile_record(int kind, cudaEvent_t start, cudaEvent_t stop);
cudaEvent_t profile_event();

// Brackets one kernel launch: records a start event in the constructor and a
// stop event in the destructor, on `st`, when profiling is on.
class ProfScope {
  public:
    ProfScope(int kind, cudaStream_t st) : kind_(kind), st_(st) {
        if (profiling_enabled()) {
            start_ = profile_event();
            cudaEventRecord(start_, st_);
        }
    }
    ~ProfScope() {
        if (start_) {
            cudaEvent_t stop = profile_event();
            cudaEventRecord(stop, st_);
            profile_record(kind_, start_, stop);
        }
    }

  private:
    int kind_;
    cudaStream_t st_;
    cudaEvent_t start_ = nullptr;
};

}  // namespace maxi
