// Scoped per-phase device timer: records a CUDA event pair on the library
// stream around a phase when timers are enabled (rmpcd_timers_enable), the
// device-side counterpart of the reference's tic/tac timers
// (src/common.f90:353-363).
#pragma once
#include <cuda_runtime.h>

namespace rmpcd {

// whether phase timers are on (their event records must not be captured
// into CUDA graphs)
bool timers_on();

class PhaseTimer {
  public:
    explicit PhaseTimer(const char *name);
    ~PhaseTimer();
    PhaseTimer(const PhaseTimer &) = delete;
    PhaseTimer &operator=(const PhaseTimer &) = delete;

  private:
    int idx_ = -1;
    cudaEvent_t a_ = nullptr;
};

}  // namespace rmpcd
