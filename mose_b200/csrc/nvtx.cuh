// nvtx.cuh -- NVTX ranges around the C-ABI entry points, so a timeline
// profiler shows each Fortran-side call (Fill_Ghost_Cell, Fluxes, ...) with
// the kernels it enqueued.  NVTX 3 is header-only: without a tool attached
// the range calls return at once and nothing is loaded.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace mose {
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace mose

#define MOSE_NVTX_RANGE(name) ::mose::NvtxRange mose_nvtx_range_(name)
