// Named ranges for a profiler's timeline (NVTX, header-only; inert unless a
// tool is attached): equilibration, solve setup, the persistent launches,
// presolve and MPS input.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace prima {

struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace prima
