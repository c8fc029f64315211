// NVTX ranges around the recipe's stages (the reference marks its timed
// iterations with one NVTX range, bench/profile.cu:31-34). NVTX 3 is header
// only: without a profiler attached a range costs a few nanoseconds and
// records nothing.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <cstdio>

namespace qpb {

class NvtxRange {
 public:
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  // "<what> <n>", e.g. "RAAR 50"
  NvtxRange(const char* what, int n) {
    char name[64];
    std::snprintf(name, sizeof(name), "%s %d", what, n);
    nvtxRangePushA(name);
  }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
  ~NvtxRange() { nvtxRangePop(); }
};

}  // namespace qpb
