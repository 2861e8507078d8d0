// NVTX ranges around the library's launches and eigenray-search rounds, so a
// timeline from Nsight Systems (or ncu --nvtx filtering) shows which entry
// point and round a kernel belongs to.  Header-only NVTX3: without an attached
// tool each range is a no-op call.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace iga_internal {

struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace iga_internal
