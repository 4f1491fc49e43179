// nvtx_range.h — NVTX ranges around the engine's host-side phases (training
// call, binning, boosting rounds, one tree, prediction), so a timeline from
// Nsight Systems or an `ncu --nvtx` filter groups the kernels by phase.
// NVTX3 is header-only: without a tool attached, a push/pop is one check of
// an unset function pointer.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace bst {

struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace bst

#define BST_NVTX_CAT2(a, b) a##b
#define BST_NVTX_CAT(a, b) BST_NVTX_CAT2(a, b)
#define BST_RANGE(name) ::bst::NvtxRange BST_NVTX_CAT(bst_nvtx_range_, __LINE__)(name)
