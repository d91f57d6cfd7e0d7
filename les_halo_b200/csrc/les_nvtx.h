// les_nvtx.h -- NVTX ranges around the library's host entry points.
//
// Every C-ABI call that does work opens a range named after itself for the
// length of the call (RAII, so every early error return closes it too); the
// time step adds one range per step and one around its graph capture and the
// SOR autotuner.  NVTX v3 is header-only: without a tool attached
// (NVTX_INJECTION64_PATH unset) each push/pop is one call through a null
// function pointer, so the ranges stay in the shipped library.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace les {

struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace les

#define LES_RANGE_CAT2(a, b) a##b
#define LES_RANGE_CAT(a, b) LES_RANGE_CAT2(a, b)
#define LES_RANGE(name) ::les::NvtxRange LES_RANGE_CAT(les_nvtx_range_, __LINE__)(name)
