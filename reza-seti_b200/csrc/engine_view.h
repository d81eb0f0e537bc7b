// Read-only view of an engine's host-side node data, for the result writers.
#pragma once

#include <cstdint>

#include "lbm_b200.h"

namespace lbm {

struct EngineView {
    int64_t n = 0;                    // nodes
    const int32_t* coords = nullptr;  // [n][3], caller order
    int64_t n_nw = 0;
    const int64_t* nearwall = nullptr;  // [n_nw] caller node indices
    int Q = 19;
};

bool engine_view(const lbm_engine* e, EngineView& v);

}  // namespace lbm
