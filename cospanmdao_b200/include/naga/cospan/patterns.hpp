// naga/cospan/patterns.hpp — leaves that run as one cspb kernel (filled in below the generic path).
#pragma once

#include "model.hpp"

namespace naga::cospan::detail {
inline void register_patterns(Runtime& rt) { rt.pattern_at.assign(rt.leaves.size(), -1); }
}  // namespace naga::cospan::detail
