// naga/cospan/cospan.hpp — the cs:: API on the cspb runtime (B200, sm_100a): include this, as with the reference.
#pragma once

#include <sycl/sycl.hpp>

#include "naga/slabkit/slabkit.hpp"

#include "core.hpp"
#include "component.hpp"
#include "system.hpp"
#include "model.hpp"
#include "patterns.hpp"
#include "finalize.hpp"
