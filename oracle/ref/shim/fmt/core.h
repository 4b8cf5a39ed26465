// Oracle shim. DACTI's integrator/domain.hpp:6 includes <fmt/core.h> for its debug dumps;
// spdlog's bundled fmt provides the same API.
#pragma once
#include <spdlog/fmt/fmt.h>
