// Oracle shim for DACTI's config/config.hpp (src/lib/config/config.hpp:11-117).
//
// Holds the Config fields that the hot path reads: side_length, active_size, IsPeriodic,
// error_threshold, error_weights, max/min refinement level, max_dt, max_cfl
// (integrator/integrator.hpp:80-86, impl/flux.hpp:68-74) and refine_zones (scene/scene.hpp:54-58),
// plus the run fields of the default driver loop.
// The runner fills them from a flat case file instead of a TOML case.
#pragma once

#include "integrator/boundary.hpp"
#include <array>
#include <memory>
#include <string>
#include <vector>

namespace oracle {
	struct CaseData;
}

namespace dacti::config {

	template<typename M>
	class Config {
	public:
		using vecn_t = typename M::vecn_t;
		using prim_t = typename M::prim_t;

		vecn_t active_size;
		scalar_t side_length = 1.0;
		scalar_t max_cfl     = 0.5;
		scalar_t max_dt      = 1.0;

		int min_refinement_level = 0;
		int max_refinement_level = 0;
		vec2_t error_threshold;
		prim_t error_weights;

		std::array<bool, M::NumDims> IsPeriodic{};

		// Refinement box with an identity transform (config/config.hpp:77-86 with Transform = id).
		struct RefineZone {
			vec3_t x0, x1;
			size_t refinement_level;

			[[nodiscard]] bool contains(const vec3_t &x) const {
				return x.cwiseLesserThan(x1).all() && x.cwiseGreaterThan(x0).all();
			}
		};
		std::vector<RefineZone> refine_zones;

		// run fields that driver/default_driver.hpp reads (config/config.hpp:28-36)
		std::string case_name       = "case";
		std::string result_out_dir  = ".";
		scalar_t io_interval        = 0.0;
		scalar_t end_time           = 0.0;
		scalar_t signal_time        = -1.0;
		scalar_t convergence_tol    = -1.0;

		const oracle::CaseData *case_data = nullptr;
	};
}    // namespace dacti::config
