// Oracle shim for DACTI's scene/scene.hpp (src/lib/scene/scene.hpp:10-62).
//
// The Integrator constructor calls Scene::init_domain and adaptive refinement calls
// Scene::can_split (integrator/integrator.hpp:95, impl/adaptive_refinement.hpp:75-76).
// init_domain here rebuilds the tree slot by slot from a flat case file, so the reference starts
// from exactly the tree the GPU path is given; can_split keeps the reference's rule
// (scene/scene.hpp:50-61).
#pragma once

#include "../../case_io.hpp"
#include "config/config.hpp"
#include "integrator/boundary.hpp"
#include "integrator/domain.hpp"
#include <unordered_set>

namespace dacti::scene {

	template<typename M>
	class Scene {
	private:
		using vecn_t   = linalg::vec<scalar_t, M::NumDims>;
		using domain_t = integrator::_internal::Domain<M>;
		using node_t   = integrator::_internal::Node<M>;
		using bnd_t    = integrator::Boundary<M>;

	public:
		const std::shared_ptr<config::Config<M>> config;

		Scene(std::shared_ptr<config::Config<M>> config) :
		    config(config) {}

		void init_domain(domain_t &domain) {
			const oracle::CaseData &c = *config->case_data;
			constexpr int D  = M::NumDims;
			constexpr int E  = M::NumEqns;
			constexpr int C  = 1 << D;
			constexpr int NF = 2 * D;

			domain.tree.resize(c.n_nodes);
			for (int i = 1; i < c.n_nodes; ++i) {
				node_t n{};
				n.parent_index = c.parent[i];
				for (int k = 0; k < C; ++k) n.child_indices[k] = c.children[i * C + k];
				n.tree_level = c.level[i];
				n.acti_level = -1;
				uint32_t fl  = c.flags[i];
				n.is_leaf      = fl & oracle::F_LEAF;
				n.is_active    = fl & oracle::F_ACTIVE;
				n.is_garbage   = fl & oracle::F_GARBAGE;
				n.can_split    = fl & oracle::F_CAN_SPLIT;
				n.can_unsplit  = fl & oracle::F_CAN_UNSPLIT;
				n.should_split = fl & oracle::F_SHOULD_SPLIT;
				n.is_boundary  = fl & oracle::F_IS_BOUNDARY;
				n.error        = -1.0;
				n.op           = integrator::_internal::creation_op::INIT;
				n.neighbors.fill(0);
				n.boundaries.fill(std::nullopt);
				for (int f = 0; f < NF; ++f) {
					int b = c.bc[i * NF + f];
					if (b >= 0) {
						const auto &e = c.bcs[b];
						bnd_t bd;
						bd.type = static_cast<typename bnd_t::Type>(e.type);
						for (int q = 0; q < E; ++q) bd.p_in[q] = e.p_in[q];
						for (int d = 0; d < D; ++d) bd.normal[d] = e.normal[d];
						bd.fade_in               = e.fade_in;
						n.boundaries.array[f]    = bd;
					}
				}
				// Cell sizes halve exactly per level from the root (integrator/domain.hpp:47,207).
				scalar_t size = config->side_length;
				for (int l = 0; l < n.tree_level; ++l) size = 0.5 * size;
				n.cell.size = size;
				n.cell.t    = 0.0;
				for (int d = 0; d < D; ++d) n.cell.center[d] = c.center[i * D + d];
				for (int q = 0; q < E; ++q) n.cell.p[q] = c.p[i * E + q];
				domain.tree[i] = n;
			}
		}

		bool can_split(vecn_t x, size_t current_level) {
			if (current_level < config->max_refinement_level)
				return true;

			for (const auto &zone: config->refine_zones) {
				if (current_level < zone.refinement_level && zone.contains(x.template project<3>())) {
					return true;
				}
			}

			return false;
		}
	};

}    // namespace dacti::scene
