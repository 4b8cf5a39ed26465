/*
 * dacti_gpu/integrator.hpp — header-only C++ adapter that re-exposes the API of DACTI's
 * dacti::integrator::Integrator<Model, Limiter, ErrorEstimator> (src/lib/integrator/integrator.hpp:
 * 14-225) on top of the C ABI in dacti_gpu.h.
 *
 * Include it inside a DACTI build (the reference's src/lib on the include path) and replace
 *     dacti::integrator::Integrator<M, L, E>    with    dacti::gpu::Integrator<M, L, E>
 * in the driver. Construction, integrate() with its substep hook and force_break flag,
 * n_active_cells(), for_each_active_cell() and the public counters keep their names and meaning:
 *
 *   - the constructor takes the same (Limiter, ErrorEstimator, Scene&, shared_ptr<Config>) and lets
 *     Scene::init_domain build the initial tree on the host exactly as the reference does
 *     (integrator/integrator.hpp:72-95); the tree is then flattened and handed to dg_create, which
 *     performs the rest of the constructor on the GPU;
 *   - integrate(hook, signal, force_break) advances one global step (impl/integrate.hpp:12-87) and
 *     calls hook(*this, level, acti_time, n_substeps, dt_level) after every level substep; inside the
 *     hook acti_clusters[level].size() is the size of the cluster that just ran;
 *   - for_each_active_cell(action) calls action(i, node) with reference Node<Model> objects holding
 *     the active cells' state (cell.center/size/t/u/p/k, tree_level, acti_level, error, max_dt, cfl),
 *     clusters 0..15 then buffers 0..15, the reference's order (integrator/integrator.hpp:172-191);
 *     they are read back once per global step, on first use.
 *
 * Differences, all outside the solver step: the tree lives on the GPU, so get_domain() does not
 * exist and `domain` holds root_index only; get_nodes() returns the whole tree renumbered breadth
 * first from the root (slot 1), with links, flags, p and metadata per node; get_node()/get_cell_index()
 * index the active cells (1-based, 0 being the null node as in the reference); acti_clusters[l] and
 * acti_buffers[l] expose
 * size() only. Refinement zones must be axis-aligned (no rotation in their Transform). Model
 * constants are read from the model's statics when the Integrator is constructed. Errors of the C
 * ABI surface as std::runtime_error, the reference's error type for configuration errors
 * (config/util.hpp:26); NaN still ends a step through force_break. Copies share one GPU solver (the
 * reference copies its whole domain), which is what default_driver needs: it keeps and steps its own
 * copy of the Integrator.
 */
#pragma once

#include "../dacti_gpu.h"

#include "integrator/domain.hpp"
#include "integrator/error_estimators.hpp"
#include "integrator/slope_limiters.hpp"
#include "scene/scene.hpp"

#include <array>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace dacti::gpu {

	namespace detail {
		inline void check(int rc, dg_solver *s, const char *what) {
			if (rc != DG_OK) {
				const char *msg = dg_last_error(s);
				throw std::runtime_error(std::string(what) + ": " + (msg ? msg : "error ") + " (status " +
				                         std::to_string(rc) + ")");
			}
		}

		template<typename L>
		constexpr int limiter_id() {
			namespace sl = dacti::integrator::slope;
			if constexpr (std::is_same_v<L, sl::minmod>) return DG_MINMOD;
			else if constexpr (std::is_same_v<L, sl::unlimited>) return DG_UNLIMITED;
			else if constexpr (std::is_same_v<L, sl::van_leer>) return DG_VAN_LEER;
			else if constexpr (std::is_same_v<L, sl::superbee>) return DG_SUPERBEE;
			else if constexpr (std::is_same_v<L, sl::von_alba_2>) return DG_VON_ALBA_2;
			else if constexpr (std::is_same_v<L, sl::koren>) return DG_KOREN;
			else if constexpr (std::is_same_v<L, sl::first_order>) return DG_FIRST_ORDER;
			else static_assert(sizeof(L) == 0, "slope limiter without a GPU counterpart");
		}

		template<typename M>
		constexpr int model_id() {
			if constexpr (M::Multiphase) return DG_MULTI;
			else if constexpr (M::Viscosity) return DG_NAVIER_STOKES;
			else return DG_EULER;
		}

		// model constants as the reference's models hold them (model/euler.hpp:34,
		// model/navier_stokes.hpp:27-31, model/multi.hpp:50-62)
		template<typename M>
		void model_params(double *prm) {
			if constexpr (M::Multiphase) {
				prm[DG_P_GAMMA1] = M::gamma1, prm[DG_P_GAMMA2] = M::gamma2;
				prm[DG_P_P1] = M::P1, prm[DG_P_P2] = M::P2;
				prm[DG_P_CP1] = M::cp1, prm[DG_P_CP2] = M::cp2, prm[DG_P_CV1] = M::cv1, prm[DG_P_CV2] = M::cv2;
				prm[DG_P_MU1] = M::mu1, prm[DG_P_MU2] = M::mu2;
				prm[DG_P_LAMBDA1] = M::lambda1, prm[DG_P_LAMBDA2] = M::lambda2;
				prm[DG_P_SIGMA] = M::sigma;
			} else {
				prm[DG_P_GAMMA] = M::gamma;
				if constexpr (M::Viscosity) prm[DG_P_NS_MU] = M::mu_, prm[DG_P_NS_LAMBDA] = M::lambda_;
			}
		}

		// refinement box in world coordinates; zones of the reference carry a Transform
		// (config/config.hpp:77-86), of which translation and positive scaling map back exactly only
		// when they are the identity
		template<typename Z>
		void zone_box(const Z &z, double *out) {
			double t[3] = {0, 0, 0}, s[3] = {1, 1, 1};
			if constexpr (requires { z.t.rotation; }) {
				for (int d = 0; d < 3; ++d) {
					if (z.t.rotation[d] != 0.0) throw std::runtime_error("rotated refinement zones are not supported");
					t[d] = z.t.translation[d], s[d] = z.t.scaling[d];
					if (s[d] <= 0.0) throw std::runtime_error("refinement zones need positive scaling");
				}
			}
			for (int d = 0; d < 3; ++d) out[d] = t[d] + s[d] * z.x0[d], out[3 + d] = t[d] + s[d] * z.x1[d];
			out[6] = (double) z.refinement_level;
		}
	}    // namespace detail

	template<typename Model, typename Limiter, typename ErrorEstimator>
	class Integrator {
	public:
		using node_t = dacti::integrator::_internal::Node<Model>;
		using vecn_t = linalg::vec<scalar_t, Model::NumDims>;

		static constexpr size_t NumDims = Model::NumDims;
		static constexpr size_t NumMeta = 4;
		static constexpr int MAX_LEVEL  = 16;
		static constexpr std::array<const char *, NumMeta> METADATA_NAMES = {"acti_level", "error", "max_dt", "cfl"};

		// size() of an ACTI cluster or buffer (integrator/integrator.hpp:46-47)
		struct level_list {
			size_t n = 0;
			size_t size() const { return n; }
			bool empty() const { return n == 0; }
		};

		scene::Scene<Model> &scene;
		std::shared_ptr<config::Config<Model>> config;
		Limiter limiter;
		ErrorEstimator error_estimator;

		// Domain::root_index (integrator/domain.hpp:23), read by htg_writer; get_nodes() puts the root there
		struct domain_index {
			size_t root_index = 1;
		} domain;

		std::array<level_list, MAX_LEVEL> acti_clusters;
		std::array<level_list, MAX_LEVEL> acti_buffers;
		std::array<int, MAX_LEVEL> acti_counter{};
		std::array<scalar_t, MAX_LEVEL> acti_time{};

		int n_substeps     = 0;
		int n_global_steps = 0;
		int max_acti_level = 0;
		unsigned long long total_cell_updates = 0;
		scalar_t global_dt = -INFINITY;

		Integrator(Limiter limiter, ErrorEstimator error_estimator, scene::Scene<Model> &scene,
		           std::shared_ptr<config::Config<Model>> config) :
		    scene(scene), config(config), limiter(limiter), error_estimator(error_estimator) {
			constexpr int D = Model::NumDims, E = Model::NumEqns, C = 1 << D, NF = 2 * D;
			static_assert(D == 2 || D == 3);
			using bnd_t = dacti::integrator::Boundary<Model>;

			// Scene::init_domain builds the initial tree as in the reference constructor
			// (integrator/integrator.hpp:77,95)
			dacti::integrator::_internal::Domain<Model> domain(MAX_LEVEL, config->side_length, config->active_size,
			                                                    config->IsPeriodic);
			scene.init_domain(domain);
			const size_t n = domain.tree.size();

			std::vector<int> parent(n, 0), children(n * C, 0), level(n, 0), bc(n * NF, -1);
			std::vector<unsigned> flags(n, 0);
			std::vector<double> center(n * D, 0.0), p(n * E, 0.0);
			std::vector<int> bc_type;
			std::vector<double> bc_p, bc_n, bc_f;
			auto bc_index = [&](const bnd_t &b) {
				for (size_t k = 0; k < bc_type.size(); ++k) {
					bool same = bc_type[k] == (int) b.type && bc_f[k] == b.fade_in;
					for (int q = 0; same && q < E; ++q) same = bc_p[k * E + q] == b.p_in[q];
					for (int d = 0; same && d < D; ++d) same = bc_n[k * D + d] == b.normal[d];
					if (same) return (int) k;
				}
				bc_type.push_back((int) b.type), bc_f.push_back(b.fade_in);
				for (int q = 0; q < E; ++q) bc_p.push_back(b.p_in[q]);
				for (int d = 0; d < D; ++d) bc_n.push_back(b.normal[d]);
				return (int) bc_type.size() - 1;
			};
			for (size_t i = 1; i < n; ++i) {
				const node_t &nd = domain.tree[i];
				parent[i] = (int) nd.parent_index;
				level[i]  = nd.tree_level;
				for (int k = 0; k < C; ++k) children[i * C + k] = (int) nd.child_indices[k];
				flags[i] = (nd.is_leaf ? DG_F_LEAF : 0) | (nd.is_active ? DG_F_ACTIVE : 0) |
				           (nd.is_garbage ? DG_F_GARBAGE : 0) | (nd.can_split ? DG_F_CAN_SPLIT : 0) |
				           (nd.can_unsplit ? DG_F_CAN_UNSPLIT : 0) | (nd.should_split ? DG_F_SHOULD_SPLIT : 0) |
				           (nd.is_boundary ? DG_F_IS_BOUNDARY : 0);
				for (int f = 0; f < NF; ++f)
					if (nd.boundaries.array[f].has_value()) bc[i * NF + f] = bc_index(*nd.boundaries.array[f]);
				for (int d = 0; d < D; ++d) center[i * D + d] = nd.cell.center[d];
				for (int q = 0; q < E; ++q) p[i * E + q] = nd.cell.p[q];
			}

			double prm[DG_N_PARAMS] = {};
			prm[DG_P_SIDE] = config->side_length;
			for (int d = 0; d < D; ++d) {
				prm[DG_P_ACTIVE0 + d]   = config->active_size[d];
				prm[DG_P_PERIODIC0 + d] = config->IsPeriodic[d] ? 1.0 : 0.0;
			}
			prm[DG_P_MAX_CFL]   = config->max_cfl;
			prm[DG_P_MAX_DT]    = config->max_dt;
			prm[DG_P_MIN_ERR]   = config->error_threshold[0];
			prm[DG_P_MAX_ERR]   = config->error_threshold[1];
			prm[DG_P_MAX_LEVEL] = (double) config->max_refinement_level;
			prm[DG_P_MIN_LEVEL] = (double) config->min_refinement_level;
			detail::model_params<Model>(prm);

			static_assert(requires { error_estimator.weights; }, "error estimator without a GPU counterpart");
			double w[7] = {};
			for (int q = 0; q < E; ++q) w[q] = error_estimator.weights[q];

			std::vector<double> zones;
			for (const auto &z: config->refine_zones) {
				double b[7];
				detail::zone_box(z, b);
				zones.insert(zones.end(), b, b + 7);
			}

			dg_case c{};
			c.model = detail::model_id<Model>(), c.dims = D;
			c.n_nodes = (int) n, c.n_bc = (int) bc_type.size(), c.n_zones = (int) (zones.size() / 7);
			c.limiter = detail::limiter_id<Limiter>();
			c.params = prm, c.weights = w, c.zones = zones.data();
			c.bc_type = bc_type.data(), c.bc_p_in = bc_p.data(), c.bc_normal = bc_n.data(), c.bc_fade_in = bc_f.data();
			c.parent = parent.data(), c.children = children.data(), c.level = level.data(), c.flags = flags.data();
			c.bc = bc.data(), c.center = center.data(), c.p = p.data();
			dg_solver *s = nullptr;
			detail::check(dg_create(&c, &s), nullptr, "dg_create");
			solver_.reset(s, deleter{});
			refresh_counters();
		}


		/* Integrator::integrate (impl/integrate.hpp:12-87) */
		scalar_t integrate(auto substep_hook, bool signal, bool &force_break) {
			struct ctx_t {
				Integrator *self;
				decltype(substep_hook) *hook;
			} ctx{this, &substep_hook};
			auto tramp = [](void *user, int level, double acti_time_l, int n_sub, double dt_level, long long size) {
				auto *c                           = static_cast<ctx_t *>(user);
				c->self->acti_clusters[level].n = (size_t) size;
				c->self->n_substeps             = n_sub;
				(*c->hook)(*c->self, level, (scalar_t) acti_time_l, n_sub, (scalar_t) dt_level);
			};
			int fb     = 0;
			double gdt = 0.0;
			detail::check(dg_step(solver_.get(), signal ? 1 : 0, &fb, &gdt, tramp, &ctx), solver_.get(), "dg_step");
			force_break = fb != 0;
			global_dt   = gdt;
			cache_valid_ = false;
			refresh_counters();
			return global_dt;
		}

		size_t n_active_cells() const {
			long long k = 0;
			detail::check(dg_cell_count(solver_.get(), &k), solver_.get(), "dg_cell_count");
			return (size_t) k;
		}

		void for_each_active_cell(auto action) const {
			load_cells();
			for (size_t i = 1; i < cells_.size(); ++i) action((int) (i - 1), cells_[i]);
		}

		/* The whole tree (Integrator::get_nodes, integrator/integrator.hpp:165), what DACTI's htg_writer
		 * walks (driver/io/htg_writer.hpp:112-161): read with dg_read_tree and renumbered breadth first,
		 * slot 0 the null node, slot 1 the root (domain.root_index), parents before children, garbage
		 * slots left out. Each node carries its links, tree level, leaf/active flags, cell.size, cell.p
		 * and get_metadata()'s acti_level, error, max_dt and cfl. The other cell fields are only in the
		 * active-cell list (for_each_active_cell, get_node). */
		std::vector<node_t> get_nodes() const {
			constexpr int E = Model::NumEqns, C = 1 << Model::NumDims;
			long long n = 0;
			detail::check(dg_tree_size(solver_.get(), &n), solver_.get(), "dg_tree_size");
			const size_t nn = (size_t) n;
			std::vector<int> parent(nn), children((size_t) C * nn), level(nn);
			std::vector<unsigned> flags(nn);
			std::vector<double> p((size_t) E * nn), meta(4 * nn);
			long long got = 0;
			detail::check(dg_read_tree(solver_.get(), parent.data(), children.data(), level.data(), flags.data(), p.data(),
			                           meta.data(), n, &got),
			              solver_.get(), "dg_read_tree");
			int root = 0;
			for (size_t i = 1; i < nn && root == 0; ++i)
				if (level[i] == 0 && !(flags[i] & DG_F_GARBAGE)) root = (int) i;
			std::vector<node_t> out(1, node_t{});
			if (root == 0) return out;
			std::vector<int> order(1, root);
			std::vector<size_t> renum(nn, 0);
			renum[root] = 1;
			for (size_t h = 0; h < order.size(); ++h) {
				const int x = order[h];
				if (flags[x] & DG_F_LEAF) continue;
				for (int c = 0; c < C; ++c) {
					const int ch = children[(size_t) c * nn + x];
					if (ch <= 0 || (size_t) ch >= nn || renum[ch] != 0)
						throw std::runtime_error("dg_read_tree: a subdivided node links an invalid child slot");
					renum[ch] = order.size() + 1;
					order.push_back(ch);
				}
			}
			out.resize(order.size() + 1);
			for (size_t k = 0; k < order.size(); ++k) {
				const int x = order[k];
				node_t nd{};
				nd.parent_index = x == root ? 0 : renum[parent[x]];
				nd.tree_level   = level[x];
				nd.is_leaf      = (flags[x] & DG_F_LEAF) != 0;
				nd.is_active    = (flags[x] & DG_F_ACTIVE) != 0;
				nd.is_garbage   = false;
				nd.child_indices.fill(0);
				if (!nd.is_leaf)
					for (int c = 0; c < C; ++c) nd.child_indices[c] = renum[children[(size_t) c * nn + x]];
				scalar_t size = config->side_length;
				for (int l = 0; l < nd.tree_level; ++l) size = 0.5 * size;
				nd.cell.size = size;
				for (int q = 0; q < E; ++q) nd.cell.p[q] = p[(size_t) q * nn + x];
				nd.acti_level = (int) meta[x];
				nd.error      = meta[nn + x];
				nd.max_dt     = meta[2 * nn + x];
				nd.cfl        = meta[3 * nn + x];
				out[k + 1]    = nd;
			}
			return out;
		}

		node_t &get_node(size_t index) const {
			load_cells();
			return cells_.at(index);
		}

		/* index (1-based, 0 if none) of the active cell that contains pos */
		size_t get_cell_index(vecn_t pos) const {
			load_cells();
			for (size_t i = 1; i < cells_.size(); ++i) {
				const auto &c = cells_[i].cell;
				bool in       = true;
				for (size_t d = 0; in && d < NumDims; ++d) in = std::abs(pos[d] - c.center[d]) <= 0.5 * c.size;
				if (in) return i;
			}
			return 0;
		}

		/* the solver handle, for the calls of dacti_gpu.h that have no reference counterpart
		 * (dg_set_form, dg_set_stream, dg_set_profiling, dg_get_stats) */
		dg_solver *handle() const { return solver_.get(); }

	private:
		struct deleter {
			void operator()(dg_solver *s) const { dg_destroy(s); }
		};
		// Copies share the GPU solver: DACTI's default_driver keeps its own copy of the Integrator
		// (driver/default_driver.hpp:20, :34-38) and steps that copy; the tree stays on the device.
		std::shared_ptr<dg_solver> solver_;
		mutable std::vector<node_t> cells_;
		mutable bool cache_valid_ = false;

		void refresh_counters() {
			dg_stats st{};
			detail::check(dg_get_stats(solver_.get(), &st), solver_.get(), "dg_get_stats");
			for (int l = 0; l < MAX_LEVEL; ++l) {
				acti_clusters[l].n = (size_t) st.n_clusters[l];
				acti_buffers[l].n  = (size_t) st.n_buffers[l];
				acti_counter[l]    = st.acti_counter[l];
				acti_time[l]       = st.acti_time[l];
			}
			n_substeps         = (int) st.n_substeps;
			n_global_steps     = (int) st.n_global_steps;
			max_acti_level     = st.max_acti_level;
			total_cell_updates = (unsigned long long) st.cell_updates;
			global_dt          = st.global_dt;
		}

		void load_cells() const {
			if (cache_valid_) return;
			constexpr int D = Model::NumDims, E = Model::NumEqns, P = Model::NumParm;
			constexpr int W = D + 1 + 2 * E + 3 + P;
			const size_t n  = n_active_cells();
			std::vector<int> lv(2 * n);
			std::vector<double> data(W * n);
			long long got = 0;
			detail::check(dg_read_cells(solver_.get(), lv.data(), data.data(), (long long) n, &got), solver_.get(),
			              "dg_read_cells");
			cells_.assign(1, node_t{});
			cells_.reserve(got + 1);
			for (long long i = 0; i < got; ++i) {
				const double *r = &data[i * W];
				node_t nd{};
				nd.tree_level = lv[2 * i], nd.acti_level = lv[2 * i + 1];
				scalar_t size = config->side_length;
				for (int l = 0; l < nd.tree_level; ++l) size = 0.5 * size;
				nd.cell.size = size;
				for (int d = 0; d < D; ++d) nd.cell.center[d] = r[d];
				nd.cell.t = r[D];
				for (int q = 0; q < E; ++q) nd.cell.u[q] = r[D + 1 + q], nd.cell.p[q] = r[D + 1 + E + q];
				nd.error  = r[D + 1 + 2 * E];
				nd.max_dt = r[D + 2 + 2 * E];
				nd.cfl    = r[D + 3 + 2 * E];
				if constexpr (P > 0)
					for (int q = 0; q < P; ++q) nd.cell.k[q] = r[D + 4 + 2 * E + q];
				nd.is_leaf = nd.is_active = true;
				cells_.push_back(nd);
			}
			// slopes for Cell::get_p (vtu_writer), gradients for DropEnergy; a case whose steps keep no
			// gradients leaves them zero
			std::vector<double> sl((size_t) D * E * (got > 0 ? got : 1));
			long long gs = 0;
			detail::check(dg_read_slopes(solver_.get(), sl.data(), got, &gs), solver_.get(), "dg_read_slopes");
			for (long long i = 0; i < gs; ++i)
				for (int d = 0; d < D; ++d)
					for (int q = 0; q < E; ++q) cells_[1 + i].cell.slope[d][q] = sl[(i * D + d) * E + q];
			if constexpr (Model::NumGrad > 0) {
				constexpr int G = Model::NumGrad;
				std::vector<double> gr((size_t) D * G * (got > 0 ? got : 1));
				const int rc = dg_read_gradients(solver_.get(), gr.data(), got, &gs);
				if (rc != DG_ERR_UNSUPPORTED) {
					detail::check(rc, solver_.get(), "dg_read_gradients");
					for (long long i = 0; i < gs; ++i)
						for (int d = 0; d < D; ++d)
							for (int g = 0; g < G; ++g) cells_[1 + i].cell.gradient[d][g] = gr[(i * D + d) * G + g];
				}
			}
			cache_valid_ = true;
		}
	};

}    // namespace dacti::gpu
