// Oracle (test infrastructure, not the product): drives DACTI's own, unmodified
// Integrator<Model, minmod, weighted_laplacian> (src/lib/integrator/integrator.hpp) on a flat case
// file, the way default_driver::run does (driver/default_driver.hpp:197-213), and writes binary
// snapshots of every active cell at the requested global steps.
//
// Usage: dacti_ref_runner <case.bin> <out_prefix> <n_global_steps> [--check s1,s2,..]
//                         [--t-end T] [--neighbor-audit] [--quiet]
//                         [--sample-substeps S --samples N]   (bounded timing samples)
//                         [--chunk-substeps S]   (one full global step timed in chunks of S substeps)
//                         [--nodes]   (with each snapshot, the whole node table of get_nodes())
// Prints one JSON line with timing (wall time of integrate() calls only), substep and
// leaf-update counts. Leaf cell-updates are counted in the substep hook as the level's cluster
// size, as impl/integrate.hpp:57-64 exposes it.
#include "case_io.hpp"

#include "integrator/error_estimators.hpp"
#include "integrator/integrator.hpp"
#include "integrator/slope_limiters.hpp"
#include "model/euler.hpp"
#include "model/multi.hpp"
#include "model/navier_stokes.hpp"
#include "scene/scene.hpp"
#ifdef DACTI_ADAPTER_CHECK
#include "dacti_gpu/integrator.hpp"
#include "driver/default_driver.hpp"
#include "driver/observer/drop_energy.hpp"
#endif

#include <chrono>
#include <iomanip>
#include <cstdio>
#include <set>
#include <sstream>

using namespace dacti;

namespace {

	struct Options {
		std::string case_path, out_prefix;
		int n_steps = 1;
		double t_end = -1.0;
		std::set<int> checks;
		bool neighbor_audit = false;
		bool quiet = false;
		int sample_substeps = 0;  // >0: each integrate() call is timed up to this many substeps
		int samples = 0;
		int chunk_substeps = 0;   // >0: one whole integrate() call, timed per chunk of this many substeps
		bool adapter_check = false;  // side-by-side run against the GPU adapter (adapter build only)
		bool driver_check  = false;  // DACTI's default_driver over the reference and over the adapter
		bool nodes         = false;  // also dump Integrator::get_nodes() beside each snapshot
	};

	template<typename Model>
	void set_model_constants(const oracle::CaseData &c) {
		using namespace oracle;
		if constexpr (Model::Multiphase) {
			Model::gamma1  = c.params[P_GAMMA1];
			Model::gamma2  = c.params[P_GAMMA2];
			Model::P1      = c.params[P_P1];
			Model::P2      = c.params[P_P2];
			Model::cp1     = c.params[P_CP1];
			Model::cp2     = c.params[P_CP2];
			Model::cv1     = c.params[P_CV1];
			Model::cv2     = c.params[P_CV2];
			Model::mu1     = c.params[P_MU1];
			Model::mu2     = c.params[P_MU2];
			Model::lambda1 = c.params[P_LAMBDA1];
			Model::lambda2 = c.params[P_LAMBDA2];
			Model::sigma   = c.params[P_SIGMA];
		} else if constexpr (Model::Viscosity) {
			Model::mu_     = c.params[P_NS_MU];
			Model::lambda_ = c.params[P_NS_LAMBDA];
		}
	}

	template<typename Model>
	std::shared_ptr<config::Config<Model>> make_config(const oracle::CaseData &c) {
		using namespace oracle;
		constexpr int D = Model::NumDims;
		constexpr int E = Model::NumEqns;
		auto cfg         = std::make_shared<config::Config<Model>>();
		cfg->case_data   = &c;
		cfg->side_length = c.params[P_SIDE];
		for (int d = 0; d < D; d++) {
			cfg->active_size[d] = c.params[P_ACTIVE0 + d];
			cfg->IsPeriodic[d]  = c.params[P_PERIODIC0 + d] != 0.0;
		}
		cfg->max_cfl              = c.params[P_MAX_CFL];
		cfg->max_dt               = c.params[P_MAX_DT];
		cfg->error_threshold      = vec2_t{c.params[P_MIN_ERR], c.params[P_MAX_ERR]};
		cfg->max_refinement_level = (int) c.params[P_MAX_LEVEL];
		cfg->min_refinement_level = (int) c.params[P_MIN_LEVEL];
		typename Model::prim_t w;
		for (int q = 0; q < E; q++) w[q] = c.weights[q];
		cfg->error_weights = w;
		for (auto &z: c.zones) {
			typename config::Config<Model>::RefineZone rz;
			rz.x0               = vec3_t{z.x0[0], z.x0[1], z.x0[2]};
			rz.x1               = vec3_t{z.x1[0], z.x1[1], z.x1[2]};
			rz.refinement_level = (size_t) z.level;
			cfg->refine_zones.push_back(rz);
		}
		return cfg;
	}

	// Counts active leaves whose stored neighbour index differs from a fresh Domain::find, i.e.
	// pointers that update_neighbors (integrator/domain.hpp:249-293) would change if called now.
	template<typename Integ>
	long audit_neighbors(Integ &in) {
		using vecn_t = typename Integ::vecn_t_pub;
		long bad     = 0;
		auto &dom    = in.domain;
		for (size_t i = 1; i < dom.tree.size(); ++i) {
			auto &node = dom.tree[i];
			if (!node.is_leaf || !node.is_active || node.is_garbage) continue;
			for (int dim = 0; dim < (int) Integ::NumDims; dim++) {
				for (int dir = 0; dir < 2; dir++) {
					if (node.boundaries.get(dim, dir).has_value()) continue;
					vecn_t loc = node.cell.center + vecn_t::unit(dim) * node.cell.size * (2 * dir - 1.0);
					size_t nb  = dom.find(loc, node.tree_level);
					if (!nb || !dom.tree[nb].is_active) continue;
					if (nb != node.neighbors.get(dim, dir)) bad++;
				}
			}
		}
		return bad;
	}

	template<typename Model, typename Limiter = integrator::slope::minmod>
	struct Runner : public integrator::Integrator<Model, Limiter, integrator::error::weighted_laplacian<Model::NumEqns>> {
		using Base       = integrator::Integrator<Model, Limiter, integrator::error::weighted_laplacian<Model::NumEqns>>;
		using vecn_t_pub = linalg::vec<scalar_t, Model::NumDims>;
		using Base::Base;
	};

	template<typename Model, typename R>
	void write_snapshot(R &in, const std::string &path, int step, double time, double updates) {
		constexpr int D = Model::NumDims;
		constexpr int E = Model::NumEqns;
		oracle::SnapWriter w(path);
		size_t n_clusters = 0;
		for (int l = 0; l < R::MAX_LEVEL; l++) n_clusters += in.acti_clusters[l].size();
		int32_t hdr[8] = {D, E, (int32_t) in.n_active_cells(), (int32_t) n_clusters, step, in.n_substeps, (int32_t) in.domain.tree.size(), 0};
		w.put("DGSNAP01", 8);
		w.put(hdr, 8);
		double hd[3] = {time, in.global_dt, updates};
		w.put(hd, 3);
		in.for_each_active_cell([&](int, auto &node) {
			int32_t lv[2] = {node.tree_level, node.acti_level};
			w.put(lv, 2);
			constexpr int NP = Model::NumParm;
			double buf[D + 1 + 2 * E + 3 + NP];
			int k = 0;
			for (int d = 0; d < D; d++) buf[k++] = node.cell.center[d];
			buf[k++] = node.cell.t;
			for (int q = 0; q < E; q++) buf[k++] = node.cell.u[q];
			for (int q = 0; q < E; q++) buf[k++] = node.cell.p[q];
			buf[k++] = node.error;
			buf[k++] = node.max_dt;
			buf[k++] = node.cfl;
			for (int q = 0; q < NP; q++) buf[k++] = node.cell.k[q];
			w.put(buf, k);
		});
	}

	// Every node of Integrator::get_nodes() (integrator/integrator.hpp:165), in tree order: the input
	// of DACTI's HTG writer (driver/io/htg_writer.hpp:112-161). "DGNODE01", int32 {D, E, n, root},
	// then per node: int32 parent, children[2^D], tree level, flags (1 leaf, 2 active, 4 garbage),
	// double p[E], get_metadata()[4].
	template<typename Model, typename R>
	void write_nodes(R &in, const std::string &path) {
		constexpr int D = Model::NumDims;
		constexpr int E = Model::NumEqns;
		const auto tree = in.get_nodes();
		oracle::SnapWriter w(path);
		int32_t hdr[4] = {D, E, (int32_t) tree.size(), (int32_t) in.domain.root_index};
		w.put("DGNODE01", 8);
		w.put(hdr, 4);
		for (const auto &node: tree) {
			int32_t iv[3 + (1 << D)];
			int k   = 0;
			iv[k++] = (int32_t) node.parent_index;
			for (int c = 0; c < (1 << D); ++c) iv[k++] = (int32_t) node.child_indices[c];
			iv[k++] = node.tree_level;
			iv[k++] = (node.is_leaf ? 1 : 0) | (node.is_active ? 2 : 0) | (node.is_garbage ? 4 : 0);
			w.put(iv, k);
			double dv[E + 4];
			for (int q = 0; q < E; ++q) dv[q] = node.cell.get_p()[q];
			const auto m = node.get_metadata();
			for (int q = 0; q < 4; ++q) dv[E + q] = m[q];
			w.put(dv, E + 4);
		}
	}

#ifdef DACTI_ADAPTER_CHECK
	// Integer cell coordinates at the cell's own level: the key under which both sides' cells are
	// matched (centres are (i + 1/2) size - side/2 on both sides).
	// Row: level, cell coordinates, ACTI level, u[E], slope[D][E], gradient[D][G].
	template<typename Node>
	std::vector<double> cell_row(const Node &node, double side, int D, int E, int G) {
		std::vector<double> r;
		r.push_back(node.tree_level);
		for (int d = 0; d < D; ++d) r.push_back(std::nearbyint((node.cell.center[d] + 0.5 * side) / node.cell.size - 0.5));
		r.push_back(node.acti_level);
		for (int q = 0; q < E; ++q) r.push_back(node.cell.u[q]);
		for (int d = 0; d < D; ++d)
			for (int q = 0; q < E; ++q) r.push_back(node.cell.slope[d][q]);
		if constexpr (requires { node.cell.gradient[0][0]; })
			for (int d = 0; d < D; ++d)
				for (int g = 0; g < G; ++g) r.push_back(node.cell.gradient[d][g]);
		return r;
	}

	// Runs the reference Integrator and dacti::gpu::Integrator (the C++ adapter over the GPU library)
	// side by side from the same Scene and Config and compares, after construction and after every
	// global step: the substep hook sequence (level, level time, substep count, cluster size), the
	// force_break flag, global_dt, the active cell set with its ACTI levels, and the conserved state.
	template<typename Model, typename Limiter>
	int adapter_check(const oracle::CaseData &c, const Options &o, std::shared_ptr<config::Config<Model>> cfg) {
		constexpr int D = Model::NumDims;
		constexpr int E = Model::NumEqns;
		using Est       = integrator::error::weighted_laplacian<E>;
		scene::Scene<Model> scene_ref(cfg), scene_gpu(cfg);
		Runner<Model, Limiter> ref{Limiter{}, Est{cfg->error_weights}, scene_ref, cfg};
		dacti::gpu::Integrator<Model, Limiter, Est> gpu{Limiter{}, Est{cfg->error_weights}, scene_gpu, cfg};
		const double side = cfg->side_length;
		int failures      = 0;
		constexpr int G   = Model::NumGrad;
		// the GPU keeps gradients only where a viscous or conduction term reads them
		bool grad_kept = G > 0;
		if constexpr (Model::Multiphase)
			grad_kept = Model::mu1 != 0.0 || Model::mu2 != 0.0 || Model::lambda1 != 0.0 || Model::lambda2 != 0.0;
		auto rows         = [&](auto &itg) {
            std::vector<std::vector<double>> v;
            itg.for_each_active_cell([&](int, auto &node) { v.push_back(cell_row(node, side, D, E, G)); });
            std::sort(v.begin(), v.end(), [&](const auto &a, const auto &b) {
                return std::lexicographical_compare(a.begin(), a.begin() + D + 1, b.begin(), b.begin() + D + 1);
            });
            return v;
		};
		auto compare = [&](int step, bool hooks_equal, bool fb_equal) {
			auto a = rows(ref), b = rows(gpu);
			bool cells_equal = a.size() == b.size();
			// relative L1 difference over columns [k0, k0 + n) of every row
			auto rel_l1 = [&](int k0, int n) {
				double num = 0.0, den = 0.0;
				for (size_t i = 0; cells_equal && i < a.size(); ++i)
					for (int k = k0; k < k0 + n; ++k) num += std::abs(a[i][k] - b[i][k]), den += std::abs(a[i][k]);
				return den > 0 ? num / den : num;
			};
			for (size_t i = 0; cells_equal && i < a.size(); ++i)
				for (int k = 0; k < D + 2; ++k) cells_equal = cells_equal && a[i][k] == b[i][k];
			const double rel   = rel_l1(D + 2, E);
			const double rel_s = rel_l1(D + 2 + E, D * E);
			// multi::get_grad_input leaves its last slot (dbeta) unset (model/multi.hpp:148-156), so the
			// reference's value there is indeterminate: compare velocity, temperature and alpha only
			const int g_cmp = Model::Multiphase ? D + 2 : G;
			double rel_g    = 0.0;
			for (int d = 0; grad_kept && d < D; ++d) rel_g += rel_l1(D + 2 + E + D * E + d * G, g_cmp);
			bool ok            = hooks_equal && fb_equal && cells_equal && ref.global_dt == gpu.global_dt &&
			          ref.n_active_cells() == gpu.n_active_cells() && rel <= 1e-10;
			if (!ok) failures++;
			std::printf("{\"step\": %d, \"hooks_equal\": %s, \"force_break_equal\": %s, \"cells_equal\": %s, "
			            "\"n_ref\": %zu, \"n_gpu\": %zu, \"global_dt_equal\": %s, \"rel_l1_u\": %.3e, "
			            "\"rel_l1_slope\": %.3e, \"rel_l1_grad\": %.3e, \"grad_compared\": %s}\n",
			            step, hooks_equal ? "true" : "false", fb_equal ? "true" : "false", cells_equal ? "true" : "false",
			            ref.n_active_cells(), gpu.n_active_cells(), ref.global_dt == gpu.global_dt ? "true" : "false", rel,
			            rel_s, rel_g, grad_kept ? "true" : "false");
		};
		compare(0, true, true);
		for (int step = 1; step <= o.n_steps; ++step) {
			std::vector<std::array<double, 4>> hr, hg;
			auto rec = [](auto &out) {
				return [&out](auto &itg, int level, scalar_t at, int ns, scalar_t) {
					out.push_back({(double) level, at, (double) ns, (double) itg.acti_clusters[level].size()});
				};
			};
			bool fr = false, fg = false;
			ref.integrate(rec(hr), true, fr);
			gpu.integrate(rec(hg), true, fg);
			compare(step, hr == hg, fr == fg);
			if (fr || fg) break;
		}
		// the whole tree as DACTI's htg_writer reads it, from both integrators after the last step
		if (o.nodes) {
			write_nodes<Model>(ref, o.out_prefix + "_ref.nodes");
			write_nodes<Model>(gpu, o.out_prefix + "_adapter.nodes");
		}
		// DACTI's own DropEnergy observer (driver/observer/drop_energy.hpp), compiled unchanged, on both
		// integrators after the last step
		if constexpr (Model::Multiphase) {
			observer::DropEnergy on_ref, on_gpu;
			on_ref.observe(ref, cfg);
			on_gpu.observe(gpu, cfg);
			const auto a = on_ref.IntegVars(), b = on_gpu.IntegVars();
			std::printf("DROP_ENERGY {\"ref\": [%.17g, %.17g], \"gpu\": [%.17g, %.17g]}\n", a[0], a[1], b[0], b[1]);
		}
		return failures ? 1 : 0;
	}
#endif

#ifdef DACTI_ADAPTER_CHECK
	// A writer for default_driver that records what it is handed: frame times and cell counts.
	struct RecordingWriter {
		std::vector<std::array<double, 3>> *frames;
		template<typename I>
		void write_data(const I &integrator, scalar_t t, int frame, std::vector<std::vector<scalar_t>> fields,
		                std::vector<std::string> names) {
			frames->push_back({t, (double) frame, (double) integrator.n_active_cells()});
		}
	};

	// DACTI's default_driver (driver/default_driver.hpp:17-217), compiled unchanged, runs the case for
	// o.n_steps global steps once over the reference Integrator and once over the GPU adapter, with a
	// frame after every step and (multiphase) the DropEnergy observer. Prints both observables files
	// and the writers' records as one line: DRIVER {...}.
	template<typename Model, typename Limiter>
	int driver_check(const oracle::CaseData &c, const Options &o, std::shared_ptr<config::Config<Model>> cfg) {
		constexpr int E = Model::NumEqns;
		using Est       = integrator::error::weighted_laplacian<E>;
		scene::Scene<Model> scene_ref(cfg), scene_gpu(cfg);
		Runner<Model, Limiter> ref{Limiter{}, Est{cfg->error_weights}, scene_ref, cfg};
		dacti::gpu::Integrator<Model, Limiter, Est> gpu{Limiter{}, Est{cfg->error_weights}, scene_gpu, cfg};
		cfg->io_interval    = 0.0;
		cfg->end_time       = (o.n_steps - 0.5) * ref.global_dt;
		cfg->result_out_dir = o.out_prefix;
		auto observers = [] {
			if constexpr (Model::Multiphase) return std::tuple{observer::DropEnergy()};
			else return std::tuple<>{};
		};
		std::vector<std::array<double, 3>> fr_ref, fr_gpu;
		cfg->case_name = "driver_ref";
		driver::default_driver d_ref{ref, RecordingWriter{&fr_ref}, cfg, observers()};
		d_ref.run();
		cfg->case_name = "driver_gpu";
		driver::default_driver d_gpu{gpu, RecordingWriter{&fr_gpu}, cfg, observers()};
		d_gpu.run();
		auto dump = [](const std::vector<std::array<double, 3>> &v) {
			std::ostringstream s;
			s << "[";
			for (size_t k = 0; k < v.size(); ++k)
				s << (k ? ", " : "") << "[" << std::setprecision(17) << v[k][0] << ", " << v[k][1] << ", " << v[k][2] << "]";
			s << "]";
			return s.str();
		};
		std::printf("DRIVER {\"frames_ref\": %s, \"frames_gpu\": %s, \"csv_ref\": \"%s/driver_ref_observables.csv\", "
		            "\"csv_gpu\": \"%s/driver_gpu_observables.csv\"}\n",
		            dump(fr_ref).c_str(), dump(fr_gpu).c_str(), o.out_prefix.c_str(), o.out_prefix.c_str());
		return 0;
	}
#endif

	template<typename Model, typename Limiter = integrator::slope::minmod>
	int run(const oracle::CaseData &c, const Options &o) {
		using R = Runner<Model, Limiter>;
		using namespace oracle;
		constexpr int D = Model::NumDims;
		constexpr int E = Model::NumEqns;
		set_model_constants<Model>(c);

		auto cfg = make_config<Model>(c);
#ifdef DACTI_ADAPTER_CHECK
		if (o.adapter_check) return adapter_check<Model, Limiter>(c, o, cfg);
		if (o.driver_check) return driver_check<Model, Limiter>(c, o, cfg);
#endif

		scene::Scene<Model> scene(cfg);
		using clk = std::chrono::steady_clock;
		auto t0   = clk::now();
		R in{Limiter{}, integrator::error::weighted_laplacian<E>{cfg->error_weights}, scene, cfg};
		double init_s = std::chrono::duration<double>(clk::now() - t0).count();

		double time = 0.0, updates = 0.0, integ_s = 0.0;
		long substeps = 0, gc_events = 0, audit_bad = 0;
		int steps_done   = 0;
		bool force_break = false;
		if (o.checks.count(0)) write_snapshot<Model>(in, o.out_prefix + "_0.snap", 0, time, updates);
		if (o.checks.count(0) && o.nodes) write_nodes<Model>(in, o.out_prefix + "_0.nodes");

		if (o.chunk_substeps > 0) {
			// One complete global step; the hook closes a chunk after every chunk_substeps substeps (and
			// after the last one), so the chunks partition the step's substeps in execution order.
			std::printf("{\"init_s\": %.6f, \"threads\": %d, \"chunks\": [", init_s, omp_get_max_threads());
			int seen = 0, in_chunk = 0, n_chunks = 0;
			double upd = 0.0;
			auto a     = clk::now();
			auto hook  = [&](auto &itg, int level, scalar_t, int, scalar_t) {
                upd += (double) itg.acti_clusters[level].size();
                ++seen;
                if (++in_chunk == o.chunk_substeps) {
                    auto b = clk::now();
                    std::printf("%s{\"substeps\": %d, \"updates\": %.0f, \"seconds\": %.6f}", n_chunks++ ? ", " : "",
                                in_chunk, upd, std::chrono::duration<double>(b - a).count());
                    std::fflush(stdout);
                    in_chunk = 0;
                    upd      = 0.0;
                    a        = clk::now();
                }
			};
			in.integrate(hook, true, force_break);
			if (in_chunk > 0)
				std::printf("%s{\"substeps\": %d, \"updates\": %.0f, \"seconds\": %.6f}", n_chunks++ ? ", " : "", in_chunk,
				            upd, std::chrono::duration<double>(clk::now() - a).count());
			std::printf("], \"substeps\": %d, \"force_break\": %d}\n", seen, force_break ? 1 : 0);
			return 0;
		}

		if (o.sample_substeps > 0) {
			// Bounded timing samples: each integrate() call is timed from its start to the hook of its
			// sample_substeps-th substep; the hook then requests the early return the NaN path uses.
			std::printf("{\"init_s\": %.6f, \"threads\": %d, \"samples\": [", init_s, omp_get_max_threads());
			for (int s = 0; s < o.samples; ++s) {
				int seen = 0;
				double upd = 0.0, took = 0.0;
				bool stop = false;
				auto a = clk::now();
				auto hook = [&](auto &itg, int level, scalar_t, int, scalar_t) {
					if (stop) return;
					upd += (double) itg.acti_clusters[level].size();
					if (++seen == o.sample_substeps) {
						took = std::chrono::duration<double>(clk::now() - a).count();
						stop = true;
						force_break = true;
					}
				};
				in.integrate(hook, true, force_break);
				if (!stop) took = std::chrono::duration<double>(clk::now() - a).count();
				force_break = false;
				std::printf("%s{\"substeps\": %d, \"updates\": %.0f, \"seconds\": %.6f}", s ? ", " : "", seen, upd, took);
				std::fflush(stdout);
			}
			std::printf("]}\n");
			return 0;
		}

		for (int step = 1; step <= o.n_steps; ++step) {
			if (o.t_end > 0 && time >= o.t_end) break;
			double step_updates = 0.0;
			bool will_gc        = false;
			auto hook           = [&](auto &itg, int level, scalar_t, int, scalar_t) {
                step_updates += (double) itg.acti_clusters[level].size();
                substeps++;
                if (level == 0) {
                    size_t n = 0;
                    for (int l = 0; l < R::MAX_LEVEL; l++) n += itg.acti_clusters[l].size();
                    will_gc = (double) n / (double) (itg.domain.tree.size() - 1) < 0.2;
                }
			};
			auto a = clk::now();
			in.integrate(hook, true, force_break);
			integ_s += std::chrono::duration<double>(clk::now() - a).count();
			time += in.global_dt;
			updates += step_updates;
			steps_done = step;
			if (will_gc) gc_events++;
			if (o.neighbor_audit) audit_bad += audit_neighbors(in);
			if (o.checks.count(step)) write_snapshot<Model>(in, o.out_prefix + "_" + std::to_string(step) + ".snap", step, time, updates);
			if (o.checks.count(step) && o.nodes) write_nodes<Model>(in, o.out_prefix + "_" + std::to_string(step) + ".nodes");
			if (force_break) break;
		}

		std::printf("{\"steps\": %d, \"time\": %.17g, \"global_dt\": %.17g, \"substeps\": %ld, \"updates\": %.0f, "
		            "\"integrate_s\": %.6f, \"init_s\": %.6f, \"updates_per_s\": %.6g, \"n_active\": %zu, "
		            "\"tree_size\": %zu, \"gc_events\": %ld, \"force_break\": %s, \"neighbor_audit_mismatch\": %ld, "
		            "\"threads\": %d}\n",
		            steps_done, time, in.global_dt, substeps, updates, integ_s, init_s,
		            integ_s > 0 ? updates / integ_s : 0.0, in.n_active_cells(), in.domain.tree.size(), gc_events,
		            force_break ? "true" : "false", audit_bad, omp_get_max_threads());
		return force_break ? 3 : 0;
	}

}    // namespace

int main(int argc, char **argv) {
	if (argc < 4) {
		std::fprintf(stderr, "usage: %s <case.bin> <out_prefix> <n_global_steps> [--check a,b] [--t-end T] [--neighbor-audit]\n", argv[0]);
		return 2;
	}
	Options o;
	o.case_path  = argv[1];
	o.out_prefix = argv[2];
	o.n_steps    = std::atoi(argv[3]);
	for (int i = 4; i < argc; ++i) {
		std::string a = argv[i];
		if (a == "--check" && i + 1 < argc) {
			std::stringstream ss(argv[++i]);
			std::string tok;
			while (std::getline(ss, tok, ',')) o.checks.insert(std::atoi(tok.c_str()));
		} else if (a == "--t-end" && i + 1 < argc) {
			o.t_end = std::atof(argv[++i]);
		} else if (a == "--neighbor-audit") {
			o.neighbor_audit = true;
		} else if (a == "--quiet") {
			o.quiet = true;
		} else if (a == "--sample-substeps" && i + 1 < argc) {
			o.sample_substeps = std::atoi(argv[++i]);
		} else if (a == "--chunk-substeps" && i + 1 < argc) {
			o.chunk_substeps = std::atoi(argv[++i]);
		} else if (a == "--samples" && i + 1 < argc) {
			o.samples = std::atoi(argv[++i]);
		} else if (a == "--adapter-check") {
			o.adapter_check = true;
		} else if (a == "--nodes") {
			o.nodes = true;
		} else if (a == "--driver-check") {
			o.driver_check = true;
		}
	}
	spdlog::set_level(spdlog::level::warn);
	oracle::CaseData c = oracle::read_case(o.case_path);
	if (c.limiter != 0 && !(c.model == 0 && c.dims == 2)) {
		std::fprintf(stderr, "limiters other than minmod are built for euler<2> only\n");
		return 2;
	}
	switch (c.model * 10 + c.dims) {
		case 2:
			switch (c.limiter) {
				case 0: return run<model::euler<2>, integrator::slope::minmod>(c, o);
				case 1: return run<model::euler<2>, integrator::slope::unlimited>(c, o);
				case 2: return run<model::euler<2>, integrator::slope::van_leer>(c, o);
				case 3: return run<model::euler<2>, integrator::slope::superbee>(c, o);
				case 4: return run<model::euler<2>, integrator::slope::von_alba_2>(c, o);
				case 5: return run<model::euler<2>, integrator::slope::koren>(c, o);
				default: return run<model::euler<2>, integrator::slope::first_order>(c, o);
			}
		case 3: return run<model::euler<3>>(c, o);
		case 12: return run<model::navier_stokes<2>>(c, o);
		case 13: return run<model::navier_stokes<3>>(c, o);
		case 22: return run<model::multi<2>>(c, o);
		case 23: return run<model::multi<3>>(c, o);
		default: std::fprintf(stderr, "unsupported model/dims %d/%d\n", c.model, c.dims); return 2;
	}
}
