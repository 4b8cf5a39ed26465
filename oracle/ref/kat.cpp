// Oracle (test infrastructure, not the product): known-answer vectors from DACTI's own model,
// boundary, limiter and estimator code (src/lib/model/*.hpp, integrator/boundary.hpp,
// integrator/slope_limiters.hpp, integrator/error_estimators.hpp), for seeded random inputs.
//
// Usage: dacti_ref_kat <out_dir>   -> <out_dir>/kat_<model><dims>.bin for the six model/dims pairs.
// Record layouts are documented in tests/test_restate_kat.py, which reads them.
#include "integrator/boundary.hpp"
#include "integrator/cell.hpp"
#include "integrator/error_estimators.hpp"
#include "integrator/neighbor.hpp"
#include "integrator/slope_limiters.hpp"
#include "model/euler.hpp"
#include "model/multi.hpp"
#include "model/navier_stokes.hpp"

#include <cstdio>
#include <random>
#include <string>
#include <vector>

using namespace dacti;

namespace {

	struct Out {
		std::vector<double> d;
		void put(double x) { d.push_back(x); }
	};

	constexpr int CELL_DOUBLES = 78;

	template<typename Model>
	void put_cell(Out &o, const integrator::_internal::Cell<Model> &c) {
		constexpr int D = Model::NumDims, E = Model::NumEqns;
		std::vector<double> v(CELL_DOUBLES, 0.0);
		v[0] = c.size;
		v[1] = c.t;
		for (int d = 0; d < D; ++d) v[2 + d] = c.center[d];
		for (int q = 0; q < E; ++q) {
			v[5 + q]  = c.u[q];
			v[12 + q] = c.p[q];
			v[19 + q] = c.rhs[q];
		}
		for (int q = 0; q < (int) Model::NumParm; ++q) v[26 + q] = c.k[q];
		for (int q = 0; q < (int) Model::NumGrad; ++q) v[33 + q] = c.t_slope[q];
		for (int d = 0; d < D; ++d)
			for (int q = 0; q < E; ++q) v[39 + 7 * d + q] = c.slope[d][q];
		for (int d = 0; d < D; ++d)
			for (int q = 0; q < (int) Model::NumGrad; ++q) v[60 + 6 * d + q] = c.gradient[d][q];
		for (double x: v) o.put(x);
	}

	template<typename Model>
	typename Model::prim_t random_state(std::mt19937_64 &g) {
		constexpr int D = Model::NumDims;
		std::uniform_real_distribution<double> U(0.0, 1.0);
		typename Model::prim_t p;
		if constexpr (Model::Multiphase) {
			double a;
			double r = U(g);
			if (r < 0.15) a = 0.0;
			else if (r < 0.3) a = 1.0;
			else if (r < 0.4) a = 1e-7;
			else if (r < 0.5) a = 1 - 1e-7;
			else a = U(g);
			p[0] = 1000.0 * a + 1e-3;
			p[1] = (1.2 + U(g)) * (1 - a) + 1e-6;
			for (int i = 0; i < D; ++i) p[Model::iu + i] = -100.0 + 200.0 * U(g);
			p[Model::ip] = 5e4 + 4.5e5 * U(g);
			p[Model::ia] = a;
		} else {
			p[0] = 0.1 + 1.9 * U(g);
			for (int i = 0; i < D; ++i) p[Model::iu + i] = -1.5 + 3.0 * U(g);
			p[Model::ip] = 0.05 + 1.95 * U(g);
		}
		return p;
	}

	template<typename Model>
	integrator::_internal::Cell<Model> random_cell(std::mt19937_64 &g) {
		constexpr int D = Model::NumDims, E = Model::NumEqns;
		std::uniform_real_distribution<double> U(-1.0, 1.0);
		integrator::_internal::Cell<Model> c{};
		int lvl = 3 + (int) (g() % 6);
		c.size  = 1.0;
		for (int l = 0; l < lvl; ++l) c.size = 0.5 * c.size;
		c.t = 0.05 * (1.0 + U(g));
		for (int d = 0; d < D; ++d) c.center[d] = 0.5 * U(g);
		c.p = random_state<Model>(g);
		c.u = Model::conserved_from_primitive(c.p);
		for (int d = 0; d < D; ++d)
			for (int q = 0; q < E; ++q) c.slope[d][q] = 0.1 * std::abs(c.p[q] + 1e-3) * U(g) / c.size;
		for (int q = 0; q < E; ++q) c.rhs[q] = 0.2 * std::abs(c.p[q] + 1e-3) * U(g);
		for (int q = 0; q < (int) Model::NumParm; ++q) c.k[q] = U(g);
		if constexpr (Model::Multiphase) c.k[Model::kappa] = 1000.0 * U(g);
		for (int q = 0; q < (int) Model::NumGrad; ++q) c.t_slope[q] = U(g);
		for (int d = 0; d < D; ++d)
			for (int q = 0; q < (int) Model::NumGrad; ++q) c.gradient[d][q] = 10.0 * U(g);
		return c;
	}

	template<typename Model>
	void set_constants() {
		if constexpr (Model::Multiphase) {
			Model::gamma1  = 4.4;
			Model::gamma2  = 1.4;
			Model::P1      = 6e8;
			Model::P2      = 0.0;
			Model::mu1     = 1e-3;
			Model::mu2     = 1.8e-5;
			Model::lambda1 = 0.6;
			Model::lambda2 = 0.026;
			Model::sigma   = 0.072;
		} else if constexpr (Model::Viscosity) {
			Model::mu_     = 2e-3;
			Model::lambda_ = 2e-3 * 1005.0 / 0.72;
		}
	}

	template<typename Model>
	void put_constants(Out &o) {
		double v[17] = {};
		if constexpr (Model::Multiphase) {
			double w[17] = {0, 0, Model::gamma1, Model::gamma2, Model::P1, Model::P2, Model::cp1, Model::cp2, Model::cv1,
			                Model::cv2, Model::mu1, Model::mu2, Model::lambda1, Model::lambda2, Model::sigma, 0, 0};
			for (int i = 0; i < 17; ++i) v[i] = w[i];
		} else if constexpr (Model::Viscosity) {
			v[0] = Model::mu_;
			v[1] = Model::lambda_;
		}
		for (double x: v) o.put(x);
	}

	template<typename Model>
	void generate(const std::string &path, int model_id, uint64_t seed) {
		constexpr int D = Model::NumDims, E = Model::NumEqns, F = Model::NumFlux;
		using cell_t = integrator::_internal::Cell<Model>;
		using face_t = integrator::_internal::CellFace<D>;
		set_constants<Model>();
		std::mt19937_64 g(seed);
		std::uniform_real_distribution<double> U(-1.0, 1.0);
		const int n_flux = 80, n_bflux = 7 * 10, n_cell = 60, n_lim = 200, n_est = 40;
		Out o;
		put_constants<Model>(o);

		for (int r = 0; r < n_flux; ++r) {
			cell_t cn = random_cell<Model>(g), cp = random_cell<Model>(g);
			int dim   = (int) (g() % D);
			typename Model::vecn_t fc;
			for (int d = 0; d < D; ++d) fc[d] = cn.center[d];
			fc[dim] = cn.center[dim] + 0.5 * cn.size;
			for (int d = 0; d < D; ++d) cp.center[d] = cn.center[d];
			cp.center[dim] = fc[dim] + 0.5 * cp.size;
			double t0 = cn.t, t1 = cn.t + 1e-3 * (1.0 + U(g));
			if constexpr (Model::Multiphase) t1 = cn.t + 1e-7 * (1.0 + U(g));
			face_t face{fc, cn.size, t0, t1, dim, 1};
			auto flux = Model::flux(cn, cp, face);
			put_cell(o, cn);
			put_cell(o, cp);
			for (int d = 0; d < 3; ++d) o.put(d < D ? fc[d] : 0.0);
			o.put(cn.size);
			o.put(t0);
			o.put(t1);
			o.put((double) dim);
			for (int q = 0; q < 11; ++q) o.put(q < F ? flux[q] : 0.0);
		}

		for (int r = 0; r < n_bflux; ++r) {
			cell_t c = random_cell<Model>(g);
			integrator::Boundary<Model> b;
			int types[7] = {0, 1, 2, 3, 4, 5, 6};
			b.type       = static_cast<typename integrator::Boundary<Model>::Type>(types[r % 7]);
			b.p_in       = random_state<Model>(g);
			double nn    = 0.0;
			for (int d = 0; d < D; ++d) {
				b.normal[d] = U(g);
				nn += b.normal[d] * b.normal[d];
			}
			for (int d = 0; d < D; ++d) b.normal[d] /= std::sqrt(nn);
			b.fade_in = (r % 2) ? 0.0 : 0.1;
			int dim   = (int) (g() % D), dir = (int) (g() % 2);
			typename Model::vecn_t fc = c.center;
			double t0 = c.t, t1 = c.t + 1e-3;
			face_t face{fc, c.size, t0, t1, dim, dir};
			auto flux = b.boundary_flux(c, face);
			put_cell(o, c);
			o.put((double) types[r % 7]);
			for (int q = 0; q < 7; ++q) o.put(q < E ? b.p_in[q] : 0.0);
			for (int d = 0; d < 3; ++d) o.put(d < D ? b.normal[d] : 0.0);
			o.put(b.fade_in);
			o.put(c.size);
			o.put(t0);
			o.put(t1);
			o.put((double) dim);
			o.put((double) dir);
			for (int q = 0; q < 11; ++q) o.put(q < F ? flux[q] : 0.0);
		}

		for (int r = 0; r < n_cell; ++r) {
			cell_t c = random_cell<Model>(g);
			typename Model::conv_t u = c.u;
			for (int q = 0; q < E; ++q) u[q] = u[q] * (1.0 + 1e-3 * U(g));
			typename Model::flux_t du;
			for (int q = 0; q < F; ++q) du[q] = 1e-3 * U(g);
			c.u       = u;
			auto prim = Model::primitive_from_conserved(u);
			auto cons = Model::conserved_from_primitive(c.p);
			double md = Model::max_delta_time(c);
			cell_t c2 = c;
			Model::compute_rhs(c2);
			typename Model::conv_t src{};
			if constexpr (Model::HasSource) src = Model::source(c, 1e-7, du);
			typename Model::grad_t gi{};
			if constexpr (Model::NumGrad > 0) gi = Model::get_grad_input(c.p);
			put_cell(o, c);
			for (int q = 0; q < 11; ++q) o.put(q < F ? du[q] : 0.0);
			for (int q = 0; q < 7; ++q) o.put(q < E ? prim[q] : 0.0);
			for (int q = 0; q < 7; ++q) o.put(q < E ? cons[q] : 0.0);
			o.put(md);
			for (int q = 0; q < 7; ++q) o.put(q < E ? c2.rhs[q] : 0.0);
			for (int q = 0; q < 7; ++q) o.put(q < E ? src[q] : 0.0);
			for (int q = 0; q < 6; ++q) o.put(q < (int) Model::NumGrad ? gi[q] : 0.0);
		}

		for (int r = 0; r < n_lim; ++r) {
			double s1 = U(g), s2 = U(g);
			if (r % 10 == 0) s1 = 0.0;
			if (r % 10 == 1) s2 = -s1;
			if (r % 10 == 2) s2 = s1;
			o.put(s1);
			o.put(s2);
			o.put(integrator::slope::minmod{}(s1, s2));
			o.put(integrator::slope::unlimited{}(s1, s2));
			o.put(integrator::slope::van_leer{}(s1, s2));
			o.put(integrator::slope::superbee{}(s1, s2));
			o.put(integrator::slope::von_alba_2{}(s1, s2));
			o.put(integrator::slope::koren{}(s1, s2));
			o.put(integrator::slope::first_order{}(s1, s2));
		}

		for (int r = 0; r < n_est; ++r) {
			cell_t c = random_cell<Model>(g);
			typename Model::prim_t w;
			for (int q = 0; q < E; ++q) w[q] = std::abs(U(g));
			integrator::_internal::Neighbor<std::optional<typename Model::prim_t>, D> nbh;
			double present[6] = {};
			double vals[6][7] = {};
			for (int dim = 0; dim < D; ++dim)
				for (int dir = 0; dir < 2; ++dir) {
					bool here = (g() % 5) != 0;
					present[2 * dim + dir] = here ? 1.0 : 0.0;
					if (here) {
						auto p = random_state<Model>(g);
						nbh.get(dim, dir) = p;
						for (int q = 0; q < E; ++q) vals[2 * dim + dir][q] = p[q];
					} else {
						nbh.get(dim, dir) = std::nullopt;
					}
				}
			integrator::error::weighted_laplacian<E> est{w};
			double e = est.estimate(c, nbh);
			put_cell(o, c);
			for (int q = 0; q < 7; ++q) o.put(q < E ? w[q] : 0.0);
			for (int k = 0; k < 6; ++k)
				for (int q = 0; q < 7; ++q) o.put(vals[k][q]);
			for (int k = 0; k < 6; ++k) o.put(present[k]);
			o.put(e);
		}

		FILE *f = std::fopen(path.c_str(), "wb");
		int32_t hdr[8] = {0x3154414b, model_id, D, n_flux, n_bflux, n_cell, n_lim, n_est};
		std::fwrite(hdr, sizeof(int32_t), 8, f);
		std::fwrite(o.d.data(), sizeof(double), o.d.size(), f);
		std::fclose(f);
	}

}    // namespace

int main(int argc, char **argv) {
	if (argc < 2) {
		std::fprintf(stderr, "usage: %s <out_dir>\n", argv[0]);
		return 2;
	}
	std::string dir = argv[1];
	generate<model::euler<2>>(dir + "/kat_euler2.bin", 0, 11);
	generate<model::euler<3>>(dir + "/kat_euler3.bin", 0, 12);
	generate<model::navier_stokes<2>>(dir + "/kat_ns2.bin", 1, 13);
	generate<model::navier_stokes<3>>(dir + "/kat_ns3.bin", 1, 14);
	generate<model::multi<2>>(dir + "/kat_multi2.bin", 2, 15);
	generate<model::multi<3>>(dir + "/kat_multi3.bin", 2, 16);
	return 0;
}
