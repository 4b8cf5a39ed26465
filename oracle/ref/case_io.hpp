// Oracle (test infrastructure, not the product): reader for the flat case files written by
// dacti_b200/casefile.py, and the binary snapshot writer used by the reference runner.
//
// A case file carries one initial tree exactly as DACTI's Scene::init_domain leaves it
// (scene/scene.cpp:369-431): every node slot with parent/children links, tree level, flags,
// per-face boundary ids, cell centre and initial primitive state, plus the solver parameters the
// Integrator constructor reads from Config (integrator/integrator.hpp:80-86).
#pragma once

#include <array>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace oracle {

	enum : uint32_t {
		F_LEAF         = 1u << 0,
		F_ACTIVE       = 1u << 1,
		F_GARBAGE      = 1u << 2,
		F_CAN_SPLIT    = 1u << 3,
		F_CAN_UNSPLIT  = 1u << 4,
		F_SHOULD_SPLIT = 1u << 5,
		F_IS_BOUNDARY  = 1u << 6,
	};

	enum Param : int {
		P_SIDE = 0,
		P_ACTIVE0 = 1,
		P_PERIODIC0 = 4,
		P_MAX_CFL = 7,
		P_MAX_DT = 8,
		P_MIN_ERR = 9,
		P_MAX_ERR = 10,
		P_MAX_LEVEL = 11,
		P_MIN_LEVEL = 12,
		P_GAMMA = 13,
		P_NS_MU = 14,
		P_NS_LAMBDA = 15,
		P_GAMMA1 = 16,
		P_GAMMA2 = 17,
		P_P1 = 18,
		P_P2 = 19,
		P_CP1 = 20,
		P_CP2 = 21,
		P_CV1 = 22,
		P_CV2 = 23,
		P_MU1 = 24,
		P_MU2 = 25,
		P_LAMBDA1 = 26,
		P_LAMBDA2 = 27,
		P_SIGMA = 28,
		N_PARAMS = 32,
	};

	struct BcEntry {
		int32_t type;
		std::vector<double> p_in;    // NumEqns
		std::vector<double> normal;  // NumDims
		double fade_in;
	};

	struct Zone {
		double x0[3], x1[3];
		double level;
	};

	struct CaseData {
		int32_t model = 0, dims = 0, n_nodes = 0, n_bc = 0, n_zones = 0, limiter = 0;
		int E = 0, C = 0, NF = 0;
		double params[N_PARAMS] = {};
		std::vector<double> weights;
		std::vector<Zone> zones;
		std::vector<BcEntry> bcs;
		std::vector<int32_t> parent, children, level, bc;
		std::vector<uint32_t> flags;
		std::vector<double> center, p;
	};

	inline int num_eqns(int model, int dims) { return model == 2 ? dims + 4 : dims + 2; }

	template<typename T>
	inline void rd(FILE *f, T *dst, size_t n) {
		if (n && std::fread(dst, sizeof(T), n, f) != n) throw std::runtime_error("case file truncated");
	}

	inline CaseData read_case(const std::string &path) {
		FILE *f = std::fopen(path.c_str(), "rb");
		if (!f) throw std::runtime_error("cannot open case file " + path);
		CaseData c;
		char magic[8];
		rd(f, magic, 8);
		if (std::memcmp(magic, "DGCASE01", 8) != 0) throw std::runtime_error("bad case magic");
		int32_t hdr[8];
		rd(f, hdr, 8);
		c.model = hdr[0], c.dims = hdr[1], c.n_nodes = hdr[2], c.n_bc = hdr[3], c.n_zones = hdr[4], c.limiter = hdr[5];
		c.E  = num_eqns(c.model, c.dims);
		c.C  = 1 << c.dims;
		c.NF = 2 * c.dims;
		rd(f, c.params, N_PARAMS);
		c.weights.resize(c.E);
		rd(f, c.weights.data(), c.E);
		c.zones.resize(c.n_zones);
		for (auto &z: c.zones) {
			rd(f, z.x0, 3);
			rd(f, z.x1, 3);
			rd(f, &z.level, 1);
		}
		c.bcs.resize(c.n_bc);
		for (auto &b: c.bcs) {
			int32_t tp[2];
			rd(f, tp, 2);
			b.type = tp[0];
			b.p_in.resize(c.E);
			b.normal.resize(c.dims);
			rd(f, b.p_in.data(), c.E);
			rd(f, b.normal.data(), c.dims);
			rd(f, &b.fade_in, 1);
		}
		size_t n = c.n_nodes;
		c.parent.resize(n);
		c.children.resize(n * c.C);
		c.level.resize(n);
		c.flags.resize(n);
		c.bc.resize(n * c.NF);
		c.center.resize(n * c.dims);
		c.p.resize(n * c.E);
		rd(f, c.parent.data(), n);
		rd(f, c.children.data(), n * c.C);
		rd(f, c.level.data(), n);
		rd(f, c.flags.data(), n);
		rd(f, c.bc.data(), n * c.NF);
		rd(f, c.center.data(), n * c.dims);
		rd(f, c.p.data(), n * c.E);
		std::fclose(f);
		return c;
	}

	// Snapshot of every active cell in for_each_active_cell order (integrator/integrator.hpp:172-191).
	// Header: "DGSNAP01", int32 {dims, E, n_cells, n_in_clusters, step, n_substeps, tree_size, pad},
	// double {time, global_dt, updates}. Then per cell int32 {tree_level, acti_level} and doubles
	// {center[D], t, u[E], p[E], error, max_dt, cfl, k[NumParm]}.
	struct SnapWriter {
		FILE *f = nullptr;
		explicit SnapWriter(const std::string &path) {
			f = std::fopen(path.c_str(), "wb");
			if (!f) throw std::runtime_error("cannot write snapshot " + path);
		}
		~SnapWriter() {
			if (f) std::fclose(f);
		}
		template<typename T>
		void put(const T *v, size_t n) { std::fwrite(v, sizeof(T), n, f); }
	};

}    // namespace oracle
