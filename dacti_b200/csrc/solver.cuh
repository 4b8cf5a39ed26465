// Host side of the solver: node-pool management, the Integrator constructor sequence and the ACTI
// level scheduler of Integrator::integrate, issuing the stage kernels of stages.cuh.
#pragma once

#include "../../include/dacti_gpu.h"
#include "stages.cuh"

#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace dg {

struct dg_error : std::runtime_error {
	int code;
	dg_error(int c, const std::string &m) :
	    std::runtime_error(m), code(c) {}
};

#define DG_CUDA(x)                                                                                     \
	do {                                                                                               \
		cudaError_t e_ = (x);                                                                          \
		if (e_ != cudaSuccess)                                                                         \
			throw ::dg::dg_error(DG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));         \
	} while (0)

class SolverBase {
public:
	virtual ~SolverBase() = default;
	virtual void step(int signal, int *force_break, double *global_dt, dg_substep_fn fn, void *user) = 0;
	virtual long long cell_count() = 0;
	virtual long long read_cells(int *levels, double *data, long long max_cells) = 0;
	virtual long long read_cells_via(int *levels, double *data, long long max_cells, void *scratch, size_t bytes) = 0;
	virtual long long read_slopes(double *data, long long max_cells) = 0;
	virtual long long read_gradients(double *data, long long max_cells) = 0;
	virtual long long forecast_features(double *data, long long max_cells) = 0;
	virtual long long tree_size() = 0;
	virtual long long read_tree(int32_t *parent, int32_t *child, int32_t *level, uint32_t *flags, double *p, double *meta,
	                            long long max_nodes) = 0;
	virtual int dims() const = 0;
	virtual void set_hold(const uint8_t *hold, long long n) = 0;
	virtual void set_coarsen_interval(int k) = 0;
	virtual void stats(dg_stats *out) = 0;
	virtual void set_stream(cudaStream_t s) = 0;
	virtual void own_stream() = 0;  // give the solver a stream of its own if it runs on the legacy default
	virtual void set_profiling(bool on) = 0;
	virtual void set_form(int form) = 0;
	virtual void set_options(int opts) = 0;
	virtual void prepare_noalloc() = 0;  // loads the read-back gather kernel on the current device
	virtual int model_id() const = 0;
	std::string last_error;
};

inline int grid_for(long long n, int max_blocks = 148 * 16) {
	long long b = (n + BLOCK - 1) / BLOCK;
	if (b < 1) b = 1;
	if (b > max_blocks) b = max_blocks;
	return (int) b;
}
// The same number of threads in blocks of `threads`.
inline int grid_threads(long long n, int threads) { return grid_for(n) * (BLOCK / threads); }

template<class M>
class Batch;

template<class M>
class Solver : public SolverBase {
	static constexpr int D = M::D, E = M::E, NC = 1 << D, NF = 2 * D;
	friend class Batch<M>;

	cudaStream_t st_ = 0;
	Consts C_{};
	BcTable B_{};
	Pool P_{};
	Lists Ls_{};
	Counters *d_cnt_ = nullptr;
	Counters *h_cnt_ = nullptr;  // pinned
	void *pool_mem_  = nullptr;
	void *spare_mem_  = nullptr;  // one field's worth of slots: target of the re-sort and gc permutations
	size_t spare_bytes_ = 0;
	void *sort_mem_  = nullptr;   // keys/values/temp storage of the re-sort
	size_t sort_bytes_ = 0;
	bool resort_     = true;
	void *list_mem_  = nullptr;
	void *bc_mem_    = nullptr;
	double *ff_mem_    = nullptr;  // face fluxes next to receivers (Pool::ff)
	double *du_mem_    = nullptr;  // face-flux sums of the running cluster (Pool::du)
	int32_t *pos_mem_  = nullptr;  // list positions of the running cluster's cells (Pool::pos)
	void *sel_mem_     = nullptr;  // stay marks of the running list and the ordered compaction's temp storage
	size_t sel_tmp_bytes_ = 0;
	int opts_          = DG_OPT_DEFAULT;  // stage implementation choices (DG_OPT_*)
	int32_t *d_leaves_ = nullptr;  // scratch list used at construction
	double *d_read_    = nullptr;
	int32_t *d_readlv_ = nullptr;
	long long read_cap_ = 0;
	int limiter_ = 0;
	int coarsen_every_ = 1;  // global steps between coarsening passes
	bool visc_   = false;  // viscous/heat terms present (multiphase with any non-zero mu or lambda)
	bool mixed_  = false;  // FP32 reconstruction and flux, FP64 update and EOS recovery
	bool sigma_  = false;  // surface tension present

	// scheduler state (integrator/integrator.hpp:46-58)
	int acti_counter_[MAX_ACTI] = {};
	double acti_time_[MAX_ACTI] = {};
	int max_acti_ = 0;
	double global_dt_ = -INFINITY;
	long long n_substeps_ = 0, n_global_ = 0, updates_ = 0, n_gc_ = 0;
	long long n_split_total_ = 0, n_unsplit_total_ = 0;
	int stamp_ = 0;
	int epoch_ = 2;           // kernel epochs of the subtree-mean memo (Pool::mod / Pool::cst)
	int max_tree_level_ = 0;  // deepest tree level any node can reach

	// launch accounting and optional per-kernel event timing
	struct Pending {
		int kind;
		cudaEvent_t a, b;
		long long cells;
	};
	bool prof_ = false;
	std::vector<cudaEvent_t> ev_free_;
	std::vector<Pending> pending_;
	double kms_[DG_NK]          = {};
	long long klaunch_[DG_NK]   = {};
	long long kcells_[DG_NK]    = {};
	long long n_launches_       = 0;

	cudaEvent_t get_event() {
		if (ev_free_.empty()) {
			cudaEvent_t e;
			DG_CUDA(cudaEventCreate(&e));
			return e;
		}
		cudaEvent_t e = ev_free_.back();
		ev_free_.pop_back();
		return e;
	}

	template<class Fn>
	void run_k(int kind, long long cells, Fn &&fn) {
		cudaEvent_t a = nullptr, b = nullptr;
		if (prof_) {
			a = get_event();
			b = get_event();
			DG_CUDA(cudaEventRecord(a, st_));
		}
		fn();
		n_launches_++;
		klaunch_[kind]++;
		kcells_[kind] += cells;
		if (prof_) {
			DG_CUDA(cudaEventRecord(b, st_));
			pending_.push_back({kind, a, b, cells});
		}
	}

	void drain_events() {
		for (auto &p: pending_) {
			float ms = 0.f;
			DG_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
			kms_[p.kind] += ms;
			ev_free_.push_back(p.a);
			ev_free_.push_back(p.b);
		}
		pending_.clear();
	}

public:
	void set_profiling(bool on) override { prof_ = on; }
	void set_options(int opts) override { opts_ = opts; }
	void set_form(int form) override {
		if (form != DG_FORM_FP64 && form != DG_FORM_MIXED) throw dg_error(DG_ERR_ARG, "unknown form");
		mixed_ = form == DG_FORM_MIXED;
	}

	explicit Solver(const dg_case &c) {
		limiter_ = c.limiter;
		setup_consts(c);
		upload_bcs(c);
		long long cap = (long long) c.n_nodes + c.n_nodes / 2 + 1024;
		if (c.params[DG_P_POOL_CAP] > 0) cap = std::max((long long) c.params[DG_P_POOL_CAP], (long long) c.n_nodes + 1024);
		if (cap > 2000000000LL) throw dg_error(DG_ERR_CAPACITY, "node pool capacity above 2e9 slots");
		alloc_pool((int) cap);
		alloc_lists(cap);
		DG_CUDA(cudaMalloc(&d_cnt_, sizeof(Counters)));
		DG_CUDA(cudaMallocHost(&h_cnt_, sizeof(Counters)));
		DG_CUDA(cudaMemset(d_cnt_, 0, sizeof(Counters)));
		upload_tree(c);
		construct();
	}

	~Solver() override {
		cudaStreamSynchronize(st_);
		cudaFree(pool_mem_);
		cudaFree(spare_mem_);
		cudaFree(sort_mem_);
		cudaFree(list_mem_);
		cudaFree(bc_mem_);
		cudaFree(ff_mem_);
		cudaFree(du_mem_);
		cudaFree(sel_mem_);
		cudaFree(pos_mem_);
		cudaFree(d_cnt_);
		cudaFreeHost(h_cnt_);
		cudaFree(d_leaves_);
		cudaFree(d_read_);
		cudaFree(d_readlv_);
		if (owned_stream_) cudaStreamDestroy(owned_stream_);
		for (auto e: ev_free_) cudaEventDestroy(e);
		for (auto &p: pending_) {
			cudaEventDestroy(p.a);
			cudaEventDestroy(p.b);
		}
	}

	void set_stream(cudaStream_t s) override { st_ = s; }

	cudaStream_t owned_stream_ = nullptr;
	void own_stream() override {
		if (st_ != 0) return;
		if (!owned_stream_) DG_CUDA(cudaStreamCreateWithFlags(&owned_stream_, cudaStreamNonBlocking));
		st_ = owned_stream_;
	}

	// ---------------------------------------------------------------------------------------
	void setup_consts(const dg_case &c) {
		const double *pr = c.params;
		C_.side = pr[DG_P_SIDE];
		for (int d = 0; d < 3; ++d) {
			C_.active[d]   = pr[DG_P_ACTIVE0 + d];
			C_.periodic[d] = pr[DG_P_PERIODIC0 + d] != 0.0;
		}
		C_.max_cfl              = pr[DG_P_MAX_CFL];
		C_.min_err              = pr[DG_P_MIN_ERR];
		C_.max_err              = pr[DG_P_MAX_ERR];
		C_.max_refinement_level = (int) pr[DG_P_MAX_LEVEL];
		max_dt_cfg_             = pr[DG_P_MAX_DT];
		pruned_                 = (long long) pr[DG_P_PRUNED];
		for (int q = 0; q < E; ++q) C_.weights[q] = c.weights[q];
		ModelConsts &m = C_.m;
		m.ns_mu = pr[DG_P_NS_MU];
		m.ns_lambda = pr[DG_P_NS_LAMBDA];
		m.gamma1 = pr[DG_P_GAMMA1];
		m.gamma2 = pr[DG_P_GAMMA2];
		m.P1 = pr[DG_P_P1];
		m.P2 = pr[DG_P_P2];
		m.cp1 = pr[DG_P_CP1];
		m.cp2 = pr[DG_P_CP2];
		m.cv1 = pr[DG_P_CV1];
		m.cv2 = pr[DG_P_CV2];
		m.mu1 = pr[DG_P_MU1];
		m.mu2 = pr[DG_P_MU2];
		m.lambda1 = pr[DG_P_LAMBDA1];
		m.lambda2 = pr[DG_P_LAMBDA2];
		m.sigma = pr[DG_P_SIGMA];
		if constexpr (M::MULTI) visc_ = m.mu1 != 0.0 || m.mu2 != 0.0 || m.lambda1 != 0.0 || m.lambda2 != 0.0;
		else visc_ = M::VISC;
		sigma_ = m.sigma != 0.0;
		C_.visc = visc_ ? 1 : 0;
		if (c.n_zones > MAX_ZONES) throw dg_error(DG_ERR_ARG, "too many refinement zones");
		C_.n_zones = c.n_zones;
		C_.coarsen = 1;
		for (int z = 0; z < c.n_zones; ++z) {
			for (int d = 0; d < 3; ++d) {
				C_.zx0[z][d] = c.zones[7 * z + d];
				C_.zx1[z][d] = c.zones[7 * z + 3 + d];
			}
			C_.zlevel[z] = (int) c.zones[7 * z + 6];
		}
		// Per-level size (exact halving from the root, integrator/domain.hpp:207), and volume/area
		// evaluated with the same std::pow calls as Cell::volume / CellFace::area
		// (integrator/cell.hpp:575-577, 622-624).
		double s = C_.side;
		for (int l = 0; l < MAX_TREE; ++l) {
			C_.size[l] = s;
			C_.vol[l]  = std::pow(s, D);
			C_.area[l] = std::pow(s, D - 1);
			for (int d = 0; d < 3; ++d) {
				if (d >= D) {
					C_.a0[l][d] = 0;
					C_.na[l][d] = 1;
					continue;
				}
				// active box [-A/2, A/2] in cells of level l of the root box [-S/2, S/2]
				double cells = C_.active[d] / s;
				double off   = 0.5 * (C_.side - C_.active[d]) / s;
				long long nc = std::llround(cells), oc = std::llround(off);
				C_.na[l][d]  = (int) nc;
				C_.a0[l][d]  = (int) oc;
				if (l >= (int) pr[DG_P_MIN_LEVEL] && (std::fabs(cells - nc) > 1e-9 || std::fabs(off - oc) > 1e-9))
					throw dg_error(DG_ERR_UNSUPPORTED, "active box not aligned with the cell grid at the base level");
			}
			s = 0.5 * s;
		}
	}

	void upload_bcs(const dg_case &c) {
		int n        = c.n_bc > 0 ? c.n_bc : 1;
		size_t bytes = sizeof(int) * n + sizeof(double) * n * (E + D + 1) + 1024;
		DG_CUDA(cudaMalloc(&bc_mem_, bytes));
		char *b   = (char *) bc_mem_;
		int *type = (int *) b;
		b += ((sizeof(int) * n + 255) / 256) * 256;
		double *pin = (double *) b;
		double *nrm = pin + (size_t) n * E;
		double *fad = nrm + (size_t) n * D;
		if (c.n_bc > 0) {
			DG_CUDA(cudaMemcpy(type, c.bc_type, sizeof(int) * c.n_bc, cudaMemcpyHostToDevice));
			DG_CUDA(cudaMemcpy(pin, c.bc_p_in, sizeof(double) * c.n_bc * E, cudaMemcpyHostToDevice));
			DG_CUDA(cudaMemcpy(nrm, c.bc_normal, sizeof(double) * c.n_bc * D, cudaMemcpyHostToDevice));
			DG_CUDA(cudaMemcpy(fad, c.bc_fade_in, sizeof(double) * c.n_bc, cudaMemcpyHostToDevice));
		}
		B_ = BcTable{c.n_bc, type, pin, nrm, fad};
	}

	// ---------------------------------------------------------------------------------------
	// Node pool: every field is an array of `cap` entries per component.
	struct Field {
		void **ptr;
		size_t elem;
		int comps;
	};

	std::vector<Field> fields(Pool &P) {
		return {
		    {(void **) &P.parent, 4, 1}, {(void **) &P.child, 4, NC}, {(void **) &P.level, 1, 1},
		    {(void **) &P.acti, 1, 1}, {(void **) &P.clu, 1, 1}, {(void **) &P.flags, 4, 1},
		    {(void **) &P.coord, 4, D}, {(void **) &P.nbr, 4, NF}, {(void **) &P.bc, 2, NF},
		    {(void **) &P.center, 8, D}, {(void **) &P.t, 8, 1}, {(void **) &P.u, 8, E},
		    {(void **) &P.p, 8, E}, {(void **) &P.rec, 8 * Rec<M>::W, 1}, {(void **) &P.avg, 8 * Avg<M>::W, 1},
		    {(void **) &P.mod, 4, 1}, {(void **) &P.cst, 4, 1}, {(void **) &P.avga, 8, 1}, {(void **) &P.csta, 4, 1},
		    {(void **) &P.k, 8, M::P}, {(void **) &P.tslope, 8, visc_ ? M::G : -1},
		    {(void **) &P.grad, 8, visc_ ? D * M::G : -1},
		    {(void **) &P.flux, 8, M::F}, {(void **) &P.err, 8, 1}, {(void **) &P.maxdt, 8, 1},
		    {(void **) &P.cfl, 8, 1}, {(void **) &P.stamp, 4, 1}, {(void **) &P.fmask, 4, 1}, {(void **) &P.op, 1, 1},
		    {(void **) &P.tmp, 8, 1}, {(void **) &P.tmp2, 8, 1},
		};
	}

	static size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

	// The spare buffer holds the largest field of the pool (the reconstruction records, in practice).
	void ensure_spare() {
		size_t need = 0;
		for (auto &f: fields(P_)) need = std::max(need, field_bytes(f, P_.cap));
		if (spare_mem_ && spare_bytes_ >= need) return;
		cudaFree(spare_mem_);
		spare_mem_ = nullptr;
		DG_CUDA(cudaMalloc(&spare_mem_, need));
		spare_bytes_ = need;
	}

	// Bytes of one field: comps < 0 marks a field this case does not store (no storage, null pointer);
	// a model without components of a field (comps 0) still gets one.
	static size_t field_bytes(const Field &f, int cap) {
		return f.comps < 0 ? 0 : align_up(f.elem * (size_t) cap * (f.comps > 0 ? f.comps : 1));
	}

	void *carve_pool(Pool &P, int cap) {
		P.cap        = cap;
		auto fs      = fields(P);
		size_t total = 0;
		for (auto &f: fs) total += field_bytes(f, cap);
		void *mem = nullptr;
		DG_CUDA(cudaMalloc(&mem, total));
		DG_CUDA(cudaMemsetAsync(mem, 0, total, st_));
		char *b = (char *) mem;
		for (auto &f: fs) {
			*f.ptr = f.comps < 0 ? nullptr : b;
			b += field_bytes(f, cap);
		}
		return mem;
	}

	void alloc_pool(int cap) {
		pool_mem_ = carve_pool(P_, cap);
		alloc_derived(cap);
	}

	// Per-substep scratch. By pool slot: pos (a running-cluster cell's list position). By list position,
	// sized to the largest list a substep has run so far (grown by a quarter when a larger one comes):
	// receiver face fluxes and face-flux sums.
	void alloc_derived(int cap) {
		cudaFree(pos_mem_);
		pos_mem_ = nullptr;
		DG_CUDA(cudaMalloc(&pos_mem_, sizeof(int32_t) * (size_t) cap));
		attach_derived();
	}

	long long scratch_cap_ = 0;
	void ensure_scratch(long long n) {
		if (n <= scratch_cap_) return;
		const long long want = std::max(std::max(n, scratch_cap_ + scratch_cap_ / 4), 1024LL);
		cudaFree(ff_mem_);
		cudaFree(du_mem_);
		cudaFree(sel_mem_);
		ff_mem_      = nullptr;
		du_mem_      = nullptr;
		sel_mem_     = nullptr;
		scratch_cap_ = 0;
		DG_CUDA(cudaMalloc(&ff_mem_, sizeof(double) * M::F * NF * (size_t) want));
		DG_CUDA(cudaMalloc(&du_mem_, sizeof(double) * M::F * (size_t) want));
		// stay marks (one byte per list position, rounded to 256) followed by the temp storage of the
		// order-keeping compaction of `want` items
		sel_tmp_bytes_ = 0;
		DG_CUDA(cub::DeviceSelect::Flagged(nullptr, sel_tmp_bytes_, (const int32_t *) nullptr, (const uint8_t *) nullptr,
		                                   (int32_t *) nullptr, (int *) nullptr, (int) want, st_));
		DG_CUDA(cudaMalloc(&sel_mem_, stay_bytes(want) + sel_tmp_bytes_));
		scratch_cap_ = want;
		attach_derived();
	}

	static size_t stay_bytes(long long want) { return ((size_t) want + 255) / 256 * 256; }
	uint8_t *stay_marks() const { return static_cast<uint8_t *>(sel_mem_); }

	void attach_derived() {
		P_.ff   = ff_mem_;
		P_.du   = du_mem_;
		P_.pos  = pos_mem_;
	}

	// The capacity a pool grows to when `need` slots must fit and `want` would be chosen: `want` when the
	// new pool and lists fit in the free device memory (counting the scratch, spare buffer and sort keys
	// that grow_pool releases first, less 1 GiB), else as many slots as fit, and never fewer than `need`.
	long long growth_target(long long need, long long want) {
		size_t free_b = 0, total_b = 0;
		DG_CUDA(cudaMemGetInfo(&free_b, &total_b));
		const size_t released = sizeof(double) * M::F * (NF + 1) * (size_t) scratch_cap_ + spare_bytes_ + sort_bytes_;
		size_t per_slot = sizeof(int32_t) * (2 * MAX_ACTI + 6);
		for (auto &f: fields(P_))
			if (f.comps >= 0) per_slot += f.elem * (size_t) (f.comps > 0 ? f.comps : 1);
		const long long avail = (long long) (free_b + released) - (1LL << 30);
		const long long fit   = avail > 0 ? avail / (long long) per_slot : 0;
		return std::max(need, std::min(want, fit));
	}

	// Grows the node pool: a new pool of new_cap slots takes every field, then the old one goes. Grows
	// between the indicator and the split of a substep, when the stages that use the list scratch are
	// done, so the scratch, the spare buffer and the re-sort keys are released first (they come back at
	// their next use) and the peak holds the two pools and the lists only.
	void grow_pool(int new_cap) {
		DG_CUDA(cudaStreamSynchronize(st_));
		cudaFree(spare_mem_);
		spare_mem_   = nullptr;
		spare_bytes_ = 0;
		cudaFree(sort_mem_);
		sort_mem_   = nullptr;
		sort_bytes_ = 0;
		cudaFree(ff_mem_);
		cudaFree(du_mem_);
		cudaFree(sel_mem_);
		ff_mem_      = nullptr;
		du_mem_      = nullptr;
		sel_mem_     = nullptr;
		scratch_cap_ = 0;
		attach_derived();
		Pool NP{};
		void *mem = carve_pool(NP, new_cap);
		auto fo = fields(P_), fn = fields(NP);
		for (size_t k = 0; k < fo.size(); ++k) {
			if (fo[k].comps <= 0) continue;
			DG_CUDA(cudaMemcpy2DAsync(*fn[k].ptr, fn[k].elem * (size_t) new_cap, *fo[k].ptr,
			                          fo[k].elem * (size_t) P_.cap, fo[k].elem * (size_t) P_.cap, fo[k].comps,
			                          cudaMemcpyDeviceToDevice, st_));
		}
		DG_CUDA(cudaStreamSynchronize(st_));
		cudaFree(pool_mem_);
		pool_mem_ = mem;
		P_        = NP;
		alloc_derived(new_cap);
		// lists grow with the pool
		Lists old = Ls_;
		void *old_mem = list_mem_;
		int old_cap   = list_cap_;
		alloc_lists(new_cap);
		const size_t bytes = sizeof(int32_t) * old_cap;
		for (int l = 0; l < MAX_ACTI; ++l) {
			DG_CUDA(cudaMemcpyAsync(Ls_.clu[l], old.clu[l], bytes, cudaMemcpyDeviceToDevice, st_));
			DG_CUDA(cudaMemcpyAsync(Ls_.buf[l], old.buf[l], bytes, cudaMemcpyDeviceToDevice, st_));
		}
		// the per-substep lists too: the pool can grow between the indicator and the split
		for (auto pr: {std::make_pair(Ls_.tmp, old.tmp), std::make_pair(Ls_.recv, old.recv),
		               std::make_pair(Ls_.split, old.split), std::make_pair(Ls_.unsplit, old.unsplit),
		               std::make_pair(Ls_.fresh, old.fresh), std::make_pair(Ls_.upd, old.upd)})
			DG_CUDA(cudaMemcpyAsync(pr.first, pr.second, bytes, cudaMemcpyDeviceToDevice, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		cudaFree(old_mem);
	}

	int list_cap_ = 0;
	void alloc_lists(int cap) {
		const int nlists = 2 * MAX_ACTI + 6;
		size_t one       = align_up(sizeof(int32_t) * (size_t) cap);
		DG_CUDA(cudaMalloc(&list_mem_, one * nlists));
		char *b = (char *) list_mem_;
		for (int l = 0; l < MAX_ACTI; ++l) {
			Ls_.clu[l] = (int32_t *) b;
			b += one;
			Ls_.buf[l] = (int32_t *) b;
			b += one;
		}
		Ls_.tmp     = (int32_t *) b;
		b += one;
		Ls_.recv    = (int32_t *) b;
		b += one;
		Ls_.split   = (int32_t *) b;
		b += one;
		Ls_.unsplit = (int32_t *) b;
		b += one;
		Ls_.fresh   = (int32_t *) b;
		b += one;
		Ls_.upd     = (int32_t *) b;
		list_cap_   = cap;
	}

	// ---------------------------------------------------------------------------------------
	template<typename T>
	void upload_soa(T *dst, const T *src_rowmajor, int n, int comps) {
		std::vector<T> tmp((size_t) n * comps);
		for (int i = 0; i < n; ++i)
			for (int c = 0; c < comps; ++c) tmp[(size_t) c * n + i] = src_rowmajor[(size_t) i * comps + c];
		for (int c = 0; c < comps; ++c)
			DG_CUDA(cudaMemcpy(dst + (size_t) c * P_.cap, tmp.data() + (size_t) c * n, sizeof(T) * n, cudaMemcpyHostToDevice));
	}

	std::vector<int32_t> active_leaves_;

	void upload_tree(const dg_case &c) {
		const int n = c.n_nodes;
		DG_CUDA(cudaStreamSynchronize(st_));
		std::vector<int8_t> lv(n), ac(n, -1), cl(n, CLU_NONE);
		std::vector<int32_t> coord((size_t) n * D, 0);
		std::vector<int16_t> bc((size_t) n * NF);
		max_tree_level_ = C_.max_refinement_level;
		for (int z = 0; z < C_.n_zones; ++z) max_tree_level_ = std::max(max_tree_level_, C_.zlevel[z]);
		for (int i = 0; i < n; ++i) {
			lv[i] = (int8_t) c.level[i];
			max_tree_level_ = std::max(max_tree_level_, (int) c.level[i]);
			for (int f = 0; f < NF; ++f) bc[(size_t) i * NF + f] = (int16_t) c.bc[(size_t) i * NF + f];
		}
		// integer coordinates, parents before children
		std::vector<int> order;
		order.reserve(n);
		if (n > 1) order.push_back(1);
		for (size_t h = 0; h < order.size(); ++h) {
			int x = order[h];
			if (c.flags[x] & DG_F_LEAF) continue;
			for (int k = 0; k < NC; ++k) {
				int ch = c.children[(size_t) x * NC + k];
				if (ch <= 0) continue;
				for (int d = 0; d < D; ++d) coord[(size_t) ch * D + d] = 2 * coord[(size_t) x * D + d] + ((k >> d) & 1);
				order.push_back(ch);
			}
		}
		upload_soa(P_.parent, c.parent, n, 1);
		upload_soa(P_.child, c.children, n, NC);
		upload_soa(P_.level, lv.data(), n, 1);
		upload_soa(P_.acti, ac.data(), n, 1);
		upload_soa(P_.clu, cl.data(), n, 1);
		upload_soa(P_.flags, (const uint32_t *) c.flags, n, 1);
		upload_soa(P_.coord, coord.data(), n, D);
		upload_soa(P_.bc, bc.data(), n, NF);
		upload_soa(P_.center, c.center, n, D);
		upload_soa(P_.p, c.p, n, E);
		// Node::error as the scene leaves it: -1 on every split child (integrator/domain.hpp:215), kept by
		// leaves that never get an estimate (inactive ones) and summed by unsplit (domain.hpp:306-309)
		{
			std::vector<double> err((size_t) n, -1.0);
			upload_soa(P_.err, err.data(), n, 1);
		}
		active_leaves_.clear();
		for (int i = 1; i < n; ++i)
			if ((c.flags[i] & DG_F_LEAF) && (c.flags[i] & DG_F_ACTIVE)) active_leaves_.push_back(i);
		h_cnt_->top = n;
		DG_CUDA(cudaMemcpy(&d_cnt_->top, &n, sizeof(int), cudaMemcpyHostToDevice));
	}

	// Integrator constructor body (integrator/integrator.hpp:100-160).
	void construct() {
		const int n = (int) active_leaves_.size();
		DG_CUDA(cudaMalloc(&d_leaves_, sizeof(int32_t) * (n > 0 ? n : 1)));
		DG_CUDA(cudaMemcpy(d_leaves_, active_leaves_.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
		const int g = grid_for(n);
		k_init_cells<M><<<g, BLOCK, 0, st_>>>(P_, C_, d_leaves_, n, d_cnt_);
		k_nbr_init<M><<<g, BLOCK, 0, st_>>>(P_, C_, d_leaves_, n);
		// every memo starts stale: mod = 1 > cst = 0
		k_fill_i32<<<grid_for(P_.cap), BLOCK, 0, st_>>>(P_.mod, 1, P_.cap);
		// neighbour values and slopes of every leaf, in pieces of the scratch's size
		ensure_scratch(std::max(n / 2, 1));
		for (int off = 0; off < n; off += (int) scratch_cap_) launch_slope(d_leaves_ + off, std::min<int>(n - off, (int) scratch_cap_));
		if constexpr (M::MULTI) multiphase_aux(d_leaves_, n, -1, 0);
		DG_CUDA(cudaGetLastError());
		sync_counters();
		global_dt_ = std::fmax(-INFINITY, h_cnt_->dmax);
		global_dt_ = std::min(0.9 * global_dt_, max_dt_cfg());
		k_assign<M><<<g, BLOCK, 0, st_>>>(P_, C_, d_leaves_, n, global_dt_, Ls_, d_cnt_);
		DG_CUDA(cudaGetLastError());
		sync_counters();
		check_status();
		cudaFree(d_leaves_);  // the constructor's list of every leaf is not used again
		d_leaves_ = nullptr;
		max_acti_ = 0;
		for (int l = 0; l < MAX_ACTI; ++l)
			if (h_cnt_->clu[l] > 0) max_acti_ = std::max(max_acti_, l);
	}

	double max_dt_cfg_ = 1.0;
	double max_dt_cfg() const { return max_dt_cfg_; }
	long long pruned_ = 0;  // node slots the host left out of the upload; part of the reference's tree size

	// The garbage-collection trigger of impl/integrate.hpp:78-84: active leaves in clusters below a fifth
	// of tree.size() - 1, the tree size counting the slots left out of the upload.
	bool gc_due() const {
		long long n_in = 0;
		for (int l = 0; l < MAX_ACTI; ++l) n_in += h_cnt_->clu[l];
		return (double) n_in / (double) (h_cnt_->top - 1 + pruned_) < 0.2;
	}

public:
	void set_max_dt(double v) { max_dt_cfg_ = v; }

private:
	// smooth_alpha x3, normal_update, curvature_update, smooth_curvature over one cell list
	// (impl/integrate.hpp:284-289, integrator/integrator.hpp:134-143).
	// Lm: the ACTI level whose cluster `list` is, or -1 when the list holds every leaf (constructor).
	// e_upd: epoch of the substep's cell update (0: no memoised volume-fraction means).
	void multiphase_aux(const int32_t *list, int n, int Lm, int e_upd) {
		if constexpr (M::MULTI) {
			constexpr int G = NF <= 4 ? 4 : 8;
			const int g  = grid_for(n);
			const int gl = grid_for((long long) n * G);
			double *alphas = P_.k + (size_t) M::ALPHAS * P_.cap;
			run_k(DG_K_AUX, n, [&] {
				k_smooth_alpha<M><<<gl, BLOCK, 0, st_>>>(P_, C_, B_, list, n, nullptr, P_.tmp, Lm, ++epoch_, e_upd, d_cnt_);
			});
			run_k(DG_K_AUX, n, [&] {
				k_smooth_alpha<M><<<gl, BLOCK, 0, st_>>>(P_, C_, B_, list, n, P_.tmp, P_.tmp2, Lm, ++epoch_, e_upd, d_cnt_);
			});
			run_k(DG_K_AUX, n, [&] {
				k_smooth_alpha<M><<<gl, BLOCK, 0, st_>>>(P_, C_, B_, list, n, P_.tmp2, alphas, Lm, ++epoch_, e_upd, d_cnt_);
			});
			run_k(DG_K_AUX, n, [&] { k_normal<M><<<gl, BLOCK, 0, st_>>>(P_, C_, B_, list, n, ++epoch_, e_upd, d_cnt_); });
			// The curvature only enters through sigma * kappa (model/multi.hpp:142, 216, 190-193); without
			// surface tension those products are zeros and the curvature stages are skipped.
			if (sigma_) {
				run_k(DG_K_AUX, n, [&] { k_curvature<M><<<g, BLOCK, 0, st_>>>(P_, C_, B_, list, n, d_cnt_); });
				run_k(DG_K_AUX, n, [&] { k_smooth_kappa<M><<<g, BLOCK, 0, st_>>>(P_, C_, B_, list, n, d_cnt_); });
				run_k(DG_K_AUX, n, [&] { k_store_tmp<<<g, BLOCK, 0, st_>>>(P_, list, n, M::KAPPA, P_.tmp); });
				run_k(DG_K_AUX, n, [&] { k_rec_k<M><<<g, BLOCK, 0, st_>>>(P_, list, n); });
			}
		}
	}

	// Face-flux sums of the running cluster into du, receivers of slower clusters into Ls_.recv.
	void launch_face_sum(const int32_t *list, int n, int L, double dtL, int stamp) {
		constexpr int G = NF <= 4 ? 4 : 8, T = FACE_THREADS;
		if (opts_ & DG_OPT_FACE_TILES) {
			constexpr int TC = FaceTile<M>::TC;
			const int gt = (int) std::max<long long>(1, ((long long) n + TC - 1) / TC);
			if (mixed_) {
				if (visc_) k_face_tile<M, true, float><<<gt, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
				else k_face_tile<M, false, float><<<gt, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
			} else {
				if (visc_) k_face_tile<M, true, double><<<gt, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
				else k_face_tile<M, false, double><<<gt, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
			}
			return;
		}
		const int g = grid_threads((long long) n * G, T);
		if (mixed_) {
			if (visc_) k_face_sum<M, true, float><<<g, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
			else k_face_sum<M, false, float><<<g, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
		} else {
			if (visc_) k_face_sum<M, true, double><<<g, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
			else k_face_sum<M, false, double><<<g, T, 0, st_>>>(P_, C_, B_, list, n, L, dtL, stamp, Ls_.recv, d_cnt_);
		}
	}

	// Slopes, Hancock rhs and (viscous) gradients of a cell list.
	void launch_slope(const int32_t *list, int n) {
		constexpr int G = NF <= 4 ? 4 : 8, T = SLOPE_THREADS;
		const int g = grid_threads((long long) n * G, T);
		if (visc_) k_slope<M, true><<<g, T, 0, st_>>>(P_, C_, B_, list, n, limiter_, ++epoch_, d_cnt_);
		else k_slope<M, false><<<g, T, 0, st_>>>(P_, C_, B_, list, n, limiter_, ++epoch_, d_cnt_);
	}

	void sync_counters() {
		DG_CUDA(cudaMemcpyAsync(h_cnt_, d_cnt_, sizeof(Counters), cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		drain_events();
	}

	void check_status() {
		uint32_t s = h_cnt_->status & ~ST_NAN;
		if (s & ST_CAPACITY) throw dg_error(DG_ERR_CAPACITY, "device list or pool capacity exceeded");
		if (s & ST_DEPTH) throw dg_error(DG_ERR_DEPTH, "tree level jump deeper than supported");
		if (s & ST_MISSING_BC) throw dg_error(DG_ERR_MISSING_BC, "face without neighbour or boundary condition");
		if (s & ST_SPLIT_UNSPLIT) throw dg_error(DG_ERR_UNSUPPORTED, "cell both split and coarsened in one substep");
	}

	// One ACTI-level substep: impl/integrate.hpp:277-299 minus the host bookkeeping.
	void substep(int L) {
		const int n      = h_cnt_->clu[L];
		const double dtL = global_dt_ / (double) (1 << L);
		ensure_scratch(n);
		// A split takes 2^D new slots. When the pool cannot take a split of every cluster cell, the
		// split requests are read back after the indicator and the pool grown to fit them.
		const bool tight = (long long) h_cnt_->top + (long long) NC * n + 16 > P_.cap;
		const int stamp_recv = ++stamp_;
		// n_recv .. status
		DG_CUDA(cudaMemsetAsync(&d_cnt_->n_recv, 0, (char *) (&d_cnt_->status + 1) - (char *) &d_cnt_->n_recv, st_));
		const int g        = grid_for(n);
		int32_t *list      = Ls_.clu[L];
		const int counterL = acti_counter_[L];

		constexpr int LPC = NF <= 4 ? 4 : 8;  // receive lanes per cell
		int e_upd = 0;                       // epoch of this substep's cell update
		run_k(DG_K_FLUX, n, [&] { launch_face_sum(list, n, L, dtL, stamp_recv); });
		run_k(DG_K_RECV, 0, [&] {
			if (mixed_) k_flux_receive<M, float><<<grid_for((long long) n * LPC), BLOCK, 0, st_>>>(P_, Ls_.recv, &d_cnt_->n_recv, L, d_cnt_);
			else k_flux_receive<M, double><<<grid_for((long long) n * LPC), BLOCK, 0, st_>>>(P_, Ls_.recv, &d_cnt_->n_recv, L, d_cnt_);
		});
		run_k(DG_K_UPDATE, n, [&] {
			e_upd = ++epoch_;
			if (visc_) k_update<M, true><<<g, BLOCK, 0, st_>>>(P_, C_, list, n, dtL, e_upd, d_cnt_);
			else k_update<M, false><<<g, BLOCK, 0, st_>>>(P_, C_, list, n, dtL, e_upd, d_cnt_);
		});
		run_k(DG_K_SLOPE, n, [&] { launch_slope(list, n); });
		if constexpr (M::MULTI) multiphase_aux(list, n, L, e_upd);
		run_k(DG_K_ESTIMATE, n, [&] {
			constexpr int GE = NF <= 4 ? 4 : 8;
			k_estimate<M><<<grid_for((long long) n * GE), BLOCK, 0, st_>>>(P_, C_, list, n, L, counterL, ++epoch_, Ls_.split,
			                                                                 d_cnt_);
		});
		if (tight) {
			sync_counters();
			check_status();
			const long long need = (long long) h_cnt_->top + (long long) NC * h_cnt_->n_split + 16;
			if (need > P_.cap) {
				const long long want = growth_target(need, std::max(need + need / 4, (long long) P_.cap * 5 / 4));
				grow_pool((int) std::min<long long>(want, 2000000000LL));
				list = Ls_.clu[L];
				ensure_scratch(n);  // the growth released the list scratch; the reassignment uses its marks
			}
		}
		const int gf = grid_for((long long) n * (NC + 1));
		run_k(DG_K_REGRID, n, [&] { k_unsplit_select<M><<<g, BLOCK, 0, st_>>>(P_, list, n, L, Ls_.unsplit, d_cnt_); });
		run_k(DG_K_REGRID, 0, [&] {
			k_split<M><<<gf, BLOCK, 0, st_>>>(P_, C_, &d_cnt_->n_split, Ls_.split, L, Ls_.fresh, ++epoch_, d_cnt_);
		});
		run_k(DG_K_REGRID, 0, [&] {
			k_unsplit<M><<<g, BLOCK, 0, st_>>>(P_, C_, &d_cnt_->n_unsplit, Ls_.unsplit, L, Ls_.fresh, ++epoch_, d_cnt_);
		});
		run_k(DG_K_REGRID, 0, [&] {
			k_nbr_fresh<M><<<gf, BLOCK, 0, st_>>>(P_, C_, &d_cnt_->n_new, Ls_.fresh, Ls_.upd, d_cnt_);
		});
		run_k(DG_K_REGRID, 0, [&] {
			k_nbr_list<M><<<grid_for((long long) n * (NC + 1) * NF), BLOCK, 0, st_>>>(P_, C_, &d_cnt_->n_upd, Ls_.upd, d_cnt_);
		});
		const bool ordered = opts_ & DG_OPT_ORDERED_LISTS;
		run_k(DG_K_REASSIGN, n, [&] {
			k_reassign<M><<<g, BLOCK, 0, st_>>>(P_, C_, list, nullptr, n, L, dtL, counterL, Ls_, d_cnt_,
			                                    ordered ? stay_marks() : nullptr);
			// the cells that stay at level L, in their list order (the count goes to n_tmp, which the
			// reassignment of the new cells then appends to)
			if (ordered) {
				size_t bytes = sel_tmp_bytes_;
				DG_CUDA(cub::DeviceSelect::Flagged(stay_marks() + stay_bytes(scratch_cap_), bytes, list, stay_marks(),
				                                   Ls_.tmp, &d_cnt_->n_tmp, n, st_));
			}
		});
		run_k(DG_K_REASSIGN, 0, [&] {
			k_reassign<M><<<gf, BLOCK, 0, st_>>>(P_, C_, Ls_.fresh, &d_cnt_->n_new, 0, L, dtL, counterL, Ls_, d_cnt_,
			                                     nullptr);
		});
		std::swap(Ls_.clu[L], Ls_.tmp);
		run_k(DG_K_OTHER, 0, [&] { k_set_count<<<1, 1, 0, st_>>>(&d_cnt_->clu[L], &d_cnt_->n_tmp); });
		DG_CUDA(cudaGetLastError());
	}

	void flush(int L) {
		if (h_cnt_->buf[L] == 0) return;
		run_k(DG_K_FLUSH, h_cnt_->buf[L], [&] {
			k_flush<<<grid_for(h_cnt_->buf[L]), BLOCK, 0, st_>>>(P_, Ls_.buf[L], &d_cnt_->buf[L], Ls_.clu[L],
			                                                   &d_cnt_->clu[L], L, d_cnt_);
		});
		DG_CUDA(cudaMemsetAsync(&d_cnt_->buf[L], 0, sizeof(int), st_));
		DG_CUDA(cudaGetLastError());
	}

public:
	// Integrator::integrate (impl/integrate.hpp:12-87)
	void step(int signal, int *force_break, double *global_dt, dg_substep_fn fn, void *user) override {
		C_.signal   = signal;
		C_.coarsen  = (n_global_ % coarsen_every_) == 0;
		*force_break = 0;
		const int top_seq = 1 << (MAX_ACTI - 1);
		int seq           = 0;
		while (true) {
			int finest = max_acti_;
			for (int l = MAX_ACTI - 1; l > finest; --l)
				if (h_cnt_->clu[l] > 0) {
					finest = l;
					break;
				}
			const int stride = 1 << (MAX_ACTI - 1 - finest);
			seq              = (seq / stride + 1) * stride;
			if (seq > top_seq) break;
			for (int l = 0; l < MAX_ACTI; ++l) {
				if (seq % (1 << l) != 0) continue;
				const int L = MAX_ACTI - l - 1;
				if (h_cnt_->clu[L] > 0 && L > max_acti_) {
					max_acti_     = L;
					acti_time_[L] = acti_time_[L - 1];
				}
				if (L > max_acti_) continue;
				substep(L);
				acti_counter_[L] = (acti_counter_[L] + 1) % 2;
				const double dtL = global_dt_ / (double) (1 << L);
				acti_time_[L] += dtL;
				flush(L);
				sync_counters();
				check_status();
				n_split_total_ += h_cnt_->n_split;
				n_unsplit_total_ += h_cnt_->n_unsplit;
				n_substeps_++;
				updates_ += h_cnt_->clu[L];
				if (h_cnt_->status & ST_NAN) {
					*force_break = 1;
					*global_dt   = global_dt_;
					return;
				}
				if (fn) fn(user, L, acti_time_[L], (int) n_substeps_, dtL, h_cnt_->clu[L]);
			}
		}
		n_global_++;
		if (gc_due()) gc();
		if (resort_) resort();
		*global_dt = global_dt_;
	}

	void set_resort(bool on) { resort_ = on; }

	// Morton re-sort of the node pool by (cluster, Z-order) at the end of a global step, when every
	// ACTI buffer is empty: each cluster becomes one contiguous slot range and its list the identity
	// over that range.
	void resort() {
		for (int l = 0; l < MAX_ACTI; ++l)
			if (h_cnt_->buf[l] != 0) return;
		const int top = h_cnt_->top;
		const int n   = top - 1;
		if (n <= 0) return;
		ensure_spare();
		size_t temp = 0;
		DG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint64_t *) nullptr, (uint64_t *) nullptr,
		                                        (int32_t *) nullptr, (int32_t *) nullptr, n, 0, 64, st_));
		const size_t need = align_up(sizeof(uint64_t) * n) * 2 + align_up(sizeof(int32_t) * n) * 2 +
		                    align_up(sizeof(int32_t) * (top + 1)) + align_up(temp);
		if (need > sort_bytes_) {
			cudaFree(sort_mem_);
			DG_CUDA(cudaMalloc(&sort_mem_, need));
			sort_bytes_ = need;
		}
		char *b          = (char *) sort_mem_;
		uint64_t *k_in   = (uint64_t *) b;
		b += align_up(sizeof(uint64_t) * n);
		uint64_t *k_out = (uint64_t *) b;
		b += align_up(sizeof(uint64_t) * n);
		int32_t *v_in = (int32_t *) b;
		b += align_up(sizeof(int32_t) * n);
		int32_t *v_out = (int32_t *) b;
		b += align_up(sizeof(int32_t) * n);
		int32_t *newidx = (int32_t *) b;
		b += align_up(sizeof(int32_t) * (top + 1));
		void *tmp = b;
		const int g = grid_for(n);
		run_k(DG_K_OTHER, 0, [&] { k_sort_keys<D><<<g, BLOCK, 0, st_>>>(P_, top, k_in, v_in); });
		DG_CUDA(cub::DeviceRadixSort::SortPairs(tmp, temp, k_in, k_out, v_in, v_out, n, 0, 64, st_));
		run_k(DG_K_OTHER, 0, [&] { k_sort_inverse<<<g, BLOCK, 0, st_>>>(v_out, n, newidx); });
		// each field in turn: permuted into the spare buffer, then copied back over slots [1, top)
		auto fo = fields(P_);
		for (size_t k = 0; k < fo.size(); ++k) {
			const int comps = fo[k].comps;
			if (comps <= 0) continue;
			const size_t elem = fo[k].elem;
			void *src = *fo[k].ptr, *dst = spare_mem_;
			run_k(DG_K_OTHER, 0, [&] {
				switch (elem) {
					case 1: k_permute<int8_t><<<g, BLOCK, 0, st_>>>((const int8_t *) src, (int8_t *) dst, comps, P_.cap, n, v_out); break;
					case 2: k_permute<int16_t><<<g, BLOCK, 0, st_>>>((const int16_t *) src, (int16_t *) dst, comps, P_.cap, n, v_out); break;
					case 4: k_permute<int32_t><<<g, BLOCK, 0, st_>>>((const int32_t *) src, (int32_t *) dst, comps, P_.cap, n, v_out); break;
					case 8: k_permute<double><<<g, BLOCK, 0, st_>>>((const double *) src, (double *) dst, comps, P_.cap, n, v_out); break;
					default:  // one record of elem bytes per node
						k_permute_words<<<grid_for((long long) n * (elem / 8)), BLOCK, 0, st_>>>(
						    (const double *) src, (double *) dst, (int) (elem / 8), n, v_out);
						break;
				}
			});
			DG_CUDA(cudaMemcpy2DAsync((char *) src + elem, elem * (size_t) P_.cap, (const char *) dst + elem,
			                          elem * (size_t) P_.cap, elem * (size_t) n, comps, cudaMemcpyDeviceToDevice, st_));
		}
		run_k(DG_K_OTHER, 0, [&] { k_remap_links<D><<<grid_for(top), BLOCK, 0, st_>>>(P_, top, newidx); });
		int first = 1;
		for (int l = 0; l < MAX_ACTI; ++l) {
			const int cnt = h_cnt_->clu[l];
			if (cnt > 0) run_k(DG_K_OTHER, 0, [&] { k_fill_range<<<grid_for(cnt), BLOCK, 0, st_>>>(Ls_.clu[l], first, cnt); });
			first += cnt;
		}
		DG_CUDA(cudaGetLastError());
		sync_counters();
	}

private:
	// Integrator::gc (impl/acti_utils.hpp:59-74): compact the node slots, then reassign every active
	// leaf to an ACTI level from its stored max_dt, resetting the hysteresis.
	void gc() {
		const int top = h_cnt_->top;
		for (int l = 0; l < MAX_ACTI; ++l)
			if (h_cnt_->buf[l] != 0) throw dg_error(DG_ERR_UNSUPPORTED, "garbage collection with non-empty ACTI buffers");
		int32_t *keep = nullptr, *newidx = nullptr;
		DG_CUDA(cudaMalloc(&keep, sizeof(int32_t) * (top + 1)));
		DG_CUDA(cudaMalloc(&newidx, sizeof(int32_t) * (top + 1)));
		const int g = grid_for(top);
		k_gc_keep<<<g, BLOCK, 0, st_>>>(P_, top, keep);
		size_t tmp_bytes = 0;
		DG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, keep, newidx, top + 1, st_));
		void *tmp = nullptr;
		DG_CUDA(cudaMalloc(&tmp, tmp_bytes));
		DG_CUDA(cudaMemsetAsync(keep + top, 0, sizeof(int32_t), st_));
		DG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, keep, newidx, top + 1, st_));
		int new_top = 0;
		DG_CUDA(cudaMemcpyAsync(&new_top, newidx + top, sizeof(int), cudaMemcpyDeviceToHost, st_));
		// each field in turn: kept slots compacted into the zeroed spare buffer, which is then copied back
		// whole (slots from new_top on end up zero)
		ensure_spare();
		auto fo = fields(P_);
		for (size_t k = 0; k < fo.size(); ++k) {
			if (fo[k].comps <= 0) continue;
			const size_t bytes = fo[k].elem * (size_t) P_.cap * fo[k].comps;
			DG_CUDA(cudaMemsetAsync(spare_mem_, 0, bytes, st_));
			k_gc_move<<<g, BLOCK, 0, st_>>>((const char *) *fo[k].ptr, (char *) spare_mem_, (int) fo[k].elem, fo[k].comps,
			                                 P_.cap, top, keep, newidx);
			DG_CUDA(cudaMemcpyAsync(*fo[k].ptr, spare_mem_, bytes, cudaMemcpyDeviceToDevice, st_));
		}
		DG_CUDA(cudaStreamSynchronize(st_));
		k_gc_remap<D><<<grid_for(new_top), BLOCK, 0, st_>>>(P_, new_top, keep, newidx);
		// full ACTI reassignment
		Counters z{};
		z.top    = new_top;
		z.status = 0;
		// the running totals that a batched step keeps on the device carry over (the host copy is current:
		// gc runs after the step's last read-back)
		z.n_split_total    = h_cnt_->n_split_total;
		z.n_unsplit_total  = h_cnt_->n_unsplit_total;
		z.n_updates_total  = h_cnt_->n_updates_total;
		z.n_substeps_total = h_cnt_->n_substeps_total;
		DG_CUDA(cudaMemcpyAsync(d_cnt_, &z, sizeof(Counters), cudaMemcpyHostToDevice, st_));
		k_collect_active_leaves<<<grid_for(new_top), BLOCK, 0, st_>>>(P_, new_top, Ls_.fresh, &d_cnt_->n_new);
		DG_CUDA(cudaStreamSynchronize(st_));
		int n_leaves = 0;
		DG_CUDA(cudaMemcpy(&n_leaves, &d_cnt_->n_new, sizeof(int), cudaMemcpyDeviceToHost));
		k_assign<M><<<grid_for(n_leaves), BLOCK, 0, st_>>>(P_, C_, Ls_.fresh, n_leaves, global_dt_, Ls_, d_cnt_);
		DG_CUDA(cudaGetLastError());
		sync_counters();
		check_status();
		cudaFree(tmp);
		cudaFree(keep);
		cudaFree(newidx);
		n_gc_++;
	}

public:
	long long cell_count() override {
		long long n = 0;
		for (int l = 0; l < MAX_ACTI; ++l) n += h_cnt_->clu[l] + h_cnt_->buf[l];
		return n;
	}

	long long read_cells(int *levels, double *data, long long max_cells) override {
		constexpr int W = D + 1 + 2 * E + 3 + M::P;
		long long n = cell_count();
		if (n > max_cells) throw dg_error(DG_ERR_ARG, "read buffer too small");
		if (n > read_cap_) {
			cudaFree(d_read_);
			cudaFree(d_readlv_);
			DG_CUDA(cudaMalloc(&d_read_, sizeof(double) * W * n));
			DG_CUDA(cudaMalloc(&d_readlv_, sizeof(int32_t) * 2 * n));
			read_cap_ = n;
		}
		long long base = 0;
		for (int pass = 0; pass < 2; ++pass) {
			for (int l = 0; l < MAX_ACTI; ++l) {
				int cnt = pass == 0 ? h_cnt_->clu[l] : h_cnt_->buf[l];
				if (cnt == 0) continue;
				const int32_t *list = pass == 0 ? Ls_.clu[l] : Ls_.buf[l];
				k_gather_cells<M><<<grid_for(cnt), BLOCK, 0, st_>>>(P_, list, cnt, (int) base, d_read_, d_readlv_);
				base += cnt;
			}
		}
		DG_CUDA(cudaGetLastError());
		DG_CUDA(cudaMemcpyAsync(data, d_read_, sizeof(double) * W * n, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaMemcpyAsync(levels, d_readlv_, sizeof(int32_t) * 2 * n, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		return n;
	}

	// `width` doubles per active cell, gathered by `launch(list, count, base, out)` in read_cells' order.
	template<class F>
	long long read_per_cell(double *data, long long max_cells, int width, const char *what, F launch) {
		const long long n = cell_count();
		if (n > max_cells) throw dg_error(DG_ERR_ARG, "read buffer too small");
		double *d_out = nullptr;
		DG_CUDA(cudaMalloc(&d_out, sizeof(double) * width * (n > 0 ? n : 1)));
		long long base = 0;
		for (int pass = 0; pass < 2; ++pass) {
			for (int l = 0; l < MAX_ACTI; ++l) {
				const int cnt = pass == 0 ? h_cnt_->clu[l] : h_cnt_->buf[l];
				if (cnt == 0) continue;
				launch(pass == 0 ? Ls_.clu[l] : Ls_.buf[l], cnt, (int) base, d_out);
				base += cnt;
			}
		}
		cudaError_t e = cudaGetLastError();
		if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(data, d_out, sizeof(double) * width * n, cudaMemcpyDeviceToHost, st_);
		if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
		cudaFree(d_out);
		if (e != cudaSuccess) throw dg_error(DG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
		return n;
	}

	// Limited slopes of the active cells, [D][E] per cell, in read_cells' order.
	long long read_slopes(double *data, long long max_cells) override {
		return read_per_cell(data, max_cells, D * E, "read_slopes", [&](const int32_t *list, int cnt, int base, double *o) {
			k_gather_slopes<M><<<grid_for(cnt), BLOCK, 0, st_>>>(P_, list, cnt, base, o);
		});
	}

	// Regrid-forecaster features, [5 + 5D] per active cell, in read_cells' order.
	long long forecast_features(double *data, long long max_cells) override {
		return read_per_cell(data, max_cells, 5 + 5 * D, "forecast_features",
		                     [&](const int32_t *list, int cnt, int base, double *o) {
			                     k_forecast_features<M><<<grid_for(cnt), BLOCK, 0, st_>>>(P_, C_, list, cnt, base, o);
		                     });
	}
	int dims() const override { return D; }

	long long tree_size() override { return h_cnt_->top; }

	// The whole node pool, slots [0, top), component-major as the pool stores it: parent[n],
	// child[C][n], level[n], flags[n], p[E][n], meta[4][n] = {acti_level, error, max_dt, cfl}. Internal,
	// inactive and garbage slots included: what a hyper-tree writer walks from the root.
	long long read_tree(int32_t *parent, int32_t *child, int32_t *level, uint32_t *flags, double *p, double *meta,
	                    long long max_nodes) override {
		const long long n = h_cnt_->top;
		if (n > max_nodes) throw dg_error(DG_ERR_ARG, "read buffer too small");
		const size_t cap = (size_t) P_.cap, nn = (size_t) n;
		std::vector<int8_t> lv(nn), ac(nn);
		auto rows = [&](void *dst, const void *src, size_t elem, int comps) {
			DG_CUDA(cudaMemcpy2DAsync(dst, elem * nn, src, elem * cap, elem * nn, comps, cudaMemcpyDeviceToHost, st_));
		};
		rows(parent, P_.parent, 4, 1);
		rows(child, P_.child, 4, NC);
		rows(lv.data(), P_.level, 1, 1);
		rows(ac.data(), P_.acti, 1, 1);
		rows(flags, P_.flags, 4, 1);
		rows(p, P_.p, 8, E);
		rows(meta + nn, P_.err, 8, 1);
		rows(meta + 2 * nn, P_.maxdt, 8, 1);
		rows(meta + 3 * nn, P_.cfl, 8, 1);
		DG_CUDA(cudaStreamSynchronize(st_));
		for (size_t i = 0; i < nn; ++i) {
			level[i] = lv[i];
			meta[i]  = (double) ac[i];
			flags[i] &= F_PUBLIC;
		}
		return n;
	}

	// Forecast-driven regrid: F_HOLD on the active cells (read_cells' order) and the interval in global
	// steps between coarsening passes (1 = every step, the reference's behaviour).
	void set_hold(const uint8_t *hold, long long n) override {
		if (n != cell_count()) throw dg_error(DG_ERR_ARG, "dg_set_hold: one entry per active cell expected");
		uint8_t *d = nullptr;
		DG_CUDA(cudaMalloc(&d, n > 0 ? n : 1));
		cudaError_t e = n > 0 ? cudaMemcpyAsync(d, hold, n, cudaMemcpyHostToDevice, st_) : cudaSuccess;
		long long base = 0;
		for (int pass = 0; e == cudaSuccess && pass < 2; ++pass) {
			for (int l = 0; l < MAX_ACTI; ++l) {
				const int cnt = pass == 0 ? h_cnt_->clu[l] : h_cnt_->buf[l];
				if (cnt == 0) continue;
				k_set_hold<M><<<grid_for(cnt), BLOCK, 0, st_>>>(P_, pass == 0 ? Ls_.clu[l] : Ls_.buf[l], cnt, (int) base, d);
				base += cnt;
			}
		}
		if (e == cudaSuccess) e = cudaGetLastError();
		if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
		cudaFree(d);
		if (e != cudaSuccess) throw dg_error(DG_ERR_CUDA, std::string("set_hold: ") + cudaGetErrorString(e));
	}
	void set_coarsen_interval(int k) override {
		if (k < 1) throw dg_error(DG_ERR_ARG, "dg_set_coarsen_interval: interval must be >= 1");
		coarsen_every_ = k;
	}

	// Gradients of the gradient inputs, [D][G] per active cell, in read_cells' order.
	long long read_gradients(double *data, long long max_cells) override {
		if constexpr (M::G == 0) {
			throw dg_error(DG_ERR_UNSUPPORTED, "dg_read_gradients: the Euler model has no gradient inputs");
		} else {
			if (!visc_)
				throw dg_error(DG_ERR_UNSUPPORTED, "dg_read_gradients: gradients are kept only when the case has viscous "
				                                   "or heat-conduction terms");
			return read_per_cell(data, max_cells, D * M::G, "read_gradients",
			                     [&](const int32_t *list, int cnt, int base, double *o) {
				                     k_gather_grads<M><<<grid_for(cnt), BLOCK, 0, st_>>>(P_, list, cnt, base, o);
			                     });
		}
	}

	// Same records as read_cells, gathered through caller-owned device scratch of `bytes` bytes;
	// allocates nothing.
	int model_id() const override { return M::ID; }

	void prepare_noalloc() override {
		cudaFuncAttributes a{};
		DG_CUDA(cudaFuncGetAttributes(&a, k_gather_cells<M>));
	}

	long long read_cells_via(int *levels, double *data, long long max_cells, void *scratch, size_t bytes) override {
		constexpr int W = D + 1 + 2 * E + 3 + M::P;
		const long long n = cell_count();
		if (n > max_cells) throw dg_error(DG_ERR_ARG, "read buffer too small");
		const size_t rec_bytes = align_up(sizeof(double) * W * (size_t) n);
		const size_t need      = rec_bytes + sizeof(int32_t) * 2 * (size_t) n;
		const size_t per_cell  = sizeof(double) * W + sizeof(int32_t) * 2;
		if (need > bytes)
			throw dg_error(DG_ERR_CAPACITY, "dg_read_cells_noalloc: " + std::to_string(n) + " active cells need " +
			                                    std::to_string(need) + " bytes of scratch; the allocation-free scratch holds " +
			                                    std::to_string(bytes) + " bytes (about " +
			                                    std::to_string((bytes - 256) / per_cell) + " cells of this model)");
		double *d_rec = (double *) scratch;
		int32_t *d_lv = (int32_t *) ((char *) scratch + rec_bytes);
		long long base = 0;
		for (int pass = 0; pass < 2; ++pass) {
			for (int l = 0; l < MAX_ACTI; ++l) {
				int cnt = pass == 0 ? h_cnt_->clu[l] : h_cnt_->buf[l];
				if (cnt == 0) continue;
				const int32_t *list = pass == 0 ? Ls_.clu[l] : Ls_.buf[l];
				k_gather_cells<M><<<grid_for(cnt), BLOCK, 0, st_>>>(P_, list, cnt, (int) base, d_rec, d_lv);
				base += cnt;
			}
		}
		DG_CUDA(cudaGetLastError());
		if (n > 0) {
			DG_CUDA(cudaMemcpyAsync(data, d_rec, sizeof(double) * W * n, cudaMemcpyDeviceToHost, st_));
			DG_CUDA(cudaMemcpyAsync(levels, d_lv, sizeof(int32_t) * 2 * n, cudaMemcpyDeviceToHost, st_));
		}
		DG_CUDA(cudaStreamSynchronize(st_));
		return n;
	}

	void stats(dg_stats *o) override {
		std::memset(o, 0, sizeof(*o));
		for (int l = 0; l < MAX_ACTI; ++l) {
			o->n_clusters[l]   = h_cnt_->clu[l];
			o->n_buffers[l]    = h_cnt_->buf[l];
			o->acti_time[l]    = acti_time_[l];
			o->acti_counter[l] = acti_counter_[l];
		}
		o->tree_size      = h_cnt_->top + pruned_;
		o->n_splits       = n_split_total_;
		o->n_unsplits     = n_unsplit_total_;
		o->n_gc           = n_gc_;
		o->n_substeps     = n_substeps_;
		o->n_global_steps = n_global_;
		o->cell_updates   = updates_;
		o->max_acti_level = max_acti_;
		o->global_dt      = global_dt_;
		o->n_launches     = n_launches_;
		for (int k = 0; k < DG_NK; ++k) {
			o->kernel_ms[k]       = kms_[k];
			o->kernel_launches[k] = klaunch_[k];
			o->kernel_cells[k]    = kcells_[k];
		}
	}
};

SolverBase *make_solver_euler(const dg_case &c);
SolverBase *make_solver_ns(const dg_case &c);
SolverBase *make_solver_multi(const dg_case &c);
class BatchBase;
BatchBase *make_batch_euler(const std::vector<SolverBase *> &s);
BatchBase *make_batch_ns(const std::vector<SolverBase *> &s);
BatchBase *make_batch_multi(const std::vector<SolverBase *> &s);

}  // namespace dg
