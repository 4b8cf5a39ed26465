// Batched trees: many independent solvers of one model advanced in lockstep by one host thread, with
// one launch per stage for all trees that run a level.
//
// Every tree keeps its own node pool, lists, counters and ACTI schedule state, so each tree computes
// exactly what it computes alone (impl/integrate.hpp:26-87 per tree). The trees' schedules are merged:
// the global-step sequence counter advances with the stride of the finest level of any tree, and at
// each sequence value a level substep runs for the trees whose schedule contains it. A tree whose
// finest level is coarser simply has no substep at sequence values that only finer levels use, which
// is the stride skip of its own schedule. The stage kernels run over a block range per tree (the
// blocks of a launch are split among the trees in proportion to their work), all counters live in one
// array that comes back with a single copy per substep, and there is one synchronisation per merged
// substep instead of one per tree and substep.
#pragma once

#include "solver.cuh"

namespace dg {

// Per-tree arguments of the batched stage kernels for one merged substep.
struct TreeArgs {
	Pool P;
	const Consts *C;  // device copy of the tree's constants
	BcTable B;
	Lists Ls;
	Counters *cnt;
	const int32_t *list;  // the tree's cluster list of the running level, as the substep starts
	int n;                // its length
	int L;
	double dtL;
	int counterL;
	int stamp;
	int epoch0;  // the tree's epoch counter before the substep (kernels use epoch0 + k)
	int limiter;
};

// The tree of the calling block: off[t] <= blockIdx.x < off[t + 1].
__device__ __forceinline__ int tree_of_block(const int *off, int nt) {
	int lo = 0, hi = nt - 1;
	const int b = (int) blockIdx.x;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (__ldg(off + mid) <= b) lo = mid;
		else hi = mid - 1;
	}
	return lo;
}

#define DG_BATCH_PROLOGUE                                     \
	if ((int) blockIdx.x >= off[nt]) return;                  \
	const int t_ = tree_of_block(off, nt);                    \
	const TreeArgs &a = A[t_];                                \
	const BlockRange g{off[t_], off[t_ + 1] - off[t_]};

// Counters n_recv .. status of every tree to zero (one block per tree).
static __global__ void kb_zero_counters(const TreeArgs *A, int nt) {
	const int t = blockIdx.x;
	if (t >= nt) return;
	Counters *c = A[t].cnt;
	char *b = (char *) &c->n_recv, *e = (char *) (&c->status + 1);
	for (int k = threadIdx.x; k < (int) (e - b) / 4; k += blockDim.x) ((int *) b)[k] = 0;
}

template<class M, bool V, class S>
__global__ void __launch_bounds__(BLOCK, 2) kb_face_sum(const TreeArgs *A, const int *off, int nt) {
	DG_BATCH_PROLOGUE
	d_face_sum<M, V, S>(g, a.P, *a.C, a.B, a.list, a.n, a.L, a.dtL, a.stamp, a.Ls.recv, a.cnt);
}

template<class M, class T>
__global__ void __launch_bounds__(BLOCK) kb_flux_receive(const TreeArgs *A, const int *off, int nt) {
	DG_BATCH_PROLOGUE
	d_flux_receive<M, T>(g, a.P, a.Ls.recv, &a.cnt->n_recv, a.L, a.cnt);
}

template<class M, bool V>
__global__ void __launch_bounds__(BLOCK, 3) kb_update(const TreeArgs *A, const int *off, int nt) {
	DG_BATCH_PROLOGUE
	d_update<M, V>(g, a.P, *a.C, a.list, a.n, a.dtL, a.epoch0 + 1, a.cnt);
}

template<class M, bool V>
__global__ void __launch_bounds__(BLOCK) kb_slope(const TreeArgs *A, const int *off, int nt) {
	DG_BATCH_PROLOGUE
	d_slope<M, V>(g, a.P, *a.C, a.B, a.list, a.n, a.limiter, a.epoch0 + 2, a.cnt);
}

// Multiphase auxiliary stages; `k` selects the stage in the order of Solver::multiphase_aux.
template<class M>
__global__ void __launch_bounds__(BLOCK) kb_aux(const TreeArgs *A, const int *off, int nt, int k) {
	DG_BATCH_PROLOGUE
	const int e_upd = a.epoch0 + 1;
	switch (k) {
		case 0: d_smooth_alpha<M>(g, a.P, *a.C, a.B, a.list, a.n, nullptr, a.P.tmp, a.L, a.epoch0 + 3, e_upd, a.cnt); break;
		case 1: d_smooth_alpha<M>(g, a.P, *a.C, a.B, a.list, a.n, a.P.tmp, a.P.tmp2, a.L, a.epoch0 + 4, e_upd, a.cnt); break;
		case 2:
			d_smooth_alpha<M>(g, a.P, *a.C, a.B, a.list, a.n, a.P.tmp2, a.P.k + (size_t) M::ALPHAS * a.P.cap, a.L, a.epoch0 + 5,
			                  e_upd, a.cnt);
			break;
		case 4: d_normal<M>(g, a.P, *a.C, a.B, a.list, a.n, a.epoch0 + 6, e_upd, a.cnt); break;
		case 5: d_curvature<M>(g, a.P, *a.C, a.B, a.list, a.n, a.cnt); break;
		case 6: d_smooth_kappa<M>(g, a.P, *a.C, a.B, a.list, a.n, a.cnt); break;
		case 7: d_store_tmp(g, a.P, a.list, a.n, M::KAPPA, a.P.tmp); break;
		default: d_rec_k<M>(g, a.P, a.list, a.n); break;
	}
}

// Epochs of one substep in the tree's own sequence (Solver::substep): update + 1, slope + 2, the four
// multiphase sweeps + 3 .. + 6, then the estimate, the split and the unsplit.
template<class M>
constexpr int EPOCH_EST = M::MULTI ? 7 : 3;

template<class M>
__global__ void __launch_bounds__(BLOCK) kb_estimate(const TreeArgs *A, const int *off, int nt) {
	DG_BATCH_PROLOGUE
	d_estimate<M>(g, a.P, *a.C, a.list, a.n, a.L, a.counterL, a.epoch0 + EPOCH_EST<M>, a.Ls.split, a.cnt);
}

// Regrid and reassignment stages in the order of Solver::substep; `k` selects the stage.
template<class M>
__global__ void kb_regrid(const TreeArgs *A, const int *off, int nt, int k) {
	DG_BATCH_PROLOGUE
	constexpr int EX = EPOCH_EST<M>;
	switch (k) {
		case 0: d_unsplit_select<M>(g, a.P, a.list, a.n, a.L, a.Ls.unsplit, a.cnt); break;
		case 1: d_split<M>(g, a.P, *a.C, &a.cnt->n_split, a.Ls.split, a.L, a.Ls.fresh, a.epoch0 + EX + 1, a.cnt); break;
		case 2: d_unsplit<M>(g, a.P, *a.C, &a.cnt->n_unsplit, a.Ls.unsplit, a.L, a.Ls.fresh, a.epoch0 + EX + 2, a.cnt); break;
		case 3: d_nbr_fresh<M>(g, a.P, *a.C, &a.cnt->n_new, a.Ls.fresh, a.Ls.upd, a.cnt); break;
		case 4: d_nbr_list<M>(g, a.P, *a.C, &a.cnt->n_upd, a.Ls.upd, a.cnt); break;
		case 5: d_reassign<M>(g, a.P, *a.C, a.list, nullptr, a.n, a.L, a.dtL, a.counterL, a.Ls, a.cnt); break;
		default: d_reassign<M>(g, a.P, *a.C, a.Ls.fresh, &a.cnt->n_new, 0, a.L, a.dtL, a.counterL, a.Ls, a.cnt); break;
	}
}

// The rebuilt cluster list's count (the lists themselves are swapped on the host).
static __global__ void kb_set_count(const TreeArgs *A, int nt) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < nt) A[t].cnt->clu[A[t].L] = A[t].cnt->n_tmp;
}

// flush_acti_buffer of level L for the listed trees, then the buffer count to zero.
static __global__ void kb_flush(const TreeArgs *A, const int *off, int nt) {
	DG_BATCH_PROLOGUE
	d_flush(g, a.P, a.Ls.buf[a.L], &a.cnt->buf[a.L], a.Ls.clu[a.L], &a.cnt->clu[a.L], a.L, a.cnt);
}
static __global__ void kb_flush_done(const TreeArgs *A, int nt) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < nt) A[t].cnt->buf[A[t].L] = 0;
}

#undef DG_BATCH_PROLOGUE

// Stage kinds of a merged substep, each with its own launch budget (blocks per SM) and timing.
enum BatchStage : int {
	BS_FACE_SUM = 0, BS_RECEIVE, BS_UPDATE, BS_SLOPE, BS_AUX, BS_ESTIMATE, BS_REGRID_CELL, BS_REGRID_FRESH,
	BS_NBR_LIST, BS_FLUSH, BS_N
};

class BatchBase {
public:
	virtual ~BatchBase() = default;
	virtual void step(int signal, int *force_break, double *global_dt) = 0;
	virtual int size() const = 0;
	virtual void set_launch(const int *blocks_per_sm, int n) = 0;
	virtual void set_profiling(bool on) = 0;
	virtual void stage_times(double *ms, long long *items, int n) = 0;
	std::string last_error;
};

template<class M>
class Batch : public BatchBase {
	static constexpr int D = M::D, NC = 1 << D, NF = 2 * D;
	static constexpr int EPOCHS = EPOCH_EST<M> + 2;  // epoch numbers one substep uses per tree
	std::vector<Solver<M> *> s_;
	cudaStream_t st_      = nullptr;
	Counters *d_cnt_      = nullptr;  // all trees' counters
	Counters *h_cnt_      = nullptr;  // pinned
	std::vector<Counters *> own_d_, own_h_;
	Consts *d_consts_     = nullptr;  // all trees' constants
	TreeArgs *d_args_     = nullptr, *h_args_ = nullptr;
	int *d_off_           = nullptr, *h_off_ = nullptr;
	int n_off_sets_       = 0;
	int device_           = 0;
	int sms_              = 148;
	bool mixed_ = false, visc_ = false, sigma_ = false;
	int bps_[BS_N];  // launch budget per stage kind: blocks per SM
	bool prof_ = false;
	struct Timed {
		int stage;
		cudaEvent_t a, b;
		long long items;
	};
	std::vector<Timed> timed_;
	std::vector<cudaEvent_t> ev_free_;
	double stage_ms_[BS_N]       = {};
	long long stage_items_[BS_N] = {};

	static constexpr int OFF_SETS = 24;  // block-offset arrays one substep may use

public:
	explicit Batch(const std::vector<SolverBase *> &solvers) {
		if (solvers.empty()) throw dg_error(DG_ERR_ARG, "empty batch");
		for (auto *b: solvers) {
			auto *s = dynamic_cast<Solver<M> *>(b);
			if (!s) throw dg_error(DG_ERR_ARG, "batched solvers must share one model and dimension");
			s_.push_back(s);
		}
		mixed_ = s_[0]->mixed_;
		visc_  = s_[0]->visc_;
		sigma_ = s_[0]->sigma_;
		for (auto *s: s_)
			if (s->mixed_ != mixed_ || s->visc_ != visc_ || s->sigma_ != sigma_)
				throw dg_error(DG_ERR_ARG, "batched solvers must share the numeric form and the viscous/tension terms");
		const int nt = (int) s_.size();
		for (int k = 0; k < BS_N; ++k) bps_[k] = 16;
		DG_CUDA(cudaGetDevice(&device_));
		DG_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
		DG_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
		DG_CUDA(cudaMalloc(&d_cnt_, sizeof(Counters) * nt));
		DG_CUDA(cudaMallocHost(&h_cnt_, sizeof(Counters) * nt));
		DG_CUDA(cudaMalloc(&d_consts_, sizeof(Consts) * nt));
		DG_CUDA(cudaMalloc(&d_args_, sizeof(TreeArgs) * nt));
		DG_CUDA(cudaMallocHost(&h_args_, sizeof(TreeArgs) * nt));
		DG_CUDA(cudaMalloc(&d_off_, sizeof(int) * (nt + 1) * OFF_SETS));
		DG_CUDA(cudaMallocHost(&h_off_, sizeof(int) * (nt + 1) * OFF_SETS));
		// every solver moves onto the batch's stream and its counters into the batch's array
		for (int t = 0; t < nt; ++t) {
			Solver<M> *s = s_[t];
			DG_CUDA(cudaStreamSynchronize(s->st_));
			s->st_ = st_;
			DG_CUDA(cudaMemcpy(d_cnt_ + t, s->d_cnt_, sizeof(Counters), cudaMemcpyDeviceToDevice));
			h_cnt_[t] = *s->h_cnt_;
			own_d_.push_back(s->d_cnt_);
			own_h_.push_back(s->h_cnt_);
			s->d_cnt_ = d_cnt_ + t;
			s->h_cnt_ = h_cnt_ + t;
		}
	}

	~Batch() override {
		cudaStreamSynchronize(st_);
		// counters and streams go back to the solvers
		for (size_t t = 0; t < s_.size(); ++t) {
			Solver<M> *s = s_[t];
			cudaMemcpy(own_d_[t], d_cnt_ + t, sizeof(Counters), cudaMemcpyDeviceToDevice);
			*own_h_[t] = h_cnt_[t];
			s->d_cnt_ = own_d_[t];
			s->h_cnt_ = own_h_[t];
			s->st_    = 0;
		}
		cudaFree(d_cnt_);
		cudaFreeHost(h_cnt_);
		cudaFree(d_consts_);
		cudaFree(d_args_);
		cudaFreeHost(h_args_);
		cudaFree(d_off_);
		cudaFreeHost(h_off_);
		for (auto &t: timed_) cudaEventDestroy(t.a), cudaEventDestroy(t.b);
		for (auto e: ev_free_) cudaEventDestroy(e);
		cudaStreamDestroy(st_);
	}

	int size() const override { return (int) s_.size(); }

	void set_launch(const int *bps, int n) override {
		for (int k = 0; k < n && k < BS_N; ++k)
			if (bps[k] < 1 || bps[k] > 64) throw dg_error(DG_ERR_ARG, "blocks per SM must lie in [1, 64]");
		for (int k = 0; k < n && k < BS_N; ++k) bps_[k] = bps[k];
	}

	void set_profiling(bool on) override { prof_ = on; }

	// Device time and work items per stage kind since the last call (profiling on), then reset.
	void stage_times(double *ms, long long *items, int n) override {
		drain();
		for (int k = 0; k < n && k < BS_N; ++k) {
			ms[k]           = stage_ms_[k];
			items[k]        = stage_items_[k];
			stage_ms_[k]    = 0.0;
			stage_items_[k] = 0;
		}
	}

private:
	cudaEvent_t event() {
		if (ev_free_.empty()) {
			cudaEvent_t e;
			DG_CUDA(cudaEventCreate(&e));
			return e;
		}
		cudaEvent_t e = ev_free_.back();
		ev_free_.pop_back();
		return e;
	}

	void drain() {
		for (auto &t: timed_) {
			float ms = 0.f;
			DG_CUDA(cudaEventSynchronize(t.b));
			DG_CUDA(cudaEventElapsedTime(&ms, t.a, t.b));
			stage_ms_[t.stage] += ms;
			stage_items_[t.stage] += t.items;
			ev_free_.push_back(t.a);
			ev_free_.push_back(t.b);
		}
		timed_.clear();
	}

	void sync() {
		DG_CUDA(cudaMemcpyAsync(h_cnt_, d_cnt_, sizeof(Counters) * s_.size(), cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		if (prof_) drain();
	}

	// One launch of a stage over the trees of `sel`: block offsets in proportion to `items` within the
	// stage's budget; `launch(grid, offsets)` issues the kernel; timed with events when profiling.
	template<class F>
	void stage(int kind, const std::vector<int> &sel, const std::vector<long long> &items, F &&launch) {
		auto o = offsets(sel, items, sms_ * bps_[kind]);
		cudaEvent_t a = nullptr, b = nullptr;
		if (prof_) {
			a = event();
			b = event();
			DG_CUDA(cudaEventRecord(a, st_));
		}
		launch(o.second, o.first);
		if (prof_) {
			DG_CUDA(cudaEventRecord(b, st_));
			long long tot = 0;
			for (auto v: items) tot += v;
			timed_.push_back({kind, a, b, tot});
		}
	}

	// Block offsets of one stage: tree k of `sel` gets blocks in proportion to its items (at least one),
	// the launch at most `cap` blocks in total unless every tree needs its one. Returns the device array
	// and the launch's block count.
	std::pair<const int *, int> offsets(const std::vector<int> &sel, const std::vector<long long> &items,
	                                    int cap = 148 * 16) {
		if (n_off_sets_ >= OFF_SETS) throw dg_error(DG_ERR_UNSUPPORTED, "batch: too many stages in one substep");
		const int nt = (int) sel.size();
		int *h       = h_off_ + (size_t) n_off_sets_ * (s_.size() + 1);
		int *d       = d_off_ + (size_t) n_off_sets_ * (s_.size() + 1);
		long long want = 0;
		std::vector<long long> nb(nt);
		for (int k = 0; k < nt; ++k) {
			nb[k] = std::max<long long>(1, (items[k] + BLOCK - 1) / BLOCK);
			want += nb[k];
		}
		if (want > cap) {
			const double f = (double) cap / (double) want;
			for (int k = 0; k < nt; ++k) nb[k] = std::max<long long>(1, (long long) (nb[k] * f));
		}
		h[0] = 0;
		for (int k = 0; k < nt; ++k) h[k + 1] = h[k] + (int) nb[k];
		DG_CUDA(cudaMemcpyAsync(d, h, sizeof(int) * (nt + 1), cudaMemcpyHostToDevice, st_));
		++n_off_sets_;
		return {d, h[nt]};
	}

	void upload_args(const std::vector<int> &sel) {
		DG_CUDA(cudaMemcpyAsync(d_args_, h_args_, sizeof(TreeArgs) * sel.size(), cudaMemcpyHostToDevice, st_));
	}

	// One merged level-L substep of the trees in `sel` (Solver::substep, tree by tree identical).
	void substep(int L, const std::vector<int> &sel) {
		const int nt = (int) sel.size();
		n_off_sets_  = 0;
		std::vector<long long> n(nt);
		bool any_tight = false;
		std::vector<char> tight(nt, 0);
		for (int k = 0; k < nt; ++k) {
			Solver<M> *s = s_[sel[k]];
			n[k]         = s->h_cnt_->clu[L];
			s->ensure_scratch(n[k]);
			tight[k] = (long long) s->h_cnt_->top + (long long) NC * n[k] + 16 > s->P_.cap;
			any_tight |= tight[k] != 0;
			TreeArgs &a = h_args_[k];
			a.P         = s->P_;
			a.C         = d_consts_ + sel[k];
			a.B         = s->B_;
			a.Ls        = s->Ls_;
			a.cnt       = s->d_cnt_;
			a.list      = s->Ls_.clu[L];
			a.n         = (int) n[k];
			a.L         = L;
			a.dtL       = s->global_dt_ / (double) (1 << L);
			a.counterL  = s->acti_counter_[L];
			a.stamp     = ++s->stamp_;
			a.epoch0    = s->epoch_;
			a.limiter   = s->limiter_;
			s->epoch_ += EPOCHS;
		}
		upload_args(sel);
		auto scaled = [&](long long mul) {
			std::vector<long long> v(nt);
			for (int k = 0; k < nt; ++k) v[k] = n[k] * mul;
			return v;
		};
		constexpr int G = NF <= 4 ? 4 : 8;
		kb_zero_counters<<<nt, 32, 0, st_>>>(d_args_, nt);
		const auto lanes = scaled(G), cells = scaled(1), fresh = scaled(NC + 1), repair = scaled((NC + 1) * NF);
		stage(BS_FACE_SUM, sel, lanes, [&](int grid, const int *off) {
			if (mixed_) {
				if (visc_) kb_face_sum<M, true, float><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
				else kb_face_sum<M, false, float><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
			} else {
				if (visc_) kb_face_sum<M, true, double><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
				else kb_face_sum<M, false, double><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
			}
		});
		stage(BS_RECEIVE, sel, lanes, [&](int grid, const int *off) {
			if (mixed_) kb_flux_receive<M, float><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
			else kb_flux_receive<M, double><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
		});
		stage(BS_UPDATE, sel, cells, [&](int grid, const int *off) {
			if (visc_) kb_update<M, true><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
			else kb_update<M, false><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
		});
		stage(BS_SLOPE, sel, lanes, [&](int grid, const int *off) {
			if (visc_) kb_slope<M, true><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
			else kb_slope<M, false><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt);
		});
		if constexpr (M::MULTI) {
			// the smoothing sweeps and the normal run a lane group per cell, the curvature stages a thread
			for (int k = 0; k < (sigma_ ? 9 : 5); ++k) {
				if (k == 3) continue;  // the last sweep writes k[ALPHAS] itself
				stage(BS_AUX, sel, k <= 4 ? lanes : cells,
				      [&](int grid, const int *off) { kb_aux<M><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt, k); });
			}
		}
		stage(BS_ESTIMATE, sel, lanes,
		      [&](int grid, const int *off) { kb_estimate<M><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt); });
		if (any_tight) {
			// split requests back; a tree whose pool cannot take them grows (Solver::substep)
			sync();
			bool grown = false;
			for (int k = 0; k < nt; ++k) {
				Solver<M> *s = s_[sel[k]];
				s->check_status();
				if (!tight[k]) continue;
				const long long need = (long long) s->h_cnt_->top + (long long) NC * s->h_cnt_->n_split + 16;
				if (need > s->P_.cap) {
					const long long want = std::max(need + need / 4, (long long) s->P_.cap * 5 / 4);
					s->grow_pool((int) std::min<long long>(want, 2000000000LL));
					h_args_[k].P    = s->P_;
					h_args_[k].Ls   = s->Ls_;
					h_args_[k].list = s->Ls_.clu[L];
					grown           = true;
				}
			}
			if (grown) upload_args(sel);
		}
		auto regrid = [&](int kind, const std::vector<long long> &items, int k) {
			stage(kind, sel, items, [&](int grid, const int *off) { kb_regrid<M><<<grid, BLOCK, 0, st_>>>(d_args_, off, nt, k); });
		};
		regrid(BS_REGRID_CELL, cells, 0);   // unsplit selection
		regrid(BS_REGRID_FRESH, fresh, 1);  // split
		regrid(BS_REGRID_CELL, cells, 2);   // unsplit
		regrid(BS_REGRID_FRESH, fresh, 3);  // neighbour repair, first pass
		regrid(BS_NBR_LIST, repair, 4);     // neighbour repair, second pass
		regrid(BS_REGRID_CELL, cells, 5);   // reassignment of the cluster
		regrid(BS_REGRID_FRESH, fresh, 6);  // reassignment of new cells
		for (int k = 0; k < nt; ++k) std::swap(s_[sel[k]]->Ls_.clu[L], s_[sel[k]]->Ls_.tmp);
		kb_set_count<<<(nt + 127) / 128, 128, 0, st_>>>(d_args_, nt);
		DG_CUDA(cudaGetLastError());
	}

	// flush_acti_buffer(L) for the trees of `sel` whose buffer L holds cells (counts from the last
	// synchronisation; a substep of level L only fills buffer L - 1).
	void flush(int L, const std::vector<int> &sel) {
		std::vector<int> fl;
		std::vector<long long> items;
		for (int t: sel)
			if (s_[t]->h_cnt_->buf[L] > 0) {
				fl.push_back(t);
				items.push_back(s_[t]->h_cnt_->buf[L]);
			}
		if (fl.empty()) return;
		// the flush stage gets its own argument rows; the substep's upload of the rows must have run first
		DG_CUDA(cudaStreamSynchronize(st_));
		TreeArgs *h = h_args_;
		for (size_t k = 0; k < fl.size(); ++k) {
			Solver<M> *s = s_[fl[k]];
			h[k].P       = s->P_;
			h[k].Ls      = s->Ls_;
			h[k].cnt     = s->d_cnt_;
			h[k].L       = L;
		}
		upload_args(fl);
		stage(BS_FLUSH, fl, items,
		      [&](int grid, const int *off) { kb_flush<<<grid, BLOCK, 0, st_>>>(d_args_, off, (int) fl.size()); });
		kb_flush_done<<<((int) fl.size() + 127) / 128, 128, 0, st_>>>(d_args_, (int) fl.size());
		DG_CUDA(cudaGetLastError());
	}

public:
	// Integrator::integrate of every tree (impl/integrate.hpp:12-87), merged.
	void step(int signal, int *force_break, double *global_dt) override {
		const int N = (int) s_.size();
		for (int t = 0; t < N; ++t) {
			Solver<M> *s = s_[t];
			s->C_.signal  = signal;
			s->C_.coarsen = (s->n_global_ % s->coarsen_every_) == 0;
			force_break[t] = 0;
			DG_CUDA(cudaMemcpyAsync(d_consts_ + t, &s->C_, sizeof(Consts), cudaMemcpyHostToDevice, st_));
		}
		std::vector<char> halted(N, 0);
		const int top_seq = 1 << (MAX_ACTI - 1);
		int seq           = 0;
		while (true) {
			int finest = 0;
			for (int t = 0; t < N; ++t) {
				if (halted[t]) continue;
				Solver<M> *s = s_[t];
				int f        = s->max_acti_;
				for (int l = MAX_ACTI - 1; l > f; --l)
					if (s->h_cnt_->clu[l] > 0) {
						f = l;
						break;
					}
				finest = std::max(finest, f);
			}
			const int stride = 1 << (MAX_ACTI - 1 - finest);
			seq              = (seq / stride + 1) * stride;
			if (seq > top_seq) break;
			for (int l = 0; l < MAX_ACTI; ++l) {
				if (seq % (1 << l) != 0) continue;
				const int L = MAX_ACTI - l - 1;
				std::vector<int> sel;
				for (int t = 0; t < N; ++t) {
					if (halted[t]) continue;
					Solver<M> *s = s_[t];
					if (s->h_cnt_->clu[L] > 0 && L > s->max_acti_) {
						s->max_acti_     = L;
						s->acti_time_[L] = s->acti_time_[L - 1];
					}
					if (L > s->max_acti_) continue;
					sel.push_back(t);
				}
				if (sel.empty()) continue;
				substep(L, sel);
				for (int t: sel) {
					Solver<M> *s        = s_[t];
					s->acti_counter_[L] = (s->acti_counter_[L] + 1) % 2;
					s->acti_time_[L] += s->global_dt_ / (double) (1 << L);
				}
				flush(L, sel);
				sync();
				for (int t: sel) {
					Solver<M> *s = s_[t];
					s->check_status();
					s->n_split_total_ += s->h_cnt_->n_split;
					s->n_unsplit_total_ += s->h_cnt_->n_unsplit;
					s->n_substeps_++;
					s->updates_ += s->h_cnt_->clu[L];
					if (s->h_cnt_->status & ST_NAN) {
						force_break[t] = 1;
						global_dt[t]   = s->global_dt_;
						halted[t]      = 1;
					}
				}
			}
		}
		for (int t = 0; t < N; ++t) {
			if (halted[t]) continue;
			Solver<M> *s = s_[t];
			s->n_global_++;
			if (s->gc_due()) s->gc();
			if (s->resort_) s->resort();
			global_dt[t] = s->global_dt_;
		}
	}
};

template<class M>
BatchBase *make_batch_for(const std::vector<SolverBase *> &solvers) {
	return new Batch<M>(solvers);
}

}  // namespace dg
