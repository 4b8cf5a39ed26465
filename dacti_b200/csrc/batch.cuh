// Batched trees: many independent solvers of one model advanced in lockstep by one host thread, with
// one launch per stage for all trees that run a level and no host synchronisation inside a global step.
//
// Every tree keeps its own node pool, lists, counters and ACTI schedule state, so each tree computes
// exactly what it computes alone (impl/integrate.hpp:26-87 per tree). The trees' schedules are merged:
// the global-step sequence counter advances with the stride of the finest level of any tree, and at
// each sequence value a level substep runs for the trees whose schedule contains it. A tree whose
// finest level is coarser simply has no substep at sequence values that only finer levels use, which
// is the stride skip of its own schedule.
//
// The host plans the global step ahead: the schedule depends on the cluster counts only through "is a
// level above the tree's finest level populated", and the cell counts only size the launches, so a run
// of substeps is planned on the counts as it starts and every substep's arguments and block offsets go
// to the device in one copy. Then all launches of the run are issued with no synchronisation. A run
// takes the rest of the step, up to a window that doubles after every run that nothing stopped (so a
// warmed-up batch plans each global step as one run) and halves after a stop.
//
// Each substep opens with a one-block guard. A tree whose last substep left a NaN halts there for the
// rest of the step, as Integrator::integrate returns on force_break; its blocks return in every later
// substep, and the other trees, which are independent, run on unchanged. Then the guard checks, on the
// live counts, what the plan assumed: no error status, no populated level above a tree's planned finest
// level, every running cluster within its tree's scratch rows. After the indicator a second guard checks
// that every tree's pool takes its split requests. A failed guard stops the run there: that substep's
// kernels and all later ones find their substep closed and return. The host then sees where the run
// stopped, replays its own bookkeeping over the substeps that ran (and, for a halted tree, over its own
// substeps before the halt), completes a half-run substep itself (growing the pool, as Solver::substep
// does), and plans again from there. The stage kernels run over a block range per tree (the blocks of a
// launch are split among the trees in proportion to their planned work); the stage bodies read the live
// cluster length, so an approximate split costs balance, never results.
#pragma once

#include <algorithm>

#include "solver.cuh"

namespace dg {

// Per-tree arguments of the batched stage kernels: fixed while a planned run executes, except the list
// pointers of the running level, which kb_swap exchanges on the device as Solver::substep does on the host.
struct TreeArgs {
	Pool P;
	const Consts *C;  // device copy of the tree's constants
	BcTable B;
	Lists Ls;
	Counters *cnt;
	long long scratch;  // rows of the tree's per-substep scratch (Pool::ff, Pool::du)
	int limiter;
	int halted;  // the tree runs no further substep in this global step (set by kb_begin on a NaN)
	int finest;  // planned finest ACTI level: a populated level above it stops the run
};

// Per-tree arguments of one merged substep.
struct SubArgs {
	int tree;  // index into the TreeArgs array
	int L;
	int n;  // cluster length as the substep starts (written by kb_begin)
	int counterL;
	int stamp;
	int epoch0;  // the tree's epoch counter before the substep (kernels use epoch0 + k)
	double dtL;
};

constexpr int STALL_NONE = 0x7f7f7f7f;  // a run that nothing stopped (memset pattern 0x7f)

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

// `on` is the substep's head or tail flag (kb_begin, kb_split_check); a halted tree's blocks return.
#define DG_BATCH_PROLOGUE                                     \
	if (!*on || (int) blockIdx.x >= off[nt]) return;          \
	const int t_      = tree_of_block(off, nt);               \
	const SubArgs &s  = SA[t_];                               \
	const TreeArgs &a = A[s.tree];                            \
	if (a.halted) return;                                     \
	const BlockRange g{off[t_], off[t_ + 1] - off[t_]};

#define DG_BATCH_PARAMS const TreeArgs *A, const SubArgs *SA, const int *off, int nt, const int *on

// Opens merged substep `idx`. A tree whose last substep left a NaN (and nothing else) halts here, as
// Integrator::integrate returns on force_break: its blocks return in every later substep of the run and
// halt_at[t] = idx records where. The trees are independent, so the others' substeps are unchanged. Then,
// in a planned run, the plan's assumptions are checked on the live counts of every running tree; if one
// fails, or an earlier substep stopped the run, the substep stays closed (both flags 0) and the first
// stop is recorded as 2 * idx. Otherwise each listed running tree's counters n_recv .. status go to
// zero, its cluster length goes into its arguments, and both flags open.
static __global__ void __launch_bounds__(256) kb_begin(TreeArgs *A, int n_trees, SubArgs *SA, int nt, int *flags,
                                                      int *stall, int *halt_at, int idx) {
	const int stopped = *stall != STALL_NONE;
	if (!stopped)
		for (int t = threadIdx.x; t < n_trees; t += blockDim.x)
			if (!A[t].halted && A[t].cnt->status == ST_NAN) {
				A[t].halted = 1;
				halt_at[t]  = idx;
			}
	int bad = 0;
	__syncthreads();
	if (!stopped) {
		for (int t = threadIdx.x; t < n_trees; t += blockDim.x) {
			const TreeArgs &a = A[t];
			if (a.halted) continue;
			const Counters *c = a.cnt;
			bad |= c->status != 0;
			for (int l = a.finest + 1; l < MAX_ACTI; ++l) bad |= c->clu[l] > 0;
		}
		for (int k = threadIdx.x; k < nt; k += blockDim.x) {
			const TreeArgs &a = A[SA[k].tree];
			bad |= !a.halted && (long long) a.cnt->clu[SA[k].L] > a.scratch;
		}
	}
	if (__syncthreads_or(bad) || stopped) {
		if (threadIdx.x == 0) {
			if (!stopped) *stall = 2 * idx;
			flags[0] = flags[1] = 0;
		}
		return;
	}
	for (int k = threadIdx.x; k < nt; k += blockDim.x) {
		SubArgs &s = SA[k];
		if (A[s.tree].halted) continue;
		Counters *c = A[s.tree].cnt;
		s.n         = c->clu[s.L];
		c->n_recv = c->n_split = c->n_unsplit = c->n_new = c->n_upd = c->n_tmp = 0;
		c->status                                                        = 0;
	}
	if (threadIdx.x == 0) flags[0] = flags[1] = 1;
}

// After the indicator: a tree whose pool cannot take a split of every requested cell stops the run
// before the split (recorded as 2 * idx + 1, tail flag closed); the host grows that pool and runs the
// rest of the substep (Solver::substep's capacity check).
template<int NC>
static __global__ void __launch_bounds__(256) kb_split_check(const TreeArgs *A, const SubArgs *SA, int nt, int *flags,
                                                            int *stall, int idx) {
	int bad = 0;
	if (flags[1])
		for (int k = threadIdx.x; k < nt; k += blockDim.x) {
			const TreeArgs &a = A[SA[k].tree];
			bad |= !a.halted && (long long) a.cnt->top + (long long) NC * a.cnt->n_split + 16 > a.P.cap;
		}
	if (__syncthreads_or(bad) && threadIdx.x == 0) {
		*stall   = 2 * idx + 1;
		flags[1] = 0;
	}
}

template<class M, bool V, class R>
__global__ void __launch_bounds__(BLOCK, 2) kb_face_sum(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_face_sum<M, V, R>(g, a.P, *a.C, a.B, a.Ls.clu[s.L], s.n, s.L, s.dtL, s.stamp, a.Ls.recv, a.cnt);
}

template<class M, class R>
__global__ void __launch_bounds__(BLOCK) kb_flux_receive(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_flux_receive<M, R>(g, a.P, a.Ls.recv, &a.cnt->n_recv, s.L, a.cnt);
}

template<class M, bool V>
__global__ void __launch_bounds__(BLOCK, 3) kb_update(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_update<M, V>(g, a.P, *a.C, a.Ls.clu[s.L], s.n, s.dtL, s.epoch0 + 1, a.cnt);
}

template<class M, bool V>
__global__ void __launch_bounds__(BLOCK) kb_slope(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_slope<M, V>(g, a.P, *a.C, a.B, a.Ls.clu[s.L], s.n, a.limiter, s.epoch0 + 2, a.cnt);
}

// Multiphase auxiliary stages; `k` selects the stage in the order of Solver::multiphase_aux.
template<class M>
__global__ void __launch_bounds__(BLOCK) kb_aux(DG_BATCH_PARAMS, int k) {
	DG_BATCH_PROLOGUE
	const int e_upd      = s.epoch0 + 1;
	const int32_t *list = a.Ls.clu[s.L];
	switch (k) {
		case 0: d_smooth_alpha<M>(g, a.P, *a.C, a.B, list, s.n, nullptr, a.P.tmp, s.L, s.epoch0 + 3, e_upd, a.cnt); break;
		case 1: d_smooth_alpha<M>(g, a.P, *a.C, a.B, list, s.n, a.P.tmp, a.P.tmp2, s.L, s.epoch0 + 4, e_upd, a.cnt); break;
		case 2:
			d_smooth_alpha<M>(g, a.P, *a.C, a.B, list, s.n, a.P.tmp2, a.P.k + (size_t) M::ALPHAS * a.P.cap, s.L, s.epoch0 + 5,
			                  e_upd, a.cnt);
			break;
		case 4: d_normal<M>(g, a.P, *a.C, a.B, list, s.n, s.epoch0 + 6, e_upd, a.cnt); break;
		case 5: d_curvature<M>(g, a.P, *a.C, a.B, list, s.n, a.cnt); break;
		case 6: d_smooth_kappa<M>(g, a.P, *a.C, a.B, list, s.n, a.cnt); break;
		case 7: d_store_tmp(g, a.P, list, s.n, M::KAPPA, a.P.tmp); break;
		default: d_rec_k<M>(g, a.P, list, s.n); break;
	}
}

// Epochs of one substep in the tree's own sequence (Solver::substep): update + 1, slope + 2, the four
// multiphase sweeps + 3 .. + 6, then the estimate, the split and the unsplit.
template<class M>
constexpr int EPOCH_EST = M::MULTI ? 7 : 3;

template<class M>
__global__ void __launch_bounds__(BLOCK) kb_estimate(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_estimate<M>(g, a.P, *a.C, a.Ls.clu[s.L], s.n, s.L, s.counterL, s.epoch0 + EPOCH_EST<M>, a.Ls.split, a.cnt);
}

// Regrid and reassignment stages in the order of Solver::substep; `k` selects the stage.
template<class M>
__global__ void kb_regrid(DG_BATCH_PARAMS, int k) {
	DG_BATCH_PROLOGUE
	constexpr int EX = EPOCH_EST<M>;
	const int L      = s.L;
	switch (k) {
		case 0: d_unsplit_select<M>(g, a.P, a.Ls.clu[L], s.n, L, a.Ls.unsplit, a.cnt); break;
		case 1: d_split<M>(g, a.P, *a.C, &a.cnt->n_split, a.Ls.split, L, a.Ls.fresh, s.epoch0 + EX + 1, a.cnt); break;
		case 2: d_unsplit<M>(g, a.P, *a.C, &a.cnt->n_unsplit, a.Ls.unsplit, L, a.Ls.fresh, s.epoch0 + EX + 2, a.cnt); break;
		case 3: d_nbr_fresh<M>(g, a.P, *a.C, &a.cnt->n_new, a.Ls.fresh, a.Ls.upd, a.cnt); break;
		case 4: d_nbr_list<M>(g, a.P, *a.C, &a.cnt->n_upd, a.Ls.upd, a.cnt); break;
		case 5: d_reassign<M>(g, a.P, *a.C, a.Ls.clu[L], nullptr, s.n, L, s.dtL, s.counterL, a.Ls, a.cnt); break;
		default: d_reassign<M>(g, a.P, *a.C, a.Ls.fresh, &a.cnt->n_new, 0, L, s.dtL, s.counterL, a.Ls, a.cnt); break;
	}
}

// The rebuilt cluster list becomes the level's list and its count the cluster count (Solver::substep's
// swap of Lists::clu[L] and Lists::tmp).
static __global__ void kb_swap(TreeArgs *A, const SubArgs *SA, int nt, const int *on) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nt || !*on) return;
	TreeArgs &a   = A[SA[k].tree];
	const int L   = SA[k].L;
	if (a.halted) return;
	int32_t *x    = a.Ls.clu[L];
	a.Ls.clu[L]   = a.Ls.tmp;
	a.Ls.tmp      = x;
	a.cnt->clu[L] = a.cnt->n_tmp;
}

// flush_acti_buffer of level L for the listed trees (impl/acti_utils.hpp:365-372).
static __global__ void kb_flush(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_flush(g, a.P, a.Ls.buf[s.L], &a.cnt->buf[s.L], a.Ls.clu[s.L], &a.cnt->clu[s.L], s.L, a.cnt);
}

// Closes a substep: buffer L to zero, then the running totals (splits, coarsenings, the cluster's
// cells after the flush, substeps).
static __global__ void kb_done(const TreeArgs *A, const SubArgs *SA, int nt, const int *on) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nt || !*on || A[SA[k].tree].halted) return;
	Counters *c = A[SA[k].tree].cnt;
	const int L = SA[k].L;
	c->buf[L]   = 0;
	c->n_split_total += (unsigned long long) c->n_split;
	c->n_unsplit_total += (unsigned long long) c->n_unsplit;
	c->n_updates_total += (unsigned long long) c->clu[L];
	c->n_substeps_total += 1ull;
}

// Status of every tree to zero as a global step starts (a tree's status holds its last substep's).
static __global__ void kb_clear_status(const TreeArgs *A, int n_trees) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < n_trees) A[t].cnt->status = 0;
}

#undef DG_BATCH_PROLOGUE
#undef DG_BATCH_PARAMS

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
	virtual void run_stats(long long *out, int n) = 0;
	std::string last_error;
};

template<class M>
class Batch : public BatchBase {
	static constexpr int D = M::D, NC = 1 << D, NF = 2 * D;
	static constexpr int EPOCHS = EPOCH_EST<M> + 2;  // epoch numbers one substep uses per tree
	static constexpr int LANES  = NF <= 4 ? 4 : 8;    // lanes per cell of the lane-group stages

	// Block-offset tables of a substep: the stage kind whose budget sizes the launch, and the work items
	// per cluster cell it is split by (lanes, cells, new cells, repair tasks, buffer cells).
	enum Table : int { T_FACE, T_RECV, T_UPD, T_SLOPE, T_AUX_L, T_AUX_C, T_EST, T_RG_CELL, T_RG_FRESH, T_NBR, T_FLUSH, TABLES };
	static constexpr int TABLE_STAGE[TABLES] = {BS_FACE_SUM, BS_RECEIVE, BS_UPDATE, BS_SLOPE, BS_AUX, BS_AUX,
	                                            BS_ESTIMATE, BS_REGRID_CELL, BS_REGRID_FRESH, BS_NBR_LIST, BS_FLUSH};
	static constexpr long long TABLE_ITEMS[TABLES] = {LANES, LANES, 1, LANES, LANES, 1, LANES, 1, NC + 1, (NC + 1) * NF, 0};

	// The schedule's position: sequence value and the next level index to look at in it (MAX_ACTI: the
	// next sequence value is due).
	struct Cursor {
		int seq = 0;
		int l   = MAX_ACTI;
	};
	// A tree's host-side schedule state, saved before a planned run and restored when it stops early.
	struct TreeState {
		int max_acti, stamp, epoch;
		int acti_counter[MAX_ACTI];
		double acti_time[MAX_ACTI];
		Lists Ls;
	};
	// One planned merged substep: its level, its trees, their arguments and its slot in the arena.
	struct Planned {
		int L;
		std::vector<int> sel;
		std::vector<SubArgs> args;
		size_t at;
		int grid[TABLES];
		long long items[TABLES];
	};

	std::vector<Solver<M> *> s_;
	cudaStream_t st_  = nullptr;
	Counters *d_cnt_  = nullptr;  // all trees' counters
	Counters *h_cnt_  = nullptr;  // pinned
	std::vector<Counters *> own_d_, own_h_;
	Consts *d_consts_ = nullptr;  // all trees' constants
	TreeArgs *d_trees_ = nullptr, *h_trees_ = nullptr;
	char *d_arena_ = nullptr, *h_arena_ = nullptr;  // substep slots: flags, SubArgs, offset tables
	size_t arena_cap_ = 0;
	int *d_stall_ = nullptr, *h_stall_ = nullptr, *h_one_ = nullptr;
	int *d_halt_ = nullptr, *h_halt_ = nullptr;  // per tree: the planned substep whose kb_begin halted it
	static constexpr int WINDOW_MIN = 64, WINDOW_MAX = 1 << 16;
	int window_ = 512;  // substeps one planned run takes at most: doubles after a run that nothing stopped,
	                    // halves after a stop
	int device_ = 0;
	int sms_    = 148;
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
	struct Base {
		long long split, unsplit, updates, substeps;
	};
	std::vector<Base> base_;  // the solvers' statistics when they joined the batch
	long long runs_ = 0, stops_ = 0, planned_ = 0, replayed_ = 0;

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
		DG_CUDA(cudaMalloc(&d_trees_, sizeof(TreeArgs) * nt));
		DG_CUDA(cudaMallocHost(&h_trees_, sizeof(TreeArgs) * nt));
		DG_CUDA(cudaMalloc(&d_stall_, sizeof(int)));
		DG_CUDA(cudaMallocHost(&h_stall_, sizeof(int)));
		DG_CUDA(cudaMallocHost(&h_one_, sizeof(int)));
		DG_CUDA(cudaMalloc(&d_halt_, sizeof(int) * nt));
		DG_CUDA(cudaMallocHost(&h_halt_, sizeof(int) * nt));
		*h_one_ = 1;
		// every solver moves onto the batch's stream and its counters into the batch's array
		for (int t = 0; t < nt; ++t) {
			Solver<M> *s = s_[t];
			DG_CUDA(cudaStreamSynchronize(s->st_));
			s->st_ = st_;
			Counters c = *s->h_cnt_;
			c.n_split_total = c.n_unsplit_total = c.n_updates_total = c.n_substeps_total = 0;
			DG_CUDA(cudaMemcpy(d_cnt_ + t, s->d_cnt_, sizeof(Counters), cudaMemcpyDeviceToDevice));
			DG_CUDA(cudaMemcpy(&d_cnt_[t].n_split_total, &c.n_split_total, 4 * sizeof(unsigned long long),
			                   cudaMemcpyHostToDevice));
			h_cnt_[t] = c;
			own_d_.push_back(s->d_cnt_);
			own_h_.push_back(s->h_cnt_);
			s->d_cnt_ = d_cnt_ + t;
			s->h_cnt_ = h_cnt_ + t;
			base_.push_back({s->n_split_total_, s->n_unsplit_total_, s->updates_, s->n_substeps_});
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
		cudaFree(d_trees_);
		cudaFreeHost(h_trees_);
		cudaFree(d_arena_);
		cudaFreeHost(h_arena_);
		cudaFree(d_stall_);
		cudaFreeHost(h_stall_);
		cudaFreeHost(h_one_);
		cudaFree(d_halt_);
		cudaFreeHost(h_halt_);
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

	// Planned runs, runs stopped by a guard, substeps planned and substeps replayed on the host after a
	// stop, since the batch was made.
	void run_stats(long long *out, int n) override {
		const long long v[4] = {runs_, stops_, planned_, replayed_};
		for (int k = 0; k < n && k < 4; ++k) out[k] = v[k];
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
		DG_CUDA(cudaMemcpyAsync(h_stall_, d_stall_, sizeof(int), cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaMemcpyAsync(h_halt_, d_halt_, sizeof(int) * s_.size(), cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		if (prof_) drain();
	}

	// ---- the schedule --------------------------------------------------------------------------

	// The next merged substep (impl/integrate.hpp:26-67 per tree, merged): its level L and the trees
	// that run it, decided on the cluster counts `cnt`; a tree whose level above its finest level is
	// populated takes that level on (max_acti_level and its time, as the reference does).
	bool next(Cursor &c, const std::vector<char> &halted, const Counters *cnt, int &L, std::vector<int> &sel) {
		const int N       = (int) s_.size();
		const int top_seq = 1 << (MAX_ACTI - 1);
		while (true) {
			if (c.l >= MAX_ACTI) {
				int finest = 0;
				for (int t = 0; t < N; ++t) {
					if (halted[t]) continue;
					int f = s_[t]->max_acti_;
					for (int l = MAX_ACTI - 1; l > f; --l)
						if (cnt[t].clu[l] > 0) {
							f = l;
							break;
						}
					finest = std::max(finest, f);
				}
				const int stride = 1 << (MAX_ACTI - 1 - finest);
				c.seq            = (c.seq / stride + 1) * stride;
				if (c.seq > top_seq) return false;
				c.l = 0;
			}
			for (; c.l < MAX_ACTI; ++c.l) {
				if (c.seq % (1 << c.l) != 0) continue;
				L = MAX_ACTI - c.l - 1;
				sel.clear();
				for (int t = 0; t < N; ++t) {
					if (halted[t]) continue;
					Solver<M> *s = s_[t];
					if (cnt[t].clu[L] > 0 && L > s->max_acti_) {
						s->max_acti_     = L;
						s->acti_time_[L] = s->acti_time_[L - 1];
					}
					if (L > s->max_acti_) continue;
					sel.push_back(t);
				}
				if (sel.empty()) continue;
				++c.l;
				return true;
			}
		}
	}

	// The substep's per-tree arguments; advances each tree's stamp and epoch counters.
	void make_args(int L, const std::vector<int> &sel, std::vector<SubArgs> &out) {
		out.resize(sel.size());
		for (size_t k = 0; k < sel.size(); ++k) {
			Solver<M> *s = s_[sel[k]];
			SubArgs &a   = out[k];
			a.tree       = sel[k];
			a.L          = L;
			a.n          = 0;
			a.counterL   = s->acti_counter_[L];
			a.stamp      = ++s->stamp_;
			a.epoch0     = s->epoch_;
			a.dtL        = s->global_dt_ / (double) (1 << L);
			s->epoch_ += EPOCHS;
		}
	}

	// The host's part of a finished substep: ACTI counter and time of level L, the list swap.
	void advance(int L, const std::vector<int> &sel) {
		for (int t: sel) {
			Solver<M> *s        = s_[t];
			s->acti_counter_[L] = (s->acti_counter_[L] + 1) % 2;
			s->acti_time_[L] += s->global_dt_ / (double) (1 << L);
			std::swap(s->Ls_.clu[L], s->Ls_.tmp);
		}
	}

	TreeState save(const Solver<M> *s) const {
		TreeState z;
		z.max_acti = s->max_acti_;
		z.stamp    = s->stamp_;
		z.epoch    = s->epoch_;
		std::copy(s->acti_counter_, s->acti_counter_ + MAX_ACTI, z.acti_counter);
		std::copy(s->acti_time_, s->acti_time_ + MAX_ACTI, z.acti_time);
		z.Ls = s->Ls_;
		return z;
	}
	void restore(Solver<M> *s, const TreeState &z) const {
		s->max_acti_ = z.max_acti;
		s->stamp_    = z.stamp;
		s->epoch_    = z.epoch;
		std::copy(z.acti_counter, z.acti_counter + MAX_ACTI, s->acti_counter_);
		std::copy(z.acti_time, z.acti_time + MAX_ACTI, s->acti_time_);
		s->Ls_ = z.Ls;
	}

	// After substeps with these trees ran: a capacity or structure error throws, a NaN halts the tree
	// for the rest of the global step (force_break).
	void post_checks(const std::vector<int> &sel, std::vector<char> &halted, int *force_break, double *global_dt) {
		for (int t: sel) {
			if (halted[t]) continue;
			Solver<M> *s = s_[t];
			s->check_status();
			if (s->h_cnt_->status & ST_NAN) {
				force_break[t] = 1;
				global_dt[t]   = s->global_dt_;
				halted[t]      = 1;
			}
		}
	}

	// ---- device side of a planned run ----------------------------------------------------------

	// Scratch rows for the clusters as they are now (and half as much again), then every tree's arguments.
	void prepare(const std::vector<char> &halted) {
		const int N = (int) s_.size();
		for (int t = 0; t < N; ++t) {
			Solver<M> *s   = s_[t];
			const Counters &c = h_cnt_[t];
			long long most = 0;
			int finest     = s->max_acti_;
			for (int l = 0; l < MAX_ACTI; ++l) {
				most = std::max<long long>(most, c.clu[l]);
				if (c.clu[l] > 0) finest = std::max(finest, l);
			}
			if (!halted[t]) s->ensure_scratch(most + most / 2);
			TreeArgs &a = h_trees_[t];
			a.P         = s->P_;
			a.C         = d_consts_ + t;
			a.B         = s->B_;
			a.Ls        = s->Ls_;
			a.cnt       = s->d_cnt_;
			a.scratch   = s->scratch_cap_;
			a.limiter   = s->limiter_;
			a.halted    = halted[t];
			a.finest    = finest;
		}
		upload_trees();
	}

	void upload_trees() {
		DG_CUDA(cudaMemcpyAsync(d_trees_, h_trees_, sizeof(TreeArgs) * s_.size(), cudaMemcpyHostToDevice, st_));
	}

	static size_t slot_bytes(int nt) {
		return Solver<M>::align_up(16 + sizeof(SubArgs) * (size_t) nt + sizeof(int) * (size_t) TABLES * (nt + 1));
	}

	void ensure_arena(size_t bytes) {
		if (bytes <= arena_cap_) return;
		DG_CUDA(cudaStreamSynchronize(st_));
		cudaFree(d_arena_);
		cudaFreeHost(h_arena_);
		d_arena_   = nullptr;
		h_arena_   = nullptr;
		arena_cap_ = 0;
		const size_t want = std::max(bytes, arena_cap_ + arena_cap_ / 2);
		DG_CUDA(cudaMalloc(&d_arena_, want));
		DG_CUDA(cudaMallocHost(&h_arena_, want));
		arena_cap_ = want;
	}

	// Block offsets of one table: tree k gets blocks in proportion to its planned items (at least one),
	// the launch at most `cap` blocks in total unless every tree needs its one. Returns the block count.
	static int fill_offsets(int *h, const std::vector<long long> &items, int cap) {
		const int nt   = (int) items.size();
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
		return h[nt];
	}

	// The slot of a planned substep in the host arena: closed flags, arguments, offset tables sized on
	// the planning counts `cnt`.
	void write_slot(Planned &p, const Counters *cnt) {
		const int nt = (int) p.sel.size();
		char *slot   = h_arena_ + p.at;
		std::memset(slot, 0, 16);
		std::memcpy(slot + 16, p.args.data(), sizeof(SubArgs) * nt);
		int *off = (int *) (slot + 16 + sizeof(SubArgs) * nt);
		std::vector<long long> items(nt);
		for (int tb = 0; tb < TABLES; ++tb) {
			long long tot = 0;
			for (int k = 0; k < nt; ++k) {
				const Counters &c = cnt[p.sel[k]];
				const long long n = c.clu[p.L];
				// the flush moves the cells that level L + 1 handed down; plan for half its cluster
				items[k] = tb == T_FLUSH ? (p.L + 1 < MAX_ACTI ? c.clu[p.L + 1] / 2 : 0) : n * TABLE_ITEMS[tb];
				tot += items[k];
			}
			p.grid[tb]  = fill_offsets(off + (size_t) tb * (nt + 1), items, sms_ * bps_[TABLE_STAGE[tb]]);
			p.items[tb] = tot;
		}
	}

	// One launch of a table's stage, timed with events when profiling.
	template<class F>
	void stage(const Planned &p, int tb, const int *off, F &&launch) {
		cudaEvent_t a = nullptr, b = nullptr;
		if (prof_) {
			a = event();
			b = event();
			DG_CUDA(cudaEventRecord(a, st_));
		}
		launch(p.grid[tb], off + (size_t) tb * (p.sel.size() + 1));
		if (prof_) {
			DG_CUDA(cudaEventRecord(b, st_));
			timed_.push_back({TABLE_STAGE[tb], a, b, p.items[tb]});
		}
	}

	// The launches of planned substep `idx`: the head (guard, fluxes, update, slopes, multiphase
	// auxiliaries, indicator, capacity guard) and the tail (regrid, reassignment, list swap, flush, totals).
	void launch(const Planned &p, int idx, bool head, bool tail) {
		const int nt          = (int) p.sel.size();
		char *slot            = d_arena_ + p.at;
		int *flags            = (int *) slot;
		SubArgs *S            = (SubArgs *) (slot + 16);
		const int *off        = (const int *) (slot + 16 + sizeof(SubArgs) * nt);
		const TreeArgs *A     = d_trees_;
		const int *on         = flags;
		if (head) {
			kb_begin<<<1, 256, 0, st_>>>(d_trees_, (int) s_.size(), S, nt, flags, d_stall_, d_halt_, idx);
			stage(p, T_FACE, off, [&](int grid, const int *o) {
				if (mixed_) {
					if (visc_) kb_face_sum<M, true, float><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
					else kb_face_sum<M, false, float><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
				} else {
					if (visc_) kb_face_sum<M, true, double><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
					else kb_face_sum<M, false, double><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
				}
			});
			stage(p, T_RECV, off, [&](int grid, const int *o) {
				if (mixed_) kb_flux_receive<M, float><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
				else kb_flux_receive<M, double><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
			});
			stage(p, T_UPD, off, [&](int grid, const int *o) {
				if (visc_) kb_update<M, true><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
				else kb_update<M, false><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
			});
			stage(p, T_SLOPE, off, [&](int grid, const int *o) {
				if (visc_) kb_slope<M, true><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
				else kb_slope<M, false><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on);
			});
			if constexpr (M::MULTI) {
				// the smoothing sweeps and the normal run a lane group per cell, the curvature stages a thread
				for (int k = 0; k < (sigma_ ? 9 : 5); ++k) {
					if (k == 3) continue;  // the last sweep writes k[ALPHAS] itself
					stage(p, k <= 4 ? T_AUX_L : T_AUX_C, off,
					      [&](int grid, const int *o) { kb_aux<M><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on, k); });
				}
			}
			stage(p, T_EST, off, [&](int grid, const int *o) { kb_estimate<M><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, on); });
			kb_split_check<NC><<<1, 256, 0, st_>>>(A, S, nt, flags, d_stall_, idx);
		}
		if (tail) {
			const int *ont = flags + 1;
			auto regrid    = [&](int tb, int k) {
				stage(p, tb, off, [&](int grid, const int *o) { kb_regrid<M><<<grid, BLOCK, 0, st_>>>(A, S, o, nt, ont, k); });
			};
			regrid(T_RG_CELL, 0);   // unsplit selection
			regrid(T_RG_FRESH, 1);  // split
			regrid(T_RG_CELL, 2);   // unsplit
			regrid(T_RG_FRESH, 3);  // neighbour repair, first pass
			regrid(T_NBR, 4);       // neighbour repair, second pass
			regrid(T_RG_CELL, 5);   // reassignment of the cluster
			regrid(T_RG_FRESH, 6);  // reassignment of new cells
			kb_swap<<<(nt + 127) / 128, 128, 0, st_>>>(d_trees_, S, nt, ont);
			stage(p, T_FLUSH, off, [&](int grid, const int *o) { kb_flush<<<grid, BLOCK, 0, st_>>>(A, S, o, nt, ont); });
			kb_done<<<(nt + 127) / 128, 128, 0, st_>>>(A, S, nt, ont);
		}
		DG_CUDA(cudaGetLastError());
	}

	// Completes planned substep `idx`, whose run stopped at the capacity guard: the pools that cannot take
	// their split requests grow (Solver::substep), then the substep's tail runs.
	void finish_substep(const Planned &p, int idx, const std::vector<char> &dev_halted) {
		bool grown = false;
		for (int t: p.sel) {
			if (dev_halted[t]) continue;
			Solver<M> *s         = s_[t];
			const long long need = (long long) s->h_cnt_->top + (long long) NC * s->h_cnt_->n_split + 16;
			if (need > s->P_.cap) {
				const long long want = std::max(need + need / 4, (long long) s->P_.cap * 5 / 4);
				s->grow_pool((int) std::min<long long>(want, 2000000000LL));
				grown = true;
			}
		}
		if (grown) {
			// the host's lists mirror the device's after the replay: every tree's row is rewritten
			for (size_t t = 0; t < s_.size(); ++t) {
				TreeArgs &a = h_trees_[t];
				a.P         = s_[t]->P_;
				a.Ls        = s_[t]->Ls_;
				a.scratch   = s_[t]->scratch_cap_;
				a.halted    = a.halted || dev_halted[t];
			}
			upload_trees();
		}
		int *flags = (int *) (d_arena_ + p.at);
		DG_CUDA(cudaMemcpyAsync(flags + 1, h_one_, sizeof(int), cudaMemcpyHostToDevice, st_));
		launch(p, idx, false, true);
		sync();
	}

	// Tree t halted on the device at planned substep h (a NaN from its substep before h): its host state
	// goes back to the run's start `z` and forward over its own substeps of the plan before h.
	void replay_tree(int t, int h, const TreeState &z, const std::vector<Planned> &plan) {
		Solver<M> *s = s_[t];
		restore(s, z);
		const std::vector<int> one{t};
		std::vector<SubArgs> tmp;
		for (int j = 0; j < h && j < (int) plan.size(); ++j) {
			const Planned &p = plan[j];
			if (!std::binary_search(p.sel.begin(), p.sel.end(), t)) continue;
			if (p.L > s->max_acti_) {  // the level next() had the tree take on
				s->max_acti_       = p.L;
				s->acti_time_[p.L] = s->acti_time_[p.L - 1];
			}
			make_args(p.L, one, tmp);
			advance(p.L, one);
		}
	}

public:
	// Integrator::integrate of every tree (impl/integrate.hpp:12-87), merged.
	void step(int signal, int *force_break, double *global_dt) override {
		const int N = (int) s_.size();
		for (int t = 0; t < N; ++t) {
			Solver<M> *s  = s_[t];
			s->C_.signal  = signal;
			s->C_.coarsen = (s->n_global_ % s->coarsen_every_) == 0;
			force_break[t] = 0;
			DG_CUDA(cudaMemcpyAsync(d_consts_ + t, &s->C_, sizeof(Consts), cudaMemcpyHostToDevice, st_));
		}
		std::vector<char> halted(N, 0);
		auto halt = [&](int t) {
			force_break[t] = 1;
			global_dt[t]   = s_[t]->global_dt_;
			halted[t]      = 1;
		};
		// a status left from before the step belongs to no substep of it
		for (int t = 0; t < N; ++t) {
			s_[t]->check_status();
			h_cnt_[t].status = 0;
		}
		prepare(halted);
		kb_clear_status<<<(N + 127) / 128, 128, 0, st_>>>(d_trees_, N);
		Cursor cur;
		std::vector<Planned> plan;
		std::vector<TreeState> saved(N);
		std::vector<Counters> pred(N);
		std::vector<int> all(N);
		for (int t = 0; t < N; ++t) all[t] = t;
		bool first = true;
		while (true) {
			// plan up to window_ substeps of the rest of the step on the counts as they are now (the
			// stream is idle, h_cnt_ current)
			if (!first) prepare(halted);
			first              = false;
			const Cursor cur0  = cur;
			const auto halted0 = halted;
			for (int t = 0; t < N; ++t) saved[t] = save(s_[t]);
			std::copy(h_cnt_, h_cnt_ + N, pred.begin());
			plan.clear();
			size_t bytes  = 0;
			bool finished = false;
			int L;
			std::vector<int> sel;
			while ((int) plan.size() < window_) {
				if (!next(cur, halted, pred.data(), L, sel)) {
					finished = true;
					break;
				}
				Planned p;
				p.L   = L;
				p.sel = sel;
				p.at  = bytes;
				make_args(L, sel, p.args);
				advance(L, sel);
				bytes += slot_bytes((int) sel.size());
				plan.push_back(std::move(p));
			}
			if (plan.empty()) break;
			ensure_arena(bytes);
			for (auto &p: plan) write_slot(p, pred.data());
			DG_CUDA(cudaMemcpyAsync(d_arena_, h_arena_, bytes, cudaMemcpyHostToDevice, st_));
			DG_CUDA(cudaMemsetAsync(d_stall_, 0x7f, sizeof(int), st_));
			DG_CUDA(cudaMemsetAsync(d_halt_, 0x7f, sizeof(int) * N, st_));
			for (size_t i = 0; i < plan.size(); ++i) launch(plan[i], (int) i, true, true);
			sync();
			++runs_;
			planned_ += (long long) plan.size();
			// trees that a NaN halted on the device, with the substep where it was seen
			std::vector<std::pair<int, int>> halts;
			std::vector<char> dev_halted(N, 0);
			for (int t = 0; t < N; ++t)
				if (h_halt_[t] != STALL_NONE) {
					halts.push_back({t, h_halt_[t]});
					dev_halted[t] = 1;
				}
			const int stop = *h_stall_;
			if (stop == STALL_NONE) {
				for (auto &th: halts) {
					replay_tree(th.first, th.second, saved[th.first], plan);
					halt(th.first);
				}
				// a NaN in a tree's last substep of the run halts it now; an error throws
				post_checks(all, halted, force_break, global_dt);
				if (finished) break;
				window_ = std::min(window_ * 2, WINDOW_MAX);
				continue;
			}
			++stops_;
			window_     = std::max(window_ / 2, WINDOW_MIN);
			const int i = stop / 2, half = stop & 1;
			if (i == 0 && !half) throw dg_error(DG_ERR_UNSUPPORTED, "batch: a planned run stopped before its first substep");
			// back to the state before the run, then forward over the substeps that ran
			cur    = cur0;
			halted = halted0;
			for (int t = 0; t < N; ++t) restore(s_[t], saved[t]);
			std::vector<SubArgs> scratch_args;
			for (int j = 0; j < i; ++j) {
				const bool more = next(cur, halted, pred.data(), L, sel);
				if (!more || L != plan[j].L || sel != plan[j].sel)
					throw dg_error(DG_ERR_UNSUPPORTED, "batch: replay left the plan at substep " + std::to_string(j) + " of " +
					                                       std::to_string(i) + (half ? " (tail stop)" : " (head stop)"));
				make_args(L, sel, scratch_args);
				advance(L, sel);
				++replayed_;
			}
			if (!half) {
				// the statuses are still those of substep i - 1 (a NaN there has halted its tree already)
				if (i > 0) post_checks(plan[i - 1].sel, halted, force_break, global_dt);
			} else {
				// substep i's head ran: its statuses are substep i's, and kb_begin(i) found every running
				// tree's status clear before it
				const bool more = next(cur, halted, pred.data(), L, sel);
				if (!more || L != plan[i].L || sel != plan[i].sel)
					throw dg_error(DG_ERR_UNSUPPORTED, "batch: replay left the plan at the stopped substep " + std::to_string(i));
				make_args(L, sel, scratch_args);
				finish_substep(plan[i], i, dev_halted);
				advance(L, sel);
				++replayed_;
				post_checks(sel, halted, force_break, global_dt);
			}
			for (auto &th: halts) {
				replay_tree(th.first, th.second, saved[th.first], plan);
				halt(th.first);
			}
		}
		for (int t = 0; t < N; ++t) {
			Solver<M> *s       = s_[t];
			const Counters &c  = h_cnt_[t];
			s->n_split_total_   = base_[t].split + (long long) c.n_split_total;
			s->n_unsplit_total_ = base_[t].unsplit + (long long) c.n_unsplit_total;
			s->updates_         = base_[t].updates + (long long) c.n_updates_total;
			s->n_substeps_      = base_[t].substeps + (long long) c.n_substeps_total;
			if (halted[t]) continue;
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
