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
// The host plans the global step ahead, in runs of substeps issued with no synchronisation. The merged
// sequence of (sequence value, level) pairs depends only on the batch's finest populated level F: the
// stride of the sequence counter is F's. Which trees run a pair's substep, and with which stamps, epochs
// and ACTI counters, is decided on the device: each tree's schedule state (max_acti_level, ACTI
// counters and times, stamp and epoch counters) lives in device memory, and the substep's opening kernel
// applies the reference's rule to the live counts, a tree taking on a newly populated level up to its
// planned headroom as Integrator::integrate does. So the plan is the pairs of the rest of the step, each
// with the trees that may run it, and one copy takes every substep's arguments and block offsets to the
// device. A run takes the rest of the step, up to a window that doubles after every run nothing stopped
// (a warmed-up batch plans each global step as one run) and halves after a stop.
//
// Each substep opens with a one-block kernel (kb_begin). A tree whose last substep left a NaN halts
// there for the rest of the step, as Integrator::integrate returns on force_break; the other trees are
// independent and run on unchanged. Then the kernel checks what the plan assumed: no error status, no
// populated level above a tree's planned headroom (a level above F changes the sequence's stride), every
// running cluster within its tree's scratch rows. After the indicator a second kernel checks that every
// pool takes its split requests. A failed check stops the run there: that substep's kernels and all
// later ones find their substep closed and return. The host reads the trees' schedule state back,
// completes a half-run substep itself (growing the pool, as Solver::substep does), and plans again from
// there. The stage kernels run over a block range per tree (the blocks of a launch are split among the
// trees in proportion to their planned work); the stage bodies read the live cluster length, so an
// approximate split costs balance, never results.
#pragma once

#include <algorithm>

#include "solver.cuh"

namespace dg {

// A tree's schedule state in the merged step (Integrator: max_acti_level, acti_counter, acti_time, and
// this port's stamp and epoch counters), kept on the device while a run executes.
struct TreeSched {
	int max_acti, stamp, epoch, pad;
	int counter[MAX_ACTI];
	double time[MAX_ACTI];
};

// Per-tree arguments of the batched stage kernels: fixed while a run executes, except the list pointers
// of the running level, which kb_swap exchanges as Solver::substep does, and the halt flag.
struct TreeArgs {
	Pool P;
	const Consts *C;  // device copy of the tree's constants
	BcTable B;
	Lists Ls;
	Counters *cnt;
	TreeSched *sch;
	long long scratch;  // rows of the tree's per-substep scratch (Pool::ff, Pool::du)
	int limiter;
	int halted;  // the tree runs no further substep in this global step (set by kb_begin on a NaN)
	int finest;  // planned headroom: the tree may run levels up to here; a populated level above stops the run
	int epochs;  // epoch numbers one substep uses
};

// Per-tree arguments of one merged substep: tree, level and dtL from the plan, the rest from kb_begin.
struct SubArgs {
	int tree;  // index into the TreeArgs array
	int L;
	int n;  // cluster length as the substep starts
	int counterL;
	int stamp;
	int epoch0;  // the tree's epoch counter before the substep (kernels use epoch0 + k)
	int active;  // the tree runs this substep
	int pad;
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

// Every block of a batched launch works for one tree: its argument row (and, where the stage reads them,
// its constants) goes to shared memory once, so the stage body finds the pool's pointers and the
// constants there instead of reloading them from global memory after its stores.
__device__ __forceinline__ void stage_tree(const TreeArgs &src, TreeArgs &a, Consts *c) {
	const long long *sa = reinterpret_cast<const long long *>(&src);
	long long *da       = reinterpret_cast<long long *>(&a);
	for (int w = threadIdx.x; w < (int) (sizeof(TreeArgs) / 8); w += blockDim.x) da[w] = sa[w];
	if (c) {
		const long long *sc = reinterpret_cast<const long long *>(src.C);
		long long *dc       = reinterpret_cast<long long *>(c);
		for (int w = threadIdx.x; w < (int) (sizeof(Consts) / 8); w += blockDim.x) dc[w] = sc[w];
	}
	__syncthreads();
}
static_assert(sizeof(TreeArgs) % 8 == 0 && sizeof(Consts) % 8 == 0, "argument rows copy as 8-byte words");

// `on` is the substep's head or tail flag (kb_begin, kb_split_check); the blocks of a tree that does not
// run the substep return (the whole block: the tree is the block's).
#define DG_BATCH_HEAD                                         \
	if (!*on || (int) blockIdx.x >= off[nt]) return;          \
	const int t_     = tree_of_block(off, nt);                \
	const SubArgs &s = SA[t_];                                \
	if (!s.active) return;                                    \
	__shared__ TreeArgs a_sh_;                                \
	const TreeArgs &a = a_sh_;                                \
	const BlockRange g{off[t_], off[t_ + 1] - off[t_]};
#define DG_BATCH_PROLOGUE                                     \
	DG_BATCH_HEAD                                             \
	__shared__ Consts c_sh_;                                  \
	stage_tree(A[s.tree], a_sh_, &c_sh_);                     \
	const Consts &cst = c_sh_;
#define DG_BATCH_PROLOGUE_NC                                  \
	DG_BATCH_HEAD                                             \
	stage_tree(A[s.tree], a_sh_, nullptr);

#define DG_BATCH_PARAMS const TreeArgs *A, const SubArgs *SA, const int *off, int nt, const int *on

// Opens merged substep `idx`. A tree whose last substep left a NaN (and nothing else) halts here, as
// Integrator::integrate returns on force_break: it runs no later substep of the step, and halt_at[t] =
// idx records where. The trees are independent, so the others' substeps are unchanged. Then, in order:
// - the run's assumptions on the live counts of every running tree: no error status, no populated level
//   above the tree's headroom, the running clusters within the scratch rows. If one fails, or an earlier
//   substep stopped the run, the substep stays closed (both flags 0) and the first stop is recorded as
//   2 * idx;
// - for each listed tree, Integrator::integrate's rule for level L (impl/integrate.hpp:32-39): a populated
//   level above max_acti_level becomes the tree's finest (its time taken from the next coarser level),
//   and the tree runs the substep if L <= max_acti_level. A running tree's counters n_recv .. status go
//   to zero and its arguments get the cluster length, the ACTI counter and the next stamp and epochs.
static __global__ void __launch_bounds__(256) kb_begin(TreeArgs *A, int n_trees, SubArgs *SA, int nt, int *flags,
                                                      int *stall, int *halt_at, int idx) {
	const int stopped = *stall != STALL_NONE;
	if (!stopped)
		for (int t = threadIdx.x; t < n_trees; t += blockDim.x)
			if (!A[t].halted && A[t].cnt->status == ST_NAN) {
				A[t].halted = 1;
				halt_at[t]  = idx;
			}
	__syncthreads();
	int bad = 0;
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
			const int L       = SA[k].L;
			const int n       = a.cnt->clu[L];
			bad |= !a.halted && (L <= a.sch->max_acti || n > 0) && (long long) n > a.scratch;
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
		SubArgs &s        = SA[k];
		const TreeArgs &a = A[s.tree];
		int run           = 0;
		if (!a.halted) {
			TreeSched &z = *a.sch;
			Counters *c  = a.cnt;
			const int L  = s.L;
			if (c->clu[L] > 0 && L > z.max_acti) {
				z.max_acti = L;
				z.time[L]  = z.time[L - 1];
			}
			run = L <= z.max_acti;
			if (run) {
				s.n        = c->clu[L];
				s.counterL = z.counter[L];
				s.stamp    = ++z.stamp;
				s.epoch0   = z.epoch;
				z.epoch += a.epochs;
				c->n_recv = c->n_split = c->n_unsplit = c->n_new = c->n_upd = c->n_tmp = 0;
				c->status                                                        = 0;
			}
		}
		s.active = run;
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
			bad |= SA[k].active && (long long) a.cnt->top + (long long) NC * a.cnt->n_split + 16 > a.P.cap;
		}
	if (__syncthreads_or(bad) && threadIdx.x == 0) {
		*stall   = 2 * idx + 1;
		flags[1] = 0;
	}
}

template<class M, bool V, class R>
__global__ void __launch_bounds__(FACE_THREADS, FACE_MIN_BLOCKS) kb_face_sum(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_face_sum<M, V, R>(g, a.P, cst, a.B, a.Ls.clu[s.L], s.n, s.L, s.dtL, s.stamp, a.Ls.recv, a.cnt);
}

template<class M, class R>
__global__ void __launch_bounds__(BLOCK) kb_flux_receive(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE_NC
	d_flux_receive<M, R>(g, a.P, a.Ls.recv, &a.cnt->n_recv, s.L, a.cnt);
}

template<class M, bool V>
__global__ void __launch_bounds__(BLOCK, 3) kb_update(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_update<M, V>(g, a.P, cst, a.Ls.clu[s.L], s.n, s.dtL, s.epoch0 + 1, a.cnt);
}

template<class M, bool V>
__global__ void __launch_bounds__(SLOPE_THREADS, SLOPE_MIN_BLOCKS) kb_slope(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE
	d_slope<M, V>(g, a.P, cst, a.B, a.Ls.clu[s.L], s.n, a.limiter, s.epoch0 + 2, a.cnt);
}

// Multiphase auxiliary stages; `k` selects the stage in the order of Solver::multiphase_aux.
template<class M>
__global__ void __launch_bounds__(BLOCK) kb_aux(DG_BATCH_PARAMS, int k) {
	DG_BATCH_PROLOGUE
	const int e_upd      = s.epoch0 + 1;
	const int32_t *list = a.Ls.clu[s.L];
	switch (k) {
		case 0: d_smooth_alpha<M>(g, a.P, cst, a.B, list, s.n, nullptr, a.P.tmp, s.L, s.epoch0 + 3, e_upd, a.cnt); break;
		case 1: d_smooth_alpha<M>(g, a.P, cst, a.B, list, s.n, a.P.tmp, a.P.tmp2, s.L, s.epoch0 + 4, e_upd, a.cnt); break;
		case 2:
			d_smooth_alpha<M>(g, a.P, cst, a.B, list, s.n, a.P.tmp2, a.P.k + (size_t) M::ALPHAS * a.P.cap, s.L, s.epoch0 + 5,
			                  e_upd, a.cnt);
			break;
		case 4: d_normal<M>(g, a.P, cst, a.B, list, s.n, s.epoch0 + 6, e_upd, a.cnt); break;
		case 5: d_curvature<M>(g, a.P, cst, a.B, list, s.n, a.cnt); break;
		case 6: d_smooth_kappa<M>(g, a.P, cst, a.B, list, s.n, a.cnt); break;
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
	d_estimate<M>(g, a.P, cst, a.Ls.clu[s.L], s.n, s.L, s.counterL, s.epoch0 + EPOCH_EST<M>, a.Ls.split, a.cnt);
}

// Regrid and reassignment stages in the order of Solver::substep; `k` selects the stage.
template<class M>
__global__ void kb_regrid(DG_BATCH_PARAMS, int k) {
	DG_BATCH_PROLOGUE
	constexpr int EX = EPOCH_EST<M>;
	const int L      = s.L;
	switch (k) {
		case 0: d_unsplit_select<M>(g, a.P, a.Ls.clu[L], s.n, L, a.Ls.unsplit, a.cnt); break;
		case 1: d_split<M>(g, a.P, cst, &a.cnt->n_split, a.Ls.split, L, a.Ls.fresh, s.epoch0 + EX + 1, a.cnt); break;
		case 2: d_unsplit<M>(g, a.P, cst, &a.cnt->n_unsplit, a.Ls.unsplit, L, a.Ls.fresh, s.epoch0 + EX + 2, a.cnt); break;
		case 3: d_nbr_fresh<M>(g, a.P, cst, &a.cnt->n_new, a.Ls.fresh, a.Ls.upd, a.cnt); break;
		case 4: d_nbr_list<M>(g, a.P, cst, &a.cnt->n_upd, a.Ls.upd, a.cnt); break;
		case 5: d_reassign<M>(g, a.P, cst, a.Ls.clu[L], nullptr, s.n, L, s.dtL, s.counterL, a.Ls, a.cnt); break;
		default: d_reassign<M>(g, a.P, cst, a.Ls.fresh, &a.cnt->n_new, 0, L, s.dtL, s.counterL, a.Ls, a.cnt); break;
	}
}

// The rebuilt cluster list becomes the level's list and its count the cluster count (Solver::substep's
// swap of Lists::clu[L] and Lists::tmp).
static __global__ void kb_swap(TreeArgs *A, const SubArgs *SA, int nt, const int *on) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nt || !*on || !SA[k].active) return;
	TreeArgs &a   = A[SA[k].tree];
	const int L   = SA[k].L;
	int32_t *x    = a.Ls.clu[L];
	a.Ls.clu[L]   = a.Ls.tmp;
	a.Ls.tmp      = x;
	a.cnt->clu[L] = a.cnt->n_tmp;
}

// flush_acti_buffer of level L for the listed trees (impl/acti_utils.hpp:365-372).
static __global__ void kb_flush(DG_BATCH_PARAMS) {
	DG_BATCH_PROLOGUE_NC
	d_flush(g, a.P, a.Ls.buf[s.L], &a.cnt->buf[s.L], a.Ls.clu[s.L], &a.cnt->clu[s.L], s.L, a.cnt);
}

// Closes a substep for each tree that ran it: the ACTI counter and time of level L advance
// (impl/integrate.hpp:56-57), buffer L goes to zero, then the running totals (splits, coarsenings, the
// cluster's cells after the flush, substeps).
static __global__ void kb_done(const TreeArgs *A, const SubArgs *SA, int nt, const int *on) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nt || !*on || !SA[k].active) return;
	const TreeArgs &a = A[SA[k].tree];
	Counters *c       = a.cnt;
	const int L       = SA[k].L;
	a.sch->counter[L] = (a.sch->counter[L] + 1) % 2;
	a.sch->time[L] += SA[k].dtL;
	c->buf[L] = 0;
	c->n_split_total += (unsigned long long) c->n_split;
	c->n_unsplit_total += (unsigned long long) c->n_unsplit;
	c->n_updates_total += (unsigned long long) c->clu[L];
	c->n_substeps_total += 1ull;
}

// Status of every tree to zero as a global step starts (a tree's status holds its last substep's).
static __global__ void kb_clear_status(Counters *cnt, int n_trees) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < n_trees) cnt[t].status = 0;
}

#undef DG_BATCH_PROLOGUE
#undef DG_BATCH_PROLOGUE_NC
#undef DG_BATCH_HEAD
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
	virtual void set_pregrow(bool on) = 0;
	std::string last_error;
};

template<class M>
class Batch : public BatchBase {
	static constexpr int D = M::D, NC = 1 << D, NF = 2 * D;
	static constexpr int EPOCHS = EPOCH_EST<M> + 2;  // epoch numbers one substep uses per tree
	static constexpr int LANES  = NF <= 4 ? 4 : 8;    // lanes per cell of the lane-group stages
	static constexpr int HEADROOM = 2;  // levels above its finest that a tree may take on within a run

	// Block-offset tables of a substep: the stage kind whose budget sizes the launch, and the work items
	// per cluster cell it is split by (lanes, cells, new cells, repair tasks, buffer cells).
	enum Table : int { T_FACE, T_RECV, T_UPD, T_SLOPE, T_AUX_L, T_AUX_C, T_EST, T_RG_CELL, T_RG_FRESH, T_NBR, T_FLUSH, TABLES };
	static constexpr int TABLE_STAGE[TABLES] = {BS_FACE_SUM, BS_RECEIVE, BS_UPDATE, BS_SLOPE, BS_AUX, BS_AUX,
	                                            BS_ESTIMATE, BS_REGRID_CELL, BS_REGRID_FRESH, BS_NBR_LIST, BS_FLUSH};
	static constexpr long long TABLE_ITEMS[TABLES] = {LANES, LANES, 1, LANES, LANES, 1, LANES, 1, NC + 1, (NC + 1) * NF, 0};
	// threads per block of each table's launches (the face sums and slopes run smaller blocks)
	static constexpr int TABLE_THREADS[TABLES] = {FACE_THREADS, BLOCK, BLOCK, SLOPE_THREADS, BLOCK, BLOCK,
	                                              BLOCK, BLOCK, BLOCK, BLOCK, BLOCK};

	// The schedule's position: sequence value and the next level index to look at in it (MAX_ACTI: the
	// next sequence value is due).
	struct Cursor {
		int seq = 0;
		int l   = MAX_ACTI;
	};
	// One planned merged substep: its level, the trees that may run it, the schedule position after it
	// and its slot in the arena.
	struct Planned {
		int L;
		std::vector<int> sel;
		Cursor after;
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
	TreeSched *d_sched_ = nullptr, *h_sched_ = nullptr;
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
	bool prof_    = false;
	bool pregrow_ = true;
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
	long long runs_ = 0, stops_ = 0, planned_ = 0, completed_ = 0;

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
		DG_CUDA(cudaMalloc(&d_sched_, sizeof(TreeSched) * nt));
		DG_CUDA(cudaMallocHost(&h_sched_, sizeof(TreeSched) * nt));
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
		cudaFree(d_sched_);
		cudaFreeHost(h_sched_);
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

	// Pools grown ahead of a run (on by default); off, a pool grows only at the capacity check.
	void set_pregrow(bool on) override { pregrow_ = on; }

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

	// Planned runs, runs a check stopped, substeps planned and substeps the host completed after a stop,
	// since the batch was made.
	void run_stats(long long *out, int n) override {
		const long long v[4] = {runs_, stops_, planned_, completed_};
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

	// Counters, the stop record, the halts, the trees' schedule state and list pointers back to the host;
	// the solvers take their schedule state and lists from the device.
	void sync() {
		const size_t N = s_.size();
		DG_CUDA(cudaMemcpyAsync(h_cnt_, d_cnt_, sizeof(Counters) * N, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaMemcpyAsync(h_stall_, d_stall_, sizeof(int), cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaMemcpyAsync(h_halt_, d_halt_, sizeof(int) * N, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaMemcpyAsync(h_sched_, d_sched_, sizeof(TreeSched) * N, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaMemcpyAsync(h_trees_, d_trees_, sizeof(TreeArgs) * N, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		if (prof_) drain();
		for (size_t t = 0; t < N; ++t) {
			Solver<M> *s       = s_[t];
			const TreeSched &z = h_sched_[t];
			s->max_acti_       = z.max_acti;
			s->stamp_          = z.stamp;
			s->epoch_          = z.epoch;
			std::copy(z.counter, z.counter + MAX_ACTI, s->acti_counter_);
			std::copy(z.time, z.time + MAX_ACTI, s->acti_time_);
			s->Ls_ = h_trees_[t].Ls;
		}
	}

	// ---- the schedule --------------------------------------------------------------------------

	// The next (sequence value, level) pair of the merged schedule (impl/integrate.hpp:25-28 per tree,
	// merged) when the batch's finest populated level is F: the sequence counter advances with F's
	// stride (values in between only have levels above F due, which are empty), and at each value the
	// due levels up to F run from the finest down.
	static bool next_pair(Cursor &c, int F, int &L) {
		const int top_seq = 1 << (MAX_ACTI - 1);
		while (true) {
			if (c.l >= MAX_ACTI) {
				const int stride = 1 << (MAX_ACTI - 1 - F);
				c.seq            = (c.seq / stride + 1) * stride;
				if (c.seq > top_seq) return false;
				c.l = 0;
			}
			for (; c.l < MAX_ACTI; ++c.l) {
				if (c.seq % (1 << c.l) != 0) continue;
				L = MAX_ACTI - c.l - 1;
				if (L > F) continue;
				++c.l;
				return true;
			}
		}
	}

	// A tree's finest level as a run starts: its max_acti_level or a populated level above it.
	int finest_of(int t) const {
		int f = s_[t]->max_acti_;
		for (int l = MAX_ACTI - 1; l > f; --l)
			if (h_cnt_[t].clu[l] > 0) return l;
		return f;
	}

	// After substeps ran: a capacity or structure error throws, a NaN halts the tree for the rest of the
	// global step (force_break).
	void post_checks(std::vector<char> &halted, int *force_break, double *global_dt) {
		for (size_t t = 0; t < s_.size(); ++t) {
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

	// Scratch rows for the clusters as they are now (and half as much again), then every tree's arguments
	// and schedule state; `head[t]` is the highest level tree t may run within the run.
	void prepare(const std::vector<char> &halted, const std::vector<int> &head) {
		const int N = (int) s_.size();
		for (int t = 0; t < N; ++t) {
			Solver<M> *s      = s_[t];
			const Counters &c = h_cnt_[t];
			long long most    = 0;
			for (int l = 0; l < MAX_ACTI; ++l) most = std::max<long long>(most, c.clu[l]);
			if (!halted[t]) {
				// at least a fifth of the tree free as a run starts, else room for half the tree again: growing
				// early only changes the capacity, never a result, and spares most runs a stop at the
				// capacity check
				const long long top = c.top;
				if (pregrow_ && top + top / 5 + 16 * NC > s->P_.cap) {
					const long long want = s->growth_target(s->P_.cap, std::max(top + top / 2 + 16 * NC, (long long) s->P_.cap * 5 / 4));
					if (want > s->P_.cap) s->grow_pool((int) std::min<long long>(want, 2000000000LL));
				}
				s->ensure_scratch(most + most / 2);
			}
			TreeArgs &a = h_trees_[t];
			a.P         = s->P_;
			a.C         = d_consts_ + t;
			a.B         = s->B_;
			a.Ls        = s->Ls_;
			a.cnt       = s->d_cnt_;
			a.sch       = d_sched_ + t;
			a.scratch   = s->scratch_cap_;
			a.limiter   = s->limiter_;
			a.halted    = halted[t];
			a.finest    = head[t];
			a.epochs    = EPOCHS;
			TreeSched &z = h_sched_[t];
			z.max_acti   = s->max_acti_;
			z.stamp      = s->stamp_;
			z.epoch      = s->epoch_;
			z.pad        = 0;
			std::copy(s->acti_counter_, s->acti_counter_ + MAX_ACTI, z.counter);
			std::copy(s->acti_time_, s->acti_time_ + MAX_ACTI, z.time);
		}
		upload_trees();
		DG_CUDA(cudaMemcpyAsync(d_sched_, h_sched_, sizeof(TreeSched) * N, cudaMemcpyHostToDevice, st_));
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
		const size_t want = std::max(bytes, arena_cap_ + arena_cap_ / 2);
		cudaFree(d_arena_);
		cudaFreeHost(h_arena_);
		d_arena_   = nullptr;
		h_arena_   = nullptr;
		arena_cap_ = 0;
		DG_CUDA(cudaMalloc(&d_arena_, want));
		DG_CUDA(cudaMallocHost(&h_arena_, want));
		arena_cap_ = want;
	}

	// Block offsets of one table: tree k gets blocks of `threads` in proportion to its planned items (at
	// least one), the launch at most `cap` blocks in total unless every tree needs its one. Returns the
	// block count.
	static int fill_offsets(int *h, const std::vector<long long> &items, int cap, int threads) {
		const int nt   = (int) items.size();
		long long want = 0;
		std::vector<long long> nb(nt);
		for (int k = 0; k < nt; ++k) {
			nb[k] = std::max<long long>(1, (items[k] + threads - 1) / threads);
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

	// The slot of a planned substep in the host arena: closed flags, the trees' rows (tree, level, dtL;
	// kb_begin writes the rest), offset tables sized on the planning counts `cnt`.
	void write_slot(Planned &p, const Counters *cnt) {
		const int nt = (int) p.sel.size();
		char *slot   = h_arena_ + p.at;
		std::memset(slot, 0, 16);
		SubArgs *S = (SubArgs *) (slot + 16);
		for (int k = 0; k < nt; ++k) {
			SubArgs a{};
			a.tree = p.sel[k];
			a.L    = p.L;
			a.dtL  = s_[p.sel[k]]->global_dt_ / (double) (1 << p.L);
			S[k]   = a;
		}
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
			p.grid[tb]  = fill_offsets(off + (size_t) tb * (nt + 1), items, sms_ * bps_[TABLE_STAGE[tb]], TABLE_THREADS[tb]);
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

	// The launches of planned substep `idx`: the head (opening and checks, fluxes, update, slopes,
	// multiphase auxiliaries, indicator, capacity check) and the tail (regrid, reassignment, list swap,
	// flush, closing).
	void launch(const Planned &p, int idx, bool head, bool tail) {
		const int nt      = (int) p.sel.size();
		char *slot        = d_arena_ + p.at;
		int *flags        = (int *) slot;
		SubArgs *S        = (SubArgs *) (slot + 16);
		const int *off    = (const int *) (slot + 16 + sizeof(SubArgs) * nt);
		const TreeArgs *A = d_trees_;
		const int *on     = flags;
		if (head) {
			kb_begin<<<1, 256, 0, st_>>>(d_trees_, (int) s_.size(), S, nt, flags, d_stall_, d_halt_, idx);
			stage(p, T_FACE, off, [&](int grid, const int *o) {
				constexpr int T = FACE_THREADS;
				if (mixed_) {
					if (visc_) kb_face_sum<M, true, float><<<grid, T, 0, st_>>>(A, S, o, nt, on);
					else kb_face_sum<M, false, float><<<grid, T, 0, st_>>>(A, S, o, nt, on);
				} else {
					if (visc_) kb_face_sum<M, true, double><<<grid, T, 0, st_>>>(A, S, o, nt, on);
					else kb_face_sum<M, false, double><<<grid, T, 0, st_>>>(A, S, o, nt, on);
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
				constexpr int T = SLOPE_THREADS;
				if (visc_) kb_slope<M, true><<<grid, T, 0, st_>>>(A, S, o, nt, on);
				else kb_slope<M, false><<<grid, T, 0, st_>>>(A, S, o, nt, on);
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

	// Completes planned substep `idx`, whose run stopped at the capacity check: the pools of the trees
	// that ran it and cannot take their split requests grow (Solver::substep), then the substep's tail runs.
	void finish_substep(const Planned &p, int idx) {
		const int nt = (int) p.sel.size();
		std::vector<SubArgs> rows(nt);
		DG_CUDA(cudaMemcpyAsync(rows.data(), d_arena_ + p.at + 16, sizeof(SubArgs) * nt, cudaMemcpyDeviceToHost, st_));
		DG_CUDA(cudaStreamSynchronize(st_));
		bool grown = false;
		for (int k = 0; k < nt; ++k) {
			if (!rows[k].active) continue;
			Solver<M> *s         = s_[p.sel[k]];
			const long long need = (long long) s->h_cnt_->top + (long long) NC * s->h_cnt_->n_split + 16;
			if (need > s->P_.cap) {
				const long long want = s->growth_target(need, std::max(need + need / 4, (long long) s->P_.cap * 5 / 4));
				s->grow_pool((int) std::min<long long>(want, 2000000000LL));
				grown = true;
			}
		}
		if (grown) {
			// the pools and lists moved; the halt flags are the device's (read back by the last sync)
			for (size_t t = 0; t < s_.size(); ++t) {
				TreeArgs &a = h_trees_[t];
				a.P         = s_[t]->P_;
				a.Ls        = s_[t]->Ls_;
				a.scratch   = s_[t]->scratch_cap_;
			}
			upload_trees();
		}
		int *flags = (int *) (d_arena_ + p.at);
		DG_CUDA(cudaMemcpyAsync(flags + 1, h_one_, sizeof(int), cudaMemcpyHostToDevice, st_));
		launch(p, idx, false, true);
		sync();
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
		// a status left from before the step belongs to no substep of it
		for (int t = 0; t < N; ++t) {
			s_[t]->check_status();
			h_cnt_[t].status = 0;
		}
		kb_clear_status<<<(N + 127) / 128, 128, 0, st_>>>(d_cnt_, N);
		Cursor cur;
		std::vector<Planned> plan;
		std::vector<Counters> pred(N);
		std::vector<int> head(N);
		while (true) {
			// a run from here, planned on the counts as they are now (the stream is idle, h_cnt_ and the
			// solvers' schedule state current): the batch's finest level F sets the pairs, a tree may run
			// levels up to HEADROOM above its own finest
			int F = -1;
			for (int t = 0; t < N; ++t) {
				head[t] = finest_of(t);
				if (!halted[t]) F = std::max(F, head[t]);
			}
			if (F < 0) break;  // every tree has halted
			for (int t = 0; t < N; ++t) head[t] = std::min(F, head[t] + HEADROOM);
			prepare(halted, head);
			std::copy(h_cnt_, h_cnt_ + N, pred.begin());
			plan.clear();
			size_t bytes  = 0;
			bool finished = false;
			while ((int) plan.size() < window_) {
				int L;
				if (!next_pair(cur, F, L)) {
					finished = true;
					break;
				}
				std::vector<int> sel;
				for (int t = 0; t < N; ++t)
					if (!halted[t] && L <= head[t]) sel.push_back(t);
				if (sel.empty()) continue;
				Planned p;
				p.L     = L;
				p.sel   = std::move(sel);
				p.after = cur;
				p.at    = bytes;
				bytes += slot_bytes((int) p.sel.size());
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
			for (int t = 0; t < N; ++t)
				if (h_halt_[t] != STALL_NONE) {
					force_break[t] = 1;
					global_dt[t]   = s_[t]->global_dt_;
					halted[t]      = 1;
				}
			const int stop = *h_stall_;
			if (stop == STALL_NONE) {
				// a NaN in a tree's last substep of the run halts it now; an error throws
				post_checks(halted, force_break, global_dt);
				if (finished) break;
				window_ = std::min(window_ * 2, WINDOW_MAX);
				continue;
			}
			++stops_;
			window_     = std::max(window_ / 2, WINDOW_MIN);
			const int i = stop / 2, half = stop & 1;
			if (i == 0 && !half) throw dg_error(DG_ERR_UNSUPPORTED, "batch: a planned run stopped before its first substep");
			if (!half) {
				// substep i did not start: the schedule resumes at it
				cur = plan[i - 1].after;
			} else {
				// substep i's head ran: complete it, then resume after it
				finish_substep(plan[i], i);
				++completed_;
				cur = plan[i].after;
			}
			post_checks(halted, force_break, global_dt);
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
