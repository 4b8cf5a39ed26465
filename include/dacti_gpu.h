/*
 * dacti_gpu.h — C ABI of the B200 octree finite-volume step.
 *
 * Drop-in replacement for the solver step of DACTI's header-only
 * dacti::integrator::Integrator<Model, Limiter, ErrorEstimator>
 * (src/lib/integrator/integrator.hpp:14-225). The reference has no FFI layer; these entry points
 * are what its class template does, flattened to plain pointers and sizes so that any host (the C++
 * adapter include/dacti_gpu/integrator.hpp, ctypes, cgo, JNI) can bind them. All functions return a
 * dg_status; nothing throws across the ABI.
 */
#ifndef DACTI_GPU_H
#define DACTI_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dg_solver dg_solver;

/* status codes */
enum {
	DG_OK              = 0,
	DG_ERR_ARG         = -1, /* invalid argument or unsupported model/dimension */
	DG_ERR_CUDA        = -2, /* CUDA runtime error (dg_last_error has the text) */
	DG_ERR_CAPACITY    = -3, /* node pool or list capacity exceeded on the device */
	DG_ERR_DEPTH       = -4, /* tree deeper than the neighbourhood walkers support */
	DG_ERR_MISSING_BC  = -5, /* a face with neither neighbour nor boundary condition */
	DG_ERR_UNSUPPORTED = -6  /* feature of the reference not supported by this build */
};

/* model ids (dacti::model::euler / navier_stokes / multi) */
enum { DG_EULER = 0, DG_NAVIER_STOKES = 1, DG_MULTI = 2 };

/* numerical forms: the reference's FP64 arithmetic, or FP32 reconstruction and HLLC flux, face fluxes
 * stored in FP32 (both sides of a face read the same value, so conservation stays exact), with the
 * flux sums, the conservative update, the conservation totals and the pressure/temperature recovery
 * in FP64 */
enum { DG_FORM_FP64 = 0, DG_FORM_MIXED = 1 };
/* Stage implementation choices of the single-tree step (dg_set_options). Every combination gives the
 * same results bit for bit; they differ only in speed.
 *   DG_OPT_ORDERED_LISTS: the reassignment rebuilds the running cluster's list in its old order (an
 *     order-keeping compaction), so lists keep the Morton order of the last re-sort through the step;
 *     without it the cells that stay are appended in the order the GPU reaches them.
 *   DG_OPT_FACE_TILES: the face sums run over tiles of consecutive list positions and evaluate a face
 *     whose two cells are both in the tile once instead of once per cell. */
enum { DG_OPT_ORDERED_LISTS = 1, DG_OPT_FACE_TILES = 2, DG_OPT_DEFAULT = DG_OPT_ORDERED_LISTS | DG_OPT_FACE_TILES };

/* limiter ids (dacti::integrator::slope, integrator/slope_limiters.hpp:7-57) */
enum { DG_MINMOD = 0, DG_UNLIMITED, DG_VAN_LEER, DG_SUPERBEE, DG_VON_ALBA_2, DG_KOREN, DG_FIRST_ORDER };

/* layout of dg_case.params (Config fields read by integrator/integrator.hpp:80-86 and model constants) */
enum {
	DG_P_SIDE = 0, DG_P_ACTIVE0 = 1, DG_P_PERIODIC0 = 4, DG_P_MAX_CFL = 7, DG_P_MAX_DT = 8, DG_P_MIN_ERR = 9,
	DG_P_MAX_ERR = 10, DG_P_MAX_LEVEL = 11, DG_P_MIN_LEVEL = 12, DG_P_GAMMA = 13, DG_P_NS_MU = 14,
	DG_P_NS_LAMBDA = 15, DG_P_GAMMA1 = 16, DG_P_GAMMA2 = 17, DG_P_P1 = 18, DG_P_P2 = 19, DG_P_CP1 = 20,
	DG_P_CP2 = 21, DG_P_CV1 = 22, DG_P_CV2 = 23, DG_P_MU1 = 24, DG_P_MU2 = 25, DG_P_LAMBDA1 = 26,
	DG_P_LAMBDA2 = 27, DG_P_SIGMA = 28,
	/* GPU solver only: node slots the host left out of the upload (subtrees without active leaves), counted
	 * in the tree size as the reference counts them; node-pool capacity in slots (0: 1.5 x n_nodes) */
	DG_P_PRUNED = 29, DG_P_POOL_CAP = 30, DG_N_PARAMS = 32
};

/* node flag bits of dg_case.flags (integrator/node.hpp:60-66) */
enum {
	DG_F_LEAF = 1, DG_F_ACTIVE = 2, DG_F_GARBAGE = 4, DG_F_CAN_SPLIT = 8, DG_F_CAN_UNSPLIT = 16,
	DG_F_SHOULD_SPLIT = 32, DG_F_IS_BOUNDARY = 64
};

/*
 * The initial tree as Scene::init_domain leaves it (scene/scene.cpp:369-431): every node slot,
 * slot 0 the null node and slot 1 the root. Arrays are row-major per node:
 * children[n][2^D], bc[n][2D] (index into the boundary table or -1), center[n][D], p[n][E].
 */
typedef struct dg_case {
	int model, dims;
	int n_nodes, n_bc, n_zones;
	int limiter;
	const double *params;     /* DG_N_PARAMS */
	const double *weights;    /* E: weighted_laplacian weights (integrator/error_estimators.hpp:336) */
	const double *zones;      /* n_zones x {x0[3], x1[3], max_level} refinement zones */
	const int *bc_type;       /* n_bc Boundary::Type values (integrator/boundary.hpp:23-32) */
	const double *bc_p_in;    /* n_bc x E */
	const double *bc_normal;  /* n_bc x D */
	const double *bc_fade_in; /* n_bc */
	const int *parent;
	const int *children;
	const int *level;
	const unsigned *flags;
	const int *bc;
	const double *center;
	const double *p;
} dg_case;

/* Called after every level substep, like the substep_hook of Integrator::integrate
 * (impl/integrate.hpp:64): (user, level, level time, substep count, level dt, cluster size). */
typedef void (*dg_substep_fn)(void *user, int level, double acti_time, int n_substeps, double dt_level,
                              long long cluster_size);

/* kernel kinds reported in dg_stats.kernel_* */
enum {
	DG_K_FLUX = 0, DG_K_RECV, DG_K_UPDATE, DG_K_SLOPE, DG_K_AUX, DG_K_ESTIMATE, DG_K_REGRID, DG_K_REASSIGN,
	DG_K_FLUSH, DG_K_INIT, DG_K_GC, DG_K_OTHER, DG_NK
};

typedef struct dg_stats {
	long long n_clusters[16];   /* cells per ACTI cluster */
	long long n_buffers[16];    /* cells waiting in ACTI buffers */
	long long tree_size;        /* node slots incl. the null slot (Domain::tree.size()) */
	long long n_splits, n_unsplits, n_gc;
	long long n_substeps, n_global_steps;
	long long cell_updates;     /* sum of cluster sizes over executed substeps */
	int max_acti_level;
	double global_dt;
	double acti_time[16];
	int acti_counter[16];
	long long n_launches;        /* kernels launched by this solver so far */
	double kernel_ms[DG_NK];     /* device time per kernel kind (when profiling is on) */
	long long kernel_launches[DG_NK];
	long long kernel_cells[DG_NK]; /* cells processed per kernel kind (cluster-sized launches) */
} dg_stats;

/* Selects the CUDA device on which the calling thread's next dg_create builds its solver; every
 * later call on that solver runs on the same device. Default: device 0. */
int dg_set_device(int ordinal);

/* Integrator constructor (integrator/integrator.hpp:72-163) on a flattened initial tree. */
int dg_create(const dg_case *c, dg_solver **out);

/* Optional CUDA stream (cudaStream_t) on which all work of this solver is issued. */
int dg_set_stream(dg_solver *s, void *cuda_stream);

/* Integrator::integrate (impl/integrate.hpp:12-87): one global step over all ACTI levels.
 * force_break is set when a cell update produced NaN (the step stops at that substep). */
int dg_step(dg_solver *s, int signal, int *force_break, double *global_dt, dg_substep_fn fn, void *user);

/* One global step of each of n independent solvers (a batch of trees, each one Integrator of the
 * reference stepped on its own), driven by up to `threads` host threads with every solver on a stream
 * of its own so that the trees' kernels overlap on the device. Results per tree are those of dg_step
 * (bitwise: the kernels are deterministic); force_break[k], global_dt[k] and status[k] per solver; the
 * return value is the first non-DG_OK status or DG_OK. A solver still on the legacy default stream gets
 * a stream of its own. No substep callback. */
int dg_step_many(dg_solver **solvers, int n, int threads, int signal, int *force_break, double *global_dt,
                 int *status);

/* A batch of independent trees of one model, numeric form and set of viscous/tension terms, stepped in
 * lockstep by one host thread (the chosen form's batched path; no counterpart in the reference, where
 * every tree is an Integrator stepped on its own, impl/integrate.hpp:12-87). The trees' ACTI schedules
 * are merged; each substep of level L launches every stage once for all trees that run L, over block
 * ranges split among them by work. The host plans the global step and issues it with no
 * synchronisation; each tree's schedule state lives on the device, which applies the reference's level
 * rule per tree and halts a tree with a NaN there. Device-side checks stop a run only where the live
 * counts leave the plan (a tree populating a level beyond its headroom, a pool that must grow), and the
 * host resumes from there.
 * Per tree the results are dg_step's, bit for bit. While in the batch, the solvers run on the batch's stream and keep their
 * counters in the batch's array: step them through dg_batch_step only, and destroy the batch before
 * its solvers. */
typedef struct dg_batch dg_batch;
int dg_batch_create(dg_solver **solvers, int n, dg_batch **out);
/* One global step of every tree: force_break[k] and global_dt[k] per tree, as dg_step's. */
int dg_batch_step(dg_batch *b, int signal, int *force_break, double *global_dt);
const char *dg_batch_last_error(dg_batch *b);
void dg_batch_destroy(dg_batch *b);

/* Stage kinds of a merged batch substep, in this order: face sums, flux receive, cell update, slopes,
 * multiphase auxiliary sweeps, indicator, per-cell regrid, regrid of new cells, neighbour repair,
 * buffer flush. */
enum { DG_BATCH_STAGES = 10 };
/* Launch budget of each stage kind in blocks per SM (1..64, default 16): a launch splits that many blocks
 * among the trees in proportion to their work. What the autotuner (dacti_b200/autotune.py) sets. */
int dg_batch_set_launch(dg_batch *b, const int *blocks_per_sm, int n_stages);
/* Per-stage device timing with CUDA events (off by default). */
int dg_batch_set_profiling(dg_batch *b, int on);
/* Device milliseconds and work items per stage kind since the previous call. */
int dg_batch_stage_times(dg_batch *b, double *ms, long long *items, int n_stages);
/* Since the batch was made: out[0] planned runs, out[1] runs a check stopped, out[2] substeps planned,
 * out[3] substeps the host completed after a stop at the capacity check (n <= 4 values). */
int dg_batch_run_stats(dg_batch *b, long long *out, int n);
/* Pools grown ahead of each planned run when less than a fifth of the tree is free, to half the tree
 * again (on by default; capacity never changes a result). Off, a pool grows only where a run stops at
 * the capacity check. */
int dg_batch_set_pregrow(dg_batch *b, int on);

/* Integrator::n_active_cells (integrator/integrator.hpp:193-202) */
int dg_cell_count(dg_solver *s, long long *n);

/* for_each_active_cell (integrator/integrator.hpp:172-191): clusters 0..15 then buffers 0..15.
 * levels[n][2] = {tree_level, acti_level}; data[n][D + 1 + 2E + 3 + P] =
 * {center[D], t, u[E], p[E], error, max_dt, cfl, k[P]} with P = NumParm (D + 4 for the
 * multiphase model: mu, unused, interface normal[D], curvature, smoothed volume fraction; 0 otherwise). */
int dg_read_cells(dg_solver *s, int *levels, double *data, long long max_cells, long long *n_out);

/* The limited slopes (Cell::slope, integrator/cell.hpp:19) of the active cells, slopes[n][D][E], in the
 * order of dg_read_cells: what a writer needs to evaluate Cell::get_p(x, t) (cell.hpp:23-31) at points
 * of the cell, as DACTI's VTU writer does at the cell vertices (driver/io/vtu_writer.hpp:40-62). */
int dg_read_slopes(dg_solver *s, double *slopes, long long max_cells, long long *n_out);

/* The gradients of the gradient inputs (Cell::gradient, integrator/cell.hpp:20; written by
 * compute_slope, impl/slopes.hpp:68-70) of the active cells, gradients[n][D][G], in the order of
 * dg_read_cells. G is NumGrad: D + 1 for Navier-Stokes (velocity, temperature), D + 3 for the
 * multiphase model (velocity, temperature, volume fraction, and a last slot that is zero here and
 * indeterminate in the reference, whose get_grad_input leaves it unset, model/multi.hpp:148-156). What
 * DACTI's DropEnergy observer reads (driver/observer/drop_energy.hpp:25-26). DG_ERR_UNSUPPORTED for
 * the Euler model (no gradient inputs) and for multiphase cases without viscosity or conduction,
 * whose steps skip the gradient computation. */
int dg_read_gradients(dg_solver *s, double *gradients, long long max_cells, long long *n_out);

/* Integrator::get_nodes (integrator/integrator.hpp:165), as DACTI's HTG writer walks it
 * (driver/io/htg_writer.hpp:112-161): every node slot [0, n) of the device pool, internal, inactive and
 * garbage slots included, component-major: parent[n], children[2^D][n], level[n] (tree level),
 * flags[n] (bit 0 leaf, bit 1 active, bit 2 garbage), p[E][n] (meaningful on leaves), meta[4][n] =
 * Node::get_metadata() = {acti_level, error, max_dt, cfl} (integrator/node.hpp:56-58). Slot 0 is the
 * null node; the root is the one non-garbage slot of level 0 (slot numbers follow the device's own
 * re-sorts, not the reference's tree indices; child order is the reference's). dg_tree_size gives n. */
int dg_tree_size(dg_solver *s, long long *n);
int dg_read_tree(dg_solver *s, int *parent, int *children, int *level, unsigned int *flags, double *p, double *meta,
                 long long max_nodes, long long *n_out);

/* ---- Initial tree on the device: Scene::init_domain (scene/scene.cpp:369-431) for analytic scenes --
 * Spheres, ellipses and polygons (droplets, bubbles and solids with a boundary condition), domain-face
 * boundaries, object faces and fix_boundary, refinement near objects, inflow_r faces, the initial jump
 * and in zones, the uniform or jump initial condition and the tanh-smeared volume fraction. Produces the
 * same nodes in the same order as the host builder; the result feeds dg_case. Object faces come back
 * with boundary id -2: the caller assigns the nearest object's condition (the surface normal differs
 * per face, so the boundary table is the caller's). */
typedef struct dg_scene {
	int model, dims;
	double side_length, active_size[3];
	int min_level, max_level, max_level_geom;
	double refinement_radius;
	int domain_bc[3][2];  /* boundary-table id of each domain face, -1 on periodic dimensions */
	int inflow_r[3][2];   /* 1 where that face's condition is inflow_r (refined to the maximum level) */
	int n_objects;        /* <= 16 */
	const double *objects; /* 29 per object: centre[3], semi-axes[3] (a sphere's radius first), cos and sin
	                          of its rotation about z, shape (0 sphere, 1 ellipse, 2 polygon), type
	                          (0 droplet, 1 bubble, 2 solid), 1 if it has a boundary condition, 1 if that
	                          is inflow_r, the polygon's vertex count (3..8, 2D) and vertices x, y [8][2] */
	int n_zones;          /* <= 16 */
	const double *zones;  /* 7 per zone: x0[3], x1[3], level */
	int refine_jump, jump_axis;
	double jump_location;
	int ic_kind, ic_axis; /* 0 uniform (ic_neg), 1 jump (ic_pos where x[ic_axis] > ic_location) */
	double ic_location;
	const double *ic_neg, *ic_pos; /* E primitive values each */
	int diffuse_ic, keep_ic_gas_density;
	double rho_ref[2];
} dg_scene;
typedef struct dg_tree dg_tree;
const char *dg_build_last_error(void);
int dg_build_tree(const dg_scene *scene, dg_tree **out);
int dg_tree_nodes(const dg_tree *t, long long *n_nodes);
/* Host copies in the layout of dg_case: parent[n], children[n][2^D], level[n], flags[n], bc[n][2D],
 * center[n][D], p[n][E]. */
int dg_tree_copy(const dg_tree *t, int *parent, int *children, int *level, unsigned int *flags, int *bc,
                 double *center, double *p);
int dg_tree_free(dg_tree *t);

/* ---- Regrid forecaster (no counterpart in the reference) -------------------------------------
 * A small network that predicts from per-leaf features whether the refinement indicator will fire
 * at a leaf's place a few global steps ahead. */

/* Forecaster inputs of the active cells, features[n][5 + 5D], in the order of dg_read_cells: for the
 * cell, log(1 + 100 x) of x = |grad rho| h / rho, |grad p| h / p and |curl v| h / (|v| + c), its tree
 * level / 16, log(1 + err / max_err) of its last indicator value, its velocity / (|v| + c) per
 * dimension; then the first two quantities of the neighbour behind each face (face order x-, x+, y-,
 * ...; the cell's own where the face is a boundary or the neighbour is refined). */
int dg_forecast_features(dg_solver *s, double *features, long long max_cells, long long *n_out);

/* Forecast-driven regrid. hold[n] (one byte per active cell, dg_read_cells' order; n must equal the
 * active cell count): a held cell is never coarsened; splitting stays with the plain indicator, which
 * keeps splitting the cells it flags at every substep. dg_set_coarsen_interval
 * runs the coarsening test only on global steps that are multiples of `steps` (1, the default, is the
 * reference's every-substep behaviour). Holds stay until the next dg_set_hold; children of a split do
 * not inherit them. */
int dg_set_hold(dg_solver *s, const unsigned char *hold, long long n);
int dg_set_coarsen_interval(dg_solver *s, int steps);

/* Multilayer perceptron n_in -> 64 -> 64 -> 1 (ReLU hidden layers, logistic output) on the current
 * device, n_in <= 32. Parameters, in order: W1[64][n_in], b1[64], W2[64][64], b2[64], W3[64], b3.
 * Training keeps FP32 master weights and Adam moments; predictions use BF16 copies of the weights.
 * Errors: negative status, text from dg_mlp_last_error (per host thread). */
typedef struct dg_mlp dg_mlp;
const char *dg_mlp_last_error(void);
/* He-uniform hidden layers and Glorot-uniform output layer from `seed`, zero biases. */
int dg_mlp_create(int n_in, unsigned long long seed, dg_mlp **out);
int dg_mlp_param_count(dg_mlp *m, long long *n);
/* Replace / read the FP32 parameters; setting them also resets the Adam state. */
int dg_mlp_set_params(dg_mlp *m, const float *params);
int dg_mlp_get_params(dg_mlp *m, float *params);
/* prob[n] = sigmoid(logit(x[n][n_in])) with the BF16 weights. */
int dg_mlp_predict(dg_mlp *m, const float *x, long long n, float *prob);
/* Sum over the n samples of the loss pw y softplus(-z) + (1 - y) softplus(z) (z the logit, FP32 master
 * weights) and of its gradient with respect to every parameter. */
int dg_mlp_loss_grad(dg_mlp *m, const float *x, const float *y, long long n, float pos_weight, float *grad,
                     double *loss_sum);
/* `epochs` passes of Adam (beta 0.9 / 0.999) over shuffled minibatches of the mean loss; mean_loss is
 * the mean over the samples of the last pass. */
int dg_mlp_train(dg_mlp *m, const float *x, const float *y, long long n, int epochs, int batch, float lr,
                 float pos_weight, unsigned long long seed, double *mean_loss);
int dg_mlp_destroy(dg_mlp *m);

/* Allocation-free variant of dg_read_cells for hosts that cannot let the library call cudaMalloc
 * (a fixed device-memory budget owned by the host's allocator, or a thread that must not take the
 * device-wide synchronisation of cudaMalloc/cudaFree). No counterpart in the reference: DACTI's
 * Integrator hands out host references to its nodes. Same records and order as dg_read_cells,
 * gathered through a 64 MiB scratch array that the library keeps resident on each device: read-backs
 * larger than that return DG_ERR_CAPACITY: a cell takes 8 (D + 2E + P + 5) bytes of it, so it holds about 289
 * thousand multi<3> cells or 559 thousand euler<2> cells. dg_create places the scratch on the solver's
 * device and looks up its address, so no call of this function allocates, the first one included.
 * Calls share the scratch, so calls whose GPU work overlaps race. */
int dg_read_cells_noalloc(dg_solver *s, int *levels, double *data, long long max_cells, long long *n_out);

int dg_get_stats(dg_solver *s, dg_stats *out);

/* Numerical form of the following steps (DG_FORM_FP64 by default). No counterpart in the reference,
 * which computes everything in FP64. */
int dg_set_form(dg_solver *s, int form);

/* Stage implementation choices (DG_OPT_* bits, DG_OPT_DEFAULT at creation). No counterpart in the
 * reference. */
int dg_set_options(dg_solver *s, int options);

/* Per-kernel device timing with CUDA events on the solver's stream (off by default). */
int dg_set_profiling(dg_solver *s, int on);

/* Text of the last error on this solver (or of the last failed dg_create when s is NULL). */
const char *dg_last_error(dg_solver *s);

void dg_destroy(dg_solver *s);

#ifdef __cplusplus
}
#endif

#endif /* DACTI_GPU_H */
