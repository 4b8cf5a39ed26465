// Device-side data layout of the octree node pool and solver constants.
#pragma once

#include <cstdint>

namespace dg {

constexpr int MAX_ACTI      = 16;  // ACTI (time) levels, integrator/integrator.hpp:28
constexpr int MAX_TREE      = 32;  // tree levels with per-level size/area/volume tables
constexpr int MAX_ZONES     = 8;
constexpr int BUF_BASE      = 16;  // membership code of buffer L is BUF_BASE + L
constexpr int8_t CLU_NONE   = -1;

// Node flag bits (mirror the bool members of integrator/node.hpp:60-66).
enum : uint32_t {
	F_LEAF         = 1u << 0,
	F_ACTIVE       = 1u << 1,
	F_GARBAGE      = 1u << 2,
	F_CAN_SPLIT    = 1u << 3,
	F_CAN_UNSPLIT  = 1u << 4,
	F_SHOULD_SPLIT = 1u << 5,
	F_IS_BOUNDARY  = 1u << 6,
	F_HOLD         = 1u << 7,  // held by the regrid forecaster: never coarsened
	F_RECV         = 1u << 8,  // the received-flux accumulator may be non-zero (set by the receive stage)
};
constexpr uint32_t F_PUBLIC = 0x7fu;  // the flag bits of include/dacti_gpu.h

// Refinement op codes written by the estimation kernel.
enum : uint8_t {
	OP_NONE   = 0,
	OP_SPLIT  = 1,  // split requested and 2:1 guard passed
	OP_UCAND  = 2,  // unsplit candidate whose neighbourhood allows coarsening
};

// Boundary::Type (integrator/boundary.hpp:23-32)
enum : int {
	BC_ZERO_GRADIENT = 0,
	BC_FREESLIP      = 1,
	BC_NOSLIP        = 2,
	BC_INFLOW        = 3,
	BC_INFLOW_R      = 4,
	BC_OUTFLOW       = 5,
	BC_DIRICHLET     = 6,
	BC_NEUMANN       = 7,
};

// Device error flags (OR-ed into Counters::status).
enum : uint32_t {
	ST_NAN          = 1u << 0,  // NaN pressure/density after a cell update (force_break)
	ST_DEPTH        = 1u << 1,  // tree deeper than the neighbourhood walkers support
	ST_CAPACITY     = 1u << 2,  // node pool or list capacity exceeded
	ST_SPLIT_UNSPLIT = 1u << 3, // a cell was both split-ready and a coarsening candidate
	ST_MISSING_BC   = 1u << 4,  // face with neither neighbour nor boundary
};

struct ModelConsts {
	double ns_mu, ns_lambda;
	double gamma1, gamma2, P1, P2, cp1, cp2, cv1, cv2, mu1, mu2, lambda1, lambda2, sigma;
};

struct Consts {
	ModelConsts m;
	double side;
	double active[3];
	int periodic[3];
	double max_cfl, min_err, max_err;
	double weights[8];
	int max_refinement_level;
	int n_zones;
	double zx0[MAX_ZONES][3], zx1[MAX_ZONES][3];
	int zlevel[MAX_ZONES];
	double size[MAX_TREE], vol[MAX_TREE], area[MAX_TREE];
	// Active box in cells per tree level and dimension: [a0, a0 + na).
	int a0[MAX_TREE][3], na[MAX_TREE][3];
	int signal;  // `signal` argument of integrate (hold-droplet-still switch)
	int coarsen; // 0 on global steps where a forecast-driven regrid skips coarsening
	int visc;    // viscous or heat terms present: gradients and their time slopes are stored
};

// Boundary table (one Boundary<M> value per entry).
struct BcTable {
	int n;
	const int *type;
	const double *p_in;    // [n][E]
	const double *normal;  // [n][D]
	const double *fade_in; // [n]
};

// Structure-of-arrays node pool. Component c of node i lives at array[c * cap + i].
struct Pool {
	int cap;
	int32_t *parent;
	int32_t *child;   // [C][cap]
	int8_t *level;    // tree level
	int8_t *acti;     // ACTI level (Node::acti_level)
	int8_t *clu;      // membership: cluster L, BUF_BASE+L for buffer L, CLU_NONE
	uint32_t *flags;
	int32_t *coord;   // [D][cap] integer cell index at its own level
	int32_t *nbr;     // [2D][cap] neighbour slot (0 = none / boundary)
	int16_t *bc;      // [2D][cap] boundary table entry or -1
	double *center;   // [D][cap]
	double *t;
	double *u;        // [E][cap]
	double *p;        // [E][cap]
	double *rec;      // [cap][W] reconstruction record: p copy, Hancock rhs, slope rows, multiphase k part
	double *avg;      // [cap][AW] non-leaf nodes: memo of the mean primitive state and time of the subtree
	int32_t *mod;     // epoch of the latest change of any leaf below the node
	int32_t *cst;     // epoch at which `avg` was computed
	double *avga;     // non-leaf nodes: memo of the mean smoothed volume fraction of the subtree
	int32_t *csta;    // epoch at which `avga` was computed
	double *k;        // [P][cap]
	double *tslope;   // [G][cap], only with viscous or heat terms (Consts::visc)
	double *grad;     // [D][G][cap], only with viscous or heat terms
	double *flux;     // [F][cap]
	double *err, *maxdt, *cfl;
	int32_t *stamp;   // per-node dedup stamp for list building
	uint32_t *fmask;  // faces (bit 2 dim + dir) whose neighbour changed in the running regrid; 0 otherwise
	uint8_t *op;      // refinement op code
	double *tmp, *tmp2;  // per-node scratch scalars (Jacobi smoothing sweeps, alternately)
	// Per-substep scratch outside the permuted fields:
	double *ff;       // [slot][2D][F] flux of each owned face next to a receiver (by the owner's list position)
	double *du;       // [slot][F] face-flux sum of each running-cluster cell (by list position)
	int32_t *pos;     // [cap] list position of each running-cluster cell, written by the face-sum stage
};

// Device counters, copied back to the host after each substep.
struct Counters {
	int clu[MAX_ACTI];
	int buf[MAX_ACTI];
	int top;          // next free node slot (== reference tree.size())
	int n_recv;
	int n_split;
	int n_unsplit;
	int n_new;        // new cluster members (children + coarsened parents)
	int n_upd;        // neighbour-update list
	int n_tmp;        // rebuilt cluster list
	uint32_t status;
	// running totals that the batched step keeps on the device (splits, coarsenings, cluster cells after
	// each substep's flush, substeps)
	unsigned long long n_split_total, n_unsplit_total, n_updates_total, n_substeps_total;
	double dmax;      // reduction result
};

// Per-level index lists on the device.
struct Lists {
	int32_t *clu[MAX_ACTI];
	int32_t *buf[MAX_ACTI];
	int32_t *tmp;      // rebuilt cluster list
	int32_t *recv;     // receivers of cross-level fluxes
	int32_t *split;    // split-ready cells
	int32_t *unsplit;  // parents to coarsen
	int32_t *fresh;    // new children and coarsened parents
	int32_t *upd;      // neighbour-update list
};

}  // namespace dg
