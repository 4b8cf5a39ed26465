// Initial tree on the device: Scene::init_domain (scene/scene.cpp:369-431) for scenes with analytic
// spheres, ellipses and polygons, level by level as the host builder does it (dacti_b200/scene.py), so that
// both produce the same nodes in the same order:
//
//  - signed distances to the objects and the nearest object (scene.cpp:47-91), sphere |x - c| - r and
//    the ellipse measure (|R^T (x - c) / a| - 1) min(a); cells inside an object with a boundary
//    condition are inactive (scene.cpp:76-82);
//  - domain-face boundaries (scene.cpp:105-108) and object faces (scene.cpp:112-127): a face whose
//    same-level neighbour (Domain::find, integrator/domain.hpp:65-82, :407-417) differs in activity,
//    or whose centre-to-centre segment meets an object (Scene::raycast, scene.cpp:31-45), is marked;
//    the host gives marked faces the nearest object's condition and surface normal;
//  - split detection (scene.cpp:150-216): below the minimum level, near an object (solids to
//    max_refinement_level_geom), on an inflow_r face, near the initial jump, inside a zone;
//  - Domain::split child placement (integrator/domain.hpp:206): parent.center + (0.25 parent.size)
//    quadrant(i); the r-th splitting node gets children first + r C + c;
//  - fix_boundary (scene.cpp:249-337) ten times: active leaves coarser than an inactive neighbour
//    split (in ascending node order, children taking the parent's boundaries on shared faces) until
//    none is left, the new leaves' faces are tested again, one-sided boundaries are dropped;
//  - leaves outside the active box inactive, uniform or jump initial condition, and the interface
//    initialisation with its tanh smear (scene.cpp:343-365).
//
// Each pass reads only what earlier kernels wrote (the activity after the distance pass, the
// boundaries before a drop pass), which is the host builder's order of evaluation.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "dacti_gpu.h"
#include "dg_types.h"

namespace {

constexpr int TPB      = 256;
constexpr int MAX_OBJ  = 16;
constexpr int MAX_ZONE = 16;
constexpr int BC_MARK  = -2;  // object boundary; the host assigns the condition
constexpr int MAX_VERT = 8;   // polygon vertices per object
constexpr int OBJ_ROW  = 13 + 2 * MAX_VERT;

struct Scene {
	int D, E, C, NF, multi, ia;
	double side, active[3];
	int periodic[3];
	int min_level, max_level, max_level_geom;
	double radius;
	int dbc[3][2], inflow_r[3][2];
	int n_obj, walls;
	double oc[MAX_OBJ][3], oa[MAX_OBJ][3], ocs[MAX_OBJ], osn[MAX_OBJ];
	int oshape[MAX_OBJ], otype[MAX_OBJ], obc[MAX_OBJ], obc_inflow_r[MAX_OBJ];  // shape 0 sphere, 1 ellipse, 2 polygon
	int onv[MAX_OBJ];
	double ov[MAX_OBJ][MAX_VERT][2];
	int n_zone;
	double zx0[MAX_ZONE][3], zx1[MAX_ZONE][3];
	int zlevel[MAX_ZONE];
	int refine_jump, jump_axis;
	double jump_loc;
	int ic_kind, ic_axis;
	double ic_loc, ic_neg[8], ic_pos[8];
	int diffuse, keep_gas;
	double rho1, rho2, h_finest;
};

struct Arrays {
	int32_t *parent, *children, *level, *bc, *mesh;
	uint32_t *flags;
	double *center, *size, *sd, *p;
	uint8_t *isb, *aux, *mark;  // object-boundary node; face-pass result; fix_boundary marks
};

thread_local std::string g_err;

constexpr double DMAX = 1.7976931348623157e308;

__device__ bool active_node(const Arrays &A, long long i) { return i != 0 && (A.flags[i] & dg::F_ACTIVE); }

// Closed polygon (2D): distance to the nearest edge, negative inside (even-odd rule), in the host
// builder's order of operations.
__device__ double polygon_distance(const Scene &S, int o, const double *x) {
	double dist = INFINITY;
	bool inside = false;
	const int nv = S.onv[o];
	for (int k = 0; k < nv; ++k) {
		const double a0 = S.ov[o][k][0], a1 = S.ov[o][k][1];
		const double b0 = S.ov[o][(k + 1) % nv][0], b1 = S.ov[o][(k + 1) % nv][1];
		const double ab0 = b0 - a0, ab1 = b1 - a1;
		double t         = ((x[0] - a0) * ab0 + (x[1] - a1) * ab1) / (ab0 * ab0 + ab1 * ab1);
		t                = fmin(fmax(t, 0.0), 1.0);
		const double e0 = x[0] - (a0 + t * ab0), e1 = x[1] - (a1 + t * ab1);
		dist            = fmin(dist, sqrt(e0 * e0 + e1 * e1));
		const bool crosses = (a1 > x[1]) != (b1 > x[1]);
		if (crosses) {
			const double xc = a0 + (x[1] - a1) * ab0 / ab1;
			if (x[0] < xc) inside = !inside;
		}
	}
	return inside ? -dist : dist;
}

__device__ double sgn(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); }

__device__ double cross3(double o0, double o1, double a0, double a1, double b0, double b1) {
	return (a0 - o0) * (b1 - o1) - (a1 - o1) * (b0 - o0);
}

// Segment p-q meets an edge of the polygon (touching counts).
__device__ bool polygon_hits(const Scene &S, int o, const double *p, const double *q) {
	const int nv = S.onv[o];
	for (int k = 0; k < nv; ++k) {
		const double a0 = S.ov[o][k][0], a1 = S.ov[o][k][1];
		const double b0 = S.ov[o][(k + 1) % nv][0], b1 = S.ov[o][(k + 1) % nv][1];
		const double d1 = cross3(a0, a1, b0, b1, p[0], p[1]), d2 = cross3(a0, a1, b0, b1, q[0], q[1]);
		const double d3 = cross3(p[0], p[1], q[0], q[1], a0, a1), d4 = cross3(p[0], p[1], q[0], q[1], b0, b1);
		if (sgn(d1) * sgn(d2) <= 0 && sgn(d3) * sgn(d4) <= 0 && fmin(p[0], q[0]) <= fmax(a0, b0) &&
		    fmax(p[0], q[0]) >= fmin(a0, b0) && fmin(p[1], q[1]) <= fmax(a1, b1) && fmax(p[1], q[1]) >= fmin(a1, b1))
			return true;
	}
	return false;
}

__device__ double signed_distance(const Scene &S, int o, const double *x) {
	if (S.oshape[o] == 2) return polygon_distance(S, o, x);
	if (S.oshape[o] == 0) {
		double s = 0.0;
		for (int d = 0; d < S.D; ++d) {
			const double y = x[d] - S.oc[o][d];
			s += y * y;
		}
		return sqrt(s) - S.oa[o][0];
	}
	double y[3];
	for (int d = 0; d < S.D; ++d) y[d] = x[d] - S.oc[o][d];
	if (S.D == 2 && (S.ocs[o] != 1.0 || S.osn[o] != 0.0)) {
		const double y0 = S.ocs[o] * y[0] + S.osn[o] * y[1];
		const double y1 = -S.osn[o] * y[0] + S.ocs[o] * y[1];
		y[0] = y0, y[1] = y1;
	}
	double s = 0.0, amin = S.oa[o][0];
	for (int d = 0; d < S.D; ++d) {
		const double q = y[d] / S.oa[o][d];
		s += q * q;
		if (S.oa[o][d] < amin) amin = S.oa[o][d];
	}
	return (sqrt(s) - 1.0) * amin;
}

// The object's frame, scaled so that its surface is the unit sphere.
__device__ void unit_frame(const Scene &S, int o, const double *x, double *y) {
	for (int d = 0; d < S.D; ++d) y[d] = x[d] - S.oc[o][d];
	if (S.oshape[o] == 0) {
		for (int d = 0; d < S.D; ++d) y[d] = y[d] / S.oa[o][0];
		return;
	}
	if (S.D == 2 && (S.ocs[o] != 1.0 || S.osn[o] != 0.0)) {
		const double y0 = S.ocs[o] * y[0] + S.osn[o] * y[1];
		const double y1 = -S.osn[o] * y[0] + S.ocs[o] * y[1];
		y[0] = y0, y[1] = y1;
	}
	for (int d = 0; d < S.D; ++d) y[d] = y[d] / S.oa[o][d];
}

// Segment a-b meets the unit sphere: its nearest point to the origin is inside or on it and its
// farthest end outside or on it.
__device__ bool hits_unit(const double *a, const double *b, int D) {
	double ab[3], den = 0.0, dot = 0.0;
	for (int d = 0; d < D; ++d) ab[d] = b[d] - a[d];
	for (int d = 0; d < D; ++d) den += ab[d] * ab[d];
	for (int d = 0; d < D; ++d) dot += a[d] * ab[d];
	double t = -dot / (den > 0 ? den : 1.0);
	t        = fmin(fmax(t, 0.0), 1.0);
	double dmin = 0.0, da = 0.0, db = 0.0;
	for (int d = 0; d < D; ++d) {
		const double nr = a[d] + t * ab[d];
		dmin += nr * nr;
	}
	for (int d = 0; d < D; ++d) da += a[d] * a[d];
	for (int d = 0; d < D; ++d) db += b[d] * b[d];
	return dmin <= 1.0 && fmax(da, db) >= 1.0;
}

// Scene::raycast over the objects in order: an object without a condition ends the search.
__device__ bool raycast(const Scene &S, const double *a, const double *b) {
	for (int o = 0; o < S.n_obj; ++o) {
		if (!S.obc[o]) return false;
		if (S.oshape[o] == 2) {
			if (polygon_hits(S, o, a, b)) return true;
			continue;
		}
		double ya[3], yb[3];
		unit_frame(S, o, a, ya);
		unit_frame(S, o, b, yb);
		if (hits_unit(ya, yb, S.D)) return true;
	}
	return false;
}

// Domain::find: the node at level <= max_lv containing x (periodic wrap; 0 outside the box).
__device__ long long find(const Scene &S, const Arrays &A, const double *x0, int max_lv) {
	double x[3];
	for (int d = 0; d < S.D; ++d) {
		x[d] = x0[d];
		const bool lo = x[d] < -0.5 * S.active[d], hi = x[d] > 0.5 * S.active[d];
		if (lo || hi) {
			if (!S.periodic[d]) return 0;
			if (lo) x[d] += S.active[d];
			else x[d] -= S.active[d];
		}
	}
	long long i = 1;
	while (!(A.flags[i] & dg::F_LEAF) && A.level[i] < max_lv) {
		int bits = 0;
		for (int d = 0; d < S.D; ++d) bits |= (x[d] > A.center[i * S.D + d] ? 1 : 0) << d;
		i = A.children[i * S.C + bits];
	}
	return i;
}

__device__ void load_center(const Scene &S, const Arrays &A, long long i, double *x) {
	x[0] = x[1] = x[2] = 0.0;
	for (int d = 0; d < S.D; ++d) x[d] = A.center[i * S.D + d];
}

// Object-face test of node i's faces that carry no boundary yet; returns whether one was marked.
__device__ bool mark_object_faces(const Scene &S, const Arrays &A, long long i) {
	double x[3];
	load_center(S, A, i, x);
	const double size = A.size[i];
	const bool me     = active_node(A, i);
	bool hit_any      = false;
	for (int d = 0; d < S.D; ++d)
		for (int dir = 0; dir < 2; ++dir) {
			const int f = 2 * d + dir;
			if (A.bc[i * S.NF + f] != -1) continue;
			double nc[3] = {x[0], x[1], x[2]};
			nc[d] += (2.0 * dir - 1.0) * size;
			const long long nb = find(S, A, nc, A.level[i]);
			if (active_node(A, nb) != me || raycast(S, x, nc)) {
				A.bc[i * S.NF + f] = BC_MARK;
				hit_any           = true;
			}
		}
	return hit_any;
}

// Pass 1 of a level: distances, activity, domain-face boundaries.
__global__ void k_distance(Scene S, Arrays A, long long f0, long long n) {
	for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long) gridDim.x * blockDim.x) {
		const long long i = f0 + t;
		double x[3];
		load_center(S, A, i, x);
		const double size = A.size[i];
		double sd         = DMAX;
		int mesh          = 0;
		for (int o = 0; o < S.n_obj; ++o) {
			const double dist = signed_distance(S, o, x);
			if (dist < sd) sd = dist, mesh = o;
		}
		A.sd[i]   = sd;
		A.mesh[i] = mesh;
		if (S.n_obj > 0) {
			const bool inside = sd < 0.0 && S.obc[mesh];
			A.flags[i]        = inside ? (A.flags[i] & ~dg::F_ACTIVE) : (A.flags[i] | dg::F_ACTIVE);
		}
		for (int d = 0; d < S.D; ++d)
			for (int dir = 0; dir < 2; ++dir) {
				const double s  = 2.0 * dir - 1.0;
				const double nc = x[d] + s * size;
				int b           = -1;
				if (S.dbc[d][dir] >= 0 && nc * s > S.active[d] / 2.0) b = S.dbc[d][dir];
				A.bc[i * S.NF + 2 * d + dir] = b;
			}
		A.aux[i] = 0;
	}
}

// Pass 2 (scenes with walls): object faces; aux bit 0 = object face, bit 1 = no open face.
__global__ void k_faces(Scene S, Arrays A, long long f0, long long n) {
	for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long) gridDim.x * blockDim.x) {
		const long long i = f0 + t;
		const bool hit    = mark_object_faces(S, A, i);
		bool open         = false;
		for (int f = 0; f < S.NF; ++f) open = open || A.bc[i * S.NF + f] == -1;
		A.aux[i] = (uint8_t) ((hit ? 1 : 0) | (open ? 0 : 2));
	}
}

// The nearest object with a condition (Scene::nearest_boundary's choice), by |signed distance|.
__device__ int nearest_wall(const Scene &S, const double *x) {
	double best = INFINITY;
	int which   = -1;
	for (int o = 0; o < S.n_obj; ++o) {
		if (!S.obc[o]) continue;
		const double dist = fabs(signed_distance(S, o, x));
		if (dist < best) best = dist, which = o;
	}
	return which;
}

// Pass 3: split decision (scene.cpp:150-216) after the face pass.
__global__ void k_decide(Scene S, Arrays A, long long f0, long long n, int *split) {
	for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long) gridDim.x * blockDim.x) {
		const long long i = f0 + t;
		double x[3];
		load_center(S, A, i, x);
		const double size = A.size[i];
		const int lvl     = A.level[i];
		const double sd   = A.sd[i];
		uint32_t fl       = A.flags[i];
		const int aux     = A.aux[i];
		if (aux & 2) fl &= ~dg::F_ACTIVE;
		if (aux & 1) A.isb[i] = 1;
		bool cu = (fl & dg::F_CAN_UNSPLIT) != 0;
		if (aux & 1) cu = false;
		bool sp = false;
		if (lvl < S.min_level) sp = true, cu = false;
		if (S.n_obj > 0 && fabs(sd) < size * S.radius) {
			if (S.otype[A.mesh[i]] == 2) {
				if (lvl < S.max_level_geom) sp = true, cu = false;
			} else if (lvl < S.max_level) {
				sp = true, cu = true;
			}
		}
		bool inflow_r_face = false;
		for (int d = 0; d < S.D; ++d)
			for (int dir = 0; dir < 2; ++dir) {
				const int b = A.bc[i * S.NF + 2 * d + dir];
				if (b >= 0 && S.inflow_r[d][dir]) inflow_r_face = true;
				if (b == BC_MARK) {
					const int w = nearest_wall(S, x);
					if (w >= 0 && S.obc_inflow_r[w]) inflow_r_face = true;
				}
			}
		if (inflow_r_face && lvl < S.max_level) sp = true, cu = true;
		if (S.refine_jump && fabs(x[S.jump_axis] - S.jump_loc) < size && lvl < S.max_level) sp = true, cu = true;
		for (int z = 0; z < S.n_zone; ++z) {
			bool in = true;
			for (int d = 0; d < 3; ++d) in = in && x[d] < S.zx1[z][d] && x[d] > S.zx0[z][d];
			if (in && lvl < S.zlevel[z]) sp = true;
		}
		fl = cu ? (fl | dg::F_CAN_UNSPLIT) : (fl & ~dg::F_CAN_UNSPLIT);
		A.flags[i] = fl;
		split[t]   = (sp && (fl & dg::F_LEAF)) ? 1 : 0;
	}
}

// Domain::split of the parents par(r) = list ? list[r] : f0 + r for the r with split[r] (or all r
// when split is null); offset[r] ranks them. With copy_bc the children take the parent's
// boundaries on shared faces, and the children are marked as new leaves of fix_boundary.
__global__ void k_children(Scene S, Arrays A, const int32_t *list, long long f0, long long n, const int *split,
                           const int *offset, long long first, int copy_bc) {
	for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long) gridDim.x * blockDim.x) {
		if (split && !split[t]) continue;
		const long long par = list ? (long long) list[t] : f0 + t;
		const long long k0  = first + (long long) (offset ? offset[t] : t) * S.C;
		const double psz    = A.size[par];
		const double q      = 0.25 * psz;
		for (int c = 0; c < S.C; ++c) {
			const long long k = k0 + c;
			A.parent[k]       = (int32_t) par;
			A.level[k]        = A.level[par] + 1;
			for (int d = 0; d < S.D; ++d) A.center[k * S.D + d] = A.center[par * S.D + d] + q * ((c >> d) & 1 ? 1.0 : -1.0);
			A.size[k]  = 0.5 * psz;
			A.flags[k] = dg::F_LEAF | dg::F_ACTIVE | dg::F_CAN_SPLIT | (A.flags[par] & dg::F_CAN_UNSPLIT);
			for (int d = 0; d < S.D; ++d)
				for (int dir = 0; dir < 2; ++dir)
					A.bc[k * S.NF + 2 * d + dir] =
					    (copy_bc && ((c >> d) & 1) == dir) ? A.bc[par * S.NF + 2 * d + dir] : -1;
			for (int cc = 0; cc < S.C; ++cc) A.children[k * S.C + cc] = 0;
			A.sd[k]                    = DMAX;
			A.mesh[k]                  = 0;
			A.isb[k]                   = 0;
			A.mark[k]                  = copy_bc ? 1 : 0;
			A.children[par * S.C + c] = (int32_t) k;
		}
		A.flags[par] &= ~(dg::F_LEAF | dg::F_SHOULD_SPLIT);
		A.mark[par] = 0;
	}
}

// fix_boundary, splitting pass: bit 1 of mark[j] for active leaves j coarser than an inactive leaf's
// same-level neighbour position (bit 0 marks the leaves this call created).
__global__ void k_fix_targets(Scene S, Arrays A, long long n) {
	for (long long i = 1 + (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		const uint32_t fl = A.flags[i];
		if (!(fl & dg::F_LEAF) || (fl & dg::F_ACTIVE)) continue;
		double x[3];
		load_center(S, A, i, x);
		for (int d = 0; d < S.D; ++d)
			for (int dir = 0; dir < 2; ++dir) {
				double nc[3] = {x[0], x[1], x[2]};
				nc[d] += (2.0 * dir - 1.0) * A.size[i];
				const long long nb = find(S, A, nc, A.level[i]);
				if (active_node(A, nb) && A.level[nb] < A.level[i]) A.mark[nb] = A.mark[nb] | 2;  // every writer sets the same bit
			}
	}
}

__global__ void k_flag_bit(const uint8_t *mark, long long n, uint8_t bit, uint8_t *out) {
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
		out[i] = (mark[i] & bit) ? 1 : 0;
}

__global__ void k_iota(int32_t *v, long long n) {
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x)
		v[i] = (int32_t) i;
}

// fix_boundary, new leaves: boundaries cleared and tested again (no domain-face branch, as there).
__global__ void k_new_leaf_faces(Scene S, Arrays A, long long n) {
	for (long long i = 1 + (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		if (!(A.mark[i] & 1) || !(A.flags[i] & dg::F_LEAF)) continue;
		for (int f = 0; f < S.NF; ++f) A.bc[i * S.NF + f] = -1;
	}
}
__global__ void k_new_leaf_faces2(Scene S, Arrays A, long long n) {
	for (long long i = 1 + (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		if (!(A.mark[i] & 1) || !(A.flags[i] & dg::F_LEAF)) continue;
		mark_object_faces(S, A, i);
	}
}

// fix_boundary, last pass: boundaries of active leaves whose neighbour has none on the opposite face.
__global__ void k_drop_find(Scene S, Arrays A, long long n, uint8_t *drop) {
	// every node, the null slot included, writes its flags: the apply pass reads all n * 2D of them
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		const uint32_t fl = A.flags[i];
		for (int f = 0; f < S.NF; ++f) drop[i * S.NF + f] = 0;
		if (!(fl & dg::F_LEAF) || !(fl & dg::F_ACTIVE)) continue;
		double x[3];
		load_center(S, A, i, x);
		for (int d = 0; d < S.D; ++d)
			for (int dir = 0; dir < 2; ++dir) {
				const int f = 2 * d + dir;
				if (A.bc[i * S.NF + f] == -1) continue;
				double nc[3] = {x[0], x[1], x[2]};
				nc[d] += (2.0 * dir - 1.0) * A.size[i];
				const long long nb = find(S, A, nc, A.level[i]);
				if (nb != 0 && A.bc[nb * S.NF + (f ^ 1)] == -1) drop[i * S.NF + f] = 1;
			}
	}
}
__global__ void k_drop_apply(Arrays A, long long total, const uint8_t *drop, int *changed) {
	for (long long k = (long long) blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long) gridDim.x * blockDim.x)
		if (drop[k]) {
			A.bc[k] = -1;
			*changed = 1;
		}
}

// Distances of nodes created by fix_boundary, for the interface initialisation.
__global__ void k_fresh_sd(Scene S, Arrays A, long long n) {
	for (long long i = 1 + (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		if (A.sd[i] != DMAX) continue;
		double x[3];
		load_center(S, A, i, x);
		for (int o = 0; o < S.n_obj; ++o) {
			const double dist = signed_distance(S, o, x);
			if (dist < A.sd[i]) A.sd[i] = dist, A.mesh[i] = o;
		}
	}
}

// Active box, boundary flag, initial condition and interface of every node [0, n) (slot 0: no flags).
__global__ void k_finish(Scene S, Arrays A, long long n) {
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		uint32_t fl = A.flags[i];
		double x[3];
		load_center(S, A, i, x);
		bool outside = false;
		for (int d = 0; d < S.D; ++d) outside = outside || x[d] > 0.5 * S.active[d] || x[d] < -0.5 * S.active[d];
		if (outside) fl &= ~dg::F_ACTIVE;
		if (i > 0 && A.isb[i]) fl |= dg::F_IS_BOUNDARY;
		A.flags[i] = fl;
		double *p  = A.p + i * S.E;
		for (int q = 0; q < S.E; ++q) p[q] = 0.0;
		if (!((fl & dg::F_LEAF) && (fl & dg::F_ACTIVE))) continue;
		const double *v = (S.ic_kind == 1 && x[S.ic_axis] > S.ic_loc) ? S.ic_pos : S.ic_neg;
		for (int q = 0; q < S.E; ++q) p[q] = v[q];
		if (!(S.multi && S.D > 1 && S.n_obj > 0)) continue;
		// Scene::init_interface (scene.cpp:343-365); solids keep the initial condition
		double sd      = A.sd[i];
		const int type = S.otype[A.mesh[i]];
		if (type == 2) continue;
		double alpha = 0.0;
		if (type == 0) {
			alpha = sd < 0 ? 1.0 : 0.0;
		} else {
			alpha = sd > 0 ? 1.0 : 0.0;
			sd    = -sd;
		}
		if (S.diffuse && fabs(sd) < A.size[i] * S.radius) alpha = 0.5 * (1.0 - tanh(sd / S.h_finest));
		double air = S.rho2;
		if (S.keep_gas) {
			const double a0 = p[S.ia];
			air             = p[1] / (a0 < 1.0 ? 1.0 - a0 : 1.0);
			if (!(air > 0)) air = S.rho2;
		}
		p[0]    = S.rho1 * alpha;
		p[1]    = air * (1.0 - alpha);
		p[S.ia] = alpha;
	}
}

int grid_of(long long n) {
	long long b = (n + TPB - 1) / TPB;
	return (int) (b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

int fail(int code, const std::string &m) {
	g_err = m;
	return code;
}

#define B_CUDA(call)                                                                        \
	do {                                                                                    \
		cudaError_t e_ = (call);                                                            \
		if (e_ != cudaSuccess) return fail(DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
	} while (0)

}  // namespace

struct dg_tree {
	long long n = 0;
	int D = 0, E = 0, C = 0, NF = 0;
	std::vector<int32_t> parent, children, level, bc;
	std::vector<uint32_t> flags;
	std::vector<double> center, p;
};

namespace {

// Device arrays of the tree being built, grown by doubling; freed on scope exit.
struct DeviceTree {
	Arrays A{};
	long long cap = 0;
	~DeviceTree() {
		cudaFree(A.parent), cudaFree(A.children), cudaFree(A.level), cudaFree(A.bc), cudaFree(A.mesh);
		cudaFree(A.flags), cudaFree(A.center), cudaFree(A.size), cudaFree(A.sd), cudaFree(A.p);
		cudaFree(A.isb), cudaFree(A.aux), cudaFree(A.mark);
	}
};

// Scratch buffers, freed on scope exit.
struct Scratch {
	std::vector<void *> bufs;
	template<class T>
	cudaError_t get(T **p, size_t count) {
		cudaError_t e = cudaMalloc(p, sizeof(T) * (count > 0 ? count : 1));
		if (e == cudaSuccess) bufs.push_back(*p);
		return e;
	}
	~Scratch() {
		for (void *q : bufs) cudaFree(q);
	}
};

template<class T>
cudaError_t grow(T *&ptr, long long old_n, long long new_n, long long width) {
	T *fresh = nullptr;
	cudaError_t e = cudaMalloc(&fresh, sizeof(T) * new_n * width);
	if (e != cudaSuccess) return e;
	if (ptr) {
		e = cudaMemcpy(fresh, ptr, sizeof(T) * old_n * width, cudaMemcpyDeviceToDevice);
		cudaFree(ptr);
	}
	ptr = fresh;
	return e;
}

cudaError_t reserve(DeviceTree &T, const Scene &S, long long need) {
	if (need <= T.cap) return cudaSuccess;
	long long cap = T.cap ? T.cap : 1024;
	while (cap < need) cap *= 2;
	Arrays &A         = T.A;
	cudaError_t e     = cudaSuccess;
	const long long o = T.cap;
	if (e == cudaSuccess) e = grow(A.parent, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.children, o, cap, S.C);
	if (e == cudaSuccess) e = grow(A.level, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.bc, o, cap, S.NF);
	if (e == cudaSuccess) e = grow(A.mesh, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.flags, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.center, o, cap, S.D);
	if (e == cudaSuccess) e = grow(A.size, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.sd, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.p, o, cap, S.E);
	if (e == cudaSuccess) e = grow(A.isb, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.aux, o, cap, 1);
	if (e == cudaSuccess) e = grow(A.mark, o, cap, 1);
	T.cap = cap;
	return e;
}

// One Scene::fix_boundary call (scene.cpp:249-337).
int fix_boundary(const Scene &S, DeviceTree &T, long long &n) {
	Arrays &A = T.A;
	B_CUDA(cudaMemset(A.mark, 0, T.cap));
	while (true) {
		k_fix_targets<<<grid_of(n), TPB>>>(S, A, n);
		B_CUDA(cudaGetLastError());
		// targets in ascending node order
		Scratch sc;
		uint8_t *flag = nullptr;
		int32_t *iota = nullptr, *sel = nullptr;
		int *n_sel    = nullptr;
		B_CUDA(sc.get(&flag, n));
		B_CUDA(sc.get(&iota, n));
		B_CUDA(sc.get(&sel, n));
		B_CUDA(sc.get(&n_sel, 1));
		k_flag_bit<<<grid_of(n), TPB>>>(A.mark, n, 2, flag);
		k_iota<<<grid_of(n), TPB>>>(iota, n);
		size_t tb = 0;
		void *tmp = nullptr;
		B_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, iota, flag, sel, n_sel, (int) n));
		B_CUDA(sc.get((char **) &tmp, tb));
		B_CUDA(cub::DeviceSelect::Flagged(tmp, tb, iota, flag, sel, n_sel, (int) n));
		int cnt = 0;
		B_CUDA(cudaMemcpy(&cnt, n_sel, sizeof(int), cudaMemcpyDeviceToHost));
		if (cnt == 0) break;
		const long long kids = (long long) cnt * S.C;
		if (n + kids > 0x7fffffffLL) return fail(DG_ERR_CAPACITY, "dg_build_tree: more than 2^31 nodes");
		B_CUDA(reserve(T, S, n + kids));
		// targets lose bit 2 below (mark[par] = 0); children become new leaves (bit 0)
		k_children<<<grid_of(cnt), TPB>>>(S, T.A, sel, 0, cnt, nullptr, nullptr, n, 1);
		B_CUDA(cudaGetLastError());
		n += kids;
	}
	k_new_leaf_faces<<<grid_of(n), TPB>>>(S, A, n);
	k_new_leaf_faces2<<<grid_of(n), TPB>>>(S, A, n);
	B_CUDA(cudaGetLastError());
	Scratch sc;
	uint8_t *drop = nullptr;
	int *changed  = nullptr;
	B_CUDA(sc.get(&drop, (size_t) n * S.NF));
	B_CUDA(sc.get(&changed, 1));
	while (true) {
		B_CUDA(cudaMemset(changed, 0, sizeof(int)));
		k_drop_find<<<grid_of(n), TPB>>>(S, A, n, drop);
		k_drop_apply<<<grid_of(n * S.NF), TPB>>>(A, n * S.NF, drop, changed);
		B_CUDA(cudaGetLastError());
		int c = 0;
		B_CUDA(cudaMemcpy(&c, changed, sizeof(int), cudaMemcpyDeviceToHost));
		if (!c) break;
	}
	return DG_OK;
}

}  // namespace

extern "C" {

const char *dg_build_last_error(void) { return g_err.c_str(); }

int dg_build_tree(const dg_scene *in, dg_tree **out) {
	if (!in || !out) return fail(DG_ERR_ARG, "dg_build_tree: null argument");
	if (in->dims < 1 || in->dims > 3) return fail(DG_ERR_ARG, "dg_build_tree: dims must be 1, 2 or 3");
	if (in->n_objects > MAX_OBJ || in->n_zones > MAX_ZONE) return fail(DG_ERR_ARG, "dg_build_tree: too many objects or zones");
	Scene S{};
	S.D = in->dims, S.C = 1 << S.D, S.NF = 2 * S.D;
	S.multi = in->model == 2;
	S.E     = S.multi ? S.D + 4 : S.D + 2;
	S.ia    = S.E - 1;
	S.side  = in->side_length;
	for (int d = 0; d < 3; ++d) S.active[d] = in->active_size[d], S.periodic[d] = 0;
	S.min_level = in->min_level, S.max_level = in->max_level, S.max_level_geom = in->max_level_geom;
	S.radius = in->refinement_radius;
	for (int d = 0; d < 3; ++d)
		for (int k = 0; k < 2; ++k) S.dbc[d][k] = in->domain_bc[d][k], S.inflow_r[d][k] = in->inflow_r[d][k];
	for (int d = 0; d < S.D; ++d) S.periodic[d] = in->domain_bc[d][0] < 0 ? 1 : 0;
	S.n_obj = in->n_objects;
	S.walls = 0;
	for (int o = 0; o < S.n_obj; ++o) {
		const double *ob = in->objects + OBJ_ROW * o;
		for (int d = 0; d < 3; ++d) S.oc[o][d] = ob[d], S.oa[o][d] = ob[3 + d];
		S.ocs[o] = ob[6], S.osn[o] = ob[7];
		S.oshape[o] = (int) ob[8], S.otype[o] = (int) ob[9], S.obc[o] = (int) ob[10], S.obc_inflow_r[o] = (int) ob[11];
		S.onv[o] = (int) ob[12];
		if (S.oshape[o] == 2 && (S.D != 2 || S.onv[o] < 3 || S.onv[o] > MAX_VERT))
			return fail(DG_ERR_ARG, "dg_build_tree: polygons are 2D with 3 to 8 vertices");
		for (int k = 0; k < MAX_VERT; ++k) S.ov[o][k][0] = ob[13 + 2 * k], S.ov[o][k][1] = ob[14 + 2 * k];
		if (S.otype[o] < 0 || S.otype[o] > 2) return fail(DG_ERR_ARG, "dg_build_tree: object type must be 0, 1 or 2");
		if (S.obc[o]) S.walls = 1;
	}
	S.n_zone = in->n_zones;
	for (int z = 0; z < S.n_zone; ++z) {
		const double *zz = in->zones + 7 * z;
		for (int d = 0; d < 3; ++d) S.zx0[z][d] = zz[d], S.zx1[z][d] = zz[3 + d];
		S.zlevel[z] = (int) zz[6];
	}
	S.refine_jump = in->refine_jump, S.jump_axis = in->jump_axis, S.jump_loc = in->jump_location;
	S.ic_kind = in->ic_kind, S.ic_axis = in->ic_axis, S.ic_loc = in->ic_location;
	for (int q = 0; q < S.E; ++q) S.ic_neg[q] = in->ic_neg[q], S.ic_pos[q] = in->ic_kind == 1 ? in->ic_pos[q] : 0.0;
	S.diffuse = in->diffuse_ic, S.keep_gas = in->keep_ic_gas_density;
	S.rho1 = in->rho_ref[0], S.rho2 = in->rho_ref[1];
	S.h_finest = in->side_length / (double) (1LL << in->max_level);

	DeviceTree T;
	B_CUDA(reserve(T, S, 2));
	// slot 0: the null node (level -1); slot 1: the root (integrator/domain.hpp:40-62)
	{
		std::vector<int32_t> i0 = {0, 0}, l0 = {-1, 0};
		std::vector<uint32_t> f0 = {0u, dg::F_LEAF | dg::F_ACTIVE | dg::F_CAN_SPLIT};
		std::vector<double> c0(2 * S.D, 0.0), s0 = {0.0, S.side}, sd0 = {-1.0, 0.0};
		std::vector<int32_t> ch0(2 * S.C, 0), bc0(2 * S.NF, -1);
		std::vector<uint8_t> z0 = {0, 0};
		B_CUDA(cudaMemcpy(T.A.parent, i0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.level, l0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.mesh, i0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.flags, f0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.center, c0.data(), sizeof(double) * 2 * S.D, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.size, s0.data(), 16, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.sd, sd0.data(), 16, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.children, ch0.data(), sizeof(int32_t) * 2 * S.C, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.bc, bc0.data(), sizeof(int32_t) * 2 * S.NF, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.isb, z0.data(), 2, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.mark, z0.data(), 2, cudaMemcpyHostToDevice));
	}
	long long n = 2, f0 = 1, fn = 1;
	while (fn > 0) {
		Scratch sc;
		int *d_split = nullptr, *d_off = nullptr;
		B_CUDA(sc.get(&d_split, fn + 1));
		B_CUDA(sc.get(&d_off, fn + 1));
		size_t tb = 0;
		void *tmp = nullptr;
		B_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_split, d_off, (int) (fn + 1)));
		B_CUDA(sc.get((char **) &tmp, tb));
		k_distance<<<grid_of(fn), TPB>>>(S, T.A, f0, fn);
		if (S.walls) k_faces<<<grid_of(fn), TPB>>>(S, T.A, f0, fn);
		k_decide<<<grid_of(fn), TPB>>>(S, T.A, f0, fn, d_split);
		B_CUDA(cudaGetLastError());
		B_CUDA(cudaMemset(d_split + fn, 0, sizeof(int)));
		B_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, d_split, d_off, (int) (fn + 1)));
		int n_split = 0;
		B_CUDA(cudaMemcpy(&n_split, d_off + fn, sizeof(int), cudaMemcpyDeviceToHost));
		if (n_split == 0) break;
		const long long kids = (long long) n_split * S.C;
		if (n + kids > 0x7fffffffLL) return fail(DG_ERR_CAPACITY, "dg_build_tree: more than 2^31 nodes");
		B_CUDA(reserve(T, S, n + kids));
		k_children<<<grid_of(fn), TPB>>>(S, T.A, nullptr, f0, fn, d_split, d_off, n, 0);
		B_CUDA(cudaGetLastError());
		f0 = n, fn = kids, n += kids;
	}
	if (S.walls) {
		for (int k = 0; k < 10; ++k) {  // init_domain calls fix_boundary ten times (scene.cpp:401-402)
			const int rc = fix_boundary(S, T, n);
			if (rc != DG_OK) return rc;
		}
		k_fresh_sd<<<grid_of(n), TPB>>>(S, T.A, n);
	}
	k_finish<<<grid_of(n), TPB>>>(S, T.A, n);
	B_CUDA(cudaGetLastError());
	B_CUDA(cudaDeviceSynchronize());

	dg_tree *t = new dg_tree();
	t->n = n, t->D = S.D, t->E = S.E, t->C = S.C, t->NF = S.NF;
	t->parent.resize(n), t->children.resize(n * S.C), t->level.resize(n), t->bc.resize(n * S.NF);
	t->flags.resize(n), t->center.resize(n * S.D), t->p.resize(n * S.E);
	cudaError_t e = cudaSuccess;
	auto get      = [&](void *dst, const void *src, size_t bytes) {
        if (e == cudaSuccess) e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
	};
	get(t->parent.data(), T.A.parent, sizeof(int32_t) * n);
	get(t->children.data(), T.A.children, sizeof(int32_t) * n * S.C);
	get(t->level.data(), T.A.level, sizeof(int32_t) * n);
	get(t->bc.data(), T.A.bc, sizeof(int32_t) * n * S.NF);
	get(t->flags.data(), T.A.flags, sizeof(uint32_t) * n);
	get(t->center.data(), T.A.center, sizeof(double) * n * S.D);
	get(t->p.data(), T.A.p, sizeof(double) * n * S.E);
	if (e != cudaSuccess) {
		delete t;
		return fail(DG_ERR_CUDA, std::string("dg_build_tree: ") + cudaGetErrorString(e));
	}
	t->flags[0] = 0;
	*out        = t;
	return DG_OK;
}

int dg_tree_nodes(const dg_tree *t, long long *n) {
	if (!t || !n) return DG_ERR_ARG;
	*n = t->n;
	return DG_OK;
}

int dg_tree_copy(const dg_tree *t, int *parent, int *children, int *level, unsigned int *flags, int *bc,
                 double *center, double *p) {
	if (!t || !parent || !children || !level || !flags || !bc || !center || !p) return DG_ERR_ARG;
	std::copy(t->parent.begin(), t->parent.end(), parent);
	std::copy(t->children.begin(), t->children.end(), children);
	std::copy(t->level.begin(), t->level.end(), level);
	std::copy(t->flags.begin(), t->flags.end(), flags);
	std::copy(t->bc.begin(), t->bc.end(), bc);
	std::copy(t->center.begin(), t->center.end(), center);
	std::copy(t->p.begin(), t->p.end(), p);
	return DG_OK;
}

int dg_tree_free(dg_tree *t) {
	delete t;
	return DG_OK;
}

}  // extern "C"
