// Initial tree on the device: Scene::init_domain (scene/scene.cpp:369-431) for scenes with analytic
// droplet/bubble objects, level by level as the host builder does it (dacti_b200/scene.py), so that
// both produce the same nodes in the same order:
//
//  - signed distances to the objects and the nearest object (scene.cpp:47-91), sphere |x - c| - r and
//    the ellipse measure (|R^T (x - c) / a| - 1) min(a);
//  - domain-face boundaries (scene.cpp:105-108);
//  - split detection (scene.cpp:150-216): below the minimum level, near an object, on an inflow_r face,
//    near the initial jump, inside a refinement zone (centre padded to 3D with zeros);
//  - Domain::split child placement (integrator/domain.hpp:206): parent.center + (0.25 parent.size)
//    quadrant(i); the r-th splitting node of a level gets children first + r C + c;
//  - leaves outside the active box inactive, uniform or jump initial condition, and the interface
//    initialisation with its tanh smear (scene.cpp:343-365).
//
// The frontier of every level is a contiguous index range, so a level costs one classification
// kernel, one exclusive scan of the split flags and one child-writing kernel.
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

struct Scene {
	int D, E, C, NF, multi, ia;
	double side, active[3];
	int min_level, max_level, max_level_geom;
	double radius;
	int dbc[3][2], inflow_r[3][2];
	int n_obj;
	double oc[MAX_OBJ][3], oa[MAX_OBJ][3], ocs[MAX_OBJ], osn[MAX_OBJ];
	int oshape[MAX_OBJ], otype[MAX_OBJ];  // shape 0 sphere, 1 ellipse; type 0 droplet, 1 bubble
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
};

thread_local std::string g_err;

__device__ double signed_distance(const Scene &S, int o, const double *x) {
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

// Classification of the frontier [f0, f0 + n): distances, domain boundaries, split decision.
__global__ void k_classify(Scene S, Arrays A, long long f0, long long n, int *split) {
	for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long) gridDim.x * blockDim.x) {
		const long long i = f0 + t;
		double x[3] = {0.0, 0.0, 0.0};
		for (int d = 0; d < S.D; ++d) x[d] = A.center[i * S.D + d];
		const double size = A.size[i];
		const int lvl     = A.level[i];
		double sd         = 1.7976931348623157e308;
		int mesh          = 0;
		for (int o = 0; o < S.n_obj; ++o) {
			const double dist = signed_distance(S, o, x);
			if (dist < sd) sd = dist, mesh = o;
		}
		A.sd[i]   = sd;
		A.mesh[i] = mesh;
		bool inflow_r_face = false;
		for (int d = 0; d < S.D; ++d)
			for (int dir = 0; dir < 2; ++dir) {
				const double s  = 2.0 * dir - 1.0;
				const double nc = x[d] + s * size;
				int b           = -1;
				if (S.dbc[d][dir] >= 0 && nc * s > S.active[d] / 2.0) b = S.dbc[d][dir];
				A.bc[i * S.NF + 2 * d + dir] = b;
				if (b >= 0 && S.inflow_r[d][dir]) inflow_r_face = true;
			}
		uint32_t fl = A.flags[i];
		bool cu     = (fl & dg::F_CAN_UNSPLIT) != 0;
		bool sp     = false;
		if (lvl < S.min_level) sp = true, cu = false;
		if (S.n_obj > 0 && fabs(sd) < size * S.radius && lvl < S.max_level) sp = true, cu = true;
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

__global__ void k_children(Scene S, Arrays A, long long f0, long long n, const int *split, const int *offset,
                           long long first) {
	for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long) gridDim.x * blockDim.x) {
		if (!split[t]) continue;
		const long long par = f0 + t;
		const long long k0  = first + (long long) offset[t] * S.C;
		const double psz    = A.size[par];
		const double q      = 0.25 * psz;
		for (int c = 0; c < S.C; ++c) {
			const long long k = k0 + c;
			A.parent[k]       = (int32_t) par;
			A.level[k]        = A.level[par] + 1;
			for (int d = 0; d < S.D; ++d) A.center[k * S.D + d] = A.center[par * S.D + d] + q * ((c >> d) & 1 ? 1.0 : -1.0);
			A.size[k]  = 0.5 * psz;
			A.flags[k] = dg::F_LEAF | dg::F_ACTIVE | dg::F_CAN_SPLIT | (A.flags[par] & dg::F_CAN_UNSPLIT);
			for (int f = 0; f < S.NF; ++f) A.bc[k * S.NF + f] = -1;
			for (int cc = 0; cc < S.C; ++cc) A.children[k * S.C + cc] = 0;
			A.sd[k]                    = 1.7976931348623157e308;
			A.mesh[k]                  = 0;
			A.children[par * S.C + c] = (int32_t) k;
		}
		A.flags[par] &= ~(dg::F_LEAF | dg::F_SHOULD_SPLIT);
	}
}

// Active box, initial condition and interface of every node [0, n) (slot 0 has no flags).
__global__ void k_finish(Scene S, Arrays A, long long n) {
	for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
		uint32_t fl = A.flags[i];
		double x[3] = {0.0, 0.0, 0.0};
		for (int d = 0; d < S.D; ++d) x[d] = A.center[i * S.D + d];
		bool outside = false;
		for (int d = 0; d < S.D; ++d) outside = outside || x[d] > 0.5 * S.active[d] || x[d] < -0.5 * S.active[d];
		if (outside) fl &= ~dg::F_ACTIVE;
		A.flags[i] = fl;
		double *p  = A.p + i * S.E;
		for (int q = 0; q < S.E; ++q) p[q] = 0.0;
		if (!((fl & dg::F_LEAF) && (fl & dg::F_ACTIVE))) continue;
		const double *v = (S.ic_kind == 1 && x[S.ic_axis] > S.ic_loc) ? S.ic_pos : S.ic_neg;
		for (int q = 0; q < S.E; ++q) p[q] = v[q];
		if (!(S.multi && S.D > 1 && S.n_obj > 0)) continue;
		// Scene::init_interface (scene.cpp:343-365)
		double sd       = A.sd[i];
		const int type  = S.otype[A.mesh[i]];
		double alpha    = 0.0;
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

struct DeviceTree {
	Arrays A{};
	long long cap = 0;
	std::vector<void *> owned;
	~DeviceTree() {
		for (void *q : owned) cudaFree(q);
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
	Arrays &A      = T.A;
	cudaError_t e  = cudaSuccess;
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
	T.cap = cap;
	return e;
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
	for (int d = 0; d < 3; ++d) S.active[d] = in->active_size[d];
	S.min_level = in->min_level, S.max_level = in->max_level, S.max_level_geom = in->max_level_geom;
	S.radius = in->refinement_radius;
	for (int d = 0; d < 3; ++d)
		for (int k = 0; k < 2; ++k) S.dbc[d][k] = in->domain_bc[d][k], S.inflow_r[d][k] = in->inflow_r[d][k];
	S.n_obj = in->n_objects;
	for (int o = 0; o < S.n_obj; ++o) {
		const double *ob = in->objects + 10 * o;
		for (int d = 0; d < 3; ++d) S.oc[o][d] = ob[d], S.oa[o][d] = ob[3 + d];
		S.ocs[o] = ob[6], S.osn[o] = ob[7];
		S.oshape[o] = (int) ob[8], S.otype[o] = (int) ob[9];
		if (S.otype[o] != 0 && S.otype[o] != 1) return fail(DG_ERR_UNSUPPORTED, "dg_build_tree: only droplet and bubble objects");
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
		B_CUDA(cudaMemcpy(T.A.parent, i0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.level, l0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.mesh, i0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.flags, f0.data(), 8, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.center, c0.data(), sizeof(double) * 2 * S.D, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.size, s0.data(), 16, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.sd, sd0.data(), 16, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.children, ch0.data(), sizeof(int32_t) * 2 * S.C, cudaMemcpyHostToDevice));
		B_CUDA(cudaMemcpy(T.A.bc, bc0.data(), sizeof(int32_t) * 2 * S.NF, cudaMemcpyHostToDevice));
	}
	long long n = 2, f0 = 1, fn = 1;
	int *d_split = nullptr, *d_off = nullptr;
	void *d_tmp  = nullptr;
	size_t tmp_bytes = 0;
	long long scratch_cap = 0;
	auto free_scratch = [&] {
		cudaFree(d_split), cudaFree(d_off), cudaFree(d_tmp);
		d_split = d_off = nullptr, d_tmp = nullptr;
	};
	while (fn > 0) {
		if (fn > scratch_cap) {
			free_scratch();
			scratch_cap = fn * 2;
			B_CUDA(cudaMalloc(&d_split, sizeof(int) * (scratch_cap + 1)));
			B_CUDA(cudaMalloc(&d_off, sizeof(int) * (scratch_cap + 1)));
			tmp_bytes = 0;
			B_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_split, d_off, (int) (scratch_cap + 1)));
			B_CUDA(cudaMalloc(&d_tmp, tmp_bytes));
		}
		k_classify<<<grid_of(fn), TPB>>>(S, T.A, f0, fn, d_split);
		B_CUDA(cudaGetLastError());
		B_CUDA(cudaMemset(d_split + fn, 0, sizeof(int)));
		B_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_split, d_off, (int) (fn + 1)));
		int n_split = 0;
		B_CUDA(cudaMemcpy(&n_split, d_off + fn, sizeof(int), cudaMemcpyDeviceToHost));
		if (n_split == 0) break;
		const long long kids = (long long) n_split * S.C;
		if (n + kids > 0x7fffffffLL) {
			free_scratch();
			return fail(DG_ERR_CAPACITY, "dg_build_tree: more than 2^31 nodes");
		}
		B_CUDA(reserve(T, S, n + kids));
		k_children<<<grid_of(fn), TPB>>>(S, T.A, f0, fn, d_split, d_off, n);
		B_CUDA(cudaGetLastError());
		f0 = n, fn = kids, n += kids;
	}
	free_scratch();
	k_finish<<<grid_of(n), TPB>>>(S, T.A, n);
	B_CUDA(cudaGetLastError());
	B_CUDA(cudaDeviceSynchronize());

	dg_tree *t = new dg_tree();
	t->n = n, t->D = S.D, t->E = S.E, t->C = S.C, t->NF = S.NF;
	t->parent.resize(n), t->children.resize(n * S.C), t->level.resize(n), t->bc.resize(n * S.NF);
	t->flags.resize(n), t->center.resize(n * S.D), t->p.resize(n * S.E);
	cudaError_t e = cudaSuccess;
	auto get = [&](void *dst, const void *src, size_t bytes) {
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
	*out = t;
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
