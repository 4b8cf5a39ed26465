// Node-pool access helpers: neighbour search, recursive child averages, boundary ghost states.
#pragma once

#include "model.cuh"

namespace dg {

__device__ __forceinline__ double at(const double *a, int cap, int c, int i) { return a[(size_t) c * cap + i]; }
__device__ __forceinline__ bool is_leaf(const Pool &P, int i) { return P.flags[i] & F_LEAF; }
__device__ __forceinline__ bool is_active(const Pool &P, int i) { return P.flags[i] & F_ACTIVE; }

template<class M>
__device__ __forceinline__ void load_p(const Pool &P, int i, double *p) {
	for (int q = 0; q < M::E; ++q) p[q] = at(P.p, P.cap, q, i);
}

__device__ __forceinline__ void set_status(uint32_t *status, uint32_t bit) { atomicOr(status, bit); }

// Domain::find(location, node.tree_level) for the face (dim, dir) of node i, as used by
// update_neighbors (integrator/domain.hpp:65-82, 249-293, 407-417). The location is the centre of
// the same-level neighbour; in integer cell coordinates the root-down descent becomes: step up to
// the common ancestor, then down towards the target until a leaf or the node's level. Returns 0 when
// the location lies outside the active box of a non-periodic dimension.
template<int D>
__device__ int find_neighbor(const Pool &P, const Consts &C, int i, int dim, int dir) {
	const int cap = P.cap;
	const int l   = P.level[i];
	int tc[3];
	for (int d = 0; d < D; ++d) tc[d] = P.coord[(size_t) d * cap + i];
	tc[dim] += 2 * dir - 1;
	const int lo = C.a0[l][dim], hi = C.a0[l][dim] + C.na[l][dim];
	if (tc[dim] < lo || tc[dim] >= hi) {
		if (!C.periodic[dim]) return 0;
		tc[dim] += (tc[dim] < lo) ? C.na[l][dim] : -C.na[l][dim];
	}
	const int own = P.coord[(size_t) dim * cap + i];
	int a = i, m = l;
	// ascend while the ancestor at level m does not contain the target along `dim`
	for (int guard = 0; guard < MAX_TREE && m > 0 && ((tc[dim] >> (l - m)) != (own >> (l - m))); ++guard) {
		a = P.parent[a];
		--m;
	}
	// descend towards the target
	for (int guard = 0; guard < MAX_TREE && !(P.flags[a] & F_LEAF) && m < l; ++guard) {
		int ci = 0;
		for (int d = 0; d < D; ++d) ci |= ((tc[d] >> (l - m - 1)) & 1) << d;
		a = P.child[(size_t) ci * cap + a];
		++m;
	}
	return a;
}

// Subtree means of non-leaf nodes. Domain::interpolate_p / interpolate_t (integrator/domain.hpp:
// 84-148) return, for a non-leaf node, the mean over its active children of the child's value (a
// leaf's own state, or recursively the child's mean). The pool keeps that mean for every non-leaf
// node in `avg` ({p[E], t}), refreshed bottom-up whenever a leaf below changes, so that a lookup is
// one record read instead of a walk over the subtree; the refresh adds the children in slot order
// from +0 and divides by their count, exactly as the recursion does.
template<class M>
struct Avg {
	static constexpr int W = (M::E + 1 + 1) & ~1;  // p[E], t, padded to 16 bytes
};

template<class M>
__device__ __forceinline__ void interp_p(const Pool &P, uint32_t *, int n, double *out) {
	if (P.flags[n] & F_LEAF) {
		load_p<M>(P, n, out);
		return;
	}
	const double *a = P.avg + (size_t) n * Avg<M>::W;
	for (int q = 0; q < M::E; ++q) out[q] = a[q];
}

template<class M>
__device__ __forceinline__ double interp_t(const Pool &P, int n) {
	if (P.flags[n] & F_LEAF) return P.t[n];
	return P.avg[(size_t) n * Avg<M>::W + M::E];
}

// Recomputes the subtree mean of non-leaf node n from its children (whose own means are current).
// Child means may have been written moments before by threads on other SMs, so they are read past
// the non-coherent L1.
template<class M>
__device__ __forceinline__ void refresh_avg(const Pool &P, int n) {
	constexpr int E = M::E, NC = 1 << M::D;
	double f[E + 1];
	for (int q = 0; q <= E; ++q) f[q] = 0.0;
	int cnt = 0;
	for (int c = 0; c < NC; ++c) {
		const int ch = P.child[(size_t) c * P.cap + n];
		const uint32_t fl = P.flags[ch];
		if (!(fl & F_ACTIVE)) continue;
		if (fl & F_LEAF) {
			for (int q = 0; q < E; ++q) f[q] = f[q] + at(P.p, P.cap, q, ch);
			f[E] = f[E] + P.t[ch];
		} else {
			const double *a = P.avg + (size_t) ch * Avg<M>::W;
			for (int q = 0; q <= E; ++q) f[q] = f[q] + __ldcg(a + q);
		}
		cnt++;
	}
	double *a = P.avg + (size_t) n * Avg<M>::W;
	for (int q = 0; q <= E; ++q) a[q] = f[q] / (double) cnt;
}

// Queues a node whose subtree changed and its ancestors for the next refresh. Every queued node counts
// its queued children in `pending`; a walk stops at the first ancestor that an earlier walk of the same
// refresh epoch queued (that walk went on to the root). `first` is the lowest node whose mean changed:
// the parent of a changed leaf, or a cell that has just been split.
__device__ __forceinline__ void mark_from(const Pool &P, int first, int epoch, int32_t *dirty, int *n_dirty, int cap,
                                          uint32_t *status) {
	int a = first;
	if (a == 0 || atomicExch(&P.mark[a], epoch) == epoch) return;
	for (int guard = 0; guard < MAX_TREE; ++guard) {
		const int pos = atomicAdd(n_dirty, 1);
		if (pos < cap) dirty[pos] = a;
		else atomicOr(status, ST_CAPACITY);
		const int b = P.parent[a];
		if (b == 0) return;
		atomicAdd(&P.pending[b], 1);
		if (atomicExch(&P.mark[b], epoch) == epoch) return;
		a = b;
	}
}

// Scalar field average (t, k[i] or p[i]); `arr` is the SoA base of that component.
template<int D>
__device__ double interp_scalar(const Pool &P, uint32_t *status, int n, const double *arr) {
	constexpr int NC = 1 << D;
	if (P.flags[n] & F_LEAF) return arr[n];
	int node[MAX_TREE], next[MAX_TREE], cnt[MAX_TREE];
	double f[MAX_TREE];
	int sp   = 1;
	node[0]  = n;
	next[0]  = 0;
	cnt[0]   = 0;
	f[0]     = 0.0;
	while (true) {
		const int k = sp - 1;
		if (next[k] < NC) {
			const int c = P.child[(size_t) next[k] * P.cap + node[k]];
			next[k]++;
			if (!(P.flags[c] & F_ACTIVE)) continue;
			if (P.flags[c] & F_LEAF) {
				f[k] += arr[c];
				cnt[k]++;
			} else if (sp < MAX_TREE) {
				node[sp] = c;
				next[sp] = 0;
				cnt[sp]  = 0;
				f[sp]    = 0.0;
				++sp;
			} else {
				set_status(status, ST_DEPTH);
			}
			continue;
		}
		const double r = f[k] / (double) cnt[k];
		--sp;
		if (sp == 0) return r;
		f[sp - 1] += r;
		cnt[sp - 1]++;
	}
}


// Boundary::boundary_value (integrator/boundary.hpp:75-123): ghost primitive state of a face.
template<class M>
__device__ void boundary_value(const ModelConsts &m, const BcTable &B, int b, const double *pc, double tc,
                               double *pb) {
	const int type = B.type[b];
	if (type == BC_FREESLIP) {
		const double *n = B.normal + (size_t) b * M::D;
		for (int q = 0; q < M::E; ++q) pb[q] = pc[q];
		double dot = 0.0;
		for (int i = 0; i < M::D; ++i) dot += pc[M::IU + i] * n[i];
		for (int i = 0; i < M::D; ++i) pb[M::IU + i] = pc[M::IU + i] - n[i] * dot;
		return;
	}
	if (type == BC_NOSLIP) {
		for (int q = 0; q < M::E; ++q) pb[q] = pc[q];
		for (int i = 0; i < M::D; ++i) pb[M::IU + i] *= -1.0;
		return;
	}
	if (type == BC_INFLOW || type == BC_INFLOW_R) {
		const double *pin = B.p_in + (size_t) b * M::E;
		for (int q = 0; q < M::E; ++q) pb[q] = pin[q];
		if (!supersonic<M>(m, pc)) pb[M::IP] = pc[M::IP];
		double fade = B.fade_in[b];
		if (fade > 0.0) {
			double vm = smin(tc / fade, 1.0);
			for (int i = 0; i < M::D; ++i) pb[M::IU + i] *= vm;
		}
		return;
	}
	if (type == BC_DIRICHLET) {
		const double *pin = B.p_in + (size_t) b * M::E;
		for (int q = 0; q < M::E; ++q) pb[q] = pin[q];
		return;
	}
	// outflow, zeroGradient (and the unused neumann)
	for (int q = 0; q < M::E; ++q) pb[q] = pc[q];
}

// Slope limiters (integrator/slope_limiters.hpp:7-57).
enum : int { LIM_MINMOD = 0, LIM_UNLIMITED, LIM_VAN_LEER, LIM_SUPERBEE, LIM_VON_ALBA_2, LIM_KOREN, LIM_FIRST_ORDER };

__device__ __forceinline__ double limit(int lim, double s1, double s2) {
	switch (lim) {
		case LIM_MINMOD:
			if (s1 * s2 <= 0.0) return 0.0;
			else if (fabs(s1) < fabs(s2)) return s1;
			else return s2;
		case LIM_UNLIMITED: return 0.5 * (s1 + s2);
		case LIM_VAN_LEER: {
			double r = s1 / s2;
			return (r + fabs(r)) / (1 + fabs(r)) * s2;
		}
		case LIM_SUPERBEE: {
			double r = s1 / s2;
			return smax(smax(0.0, smin(2.0 * r, 1.0)), smin(r, 2.0)) * s2;
		}
		case LIM_VON_ALBA_2: {
			double r = s1 / s2;
			return 2.0 * r / (r * r + 1) * s2;
		}
		case LIM_KOREN: {
			double r = (s1 + 1e-9) / (s2 + 1e-9);
			return smax(0.0, smin(2.0 * r, smin((1.0 + 2.0 * r) / 3.0, 2.))) * s2;
		}
		default: return 0.0;
	}
}

}  // namespace dg
