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

template<class M>
struct Rec {
	static constexpr int E = M::E, D = M::D;
	static constexpr int ES  = (E + 1) & ~1;  // slope row stride
	static constexpr int P0  = 0, R0 = E;     // p and rhs, adjacent (2E doubles)
	static constexpr int S0  = 2 * E;         // slope row d at S0 + d * ES
	static constexpr int K0  = S0 + D * ES;   // multiphase: curvature, then the normal's D components
	static constexpr int RAW = K0 + (M::MULTI ? 1 + D : 0);
	static constexpr int W   = (RAW + 1) & ~1;
};

__device__ __forceinline__ double *rec_of(const Pool &P, int i, int W) { return P.rec + (size_t) i * W; }

// Primitive state of node i from the head of its record: one or two 32-byte sectors instead of E
// scattered ones. The record's p equals the SoA p of every cell whenever another cell reads it
// (the update, split, unsplit and initialisation write both).
template<class M>
__device__ __forceinline__ void load_p_rec(const Pool &P, int i, double *p) {
	const double *r = P.rec + (size_t) i * Rec<M>::W;
	const double2 *r2 = reinterpret_cast<const double2 *>(r);
#pragma unroll
	for (int k = 0; k < M::E / 2; ++k) {
		const double2 v = r2[k];
		p[2 * k] = v.x, p[2 * k + 1] = v.y;
	}
	if constexpr (M::E % 2) p[M::E - 1] = r[M::E - 1];
}

template<class M>
__device__ __forceinline__ void store_p_rec(const Pool &P, int i, const double *p) {
	double *r   = P.rec + (size_t) i * Rec<M>::W;
	double2 *r2 = reinterpret_cast<double2 *>(r);
#pragma unroll
	for (int k = 0; k < M::E / 2; ++k) r2[k] = make_double2(p[2 * k], p[2 * k + 1]);
	if constexpr (M::E % 2) r[M::E - 1] = p[M::E - 1];
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
// leaf's own state, or recursively the child's mean). The walk below computes the same recursion
// (children in slot order, sums from +0, divided by the count), but memoises every non-leaf mean it
// forms in `avg` with the epoch of the computing kernel (`cst`), and reuses a memo instead of
// descending when no leaf below has changed since (`mod`, stamped upwards by every kernel that changes
// a leaf's state or the tree). A memo is only trusted when a previous kernel wrote it, so threads of
// one kernel never read each other's partial writes.
template<class M>
struct Avg {
	static constexpr int W = (M::E + 1 + 1) & ~1;  // p[E], t, padded to 16 bytes
};

__device__ __forceinline__ bool memo_ok(const Pool &P, int n, int epoch) {
	const int c = __ldcg(P.cst + n);
	return c > __ldcg(P.mod + n) && c < epoch;
}

// Mean primitive state and time of node n ({p[E], t} in out); `epoch` is the calling kernel's.
template<class M>
__device__ void interp_pt(const Pool &P, uint32_t *status, int n, int epoch, double *out) {
	constexpr int E = M::E, NC = 1 << M::D, AW = Avg<M>::W;
	if (P.flags[n] & F_LEAF) {
		load_p_rec<M>(P, n, out);
		out[E] = P.t[n];
		return;
	}
	if (memo_ok(P, n, epoch)) {
		for (int q = 0; q <= E; ++q) out[q] = __ldcg(P.avg + (size_t) n * AW + q);
		return;
	}
	struct Frame {
		int node, next, cnt;
		double f[E + 1];
	};
	Frame st[MAX_TREE];
	st[0].node = n;
	st[0].next = 0;
	st[0].cnt  = 0;
	for (int q = 0; q <= E; ++q) st[0].f[q] = 0.0;
	int sp = 1;
	while (true) {
		Frame &fr = st[sp - 1];
		if (fr.next < NC) {
			const int c = P.child[(size_t) fr.next * P.cap + fr.node];
			fr.next++;
			const uint32_t fl = P.flags[c];
			if (!(fl & F_ACTIVE)) continue;
			if (fl & F_LEAF) {
				double pc[E];
				load_p_rec<M>(P, c, pc);
				for (int q = 0; q < E; ++q) fr.f[q] = fr.f[q] + pc[q];
				fr.f[E] = fr.f[E] + P.t[c];
				fr.cnt++;
			} else if (memo_ok(P, c, epoch)) {
				for (int q = 0; q <= E; ++q) fr.f[q] = fr.f[q] + __ldcg(P.avg + (size_t) c * AW + q);
				fr.cnt++;
			} else if (sp < MAX_TREE) {
				Frame &nf = st[sp++];
				nf.node   = c;
				nf.next   = 0;
				nf.cnt    = 0;
				for (int q = 0; q <= E; ++q) nf.f[q] = 0.0;
			} else {
				set_status(status, ST_DEPTH);
			}
			continue;
		}
		double r[E + 1];
		for (int q = 0; q <= E; ++q) r[q] = fr.f[q] / (double) fr.cnt;
		double *memo = P.avg + (size_t) fr.node * AW;
		for (int q = 0; q <= E; ++q) memo[q] = r[q];
		P.cst[fr.node] = epoch;
		--sp;
		if (sp == 0) {
			for (int q = 0; q <= E; ++q) out[q] = r[q];
			return;
		}
		Frame &pf = st[sp - 1];
		for (int q = 0; q <= E; ++q) pf.f[q] = pf.f[q] + r[q];
		pf.cnt++;
	}
}

// Stamps a changed subtree: `first` (the parent of a changed leaf, or a cell that has just been
// split) and its ancestors get mod = epoch; a walk stops at the first ancestor already stamped in this
// epoch (that walk continues to the root).
__device__ __forceinline__ void mark_up(const Pool &P, int first, int epoch) {
	for (int a = first, guard = 0; a != 0 && guard < MAX_TREE; a = P.parent[a], ++guard) {
		if (__ldcg(P.mod + a) == epoch) break;
		P.mod[a] = epoch;
	}
}

// mark_up for a warp at once: lanes that name the same node leave it to one of them, so a node shared
// by many cells of the warp (their parent, grandparent, ...) is read and written once per warp instead
// of once per cell, and the cells of the first wave no longer all store to the same ancestors. The
// stamped set is mark_up's. Every lane of the warp calls it (first = 0 for a lane with nothing to stamp).
__device__ __forceinline__ void mark_up_warp(const Pool &P, int first, int epoch) {
	const int lane = threadIdx.x & 31;
	int a          = first;
	for (int guard = 0; guard < MAX_TREE; ++guard) {
		if (!__any_sync(0xffffffffu, a != 0)) break;
		const unsigned same = __match_any_sync(0xffffffffu, a);
		int next            = 0;
		if (a != 0 && __ffs(same) - 1 == lane && __ldcg(P.mod + a) != epoch) {
			P.mod[a] = epoch;
			next     = P.parent[a];
		}
		a = next;
	}
}

// Mean of a per-node scalar over the subtree of n (the leaf's own value for a leaf), children in slot
// order as the recursion of interpolate_k visits them; `val(x)` gives a leaf's value.
template<int D, class Val>
__device__ double interp_fn(const Pool &P, uint32_t *status, int n, Val val) {
	constexpr int NC = 1 << D;
	if (P.flags[n] & F_LEAF) return val(n);
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
				f[k] += val(c);
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

// The same recursion for the smoothed volume fraction, memoised like the primitive-state means but
// only for subtrees without a leaf changed in the running substep (mod below `e_upd`, the epoch of the
// substep's cell update): below those, the list's cells change from one Jacobi sweep to the next.
// e_upd = 0 disables the memo.
template<int D, class Val>
__device__ double interp_alpha(const Pool &P, uint32_t *status, int n, Val val, int epoch, int e_upd) {
	constexpr int NC = 1 << D;
	auto ok = [&](int x) {
		const int c = __ldcg(P.csta + x), m = __ldcg(P.mod + x);
		return c > m && c < epoch && m < e_upd;
	};
	if (P.flags[n] & F_LEAF) return val(n);
	if (ok(n)) return __ldcg(P.avga + n);
	int node[MAX_TREE], next[MAX_TREE], cnt[MAX_TREE];
	double f[MAX_TREE];
	int sp  = 1;
	node[0] = n;
	next[0] = 0;
	cnt[0]  = 0;
	f[0]    = 0.0;
	while (true) {
		const int k = sp - 1;
		if (next[k] < NC) {
			const int c = P.child[(size_t) next[k] * P.cap + node[k]];
			next[k]++;
			const uint32_t fl = P.flags[c];
			if (!(fl & F_ACTIVE)) continue;
			if (fl & F_LEAF) {
				f[k] += val(c);
				cnt[k]++;
			} else if (ok(c)) {
				f[k] += __ldcg(P.avga + c);
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
		if (__ldcg(P.mod + node[k]) < e_upd) {
			P.avga[node[k]] = r;
			P.csta[node[k]] = epoch;
		}
		--sp;
		if (sp == 0) return r;
		f[sp - 1] += r;
		cnt[sp - 1]++;
	}
}

// Scalar field average (t, k[i] or p[i]); `arr` is the SoA base of that component.
template<int D>
__device__ double interp_scalar(const Pool &P, uint32_t *status, int n, const double *arr) {
	return interp_fn<D>(P, status, n, [arr](int x) { return arr[x]; });
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
