// Stage kernels of one ACTI-level substep (impl/integrate.hpp:26-67).
//
// Flux accumulation is free of floating-point atomics. Every face that carries a flux in a substep
// has one owner (impl/flux.hpp:58-59), which evaluates it once into its face-flux slot; each cell of
// the running cluster then sums the slots of its faces in a fixed order, and the cells of slower
// time levels that receive fluxes (the coarse side of the LTS coupling, impl/flux.hpp:82-91) are
// collected into a receiver list and gather the same way. The result is independent of list order
// and of scheduling, so runs are bitwise reproducible.
#pragma once

#include "tree.cuh"

namespace dg {

constexpr int BLOCK = 256;
// The face-sum and slope stages run 128-thread blocks of five resident blocks per SM: at the register
// count that allows (96), 20 warps per SM stay resident where 256-thread blocks at their natural count
// held 16 (measured 2-3% faster each on the whole step).
constexpr int FACE_THREADS = 128, FACE_MIN_BLOCKS = 5;
constexpr int SLOPE_THREADS = 128, SLOPE_MIN_BLOCKS = 5;

__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int gstride() { return gridDim.x * blockDim.x; }

// Thread index and grid stride of the grid-stride loops of the stage bodies: the launch's own grid, or
// (batched trees) the range of blocks a launch gives one tree.
struct PlainGrid {
	__device__ __forceinline__ int tid() const { return blockIdx.x * blockDim.x + threadIdx.x; }
	__device__ __forceinline__ int stride() const { return gridDim.x * blockDim.x; }
};
struct BlockRange {
	int first, count;  // blocks [first, first + count) of the launch
	__device__ __forceinline__ int tid() const { return ((int) blockIdx.x - first) * blockDim.x + threadIdx.x; }
	__device__ __forceinline__ int stride() const { return count * blockDim.x; }
};

__device__ __forceinline__ void append(int32_t *list, int *count, int value, int cap, uint32_t *status) {
	int pos = atomicAdd(count, 1);
	if (pos < cap) list[pos] = value;
	else set_status(status, ST_CAPACITY);
}

// --------------------------------------------------------------------------------------------
// Reconstruction records (Rec, declared with the tree helpers). Everything a face flux needs from one
// side, apart from centre and time, sits in one contiguous FP64 record per node: the primitive state (a
// copy of the pool's p, also what neighbour gathers read), the
// Hancock rhs, the limited slope rows (each padded to an even length so that rows start on 16-byte
// boundaries) and, for the multiphase model, the curvature and interface normal. A neighbour's
// face state is then a handful of 16-byte vector loads from a few cache lines instead of 3E + 2
// scattered structure-of-arrays loads. The record is the only storage of slope and rhs.
// --------------------------------------------------------------------------------------------

// Loads the face-dim part of node i's record, rounded to S: p, rhs, slope row `dim`, and (multiphase)
// curvature and normal component `dim`.
template<class M, class S>
__device__ __forceinline__ void load_face_rec(const Pool &P, int i, int dim, S *p, S *rhs, S *sl, S &kap, S &nrm) {
	using R = Rec<M>;
	constexpr int E = M::E;
	const double2 *r = reinterpret_cast<const double2 *>(rec_of(P, i, R::W));
	double a[2 * E];
#pragma unroll
	for (int k = 0; k < E; ++k) {
		const double2 v = __ldg(r + k);
		a[2 * k] = v.x, a[2 * k + 1] = v.y;
	}
#pragma unroll
	for (int q = 0; q < E; ++q) p[q] = (S) a[R::P0 + q], rhs[q] = (S) a[R::R0 + q];
	const double2 *sr = r + (R::S0 + dim * R::ES) / 2;
#pragma unroll
	for (int k = 0; k < R::ES / 2; ++k) {
		const double2 v = __ldg(sr + k);
		if (2 * k < E) sl[2 * k] = (S) v.x;
		if (2 * k + 1 < E) sl[2 * k + 1] = (S) v.y;
	}
	if constexpr (M::MULTI) {
		const double *kr = rec_of(P, i, R::W) + R::K0;
		kap = (S) __ldg(kr);
		nrm = (S) pick<0, M::D>(kr + 1, dim);
	}
}

// Slope component q along d of node i.
template<class M>
__device__ __forceinline__ double rec_slope(const Pool &P, int i, int d, int q) {
	return rec_of(P, i, Rec<M>::W)[Rec<M>::S0 + d * Rec<M>::ES + q];
}

// Multiphase k part of the record (curvature, normal) from the pool's parameters.
template<class M>
__device__ __forceinline__ void write_rec_k(const Pool &P, int i) {
	if constexpr (M::MULTI) {
		double *kr = rec_of(P, i, Rec<M>::W) + Rec<M>::K0;
		kr[0] = at(P.k, P.cap, M::KAPPA, i);
		for (int d = 0; d < M::D; ++d) kr[1 + d] = at(P.k, P.cap, M::IKN + d, i);
	}
}

template<class M, class Grid>
__device__ __forceinline__ void d_rec_k(const Grid &g, const Pool &P, const int32_t *list, int n) {
	for (int tid = g.tid(); tid < n; tid += g.stride()) write_rec_k<M>(P, list[tid]);
}
template<class M>
__global__ void k_rec_k(Pool P, const int32_t *list, int n) {
	d_rec_k<M>(PlainGrid{}, P, list, n);
}

// du[dim * G + DT] (temperature gradient along the face normal) for a run-time dim.
template<class M, class S>
__device__ __forceinline__ S pick_row_dt(const S *du, int dim) {
	S r = du[M::DT];
#pragma unroll
	for (int j = 1; j < M::D; ++j)
		if (dim == j) r = du[j * M::G + M::DT];
	return r;
}

// --------------------------------------------------------------------------------------------
// Interior face flux: Model::flux(left, right, face) with the face of the owning cell
// (impl/flux.hpp:32-39, 80-91; model/euler.hpp:156-200, navier_stokes.hpp:387-408,
// multi.hpp:249-302). `dir_o` is the owner's direction towards `other`; for dir_o == 0 the owner is
// the right state and the face keeps the owner's centre (the reference relabels face.dir = 1).
// Across a periodic wrap the non-owner's centre moves by the active size.
// --------------------------------------------------------------------------------------------
template<class M, bool V, class S>
__device__ __forceinline__ void interior_flux(const Pool &P, const Consts &C, int owner, int other, int dim, int dir_o,
                                              double dtL, double *Fout) {
	constexpr int E = M::E, D = M::D;
	const int cap   = P.cap;
	const int lo    = P.level[owner];
	const double so = C.size[lo];
	const double co = at(P.center, cap, dim, owner);
	const double fc = co + so * (dir_o - 0.5);
	const double t0 = P.t[owner];
	const double t1 = t0 + dtL;
	const double area = C.area[lo];

	double cx = at(P.center, cap, dim, other);
	if (C.periodic[dim]) {
		if (dir_o == 1) {
			if (co + so > 0.5 * C.active[dim]) cx += C.active[dim];
		} else {
			if (co - so < -0.5 * C.active[dim]) cx -= C.active[dim];
		}
	}
	const int iL = dir_o == 1 ? owner : other;
	const int iR = dir_o == 1 ? other : owner;
	const double cL = dir_o == 1 ? co : cx;
	const double cR = dir_o == 1 ? cx : co;

	S pl[E], hl[E], sl[E], pr[E], hr[E], sr[E], kl = 0, kr = 0, nl = 0, nr = 0;
	load_face_rec<M, S>(P, iL, dim, pl, hl, sl, kl, nl);
	load_face_rec<M, S>(P, iR, dim, pr, hr, sr, kr, nr);
	const double tm   = 0.5 * (t1 + t0);
	const double dt_n = tm - P.t[iL];
	const double dt_p = tm - P.t[iR];
	// Hancock predictor at the face (reconstruction); geometry and time offsets stay FP64
	const S xl = (S) (fc - cL), xr = (S) (fc - cR), tl = (S) dt_n, tr = (S) dt_p;
	S pn[E], pp[E];
	for (int q = 0; q < E; ++q) {
		S v   = pl[q] + sl[q] * xl;
		pn[q] = v - hl[q] * tl;
		S w   = pr[q] + sr[q] * xr;
		pp[q] = w - hr[q] * tr;
	}
	S ka = 0;
	if constexpr (M::MULTI) ka = (S) 0.5 * (kl + kr);
	S pm[E], F[M::F];
	middle_state<M, S>(C.m, pn, pp, ka, dim, pm);
	phys_flux<M, S>(C.m, pm, (S) 0, dim, false, F);
	const double dtf = t1 - t0;

	if constexpr (M::MULTI) {
		constexpr int IA = M::IA, IU = M::IU, IP = M::IP;
		const S a = pm[IA];
		if (a > (S) 1e-5 && a < 1 - (S) 1e-5) {
			S n  = (S) 0.5 * (nl + nr);
			S uc = (S) MULTI_UC * fabs(pick<IU, D>(pm, dim)) * n;
			S ke = 0;
			for (int i = 0; i < D; ++i) {
				F[IU + i] += uc * ((1 - a) * pm[0] - a * pm[1]) * pm[IU + i];
				ke += (S) 0.5 * pm[IU + i] * pm[IU + i];
			}
			F[0] += uc * (1 - a) * pm[0];
			F[1] += uc * (-a) * pm[1];
			const ModelConsts &m = C.m;
			const S g1 = (S) m.gamma1, g2 = (S) m.gamma2, P1 = (S) m.P1, P2 = (S) m.P2;
			F[IP] += uc * ((1 - a) * pm[0] - a * pm[1]) * ke +
			         uc * (1 - a) * a * (pm[IP] * (1 / (g1 - 1) - 1 / (g2 - 1)) + g1 * P1 / (g1 - 1) - g2 * P2 / (g2 - 1));
			F[IA] += uc * (1 - a) * a;
		}
	}
	if constexpr (M::VISC && V) {
		constexpr int G = M::G;
		S du[D * G], vel[D], fv[D + 1];
		for (int i = 0; i < D; ++i)
			for (int g = 0; g < G; ++g)
				du[i * G + g] = (S) 0.5 * ((S) at(P.grad, cap, i * G + g, iL) + (S) at(P.grad, cap, i * G + g, iR));
		for (int i = 0; i < D; ++i) vel[i] = (S) 0.5 * (pl[M::IU + i] + pr[M::IU + i]);
		if constexpr (M::MULTI) {
			// multi.hpp:287-301: viscous and heat terms enter before the area * dt scaling
			visc_flux<D, G, S>(du, vel, visc_mu<M, S>(C.m, pm), dim, fv);
			for (int i = 0; i <= D; ++i) F[M::IU + i] -= fv[i];
			F[M::IU + D] -= pick_row_dt<M, S>(du, dim) * visc_lambda<M, S>(C.m, pm);
			for (int q = 0; q < M::F; ++q) Fout[q] = (double) F[q] * area * dtf;
		} else {
			// navier_stokes.hpp:387-408: convective part scaled first, then scaled viscous/heat terms
			for (int q = 0; q < M::F; ++q) Fout[q] = (double) F[q] * area * dtf;
			visc_flux<D, G, S>(du, vel, (S) C.m.ns_mu, dim, fv);
			for (int i = 0; i <= D; ++i) Fout[M::IU + i] -= (double) fv[i] * area * dtf;
			const double fh = (double) ((S) C.m.ns_lambda * pick_row_dt<M, S>(du, dim)) * area * dtf;
			Fout[M::IU + D] -= fh;
		}
	} else {
		for (int q = 0; q < M::F; ++q) Fout[q] = (double) F[q] * area * dtf;
	}
}

// Boundary::boundary_flux (integrator/boundary.hpp:130-160), from the cell-centre state.
template<class M, bool V, class S>
__device__ __forceinline__ void boundary_flux(const Pool &P, const Consts &C, const BcTable &B, int i, int b, int dim,
                                              int dir, double dtL, double *Fout) {
	constexpr int E = M::E, D = M::D;
	const int cap = P.cap;
	double pcd[E], pbd[E];
	load_p<M>(P, i, pcd);
	const double t0 = P.t[i];
	const double t1 = t0 + dtL;
	boundary_value<M>(C.m, B, b, pcd, t0, pbd);
	S pc[E], pb[E], F[M::F];
	for (int q = 0; q < E; ++q) {
		pc[q] = (S) pcd[q];
		pb[q] = (S) pbd[q];
	}
	const int type = B.type[b];
	if (type == BC_FREESLIP) {
		phys_flux<M, S>(C.m, pc, pick<M::IU, D>(pb, dim), dim, true, F);
	} else if (type == BC_NOSLIP) {
		for (int q = 0; q < M::F; ++q) F[q] = 0;
		put<M::IU, D>(F, dim, pb[M::IP]);
	} else {
		S pm[E];
		middle_state<M, S>(C.m, pb, pc, (S) 0, dim, pm);
		phys_flux<M, S>(C.m, pm, (S) 0, dim, false, F);
	}
	if constexpr (M::VISC && V) {
		constexpr int G = M::G;
		S g[D * G], z[D], fv[D + 1];
		for (int c = 0; c < D * G; ++c) g[c] = (S) at(P.grad, cap, c, i);
		for (int d = 0; d < D; ++d) z[d] = 0;
		visc_flux<D, G, S>(g, z, visc_mu<M, S>(C.m, pc), dim, fv);
		for (int k = 0; k <= D; ++k) F[M::IU + k] -= fv[k];
	}
	const double area = C.area[P.level[i]];
	const double dirn = (double) (2 * dir - 1);
	for (int q = 0; q < M::F; ++q) Fout[q] = (double) F[q] * area * (t1 - t0) * dirn;
}

// The c-th owner of a flux across face (dim, dir) of cell i at this substep (impl/flux.hpp:58-59 seen
// from either side). c = 0: the cell itself (cluster_mode) or its same-level neighbour; c >= 1: the
// finer cells behind a non-leaf neighbour, adjacent child a and, when that child is split, its
// adjacent child b - 1 (c - 1 = a (2^(D-1) + 1) + b). Returns the owner or -1; `dn` is the owner's
// direction towards the other cell and `plus` whether cell i adds the flux.
template<class M>
__device__ __forceinline__ int face_owner(const Pool &P, uint32_t *status, int i, int nb, int dim, int dir, int L, int li,
                                          int ai, int c, bool cluster_mode, int &dn, bool &plus) {
	constexpr int NSUB = 1 << (M::D - 1);
	const int cap = P.cap;
	if (c == 0) {
		const uint32_t fn = P.flags[nb];
		if (!(fn & F_LEAF)) return -1;
		const int ln = P.level[nb], an = P.acti[nb];
		if (cluster_mode && an <= ai && (ln < li || (ln == li && (dir == 1 || an < ai)))) {
			dn   = dir;
			plus = dir == 0;
			return i;
		}
		if (ln == li && P.clu[nb] == L && ai <= an && ((1 - dir) == 1 || ai < an)) {
			dn   = 1 - dir;
			plus = dn == 1;
			return nb;
		}
		return -1;
	}
	dn   = 1 - dir;
	plus = dn == 1;
	const int k = c - 1, a = k / (NSUB + 1), b = k % (NSUB + 1);
	const int mask = (1 << dim) - 1;
	const int ca   = (a & mask) | (dn << dim) | ((a >> dim) << (dim + 1));
	const int ch   = P.child[(size_t) ca * cap + nb];
	if (ch == 0) return -1;  // left out by the host: an inactive leaf or subtree, which owns no flux
	const bool ch_leaf = P.flags[ch] & F_LEAF;
	if (b == 0) return (ch_leaf && P.clu[ch] == L && ai <= P.acti[ch]) ? ch : -1;
	if (ch_leaf) return -1;
	const int gb = b - 1;
	const int cg = (gb & mask) | (dn << dim) | ((gb >> dim) << (dim + 1));
	const int gc = P.child[(size_t) cg * cap + ch];
	if (gc == 0) return -1;
	if (!(P.flags[gc] & F_LEAF)) {
		set_status(status, ST_DEPTH);
		return -1;
	}
	return (P.clu[gc] == L && ai <= P.acti[gc]) ? gc : -1;
}

// Face-flux slot of face f of the cell at list position `slot`, written for owned faces next to a receiver. The slots hold FP64
// values in the FP64 form and FP32 values in the mixed form (T = float: the same array read with a
// compact FP32 stride).
template<class T = double>
__device__ __forceinline__ T *face_flux(const Pool &P, int slot, int f, int nflux, int nfaces) {
	return reinterpret_cast<T *>(P.ff) + ((size_t) slot * nfaces + f) * nflux;
}

// flux_update, receiving side: each queued receiver sums, in a fixed face order, the fluxes that
// running-cluster cells own across its faces. A group of 2D lanes (padded to 4 or 8) serves one
// cell; lane f walks the owners across face (dim, dir) = (f / 2, f % 2) and the lane sums are
// combined with a fixed butterfly, so the total does not depend on scheduling.
template<class M, class T = double, class Grid>
__device__ __forceinline__ void d_flux_receive(const Grid &g, const Pool &P, const int32_t *list, const int *n_ptr, int L, Counters *cnt) {
	constexpr int NF   = 2 * M::D;
	constexpr int G    = NF <= 4 ? 4 : 8;
	constexpr int GW   = 32 / G;
	constexpr int NSUB = 1 << (M::D - 1);
	const int n      = *n_ptr;
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int sub    = lane & (G - 1);
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot = wbase + lane / G;
		double acc[M::F];
#pragma unroll
		for (int q = 0; q < M::F; ++q) acc[q] = 0.0;
		if (slot < n && sub < NF) {
			const int i   = list[slot];
			const int dim = sub >> 1, dir = sub & 1;
			const int li = P.level[i], ai = P.acti[i];
			const int nb = P.nbr[(size_t) sub * cap + i];
			if (nb != 0) {
				const int ncand = (P.flags[nb] & F_LEAF) ? 1 : 1 + NSUB * (NSUB + 1);
				for (int c = 0; c < ncand; ++c) {
					int dn;
					bool plus;
					const int owner = face_owner<M>(P, &cnt->status, i, nb, dim, dir, L, li, ai, c, false, dn, plus);
					if (owner < 0) continue;
					const T *F = face_flux<T>(P, P.pos[owner], 2 * dim + dn, M::F, NF);
					if (plus) {
#pragma unroll
						for (int q = 0; q < M::F; ++q) acc[q] += F[q];
					} else {
#pragma unroll
						for (int q = 0; q < M::F; ++q) acc[q] -= F[q];
					}
				}
			}
		}
		// fixed-order butterfly over the group's lanes
#pragma unroll
		for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
			for (int q = 0; q < M::F; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
		if (slot < n) {
			const int i = list[slot];
#pragma unroll
			for (int q = 0; q < M::F; ++q)
				if ((q & (G - 1)) == sub) P.flux[(size_t) q * cap + i] += acc[q];
			if (sub == 0) atomicOr(&P.flags[i], (uint32_t) F_RECV);
		}
	}
}
template<class M, class T = double>
__global__ void __launch_bounds__(BLOCK) k_flux_receive(Pool P, const int32_t *list, const int *n_ptr, int L,
                                                        Counters *cnt) {
	d_flux_receive<M, T>(PlainGrid{}, P, list, n_ptr, L, cnt);
}

// flux_update (impl/flux.hpp:11-97) seen from each running-cluster cell: the signed sum of the fluxes
// that cross its faces in this substep, one lane per face (groups of 4 lanes in 2D, 8 cells a warp; of
// 6 lanes in 3D, 5 cells a warp, the warp's last two lanes idle). Lane f evaluates the flux across face f: the cell's own when it owns the face (the finer
// side, at equal levels the slower cell or the cell on the left), the same-level neighbour's when the
// neighbour owns it, the boundary flux, or the sum over the finer owners behind a non-leaf neighbour in
// candidate order. Every interior flux is evaluated with the owner's arguments (owner, the owner's
// neighbour, the owner's direction), so the two cells of a face obtain identical bits and the update
// stays conservative without a face-flux array or atomics. The lane terms combine in a fixed butterfly,
// ((f0 + f4) + (f2 + 0)) + ((f1 + f5) + (f3 + 0)) in 3D, into du[slot]. An owned face next to a cell of
// a slower cluster (the coarse-time side of the LTS coupling, impl/flux.hpp:82-91) also goes to the
// owner's face-flux slot, and that cell joins the receiver list. In the mixed form every flux is rounded
// to FP32 once, as both sides read it; sums stay FP64.
template<class M, bool V, class S = double, class Grid>
__device__ __forceinline__ void d_face_sum(const Grid &g, const Pool &P, const Consts &C, const BcTable &B, const int32_t *list, int n, int L, double dtL, int stamp, int32_t *recv, Counters *cnt) {
	constexpr int NF = 2 * M::D, G = NF, GW = 32 / G, NSUB = 1 << (M::D - 1), F = M::F;
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int grp    = lane / G;  // the lane's cell within the warp; lanes past GW * G idle
	const int sub    = lane - grp * G;
	const int base   = grp * G;
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot    = wbase + grp;
		const bool active = grp < GW && slot < n;
		double acc[F];
#pragma unroll
		for (int q = 0; q < F; ++q) acc[q] = 0.0;
		if (active) {
			const int i   = list[slot];
			if (sub == 0) P.pos[i] = slot;
			const int f   = sub, dim = f >> 1, dir = f & 1;
			const int nb  = P.nbr[(size_t) f * cap + i];
			if (nb == 0) {
				const int b = P.bc[(size_t) f * cap + i];
				if (b < 0) {
					set_status(&cnt->status, ST_MISSING_BC);
				} else {
					double Fb[F];
					boundary_flux<M, V, S>(P, C, B, i, b, dim, dir, dtL, Fb);
#pragma unroll
					for (int q = 0; q < F; ++q) acc[q] = 0.0 - (double) (S) Fb[q];
				}
			} else if (!(P.flags[nb] & F_LEAF)) {
				const int li = P.level[i], ai = P.acti[i];
				double w[F];
#pragma unroll
				for (int q = 0; q < F; ++q) w[q] = 0.0;
				for (int c = 1; c < 1 + NSUB * (NSUB + 1); ++c) {
					int dn;
					bool plus;
					const int owner = face_owner<M>(P, &cnt->status, i, nb, dim, dir, L, li, ai, c, true, dn, plus);
					if (owner < 0) continue;
					const int fo = 2 * dim + dn;
					double Fw[F];
					interior_flux<M, V, S>(P, C, owner, P.nbr[(size_t) fo * cap + owner], dim, dn, dtL, Fw);
					if (plus) {
#pragma unroll
						for (int q = 0; q < F; ++q) w[q] += (double) (S) Fw[q];
					} else {
#pragma unroll
						for (int q = 0; q < F; ++q) w[q] -= (double) (S) Fw[q];
					}
				}
#pragma unroll
				for (int q = 0; q < F; ++q) acc[q] = 0.0 + (double) (S) w[q];
			} else {
				const int li = P.level[i], ai = P.acti[i], ln = P.level[nb], an = P.acti[nb];
				int own = -1, fo = f;
				if (an <= ai && (ln < li || (ln == li && (dir == 1 || an < ai)))) {
					own = i;
				} else if (ln == li && P.clu[nb] == L && ai <= an && (dir == 0 || ai < an)) {
					own = nb;
					fo  = f ^ 1;
				}
				if (own >= 0) {
					const int other = own == i ? nb : P.nbr[(size_t) fo * cap + nb];
					double Fi[F];
					interior_flux<M, V, S>(P, C, own, other, dim, fo & 1, dtL, Fi);
					if (own == i && P.clu[nb] != L) {
						S *dst = face_flux<S>(P, slot, f, F, NF);
#pragma unroll
						for (int q = 0; q < F; ++q) dst[q] = (S) Fi[q];
						if (atomicExch(&P.stamp[nb], stamp) != stamp) append(recv, &cnt->n_recv, nb, cap, &cnt->status);
					}
#pragma unroll
					for (int q = 0; q < F; ++q) {
						const double v = (double) (S) Fi[q];
						acc[q] = dir ? 0.0 - v : 0.0 + v;
					}
				}
			}
		}
		// the group's face terms in the fixed pairing order, on every lane of the group
		double sum[F];
		if constexpr (NF == 4) {
			// (f0 + f2) + (f1 + f3): a butterfly over the aligned group of four
#pragma unroll
			for (int q = 0; q < F; ++q) {
				double v = acc[q] + __shfl_xor_sync(0xffffffffu, acc[q], 2);
				sum[q]   = v + __shfl_xor_sync(0xffffffffu, v, 1);
			}
		} else {
			// ((f0 + f4) + (f2 + 0)) + ((f1 + f5) + (f3 + 0))
#pragma unroll
			for (int q = 0; q < F; ++q) {
				double f[6];
#pragma unroll
				for (int k = 0; k < 6; ++k) f[k] = __shfl_sync(0xffffffffu, acc[q], min(base + k, 31));
				sum[q] = ((f[0] + f[4]) + (f[2] + 0.0)) + ((f[1] + f[5]) + (f[3] + 0.0));
			}
		}
		if (active) {
			double *dst = P.du + (size_t) slot * F;
#pragma unroll
			for (int q = 0; q < F; ++q)
				if (q % G == sub) dst[q] = sum[q];
		}
	}
}
template<class M, bool V, class S = double>
__global__ void __launch_bounds__(FACE_THREADS, FACE_MIN_BLOCKS) k_face_sum(Pool P, Consts C, BcTable B, const int32_t *list, int n, int L,
                                                    double dtL, int stamp, int32_t *recv, Counters *cnt) {
	d_face_sum<M, V, S>(PlainGrid{}, P, C, B, list, n, L, dtL, stamp, recv, cnt);
}

// The same face sums over tiles of TC consecutive list positions, one 128-thread block per tile. After
// the Morton re-sort (and with the order-keeping list rebuild) a tile is a compact patch of cells, and
// most faces have both cells in it; such a face is evaluated once, by the task of its owner, instead of
// once by each of its cells. Per tile:
//   1. every (cell, face) incidence is classified as d_face_sum classifies its lane: boundary, non-leaf
//      neighbour (the sum over the finer owners), a flux owned by the cell, a flux owned by the
//      same-level neighbour, or none. A flux owned by the neighbour becomes a reference to the
//      neighbour's own incidence when the neighbour is in the tile (it then evaluates that face as its
//      own), else a task of this cell; every other flux is a task;
//   2. the block's threads run the tasks, interior fluxes first (compacted at the low end of the task
//      list, boundary and non-leaf sums at the high end, so that warps diverge less), into shared memory;
//   3. each (cell, component) thread combines the cell's face terms in d_face_sum's fixed pairing order
//      and writes du.
// Every flux is the same call with the same arguments as in d_face_sum (the owner's), and the terms are
// combined in the same order with the same signs, so du is the same bit for bit.
template<class M>
struct FaceTile {
	static constexpr int NF = 2 * M::D, F = M::F;
	static constexpr int TC0 = 40960 / (NF * F * 8);  // the tile's face results within 40 KB
	static constexpr int TC  = TC0 >= 128 ? 128 : TC0 >= 64 ? 64 : 32;
	static constexpr int NI  = TC * NF;  // (cell, face) incidences of a tile
	static_assert(NI < 32768, "task indices are 16-bit");
};
enum : uint8_t { FT_NONE = 0, FT_BND = 1, FT_HANG = 2, FT_INT = 3, FT_INT_FF = 4, FT_REF = 5 };

template<class M, bool V, class S>
__global__ void __launch_bounds__(FACE_THREADS, FACE_MIN_BLOCKS)
k_face_tile(Pool P, Consts C, BcTable B, const int32_t *list, int n, int L, double dtL, int stamp, int32_t *recv,
            Counters *cnt) {
	using T = FaceTile<M>;
	constexpr int NF = T::NF, F = T::F, TC = T::TC, NI = T::NI, NSUB = 1 << (M::D - 1);
	__shared__ double s_res[NI * F];  // face results by incidence
	__shared__ int32_t s_a[NI];       // owner of a task, or the partner incidence of a reference
	__shared__ int32_t s_b[NI];       // the task's other cell, boundary id or non-leaf neighbour
	__shared__ int16_t s_task[NI];
	__shared__ int32_t s_cell[TC];
	__shared__ uint8_t s_kind[NI];
	__shared__ int s_lo, s_hi;
	const int cap = P.cap;
	for (int t0 = blockIdx.x * TC; t0 < n; t0 += gridDim.x * TC) {
		for (int c = threadIdx.x; c < TC; c += blockDim.x) {
			const int slot = t0 + c;
			int i          = -1;
			if (slot < n) {
				i        = list[slot];
				P.pos[i] = slot;
			}
			s_cell[c] = i;
		}
		if (threadIdx.x == 0) s_lo = 0, s_hi = 0;
		__syncthreads();
		// 1. classification
		for (int inc = threadIdx.x; inc < NI; inc += blockDim.x) {
			const int c = inc / NF, f = inc - c * NF, dir = f & 1;
			const int i = s_cell[c];
			uint8_t kind = FT_NONE;
			int a = 0, b = 0;
			bool low = true;
			if (i >= 0) {
				const int nb = P.nbr[(size_t) f * cap + i];
				if (nb == 0) {
					b = P.bc[(size_t) f * cap + i];
					if (b < 0) set_status(&cnt->status, ST_MISSING_BC);
					else kind = FT_BND, low = false;
				} else if (!(P.flags[nb] & F_LEAF)) {
					kind = FT_HANG, b = nb, low = false;
				} else {
					const int li = P.level[i], ai = P.acti[i], ln = P.level[nb], an = P.acti[nb];
					if (an <= ai && (ln < li || (ln == li && (dir == 1 || an < ai)))) {
						kind = FT_INT, a = i, b = nb;
						if (P.clu[nb] != L) {
							kind = FT_INT_FF;
							if (atomicExch(&P.stamp[nb], stamp) != stamp) append(recv, &cnt->n_recv, nb, cap, &cnt->status);
						}
					} else if (ln == li && P.clu[nb] == L && ai <= an && (dir == 0 || ai < an)) {
						// pos of a cell of this tile was written above, before the barrier; pos of any
						// other cell may be stale or being written by another block, so only the
						// s_cell check decides membership
						const int other = P.nbr[(size_t) (f ^ 1) * cap + nb];
						const int cn    = __ldcg(P.pos + nb) - t0;
						if (other == i && cn >= 0 && cn < TC && s_cell[cn] == nb) {
							kind = FT_REF, a = cn * NF + (f ^ 1);
						} else {
							kind = FT_INT, a = nb, b = other;
						}
					}
				}
			}
			s_kind[inc] = kind;
			s_a[inc]    = a;
			s_b[inc]    = b;
			if (kind != FT_NONE && kind != FT_REF) {
				if (low) s_task[atomicAdd(&s_lo, 1)] = (int16_t) inc;
				else s_task[NI - 1 - atomicAdd(&s_hi, 1)] = (int16_t) inc;
			}
		}
		__syncthreads();
		// 2. the tasks
		const int nlo = s_lo, ntask = s_lo + s_hi;
		for (int k = threadIdx.x; k < ntask; k += blockDim.x) {
			const int inc = k < nlo ? s_task[k] : s_task[NI - 1 - (k - nlo)];
			const int c = inc / NF, f = inc - c * NF, dim = f >> 1, dir = f & 1;
			const int i = s_cell[c];
			const uint8_t kind = s_kind[inc];
			double *res = s_res + (size_t) inc * F;
			if (kind == FT_BND) {
				double Fb[F];
				boundary_flux<M, V, S>(P, C, B, i, s_b[inc], dim, dir, dtL, Fb);
#pragma unroll
				for (int q = 0; q < F; ++q) res[q] = 0.0 - (double) (S) Fb[q];
			} else if (kind == FT_HANG) {
				const int nb = s_b[inc];
				const int li = P.level[i], ai = P.acti[i];
				double w[F];
#pragma unroll
				for (int q = 0; q < F; ++q) w[q] = 0.0;
				for (int cc = 1; cc < 1 + NSUB * (NSUB + 1); ++cc) {
					int dn;
					bool plus;
					const int owner = face_owner<M>(P, &cnt->status, i, nb, dim, dir, L, li, ai, cc, true, dn, plus);
					if (owner < 0) continue;
					const int fo = 2 * dim + dn;
					double Fw[F];
					interior_flux<M, V, S>(P, C, owner, P.nbr[(size_t) fo * cap + owner], dim, dn, dtL, Fw);
					if (plus) {
#pragma unroll
						for (int q = 0; q < F; ++q) w[q] += (double) (S) Fw[q];
					} else {
#pragma unroll
						for (int q = 0; q < F; ++q) w[q] -= (double) (S) Fw[q];
					}
				}
#pragma unroll
				for (int q = 0; q < F; ++q) res[q] = 0.0 + (double) (S) w[q];
			} else {
				const int own = s_a[inc];
				const int dir_o = own == i ? dir : 1 - dir;
				double Fi[F];
				interior_flux<M, V, S>(P, C, own, s_b[inc], dim, dir_o, dtL, Fi);
#pragma unroll
				for (int q = 0; q < F; ++q) res[q] = (double) (S) Fi[q];
				if (kind == FT_INT_FF) {
					S *dst = face_flux<S>(P, t0 + c, f, F, NF);
#pragma unroll
					for (int q = 0; q < F; ++q) dst[q] = (S) Fi[q];
				}
			}
		}
		__syncthreads();
		// 3. each cell's face terms in d_face_sum's pairing order
		for (int idx = threadIdx.x; idx < TC * F; idx += blockDim.x) {
			const int c = idx / F, q = idx - c * F;
			if (t0 + c >= n) continue;
			double fv[NF];
#pragma unroll
			for (int k = 0; k < NF; ++k) {
				const int inc = c * NF + k;
				const uint8_t kind = s_kind[inc];
				double v = 0.0;
				if (kind == FT_BND || kind == FT_HANG) {
					v = s_res[inc * F + q];
				} else if (kind != FT_NONE) {
					const double raw = s_res[(kind == FT_REF ? s_a[inc] : inc) * F + q];
					v = (k & 1) ? 0.0 - raw : 0.0 + raw;
				}
				fv[k] = v;
			}
			double sum;
			if constexpr (NF == 4) sum = (fv[0] + fv[2]) + (fv[1] + fv[3]);
			else sum = ((fv[0] + fv[4]) + (fv[2] + 0.0)) + ((fv[1] + fv[5]) + (fv[3] + 0.0));
			P.du[(size_t) (t0 + c) * F + q] = sum;
		}
		__syncthreads();
	}
}

// cell_update (impl/cell_update.hpp:10-90) of the running cluster, one thread per cell: du = (received
// fluxes + the face sum of k_face_sum) / volume, the multiphase source from the pre-update state, the
// EOS recovery, floors and the conservative state. The received-flux accumulator is read (and reset)
// only when the receive stage has marked the cell. Without viscous terms (V = false) the gradient
// inputs are never read, so t_slope is not maintained.
template<class M, bool V, class Grid>
__device__ __forceinline__ void d_update(const Grid &g, const Pool &P, const Consts &C, const int32_t *list, int n, double dtL, int epoch, Counters *cnt) {
	constexpr int E = M::E;
	const int cap  = P.cap;
	const int lane = threadIdx.x & 31;
	// warp-uniform loop: the whole warp stamps the updated cells' ancestors together
	for (int t0 = g.tid() - lane; t0 < n; t0 += g.stride()) {
		const int tid = t0 + lane;
		int up        = 0;
		if (tid < n) {
			const int i  = list[tid];
			const int li = P.level[i];
			const double vol  = C.vol[li];
			const uint32_t fl0 = P.flags[i];
			const bool rcv     = fl0 & F_RECV;
			const double *s_in = P.du + (size_t) tid * M::F;
			double du[M::F];
	#pragma unroll
			for (int q = 0; q < M::F; ++q) du[q] = ((rcv ? at(P.flux, cap, q, i) : 0.0) + s_in[q]) / vol;

			double pold[E], u[E], p[E];
			load_p<M>(P, i, pold);
			for (int q = 0; q < E; ++q) u[q] = at(P.u, cap, q, i);
			double gold[M::G > 0 ? M::G : 1];
			if constexpr (V) grad_input<M>(C.m, pold, gold);
			for (int q = 0; q < E; ++q) u[q] += du[q];
			if constexpr (M::MULTI) {
				if (!C.signal) {
					if (u[M::IA] > 0.001)
						for (int k = M::IU; k < M::IU + M::D; ++k) u[k] = 0.0;
				}
				// source (model/multi.hpp:186-203) from the pre-update state
				const double kap = at(P.k, cap, M::KAPPA, i);
				const double sg  = C.m.sigma;
				double s[E];
				for (int q = 0; q < E; ++q) s[q] = 0.0;
				for (int d = 0; d < M::D; ++d) s[M::IU + d] = -sg * kap * du[M::IA + 2 + d];
				s[M::IP] = sg * kap * (-du[M::IA] + pold[M::IA] * du[M::IA + 1]);
				s[M::IA] = -pold[M::IA] * du[M::IA + 1];
				for (int q = 0; q < E; ++q) u[q] = u[q] + s[q];
			}
			prim_from_cons<M>(C.m, u, p);
			if (isnan(p[M::IP]) || isnan(p[0])) set_status(&cnt->status, ST_NAN);
			if constexpr (M::MULTI) {
				p[0] = smax(p[0], 1e-3);
				p[1] = smax(p[1], 1e-6);
			} else {
				p[0] = smax(p[0], 1e-3);
			}
			p[M::IP] = smax(p[M::IP], 1e-3);
			cons_from_prim<M>(C.m, p, u);
			if constexpr (M::G > 0 && V) {
				double gnew[M::G];
				grad_input<M>(C.m, p, gnew);
				for (int g = 0; g < M::G; ++g) P.tslope[(size_t) g * cap + i] = (gnew[g] - gold[g]) / dtL;
			}
			if constexpr (M::MULTI) {
				P.k[(size_t) 0 * cap + i]        = C.m.mu1 * p[M::IA] + C.m.mu2 * (1 - p[M::IA]);
				P.k[(size_t) M::ALPHAS * cap + i] = p[M::IA];
			}
			for (int q = 0; q < E; ++q) {
				P.u[(size_t) q * cap + i] = u[q];
				P.p[(size_t) q * cap + i] = p[q];
			}
			store_p_rec<M>(P, i, p);
			if (rcv) {
				for (int q = 0; q < M::F; ++q) P.flux[(size_t) q * cap + i] = 0.0;
				P.flags[i] = fl0 & ~F_RECV;
			}
			P.t[i] = P.t[i] + dtL;
			up     = P.parent[i];
		}
		mark_up_warp(P, up, epoch);
	}
}
template<class M, bool V>
__global__ void __launch_bounds__(BLOCK, 3) k_update(Pool P, Consts C, const int32_t *list, int n, double dtL, int epoch,
                                                     Counters *cnt) {
	d_update<M, V>(PlainGrid{}, P, C, list, n, dtL, epoch, cnt);
}



// Neighbour facts of a face as the slope and estimation stages read them: presence, leaf flag, tree
// level and ACTI level of the face neighbour.
constexpr int32_t NB_LEAF = 1 << 8, NB_PRESENT = 1 << 9;

__device__ __forceinline__ int nb_level(int32_t code) { return code & 0xff; }
__device__ __forceinline__ int nb_acti(int32_t code) { return ((code >> 16) & 0xff) - 1; }

// The value compute_slope and the error estimator see across face f of cell i (impl/slopes.hpp:24-58,
// impl/adaptive_refinement.hpp:16-60): the neighbour's primitive state and time (its own, or the mean
// over a non-leaf neighbour's subtree, integrator/domain.hpp:84-148) and the centre distance
// 0.5 (h + h_n); returns the neighbour facts, 0 when the face has no neighbour.
template<class M>
__device__ __forceinline__ int32_t neighbour_value(const Pool &P, const Consts &C, uint32_t *status, int i, int f, int epoch,
                                                   double *v /*[E]*/, double &tv, double &dist) {
	constexpr int E = M::E;
	const int nb = P.nbr[(size_t) f * P.cap + i];
	if (nb == 0) return 0;
	const uint32_t fl = P.flags[nb];
	const int ln      = P.level[nb];
	double w[E + 1];
	if (!(fl & F_LEAF)) {
		interp_pt<M>(P, status, nb, epoch, w);
	} else {
		load_p_rec<M>(P, nb, w);
		w[E] = P.t[nb];
	}
#pragma unroll
	for (int q = 0; q < E; ++q) v[q] = w[q];
	tv   = w[E];
	dist = 0.5 * (C.size[P.level[i]] + C.size[ln]);
	return NB_PRESENT | ((fl & F_LEAF) ? NB_LEAF : 0) | ln | ((P.acti[nb] + 1) << 16);
}

// compute_slope (impl/slopes.hpp:16-76) of a cell list: limited primitive slopes, gradients (only read
// by the viscous terms, so computed when V) and the Hancock rhs, written to the record's [0, K0) part
// (p, rhs, slope rows); the gradients go to the pool. A group of G = 2D lanes serves one cell (8 cells a
// warp in 2D, 5 in 3D with the warp's last two lanes idle): lane f fetches the value across face f (the
// neighbour's, or the boundary ghost at distance h), the two lanes of a dimension meet to limit that
// dimension's slope row, and the group's first lane forms the rhs from all rows. The neighbour loads of a cell's faces thus run in parallel and nothing
// goes through memory between the fetch and the slope.
template<class M, bool V, class Grid>
__device__ __forceinline__ void d_slope(const Grid &g, const Pool &P, const Consts &C, const BcTable &B,
                                        const int32_t *list, int n, int lim, int epoch, Counters *cnt) {
	using R = Rec<M>;
	constexpr int E = M::E, D = M::D, NF = 2 * D, G = NF, GW = 32 / G;  // lanes per cell, cells per warp
	static_assert(R::K0 % 2 == 0, "record rows are 16-byte aligned");
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int grp    = lane / G;  // the lane's cell within the warp; lanes past GW * G idle
	const int sub    = lane - grp * G;
	const int base   = grp * G;
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot    = wbase + grp;
		const bool active = grp < GW && slot < n;
		const int i       = active ? list[slot] : 0;
		double pc[E];
		if (active) load_p<M>(P, i, pc);
		else
#pragma unroll
			for (int q = 0; q < E; ++q) pc[q] = 0.0;
		const double h  = active ? C.size[P.level[i]] : 1.0;
		const double ti = active ? P.t[i] : 0.0;
		// this lane's face: the value, its distance and time
		double pv[E], x = 0.0, tv = 0.0;
#pragma unroll
		for (int q = 0; q < E; ++q) pv[q] = pc[q];
		if (active && sub < NF) {
			const int f = sub, dir = f & 1;
			double dist;
			const int32_t code = neighbour_value<M>(P, C, &cnt->status, i, f, epoch, pv, tv, dist);
			if (!(code & NB_PRESENT)) {
				const int b = P.bc[(size_t) f * cap + i];
				if (b < 0) {
					set_status(&cnt->status, ST_MISSING_BC);
					for (int q = 0; q < E; ++q) pv[q] = pc[q];
				} else {
					boundary_value<M>(C.m, B, b, pc, ti, pv);
				}
				x  = dir == 0 ? -h : h;
				tv = ti;
			} else {
				x = dir == 0 ? -dist : dist;
			}
		}
		// the + side of each dimension moves to the dimension's first lane
		const int partner = base + (sub | 1);
		double pp[E];
#pragma unroll
		for (int q = 0; q < E; ++q) pp[q] = __shfl_sync(0xffffffffu, pv[q], partner);
		const double xp = __shfl_sync(0xffffffffu, x, partner);
		const double tp = __shfl_sync(0xffffffffu, tv, partner);
		double row[E];
#pragma unroll
		for (int q = 0; q < E; ++q) row[q] = 0.0;
		if (active && sub < NF && !(sub & 1)) {
			const int dim   = sub >> 1;
			const double xc = 0.0, xn = x, tn = tv;
			for (int q = 0; q < E; ++q) {
				double sn = (pc[q] - pv[q]) / (xc - xn);
				double sp = (pp[q] - pc[q]) / (xp - xc);
				row[q]    = limit(lim, sn, sp);
			}
			if constexpr (M::G > 0 && V) {
				double gp[M::G], gn[M::G];
				grad_input<M>(C.m, pp, gp);
				grad_input<M>(C.m, pv, gn);
				for (int k = 0; k < M::G; ++k) {
					double ts = at(P.tslope, cap, k, i);
					P.grad[(size_t) (dim * M::G + k) * cap + i] = (gp[k] - gn[k] - ts * (tp - tn)) / (xp - xn);
				}
			}
			// slope row `dim` of the record
			double2 *dst = reinterpret_cast<double2 *>(rec_of(P, i, R::W) + R::S0 + dim * R::ES);
#pragma unroll
			for (int k = 0; k < R::ES / 2; ++k) dst[k] = make_double2(row[2 * k], 2 * k + 1 < E ? row[2 * k + 1] : 0.0);
		}
		// all rows to the group's first lane, which forms the rhs
		double slope[D * E];
#pragma unroll
		for (int d = 0; d < D; ++d)
#pragma unroll
			for (int q = 0; q < E; ++q) slope[d * E + q] = __shfl_sync(0xffffffffu, row[q], min(base + 2 * d, 31));
		if (active && sub == 0) {
			double rhs[E];
			double kap = 0.0;
			if constexpr (M::MULTI) kap = at(P.k, cap, M::KAPPA, i);
			compute_rhs<M>(C.m, pc, slope, kap, rhs);
			double out[2 * E];
#pragma unroll
			for (int q = 0; q < E; ++q) out[R::P0 + q] = pc[q], out[R::R0 + q] = rhs[q];
			double2 *dst = reinterpret_cast<double2 *>(rec_of(P, i, R::W));
#pragma unroll
			for (int k = 0; k < E; ++k) dst[k] = make_double2(out[2 * k], out[2 * k + 1]);
		}
	}
}
template<class M, bool V>
__global__ void __launch_bounds__(SLOPE_THREADS, SLOPE_MIN_BLOCKS) k_slope(Pool P, Consts C, BcTable B, const int32_t *list, int n, int lim, int epoch,
                                                 Counters *cnt) {
	d_slope<M, V>(PlainGrid{}, P, C, B, list, n, lim, epoch, cnt);
}

// Recompute the Hancock rhs from the stored slope (used for split parents, whose curvature may
// have changed since the slope stage; impl/adaptive_refinement.hpp:169).
template<class M>
__device__ void recompute_rhs(const Pool &P, const Consts &C, int i) {
	constexpr int E = M::E, D = M::D;
	const int cap = P.cap;
	double pc[E], slope[D * E], rhs[E];
	load_p<M>(P, i, pc);
	for (int d = 0; d < D; ++d)
		for (int q = 0; q < E; ++q) slope[d * E + q] = rec_slope<M>(P, i, d, q);
	double kap = 0.0;
	if constexpr (M::MULTI) kap = at(P.k, cap, M::KAPPA, i);
	compute_rhs<M>(C.m, pc, slope, kap, rhs);
	double *r = rec_of(P, i, Rec<M>::W);
	for (int q = 0; q < E; ++q) r[Rec<M>::R0 + q] = rhs[q];
}

// Scene::can_split (scene/scene.hpp:50-61) with identity-transform refinement zones.
template<int D>
__device__ bool can_split_at(const Pool &P, const Consts &C, int i) {
	const int l = P.level[i];
	if (l < C.max_refinement_level) return true;
	for (int z = 0; z < C.n_zones; ++z) {
		if (l < C.zlevel[z]) {
			bool in = true;
			for (int d = 0; d < 3; ++d) {
				double x = d < D ? at(P.center, P.cap, d, i) : 0.0;
				in = in && (x < C.zx1[z][d]) && (x > C.zx0[z][d]);
			}
			if (in) return true;
		}
	}
	return false;
}

// Error estimation and split/unsplit detection (impl/adaptive_refinement.hpp:16-149) with the
// weighted_laplacian estimator (integrator/error_estimators.hpp:19-37). A group of G lanes per cell,
// as in the slope stage: lane f fetches the value across face f (a coarser leaf's state extrapolated
// to the same-level position with its slope), the two lanes of a dimension meet to form that
// dimension's second difference, and the group's first lane sums the dimensions in order and decides.
template<class M, class Grid>
__device__ __forceinline__ void d_estimate(const Grid &g, const Pool &P, const Consts &C, const int32_t *list, int n, int L,
                                           int counter_L, int epoch, int32_t *split_list, Counters *cnt) {
	constexpr int E = M::E, D = M::D, NF = 2 * D, G = NF, GW = 32 / G;  // lanes per cell, cells per warp
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int grp    = lane / G;  // the lane's cell within the warp; lanes past GW * G idle
	const int sub    = lane - grp * G;
	const int base   = grp * G;
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot    = wbase + grp;
		const bool active = grp < GW && slot < n;
		const int i       = active ? list[slot] : 0;
		const int li      = active ? P.level[i] : 0;
		double pc[E];
		if (active) load_p<M>(P, i, pc);
		else
#pragma unroll
			for (int q = 0; q < E; ++q) pc[q] = 0.0;
		double v[E];
#pragma unroll
		for (int q = 0; q < E; ++q) v[q] = 0.0;
		int32_t code = 0;
		if (active && sub < NF) {
			const int f = sub, dim = f >> 1, dir = f & 1;
			double tv, dist;
			code = neighbour_value<M>(P, C, &cnt->status, i, f, epoch, v, tv, dist);
			if ((code & NB_PRESENT) && (code & NB_LEAF) && nb_level(code) < li) {
				// a coarser leaf: its state extrapolated to the same-level position
				const int nb   = P.nbr[(size_t) f * cap + i];
				const double h = C.size[li];
				double x[D];
				for (int d = 0; d < D; ++d) x[d] = at(P.center, cap, d, i) + (d == dim ? h * (2 * dir - 1.0) : 0.0 * h);
				if (C.periodic[dim] && dir == 0 && x[dim] < -0.5 * C.active[dim]) x[dim] += C.active[dim];
				if (C.periodic[dim] && dir == 1 && x[dim] > 0.5 * C.active[dim]) x[dim] -= C.active[dim];
				for (int d = 0; d < D; ++d) {
					const double off = x[d] - at(P.center, cap, d, nb);
					for (int q = 0; q < E; ++q) v[q] = v[q] + rec_slope<M>(P, nb, d, q) * off;
				}
			}
		}
		// second difference of each dimension on the dimension's first lane
		const int partner = base + (sub | 1);
		double vp[E];
#pragma unroll
		for (int q = 0; q < E; ++q) vp[q] = __shfl_sync(0xffffffffu, v[q], partner);
		const int32_t code_p = __shfl_sync(0xffffffffu, code, partner);
		double sq = 0.0;
		if (active && sub < NF && !(sub & 1)) {
			double d2[E];
			for (int q = 0; q < E; ++q) d2[q] = pc[q] * -2.0;
			bool missing = !(code & NB_PRESENT);
			if (!missing) {
				for (int q = 0; q < E; ++q) d2[q] = d2[q] + v[q];
				missing = !(code_p & NB_PRESENT);
				if (!missing)
					for (int q = 0; q < E; ++q) d2[q] = d2[q] + vp[q];
			}
			if (missing)
				for (int q = 0; q < E; ++q) d2[q] = 0.0;
			for (int q = 0; q < E; ++q) {
				const double w = d2[q] * C.weights[q];
				sq += w * w;
			}
		}
		double sqd[D];
#pragma unroll
		for (int d = 0; d < D; ++d) sqd[d] = __shfl_sync(0xffffffffu, sq, min(base + 2 * d, 31));
		// neighbour facts of the whole group: a present face more than one level coarser; a present face
		// that is not a leaf or belongs to a faster cluster
		const bool coarse2         = (code & NB_PRESENT) && nb_level(code) < li - 1;
		const bool busy            = (code & NB_PRESENT) && (!(code & NB_LEAF) || nb_acti(code) > L);
		const unsigned gmask       = ((1u << G) - 1u) << base;
		const unsigned any_coarse2 = __ballot_sync(0xffffffffu, coarse2) & gmask;
		const unsigned any_busy    = __ballot_sync(0xffffffffu, busy) & gmask;
		if (!active || sub != 0) continue;
		double error = 0.0;
		for (int d = 0; d < D; ++d) error += sqd[d];
		error = sqrt(error);
		P.err[i] = error;

		uint32_t fl = P.flags[i];
		if (fl & F_CAN_SPLIT) {
			if (!can_split_at<D>(P, C, i)) {
				fl &= ~F_CAN_SPLIT;
				P.flags[i] = fl;
			}
		}
		uint8_t op = OP_NONE;
		const bool want_split = (error > C.max_err && (fl & F_CAN_SPLIT)) || (fl & F_SHOULD_SPLIT);
		if (want_split && !any_coarse2) op |= OP_SPLIT;
		if (error < C.min_err && (fl & F_CAN_UNSPLIT) && li > 0 && counter_L == 1 && C.coarsen && !(fl & F_HOLD) && !any_busy)
			op |= OP_UCAND;
		P.op[i] = op;
		if (op & OP_SPLIT) append(split_list, &cnt->n_split, i, cap, &cnt->status);
	}
}
template<class M>
__global__ void __launch_bounds__(BLOCK) k_estimate(Pool P, Consts C, const int32_t *list, int n, int L, int counter_L,
                                                    int epoch, int32_t *split_list, Counters *cnt) {
	d_estimate<M>(PlainGrid{}, P, C, list, n, L, counter_L, epoch, split_list, cnt);
}

// A parent coarsens when all its children are coarsening candidates of this cluster
// (impl/adaptive_refinement.hpp:198-209); the first child decides.
template<class M, class Grid>
__device__ __forceinline__ void d_unsplit_select(const Grid &g, const Pool &P, const int32_t *list, int n, int L, int32_t *unsplit_list, Counters *cnt) {
	const int cap = P.cap;
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int i = list[tid];
		if (!(P.op[i] & OP_UCAND)) continue;
		const int par = P.parent[i];
		if (P.child[par] != i) continue;
		bool all = true;
		for (int c = 0; c < (1 << M::D); ++c) {
			const int ch = P.child[(size_t) c * cap + par];
			const uint8_t o = P.op[ch];
			if (P.clu[ch] != L || !(o & OP_UCAND)) all = false;
			if (P.clu[ch] == L && (o & OP_SPLIT) && (o & OP_UCAND)) {
				set_status(&cnt->status, ST_SPLIT_UNSPLIT);
				all = false;
			}
		}
		if (all) append(unsplit_list, &cnt->n_unsplit, par, cap, &cnt->status);
	}
}
template<class M>
__global__ void k_unsplit_select(Pool P, const int32_t *list, int n, int L, int32_t *unsplit_list, Counters *cnt) {
	d_unsplit_select<M>(PlainGrid{}, P, list, n, L, unsplit_list, cnt);
}

// Domain::split (integrator/domain.hpp:192-247) plus the child set-up of
// impl/adaptive_refinement.hpp:167-195. Children take the parent's primitive state extrapolated
// with its slope, reuse the parent's old child slots when it has any, start with a zero Hancock
// rhs, and join the running cluster.
template<class M, class Grid>
__device__ __forceinline__ void d_split(const Grid &g, const Pool &P, const Consts &C, const int *n_ptr, const int32_t *split_list, int L, int32_t *fresh, int epoch, Counters *cnt) {
	constexpr int E = M::E, D = M::D, NC = 1 << D, GW = 32 / NC;
	using R = Rec<M>;
	const int n      = *n_ptr;
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int c      = lane & (NC - 1);  // the child this lane sets up
	const int lead   = lane & ~(NC - 1);
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	// one group of 2^D lanes per parent: the group's first lane allocates, every lane builds one child
	for (int base = warp * GW; base < n; base += nwarps * GW) {
		const int slot    = base + lane / NC;
		const bool active = slot < n;
		const int par     = active ? split_list[slot] : 0;
		int first = 0, reuse = 0, fail = 0;
		if (active && c == 0) {
			if constexpr (M::MULTI) recompute_rhs<M>(P, C, par);
			reuse = P.child[par] != 0;
			if (!reuse) {
				first = atomicAdd(&cnt->top, NC);
				if (first + NC > cap) {
					set_status(&cnt->status, ST_CAPACITY);
					fail = 1;
				}
			}
		}
		first = __shfl_sync(0xffffffffu, first, lead);
		reuse = __shfl_sync(0xffffffffu, reuse, lead);
		fail  = __shfl_sync(0xffffffffu, fail, lead);
		if (active && !fail) {
			const int s = reuse ? P.child[(size_t) c * cap + par] : first + c;
			if (!reuse) P.child[(size_t) c * cap + par] = s;
			const int lp   = P.level[par];
			const double q = 0.25 * C.size[lp];
			double pp[E], pc[D];
			load_p<M>(P, par, pp);
			for (int d = 0; d < D; ++d) pc[d] = at(P.center, cap, d, par);
			const double *rp = rec_of(P, par, R::W);
			P.parent[s] = par;
			P.level[s]  = (int8_t) (lp + 1);
			P.acti[s]   = (int8_t) L;
			P.clu[s]    = (int8_t) L;
			P.flags[s]  = F_LEAF | F_ACTIVE | F_CAN_SPLIT | F_CAN_UNSPLIT;
			double cc[D];
			for (int d = 0; d < D; ++d) {
				const double qd = (c >> d) & 1 ? 1.0 : -1.0;
				cc[d] = pc[d] + q * qd;
				P.center[(size_t) d * cap + s] = cc[d];
				P.coord[(size_t) d * cap + s]  = 2 * P.coord[(size_t) d * cap + par] + ((c >> d) & 1);
			}
			P.t[s] = P.t[par];
			double p[E], u[E];
			for (int k = 0; k < E; ++k) p[k] = pp[k];
			for (int d = 0; d < D; ++d) {
				const double off = cc[d] - pc[d];
				for (int k = 0; k < E; ++k) p[k] = p[k] + rp[R::S0 + d * R::ES + k] * off;
			}
			cons_from_prim<M>(C.m, p, u);
			double *rs = rec_of(P, s, R::W);
			for (int k = 0; k < E; ++k) {
				P.p[(size_t) k * cap + s] = p[k];
				P.u[(size_t) k * cap + s] = u[k];
				rs[R::P0 + k]             = p[k];
				rs[R::R0 + k]             = 0.0;
			}
			for (int k = 0; k < D * R::ES; ++k) rs[R::S0 + k] = rp[R::S0 + k];
			for (int k = 0; k < M::P; ++k) P.k[(size_t) k * cap + s] = at(P.k, cap, k, par);
			write_rec_k<M>(P, s);
			if (C.visc) {
				for (int k = 0; k < M::G; ++k) P.tslope[(size_t) k * cap + s] = at(P.tslope, cap, k, par);
				for (int k = 0; k < D * M::G; ++k) P.grad[(size_t) k * cap + s] = at(P.grad, cap, k, par);
			}
			for (int k = 0; k < M::F; ++k) P.flux[(size_t) k * cap + s] = 0.0;
			P.err[s] = -1.0;
			for (int dim = 0; dim < D; ++dim) {
				for (int dir = 0; dir < 2; ++dir) {
					const int f = 2 * dim + dir;
					P.nbr[(size_t) f * cap + s] = 0;
					P.bc[(size_t) f * cap + s]  = ((c & (1 << dim)) == (dir << dim)) ? P.bc[(size_t) f * cap + par] : (int16_t) -1;
				}
			}
			if (!reuse)
				for (int k = 0; k < NC; ++k) P.child[(size_t) k * cap + s] = 0;
			append(fresh, &cnt->n_new, s, cap, &cnt->status);
		}
		__syncwarp();
		if (active && !fail && c == 0) {
			P.flags[par] &= ~(F_LEAF | F_SHOULD_SPLIT);
			mark_up(P, par, epoch);
		}
	}
}
template<class M>
__global__ void k_split(Pool P, Consts C, const int *n_ptr, const int32_t *split_list, int L, int32_t *fresh,
                        int epoch, Counters *cnt) {
	d_split<M>(PlainGrid{}, P, C, n_ptr, split_list, L, fresh, epoch, cnt);
}

// Domain::unsplit with interpolated_cell (integrator/domain.hpp:150-180, 296-325): the parent takes
// the children's mean t, u, k, t_slope and gradient (the gradient sum starts from the parent's own
// stale gradient, as interpolated_cell does not reset it) and keeps its old slope and rhs.
template<class M, class Grid>
__device__ __forceinline__ void d_unsplit(const Grid &g, const Pool &P, const Consts &C, const int *n_ptr, const int32_t *unsplit_list, int L, int32_t *fresh, int epoch, Counters *cnt) {
	constexpr int E = M::E, D = M::D, NC = 1 << D, G = M::G;
	const int n   = *n_ptr;
	const int cap = P.cap;
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int par = unsplit_list[tid];
		double t = 0.0, u[E], kk[M::P > 0 ? M::P : 1], ts[G > 0 ? G : 1], gr[D * G > 0 ? D * G : 1];
		for (int q = 0; q < E; ++q) u[q] = 0.0;
		for (int q = 0; q < M::P; ++q) kk[q] = 0.0;
		for (int q = 0; q < G; ++q) ts[q] = 0.0;
		for (int q = 0; q < D * G; ++q) gr[q] = C.visc ? at(P.grad, cap, q, par) : 0.0;
		double error = 0.0;
		for (int c = 0; c < NC; ++c) {
			const int ch = P.child[(size_t) c * cap + par];
			t += P.t[ch];
			for (int q = 0; q < E; ++q) u[q] = u[q] + at(P.u, cap, q, ch);
			for (int q = 0; q < M::P; ++q) kk[q] = kk[q] + at(P.k, cap, q, ch);
			if (C.visc) {
				for (int q = 0; q < D * G; ++q) gr[q] = gr[q] + at(P.grad, cap, q, ch);
				for (int q = 0; q < G; ++q) ts[q] = ts[q] + at(P.tslope, cap, q, ch);
			}
		}
		for (int c = 0; c < NC; ++c) {
			const int ch = P.child[(size_t) c * cap + par];
			error += P.err[ch];
			P.flags[ch] |= F_GARBAGE | F_LEAF;
		}
		t = t / (double) NC;
		for (int q = 0; q < G; ++q) ts[q] = ts[q] / (double) NC;
		for (int q = 0; q < E; ++q) u[q] = u[q] / (double) NC;
		double p[E];
		prim_from_cons<M>(C.m, u, p);
		for (int q = 0; q < M::P; ++q) kk[q] = kk[q] / (double) NC;
		for (int q = 0; q < D * G; ++q) gr[q] = gr[q] / (double) NC;
		P.t[par] = t;
		double *rpar = rec_of(P, par, Rec<M>::W);
		for (int q = 0; q < E; ++q) {
			P.u[(size_t) q * cap + par] = u[q];
			P.p[(size_t) q * cap + par] = p[q];
			rpar[Rec<M>::P0 + q]        = p[q];
		}
		for (int q = 0; q < M::P; ++q) P.k[(size_t) q * cap + par] = kk[q];
		write_rec_k<M>(P, par);
		if (C.visc) {
			for (int q = 0; q < G; ++q) P.tslope[(size_t) q * cap + par] = ts[q];
			for (int q = 0; q < D * G; ++q) P.grad[(size_t) q * cap + par] = gr[q];
		}
		for (int q = 0; q < M::F; ++q) P.flux[(size_t) q * cap + par] = 0.0;
		for (int f = 0; f < 2 * D; ++f) P.nbr[(size_t) f * cap + par] = 0;
		P.err[par]   = error;
		P.flags[par] = (P.flags[par] | F_LEAF | F_ACTIVE | F_CAN_SPLIT) & ~F_GARBAGE;
		P.acti[par]  = (int8_t) L;
		P.clu[par]   = (int8_t) L;
		append(fresh, &cnt->n_new, par, cap, &cnt->status);
		mark_up(P, P.parent[par], epoch);
	}
}
template<class M>
__global__ void k_unsplit(Pool P, Consts C, const int *n_ptr, const int32_t *unsplit_list, int L, int32_t *fresh,
                          int epoch, Counters *cnt) {
	d_unsplit<M>(PlainGrid{}, P, C, n_ptr, unsplit_list, L, fresh, epoch, cnt);
}

// Domain::update_neighbors for one active leaf (integrator/domain.hpp:249-293): faces without a
// boundary get the node found at the same level (or the coarser leaf); a neighbour more than one
// level coarser is flagged should_split.
template<class M>
__device__ void update_neighbor_face(const Pool &P, const Consts &C, int i, int dim, int dir) {
	const int cap = P.cap;
	const int f   = 2 * dim + dir;
	if (P.bc[(size_t) f * cap + i] >= 0) return;
	const int nb = find_neighbor<M::D>(P, C, i, dim, dir);
	if (nb == 0 || !(P.flags[nb] & F_ACTIVE)) return;
	P.nbr[(size_t) f * cap + i] = nb;
	if (P.level[nb] < P.level[i] - 1) atomicOr(&P.flags[nb], (uint32_t) F_SHOULD_SPLIT);
}

template<class M>
__device__ void update_neighbors_leaf(const Pool &P, const Consts &C, int i) {
	for (int dim = 0; dim < M::D; ++dim)
		for (int dir = 0; dir < 2; ++dir) update_neighbor_face<M>(P, C, i, dim, dir);
}

// update_neighbors restricted to one face of a node: the leaves of its subtree that touch face
// (dim, dir) get that face's neighbour recomputed. Used for the neighbours of new cells: a leaf of such a
// neighbour's subtree that does not touch the face towards the new cell finds the same neighbours as
// before, so the reference's full subtree update leaves it unchanged.
template<class M>
__device__ void update_face_subtree(const Pool &P, const Consts &C, uint32_t *status, int root, int dim, int dir) {
	constexpr int NC = 1 << M::D, NH = NC / 2;
	constexpr int CAP = NH * MAX_TREE;
	int stack[CAP];
	int sp = 0;
	stack[sp++] = root;
	while (sp > 0) {
		const int x = stack[--sp];
		if (x == 0) continue;  // a subtree without active leaves that the host left out
		const uint32_t fl = P.flags[x];
		if (fl & F_LEAF) {
			if (fl & F_ACTIVE) update_neighbor_face<M>(P, C, x, dim, dir);
			continue;
		}
		for (int c = NC - 1; c >= 0; --c) {
			if (((c >> dim) & 1) != dir) continue;
			if (sp >= CAP) {
				set_status(status, ST_DEPTH);
				break;
			}
			stack[sp++] = P.child[(size_t) c * P.cap + x];
		}
	}
}

// update_neighbors applied to a node: leaves directly, non-leaves through all their descendants.
template<class M>
__device__ void update_neighbors_subtree(const Pool &P, const Consts &C, uint32_t *status, int root) {
	constexpr int NC = 1 << M::D;
	constexpr int CAP = 8 * MAX_TREE;
	int stack[CAP];
	int sp = 0;
	stack[sp++] = root;
	while (sp > 0) {
		const int x = stack[--sp];
		if (x == 0) continue;  // a subtree without active leaves that the host left out
		const uint32_t fl = P.flags[x];
		if (fl & F_LEAF) {
			if (fl & F_ACTIVE) update_neighbors_leaf<M>(P, C, x);
			continue;
		}
		for (int c = NC - 1; c >= 0; --c) {
			if (sp >= CAP) {
				set_status(status, ST_DEPTH);
				break;
			}
			stack[sp++] = P.child[(size_t) c * P.cap + x];
		}
	}
}

// Neighbour repair, first pass (impl/adaptive_refinement.hpp:236-249): new children and coarsened
// parents, then queue their neighbours for the second pass.
// Each neighbour is queued once with the mask of its faces towards new cells. A group of lanes serves one
// new cell (4 in 2D, 8 in 3D with 6 busy), lane f repairing face f and queueing the neighbour across it,
// so the tree walks of a cell's faces run side by side instead of one after another in one thread. New
// cells are leaves; a non-leaf (which the stages do not produce) is repaired whole by its group's first
// lane, as Domain::update_neighbors repairs a subtree.
template<class M, class Grid>
__device__ __forceinline__ void d_nbr_fresh(const Grid &g, const Pool &P, const Consts &C, const int *n_ptr, const int32_t *fresh, int32_t *upd, Counters *cnt) {
	constexpr int NF = 2 * M::D, G = NF <= 4 ? 4 : 8, GW = 32 / G;
	const int n      = *n_ptr;
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int sub    = lane & (G - 1);
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	auto queue = [&](int i, int f) {
		const int nb = P.nbr[(size_t) f * cap + i];
		if (nb != 0 && ((P.flags[nb] & F_ACTIVE) || !(P.flags[nb] & F_LEAF))) {
			if (atomicOr(&P.fmask[nb], 1u << (f ^ 1)) == 0) append(upd, &cnt->n_upd, nb, cap, &cnt->status);
		}
	};
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot = wbase + lane / G;
		if (slot >= n || sub >= NF) continue;
		const int i       = fresh[slot];
		const uint32_t fl = P.flags[i];
		if (fl & F_LEAF) {
			if (fl & F_ACTIVE) update_neighbor_face<M>(P, C, i, sub >> 1, sub & 1);
			queue(i, sub);
		} else if (sub == 0) {
			update_neighbors_subtree<M>(P, C, &cnt->status, i);
			for (int f = 0; f < NF; ++f) queue(i, f);
		}
	}
}
template<class M>
__global__ void k_nbr_fresh(Pool P, Consts C, const int *n_ptr, const int32_t *fresh, int32_t *upd, Counters *cnt) {
	d_nbr_fresh<M>(PlainGrid{}, P, C, n_ptr, fresh, upd, cnt);
}

// Neighbour repair, second pass: the queued neighbours' faces towards new cells, one lane per face (the
// lane groups of the first pass). The group reads the face mask before its first lane clears it.
template<class M, class Grid>
__device__ __forceinline__ void d_nbr_list(const Grid &g, const Pool &P, const Consts &C, const int *n_ptr, const int32_t *list, Counters *cnt) {
	constexpr int NF = 2 * M::D, G = NF <= 4 ? 4 : 8, GW = 32 / G;
	const int n      = *n_ptr;
	const int lane   = threadIdx.x & 31;
	const int sub    = lane & (G - 1);
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot = wbase + lane / G;
		const bool act = slot < n && sub < NF;
		const int x      = act ? list[slot] : 0;
		const uint32_t m = act ? P.fmask[x] : 0u;
		__syncwarp();
		if (act && (m & (1u << sub))) update_face_subtree<M>(P, C, &cnt->status, x, sub >> 1, sub & 1);
		if (act && sub == 0) P.fmask[x] = 0;
	}
}
template<class M>
__global__ void k_nbr_list(Pool P, Consts C, const int *n_ptr, const int32_t *list, Counters *cnt) {
	d_nbr_list<M>(PlainGrid{}, P, C, n_ptr, list, cnt);
}

// ACTI reassignment (impl/adaptive_refinement.hpp:264-322): per-cell CFL decides whether a cell
// stays, drops one time level (into the buffer of L-1, only when level L is synchronised with L-1)
// or rises by floor(log2(cfl/max_cfl))+1 levels.
//
// `stay` (optional, one byte per list position): instead of appending the cells that stay at level L to
// the rebuilt list with an atomic counter (which leaves them in the order the warps reach the counter),
// mark them, so that an order-keeping compaction can rebuild the list in the old list's order. After the
// Morton re-sort that keeps each cluster list in Morton order through the whole global step.
template<class M, class Grid>
__device__ __forceinline__ void d_reassign(const Grid &g, const Pool &P, const Consts &C, const int32_t *list, const int *n_ptr, int n_host, int L, double dtL, int counter_L, const Lists &Ls, Counters *cnt, uint8_t *stay = nullptr) {
	const int n   = n_ptr ? *n_ptr : n_host;
	const int cap = P.cap;
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int i = list[tid];
		double p[M::E];
		load_p<M>(P, i, p);
		const double mdt = max_delta_time<M>(C.m, p, C.size[P.level[i]]);
		P.maxdt[i]       = mdt;
		double cfl       = dtL / mdt;
		const uint32_t fl = P.flags[i];
		if (stay) stay[tid] = 0;
		if (!(fl & F_LEAF) || (fl & F_GARBAGE)) {
			P.cfl[i] = cfl;
			P.clu[i] = CLU_NONE;
			continue;
		}
		if (cfl < 0.5 * C.max_cfl && counter_L == 1 && L > 0) {
			append(Ls.buf[L - 1], &cnt->buf[L - 1], i, cap, &cnt->status);
			cfl *= 2;
			P.clu[i] = (int8_t) (BUF_BASE + L - 1);
		} else if (cfl > C.max_cfl && L < MAX_ACTI - 1) {
			const int raise = (int) log2(cfl / C.max_cfl) + 1;
			if (L + raise < MAX_ACTI) {
				append(Ls.clu[L + raise], &cnt->clu[L + raise], i, cap, &cnt->status);
				P.acti[i] = (int8_t) (L + raise);
				cfl /= (double) (1 << raise);
				P.clu[i] = (int8_t) (L + raise);
			} else {
				P.clu[i] = CLU_NONE;
			}
		} else {
			if (stay) stay[tid] = 1;
			else append(Ls.tmp, &cnt->n_tmp, i, cap, &cnt->status);
			P.clu[i] = (int8_t) L;
		}
		P.cfl[i] = cfl;
	}
}
template<class M>
__global__ void k_reassign(Pool P, Consts C, const int32_t *list, const int *n_ptr, int n_host, int L, double dtL,
                           int counter_L, Lists Ls, Counters *cnt, uint8_t *stay) {
	d_reassign<M>(PlainGrid{}, P, C, list, n_ptr, n_host, L, dtL, counter_L, Ls, cnt, stay);
}

// flush_acti_buffer (impl/acti_utils.hpp:365-372)
template<class Grid>
__device__ __forceinline__ void d_flush(const Grid &g, const Pool &P, const int32_t *buf, const int *n_ptr, int32_t *clu_list, int *clu_count, int L, Counters *cnt) {
	const int n = *n_ptr;
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int i = buf[tid];
		append(clu_list, clu_count, i, P.cap, &cnt->status);
		P.acti[i] = (int8_t) L;
		P.clu[i]  = (int8_t) L;
	}
}
static __global__ void k_flush(Pool P, const int32_t *buf, const int *n_ptr, int32_t *clu_list, int *clu_count, int L,
                        Counters *cnt) {
	d_flush(PlainGrid{}, P, buf, n_ptr, clu_list, clu_count, L, cnt);
}

static __global__ void k_set_count(int *dst, const int *src) { *dst = *src; }

// --------------------------------------------------------------------------------------------
// Initialisation (integrator/integrator.hpp:100-160)
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_pos_double(double *addr, double v) {
	// non-negative doubles order like their bit patterns as signed 64-bit integers
	atomicMax(reinterpret_cast<long long *>(addr), __double_as_longlong(v));
}

template<class M>
__global__ void k_init_cells(Pool P, Consts C, const int32_t *list, int n, Counters *cnt) {
	constexpr int E = M::E;
	const int cap = P.cap;
	double local_max = -INFINITY;
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		double p[E], u[E];
		load_p<M>(P, i, p);
		store_p_rec<M>(P, i, p);
		cons_from_prim<M>(C.m, p, u);
		for (int q = 0; q < E; ++q) P.u[(size_t) q * cap + i] = u[q];
		if constexpr (M::MULTI) {
			P.k[(size_t) 0 * cap + i]         = C.m.mu1 * p[M::IA] + C.m.mu2 * (1 - p[M::IA]);
			P.k[(size_t) M::ALPHAS * cap + i] = p[M::IA];
		}
		if (C.visc)
			for (int g = 0; g < M::G; ++g) P.tslope[(size_t) g * cap + i] = 0.0;
		const double mdt = max_delta_time<M>(C.m, p, C.size[P.level[i]]);
		P.maxdt[i] = mdt;
		for (int q = 0; q < M::F; ++q) P.flux[(size_t) q * cap + i] = 0.0;
		local_max = smax(local_max, mdt);
	}
	// warp-shuffle max, then one atomic per warp
	for (int off = 16; off > 0; off >>= 1) local_max = smax(local_max, __shfl_xor_sync(0xffffffffu, local_max, off));
	if ((threadIdx.x & 31) == 0 && local_max > 0) atomic_max_pos_double(&cnt->dmax, local_max);
}

template<class M>
__global__ void k_nbr_init(Pool P, Consts C, const int32_t *list, int n) {
	for (int tid = gtid(); tid < n; tid += gstride()) update_neighbors_leaf<M>(P, C, list[tid]);
}

// assign_to_acti_clusters (impl/acti_utils.hpp:11-24)
template<class M>
__global__ void k_assign(Pool P, Consts C, const int32_t *list, int n, double global_dt, Lists Ls, Counters *cnt) {
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		const uint32_t fl = P.flags[i];
		if (!(fl & F_ACTIVE) || !(fl & F_LEAF)) continue;
		double cfl = global_dt / P.maxdt[i];
		int lvl    = (int) log2(cfl / C.max_cfl);
		lvl        = lvl < 0 ? 0 : (lvl > MAX_ACTI - 1 ? MAX_ACTI - 1 : lvl);
		cfl /= (double) (1 << lvl);
		P.cfl[i]  = cfl;
		P.acti[i] = (int8_t) lvl;
		P.clu[i]  = (int8_t) lvl;
		append(Ls.clu[lvl], &cnt->clu[lvl], i, P.cap, &cnt->status);
	}
}

// Gather of the active cells' limited slopes ([D][E] per cell) for the read-back API.
template<class M>
__global__ void k_gather_slopes(Pool P, const int32_t *list, int n, int base, double *out) {
	constexpr int E = M::E, D = M::D;
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		double *o   = out + (size_t) (base + tid) * D * E;
		for (int d = 0; d < D; ++d)
			for (int q = 0; q < E; ++q) o[d * E + q] = rec_slope<M>(P, i, d, q);
	}
}

// Gradients (Cell::gradient, [D][G]) of the listed cells, for the read-back API.
template<class M>
__global__ void k_gather_grads(Pool P, const int32_t *list, int n, int base, double *out) {
	constexpr int G = M::G, D = M::D;
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		double *o   = out + (size_t) (base + tid) * D * G;
		for (int k = 0; k < D * G; ++k) o[k] = at(P.grad, P.cap, k, i);
	}
}

// Inputs of the regrid forecaster (no reference counterpart). For leaf i with size h, from its
// primitive state and limited slopes: a = |grad rho| h / rho, b = |grad p| h / p, w = |curl v| h / (|v| + c);
// compressed as log(1 + 100 x).
template<class M>
__device__ __forceinline__ void forecast_scales(const Pool &P, const Consts &C, int i, double *abw, double *vel) {
	constexpr int D = M::D, E = M::E;
	double p[E];
	load_p<M>(P, i, p);
	const double h   = C.size[P.level[i]];
	const double rho = M::MULTI ? p[0] + p[1] : p[0];
	double gr = 0.0, gp = 0.0, v2 = 0.0;
	for (int d = 0; d < D; ++d) {
		const double sr = M::MULTI ? rec_slope<M>(P, i, d, 0) + rec_slope<M>(P, i, d, 1) : rec_slope<M>(P, i, d, 0);
		const double sp = rec_slope<M>(P, i, d, M::IP);
		gr += sr * sr;
		gp += sp * sp;
		v2 += p[M::IU + d] * p[M::IU + d];
	}
	double w2 = 0.0;
	if constexpr (D == 2) {
		const double w = rec_slope<M>(P, i, 0, M::IU + 1) - rec_slope<M>(P, i, 1, M::IU);
		w2 = w * w;
	} else if constexpr (D == 3) {
		for (int a = 0; a < 3; ++a) {
			const int b = (a + 1) % 3, c = (a + 2) % 3;
			const double w = rec_slope<M>(P, i, b, M::IU + c) - rec_slope<M>(P, i, c, M::IU + b);
			w2 += w * w;
		}
	}
	const double cs   = sound_speed<M>(C.m, p);
	const double vref = sqrt(v2) + cs;
	abw[0] = log1p(100.0 * sqrt(gr) * h / fabs(rho));
	abw[1] = log1p(100.0 * sqrt(gp) * h / fabs(p[M::IP]));
	abw[2] = log1p(100.0 * sqrt(w2) * h / vref);
	for (int d = 0; d < D; ++d) vel[d] = p[M::IU + d] / vref;
}

// Forecaster features of the listed leaves, FORECAST_F(D) = 5 + 5D doubles each: the cell's a, b, w,
// level / 16 and log(1 + err / max_err), its velocity over (|v| + c) per dimension, then a and b of the
// neighbour behind each face (the cell's own where the face is a boundary or the neighbour is refined).
template<class M>
__global__ void k_forecast_features(Pool P, Consts C, const int32_t *list, int n, int base, double *out) {
	constexpr int D = M::D, NF = 2 * D, F = 5 + 5 * D;
	const int cap = P.cap;
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		double *o   = out + (size_t) (base + tid) * F;
		double abw[3], vel[D];
		forecast_scales<M>(P, C, i, abw, vel);
		o[0] = abw[0];
		o[1] = abw[1];
		o[2] = abw[2];
		o[3] = P.level[i] / 16.0;
		o[4] = log1p(fmax(P.err[i], 0.0) / C.max_err);
		for (int d = 0; d < D; ++d) o[5 + d] = vel[d];
		for (int f = 0; f < NF; ++f) {
			const int j = P.nbr[(size_t) f * cap + i];
			double a = abw[0], b = abw[1];
			if (j > 0 && (P.flags[j] & F_LEAF)) {
				double nabw[3], nvel[D];
				forecast_scales<M>(P, C, j, nabw, nvel);
				a = nabw[0], b = nabw[1];
			}
			o[5 + D + 2 * f]     = a;
			o[5 + D + 2 * f + 1] = b;
		}
	}
}

// Sets (hold[base + tid] != 0) or clears F_HOLD on the listed leaves.
template<class M>
__global__ void k_set_hold(Pool P, const int32_t *list, int n, int base, const uint8_t *hold) {
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		P.flags[i]  = hold[base + tid] ? (P.flags[i] | F_HOLD) : (P.flags[i] & ~F_HOLD);
	}
}

// Gather of active-cell records for the read-back API.
template<class M>
__global__ void k_gather_cells(Pool P, const int32_t *list, int n, int base, double *out, int32_t *lv) {
	constexpr int E = M::E, D = M::D, W = D + 1 + 2 * E + 3 + M::P;
	const int cap = P.cap;
	for (int tid = gtid(); tid < n; tid += gstride()) {
		const int i = list[tid];
		const int r = base + tid;
		lv[2 * r]     = P.level[i];
		lv[2 * r + 1] = P.acti[i];
		double *o     = out + (size_t) r * W;
		int k         = 0;
		for (int d = 0; d < D; ++d) o[k++] = at(P.center, cap, d, i);
		o[k++] = P.t[i];
		for (int q = 0; q < E; ++q) o[k++] = at(P.u, cap, q, i);
		for (int q = 0; q < E; ++q) o[k++] = at(P.p, cap, q, i);
		o[k++] = P.err[i];
		o[k++] = P.maxdt[i];
		o[k++] = P.cfl[i];
		for (int q = 0; q < M::P; ++q) o[k++] = at(P.k, cap, q, i);
	}
}

}  // namespace dg

namespace dg {

// --------------------------------------------------------------------------------------------
// Multiphase auxiliary stages (impl/smooth.hpp, impl/normal_curvature.hpp)
// --------------------------------------------------------------------------------------------

// Value of a parameter component on the far side of face (dim, dir): the boundary ghost's volume
// fraction, the recursive child mean of k[comp] for finer neighbours, else the neighbour's k[comp].
// `x` receives the centre distance used by compute_normal/compute_curvature (half a cell at a
// boundary, impl/normal_curvature.hpp:161-183).
// The smoothed volume fraction of node x during the Jacobi sweeps of a cell list: the previous sweep's
// result for members of the list (cur, after the first sweep), the stored k[ALPHAS] for everyone else.
// Lm >= 0: members are the cells of cluster Lm; Lm < 0: every leaf (the constructor's list).
template<class M>
__device__ __forceinline__ double alpha_now(const Pool &P, int x, const double *cur, int Lm) {
	if (cur && (Lm < 0 || P.clu[x] == Lm)) return cur[x];
	return at(P.k, P.cap, M::ALPHAS, x);
}

template<class M>
__device__ double k_side(const Pool &P, const Consts &C, const BcTable &B, uint32_t *status, int i, int dim, int dir,
                         int comp, bool zero_at_boundary, double &x, const double *cur = nullptr, int Lm = -1,
                         int epoch = 0, int e_upd = 0) {
	const int cap  = P.cap;
	const int nb   = P.nbr[(size_t) (2 * dim + dir) * cap + i];
	const double h = C.size[P.level[i]];
	if (nb == 0) {
		x = dir == 0 ? -0.5 * h : 0.5 * h;
		if (zero_at_boundary) return 0.0;
		const int b = P.bc[(size_t) (2 * dim + dir) * cap + i];
		double pc[M::E], pb[M::E];
		load_p<M>(P, i, pc);
		if (b < 0) {
			set_status(status, ST_MISSING_BC);
			return pc[M::IA];
		}
		boundary_value<M>(C.m, B, b, pc, P.t[i], pb);
		return pb[M::IA];
	}
	const double hn = C.size[P.level[nb]];
	x = dir == 0 ? -0.5 * (h + hn) : 0.5 * (h + hn);
	if (comp == M::ALPHAS) {
		auto val = [&](int y) { return alpha_now<M>(P, y, cur, Lm); };
		if (!(P.flags[nb] & F_LEAF)) return interp_alpha<M::D>(P, status, nb, val, epoch, e_upd);
		return val(nb);
	}
	if (!(P.flags[nb] & F_LEAF)) return interp_scalar<M::D>(P, status, nb, P.k + (size_t) comp * cap);
	return at(P.k, cap, comp, nb);
}

// smooth_alpha, one Jacobi sweep (impl/smooth.hpp:10-51): reads the previous sweep's values of the
// list's cells from `cur` (nullptr for the first sweep: everything from k[ALPHAS]) and writes `out`;
// the sweeps alternate between two scratch arrays and the last writes k[ALPHAS] itself (the list's own
// values are read from `cur` throughout, so that write races with no read). A group of G lanes per cell:
// lane f fetches the smoothed volume fraction across face f, the dimension's two lanes form its term
// 0.5 (a_n + a_p) + a_c, and the group's first lane sums the dimensions in order.
template<class M, class Grid>
__device__ __forceinline__ void d_smooth_alpha(const Grid &g, const Pool &P, const Consts &C, const BcTable &B,
                                               const int32_t *list, int n, const double *cur, double *out, int Lm,
                                               int epoch, int e_upd, Counters *cnt) {
	constexpr int D = M::D, NF = 2 * D, G = NF, GW = 32 / G;  // lanes per cell, cells per warp
	const int lane   = threadIdx.x & 31;
	const int grp    = lane / G;  // the lane's cell within the warp; lanes past GW * G idle
	const int sub    = lane - grp * G;
	const int base   = grp * G;
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot    = wbase + grp;
		const bool active = grp < GW && slot < n;
		const int i       = active ? list[slot] : 0;
		double v = 0.0, x = 0.0;
		if (active && sub < NF) v = k_side<M>(P, C, B, &cnt->status, i, sub >> 1, sub & 1, M::ALPHAS, false, x, cur, Lm, epoch, e_upd);
		const double vp = __shfl_sync(0xffffffffu, v, base + (sub | 1));
		double term = 0.0;
		if (active && sub < NF && !(sub & 1)) {
			const double ac = cur ? cur[i] : at(P.k, P.cap, M::ALPHAS, i);
			term = 0.5 * (v + vp) + ac;
		}
		double terms[D];
#pragma unroll
		for (int d = 0; d < D; ++d) terms[d] = __shfl_sync(0xffffffffu, term, min(base + 2 * d, 31));
		if (active && sub == 0) {
			double s = 0.0;
			for (int d = 0; d < D; ++d) s += terms[d];
			out[i] = s / (double) (2 * D);
		}
	}
}
template<class M>
__global__ void __launch_bounds__(BLOCK) k_smooth_alpha(Pool P, Consts C, BcTable B, const int32_t *list, int n,
                                                        const double *cur, double *out, int Lm, int epoch, int e_upd,
                                                        Counters *cnt) {
	d_smooth_alpha<M>(PlainGrid{}, P, C, B, list, n, cur, out, Lm, epoch, e_upd, cnt);
}

template<class Grid>
__device__ __forceinline__ void d_store_tmp(const Grid &g, const Pool &P, const int32_t *list, int n, int comp, const double *src) {
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int i = list[tid];
		P.k[(size_t) comp * P.cap + i] = src[i];
	}
}
static __global__ void k_store_tmp(Pool P, const int32_t *list, int n, int comp, const double *src) {
	d_store_tmp(PlainGrid{}, P, list, n, comp, src);
}

// compute_normal (impl/normal_curvature.hpp:7-55), a group of G lanes per cell as in smooth_alpha:
// lane f fetches the volume fraction across face f and its centre distance, the dimension's two lanes
// form that gradient component, the first lane normalises and writes.
template<class M, class Grid>
__device__ __forceinline__ void d_normal(const Grid &g, const Pool &P, const Consts &C, const BcTable &B,
                                         const int32_t *list, int n, int epoch, int e_upd, Counters *cnt) {
	constexpr int D = M::D, NF = 2 * D, G = NF, GW = 32 / G;  // lanes per cell, cells per warp
	const int cap    = P.cap;
	const int lane   = threadIdx.x & 31;
	const int grp    = lane / G;  // the lane's cell within the warp; lanes past GW * G idle
	const int sub    = lane - grp * G;
	const int base   = grp * G;
	const int warp   = g.tid() >> 5;
	const int nwarps = g.stride() >> 5;
	for (int wbase = warp * GW; wbase < n; wbase += nwarps * GW) {
		const int slot    = wbase + grp;
		const bool active = grp < GW && slot < n;
		const int i       = active ? list[slot] : 0;
		double v = 0.0, x = 0.0;
		if (active && sub < NF) v = k_side<M>(P, C, B, &cnt->status, i, sub >> 1, sub & 1, M::ALPHAS, false, x, nullptr, -1, epoch, e_upd);
		const double vp = __shfl_sync(0xffffffffu, v, base + (sub | 1));
		const double xp = __shfl_sync(0xffffffffu, x, base + (sub | 1));
		double comp = 0.0;
		if (active && sub < NF && !(sub & 1)) comp = (vp - v) / (xp - x);
		double nrm[D];
#pragma unroll
		for (int d = 0; d < D; ++d) nrm[d] = __shfl_sync(0xffffffffu, comp, min(base + 2 * d, 31));
		if (!active || sub != 0) continue;
		double sq = 0.0;
		for (int d = 0; d < D; ++d) sq += nrm[d] * nrm[d];
		const double len = sqrt(sq);
		for (int d = 0; d < D; ++d) nrm[d] = (len < 1e-10) ? 0.0 : nrm[d] / len;
		for (int d = 0; d < D; ++d) P.k[(size_t) (M::IKN + d) * cap + i] = nrm[d];
		// the record's multiphase part (curvature is final here unless surface tension recomputes it)
		double *kr = rec_of(P, i, Rec<M>::W) + Rec<M>::K0;
		kr[0] = at(P.k, cap, M::KAPPA, i);
		for (int d = 0; d < D; ++d) kr[1 + d] = nrm[d];
	}
}
template<class M>
__global__ void __launch_bounds__(BLOCK) k_normal(Pool P, Consts C, BcTable B, const int32_t *list, int n, int epoch,
                                                  int e_upd, Counters *cnt) {
	d_normal<M>(PlainGrid{}, P, C, B, list, n, epoch, e_upd, cnt);
}

// compute_curvature (impl/normal_curvature.hpp:59-102)
template<class M, class Grid>
__device__ __forceinline__ void d_curvature(const Grid &g, const Pool &P, const Consts &C, const BcTable &B, const int32_t *list, int n, Counters *cnt) {
	const int cap = P.cap;
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int i  = list[tid];
		double kappa = 0.0;
		for (int dim = 0; dim < M::D; ++dim) {
			double xn, xp;
			const double nn = k_side<M>(P, C, B, &cnt->status, i, dim, 0, M::IKN + dim, true, xn);
			const double np = k_side<M>(P, C, B, &cnt->status, i, dim, 1, M::IKN + dim, true, xp);
			kappa -= (np - nn) / (xp - xn);
		}
		P.k[(size_t) M::KAPPA * cap + i] = kappa;
	}
}
template<class M>
__global__ void k_curvature(Pool P, Consts C, BcTable B, const int32_t *list, int n, Counters *cnt) {
	d_curvature<M>(PlainGrid{}, P, C, B, list, n, cnt);
}

// smooth_curvature, one weighted sweep into P.tmp (impl/smooth.hpp:63-133)
template<class M, class Grid>
__device__ __forceinline__ void d_smooth_kappa(const Grid &g, const Pool &P, const Consts &C, const BcTable &B, const int32_t *list, int n, Counters *cnt) {
	const int cap = P.cap;
	for (int tid = g.tid(); tid < n; tid += g.stride()) {
		const int i     = list[tid];
		const double kc = at(P.k, cap, M::KAPPA, i);
		const double as = at(P.k, cap, M::ALPHAS, i);
		const double xc = as * (1 - as);
		const double wc = xc * xc;
		double ks = 0.0, w = 0.0;
		for (int dim = 0; dim < M::D; ++dim) {
			double kv[2], av[2];
			for (int dir = 0; dir < 2; ++dir) {
				const int nb = P.nbr[(size_t) (2 * dim + dir) * cap + i];
				if (nb == 0) {
					kv[dir] = 0.0;
					const int b = P.bc[(size_t) (2 * dim + dir) * cap + i];
					double pc[M::E], pb[M::E];
					load_p<M>(P, i, pc);
					if (b < 0) {
						set_status(&cnt->status, ST_MISSING_BC);
						av[dir] = pc[M::IA];
					} else {
						boundary_value<M>(C.m, B, b, pc, P.t[i], pb);
						av[dir] = pb[M::IA];
					}
				} else if (!(P.flags[nb] & F_LEAF)) {
					kv[dir] = interp_scalar<M::D>(P, &cnt->status, nb, P.k + (size_t) M::KAPPA * cap);
					av[dir] = interp_scalar<M::D>(P, &cnt->status, nb, P.p + (size_t) M::IA * cap);
				} else {
					kv[dir] = at(P.k, cap, M::KAPPA, nb);
					av[dir] = at(P.p, cap, M::IA, nb);
				}
			}
			const double xn = av[0] * (1 - av[0]), xp = av[1] * (1 - av[1]);
			const double wn = xn * xn, wp = xp * xp;
			ks += 0.5 * (wn * kv[0] + wp * kv[1]) + kc * wc;
			w += 0.5 * (wn + wp) + wc;
		}
		P.tmp[i] = (w > 1e-6) ? ks / w : 0.0;
	}
}
template<class M>
__global__ void k_smooth_kappa(Pool P, Consts C, BcTable B, const int32_t *list, int n, Counters *cnt) {
	d_smooth_kappa<M>(PlainGrid{}, P, C, B, list, n, cnt);
}

// --------------------------------------------------------------------------------------------
// Garbage collection (integrator/domain.hpp:327-356): order-preserving compaction of the non-garbage
// slots with every link remapped (links to removed slots become 0).
// --------------------------------------------------------------------------------------------
static __global__ void k_gc_keep(Pool P, int top, int32_t *keep) {
	for (int i = gtid(); i < top; i += gstride()) keep[i] = (i == 0 || !(P.flags[i] & F_GARBAGE)) ? 1 : 0;
}

// Moves component c of every kept slot of `src` to its new index in `dst` (elem bytes per entry).
static __global__ void k_gc_move(const char *src, char *dst, int elem, int comps, int cap, int top, const int32_t *keep,
                          const int32_t *newidx) {
	for (int i = gtid(); i < top; i += gstride()) {
		if (!keep[i]) continue;
		const int j = newidx[i];
		for (int c = 0; c < comps; ++c) {
			const size_t so = ((size_t) c * cap + i) * elem, dof = ((size_t) c * cap + j) * elem;
			if (elem % 8 == 0) {
				for (int b = 0; b < elem; b += 8) *(double *) (dst + dof + b) = *(const double *) (src + so + b);
			} else {
				for (int b = 0; b < elem; ++b) dst[dof + b] = src[so + b];
			}
		}
	}
}

template<int D>
__global__ void k_gc_remap(Pool P, int new_top, const int32_t *keep, const int32_t *newidx) {
	constexpr int NC = 1 << D, NF = 2 * D;
	const int cap = P.cap;
	for (int j = gtid(); j < new_top; j += gstride()) {
		auto mapv = [&](int32_t old) { return (old > 0 && keep[old]) ? newidx[old] : 0; };
		P.parent[j] = mapv(P.parent[j]);
		for (int c = 0; c < NC; ++c) P.child[(size_t) c * cap + j] = mapv(P.child[(size_t) c * cap + j]);
		for (int f = 0; f < NF; ++f) P.nbr[(size_t) f * cap + j] = mapv(P.nbr[(size_t) f * cap + j]);
		P.clu[j] = CLU_NONE;
	}
}

static __global__ void k_collect_active_leaves(Pool P, int top, int32_t *out, int *count) {
	for (int i = gtid(); i < top; i += gstride()) {
		if (i == 0) continue;
		const uint32_t f = P.flags[i];
		if ((f & F_LEAF) && (f & F_ACTIVE) && !(f & F_GARBAGE)) {
			int pos  = atomicAdd(count, 1);
			out[pos] = i;
		}
	}
}

}  // namespace dg

namespace dg {

// --------------------------------------------------------------------------------------------
// Level-bucketed Morton re-sort of the node pool. Leaves of cluster L (then of buffer L) become one
// contiguous, Z-ordered slot range; other slots keep their relative order after them. A pure
// permutation: links are remapped and nothing the reference can observe changes.
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t spread2(uint64_t x) {  // 29 bits -> even positions
	x &= 0x1fffffffull;
	x = (x | (x << 16)) & 0x0000ffff0000ffffull;
	x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
	x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
	x = (x | (x << 2)) & 0x3333333333333333ull;
	x = (x | (x << 1)) & 0x5555555555555555ull;
	return x;
}
__device__ __forceinline__ uint64_t spread3(uint64_t x) {  // 19 bits -> every third position
	x &= 0x7ffffull;
	x = (x | (x << 32)) & 0x1f00000000ffffull;
	x = (x | (x << 16)) & 0x1f0000ff0000ffull;
	x = (x | (x << 8)) & 0x100f00f00f00f00full;
	x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
	x = (x | (x << 2)) & 0x1249249249249249ull;
	return x;
}

template<int D>
__global__ void k_sort_keys(Pool P, int top, uint64_t *keys, int32_t *vals) {
	constexpr int LMAX = D == 2 ? 29 : 19;
	for (int j = gtid(); j < top - 1; j += gstride()) {
		const int i     = j + 1;
		const int8_t cl = P.clu[i];
		uint64_t code   = cl >= 0 ? (uint64_t) cl : 63ull;
		uint64_t m      = 0;
		if (cl >= 0) {
			const int l  = P.level[i];
			const int sh = LMAX - l;
			for (int d = 0; d < D; ++d) {
				uint64_t c = (uint64_t) P.coord[(size_t) d * P.cap + i];
				c          = sh >= 0 ? (c << sh) : (c >> (-sh));
				m |= (D == 2 ? spread2(c) : spread3(c)) << d;
			}
		} else {
			m = (uint64_t) i;
		}
		keys[j] = (code << 58) | (m & ((1ull << 58) - 1));
		vals[j] = i;
	}
}

static __global__ void k_sort_inverse(const int32_t *sorted_vals, int n, int32_t *newidx) {
	for (int j = gtid(); j < n; j += gstride()) newidx[sorted_vals[j]] = j + 1;
	if (gtid() == 0) newidx[0] = 0;
}

template<typename T>
__global__ void k_permute(const T *__restrict__ src, T *__restrict__ dst, int comps, int cap, int n,
                          const int32_t *__restrict__ perm) {
	for (int j = gtid(); j < n; j += gstride()) {
		const int o = perm[j];
		for (int c = 0; c < comps; ++c) dst[(size_t) c * cap + j + 1] = src[(size_t) c * cap + o];
	}
}

// Permutation of a field holding one record of w 8-byte words per node: word-parallel copies.
static __global__ void k_permute_words(const double *__restrict__ src, double *__restrict__ dst, int w, int n,
                                       const int32_t *__restrict__ perm) {
	const long long total = (long long) n * w;
	for (long long t = gtid(); t < total; t += gstride()) {
		const int j = (int) (t / w), k = (int) (t % w);
		dst[(size_t) (j + 1) * w + k] = src[(size_t) perm[j] * w + k];
	}
}

template<int D>
__global__ void k_remap_links(Pool P, int top, const int32_t *newidx) {
	constexpr int NC = 1 << D, NF = 2 * D;
	const int cap = P.cap;
	for (int j = gtid(); j < top; j += gstride()) {
		if (j == 0) continue;
		P.parent[j] = newidx[P.parent[j]];
		for (int c = 0; c < NC; ++c) P.child[(size_t) c * cap + j] = newidx[P.child[(size_t) c * cap + j]];
		for (int f = 0; f < NF; ++f) P.nbr[(size_t) f * cap + j] = newidx[P.nbr[(size_t) f * cap + j]];
	}
}

static __global__ void k_fill_i32(int32_t *a, int v, int n) {
	for (int j = gtid(); j < n; j += gstride()) a[j] = v;
}

static __global__ void k_fill_range(int32_t *list, int first, int n) {
	for (int j = gtid(); j < n; j += gstride()) list[j] = first + j;
}

}  // namespace dg
