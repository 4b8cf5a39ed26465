// Physics of the three DACTI model policies as device functions.
//
// Every function keeps the reference's floating-point operation order (left-to-right C++
// evaluation, no reassociation) so that, compiled with --fmad=false, the FP64 results are
// bit-identical to the reference CPU solver. Line citations are to the reference's model headers.
#pragma once

#include "dg_types.h"

namespace dg {

// std::min / std::max semantics (first argument returned on ties and NaN comparisons).
template<class S>
__host__ __device__ __forceinline__ S smin(S a, S b) { return (b < a) ? b : a; }
template<class S>
__host__ __device__ __forceinline__ S smax(S a, S b) { return (a < b) ? b : a; }

// a[LO + k] and a[LO + k] (+)= v for a run-time k in [0, N): unrolled selects keep small state arrays in
// registers where a dynamic index would move them to local memory.
template<int LO, int N, class S>
__device__ __forceinline__ S pick(const S *a, int k) {
	S r = a[LO];
#pragma unroll
	for (int j = 1; j < N; ++j)
		if (k == j) r = a[LO + j];
	return r;
}
template<int LO, int N, class S>
__device__ __forceinline__ void put(S *a, int k, S v) {
#pragma unroll
	for (int j = 0; j < N; ++j)
		if (k == j) a[LO + j] = v;
}
template<int LO, int N, class S>
__device__ __forceinline__ void put_add(S *a, int k, S v) {
#pragma unroll
	for (int j = 0; j < N; ++j)
		if (k == j) a[LO + j] += v;
}

// --------------------------------------------------------------------------------------------
// Model traits (compile-time sizes of model/euler.hpp:26-32, navier_stokes.hpp:351, multi.hpp:27-42)
// --------------------------------------------------------------------------------------------
template<int D_>
struct Euler {
	static constexpr int D = D_, E = D + 2, F = E, G = 0, P = 0, IU = 1, IP = E - 1, IA = -1;
	static constexpr bool MULTI = false, VISC = false, HEAT = false, SOURCE = false;
	static constexpr int ID = 0;
};
template<int D_>
struct NavierStokes {
	static constexpr int D = D_, E = D + 2, F = E, G = D + 1, P = 0, IU = 1, IP = E - 1, IA = -1;
	static constexpr int DT = D;
	static constexpr bool MULTI = false, VISC = true, HEAT = true, SOURCE = false;
	static constexpr int ID = 1;
};
template<int D_>
struct Multi {
	static constexpr int D = D_, E = D + 4, F = E + D + 1, G = D + 3, P = D + 4, IU = 2, IP = E - 2, IA = E - 1;
	static constexpr int IKN = 2, KAPPA = IKN + D, ALPHAS = KAPPA + 1, DT = D, DA = D + 1;
	static constexpr bool MULTI = true, VISC = true, HEAT = true, SOURCE = true;
	static constexpr int ID = 2;
};

constexpr double EULER_GAMMA = 1.4;      // model/euler.hpp:34
constexpr double NS_CP       = 1005.0;   // model/navier_stokes.hpp:353
constexpr double NS_R        = 287.0;    // model/navier_stokes.hpp:354
constexpr double MULTI_EPS   = 1e-20;    // model/multi.hpp:47
constexpr double MULTI_UC    = 1.0;      // model/multi.hpp:48

// --------------------------------------------------------------------------------------------
// Stiffened-gas mixture closures (model/multi.hpp:367-430)
// --------------------------------------------------------------------------------------------
template<class S = double>
__device__ __forceinline__ S mix_gamma(const ModelConsts &m, S a) {
	const S g1 = (S) m.gamma1, g2 = (S) m.gamma2;
	if (a < (S) MULTI_EPS) return g2;
	else if (a > 1 - (S) MULTI_EPS) return g1;
	else return 1 + 1 / (a / (g1 - 1) + (1 - a) / (g2 - 1));
}
template<class S = double>
__device__ __forceinline__ S mix_p0(const ModelConsts &m, S a) {
	const S g1 = (S) m.gamma1, g2 = (S) m.gamma2, P1 = (S) m.P1, P2 = (S) m.P2;
	if (a < (S) MULTI_EPS) return P2;
	else if (a > 1 - (S) MULTI_EPS) return P1;
	else return (a * g1 * P1 / (g1 - 1) + (1 - a) * g2 * P2 / (g2 - 1)) / (1 + a / (g1 - 1) + (1 - a) / (g2 - 1));
}
__device__ __forceinline__ double mix_temperature(const ModelConsts &m, double r0, double r1, double p, double a) {
	if (a < MULTI_EPS) return (p + m.P2) / ((m.gamma2 - 1) * r1 * m.cv2);
	else if (a > 1 - MULTI_EPS) return (p + m.P1) / ((m.gamma1 - 1) * r0 * m.cv1);
	else
		return (p / (mix_gamma(m, a) - 1) + a * m.P1 / (m.gamma1 - 1) + (1 - a) * m.P2 / (m.gamma2 - 1)) /
		       (r0 * m.cv1 + r1 * m.cv2);
}

// --------------------------------------------------------------------------------------------
// Sound speed, pressure and variable conversions
// --------------------------------------------------------------------------------------------
template<class M, class S = double>
__device__ __forceinline__ S sound_speed_rp(const ModelConsts &m, S r0, S r1, S p, S a) {
	if constexpr (M::MULTI) return sqrt(mix_gamma<S>(m, a) * (p + mix_p0<S>(m, a)) / (r0 + r1));
	else return sqrt((S) EULER_GAMMA * p / r0);
}
template<class M>
__device__ __forceinline__ double sound_speed(const ModelConsts &m, const double *p) {
	if constexpr (M::MULTI) return sqrt(mix_gamma(m, p[M::IA]) * (p[M::IP] + mix_p0(m, p[M::IA])) / (p[0] + p[1]));
	else return sqrt(EULER_GAMMA * p[M::IP] / p[0]);
}
template<class M, class S = double>
__device__ __forceinline__ S sound_speed_2(const ModelConsts &m, S r0, S r1, S p, S a) {
	if constexpr (M::MULTI) return mix_gamma<S>(m, a) * (p + mix_p0<S>(m, a)) / (r0 + r1);
	else return (S) EULER_GAMMA * p / r0;
}

// supersonic (model/euler.hpp:250-256, model/multi.hpp:432-438). The multiphase version passes
// the scalar p[0] where a pair of phase densities is expected, so the "mixture" density is
// (alpha1 rho1, 0) and only p[0] enters the sound speed.
template<class M, class S = double>
__device__ __forceinline__ bool supersonic(const ModelConsts &m, const S *p) {
	S u2 = 0;
	for (int i = 0; i < M::D; ++i) u2 += p[M::IU + i] * p[M::IU + i];
	if constexpr (M::MULTI) return u2 > sound_speed_2<M, S>(m, p[0], (S) 0, p[M::IP], p[M::IA]);
	else return u2 > sound_speed_2<M, S>(m, p[0], (S) 0, p[M::IP], (S) 0);
}

template<class M>
__device__ __forceinline__ double pressure(const ModelConsts &m, const double *u) {
	double ke = 0;
	for (int i = 0; i < M::D; ++i) ke += 0.5 * u[M::IU + i] * u[M::IU + i];
	if constexpr (M::MULTI) {
		double g = mix_gamma(m, u[M::IA]);
		return (g - 1) * (u[M::IP] - ke / (u[0] + u[1])) - mix_gamma(m, u[M::IA]) * mix_p0(m, u[M::IA]);
	} else {
		return (EULER_GAMMA - 1) * (u[M::IP] - ke / u[0]);
	}
}

// primitive_variables (model/euler.hpp:266-274, model/multi.hpp:448-458)
template<class M>
__device__ __forceinline__ void prim_from_cons(const ModelConsts &m, const double *u, double *p) {
	if constexpr (M::MULTI) {
		p[0] = u[0];
		p[1] = u[1];
		for (int i = 0; i < M::D; ++i) p[M::IU + i] = u[M::IU + i] / (u[0] + u[1]);
		p[M::IP] = pressure<M>(m, u);
		p[M::IA] = u[M::IA];
	} else {
		p[0] = u[0];
		for (int i = 0; i < M::D; ++i) p[M::IU + i] = u[M::IU + i] / u[0];
		p[M::IP] = pressure<M>(m, u);
	}
}

// conserved_variables (model/euler.hpp:276-286, model/multi.hpp:460-472)
template<class M>
__device__ __forceinline__ void cons_from_prim(const ModelConsts &m, const double *p, double *u) {
	double ke = 0;
	if constexpr (M::MULTI) {
		u[0] = p[0];
		u[1] = p[1];
		for (int i = 0; i < M::D; ++i) {
			u[M::IU + i] = (p[0] + p[1]) * p[M::IU + i];
			ke += 0.5 * p[M::IU + i] * p[M::IU + i];
		}
		double a = p[M::IA];
		u[M::IP] = (p[M::IP] + mix_gamma(m, a) * mix_p0(m, a)) / (mix_gamma(m, a) - 1) + (p[0] + p[1]) * ke;
		u[M::IA] = p[M::IA];
	} else {
		u[0] = p[0];
		for (int i = 0; i < M::D; ++i) {
			u[M::IU + i] = p[0] * p[M::IU + i];
			ke += 0.5 * p[M::IU + i] * p[M::IU + i];
		}
		u[M::IP] = p[M::IP] / (EULER_GAMMA - 1) + p[0] * ke;
	}
}

// get_grad_input (model/navier_stokes.hpp:377-385, model/multi.hpp:148-156)
template<class M>
__device__ __forceinline__ void grad_input(const ModelConsts &m, const double *p, double *g) {
	if constexpr (M::G > 0) {
		for (int i = 0; i < M::D; ++i) g[i] = p[M::IU + i];
		if constexpr (M::MULTI) {
			g[M::DT] = mix_temperature(m, p[0], p[1], p[M::IP], p[M::IA]);
			g[M::DA] = p[M::IA];
			g[M::DA + 1] = 0.0;  // dbeta: never read; left unset by multi::get_grad_input
		} else {
			g[M::DT] = p[M::IP] / (p[0] * NS_R);
		}
	}
}

// mu / lambda (model/navier_stokes.hpp:419-425, model/multi.hpp:313-319)
template<class M, class S = double>
__device__ __forceinline__ S visc_mu(const ModelConsts &m, const S *p) {
	if constexpr (M::MULTI) return (S) m.mu1 * p[M::IA] + (S) m.mu2 * (1 - p[M::IA]);
	else return (S) m.ns_mu;
}
template<class M, class S = double>
__device__ __forceinline__ S visc_lambda(const ModelConsts &m, const S *p) {
	if constexpr (M::MULTI) return (S) m.lambda1 * p[M::IA] + (S) m.lambda2 * (1 - p[M::IA]);
	else return (S) m.ns_lambda;
}

// max_delta_time (model/euler.hpp:203-215, navier_stokes.hpp:427-440, multi.hpp:322-346)
template<class M>
__device__ __forceinline__ double max_delta_time(const ModelConsts &m, const double *p, double size) {
	double c = sound_speed<M>(m, p);
	double mn = 0;
	for (int i = 0; i < M::D; ++i) {
		double dti = size / (c + fabs(p[M::IU + i]));
		mn = (i == 0) ? dti : smin(mn, dti);
	}
	if constexpr (!M::VISC) {
		return mn;
	} else if constexpr (M::MULTI) {
		double k = smax(visc_mu<M>(m, p), visc_lambda<M>(m, p) / smin(m.cp1, m.cp2));
		if (k < 1e-15) return mn;
		double dv = size * size / k / 4.0;
		return smin(mn, dv);
	} else {
		double k = smax(m.ns_mu, m.ns_lambda / NS_CP);
		if (k < 1e-15) return mn;
		double dv = size * size / k * 0.5;
		return smin(mn, dv);
	}
}

// --------------------------------------------------------------------------------------------
// Physical fluxes (model/euler.hpp:50-83, model/multi.hpp:78-123). `F` must be zeroed by the caller
// semantics: every component not written here is 0.
// --------------------------------------------------------------------------------------------
template<class M, class S = double>
__device__ __forceinline__ void phys_flux(const ModelConsts &m, const S *p, S un, int dim, bool projected, S *F) {
	constexpr int D = M::D;
	S vn         = projected ? un : pick<M::IU, D>(p, dim);
	S ke         = 0;
	for (int q = 0; q < M::F; ++q) F[q] = 0;
	if constexpr (M::MULTI) {
		for (int i = 0; i < M::D; ++i) {
			F[M::IU + i] = (p[0] + p[1]) * vn * p[M::IU + i];
			ke += 0.5 * p[M::IU + i] * p[M::IU + i];
		}
		F[0] = vn * p[0];
		F[1] = vn * p[1];
		put_add<M::IU, D>(F, dim, p[M::IP]);
		S a      = p[M::IA];
		F[M::IP] = vn * (mix_gamma<S>(m, a) / (mix_gamma<S>(m, a) - 1) * (p[M::IP] + mix_p0<S>(m, a)) + ke * (p[0] + p[1]));
		F[M::IA] = vn * p[M::IA];
		F[M::IA + 1] = vn;
		put<M::IA + 2, D>(F, dim, p[M::IA]);
	} else {
		for (int i = 0; i < M::D; ++i) {
			F[M::IU + i] = p[0] * vn * p[M::IU + i];
			ke += 0.5 * p[M::IU + i] * p[M::IU + i];
		}
		F[0] = vn * p[0];
		put_add<M::IU, D>(F, dim, p[M::IP]);
		F[M::IP] = vn * ((S) (EULER_GAMMA / (EULER_GAMMA - 1)) * p[M::IP] + ke * p[0]);
	}
}

// middle_state (model/euler.hpp:118-153, model/multi.hpp:205-246): the HLLC-type star state in
// primitive variables; `ka` enters only the multiphase contact speed.
template<class M, class S = double>
__device__ __forceinline__ void middle_state(const ModelConsts &m, const S *pn, const S *pp, S ka, int dim, S *pm) {
	constexpr int D = M::D;
	const int ip = M::IP;
	const S un = pick<M::IU, D>(pn, dim), up = pick<M::IU, D>(pp, dim);
	S c_n, c_p, rn, rp;
	if constexpr (M::MULTI) {
		c_n = sound_speed_rp<M, S>(m, pn[0], pn[1], pn[ip], pn[M::IA]);
		c_p = sound_speed_rp<M, S>(m, pp[0], pp[1], pp[ip], pp[M::IA]);
		rn  = pn[0] + pn[1];
		rp  = pp[0] + pp[1];
	} else {
		c_n = sqrt((S) EULER_GAMMA * pn[ip] / pn[0]);
		c_p = sqrt((S) EULER_GAMMA * pp[ip] / pp[0]);
		rn  = pn[0];
		rp  = pp[0];
	}
	S u  = (S) 0.5 * (un + up);
	S c  = (S) 0.5 * (c_n + c_p);
	S Sn = smin<S>(u - c, un - c_n);
	S Sp = smax<S>(u + c, up + c_p);
	S Sm;
	if constexpr (M::MULTI)
		Sm = (pp[ip] - pn[ip] + rn * un * (Sn - un) - rp * up * (Sp - up) - (S) m.sigma * ka * (pp[M::IA] - pn[M::IA])) /
		     (rn * (Sn - un) - rp * (Sp - up));
	else
		Sm = (pp[ip] - pn[ip] + pn[0] * un * (Sn - un) - pp[0] * up * (Sp - up)) /
		     (pn[0] * (Sn - un) - pp[0] * (Sp - up));

	for (int q = 0; q < M::E; ++q) pm[q] = 0;
	if (Sn > 0) {
		for (int q = 0; q < M::E; ++q) pm[q] = pn[q];
	} else if (Sp < 0) {
		for (int q = 0; q < M::E; ++q) pm[q] = pp[q];
	} else if (Sm > 0 && Sn < 0) {
		if constexpr (M::MULTI) {
			pm[0]      = pn[0] * (Sn - un) / (Sn - Sm);
			pm[1]      = pn[1] * (Sn - un) / (Sn - Sm);
			pm[ip]     = pn[ip] + (pn[0] + pn[1]) * (Sn - un) * (Sm - un);
			pm[M::IA]  = pn[M::IA];
		} else {
			pm[0]  = pn[0] * (Sn - un) / (Sn - Sm);
			pm[ip] = pn[ip] + pn[0] * (Sn - un) * (Sm - un);
		}
		for (int i = 0; i < M::D; ++i) pm[M::IU + i] = pn[M::IU + i];
		put<M::IU, D>(pm, dim, Sm);
	} else {
		if constexpr (M::MULTI) {
			pm[0]     = pp[0] * (Sp - up) / (Sp - Sm);
			pm[1]     = pp[1] * (Sp - up) / (Sp - Sm);
			pm[ip]    = pp[ip] + (pp[0] + pp[1]) * (Sp - up) * (Sm - up);
			pm[M::IA] = pp[M::IA];
		} else {
			pm[0]  = pp[0] * (Sp - up) / (Sp - Sm);
			pm[ip] = pp[ip] + pp[0] * (Sp - up) * (Sm - up);
		}
		for (int i = 0; i < M::D; ++i) pm[M::IU + i] = pp[M::IU + i];
		put<M::IU, D>(pm, dim, Sm);
	}
}

// multi::A receives the curvature through a `const size_t ka` parameter (model/multi.hpp:126): the
// double is truncated to an integer and a negative value wraps modulo 2^64 before re-entering the
// product as a double. Reproduced as the reference build converts it (signed 64-bit truncation read as
// unsigned).
__device__ __forceinline__ double jacobian_kappa(double k) {
	return (double) (unsigned long long) (long long) k;
}

// compute_rhs (model/euler.hpp:105-116, model/multi.hpp:158-169): rhs = sum_j A_j(p) slope_j with
// the primitive Jacobians A (model/euler.hpp:86-103, model/multi.hpp:126-145). Products with
// structurally zero entries of A are skipped: adding an exact zero never changes a running sum
// that starts at +0.
template<class M>
__device__ __forceinline__ void compute_rhs(const ModelConsts &m, const double *p, const double *slope /*[D][E]*/,
                                            double kappa, double *rhs) {
	constexpr int E = M::E, D = M::D, IP = M::IP, IU = M::IU;
	double rho = M::MULTI ? (p[0] + p[1]) : p[0];
	double c2;
	if constexpr (M::MULTI) c2 = sound_speed_2<M>(m, p[0], p[1], p[IP], p[M::IA]);
	else c2 = sound_speed_2<M>(m, p[0], 0.0, p[IP], 0.0);
	double a_pin = M::MULTI ? rho * c2 : p[0] * c2;  // A[ip][in]
	double a_inp = 1.0 / rho;                         // A[in][ip]
	double a_ina = 0.0;                               // A[in][ia]
	if constexpr (M::MULTI) a_ina = m.sigma * jacobian_kappa(kappa) / (p[0] + p[1]);
	for (int i = 0; i < E; ++i) {
		double r = 0.0;
		for (int j = 0; j < D; ++j) {
			const int in  = IU + j;
			const double *s = slope + j * E;
			double diag     = p[in];
			if (i == 0) {
				r += diag * s[0];
				r += p[0] * s[in];
			} else if (M::MULTI && i == 1) {
				r += diag * s[1];
				r += p[1] * s[in];
			} else if (i == IP) {
				r += a_pin * s[in];
				r += diag * s[IP];
			} else if (i == in) {
				r += diag * s[i];
				r += a_inp * s[IP];
				if constexpr (M::MULTI) r += a_ina * s[M::IA];
			} else {
				r += diag * s[i];
			}
		}
		rhs[i] = r;
	}
}

// Fv<D> (model/common.hpp:8-24): viscous stress row (and work term) for face normal `dim`, times mu.
// du is [D][G].
template<int D, int G, class S = double>
__device__ __forceinline__ void visc_flux(const S *du, const S *vel, S mu, int dim, S *fv /*[D+1]*/) {
	for (int i = 0; i <= D; ++i) fv[i] = 0;
	S trace = 0;
#pragma unroll
	for (int i = 0; i < D; ++i) {
		S row = du[i], col = du[i * G];  // du[dim * G + i] and du[i * G + dim] for dim == 0
#pragma unroll
		for (int j = 1; j < D; ++j)
			if (dim == j) row = du[j * G + i], col = du[i * G + j];
		fv[i] = row + col;
		trace += du[i * G + i];
	}
	put_add<0, D>(fv, dim, -((S) (2.0 / 3.0) * trace));
	for (int i = 0; i < D; ++i) fv[D] += fv[i] * vel[i];
	for (int i = 0; i <= D; ++i) fv[i] = fv[i] * mu;
}

}  // namespace dg
