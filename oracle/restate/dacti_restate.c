/*
 * Oracle (test infrastructure, not the product): plain-C restatement of DACTI's model arithmetic.
 * See dacti_restate.h. Citations are reference file:line; expressions keep the reference's
 * left-to-right evaluation order. Build without FMA contraction (-ffp-contract=off).
 */
#include "dacti_restate.h"

#include <math.h>
#include <string.h>

#define EULER_GAMMA 1.4      /* model/euler.hpp:34 */
#define NS_CP 1005.0         /* model/navier_stokes.hpp:353 */
#define NS_R 287.0           /* model/navier_stokes.hpp:354 */
#define MULTI_EPS 1e-20      /* model/multi.hpp:47 */

static double mn(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double mx(double a, double b) { return (a < b) ? b : a; } /* std::max */

static int is_multi(const ro_model *m) { return m->model == RO_MULTI; }
static int iu_of(const ro_model *m) { return is_multi(m) ? 2 : 1; }

int ro_num_eqns(const ro_model *m) { return m->dims + (is_multi(m) ? 4 : 2); }
int ro_num_flux(const ro_model *m) { return ro_num_eqns(m) + (is_multi(m) ? m->dims + 1 : 0); }
static int ip_of(const ro_model *m) { return is_multi(m) ? ro_num_eqns(m) - 2 : ro_num_eqns(m) - 1; }
static int ia_of(const ro_model *m) { return ro_num_eqns(m) - 1; }

/* multi::gamma, multi::p0, multi::temperature (model/multi.hpp:367-401) */
static double gam(const ro_model *m, double a) {
	if (a < MULTI_EPS) return m->gamma2;
	else if (a > 1 - MULTI_EPS) return m->gamma1;
	return 1 + 1 / (a / (m->gamma1 - 1) + (1 - a) / (m->gamma2 - 1));
}
static double p0(const ro_model *m, double a) {
	if (a < MULTI_EPS) return m->P2;
	else if (a > 1 - MULTI_EPS) return m->P1;
	return (a * m->gamma1 * m->P1 / (m->gamma1 - 1) + (1 - a) * m->gamma2 * m->P2 / (m->gamma2 - 1)) /
	       (1 + a / (m->gamma1 - 1) + (1 - a) / (m->gamma2 - 1));
}
static double temperature_multi(const ro_model *m, double r0, double r1, double p, double a) {
	if (a < MULTI_EPS) return (p + m->P2) / ((m->gamma2 - 1) * r1 * m->cv2);
	else if (a > 1 - MULTI_EPS) return (p + m->P1) / ((m->gamma1 - 1) * r0 * m->cv1);
	return (p / (gam(m, a) - 1) + a * m->P1 / (m->gamma1 - 1) + (1 - a) * m->P2 / (m->gamma2 - 1)) /
	       (r0 * m->cv1 + r1 * m->cv2);
}

/* sound_speed_2 (model/euler.hpp:246-248, model/multi.hpp:428-430) */
static double c2(const ro_model *m, double r0, double r1, double p, double a) {
	if (is_multi(m)) return gam(m, a) * (p + p0(m, a)) / (r0 + r1);
	return EULER_GAMMA * p / r0;
}
static double cs(const ro_model *m, double r0, double r1, double p, double a) {
	if (is_multi(m)) return sqrt(gam(m, a) * (p + p0(m, a)) / (r0 + r1));
	return sqrt(EULER_GAMMA * p / r0);
}

/* pressure (model/euler.hpp:230-236, model/multi.hpp:407-414) */
static double pressure(const ro_model *m, const double *u) {
	const int D = m->dims, iu = iu_of(m), ip = ip_of(m);
	double ke = 0;
	for (int i = 0; i < D; ++i) ke += 0.5 * u[iu + i] * u[iu + i];
	if (is_multi(m)) {
		const int ia = ia_of(m);
		return (gam(m, u[ia]) - 1) * (u[ip] - ke / (u[0] + u[1])) - gam(m, u[ia]) * p0(m, u[ia]);
	}
	return (EULER_GAMMA - 1) * (u[ip] - ke / u[0]);
}

/* primitive_variables (model/euler.hpp:266-274, model/multi.hpp:448-458) */
void ro_prim_from_cons(const ro_model *m, const double *u, double *p) {
	const int D = m->dims, iu = iu_of(m), ip = ip_of(m);
	if (is_multi(m)) {
		p[0] = u[0];
		p[1] = u[1];
		for (int i = 0; i < D; ++i) p[iu + i] = u[iu + i] / (u[0] + u[1]);
		p[ip]        = pressure(m, u);
		p[ia_of(m)] = u[ia_of(m)];
	} else {
		p[0] = u[0];
		for (int i = 0; i < D; ++i) p[iu + i] = u[iu + i] / u[0];
		p[ip] = pressure(m, u);
	}
}

/* conserved_variables (model/euler.hpp:276-286, model/multi.hpp:460-472) */
void ro_cons_from_prim(const ro_model *m, const double *p, double *u) {
	const int D = m->dims, iu = iu_of(m), ip = ip_of(m);
	double ke = 0;
	if (is_multi(m)) {
		const int ia = ia_of(m);
		u[0] = p[0];
		u[1] = p[1];
		for (int i = 0; i < D; ++i) {
			u[iu + i] = (p[0] + p[1]) * p[iu + i];
			ke += 0.5 * p[iu + i] * p[iu + i];
		}
		u[ip] = (p[ip] + gam(m, p[ia]) * p0(m, p[ia])) / (gam(m, p[ia]) - 1) + (p[0] + p[1]) * ke;
		u[ia] = p[ia];
	} else {
		u[0] = p[0];
		for (int i = 0; i < D; ++i) {
			u[iu + i] = p[0] * p[iu + i];
			ke += 0.5 * p[iu + i] * p[iu + i];
		}
		u[ip] = p[ip] / (EULER_GAMMA - 1) + p[0] * ke;
	}
}

static double mu_of(const ro_model *m, const double *p) {
	if (is_multi(m)) return m->mu1 * p[ia_of(m)] + m->mu2 * (1 - p[ia_of(m)]); /* model/multi.hpp:313-315 */
	return m->ns_mu;                                                        /* model/navier_stokes.hpp:419-421 */
}
static double lambda_of(const ro_model *m, const double *p) {
	if (is_multi(m)) return m->lambda1 * p[ia_of(m)] + m->lambda2 * (1 - p[ia_of(m)]);
	return m->ns_lambda;
}

/* max_delta_time (model/euler.hpp:203-215, navier_stokes.hpp:427-440, multi.hpp:322-346) */
double ro_max_delta_time(const ro_model *m, const ro_cell *c) {
	const int D = m->dims, iu = iu_of(m), ip = ip_of(m);
	const double *p = c->p;
	double sc       = is_multi(m) ? cs(m, p[0], p[1], p[ip], p[ia_of(m)]) : cs(m, p[0], 0.0, p[ip], 0.0);
	double dt[3];
	for (int i = 0; i < D; ++i) dt[i] = c->size / (sc + fabs(p[iu + i]));
	double dmin = dt[0];
	for (int i = 1; i < D; ++i) dmin = mn(dmin, dt[i]);
	if (m->model == RO_EULER) return dmin;
	if (is_multi(m)) {
		double k = mx(mu_of(m, p), lambda_of(m, p) / mn(m->cp1, m->cp2));
		if (k < 1e-15) return dmin;
		return mn(dmin, c->size * c->size / k / 4.0);
	}
	double k = mx(m->ns_mu, m->ns_lambda / NS_CP);
	if (k < 1e-15) return dmin;
	return mn(dmin, c->size * c->size / k * 0.5);
}

/* multi::A takes the curvature as `const size_t ka` (model/multi.hpp:126): the double is truncated
 * to an integer and, when negative, wraps modulo 2^64 (the conversion the oracle build performs:
 * signed 64-bit truncation reinterpreted as unsigned); that value re-enters the product as a double. */
static double jacobian_kappa(double k) { return (double) (unsigned long long) (long long) k; }

/* compute_rhs with the full primitive Jacobians A (model/euler.hpp:86-116, model/multi.hpp:126-169) */
void ro_compute_rhs(const ro_model *m, ro_cell *c) {
	const int D = m->dims, E = ro_num_eqns(m), iu = iu_of(m), ip = ip_of(m);
	const double *p = c->p;
	for (int i = 0; i < E; ++i) c->rhs[i] = 0.0;
	for (int i = 0; i < E; ++i) {
		for (int j = 0; j < D; ++j) {
			double A[7][7];
			const int in = iu + j;
			for (int r = 0; r < E; ++r)
				for (int s = 0; s < E; ++s) A[r][s] = (r == s) ? p[in] : 0.0;
			if (is_multi(m)) {
				const int ia = ia_of(m);
				A[0][in]  = p[0];
				A[1][in]  = p[1];
				A[ip][in] = (p[0] + p[1]) * c2(m, p[0], p[1], p[ip], p[ia]);
				A[in][ip] = 1.0 / (p[0] + p[1]);
				A[in][ia] = m->sigma * jacobian_kappa(c->k[2 + D]) / (p[0] + p[1]);
			} else {
				A[0][in]  = p[0];
				A[ip][in] = p[0] * c2(m, p[0], 0.0, p[ip], 0.0);
				A[in][ip] = 1.0 / p[0];
			}
			for (int k = 0; k < E; ++k) c->rhs[i] += A[i][k] * c->slope[j][k];
		}
	}
}

/* F(p, dim) and the projected F(p, u, dim) (model/euler.hpp:50-83, model/multi.hpp:78-123) */
void ro_phys_flux(const ro_model *m, const double *p, double un, int dim, int projected, double *F) {
	const int D = m->dims, iu = iu_of(m), ip = ip_of(m), NFL = ro_num_flux(m), in = iu + dim;
	const double vn = projected ? un : p[in];
	double ke       = 0.0;
	for (int q = 0; q < NFL; ++q) F[q] = 0.0;
	if (is_multi(m)) {
		const int ia = ia_of(m);
		for (int i = 0; i < D; ++i) {
			F[iu + i] = (p[0] + p[1]) * vn * p[iu + i];
			ke += 0.5 * p[iu + i] * p[iu + i];
		}
		F[0] = vn * p[0];
		F[1] = vn * p[1];
		F[in] += p[ip];
		F[ip]           = vn * (gam(m, p[ia]) / (gam(m, p[ia]) - 1) * (p[ip] + p0(m, p[ia])) + ke * (p[0] + p[1]));
		F[ia]           = vn * p[ia];
		F[ia + 1]       = vn;
		F[ia + 2 + dim] = p[ia];
	} else {
		for (int i = 0; i < D; ++i) {
			F[iu + i] = p[0] * vn * p[iu + i];
			ke += 0.5 * p[iu + i] * p[iu + i];
		}
		F[0] = vn * p[0];
		F[in] += p[ip];
		F[ip] = vn * (EULER_GAMMA / (EULER_GAMMA - 1) * p[ip] + ke * p[0]);
	}
}

/* middle_state (model/euler.hpp:118-153, model/multi.hpp:205-246) */
void ro_middle_state(const ro_model *m, const double *pn, const double *pp, double ka, int dim, double *pm) {
	const int D = m->dims, E = ro_num_eqns(m), iu = iu_of(m), ip = ip_of(m), in = iu + dim;
	double c_n, c_p, Sm;
	if (is_multi(m)) {
		const int ia = ia_of(m);
		c_n = cs(m, pn[0], pn[1], pn[ip], pn[ia]);
		c_p = cs(m, pp[0], pp[1], pp[ip], pp[ia]);
	} else {
		c_n = cs(m, pn[0], 0.0, pn[ip], 0.0);
		c_p = cs(m, pp[0], 0.0, pp[ip], 0.0);
	}
	double u  = 0.5 * (pn[in] + pp[in]);
	double c  = 0.5 * (c_n + c_p);
	double Sn = mn(u - c, pn[in] - c_n);
	double Sp = mx(u + c, pp[in] + c_p);
	if (is_multi(m)) {
		const int ia = ia_of(m);
		Sm = (pp[ip] - pn[ip] + (pn[0] + pn[1]) * pn[in] * (Sn - pn[in]) - (pp[0] + pp[1]) * pp[in] * (Sp - pp[in]) -
		      m->sigma * ka * (pp[ia] - pn[ia])) /
		     ((pn[0] + pn[1]) * (Sn - pn[in]) - (pp[0] + pp[1]) * (Sp - pp[in]));
	} else {
		Sm = (pp[ip] - pn[ip] + pn[0] * pn[in] * (Sn - pn[in]) - pp[0] * pp[in] * (Sp - pp[in])) /
		     (pn[0] * (Sn - pn[in]) - pp[0] * (Sp - pp[in]));
	}
	for (int q = 0; q < E; ++q) pm[q] = 0.0;
	if (Sn > 0) {
		memcpy(pm, pn, sizeof(double) * E);
	} else if (Sp < 0) {
		memcpy(pm, pp, sizeof(double) * E);
	} else {
		const double *s = (Sm > 0 && Sn < 0) ? pn : pp;
		const double S  = (Sm > 0 && Sn < 0) ? Sn : Sp;
		if (is_multi(m)) {
			pm[0]        = s[0] * (S - s[in]) / (S - Sm);
			pm[1]        = s[1] * (S - s[in]) / (S - Sm);
			pm[ip]       = s[ip] + (s[0] + s[1]) * (S - s[in]) * (Sm - s[in]);
			pm[ia_of(m)] = s[ia_of(m)];
		} else {
			pm[0]  = s[0] * (S - s[in]) / (S - Sm);
			pm[ip] = s[ip] + s[0] * (S - s[in]) * (Sm - s[in]);
		}
		for (int i = 0; i < D; ++i) pm[iu + i] = s[iu + i];
		pm[in] = Sm;
	}
}

/* Fv<D> (model/common.hpp:8-24) */
static void fvisc(int D, const double *du /*[D][G]*/, int G, const double *vel, double mu, int dim, double *fv) {
	double trace = 0.0;
	for (int i = 0; i <= D; ++i) fv[i] = 0.0;
	for (int i = 0; i < D; ++i) {
		fv[i] = du[dim * G + i] + du[i * G + dim];
		trace += du[i * G + i];
	}
	fv[dim] -= (2.0 / 3.0 * trace);
	for (int i = 0; i < D; ++i) fv[D] += fv[i] * vel[i];
	for (int i = 0; i <= D; ++i) fv[i] = fv[i] * mu;
}

static int num_grad(const ro_model *m) {
	return m->model == RO_MULTI ? m->dims + 3 : (m->model == RO_NAVIER_STOKES ? m->dims + 1 : 0);
}

/* Model::flux (model/euler.hpp:156-200, navier_stokes.hpp:387-408, multi.hpp:249-302) */
void ro_flux(const ro_model *m, const ro_cell *cn, const ro_cell *cp, const double *face_center, double side,
             double t0, double t1, int dim, double *F) {
	const int D = m->dims, E = ro_num_eqns(m), NFL = ro_num_flux(m), iu = iu_of(m), ip = ip_of(m), G = num_grad(m);
	const double area = pow(side, D - 1); /* CellFace::area (integrator/cell.hpp:622-624) */
	double dt_n = 0.5 * (t1 + t0) - cn->t;
	double dt_p = 0.5 * (t1 + t0) - cp->t;
	double pn[7], pp[7], pm[7];
	for (int q = 0; q < E; ++q) {
		pn[q] = cn->p[q] + cn->slope[dim][q] * (face_center[dim] - cn->center[dim]);
		pp[q] = cp->p[q] + cp->slope[dim][q] * (face_center[dim] - cp->center[dim]);
	}
	for (int q = 0; q < E; ++q) {
		pn[q] = pn[q] - cn->rhs[q] * dt_n;
		pp[q] = pp[q] - cp->rhs[q] * dt_p;
	}
	double ka = 0.0;
	if (is_multi(m)) ka = 0.5 * (cn->k[2 + D] + cp->k[2 + D]);
	ro_middle_state(m, pn, pp, ka, dim, pm);
	ro_phys_flux(m, pm, 0.0, dim, 0, F);
	if (is_multi(m)) {
		const int ia = ia_of(m);
		const double a = pm[ia];
		if (pm[ia] > 1e-5 && pm[ia] < 1 - 1e-5) {
			double n  = 0.5 * (cn->k[2 + dim] + cp->k[2 + dim]);
			double uc = 1.0 * fabs(pm[iu + dim]) * n;
			double ke = 0.0;
			for (int i = 0; i < D; ++i) {
				F[iu + i] += uc * ((1 - a) * pm[0] - a * pm[1]) * pm[iu + i];
				ke += 0.5 * pm[iu + i] * pm[iu + i];
			}
			F[0] += uc * (1 - a) * pm[0];
			F[1] += uc * (-a) * pm[1];
			F[ip] += uc * ((1 - a) * pm[0] - a * pm[1]) * ke +
			         uc * (1 - a) * a *
			             (pm[ip] * (1 / (m->gamma1 - 1) - 1 / (m->gamma2 - 1)) + m->gamma1 * m->P1 / (m->gamma1 - 1) -
			              m->gamma2 * m->P2 / (m->gamma2 - 1));
			F[ia] += uc * (1 - a) * a;
		}
	}
	if (G > 0) {
		double du[18], vel[3], fv[4];
		for (int i = 0; i < D; ++i)
			for (int g = 0; g < G; ++g) du[i * G + g] = 0.5 * (cn->gradient[i][g] + cp->gradient[i][g]);
		for (int i = 0; i < D; ++i) vel[i] = 0.5 * (cn->p[iu + i] + cp->p[iu + i]);
		if (is_multi(m)) {
			fvisc(D, du, G, vel, mu_of(m, pm), dim, fv);
			for (int i = 0; i <= D; ++i) F[iu + i] -= fv[i];
			F[iu + D] -= du[dim * G + D] * lambda_of(m, pm);
			for (int q = 0; q < NFL; ++q) F[q] = F[q] * area * (t1 - t0);
		} else {
			for (int q = 0; q < NFL; ++q) F[q] = F[q] * area * (t1 - t0);
			fvisc(D, du, G, vel, m->ns_mu, dim, fv);
			for (int i = 0; i <= D; ++i) F[iu + i] -= fv[i] * area * (t1 - t0);
			F[iu + D] -= m->ns_lambda * du[dim * G + D] * area * (t1 - t0);
		}
	} else {
		for (int q = 0; q < NFL; ++q) F[q] = F[q] * area * (t1 - t0);
	}
}

/* Boundary::boundary_value (integrator/boundary.hpp:75-123) */
void ro_boundary_value(const ro_model *m, const ro_bc *b, const ro_cell *c, double *pb) {
	const int D = m->dims, E = ro_num_eqns(m), iu = iu_of(m), ip = ip_of(m);
	const double *pc = c->p;
	if (b->type == 1) { /* freeslip */
		double dot = 0.0;
		memcpy(pb, pc, sizeof(double) * E);
		for (int i = 0; i < D; ++i) dot += pc[iu + i] * b->normal[i];
		for (int i = 0; i < D; ++i) pb[iu + i] = pc[iu + i] - b->normal[i] * dot;
		return;
	}
	if (b->type == 2) { /* noslip */
		memcpy(pb, pc, sizeof(double) * E);
		for (int i = 0; i < D; ++i) pb[iu + i] *= -1.0;
		return;
	}
	if (b->type == 3 || b->type == 4) { /* inflow, inflow_r */
		double u2 = 0;
		memcpy(pb, b->p_in, sizeof(double) * E);
		for (int i = 0; i < D; ++i) u2 += pc[iu + i] * pc[iu + i];
		/* supersonic (model/euler.hpp:250-256; multi.hpp:432-438 passes p[0] as the density pair) */
		int sup = is_multi(m) ? u2 > c2(m, pc[0], 0.0, pc[ip], pc[ia_of(m)]) : u2 > c2(m, pc[0], 0.0, pc[ip], 0.0);
		if (!sup) pb[ip] = pc[ip];
		if (b->fade_in > 0.0) {
			double vm = mn(c->t / b->fade_in, 1.0);
			for (int i = 0; i < D; ++i) pb[iu + i] *= vm;
		}
		return;
	}
	if (b->type == 6) { /* dirichlet */
		memcpy(pb, b->p_in, sizeof(double) * E);
		return;
	}
	memcpy(pb, pc, sizeof(double) * E); /* outflow, zeroGradient */
}

/* Boundary::boundary_flux (integrator/boundary.hpp:130-160) */
void ro_boundary_flux(const ro_model *m, const ro_bc *b, const ro_cell *c, double side, double t0, double t1, int dim,
                      int dir, double *F) {
	const int D = m->dims, NFL = ro_num_flux(m), iu = iu_of(m), ip = ip_of(m), G = num_grad(m);
	double pb[7], pm[7];
	ro_boundary_value(m, b, c, pb);
	if (b->type == 1) {
		ro_phys_flux(m, c->p, pb[iu + dim], dim, 1, F);
	} else if (b->type == 2) {
		for (int q = 0; q < NFL; ++q) F[q] = 0.0;
		F[iu + dim] = pb[ip];
	} else {
		ro_middle_state(m, pb, c->p, 0.0, dim, pm);
		ro_phys_flux(m, pm, 0.0, dim, 0, F);
	}
	if (G > 0) {
		double g[18], z[3] = {0, 0, 0}, fv[4];
		for (int i = 0; i < D; ++i)
			for (int k = 0; k < G; ++k) g[i * G + k] = c->gradient[i][k];
		fvisc(D, g, G, z, mu_of(m, c->p), dim, fv);
		for (int k = 0; k <= D; ++k) F[iu + k] -= fv[k];
	}
	const double area = pow(side, D - 1);
	for (int q = 0; q < NFL; ++q) F[q] = F[q] * area * (t1 - t0) * (double) (2 * dir - 1);
}

/* multi::source (model/multi.hpp:186-203) */
void ro_source(const ro_model *m, const ro_cell *c, const double *du, double *s) {
	const int D = m->dims, E = ro_num_eqns(m), iu = iu_of(m), ip = ip_of(m), ia = ia_of(m);
	for (int q = 0; q < E; ++q) s[q] = 0.0;
	if (!is_multi(m)) return;
	const double kap = c->k[2 + D];
	for (int i = 0; i < D; ++i) s[iu + i] = -m->sigma * kap * du[ia + 2 + i];
	s[ip] = m->sigma * kap * (-du[ia] + c->p[ia] * du[ia + 1]);
	s[ia] = -c->p[ia] * du[ia + 1];
}

/* get_grad_input (model/navier_stokes.hpp:377-385, model/multi.hpp:148-156) */
void ro_grad_input(const ro_model *m, const double *p, double *g) {
	const int D = m->dims, iu = iu_of(m), ip = ip_of(m);
	for (int i = 0; i < D; ++i) g[i] = p[iu + i];
	if (is_multi(m)) {
		g[D]     = temperature_multi(m, p[0], p[1], p[ip], p[ia_of(m)]);
		g[D + 1] = p[ia_of(m)];
		g[D + 2] = 0.0;
	} else {
		g[D] = p[ip] / (p[0] * NS_R);
	}
}

/* slope limiters (integrator/slope_limiters.hpp:7-57) */
double ro_limit(int lim, double s1, double s2) {
	double r;
	switch (lim) {
		case 0:
			if (s1 * s2 <= 0.0) return 0.0;
			return fabs(s1) < fabs(s2) ? s1 : s2;
		case 1: return 0.5 * (s1 + s2);
		case 2: r = s1 / s2; return (r + fabs(r)) / (1 + fabs(r)) * s2;
		case 3: r = s1 / s2; return mx(mx(0.0, mn(2.0 * r, 1.0)), mn(r, 2.0)) * s2;
		case 4: r = s1 / s2; return 2.0 * r / (r * r + 1) * s2;
		case 5: r = (s1 + 1e-9) / (s2 + 1e-9); return mx(0.0, mn(2.0 * r, mn((1.0 + 2.0 * r) / 3.0, 2.))) * s2;
		default: return 0.0;
	}
}

/* weighted_laplacian::estimate (integrator/error_estimators.hpp:19-37) */
double ro_estimate(const ro_model *m, const double *w, const ro_cell *c, const double *nbh, const int *present) {
	const int D = m->dims, E = ro_num_eqns(m);
	double error = 0.0;
	for (int dim = 0; dim < D; ++dim) {
		double d2[7], sq = 0.0;
		for (int q = 0; q < E; ++q) d2[q] = c->p[q] * -2.0;
		for (int dir = 0; dir < 2; ++dir) {
			if (!present[dim * 2 + dir]) {
				for (int q = 0; q < E; ++q) d2[q] = 0.0;
				break;
			}
			for (int q = 0; q < E; ++q) d2[q] = d2[q] + nbh[(dim * 2 + dir) * 7 + q];
		}
		for (int q = 0; q < E; ++q) sq += (d2[q] * w[q]) * (d2[q] * w[q]);
		error += sq;
	}
	return sqrt(error);
}
