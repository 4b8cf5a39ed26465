/*
 * Oracle (test infrastructure, not the product): a plain-C restatement of the per-face and per-cell
 * arithmetic of DACTI's three models, its slope limiters, boundary conditions and refinement
 * indicator. Every function names the reference lines it follows and keeps their floating-point
 * operation order, so (compiled without FMA contraction) its results equal the reference's bit for
 * bit; tests/test_restate_kat.py checks that against known-answer vectors produced by the
 * reference's own headers (oracle/ref/kat.cpp).
 */
#ifndef DACTI_RESTATE_H
#define DACTI_RESTATE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { RO_EULER = 0, RO_NAVIER_STOKES = 1, RO_MULTI = 2 };

typedef struct ro_model {
	int model, dims;
	double ns_mu, ns_lambda;
	double gamma1, gamma2, P1, P2, cp1, cp2, cv1, cv2, mu1, mu2, lambda1, lambda2, sigma;
} ro_model;

/* One Cell<Model> (integrator/cell.hpp:8-107) with room for the largest model. */
typedef struct ro_cell {
	double size, t;
	double center[3];
	double u[7], p[7], rhs[7], k[7], t_slope[6];
	double slope[3][7];
	double gradient[3][6];
} ro_cell;

/* One Boundary<Model> value (integrator/boundary.hpp:34-37). */
typedef struct ro_bc {
	int type;
	double p_in[7];
	double normal[3];
	double fade_in;
} ro_bc;

int ro_num_eqns(const ro_model *m);
int ro_num_flux(const ro_model *m);

void ro_prim_from_cons(const ro_model *m, const double *u, double *p);
void ro_cons_from_prim(const ro_model *m, const double *p, double *u);
double ro_max_delta_time(const ro_model *m, const ro_cell *c);
void ro_compute_rhs(const ro_model *m, ro_cell *c);
void ro_middle_state(const ro_model *m, const double *pn, const double *pp, double ka, int dim, double *pm);
void ro_phys_flux(const ro_model *m, const double *p, double un, int dim, int projected, double *F);

/* Model::flux(cn, cp, face) with face = {center, side_length, t_0, t_1, dim} */
void ro_flux(const ro_model *m, const ro_cell *cn, const ro_cell *cp, const double *face_center, double side,
             double t0, double t1, int dim, double *F);

void ro_boundary_value(const ro_model *m, const ro_bc *b, const ro_cell *c, double *pb);
void ro_boundary_flux(const ro_model *m, const ro_bc *b, const ro_cell *c, double side, double t0, double t1, int dim,
                      int dir, double *F);

void ro_source(const ro_model *m, const ro_cell *c, const double *du, double *s);
void ro_grad_input(const ro_model *m, const double *p, double *g);

/* slope limiters by id: minmod, unlimited, van_leer, superbee, von_alba_2, koren, first_order */
double ro_limit(int lim, double s1, double s2);

/* weighted_laplacian::estimate (integrator/error_estimators.hpp:19-37); nbh[dim][dir] is the
 * neighbour state or absent when present[dim][dir] == 0 */
double ro_estimate(const ro_model *m, const double *weights, const ro_cell *c, const double *nbh /*[3][2][7]*/,
                   const int *present /*[3][2]*/);

#ifdef __cplusplus
}
#endif

#endif
