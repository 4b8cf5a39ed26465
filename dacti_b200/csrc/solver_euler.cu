// Instantiation of the solver for the Euler model in 2D and 3D.
#include "batch.cuh"

namespace dg {
SolverBase *make_solver_euler(const dg_case &c) {
	if (c.dims == 2) return new Solver<Euler<2>>(c);
	if (c.dims == 3) return new Solver<Euler<3>>(c);
	throw dg_error(DG_ERR_ARG, "dims must be 2 or 3");
}
BatchBase *make_batch_euler(const std::vector<SolverBase *> &s) {
	if (s.empty()) throw dg_error(DG_ERR_ARG, "empty batch");
	if (s[0]->dims() == 2) return make_batch_for<Euler<2>>(s);
	return make_batch_for<Euler<3>>(s);
}
}  // namespace dg
