// Instantiation of the solver for the Multi model in 2D and 3D.
#include "batch.cuh"

namespace dg {
SolverBase *make_solver_multi(const dg_case &c) {
	if (c.dims == 2) return new Solver<Multi<2>>(c);
	if (c.dims == 3) return new Solver<Multi<3>>(c);
	throw dg_error(DG_ERR_ARG, "dims must be 2 or 3");
}
BatchBase *make_batch_multi(const std::vector<SolverBase *> &s) {
	if (s.empty()) throw dg_error(DG_ERR_ARG, "empty batch");
	if (s[0]->dims() == 2) return make_batch_for<Multi<2>>(s);
	return make_batch_for<Multi<3>>(s);
}
}  // namespace dg
