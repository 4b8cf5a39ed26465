// Layout of the opaque dg_solver handle, shared by the C-ABI translation units.
#pragma once

#include "batch.cuh"

namespace dg {
void noalloc_prepare(int device);  // noalloc.cu
}

struct dg_solver {
	dg::SolverBase *impl;
	int device;
};

struct dg_batch {
	dg::BatchBase *impl;
	int device;
};
