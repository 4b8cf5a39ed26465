// extern "C" entry points of include/dacti_gpu.h.
#include "capi_internal.h"

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <vector>

namespace {
thread_local std::string g_create_error;
thread_local int g_device = 0;

template<typename Fn>
int guarded(dg_solver *s, Fn &&fn) {
	try {
		cudaError_t e = cudaSetDevice(s ? s->device : g_device);
		if (e != cudaSuccess) throw dg::dg_error(DG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
		fn();
		return DG_OK;
	} catch (const dg::dg_error &e) {
		if (s && s->impl) s->impl->last_error = e.what();
		else g_create_error = e.what();
		return e.code;
	} catch (const std::exception &e) {
		if (s && s->impl) s->impl->last_error = e.what();
		else g_create_error = e.what();
		return DG_ERR_ARG;
	}
}

template<typename Fn>
int batch_guarded(dg_batch *b, Fn &&fn) {
	if (!b) return DG_ERR_ARG;
	try {
		cudaError_t e = cudaSetDevice(b->device);
		if (e != cudaSuccess) throw dg::dg_error(DG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
		fn();
		return DG_OK;
	} catch (const dg::dg_error &e) {
		b->impl->last_error = e.what();
		return e.code;
	} catch (const std::exception &e) {
		b->impl->last_error = e.what();
		return DG_ERR_ARG;
	}
}
}  // namespace

extern "C" {

int dg_create(const dg_case *c, dg_solver **out) {
	if (!c || !out) return DG_ERR_ARG;
	*out = nullptr;
	return guarded(nullptr, [&] {
		dg::SolverBase *impl = nullptr;
		switch (c->model) {
			case DG_EULER: impl = dg::make_solver_euler(*c); break;
			case DG_NAVIER_STOKES: impl = dg::make_solver_ns(*c); break;
			case DG_MULTI: impl = dg::make_solver_multi(*c); break;
			default: throw dg::dg_error(DG_ERR_ARG, "unknown model id");
		}
		// the allocation-free read-back's scratch and gather kernel are placed on the device now, so
		// that dg_read_cells_noalloc never allocates, not even on its first call
		try {
			dg::noalloc_prepare(g_device);
			impl->prepare_noalloc();
		} catch (...) {
			delete impl;
			throw;
		}
		*out = new dg_solver{impl, g_device};
	});
}

int dg_set_device(int ordinal) {
	if (ordinal < 0) return DG_ERR_ARG;
	g_device = ordinal;
	return DG_OK;
}

int dg_set_stream(dg_solver *s, void *stream) {
	if (!s) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->set_stream((cudaStream_t) stream); });
}

int dg_step(dg_solver *s, int signal, int *force_break, double *global_dt, dg_substep_fn fn, void *user) {
	if (!s || !force_break || !global_dt) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->step(signal, force_break, global_dt, fn, user); });
}

int dg_step_many(dg_solver **s, int n, int threads, int signal, int *force_break, double *global_dt, int *status) {
	if (!s || n < 0 || threads < 1 || !force_break || !global_dt || !status) return DG_ERR_ARG;
	for (int k = 0; k < n; ++k)
		if (!s[k]) return DG_ERR_ARG;
	// every solver on a stream of its own, so that the solvers' kernels can overlap on the device
	for (int k = 0; k < n; ++k) {
		const int rc = guarded(s[k], [&] { s[k]->impl->own_stream(); });
		if (rc != DG_OK) return rc;
	}
	// largest trees first (cells as the work estimate), so that no large tree is left for the end
	std::vector<long long> cells(n, 0);
	std::vector<int> order(n);
	for (int k = 0; k < n; ++k) {
		order[k] = k;
		guarded(s[k], [&] { cells[k] = s[k]->impl->cell_count(); });
	}
	std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells[a] > cells[b]; });
	std::atomic<int> next{0};
	auto worker = [&] {
		for (int j = next++; j < n; j = next++) {
			const int k    = order[j];
			force_break[k] = 0;
			status[k]      = guarded(s[k], [&] { s[k]->impl->step(signal, &force_break[k], &global_dt[k], nullptr, nullptr); });
		}
	};
	const int nt = threads < n ? threads : (n > 0 ? n : 1);
	std::vector<std::thread> pool;
	for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
	worker();
	for (auto &th: pool) th.join();
	for (int k = 0; k < n; ++k)
		if (status[k] != DG_OK) return status[k];
	return DG_OK;
}

int dg_cell_count(dg_solver *s, long long *n) {
	if (!s || !n) return DG_ERR_ARG;
	return guarded(s, [&] { *n = s->impl->cell_count(); });
}

int dg_read_cells(dg_solver *s, int *levels, double *data, long long max_cells, long long *n_out) {
	if (!s || !levels || !data) return DG_ERR_ARG;
	return guarded(s, [&] {
		long long n = s->impl->read_cells(levels, data, max_cells);
		if (n_out) *n_out = n;
	});
}

int dg_read_slopes(dg_solver *s, double *slopes, long long max_cells, long long *n_out) {
	if (!s || !slopes) return DG_ERR_ARG;
	return guarded(s, [&] {
		long long n = s->impl->read_slopes(slopes, max_cells);
		if (n_out) *n_out = n;
	});
}

int dg_read_gradients(dg_solver *s, double *gradients, long long max_cells, long long *n_out) {
	if (!s || !gradients) return DG_ERR_ARG;
	return guarded(s, [&] {
		long long n = s->impl->read_gradients(gradients, max_cells);
		if (n_out) *n_out = n;
	});
}

int dg_forecast_features(dg_solver *s, double *features, long long max_cells, long long *n_out) {
	if (!s || !features) return DG_ERR_ARG;
	return guarded(s, [&] {
		long long n = s->impl->forecast_features(features, max_cells);
		if (n_out) *n_out = n;
	});
}

int dg_tree_size(dg_solver *s, long long *n) {
	if (!s || !n) return DG_ERR_ARG;
	return guarded(s, [&] { *n = s->impl->tree_size(); });
}

int dg_read_tree(dg_solver *s, int *parent, int *children, int *level, unsigned int *flags, double *p, double *meta,
                 long long max_nodes, long long *n_out) {
	if (!s || !parent || !children || !level || !flags || !p || !meta) return DG_ERR_ARG;
	return guarded(s, [&] {
		long long n = s->impl->read_tree(parent, children, level, flags, p, meta, max_nodes);
		if (n_out) *n_out = n;
	});
}

int dg_set_hold(dg_solver *s, const unsigned char *hold, long long n) {
	if (!s || (!hold && n > 0)) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->set_hold(hold, n); });
}

int dg_set_coarsen_interval(dg_solver *s, int steps) {
	if (!s) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->set_coarsen_interval(steps); });
}

int dg_get_stats(dg_solver *s, dg_stats *out) {
	if (!s || !out) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->stats(out); });
}

int dg_set_form(dg_solver *s, int form) {
	if (!s) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->set_form(form); });
}

int dg_set_options(dg_solver *s, int options) {
	if (!s || (options & ~(DG_OPT_ORDERED_LISTS | DG_OPT_FACE_TILES))) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->set_options(options); });
}

int dg_set_profiling(dg_solver *s, int on) {
	if (!s) return DG_ERR_ARG;
	return guarded(s, [&] { s->impl->set_profiling(on != 0); });
}

int dg_batch_create(dg_solver **s, int n, dg_batch **out) {
	if (!s || n < 1 || !out) return DG_ERR_ARG;
	*out = nullptr;
	for (int k = 0; k < n; ++k)
		if (!s[k] || s[k]->device != s[0]->device) return DG_ERR_ARG;
	return guarded(s[0], [&] {
		std::vector<dg::SolverBase *> v;
		for (int k = 0; k < n; ++k) v.push_back(s[k]->impl);
		const int model = v[0]->model_id(), dims = v[0]->dims();
		for (auto *x: v)
			if (x->model_id() != model || x->dims() != dims)
				throw dg::dg_error(DG_ERR_ARG, "batched solvers must share one model and dimension");
		dg::BatchBase *impl = nullptr;
		switch (model) {
			case DG_EULER: impl = dg::make_batch_euler(v); break;
			case DG_NAVIER_STOKES: impl = dg::make_batch_ns(v); break;
			default: impl = dg::make_batch_multi(v); break;
		}
		*out = new dg_batch{impl, s[0]->device};
	});
}

int dg_batch_step(dg_batch *b, int signal, int *force_break, double *global_dt) {
	if (!b || !force_break || !global_dt) return DG_ERR_ARG;
	try {
		cudaError_t e = cudaSetDevice(b->device);
		if (e != cudaSuccess) throw dg::dg_error(DG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
		b->impl->step(signal, force_break, global_dt);
		return DG_OK;
	} catch (const dg::dg_error &e) {
		b->impl->last_error = e.what();
		return e.code;
	} catch (const std::exception &e) {
		b->impl->last_error = e.what();
		return DG_ERR_ARG;
	}
}

int dg_batch_set_launch(dg_batch *b, const int *bps, int n) {
	if (!bps || n < 0) return DG_ERR_ARG;
	return batch_guarded(b, [&] { b->impl->set_launch(bps, n); });
}

int dg_batch_set_profiling(dg_batch *b, int on) {
	return batch_guarded(b, [&] { b->impl->set_profiling(on != 0); });
}

int dg_batch_stage_times(dg_batch *b, double *ms, long long *items, int n) {
	if (!ms || !items || n < 0) return DG_ERR_ARG;
	return batch_guarded(b, [&] { b->impl->stage_times(ms, items, n); });
}

int dg_batch_set_pregrow(dg_batch *b, int on) {
	return batch_guarded(b, [&] { b->impl->set_pregrow(on != 0); });
}

int dg_batch_run_stats(dg_batch *b, long long *out, int n) {
	if (!out || n < 0) return DG_ERR_ARG;
	return batch_guarded(b, [&] { b->impl->run_stats(out, n); });
}

const char *dg_batch_last_error(dg_batch *b) {
	if (!b) return g_create_error.c_str();
	return b->impl->last_error.c_str();
}

void dg_batch_destroy(dg_batch *b) {
	if (!b) return;
	cudaSetDevice(b->device);
	delete b->impl;
	delete b;
}

const char *dg_last_error(dg_solver *s) {
	if (!s) return g_create_error.c_str();
	return s->impl->last_error.c_str();
}

void dg_destroy(dg_solver *s) {
	if (!s) return;
	cudaSetDevice(s->device);
	delete s->impl;
	delete s;
}

}  // extern "C"
