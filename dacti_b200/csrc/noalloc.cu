// dg_read_cells_noalloc: the cell read-back of dg_read_cells without any device allocation.
//
// Some hosts cannot let a library call cudaMalloc: an application that hands all device memory to
// its own pool allocator up front and runs the solver under that fixed budget, or a latency-bound
// driver thread that must not hit the implicit device-wide synchronisation of cudaMalloc/cudaFree.
// dg_read_cells allocates its device gather buffer on first use (and again whenever the cell count
// grows); this variant gathers through the file-scope array below instead, which is the only device
// memory it touches besides the solver's own state.
//
// Limits and sharing:
// - the scratch holds kScratchBytes (64 MiB), i.e. 64 MiB / (8 (D + 2E + P + 5)) cells: about 289
//   thousand cells of multi<3> (232 bytes each) and about 559 thousand cells of euler<2> (120 bytes);
//   larger read-backs are rejected with DG_ERR_CAPACITY and a message that states the sizes;
// - the array belongs to the library's module and stays resident on every GPU that loads it until
//   the process exits. Under CUDA's lazy module loading the module, and with it the array, is only
//   placed on a device when something first touches it, which would be an allocation; dg_create
//   therefore resolves the array's address (and loads the gather kernel) on the solver's device
//   while it builds the solver, so the array is committed before the first read-back;
// - all calls share it and it keeps the last call's contents: every record is rewritten by each
//   call, so nothing needs clearing, but two calls whose work overlaps on the GPU (different
//   solvers on different streams) race on it and must be serialised by the caller;
// - the array's device address is looked up (cudaGetSymbolAddress) once per device with that device
//   current, by dg_create; no read-back has to come first, and none touches the lookup again.
#include "capi_internal.h"

#include <mutex>
#include <string>

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices      = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device. In host code the symbol's name is
// only a host-side stand-in; the kernel must be given this address.
void *scratch_address(int device) {
	if (device < 0 || device >= kMaxDevices) throw dg::dg_error(DG_ERR_ARG, "device ordinal out of range");
	std::lock_guard<std::mutex> lk(g_mu);
	if (!g_scratch_addr[device]) {
		void *p       = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess)
			throw dg::dg_error(DG_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
		g_scratch_addr[device] = p;
	}
	return g_scratch_addr[device];
}

}  // namespace

namespace dg {
// Called by dg_create with the solver's device current: commits the scratch array on that device.
void noalloc_prepare(int device) { (void) scratch_address(device); }
}  // namespace dg

extern "C" int dg_read_cells_noalloc(dg_solver *s, int *levels, double *data, long long max_cells, long long *n_out) {
	if (!s || !levels || !data) return DG_ERR_ARG;
	try {
		cudaError_t e = cudaSetDevice(s->device);
		if (e != cudaSuccess) throw dg::dg_error(DG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
		void *scratch = scratch_address(s->device);
		long long n   = s->impl->read_cells_via(levels, data, max_cells, scratch, kScratchBytes);
		if (n_out) *n_out = n;
		return DG_OK;
	} catch (const dg::dg_error &err) {
		s->impl->last_error = err.what();
		return err.code;
	} catch (const std::exception &err) {
		s->impl->last_error = err.what();
		return DG_ERR_ARG;
	}
}
