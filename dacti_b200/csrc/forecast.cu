// Regrid forecaster network: a multilayer perceptron n_in -> 64 -> 64 -> 1 (ReLU, logistic output)
// that predicts, from per-leaf features, whether the refinement indicator will fire at that place a
// few global steps ahead. No counterpart in the reference. Training keeps FP32 master weights with Adam
// moments; inference reads BF16 copies of the weights, refreshed after every optimiser step.
//
// Parameter layout (FP32 master and BF16 copies alike): W1[H][n_in], b1[H], W2[H][H], b2[H], W3[H], b3.
// Loss: binary cross-entropy on the logit z with a weight on the positive class,
//   l = pw y softplus(-z) + (1 - y) softplus(z),   dl/dz = sigmoid(z) (pw y + 1 - y) - pw y.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "dacti_gpu.h"

namespace {

constexpr int H      = 64;   // hidden width
constexpr int MAX_IN = 32;   // largest input width
constexpr int TPB    = 128;  // threads per block (one sample each)

thread_local std::string g_mlp_error;

struct Layout {
	int nin;
	long long w1, b1, w2, b2, w3, b3, n;
	explicit Layout(int in) : nin(in) {
		w1 = 0;
		b1 = w1 + (long long) H * nin;
		w2 = b1 + H;
		b2 = w2 + (long long) H * H;
		w3 = b2 + H;
		b3 = w3 + H;
		n  = b3 + 1;
	}
};

__device__ __forceinline__ float softplus(float z) { return z > 0.f ? z + log1pf(expf(-z)) : log1pf(expf(z)); }
__device__ __forceinline__ float sigmoidf(float z) { return 1.f / (1.f + expf(-z)); }

// Forward pass of one sample with weights `w` (shared memory, FP32); leaves the hidden activations in
// a1/a2 and returns the logit.
__device__ __forceinline__ float forward(const float *w, const Layout &L, const float *x, float *a1, float *a2) {
#pragma unroll
	for (int j = 0; j < H; ++j) {
		float z = w[L.b1 + j];
		for (int i = 0; i < L.nin; ++i) z += w[L.w1 + j * L.nin + i] * x[i];
		a1[j] = fmaxf(z, 0.f);
	}
#pragma unroll 4
	for (int k = 0; k < H; ++k) {
		float z = w[L.b2 + k];
#pragma unroll
		for (int j = 0; j < H; ++j) z += w[L.w2 + k * H + j] * a1[j];
		a2[k] = fmaxf(z, 0.f);
	}
	float z = w[L.b3];
#pragma unroll
	for (int k = 0; k < H; ++k) z += w[L.w3 + k] * a2[k];
	return z;
}

__global__ void k_predict(const __nv_bfloat16 *wb, Layout L, const float *x, long long n, float *prob) {
	extern __shared__ float sw[];
	for (long long p = threadIdx.x; p < L.n; p += blockDim.x) sw[p] = __bfloat162float(wb[p]);
	__syncthreads();
	float a1[H], a2[H], xi[MAX_IN];
	for (long long s = (long long) blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (long long) gridDim.x * blockDim.x) {
		for (int i = 0; i < L.nin; ++i) xi[i] = x[s * L.nin + i];
		prob[s] = sigmoidf(forward(sw, L, xi, a1, a2));
	}
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Adds v, summed over the warp, to sg[p] (one shared-memory atomic per warp).
__device__ __forceinline__ void acc(float *sg, long long p, float v) {
	v = warp_sum(v);
	if ((threadIdx.x & 31) == 0) atomicAdd(sg + p, v);
}

// Sums of the loss and of its gradient over samples [first, first + count) of the order `perm` (or
// the identity when perm is null) into loss_sum / grad (global, FP32 gradient, FP64 loss).
__global__ void __launch_bounds__(TPB) k_grad(const float *w, Layout L, const float *x, const float *y, const int *perm,
                                              long long first, long long count, float pw, float *grad, double *loss_sum) {
	extern __shared__ float sm[];
	float *sw = sm;
	float *sg = sm + L.n;
	for (long long p = threadIdx.x; p < L.n; p += blockDim.x) sw[p] = w[p], sg[p] = 0.f;
	__syncthreads();
	double lsum = 0.0;
	for (long long base = (long long) blockIdx.x * blockDim.x; base < count; base += (long long) gridDim.x * blockDim.x) {
		const long long t = base + threadIdx.x;
		const bool live   = t < count;
		float xi[MAX_IN], a1[H], a2[H];
		float yt = 0.f;
		if (live) {
			const long long s = perm ? (long long) perm[first + t] : first + t;
			for (int i = 0; i < L.nin; ++i) xi[i] = x[s * L.nin + i];
			yt = y[s];
		} else {
			for (int i = 0; i < L.nin; ++i) xi[i] = 0.f;
		}
		const float z  = forward(sw, L, xi, a1, a2);
		float dz       = sigmoidf(z) * (pw * yt + 1.f - yt) - pw * yt;
		if (!live) dz = 0.f;
		if (live) lsum += (double) (pw * yt * softplus(-z) + (1.f - yt) * softplus(z));
		// output layer
		acc(sg, L.b3, dz);
		float dz2[H];
#pragma unroll
		for (int k = 0; k < H; ++k) {
			acc(sg, L.w3 + k, dz * a2[k]);
			dz2[k] = a2[k] > 0.f ? dz * sw[L.w3 + k] : 0.f;
		}
		// second hidden layer
		float dz1[H];
#pragma unroll
		for (int j = 0; j < H; ++j) dz1[j] = 0.f;
#pragma unroll 1
		for (int k = 0; k < H; ++k) {
			const float d = dz2[k];
			acc(sg, L.b2 + k, d);
#pragma unroll
			for (int j = 0; j < H; ++j) {
				acc(sg, L.w2 + k * H + j, d * a1[j]);
				dz1[j] += sw[L.w2 + k * H + j] * d;
			}
		}
		// first hidden layer
#pragma unroll
		for (int j = 0; j < H; ++j) {
			const float d = a1[j] > 0.f ? dz1[j] : 0.f;
			acc(sg, L.b1 + j, d);
			for (int i = 0; i < L.nin; ++i) acc(sg, L.w1 + j * L.nin + i, d * xi[i]);
		}
	}
	__syncthreads();
	for (long long p = threadIdx.x; p < L.n; p += blockDim.x) atomicAdd(grad + p, sg[p]);
	// loss: one atomic per warp
	for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
	if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, lsum);
}

// One Adam step on the mean gradient (grad * scale); refreshes the BF16 copies and clears grad.
__global__ void k_adam(float *w, __nv_bfloat16 *wb, float *grad, float *m, float *v, long long n, float lr, float scale,
                       float bc1, float bc2) {
	constexpr float B1 = 0.9f, B2 = 0.999f, EPS = 1e-8f;
	for (long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long) gridDim.x * blockDim.x) {
		const float g = grad[p] * scale;
		m[p]          = B1 * m[p] + (1.f - B1) * g;
		v[p]          = B2 * v[p] + (1.f - B2) * g * g;
		w[p] -= lr * (m[p] / bc1) / (sqrtf(v[p] / bc2) + EPS);
		wb[p]    = __float2bfloat16(w[p]);
		grad[p]  = 0.f;
	}
}

__global__ void k_to_bf16(const float *w, __nv_bfloat16 *wb, long long n) {
	for (long long p = (long long) blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long) gridDim.x * blockDim.x)
		wb[p] = __float2bfloat16(w[p]);
}

uint64_t splitmix(uint64_t &s) {
	uint64_t z = (s += 0x9E3779B97F4A7C15ull);
	z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}
double uniform01(uint64_t &s) { return (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

int grid_of(long long n) {
	long long b = (n + TPB - 1) / TPB;
	return (int) (b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

}  // namespace

struct dg_mlp {
	Layout L{1};
	int device = 0;
	cudaStream_t st = nullptr;
	float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
	__nv_bfloat16 *wb = nullptr;
	double *loss = nullptr;
	int t = 0;
};

namespace {

int fail(int code, const std::string &msg) {
	g_mlp_error = msg;
	return code;
}

#define MLP_CUDA(call)                                                                        \
	do {                                                                                      \
		cudaError_t e_ = (call);                                                              \
		if (e_ != cudaSuccess) return fail(DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
	} while (0)

size_t smem_predict(const Layout &L) { return sizeof(float) * L.n; }
size_t smem_grad(const Layout &L) { return 2 * sizeof(float) * L.n; }

// Device copies of host arrays, freed on scope exit.
struct DevBuf {
	void *p = nullptr;
	~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

extern "C" {

const char *dg_mlp_last_error(void) { return g_mlp_error.c_str(); }

static int mlp_create_steps(dg_mlp *h, int n_in, unsigned long long seed) {
	h->L = Layout(n_in);
	const long long n = h->L.n;
	MLP_CUDA(cudaGetDevice(&h->device));
	MLP_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
	MLP_CUDA(cudaMalloc(&h->w, sizeof(float) * n));
	MLP_CUDA(cudaMalloc(&h->g, sizeof(float) * n));
	MLP_CUDA(cudaMalloc(&h->m, sizeof(float) * n));
	MLP_CUDA(cudaMalloc(&h->v, sizeof(float) * n));
	MLP_CUDA(cudaMalloc(&h->wb, sizeof(__nv_bfloat16) * n));
	MLP_CUDA(cudaMalloc(&h->loss, sizeof(double)));
	MLP_CUDA(cudaFuncSetAttribute(k_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_grad(h->L)));
	MLP_CUDA(cudaFuncSetAttribute(k_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_predict(h->L)));
	// He-uniform hidden layers, Glorot-uniform output layer, zero biases
	std::vector<float> w(n, 0.f);
	uint64_t s = seed;
	auto fill = [&](long long off, long long cnt, double lim) {
		for (long long k = 0; k < cnt; ++k) w[off + k] = (float) ((2.0 * uniform01(s) - 1.0) * lim);
	};
	fill(h->L.w1, (long long) H * n_in, std::sqrt(6.0 / n_in));
	fill(h->L.w2, (long long) H * H, std::sqrt(6.0 / H));
	fill(h->L.w3, H, std::sqrt(6.0 / (H + 1)));
	return dg_mlp_set_params(h, w.data());
}

int dg_mlp_create(int n_in, unsigned long long seed, dg_mlp **out) {
	if (!out || n_in < 1 || n_in > MAX_IN) return fail(DG_ERR_ARG, "dg_mlp_create: n_in must be in [1, 32]");
	*out = nullptr;
	dg_mlp *h = new dg_mlp();
	const int rc = mlp_create_steps(h, n_in, seed);
	if (rc != DG_OK) {
		// release whatever the failed step left allocated; the error text of the failure is kept
		const std::string msg = g_mlp_error;
		dg_mlp_destroy(h);
		g_mlp_error = msg;
		return rc;
	}
	*out = h;
	return DG_OK;
}

int dg_mlp_param_count(dg_mlp *h, long long *n) {
	if (!h || !n) return fail(DG_ERR_ARG, "dg_mlp_param_count: null argument");
	*n = h->L.n;
	return DG_OK;
}

int dg_mlp_set_params(dg_mlp *h, const float *params) {
	if (!h || !params) return fail(DG_ERR_ARG, "dg_mlp_set_params: null argument");
	const long long n = h->L.n;
	MLP_CUDA(cudaSetDevice(h->device));
	MLP_CUDA(cudaMemcpyAsync(h->w, params, sizeof(float) * n, cudaMemcpyHostToDevice, h->st));
	MLP_CUDA(cudaMemsetAsync(h->g, 0, sizeof(float) * n, h->st));
	MLP_CUDA(cudaMemsetAsync(h->m, 0, sizeof(float) * n, h->st));
	MLP_CUDA(cudaMemsetAsync(h->v, 0, sizeof(float) * n, h->st));
	k_to_bf16<<<grid_of(n), TPB, 0, h->st>>>(h->w, h->wb, n);
	MLP_CUDA(cudaGetLastError());
	MLP_CUDA(cudaStreamSynchronize(h->st));
	h->t = 0;
	return DG_OK;
}

int dg_mlp_get_params(dg_mlp *h, float *params) {
	if (!h || !params) return fail(DG_ERR_ARG, "dg_mlp_get_params: null argument");
	MLP_CUDA(cudaSetDevice(h->device));
	MLP_CUDA(cudaMemcpyAsync(params, h->w, sizeof(float) * h->L.n, cudaMemcpyDeviceToHost, h->st));
	MLP_CUDA(cudaStreamSynchronize(h->st));
	return DG_OK;
}

int dg_mlp_predict(dg_mlp *h, const float *x, long long n, float *prob) {
	if (!h || (!x && n > 0) || (!prob && n > 0) || n < 0) return fail(DG_ERR_ARG, "dg_mlp_predict: bad argument");
	if (n == 0) return DG_OK;
	MLP_CUDA(cudaSetDevice(h->device));
	DevBuf dx, dp;
	MLP_CUDA(cudaMalloc(&dx.p, sizeof(float) * n * h->L.nin));
	MLP_CUDA(cudaMalloc(&dp.p, sizeof(float) * n));
	MLP_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(float) * n * h->L.nin, cudaMemcpyHostToDevice, h->st));
	k_predict<<<grid_of(n), TPB, smem_predict(h->L), h->st>>>(h->wb, h->L, (const float *) dx.p, n, (float *) dp.p);
	MLP_CUDA(cudaGetLastError());
	MLP_CUDA(cudaMemcpyAsync(prob, dp.p, sizeof(float) * n, cudaMemcpyDeviceToHost, h->st));
	MLP_CUDA(cudaStreamSynchronize(h->st));
	return DG_OK;
}

int dg_mlp_loss_grad(dg_mlp *h, const float *x, const float *y, long long n, float pos_weight, float *grad,
                     double *loss) {
	if (!h || !x || !y || !grad || !loss || n <= 0) return fail(DG_ERR_ARG, "dg_mlp_loss_grad: bad argument");
	MLP_CUDA(cudaSetDevice(h->device));
	DevBuf dx, dy;
	MLP_CUDA(cudaMalloc(&dx.p, sizeof(float) * n * h->L.nin));
	MLP_CUDA(cudaMalloc(&dy.p, sizeof(float) * n));
	MLP_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(float) * n * h->L.nin, cudaMemcpyHostToDevice, h->st));
	MLP_CUDA(cudaMemcpyAsync(dy.p, y, sizeof(float) * n, cudaMemcpyHostToDevice, h->st));
	MLP_CUDA(cudaMemsetAsync(h->g, 0, sizeof(float) * h->L.n, h->st));
	MLP_CUDA(cudaMemsetAsync(h->loss, 0, sizeof(double), h->st));
	k_grad<<<grid_of(n), TPB, smem_grad(h->L), h->st>>>(h->w, h->L, (const float *) dx.p, (const float *) dy.p, nullptr,
	                                                     0, n, pos_weight, h->g, h->loss);
	MLP_CUDA(cudaGetLastError());
	MLP_CUDA(cudaMemcpyAsync(grad, h->g, sizeof(float) * h->L.n, cudaMemcpyDeviceToHost, h->st));
	MLP_CUDA(cudaMemcpyAsync(loss, h->loss, sizeof(double), cudaMemcpyDeviceToHost, h->st));
	MLP_CUDA(cudaMemsetAsync(h->g, 0, sizeof(float) * h->L.n, h->st));
	MLP_CUDA(cudaStreamSynchronize(h->st));
	return DG_OK;
}

int dg_mlp_train(dg_mlp *h, const float *x, const float *y, long long n, int epochs, int batch, float lr,
                 float pos_weight, unsigned long long seed, double *mean_loss) {
	if (!h || !x || !y || n <= 0 || epochs < 1 || batch < 1 || lr <= 0.f)
		return fail(DG_ERR_ARG, "dg_mlp_train: bad argument");
	MLP_CUDA(cudaSetDevice(h->device));
	DevBuf dx, dy, dperm;
	MLP_CUDA(cudaMalloc(&dx.p, sizeof(float) * n * h->L.nin));
	MLP_CUDA(cudaMalloc(&dy.p, sizeof(float) * n));
	MLP_CUDA(cudaMalloc(&dperm.p, sizeof(int) * n));
	MLP_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(float) * n * h->L.nin, cudaMemcpyHostToDevice, h->st));
	MLP_CUDA(cudaMemcpyAsync(dy.p, y, sizeof(float) * n, cudaMemcpyHostToDevice, h->st));
	std::vector<int> perm(n);
	for (long long k = 0; k < n; ++k) perm[k] = (int) k;
	uint64_t s = seed;
	double last = 0.0;
	for (int e = 0; e < epochs; ++e) {
		for (long long k = n - 1; k > 0; --k) std::swap(perm[k], perm[(long long) (splitmix(s) % (uint64_t) (k + 1))]);
		MLP_CUDA(cudaMemcpyAsync(dperm.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->st));
		MLP_CUDA(cudaMemsetAsync(h->loss, 0, sizeof(double), h->st));
		for (long long first = 0; first < n; first += batch) {
			const long long cnt = std::min<long long>(batch, n - first);
			k_grad<<<grid_of(cnt), TPB, smem_grad(h->L), h->st>>>(h->w, h->L, (const float *) dx.p, (const float *) dy.p,
			                                                       (const int *) dperm.p, first, cnt, pos_weight, h->g,
			                                                       h->loss);
			h->t++;
			const float bc1 = 1.f - std::pow(0.9f, (float) h->t), bc2 = 1.f - std::pow(0.999f, (float) h->t);
			k_adam<<<grid_of(h->L.n), TPB, 0, h->st>>>(h->w, h->wb, h->g, h->m, h->v, h->L.n, lr, 1.f / (float) cnt, bc1,
			                                            bc2);
		}
		MLP_CUDA(cudaGetLastError());
		double sum = 0.0;
		MLP_CUDA(cudaMemcpyAsync(&sum, h->loss, sizeof(double), cudaMemcpyDeviceToHost, h->st));
		MLP_CUDA(cudaStreamSynchronize(h->st));
		last = sum / (double) n;
	}
	if (mean_loss) *mean_loss = last;
	return DG_OK;
}

int dg_mlp_destroy(dg_mlp *h) {
	if (!h) return DG_OK;
	cudaSetDevice(h->device);
	if (h->st) cudaStreamSynchronize(h->st);
	cudaFree(h->w);
	cudaFree(h->g);
	cudaFree(h->m);
	cudaFree(h->v);
	cudaFree(h->wb);
	cudaFree(h->loss);
	if (h->st) cudaStreamDestroy(h->st);
	delete h;
	return DG_OK;
}

}  // extern "C"
