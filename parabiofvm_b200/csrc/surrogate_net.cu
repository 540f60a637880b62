// The learned surrogate network: a 3D convolutional operator that advances the field 16 steps at
// once from the current field and the agents' voxelised source and sink rates.
//
//   features  [B][V][32] bf16: field (S), sources x 16 (S), sinks x 16 (S), zeros
//   h0 = relu(conv0(features))
//   h_{k+1} = h_k + conv_{2k+2}(relu(conv_{2k+1}(h_k)))          k = 0..3
//   field(t + 16 dt) = field(t) + conv9(h4)[:S]                  (f32)
//
// Ten convolutions (surrogate.cu), bf16 weights and activations with f32 accumulation, trained on
// the mean squared error with Adam on f32 master weights.  The backward pass runs the same
// convolution kernel on the gradients with flipped weights and the weight-gradient kernel; the
// element-wise steps (features, loss, bias gradients, weight casts, Adam) are the small kernels
// below.  Data for training comes from the plain solver: sources and sinks per voxel are the
// secretion terms of one step (src/solver/host/cell_solver.cpp:63-85), summed over the voxel's
// agents.

#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "bfvm_internal.h"
#include "surrogate.h"

namespace bfvm {

static constexpr float SUR_FEATURE_SCALE = 16.f; // rates per step -> per macro-step of 16 steps
static constexpr int SUR_PARAMS = SUR_LAYERS * SUR_LAYER_PARAMS;

__global__ void sur_features_kernel(long long n, int S, const float* __restrict__ field, const float* __restrict__ src,
									const float* __restrict__ sink, __nv_bfloat16* __restrict__ feat)
{
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
	{
		__nv_bfloat16* f = feat + v * SUR_C;
		for (int c = 0; c < SUR_C; c++)
		{
			float x = 0.f;
			if (c < S)
				x = field[v * S + c];
			else if (c < 2 * S)
				x = src[v * S + c - S] * SUR_FEATURE_SCALE;
			else if (c < 3 * S)
				x = sink[v * S + c - 2 * S] * SUR_FEATURE_SCALE;
			f[c] = __float2bfloat16_rn(x);
		}
	}
}

// forward weights wf[l][t][co][ci] and the backward ones wb[l][26 - t][ci][co], both bf16
__global__ void sur_weights_kernel(const float* __restrict__ params, __nv_bfloat16* __restrict__ wf,
								   __nv_bfloat16* __restrict__ wb)
{
	const int per = SUR_TAPS * SUR_C * SUR_C;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < SUR_LAYERS * per; i += gridDim.x * blockDim.x)
	{
		const int l = i / per, r = i % per;
		const int t = r / (SUR_C * SUR_C), co = (r / SUR_C) % SUR_C, ci = r % SUR_C;
		const __nv_bfloat16 w = __float2bfloat16_rn(params[(size_t)l * SUR_LAYER_PARAMS + r]);
		wf[i] = w;
		wb[(size_t)l * per + ((size_t)(SUR_TAPS - 1 - t) * SUR_C + ci) * SUR_C + co] = w;
	}
}

// loss += sum (pred - target)^2 over the S channels; g = d(mean)/d(pred) as bf16 [n][32]
__global__ void sur_loss_kernel(long long n, int S, const float* __restrict__ pred, const float* __restrict__ target,
								__nv_bfloat16* __restrict__ g, float inv_count, float* __restrict__ loss)
{
	float acc = 0.f;
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
	{
		__nv_bfloat16* gv = g + v * SUR_C;
		for (int c = 0; c < SUR_C; c++)
		{
			float d = 0.f;
			if (c < S)
			{
				d = pred[v * S + c] - target[v * S + c];
				acc += d * d;
			}
			gv[c] = __float2bfloat16_rn(2.f * d * inv_count);
		}
	}
	for (int o = 16; o > 0; o >>= 1)
		acc += __shfl_xor_sync(0xffffffffu, acc, o);
	__shared__ float part[32];
	if ((threadIdx.x & 31) == 0)
		part[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x < 32)
	{
		float a = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.f;
		for (int o = 16; o > 0; o >>= 1)
			a += __shfl_xor_sync(0xffffffffu, a, o);
		if (threadIdx.x == 0)
			atomicAdd(loss, a);
	}
}

// db[c] += sum over voxels of g[v][c]; thread c % 32 of each warp owns channel c
__global__ void sur_bias_grad_kernel(long long n, const __nv_bfloat16* __restrict__ g, float* __restrict__ db)
{
	const int c = threadIdx.x & 31;
	const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
	const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
	float acc = 0.f;
	for (long long v = w0; v < n; v += nw)
		acc += __bfloat162float(g[v * SUR_C + c]);
	__shared__ float part[8][32];
	part[threadIdx.x >> 5][c] = acc;
	__syncthreads();
	if (threadIdx.x < 32)
	{
		float a = 0.f;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++)
			a += part[w][threadIdx.x];
		atomicAdd(&db[threadIdx.x], a);
	}
}

__global__ void sur_adam_kernel(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
								float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const float gi = g[i];
		const float mi = b1 * m[i] + (1.f - b1) * gi;
		const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
		m[i] = mi;
		v[i] = vi;
		p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
	}
}

// One step's secretion terms of every agent, summed per voxel (cell_solver.cpp:63-85 of the
// reference): sources += S T dt vol / V_vox + N dt / V_vox, sinks += (U + S) dt vol / V_vox.
__global__ void sur_agent_rates_kernel(int A, int S, const float* __restrict__ sec, const float* __restrict__ sat,
									   const float* __restrict__ upt, const float* __restrict__ nex,
									   const float* __restrict__ vol, const float* __restrict__ pos, int3 bmin, int3 vox,
									   int3 grid, float dt, float* __restrict__ src, float* __restrict__ sink,
									   int* __restrict__ err)
{
	const long long total = (long long)A * S;
	const float vv = (float)vox.x * vox.y * vox.z;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
		 i += (long long)gridDim.x * blockDim.x)
	{
		const int a = (int)(i / S), s = (int)(i % S);
		const float* p = pos + (size_t)a * 3;
		const float tx = __fdiv_rn(__fsub_rn(p[0], (float)bmin.x), (float)vox.x);
		const float ty = __fdiv_rn(__fsub_rn(p[1], (float)bmin.y), (float)vox.y);
		const float tz = __fdiv_rn(__fsub_rn(p[2], (float)bmin.z), (float)vox.z);
		if (!(tx > -1.f && tx < grid.x && ty > -1.f && ty < grid.y && tz > -1.f && tz < grid.z))
		{
			if (s == 0 && err)
				atomicOr(err, DEVERR_AGENT_OUTSIDE);
			continue;
		}
		const long long v = (long long)(int)tx + (long long)grid.x * ((long long)(int)ty + (long long)grid.y * (int)tz);
		const float w = dt * vol[a] / vv;
		atomicAdd(&src[v * S + s], sec[i] * sat[i] * w + nex[i] * dt / vv);
		atomicAdd(&sink[v * S + s], (upt[i] + sec[i]) * w);
	}
}

// field[v][s] = sum over bumps of amp * exp(-|x - c|^2 / (2 w^2)), bump parameters [S][bumps][5]
// = (cx, cy, cz, w, amp) in voxel units, passed by value (at most 10 substrates x 16 bumps)
static constexpr int SUR_MAX_BUMPS = 16;
struct bump_set
{
	float p[10 * SUR_MAX_BUMPS * 5];
};

__global__ void sur_bumps_kernel(long long V, int S, int X, int Y, int bumps, const __grid_constant__ bump_set bs,
								 float* __restrict__ field)
{
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < V * S; i += (long long)gridDim.x * blockDim.x)
	{
		const long long v = i / S;
		const int s = (int)(i % S);
		const float x = (float)(v % X), y = (float)((v / X) % Y), z = (float)(v / ((long long)X * Y));
		float acc = 0.f;
		for (int k = 0; k < bumps; k++)
		{
			const float* b = bs.p + ((size_t)s * bumps + k) * 5;
			const float dx = x - b[0], dy = y - b[1], dz = z - b[2];
			acc += b[4] * __expf(-(dx * dx + dy * dy + dz * dz) / (2.f * b[3] * b[3]));
		}
		field[i] = acc;
	}
}

static int grid_for(long long n, int threads = 256)
{
	return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16));
}

} // namespace bfvm

using namespace bfvm;

struct bfvm_surrogate
{
	int device = 0;
	cudaStream_t stream = nullptr, own_stream = nullptr;
	int X = 0, Y = 0, Z = 0, S = 0, max_batch = 0;
	long long V = 0;
	float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
	__nv_bfloat16 *wf = nullptr, *wb = nullptr;
	__nv_bfloat16 *feat = nullptr, *h[5] = {}, *t[4] = {}, *g[3] = {};
	float* loss = nullptr;
	float* host_loss = nullptr;
	int* dev_error = nullptr;
	int* host_error = nullptr;
	long long adam_steps = 0;
	bool weights_dirty = true;
};

namespace {

void sur_free(bfvm_surrogate* n)
{
	if (n->device >= 0)
		cudaSetDevice(n->device);
	device_free(n->params);
	device_free(n->grads);
	device_free(n->adam_m);
	device_free(n->adam_v);
	device_free(n->wf);
	device_free(n->wb);
	device_free(n->feat);
	for (auto& p : n->h)
		device_free(p);
	for (auto& p : n->t)
		device_free(p);
	for (auto& p : n->g)
		device_free(p);
	device_free(n->loss);
	device_free(n->dev_error);
	if (n->host_loss)
		cudaFreeHost(n->host_loss);
	if (n->host_error)
		cudaFreeHost(n->host_error);
	if (n->own_stream)
		cudaStreamDestroy(n->own_stream);
}

int refresh_weights(bfvm_surrogate* n)
{
	if (!n->weights_dirty)
		return BFVM_OK;
	sur_weights_kernel<<<grid_for((long long)SUR_LAYERS * SUR_TAPS * SUR_C * SUR_C), 256, 0, n->stream>>>(n->params, n->wf,
																										   n->wb);
	BFVM_CUDA(cudaGetLastError());
	n->weights_dirty = false;
	return BFVM_OK;
}

const __nv_bfloat16* wf_of(const bfvm_surrogate* n, int l) { return n->wf + (size_t)l * SUR_TAPS * SUR_C * SUR_C; }
const __nv_bfloat16* wb_of(const bfvm_surrogate* n, int l) { return n->wb + (size_t)l * SUR_TAPS * SUR_C * SUR_C; }
const float* bias_of(const bfvm_surrogate* n, int l)
{
	return n->params + (size_t)l * SUR_LAYER_PARAMS + SUR_TAPS * SUR_C * SUR_C;
}

conv_params base_params(const bfvm_surrogate* n, int batch)
{
	conv_params p;
	std::memset(&p, 0, sizeof(p));
	p.X = n->X;
	p.Y = n->Y;
	p.Z = n->Z;
	p.B = batch;
	p.err = n->dev_error;
	return p;
}

int conv(const bfvm_surrogate* n, const __nv_bfloat16* in, const __nv_bfloat16* w, const conv_params& p)
{
	return launch_sur_conv(in, w, p, n->device, n->stream);
}

// features -> prediction; keeps every activation the backward pass needs
int forward(bfvm_surrogate* n, int batch, const float* field, const float* src, const float* sink, float* pred)
{
	int st;
	if ((st = refresh_weights(n)))
		return st;
	const long long nv = n->V * batch;
	sur_features_kernel<<<grid_for(nv), 256, 0, n->stream>>>(nv, n->S, field, src, sink, n->feat);
	BFVM_CUDA(cudaGetLastError());
	conv_params p = base_params(n, batch);
	p.bias = bias_of(n, 0);
	p.relu = 1;
	p.out = n->h[0];
	if ((st = conv(n, n->feat, wf_of(n, 0), p)))
		return st;
	for (int k = 0; k < 4; k++)
	{
		p = base_params(n, batch);
		p.bias = bias_of(n, 2 * k + 1);
		p.relu = 1;
		p.out = n->t[k];
		if ((st = conv(n, n->h[k], wf_of(n, 2 * k + 1), p)))
			return st;
		p = base_params(n, batch);
		p.bias = bias_of(n, 2 * k + 2);
		p.residual = n->h[k];
		p.out = n->h[k + 1];
		if ((st = conv(n, n->t[k], wf_of(n, 2 * k + 2), p)))
			return st;
	}
	p = base_params(n, batch);
	p.bias = bias_of(n, 9);
	p.out_f32 = pred;
	p.base_f32 = field;
	p.out_ch = n->S;
	return conv(n, n->h[4], wf_of(n, 9), p);
}

int wgrad(bfvm_surrogate* n, int batch, int layer, const __nv_bfloat16* in, const __nv_bfloat16* g)
{
	float* dW = n->grads + (size_t)layer * SUR_LAYER_PARAMS;
	int st = launch_sur_wgrad(in, g, dW, base_params(n, batch), n->device, n->stream);
	if (st)
		return st;
	const long long nv = n->V * batch;
	sur_bias_grad_kernel<<<grid_for(nv * 32, 256), 256, 0, n->stream>>>(nv, g, dW + SUR_TAPS * SUR_C * SUR_C);
	BFVM_CUDA(cudaGetLastError());
	return BFVM_OK;
}

// loss and gradients of every parameter (n->grads) for one batch
int gradients(bfvm_surrogate* n, int batch, const float* field, const float* src, const float* sink,
			  const float* target, float* pred)
{
	int st;
	if ((st = forward(n, batch, field, src, sink, pred)))
		return st;
	const long long nv = n->V * batch;
	BFVM_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(float), n->stream));
	BFVM_CUDA(cudaMemsetAsync(n->grads, 0, (size_t)SUR_PARAMS * sizeof(float), n->stream));
	sur_loss_kernel<<<grid_for(nv), 256, 0, n->stream>>>(nv, n->S, pred, target, n->g[0], 1.f / (float)(nv * n->S),
														 n->loss);
	BFVM_CUDA(cudaGetLastError());
	// projection
	if ((st = wgrad(n, batch, 9, n->h[4], n->g[0])))
		return st;
	conv_params p = base_params(n, batch);
	p.out = n->g[1];
	if ((st = conv(n, n->g[0], wb_of(n, 9), p)))
		return st;
	int gh = 1; // buffer holding dL/dh_{k+1}
	for (int k = 3; k >= 0; k--)
	{
		// h_{k+1} = h_k + conv_{2k+2}(t_k),  t_k = relu(conv_{2k+1}(h_k))
		if ((st = wgrad(n, batch, 2 * k + 2, n->t[k], n->g[gh])))
			return st;
		p = base_params(n, batch);
		p.mask = n->t[k];
		p.out = n->g[2];
		if ((st = conv(n, n->g[gh], wb_of(n, 2 * k + 2), p)))
			return st;
		if ((st = wgrad(n, batch, 2 * k + 1, n->h[k], n->g[2])))
			return st;
		const int next = gh == 1 ? 0 : 1;
		p = base_params(n, batch);
		p.residual = n->g[gh];
		if (k == 0)
			p.mask = n->h[0]; // h0 = relu(conv0(features))
		p.out = n->g[next];
		if ((st = conv(n, n->g[2], wb_of(n, 2 * k + 1), p)))
			return st;
		gh = next;
	}
	return wgrad(n, batch, 0, n->feat, n->g[gh]);
}

int check_batch(const bfvm_surrogate* n, int batch)
{
	if (batch < 1 || batch > n->max_batch)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "batch must be 1.." + std::to_string(n->max_batch));
	return BFVM_OK;
}

int read_loss(bfvm_surrogate* n, int batch, float* loss)
{
	if (!loss)
		return BFVM_OK;
	BFVM_CUDA(cudaMemcpyAsync(n->host_loss, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
	BFVM_CUDA(cudaMemcpyAsync(n->host_error, n->dev_error, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
	BFVM_CUDA(cudaStreamSynchronize(n->stream));
	if (*n->host_error)
		return fail(BFVM_ERR_TIMEOUT, "a surrogate kernel timed out waiting for a copy or an MMA");
	*loss = *n->host_loss / (float)(n->V * batch * n->S);
	return BFVM_OK;
}

} // namespace

#define CHECK_NET(n)                                                                                                   \
	do                                                                                                                 \
	{                                                                                                                  \
		if (!(n))                                                                                                      \
			return fail(BFVM_ERR_INVALID_ARGUMENT, "null surrogate");                                                  \
		if (cudaSetDevice((n)->device) != cudaSuccess)                                                                 \
			return cuda_fail(cudaGetLastError(), "cudaSetDevice");                                                     \
	} while (0)

extern "C" {

int bfvm_sur_create(bfvm_surrogate** out, int device, const int32_t grid_shape[3], int32_t substrates,
					int32_t max_batch, uint64_t seed)
{
	if (!out || !grid_shape)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	*out = nullptr;
	if (substrates < 1 || 3 * substrates > SUR_C)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "the surrogate takes 1..10 substrates (3 feature channels each)");
	if (max_batch < 1)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "max_batch must be positive");
	int st;
	if ((st = sur_check_shape(grid_shape[0], grid_shape[1], grid_shape[2], max_batch)))
		return st;
	auto* n = new (std::nothrow) bfvm_surrogate();
	if (!n)
		return fail(BFVM_ERR_OUT_OF_MEMORY, "host allocation failed");
	n->device = device;
	n->X = grid_shape[0];
	n->Y = grid_shape[1];
	n->Z = grid_shape[2];
	n->S = substrates;
	n->max_batch = max_batch;
	n->V = (long long)n->X * n->Y * n->Z;
	do
	{
		if (cudaSetDevice(device) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "cudaSetDevice");
			break;
		}
		if (cudaStreamCreateWithFlags(&n->own_stream, cudaStreamNonBlocking) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "cudaStreamCreate");
			break;
		}
		n->stream = n->own_stream;
		const size_t act = (size_t)n->V * max_batch * SUR_C;
		const size_t wsz = (size_t)SUR_LAYERS * SUR_TAPS * SUR_C * SUR_C;
		if ((st = device_alloc(&n->params, (size_t)SUR_PARAMS)) || (st = device_alloc(&n->grads, (size_t)SUR_PARAMS))
			|| (st = device_alloc(&n->adam_m, (size_t)SUR_PARAMS)) || (st = device_alloc(&n->adam_v, (size_t)SUR_PARAMS))
			|| (st = device_alloc(&n->wf, wsz)) || (st = device_alloc(&n->wb, wsz)) || (st = device_alloc(&n->feat, act))
			|| (st = device_alloc(&n->loss, 1)) || (st = device_alloc(&n->dev_error, 1)))
			break;
		for (auto& p : n->h)
			if (!st)
				st = device_alloc(&p, act);
		for (auto& p : n->t)
			if (!st)
				st = device_alloc(&p, act);
		for (auto& p : n->g)
			if (!st)
				st = device_alloc(&p, act);
		if (st)
			break;
		if (cudaMallocHost((void**)&n->host_loss, sizeof(float)) != cudaSuccess
			|| cudaMallocHost((void**)&n->host_error, sizeof(int)) != cudaSuccess)
		{
			(void)cudaGetLastError();
			st = fail(BFVM_ERR_OUT_OF_MEMORY, "pinned host allocation failed");
			break;
		}
		// He-uniform weights (fan-in 27 x 32), the last convolution of every residual branch and
		// the projection scaled by 0.1 so that the untrained network stays close to the identity;
		// zero biases and Adam moments
		std::vector<float> init((size_t)SUR_PARAMS, 0.f);
		std::mt19937_64 rng(seed);
		const float a = std::sqrt(6.f / (SUR_TAPS * SUR_C));
		std::uniform_real_distribution<float> U(-a, a);
		for (int l = 0; l < SUR_LAYERS; l++)
		{
			const float scale = (l == 9 || (l > 0 && l % 2 == 0)) ? 0.1f : 1.f;
			for (int i = 0; i < SUR_TAPS * SUR_C * SUR_C; i++)
				init[(size_t)l * SUR_LAYER_PARAMS + i] = scale * U(rng);
		}
		if (cudaMemcpy(n->params, init.data(), init.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess
			|| cudaMemset(n->adam_m, 0, (size_t)SUR_PARAMS * sizeof(float)) != cudaSuccess
			|| cudaMemset(n->adam_v, 0, (size_t)SUR_PARAMS * sizeof(float)) != cudaSuccess
			|| cudaMemset(n->grads, 0, (size_t)SUR_PARAMS * sizeof(float)) != cudaSuccess
			|| cudaMemset(n->dev_error, 0, sizeof(int)) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "surrogate initialisation");
			break;
		}
		*n->host_error = 0;
	} while (0);
	if (st)
	{
		sur_free(n);
		delete n;
		return st;
	}
	*out = n;
	return BFVM_OK;
}

int bfvm_sur_destroy(bfvm_surrogate* n)
{
	if (!n)
		return BFVM_OK;
	sur_free(n);
	delete n;
	return BFVM_OK;
}

int bfvm_sur_set_stream(bfvm_surrogate* n, void* stream)
{
	CHECK_NET(n);
	n->stream = stream ? static_cast<cudaStream_t>(stream) : n->own_stream;
	return BFVM_OK;
}

int bfvm_sur_parameter_count(const bfvm_surrogate* n, int64_t* count)
{
	if (!n || !count)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	*count = SUR_PARAMS;
	return BFVM_OK;
}

int bfvm_sur_load(bfvm_surrogate* n, const float* params)
{
	CHECK_NET(n);
	if (!params)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null parameters");
	BFVM_CUDA(cudaMemcpyAsync(n->params, params, (size_t)SUR_PARAMS * sizeof(float), cudaMemcpyHostToDevice, n->stream));
	BFVM_CUDA(cudaMemsetAsync(n->adam_m, 0, (size_t)SUR_PARAMS * sizeof(float), n->stream));
	BFVM_CUDA(cudaMemsetAsync(n->adam_v, 0, (size_t)SUR_PARAMS * sizeof(float), n->stream));
	BFVM_CUDA(cudaStreamSynchronize(n->stream));
	n->adam_steps = 0;
	n->weights_dirty = true;
	return BFVM_OK;
}

int bfvm_sur_save(bfvm_surrogate* n, float* params)
{
	CHECK_NET(n);
	if (!params)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null parameters");
	BFVM_CUDA(cudaMemcpyAsync(params, n->params, (size_t)SUR_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
	BFVM_CUDA(cudaStreamSynchronize(n->stream));
	return BFVM_OK;
}

int bfvm_sur_infer(bfvm_surrogate* n, int32_t batch, const float* field, const float* sources, const float* sinks,
				   float* out)
{
	CHECK_NET(n);
	int st;
	if ((st = check_batch(n, batch)))
		return st;
	if (!field || !sources || !sinks || !out)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null device buffer");
	return forward(n, batch, field, sources, sinks, out);
}

int bfvm_sur_gradients(bfvm_surrogate* n, int32_t batch, const float* field, const float* sources, const float* sinks,
					   const float* target, float* prediction, float* loss)
{
	CHECK_NET(n);
	int st;
	if ((st = check_batch(n, batch)))
		return st;
	if (!field || !sources || !sinks || !target || !prediction)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null device buffer");
	if ((st = gradients(n, batch, field, sources, sinks, target, prediction)))
		return st;
	return read_loss(n, batch, loss);
}

int bfvm_sur_load_gradients(bfvm_surrogate* n, float* grads)
{
	CHECK_NET(n);
	if (!grads)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null gradients");
	BFVM_CUDA(cudaMemcpyAsync(grads, n->grads, (size_t)SUR_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
	BFVM_CUDA(cudaStreamSynchronize(n->stream));
	return BFVM_OK;
}

int bfvm_sur_train_step(bfvm_surrogate* n, int32_t batch, const float* field, const float* sources,
						const float* sinks, const float* target, float* prediction, float learning_rate, float* loss)
{
	CHECK_NET(n);
	int st;
	if ((st = check_batch(n, batch)))
		return st;
	if (!field || !sources || !sinks || !target || !prediction)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null device buffer");
	if ((st = gradients(n, batch, field, sources, sinks, target, prediction)))
		return st;
	n->adam_steps++;
	const float b1 = 0.9f, b2 = 0.999f;
	const float bc1 = 1.f - std::pow(b1, (float)n->adam_steps), bc2 = 1.f - std::pow(b2, (float)n->adam_steps);
	sur_adam_kernel<<<grid_for(SUR_PARAMS), 256, 0, n->stream>>>(SUR_PARAMS, n->params, n->grads, n->adam_m, n->adam_v,
																 learning_rate, b1, b2, 1e-8f, bc1, bc2);
	BFVM_CUDA(cudaGetLastError());
	n->weights_dirty = true;
	return read_loss(n, batch, loss);
}

int bfvm_sur_synchronize(bfvm_surrogate* n)
{
	CHECK_NET(n);
	BFVM_CUDA(cudaMemcpyAsync(n->host_error, n->dev_error, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
	BFVM_CUDA(cudaStreamSynchronize(n->stream));
	if (*n->host_error)
		return fail(BFVM_ERR_TIMEOUT, "a surrogate kernel timed out waiting for a copy or an MMA");
	return BFVM_OK;
}

int bfvm_sur_agent_rates(const int32_t bounding_box_mins[3], const int32_t voxel_shape[3], const int32_t grid_shape[3],
						 int32_t substrates, float time_step, int32_t agent_count, const float* secretion_rates,
						 const float* saturation_densities, const float* uptake_rates, const float* net_export_rates,
						 const float* volumes, const float* positions, float* sources, float* sinks,
						 int32_t* error_flags, void* stream)
{
	if (!bounding_box_mins || !voxel_shape || !grid_shape || !sources || !sinks || substrates < 1 || agent_count < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "bad argument");
	if (agent_count > 0
		&& (!secretion_rates || !saturation_densities || !uptake_rates || !net_export_rates || !volumes || !positions))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent arrays must not be null");
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	const size_t cells = (size_t)grid_shape[0] * grid_shape[1] * grid_shape[2] * substrates;
	BFVM_CUDA(cudaMemsetAsync(sources, 0, cells * sizeof(float), s));
	BFVM_CUDA(cudaMemsetAsync(sinks, 0, cells * sizeof(float), s));
	if (agent_count == 0)
		return BFVM_OK;
	const long long total = (long long)agent_count * substrates;
	sur_agent_rates_kernel<<<grid_for(total), 256, 0, s>>>(
		agent_count, substrates, secretion_rates, saturation_densities, uptake_rates, net_export_rates, volumes, positions,
		make_int3(bounding_box_mins[0], bounding_box_mins[1], bounding_box_mins[2]),
		make_int3(voxel_shape[0], voxel_shape[1], voxel_shape[2]), make_int3(grid_shape[0], grid_shape[1], grid_shape[2]),
		time_step, sources, sinks, error_flags);
	BFVM_CUDA(cudaGetLastError());
	return BFVM_OK;
}

int bfvm_sur_random_field(const int32_t grid_shape[3], int32_t substrates, int32_t bumps, const float* bump_params,
						  float* field, void* stream)
{
	if (!grid_shape || !bump_params || !field || substrates < 1 || substrates > 10 || bumps < 1
		|| bumps > SUR_MAX_BUMPS)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "random fields take 1..10 substrates and 1..16 bumps");
	bump_set bs;
	std::memcpy(bs.p, bump_params, (size_t)substrates * bumps * 5 * sizeof(float));
	const long long V = (long long)grid_shape[0] * grid_shape[1] * grid_shape[2];
	sur_bumps_kernel<<<grid_for(V * substrates), 256, 0, static_cast<cudaStream_t>(stream)>>>(
		V, substrates, grid_shape[0], grid_shape[1], bumps, bs, field);
	BFVM_CUDA(cudaGetLastError());
	return BFVM_OK;
}

int bfvm_sur_conv3d(const int32_t shape[4], const void* input, const void* weights, const float* bias,
					const void* residual, int32_t relu, const void* mask, void* out, float* out_f32,
					const float* base_f32, int32_t out_channels, int32_t* error_flags, void* stream)
{
	if (!shape || !input || !weights || !error_flags || (!out && !out_f32))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	if (out_f32 && (out_channels < 1 || out_channels > SUR_C))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "out_channels must be 1..32");
	int dev = 0;
	cudaGetDevice(&dev);
	conv_params p;
	std::memset(&p, 0, sizeof(p));
	p.X = shape[0];
	p.Y = shape[1];
	p.Z = shape[2];
	p.B = shape[3];
	p.bias = bias;
	p.residual = static_cast<const __nv_bfloat16*>(residual);
	p.relu = relu;
	p.mask = static_cast<const __nv_bfloat16*>(mask);
	p.out = static_cast<__nv_bfloat16*>(out);
	p.out_f32 = out_f32;
	p.base_f32 = base_f32;
	p.out_ch = out_channels;
	p.err = error_flags;
	return launch_sur_conv(static_cast<const __nv_bfloat16*>(input), static_cast<const __nv_bfloat16*>(weights), p, dev,
						   static_cast<cudaStream_t>(stream));
}

int bfvm_sur_conv3d_wgrad(const int32_t shape[4], const void* input, const void* grad, float* weight_grad,
						  int32_t* error_flags, void* stream)
{
	if (!shape || !input || !grad || !weight_grad || !error_flags)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	int dev = 0;
	cudaGetDevice(&dev);
	conv_params p;
	std::memset(&p, 0, sizeof(p));
	p.X = shape[0];
	p.Y = shape[1];
	p.Z = shape[2];
	p.B = shape[3];
	p.err = error_flags;
	return launch_sur_wgrad(static_cast<const __nv_bfloat16*>(input), static_cast<const __nv_bfloat16*>(grad),
							weight_grad, p, dev, static_cast<cudaStream_t>(stream));
}

} // extern "C"
