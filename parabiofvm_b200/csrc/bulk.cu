// Bulk supply and uptake (paraBioFVM src/solver/host/bulk_solver.cpp:20-33): for every voxel and
// substrate
//   D = (D + dt * S * T) / (1 + dt * (U + S))
// with supply rate S, uptake rate U and supply target density T.  The reference evaluates three
// host callbacks per voxel on every call; here the rates are tabulated when they are set (one row
// for the whole mesh, or one per voxel), and the two terms that do not depend on D are prepared
// once on the device with the reference's operation order:
//   add = (dt * S) * T,   den = 1 + dt * (U + S)
// so a step is one read-modify-write of the field, D = (D + add) / den, bit for bit the reference.

#include <algorithm>

#include "bfvm_internal.h"

namespace bfvm {

__global__ void bulk_prepare_kernel(long long n, float dt, const float* __restrict__ supply,
									const float* __restrict__ uptake, const float* __restrict__ target,
									float* __restrict__ add, float* __restrict__ den)
{
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
	{
		const float s = supply[t];
		add[t] = __fmul_rn(__fmul_rn(dt, s), target[t]);
		den[t] = __fadd_rn(1.f, __fmul_rn(dt, __fadd_rn(uptake[t], s)));
	}
}

// per-voxel tables: element t of the field uses add[t], den[t]
__global__ void bulk_apply_voxels_kernel(long long n, float* __restrict__ dens, const float* __restrict__ add,
										 const float* __restrict__ den)
{
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
		dens[t] = __fdiv_rn(__fadd_rn(dens[t], __ldg(&add[t])), __ldg(&den[t]));
}

// one row for the mesh: element t uses add[t % S], den[t % S]
__global__ void bulk_apply_uniform_kernel(long long n, int S, float* __restrict__ dens, const float* __restrict__ add,
										  const float* __restrict__ den)
{
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
	{
		const int s = (int)(t % S);
		dens[t] = __fdiv_rn(__fadd_rn(dens[t], __ldg(&add[s])), __ldg(&den[s]));
	}
}

static unsigned grid_for(long long n, int threads)
{
	return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 32));
}

void free_bulk(bfvm_solver* s)
{
	device_free(s->bulk_add);
	device_free(s->bulk_den);
	s->bulk_rows = 0;
}

// Tabulate the rates: [V][S] when per_voxel, else [S].  Per-voxel tables go up in chunks through
// a small staging buffer, so no full-size copy of the three host tables is held on the device.
int set_bulk_rates(bfvm_solver* s, int per_voxel, const float* supply, const float* uptake, const float* target)
{
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	free_bulk(s);
	if (!supply)
		return BFVM_OK;
	const long long rows = per_voxel ? s->V : 1;
	const long long n = rows * s->S;
	int st;
	if ((st = device_alloc(&s->bulk_add, (size_t)n)) || (st = device_alloc(&s->bulk_den, (size_t)n)))
	{
		free_bulk(s);
		return st;
	}
	const long long chunk = std::min<long long>(n, 1LL << 22);
	float* stage = nullptr;
	if ((st = device_alloc(&stage, (size_t)(3 * chunk))))
	{
		free_bulk(s);
		return st;
	}
	for (long long off = 0; off < n && !st; off += chunk)
	{
		const long long m = std::min(chunk, n - off);
		cudaError_t e = cudaMemcpyAsync(stage, supply + off, m * sizeof(float), cudaMemcpyHostToDevice, s->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(stage + chunk, uptake + off, m * sizeof(float), cudaMemcpyHostToDevice, s->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(stage + 2 * chunk, target + off, m * sizeof(float), cudaMemcpyHostToDevice, s->stream);
		if (e != cudaSuccess)
		{
			st = cuda_fail(e, "cudaMemcpyAsync(bulk rates)");
			break;
		}
		bulk_prepare_kernel<<<grid_for(m, 256), 256, 0, s->stream>>>(m, s->dt, stage, stage + chunk, stage + 2 * chunk,
																	  s->bulk_add + off, s->bulk_den + off);
		st = check_launch(s, "bulk_prepare_kernel");
	}
	cudaError_t e = cudaStreamSynchronize(s->stream);
	device_free(stage);
	if (!st && e != cudaSuccess)
		st = cuda_fail(e, "cudaStreamSynchronize(bulk rates)");
	if (st)
	{
		free_bulk(s);
		return st;
	}
	s->bulk_rows = rows;
	return BFVM_OK;
}

int launch_bulk(bfvm_solver* s)
{
	if (!s->bulk_rows)
		return fail(BFVM_ERR_STATE, "no bulk rates set (bfvm_set_bulk_rates)");
	const long long n = s->V * s->S;
	if (s->bulk_rows == 1)
		bulk_apply_uniform_kernel<<<grid_for(n, 256), 256, 0, s->stream>>>(n, s->S, s->dens, s->bulk_add, s->bulk_den);
	else
		bulk_apply_voxels_kernel<<<grid_for(n, 256), 256, 0, s->stream>>>(n, s->dens, s->bulk_add, s->bulk_den);
	return check_launch(s, "bulk_apply_kernel");
}

} // namespace bfvm
