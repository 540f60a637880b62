// Autotuning of the staged sweeps' launch shape: warp groups per CTA (how many tiles of 32 lines a
// CTA solves at once) and pipeline stages per group (how many tiles are in flight).  The built-in
// choice follows the shared-memory budget and the tile count; bfvm_autotune measures every shape
// that fits, per axis, on a scratch copy of the field, keeps the fastest in the solver, and records
// it in a process-wide cache keyed by the mesh shape, so later solvers of the same shape (the
// members of a batch, say) use it without measuring.  Results do not depend on the launch shape:
// every line is solved with the same arithmetic whichever CTA and group hold it.

#include <map>
#include <mutex>
#include <tuple>

#include "bfvm_internal.h"

namespace bfvm {

using tuning_key = std::tuple<int, int, int, int, int, int, int>; // device SMs, axis, dims, X, Y, Z, S

static std::mutex cache_lock;
static std::map<tuning_key, sweep_tuning> cache;

static tuning_key key_of(const bfvm_solver* s, int axis)
{
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	return tuning_key(sms, axis, s->dims, s->grid[0], s->grid[1], s->grid[2], s->S);
}

bool cached_tuning(const bfvm_solver* s, int axis, sweep_tuning& out)
{
	std::lock_guard<std::mutex> guard(cache_lock);
	if (cache.empty())
		return false;
	auto it = cache.find(key_of(s, axis));
	if (it == cache.end())
		return false;
	out = it->second;
	return true;
}

// mean time of `reps` launches of the staged sweep of `axis` with shape `t`, after one warm-up
static int time_shape(bfvm_solver* s, int axis, const sweep_tuning& t, int reps, float* ms)
{
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	BFVM_CUDA(cudaEventCreate(&e0));
	BFVM_CUDA(cudaEventCreate(&e1));
	int st = BFVM_OK;
	bool handled = false;
	for (int r = -1; r < reps && !st; r++)
	{
		if (r == 0)
			cudaEventRecord(e0, s->stream);
		st = launch_staged_sweep(s, axis, t, handled);
		if (!st && !handled)
			st = fail(BFVM_ERR_STATE, "the staged sweep declined a shape it listed");
	}
	if (!st)
	{
		cudaEventRecord(e1, s->stream);
		cudaError_t e = cudaEventSynchronize(e1);
		if (e == cudaSuccess)
			e = cudaEventElapsedTime(ms, e0, e1);
		if (e != cudaSuccess)
			st = cuda_fail(e, "sweep timing");
		*ms /= reps;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	return st;
}

} // namespace bfvm

using namespace bfvm;

extern "C" int bfvm_autotune(bfvm_solver* s, int32_t* choices)
{
	if (!s)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null solver");
	BFVM_CUDA(cudaSetDevice(s->device));
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	// the sweeps run on a scratch copy of the field
	float* scratch = nullptr;
	int st = device_alloc(&scratch, (size_t)s->V * s->S);
	if (st)
		return st;
	cudaError_t e = cudaMemcpyAsync(scratch, s->dens, (size_t)s->V * s->S * sizeof(float), cudaMemcpyDeviceToDevice,
									s->stream);
	if (e != cudaSuccess)
	{
		device_free(scratch);
		return cuda_fail(e, "cudaMemcpyAsync(scratch field)");
	}
	float* field = s->dens;
	s->dens = scratch;
	for (int axis = 0; axis < s->dims && !st; axis++)
	{
		const std::vector<sweep_tuning> shapes = staged_sweep_shapes(s, axis);
		sweep_tuning best;
		float best_ms = 0.f;
		for (const sweep_tuning& t : shapes)
		{
			float ms = 0.f;
			if ((st = time_shape(s, axis, t, 3, &ms)))
				break;
			if (best.groups == 0 || ms < best_ms)
			{
				best = t;
				best_ms = ms;
			}
		}
		if (st)
			break;
		s->tune[axis] = best; // groups 0 when the staged path does not take this axis
		if (best.groups > 0)
		{
			std::lock_guard<std::mutex> guard(cache_lock);
			cache[key_of(s, axis)] = best;
		}
		if (choices)
		{
			choices[2 * axis] = best.groups;
			choices[2 * axis + 1] = best.stages;
		}
	}
	e = cudaStreamSynchronize(s->stream);
	s->dens = field;
	device_free(scratch);
	if (!st && e != cudaSuccess)
		st = cuda_fail(e, "cudaStreamSynchronize(autotune)");
	// launch shapes changed: the step graphs are rebuilt
	for (auto& g : s->step_graph)
		if (g)
		{
			cudaGraphExecDestroy(g);
			g = nullptr;
		}
	s->graph_epoch++;
	return st;
}
