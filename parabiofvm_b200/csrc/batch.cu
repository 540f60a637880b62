// Batched ensembles: many independent microenvironments (parameter sweeps of an agent-based
// model, with uneven meshes, substrate and agent counts) stepped together on one GPU.
//
// A batch groups existing solvers.  Its step is one CUDA graph built around the ensemble kernels
// (batch_kernels.cu): one launch per phase (Dirichlet, x/y/z sweeps, gradient, secretion) covers
// every mesh those kernels take, so a step of 256 meshes is about a dozen launches, not
// thousands.  Around that chain the graph has parallel branches, on branch streams the batch owns:
// on recompute steps each mesh with agents rebuilds its voxel binning (it reads agent data only, so
// it overlaps the diffusion), and a mesh the ensemble kernels do not take (an axis of one voxel,
// lines of more than 512 voxels, more than 32 substrates) runs its own step.  As for one solver
// there is one graph for recompute steps and one for the others, rebuilt when any instance changes
// (its graph epoch advances).

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "agent_kernels.cuh"
#include "ensemble.h"

struct bfvm_batch
{
	int device = 0;
	std::vector<bfvm_solver*> inst;
	cudaStream_t stream = nullptr;
	cudaEvent_t fork = nullptr;
	std::vector<cudaEvent_t> join;		 // one per instance
	std::vector<cudaStream_t> branch;	 // capture stream of each instance
	cudaGraphExec_t graph[2] = { nullptr, nullptr }; // [recompute]
	std::vector<long long> kernels[2];	 // kernel nodes of each instance in graph[rc]
	std::vector<long long> epochs[2];	 // instance graph epochs when graph[rc] was captured
	// whether each instance's agent terms were in sorted order before graph[rc] (what it launches
	// depends on it) and are after it (the host state advances as the captured step did)
	std::vector<char> sorted_before[2], sorted_after[2];
	bfvm::ensemble_plan ens[2];			 // descriptors of the ensemble meshes captured in graph[rc]
	long long ens_kernels[2] = { 0, 0 }; // ensemble launches in graph[rc] (counted on the first mesh)
	bool holds_refs = false;			 // the instances count this batch in batch_refs
	bool tuned = false;					 // bfvm_batch_autotune chose `tune`
	bfvm::ens_tuning tune;
};

namespace bfvm {

static void batch_free_graph(bfvm_batch* b, int rc)
{
	if (b->graph[rc])
		cudaGraphExecDestroy(b->graph[rc]);
	b->graph[rc] = nullptr;
}

static bool batch_graph_current(const bfvm_batch* b, int rc)
{
	if (!b->graph[rc])
		return false;
	for (size_t i = 0; i < b->inst.size(); i++)
		if (b->epochs[rc][i] != b->inst[i]->graph_epoch || b->sorted_before[rc][i] != (b->inst[i]->ag.sorted ? 1 : 0))
			return false;
	return true;
}

// The autotuner's choices for batches of the same meshes, for the rest of the process.
static std::mutex g_tune_lock;
static std::map<std::string, ens_tuning> g_tune_cache;

static std::vector<bfvm_solver*> ensemble_members(const bfvm_batch* b)
{
	std::vector<bfvm_solver*> m;
	for (bfvm_solver* s : b->inst)
		if (ensemble_eligible(s))
			m.push_back(s);
	return m;
}

// the shapes the ensemble kernels see: per member dims, grid, substrates and blocks per line
static std::string ensemble_signature(const std::vector<bfvm_solver*>& members)
{
	std::string sig;
	for (const bfvm_solver* s : members)
	{
		sig += std::to_string(s->dims) + ":" + std::to_string(s->grid[0]) + "," + std::to_string(s->grid[1]) + ","
			   + std::to_string(s->grid[2]) + "x" + std::to_string(s->S);
		for (int d = 0; d < s->dims; d++)
			sig += "/" + std::to_string(s->plan[d].vP);
		sig += ";";
	}
	return sig;
}

static ens_tuning batch_tuning(const bfvm_batch* b, const std::vector<bfvm_solver*>& members)
{
	if (b->tuned)
		return b->tune;
	std::lock_guard<std::mutex> g(g_tune_lock);
	const auto it = g_tune_cache.find(ensemble_signature(members));
	return it == g_tune_cache.end() ? ens_tuning() : it->second;
}

static int batch_capture(bfvm_batch* b, int rc)
{
	batch_free_graph(b, rc);
	const size_t n = b->inst.size();
	b->kernels[rc].assign(n, 0);
	b->epochs[rc].assign(n, 0);
	b->sorted_before[rc].assign(n, 0);
	b->sorted_after[rc].assign(n, 0);
	for (size_t i = 0; i < n; i++)
		b->sorted_before[rc][i] = b->inst[i]->ag.sorted ? 1 : 0;
	std::vector<bfvm_solver*> members;
	std::vector<char> in_ens(n, 0);
	for (size_t i = 0; i < n; i++)
		if (ensemble_eligible(b->inst[i]))
		{
			members.push_back(b->inst[i]);
			in_ens[i] = 1;
		}
	// a recompute step rebins every ensemble mesh with agents first (in a side branch), which
	// leaves its agent terms sorted when it tracks internalized substrates
	int st = ensemble_build(b->ens[rc], members, batch_tuning(b, members), nullptr, rc == 1, true);
	if (!st)
		st = ensemble_build_dirichlet(b->ens[rc]);
	if (st)
		return st;
	const ensemble_plan& plan = b->ens[rc];

	BFVM_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
	cudaError_t e = cudaEventRecord(b->fork, b->stream);
	if (e != cudaSuccess)
		st = cuda_fail(e, "cudaEventRecord(fork)");
	// side branches: rebinning of ensemble meshes (recompute steps), whole steps of the others
	std::vector<char> branched(n, 0), binning(n, 0);
	for (size_t i = 0; i < n && !st; i++)
	{
		bfvm_solver* s = b->inst[i];
		const bool rebin = in_ens[i] && rc == 1 && s->ag.count > 0;
		if (in_ens[i] && !rebin)
			continue;
		cudaStream_t br = b->branch[i];
		if ((e = cudaStreamWaitEvent(br, b->fork, 0)) != cudaSuccess)
		{
			st = cuda_fail(e, "cudaStreamWaitEvent(fork)");
			break;
		}
		branched[i] = 1;
		binning[i] = rebin ? 1 : 0;
		cudaStream_t own = s->stream;
		s->stream = br;
		const long long before = s->launches;
		st = rebin ? prepare_agent_terms(s, true) : one_step(s, rc == 1);
		b->kernels[rc][i] = s->launches - before;
		s->launches = before;
		s->stream = own;
		if ((e = cudaEventRecord(b->join[i], br)) != cudaSuccess && !st)
			st = cuda_fail(e, "cudaEventRecord(join)");
	}
	// the ensemble chain on the batch's stream
	long long ens_launches = 0;
	auto count = [&](int r) {
		if (!r)
			ens_launches++;
		return r;
	};
	if (!st && plan.count > 0)
	{
		int maxdims = 0;
		for (bfvm_solver* m : members)
			maxdims = std::max(maxdims, m->dims);
		// the overwrites after the sweeps launch nothing when the sweeps write every condition
		auto overwrite = [&](int phase) {
			const int r = ensemble_dirichlet(plan, phase, b->stream);
			if (!r && ensemble_dirichlet_entries(plan, phase) > 0)
				ens_launches++;
			return r;
		};
		for (int axis = 0; axis < maxdims && !st; axis++)
		{
			if ((st = overwrite(axis)))
				break;
			st = count(ensemble_sweep(plan, axis, b->stream));
		}
		if (!st)
			st = overwrite(maxdims);
		if (!st)
			st = count(ensemble_gradient(plan, b->stream));
		// the secretion update waits for the rebinning branches
		for (size_t i = 0; i < n && !st; i++)
			if (binning[i] && (e = cudaStreamWaitEvent(b->stream, b->join[i], 0)) != cudaSuccess)
				st = cuda_fail(e, "join of a binning branch");
		if (!st)
			st = count(ensemble_secretion(plan, b->stream));
	}
	// join every branch (also after a failure, so the capture ends cleanly)
	for (size_t i = 0; i < n; i++)
		if (branched[i])
			cudaStreamWaitEvent(b->stream, b->join[i], 0);
	cudaGraph_t g = nullptr;
	e = cudaStreamEndCapture(b->stream, &g);
	if (!st && e != cudaSuccess)
		st = cuda_fail(e, "cudaStreamEndCapture(batch)");
	if (!st)
	{
		e = cudaGraphInstantiate(&b->graph[rc], g, 0);
		if (e != cudaSuccess)
		{
			b->graph[rc] = nullptr;
			st = cuda_fail(e, "cudaGraphInstantiate(batch)");
		}
	}
	if (g)
		cudaGraphDestroy(g);
	for (size_t i = 0; i < n; i++)
	{
		b->sorted_after[rc][i] = b->inst[i]->ag.sorted ? 1 : 0;
		b->inst[i]->ag.sorted = b->sorted_before[rc][i] != 0; // set again after every launch of the graph
	}
	if (st)
		return st;
	b->ens_kernels[rc] = ens_launches;
	for (size_t i = 0; i < n; i++)
		b->epochs[rc][i] = b->inst[i]->graph_epoch;
	return BFVM_OK;
}

// Work on the batch's stream after everything already queued on the instances' streams, and the
// other way round (calls on one solver afterwards see the batch's steps).
static int batch_wait_instances(bfvm_batch* b)
{
	for (size_t i = 0; i < b->inst.size(); i++)
	{
		int st;
		if ((st = order_after_copies(b->inst[i]))) // an instance's pending agent copies come first
			return st;
		BFVM_CUDA(cudaEventRecord(b->join[i], b->inst[i]->stream));
		BFVM_CUDA(cudaStreamWaitEvent(b->stream, b->join[i], 0));
	}
	return BFVM_OK;
}

static int instances_wait_batch(bfvm_batch* b)
{
	BFVM_CUDA(cudaEventRecord(b->fork, b->stream));
	for (bfvm_solver* s : b->inst)
		BFVM_CUDA(cudaStreamWaitEvent(s->stream, b->fork, 0));
	return BFVM_OK;
}

} // namespace bfvm

using namespace bfvm;

extern "C" {

int bfvm_batch_create(bfvm_batch** out, int32_t count, bfvm_solver* const* solvers)
{
	if (!out)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null output pointer");
	*out = nullptr;
	if (count <= 0 || !solvers)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "a batch needs at least one solver");
	for (int32_t i = 0; i < count; i++)
	{
		if (!solvers[i])
			return fail(BFVM_ERR_INVALID_ARGUMENT, "null solver in the batch");
		if (solvers[i]->device != solvers[0]->device)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "the solvers of a batch must share one device");
		if (solvers[i]->slab_count > 1)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "a slab of a split mesh steps through bfvm_slab_*, not in a batch");
		for (int32_t k = 0; k < i; k++)
			if (solvers[k] == solvers[i])
				return fail(BFVM_ERR_INVALID_ARGUMENT, "a solver appears twice in the batch");
	}
	auto* b = new (std::nothrow) bfvm_batch();
	if (!b)
		return fail(BFVM_ERR_OUT_OF_MEMORY, "host allocation failed");
	b->device = solvers[0]->device;
	b->inst.assign(solvers, solvers + count);
	b->join.assign(count, nullptr);
	b->branch.assign(count, nullptr);
	int st = BFVM_OK;
	cudaError_t e = cudaSetDevice(b->device);
	if (e == cudaSuccess)
		e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
	if (e == cudaSuccess)
		e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
	for (int32_t i = 0; i < count && e == cudaSuccess; i++)
	{
		e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
		if (e == cudaSuccess)
			e = cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking);
	}
	if (e != cudaSuccess)
		st = cuda_fail(e, "batch stream and events");
	// the instances' own step graphs are dropped (what they capture depends on batch_refs)
	for (int32_t i = 0; i < count && !st; i++)
		st = solver_drop_graphs(b->inst[i]);
	if (!st)
	{
		for (bfvm_solver* s : b->inst)
			s->batch_refs++;
		b->holds_refs = true;
	}
	if (st)
	{
		bfvm_batch_destroy(b);
		return st;
	}
	*out = b;
	return BFVM_OK;
}

int bfvm_batch_destroy(bfvm_batch* b)
{
	if (!b)
		return BFVM_OK;
	cudaSetDevice(b->device);
	if (b->stream)
		cudaStreamSynchronize(b->stream);
	batch_free_graph(b, 0);
	batch_free_graph(b, 1);
	if (b->holds_refs)
		for (bfvm_solver* s : b->inst)
		{
			s->batch_refs--;
			solver_drop_graphs(s); // what its own step graphs capture depends on batch_refs
		}
	ensemble_free(b->ens[0]);
	ensemble_free(b->ens[1]);
	for (cudaEvent_t ev : b->join)
		if (ev)
			cudaEventDestroy(ev);
	for (cudaStream_t st : b->branch)
		if (st)
			cudaStreamDestroy(st);
	if (b->fork)
		cudaEventDestroy(b->fork);
	if (b->stream)
		cudaStreamDestroy(b->stream);
	delete b;
	return BFVM_OK;
}

int bfvm_batch_run_steps(bfvm_batch* b, int32_t steps, int32_t first_step)
{
	if (!b)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null batch");
	if (steps < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "steps must not be negative");
	BFVM_CUDA(cudaSetDevice(b->device));
	int st;
	if ((st = batch_wait_instances(b)))
		return st;
	for (int32_t i = 0; i < steps; i++)
	{
		const int rc = ((first_step + i) % 10 == 0) ? 1 : 0;
		bool eager = false;
		for (bfvm_solver* s : b->inst)
			eager = eager || (!rc && s->ag.count > 0 && !s->ag.binned);
		if (eager)
		{
			// an instance whose agents were never binned rebins on its own stream this once
			if ((st = instances_wait_batch(b)))
				return st;
			for (bfvm_solver* s : b->inst)
				if ((st = one_step(s, false)))
					return st;
			if ((st = batch_wait_instances(b)))
				return st;
			continue;
		}
		if (rc)
		{
			// a recompute graph writes sorted agent terms back to agent order before it rebins, so
			// what it launches depends on the order it finds.  Instances with internalized
			// substrates whose terms are not sorted yet (agents never binned) are binned and sorted
			// on their own streams first, so this graph finds the order every later recompute step
			// finds and is captured once.
			bool sort_first = false;
			for (bfvm_solver* s : b->inst)
				sort_first = sort_first || (s->ag.count > 0 && s->internalized && !s->ag.sorted);
			if (sort_first)
			{
				if ((st = instances_wait_batch(b)))
					return st;
				for (bfvm_solver* s : b->inst)
					if (s->ag.count > 0 && s->internalized && !s->ag.sorted && (st = prepare_agent_terms(s, false)))
						return st;
				if ((st = batch_wait_instances(b)))
					return st;
			}
		}
		if (!batch_graph_current(b, rc) && (st = batch_capture(b, rc)))
			return st;
		BFVM_CUDA(cudaGraphLaunch(b->graph[rc], b->stream));
		for (size_t k = 0; k < b->inst.size(); k++)
		{
			bfvm_solver* s = b->inst[k];
			s->launches += b->kernels[rc][k];
			if (s->ag.count > 0)
			{
				s->ag.binned = true;
				s->ag.sorted = b->sorted_after[rc][k] != 0;
			}
		}
		b->inst[0]->launches += b->ens_kernels[rc];
	}
	return instances_wait_batch(b);
}

// Time each launch choice of the ensemble kernels on scratch copies of the members' fields and
// gradients (so the instances' state is untouched), phase by phase, and keep the fastest.
int bfvm_batch_autotune(bfvm_batch* b, int32_t* choices)
{
	if (!b)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null batch");
	BFVM_CUDA(cudaSetDevice(b->device));
	const std::vector<bfvm_solver*> members = ensemble_members(b);
	ens_tuning best;
	int st = BFVM_OK;
	if (!members.empty())
	{
		if ((st = batch_wait_instances(b)))
			return st;
		// one scratch block: each member's field then its gradient
		std::vector<std::pair<float*, float*>> bufs(members.size());
		size_t total = 0;
		for (const bfvm_solver* s : members)
			total += (size_t)s->V * s->S * (1 + s->dims);
		float* scratch = nullptr;
		if ((st = device_alloc(&scratch, total)))
			return st;
		size_t at = 0;
		for (size_t i = 0; i < members.size() && !st; i++)
		{
			const bfvm_solver* s = members[i];
			const size_t vs = (size_t)s->V * s->S;
			bufs[i] = { scratch + at, scratch + at + vs };
			at += vs * (1 + s->dims);
			const cudaError_t e = cudaMemcpyAsync(bufs[i].first, s->dens, vs * sizeof(float), cudaMemcpyDeviceToDevice,
												  b->stream);
			if (e != cudaSuccess)
				st = cuda_fail(e, "cudaMemcpyAsync(autotune scratch)");
		}
		cudaEvent_t e0 = nullptr, e1 = nullptr;
		if (!st && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
			st = cuda_fail(cudaGetLastError(), "cudaEventCreate");
		ensemble_plan plan;
		// device time of `phase` under tuning t: one launch to warm up, the mean of three
		auto time_phase = [&](const ens_tuning& t, auto phase, float& ms) -> int {
			int r = ensemble_build(plan, members, t, &bufs, false, true);
			if (!r)
				r = phase(plan);
			for (int k = 0; k < 3 && !r; k++)
			{
				if (k == 0)
					BFVM_CUDA(cudaEventRecord(e0, b->stream));
				r = phase(plan);
			}
			if (r)
				return r;
			BFVM_CUDA(cudaEventRecord(e1, b->stream));
			BFVM_CUDA(cudaEventSynchronize(e1));
			BFVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
			return BFVM_OK;
		};
		int maxdims = 0;
		for (const bfvm_solver* s : members)
			maxdims = std::max(maxdims, s->dims);
		for (int axis = 0; axis < maxdims && !st; axis++)
		{
			float best_ms = 0.f;
			ens_tuning keep = best;
			bool first = true;
			static constexpr int sweep_choices[6][2] = { { 2, 1 }, { 2, 2 }, { 2, 4 }, { 1, 1 }, { 1, 2 }, { 1, 4 } };
			for (int c = 0; c < 6 && !st; c++)
			{
				ens_tuning t = best;
				t.sweep_minb[axis] = sweep_choices[c][0];
				t.sweep_split[axis] = sweep_choices[c][1];
				float ms = 0.f;
				st = time_phase(t, [&](const ensemble_plan& p) { return ensemble_sweep(p, axis, b->stream); }, ms);
				if (!st && (first || ms < best_ms))
				{
					best_ms = ms;
					keep = t;
					first = false;
				}
			}
			best = keep;
		}
		if (!st)
		{
			float best_ms = 0.f;
			ens_tuning keep = best;
			bool first = true;
			static constexpr int grad_choices[6][2] = { { 64, 8 }, { 64, 4 }, { 32, 8 }, { 32, 4 }, { 128, 8 }, { 128, 4 } };
			for (int c = 0; c < 6 && !st; c++)
			{
				ens_tuning t = best;
				t.grad_zc = grad_choices[c][0];
				t.grad_zu = grad_choices[c][1];
				float ms = 0.f;
				st = time_phase(t, [&](const ensemble_plan& p) { return ensemble_gradient(p, b->stream); }, ms);
				if (!st && (first || ms < best_ms))
				{
					best_ms = ms;
					keep = t;
					first = false;
				}
			}
			best = keep;
		}
		cudaStreamSynchronize(b->stream);
		ensemble_free(plan);
		if (e0)
			cudaEventDestroy(e0);
		if (e1)
			cudaEventDestroy(e1);
		device_free(scratch);
		if (st)
			return st;
		std::lock_guard<std::mutex> g(g_tune_lock);
		g_tune_cache[ensemble_signature(members)] = best;
	}
	b->tune = best;
	b->tuned = true;
	batch_free_graph(b, 0);
	batch_free_graph(b, 1);
	if (choices)
	{
		for (int d = 0; d < 3; d++)
		{
			choices[d] = best.sweep_minb[d];
			choices[3 + d] = best.sweep_split[d];
		}
		choices[6] = best.grad_zc;
		choices[7] = best.grad_zu;
	}
	return BFVM_OK;
}

int bfvm_batch_synchronize(bfvm_batch* b)
{
	if (!b)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null batch");
	BFVM_CUDA(cudaSetDevice(b->device));
	BFVM_CUDA(cudaStreamSynchronize(b->stream));
	int first = BFVM_OK;
	for (bfvm_solver* s : b->inst)
	{
		const int st = check_device_errors(s);
		if (st && !first)
			first = st;
	}
	return first;
}

} // extern "C"
