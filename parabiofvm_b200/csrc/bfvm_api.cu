// C ABI entry points (include/bfvm.h): solver lifecycle, data movement, solver calls, step graphs.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "bfvm_internal.h"
#include "ensemble.h"

namespace bfvm {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg)
{
	g_last_error = msg;
	return status;
}

int cuda_fail(cudaError_t e, const char* what)
{
	(void)cudaGetLastError();
	return fail(BFVM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Sweep block capacity for a line of n elements: 32 registers per block while that keeps the
// blocks of a line within one CTA (n <= 1024), 64 up to n = 2048.
static int pick_block_capacity(int n) { return n <= 1024 ? 32 : 64; }

static int upload_plan(bfvm_solver* s, int axis)
{
	sweep_plan& p = s->plan[axis];
	const int n = s->grid[axis];
	std::vector<float> bp, ep, g, G, c, gq, Gp;
	p.n = n;
	p.M = pick_block_capacity(n);
	precompute_axis(n, s->voxel[axis], s->dims, s->S, s->dt, s->D.data(), s->decay.data(), p.M, bp, ep, g, G, c, gq,
					Gp, p.P, p.base_len, p.extra);
	int st;
	const size_t nS = (size_t)n * s->S;
	if ((st = device_alloc(&p.bp, nS)) || (st = device_alloc(&p.c, (size_t)s->S))
		|| (st = device_alloc(&p.gq, gq.size())) || (st = device_alloc(&p.Gp, Gp.size())))
		return st;
	BFVM_CUDA(cudaMemcpy(p.gq, gq.data(), gq.size() * sizeof(float), cudaMemcpyHostToDevice));
	BFVM_CUDA(cudaMemcpy(p.Gp, Gp.data(), Gp.size() * sizeof(float), cudaMemcpyHostToDevice));
	BFVM_CUDA(cudaMemcpy(p.bp, bp.data(), nS * sizeof(float), cudaMemcpyHostToDevice));
	BFVM_CUDA(cudaMemcpy(p.c, c.data(), (size_t)s->S * sizeof(float), cudaMemcpyHostToDevice));
	if (n >= 2)
	{
		std::vector<float> vt;
		if (axis == 2 && s->slab_global_z > 0)
		{
			// a z-slab: the whole line's b', restricted to the slab's planes
			std::vector<float> wbp, wep, wg, wG, wc, wgq, wGp;
			int wP, wbl, wex;
			precompute_axis(s->slab_global_z, s->voxel[2], s->dims, s->S, s->dt, s->D.data(), s->decay.data(), 32, wbp,
							wep, wg, wG, wc, wgq, wGp, wP, wbl, wex);
			precompute_padded_range(s->slab_global_z, s->slab_z0, s->slab_z0 + n, s->S, wbp, wc, p.vP, p.pad, vt);
		}
		else
			precompute_padded(n, s->S, bp, c, p.vP, p.pad, vt);
		if ((st = device_alloc(&p.vtab, vt.size())))
			return st;
		BFVM_CUDA(cudaMemcpy(p.vtab, vt.data(), vt.size() * sizeof(float), cudaMemcpyHostToDevice));
		if (s->slab_global_z == 0 && (st = build_chunks(s, axis, bp, c)))
			return st;
	}
	return BFVM_OK;
}

static void free_plan(sweep_plan& p)
{
	device_free(p.bp);
	device_free(p.c);
	device_free(p.gq);
	device_free(p.Gp);
	device_free(p.vtab);
	free_chunks(p);
}

static void free_graphs(bfvm_solver* s)
{
	for (auto& g : s->step_graph)
		if (g)
		{
			cudaGraphExecDestroy(g);
			g = nullptr;
		}
	s->graphs_dirty = true;
	s->graph_epoch++; // graphs that captured this solver's buffers (its own, a batch's) are stale
}

int solver_drop_graphs(bfvm_solver* s)
{
	BFVM_CUDA(cudaSetDevice(s->device));
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	free_graphs(s);
	return BFVM_OK;
}

static void destroy_all(bfvm_solver* s)
{
	if (s->device >= 0)
		cudaSetDevice(s->device);
	free_graphs(s);
	for (auto& p : s->plan)
		free_plan(p);
	cell_free(s);
	free_dirichlet(s);
	device_free(s->grad_tile_done);
	device_free(s->grad_deferred);
	s->grad_tiles = 0;
	free_bulk(s);
	if (s->self_plan)
	{
		ensemble_free(*s->self_plan);
		delete s->self_plan;
		s->self_plan = nullptr;
	}
	device_free(s->dens);
	device_free(s->grad);
	device_free(s->slab_coef);
	device_free(s->slab_carry);
	device_free(s->slab_rw);
	device_free(s->dev_error);
	if (s->copy_stream)
	{
		cudaStreamSynchronize(s->copy_stream);
		cudaStreamDestroy(s->copy_stream);
		cudaEventDestroy(s->copy_ready);
		cudaEventDestroy(s->copy_done);
	}
	if (s->host_error)
		cudaFreeHost(s->host_error);
	if (s->own_stream)
		cudaStreamDestroy(s->own_stream);
}

// error flags raised by kernels since the last check
int check_device_errors(bfvm_solver* s)
{
	BFVM_CUDA(cudaMemcpyAsync(s->host_error, s->dev_error, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	const int e = *s->host_error;
	if (e)
	{
		BFVM_CUDA(cudaMemsetAsync(s->dev_error, 0, sizeof(int), s->stream));
		if (e & DEVERR_TIMEOUT)
			return fail(BFVM_ERR_TIMEOUT, "a sweep kernel timed out waiting for a tile copy; the field is not valid");
		if (e & DEVERR_AGENT_OUTSIDE)
			return fail(BFVM_ERR_AGENT_OUTSIDE, "an agent position lies outside the mesh; it was left out of "
												"secretion/uptake");
	}
	return BFVM_OK;
}

static int diffusion(bfvm_solver* s) { return launch_diffusion(s); }

int order_after_copies(bfvm_solver* s)
{
	if (!s->copy_pending)
		return BFVM_OK;
	BFVM_CUDA(cudaStreamWaitEvent(s->stream, s->copy_done, 0));
	s->copy_pending = false;
	return BFVM_OK;
}

static int ensure_copy_stream(bfvm_solver* s)
{
	if (!s->copy_stream)
	{
		BFVM_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
		BFVM_CUDA(cudaEventCreateWithFlags(&s->copy_ready, cudaEventDisableTiming));
		BFVM_CUDA(cudaEventCreateWithFlags(&s->copy_done, cudaEventDisableTiming));
	}
	return BFVM_OK;
}

// the copy stream starts after everything queued on the solver's stream so far
static int begin_async_copy(bfvm_solver* s)
{
	int st;
	if ((st = ensure_copy_stream(s)))
		return st;
	BFVM_CUDA(cudaEventRecord(s->copy_ready, s->stream));
	BFVM_CUDA(cudaStreamWaitEvent(s->copy_stream, s->copy_ready, 0));
	return BFVM_OK;
}

static int end_async_copy(bfvm_solver* s)
{
	BFVM_CUDA(cudaEventRecord(s->copy_done, s->copy_stream));
	s->copy_pending = true;
	return BFVM_OK;
}

// diffusion, gradient (inside the z sweep where it can be), secretion.  Only secretion touches
// agent data, so the wait for the asynchronous agent copies (the copy stream's last event; inside
// a capture, an external event node that waits for the copies issued before each launch of the
// graph) comes right before it, and the diffusion overlaps the copies.
int one_step(bfvm_solver* s, bool recompute)
{
	int st;
	bool gradient_done = false;
	if ((st = launch_diffusion(s, true, &gradient_done)))
		return st;
	if (!gradient_done && (st = launch_gradient(s)))
		return st;
	if (s->copy_stream && s->ag.count > 0)
	{
		cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
		BFVM_CUDA(cudaStreamIsCapturing(s->stream, &cs));
		BFVM_CUDA(cudaStreamWaitEvent(s->stream, s->copy_done,
									  cs == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0));
	}
	return launch_secretion(s, recompute);
}

} // namespace bfvm

using namespace bfvm;

#define CHECK_SOLVER(s)                                                                                                \
	do                                                                                                                 \
	{                                                                                                                  \
		if (!(s))                                                                                                      \
			return fail(BFVM_ERR_INVALID_ARGUMENT, "null solver");                                                     \
		if (cudaSetDevice((s)->device) != cudaSuccess)                                                                 \
			return cuda_fail(cudaGetLastError(), "cudaSetDevice");                                                     \
	} while (0)

// the slab a solver created by bfvm_create_slab holds
struct slab_spec
{
	int count = 1, index = 0;
	std::vector<int> bounds; // [count + 1] plane boundaries of the mesh
};

// multi-slab solvers step through bfvm_slab_*; the whole-mesh calls that cross z refuse them
#define REFUSE_SLABS(s, what)                                                                                          \
	do                                                                                                                 \
	{                                                                                                                  \
		if ((s)->slab_count > 1)                                                                                       \
			return fail(BFVM_ERR_STATE, std::string(what) + " couples the slabs of a mesh: use bfvm_slab_*");         \
	} while (0)

static int create_solver(bfvm_solver** out, int device, int dims, const int32_t bounding_box_mins[3],
						 const int32_t bounding_box_maxs[3], const int32_t voxel_shape[3], int32_t substrates,
						 float time_step, const float* diffusion_coefficients, const float* decay_rates,
						 int compute_internalized_substrates, const slab_spec* slab);

extern "C" {

const char* bfvm_last_error(void) { return g_last_error.c_str(); }

const char* bfvm_status_string(int status)
{
	switch (status)
	{
	case BFVM_OK: return "ok";
	case BFVM_ERR_INVALID_ARGUMENT: return "invalid argument";
	case BFVM_ERR_OUT_OF_MEMORY: return "out of memory";
	case BFVM_ERR_CUDA: return "CUDA error";
	case BFVM_ERR_NO_DEVICE: return "no usable CUDA device";
	case BFVM_ERR_STATE: return "invalid state";
	case BFVM_ERR_AGENT_OUTSIDE: return "agent outside the mesh";
	case BFVM_ERR_TIMEOUT: return "device wait timed out";
	default: return "unknown status";
	}
}

int bfvm_version(void) { return 10000; }

int bfvm_create(bfvm_solver** out, int device, int dims, const int32_t bounding_box_mins[3],
				const int32_t bounding_box_maxs[3], const int32_t voxel_shape[3], int32_t substrates, float time_step,
				const float* diffusion_coefficients, const float* decay_rates, int compute_internalized_substrates)
{
	return create_solver(out, device, dims, bounding_box_mins, bounding_box_maxs, voxel_shape, substrates, time_step,
						 diffusion_coefficients, decay_rates, compute_internalized_substrates, nullptr);
}

int bfvm_create_slab(bfvm_solver** out, int device, const int32_t bounding_box_mins[3],
					 const int32_t bounding_box_maxs[3], const int32_t voxel_shape[3], int32_t substrates,
					 float time_step, const float* diffusion_coefficients, const float* decay_rates,
					 int compute_internalized_substrates, int32_t slab_count, const int32_t* slab_planes, int32_t slab)
{
	g_last_error.clear();
	if (!out)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "out is null");
	*out = nullptr;
	if (!bounding_box_mins || !bounding_box_maxs || !voxel_shape || !slab_planes)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "mesh and slab arrays must not be null");
	if (voxel_shape[2] <= 0 || bounding_box_maxs[2] <= bounding_box_mins[2])
		return fail(BFVM_ERR_INVALID_ARGUMENT, "the mesh needs a positive z extent");
	const int Z = (bounding_box_maxs[2] - bounding_box_mins[2] + voxel_shape[2] - 1) / voxel_shape[2];
	if (slab_count < 1 || slab_count > 64)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "slab_count must be 1..64");
	if (slab < 0 || slab >= slab_count)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "slab index out of range");
	if (slab_planes[0] != 0 || slab_planes[slab_count] != Z)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "slab_planes must run from 0 to the mesh's " + std::to_string(Z)
												   + " z planes");
	for (int k = 0; k < slab_count; k++)
		if (slab_planes[k + 1] - slab_planes[k] < 2)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "every slab needs at least 2 planes");
	const int z0 = slab_planes[slab], z1 = slab_planes[slab + 1];
	if (slab_count > 1 && z1 - z0 > 512)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "a slab holds at most 512 planes");
	slab_spec spec;
	spec.count = slab_count;
	spec.index = slab;
	spec.bounds.assign(slab_planes, slab_planes + slab_count + 1);
	int32_t mins[3] = { bounding_box_mins[0], bounding_box_mins[1], bounding_box_mins[2] + z0 * voxel_shape[2] };
	int32_t maxs[3] = { bounding_box_maxs[0], bounding_box_maxs[1],
						z1 == Z ? bounding_box_maxs[2] : bounding_box_mins[2] + z1 * voxel_shape[2] };
	return create_solver(out, device, 3, mins, maxs, voxel_shape, substrates, time_step, diffusion_coefficients,
						 decay_rates, compute_internalized_substrates, &spec);
}

} // extern "C"

static int create_solver(bfvm_solver** out, int device, int dims, const int32_t bounding_box_mins[3],
						 const int32_t bounding_box_maxs[3], const int32_t voxel_shape[3], int32_t substrates,
						 float time_step, const float* diffusion_coefficients, const float* decay_rates,
						 int compute_internalized_substrates, const slab_spec* slab)
{
	g_last_error.clear();
	if (!out)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "out is null");
	*out = nullptr;
	if (dims < 1 || dims > 3)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "dims must be 1, 2 or 3");
	if (!bounding_box_mins || !bounding_box_maxs || !voxel_shape)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "mesh arrays must not be null");
	if (substrates < 1)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "at least one substrate is required");
	if (!diffusion_coefficients || !decay_rates)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "diffusion coefficients and decay rates are required");
	int grid[3] = { 1, 1, 1 };
	for (int d = 0; d < dims; d++)
	{
		if (voxel_shape[d] <= 0)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "voxel_shape must be positive along every used axis");
		if (bounding_box_maxs[d] <= bounding_box_mins[d])
			return fail(BFVM_ERR_INVALID_ARGUMENT, "bounding box max must exceed min along every used axis");
		grid[d] = (bounding_box_maxs[d] - bounding_box_mins[d] + voxel_shape[d] - 1) / voxel_shape[d];
		if (grid[d] > 2048)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "a mesh axis longer than 2048 voxels is not supported");
	}
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
	{
		(void)cudaGetLastError();
		return fail(BFVM_ERR_NO_DEVICE, "no CUDA device is available");
	}
	if (device < 0 || device >= ndev)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "device index out of range");

	auto* s = new (std::nothrow) bfvm_solver();
	if (!s)
		return fail(BFVM_ERR_OUT_OF_MEMORY, "host allocation failed");
	s->device = device;
	s->dims = dims;
	for (int d = 0; d < 3; d++)
	{
		s->bbox_min[d] = bounding_box_mins[d];
		s->bbox_max[d] = bounding_box_maxs[d];
		s->voxel[d] = voxel_shape[d];
		s->grid[d] = grid[d];
	}
	s->S = substrates;
	s->dt = time_step;
	s->D.assign(diffusion_coefficients, diffusion_coefficients + substrates);
	s->decay.assign(decay_rates, decay_rates + substrates);
	s->internalized = compute_internalized_substrates != 0;
	s->V = (long long)grid[0] * grid[1] * grid[2];
	s->face_vals_h.assign(6 * (size_t)substrates, 0.f);
	s->face_conds_h.assign(6 * (size_t)substrates, 0);
	if (slab)
	{
		s->slab_count = slab->count;
		s->slab_index = slab->index;
		s->slab_z0 = slab->bounds[slab->index];
		s->slab_global_z = slab->bounds[slab->count];
	}

	int st = BFVM_OK;
	do
	{
		if (cudaSetDevice(device) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "cudaSetDevice");
			break;
		}
		cudaDeviceProp prop;
		if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "cudaGetDeviceProperties");
			break;
		}
		if (prop.major != 10)
		{
			st = fail(BFVM_ERR_NO_DEVICE, std::string("this library is built for sm_100a; device is ") + prop.name);
			break;
		}
		if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "cudaStreamCreate");
			break;
		}
		s->stream = s->own_stream;
		if ((st = device_alloc(&s->dens, (size_t)s->V * s->S)) || (st = device_alloc(&s->grad, (size_t)s->V * s->S * dims))
			|| (st = device_alloc(&s->dev_error, 1)))
			break;
		if (cudaMallocHost((void**)&s->host_error, sizeof(int)) != cudaSuccess)
		{
			(void)cudaGetLastError();
			st = fail(BFVM_ERR_OUT_OF_MEMORY, "pinned host allocation failed");
			break;
		}
		*s->host_error = 0;
		if (cudaMemset(s->dens, 0, (size_t)s->V * s->S * sizeof(float)) != cudaSuccess
			|| cudaMemset(s->grad, 0, (size_t)s->V * s->S * dims * sizeof(float)) != cudaSuccess
			|| cudaMemset(s->dev_error, 0, sizeof(int)) != cudaSuccess)
		{
			st = cuda_fail(cudaGetLastError(), "cudaMemset");
			break;
		}
		for (int d = 0; d < dims && !st; d++)
			st = upload_plan(s, d);
		if (st)
			break;
		if (slab)
		{
			if (slab->count > 1 && (long long)grid[0] * substrates % 4 != 0)
			{
				st = fail(BFVM_ERR_INVALID_ARGUMENT, "slabs need X * substrates to be a multiple of 4");
				break;
			}
			std::vector<float> bp, ep, g, G, c, gq, Gp, coef;
			int P, bl, ex;
			precompute_axis(s->slab_global_z, s->voxel[2], 3, s->S, s->dt, s->D.data(), s->decay.data(), 32, bp, ep, g,
							G, c, gq, Gp, P, bl, ex);
			slab_coefficients(s->slab_global_z, s->S, bp, c, slab->count, slab->bounds.data(), coef);
			std::vector<float> rw;
			int a_first;
			slab_reduce_weights(s->slab_global_z, s->slab_z0, s->slab_z0 + grid[2], s->S, bp, c, rw, a_first, s->slab_na,
								s->slab_nb);
			s->slab_a0 = a_first - s->slab_z0;
			const size_t lines = (size_t)grid[0] * grid[1] * substrates;
			if ((st = device_alloc(&s->slab_coef, coef.size())) || (st = device_alloc(&s->slab_carry, 2 * lines))
				|| (st = device_alloc(&s->slab_rw, std::max<size_t>(rw.size(), 4))))
				break;
			if (cudaMemcpy(s->slab_coef, coef.data(), coef.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess
				|| (!rw.empty()
					&& cudaMemcpy(s->slab_rw, rw.data(), rw.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess))
			{
				st = cuda_fail(cudaGetLastError(), "cudaMemcpy");
				break;
			}
		}
		s->self_plan = new (std::nothrow) ensemble_plan();
		if (!s->self_plan)
		{
			st = fail(BFVM_ERR_OUT_OF_MEMORY, "host allocation failed");
			break;
		}
		st = ensemble_build(*s->self_plan, { s });
	} while (0);

	if (st)
	{
		destroy_all(s);
		delete s;
		return st;
	}
	*out = s;
	return BFVM_OK;
}

extern "C" {

int bfvm_destroy(bfvm_solver* s)
{
	if (!s)
		return BFVM_OK;
	destroy_all(s);
	delete s;
	return BFVM_OK;
}

int bfvm_get_shape(const bfvm_solver* s, int32_t grid_shape[3], int64_t* voxel_count, int32_t* substrates, int32_t* dims)
{
	if (!s)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null solver");
	if (grid_shape)
		for (int d = 0; d < 3; d++)
			grid_shape[d] = s->grid[d];
	if (voxel_count)
		*voxel_count = s->V;
	if (substrates)
		*substrates = s->S;
	if (dims)
		*dims = s->dims;
	return BFVM_OK;
}

int bfvm_set_stream(bfvm_solver* s, void* stream)
{
	CHECK_SOLVER(s);
	cudaStream_t ns = stream ? (cudaStream_t)stream : s->own_stream;
	if (ns != s->stream)
	{
		BFVM_CUDA(cudaStreamSynchronize(s->stream));
		s->stream = ns;
		free_graphs(s);
	}
	return BFVM_OK;
}

int bfvm_set_boundary_dirichlet(bfvm_solver* s, int dim, int is_max, const float* values, const uint8_t* conditions)
{
	CHECK_SOLVER(s);
	if (dim < 0 || dim >= s->dims)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "dim must be in [0, dims)");
	const int face = 2 * dim + (is_max ? 1 : 0);
	if (!values)
	{
		s->face_mask &= ~(1 << face);
		for (int k = 0; k < s->S; k++)
		{
			s->face_vals_h[(size_t)face * s->S + k] = 0.f;
			s->face_conds_h[(size_t)face * s->S + k] = 0;
		}
	}
	else
	{
		if (!conditions)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "conditions must accompany values");
		s->face_mask |= 1 << face;
		for (int k = 0; k < s->S; k++)
		{
			s->face_vals_h[(size_t)face * s->S + k] = values[k];
			s->face_conds_h[(size_t)face * s->S + k] = conditions[k] ? 1 : 0;
		}
	}
	// the step graphs and kernels in flight use the current overwrite list
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	free_graphs(s);
	return rebuild_dirichlet(s);
}

int bfvm_set_interior_dirichlet(bfvm_solver* s, int32_t count, const int32_t* voxels, const float* values,
								const uint8_t* conditions)
{
	CHECK_SOLVER(s);
	if (count < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "count must not be negative");
	if (count > 0 && (!voxels || !values || !conditions))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "voxels, values and conditions are required");
	const int S = s->S;
	// merge duplicates in list order: a later listed condition overwrites an earlier one
	std::map<long long, int> row_of;
	std::vector<float> vals;
	std::vector<unsigned char> conds;
	for (int i = 0; i < count; i++)
	{
		int c[3] = { 0, 0, 0 };
		for (int d = 0; d < s->dims; d++)
		{
			c[d] = voxels[(size_t)i * s->dims + d];
			if (c[d] < 0 || c[d] >= s->grid[d])
				return fail(BFVM_ERR_INVALID_ARGUMENT, "interior Dirichlet voxel " + std::to_string(i) + " is outside the mesh");
		}
		const long long v = c[0] + (long long)s->grid[0] * (c[1] + (long long)s->grid[1] * c[2]);
		auto it = row_of.find(v);
		int row;
		if (it == row_of.end())
		{
			row = (int)row_of.size();
			row_of.emplace(v, row);
			vals.resize((size_t)(row + 1) * S, 0.f);
			conds.resize((size_t)(row + 1) * S, 0);
		}
		else
			row = it->second;
		for (int k = 0; k < S; k++)
			if (conditions[(size_t)i * S + k])
			{
				vals[(size_t)row * S + k] = values[(size_t)i * S + k];
				conds[(size_t)row * S + k] = 1;
			}
	}
	// rows in voxel order
	s->int_vids_h.clear();
	s->int_vals_h.assign(row_of.size() * (size_t)S, 0.f);
	s->int_conds_h.assign(row_of.size() * (size_t)S, 0);
	size_t r = 0;
	for (auto& kv : row_of)
	{
		s->int_vids_h.push_back(kv.first);
		std::memcpy(&s->int_vals_h[r * S], &vals[(size_t)kv.second * S], S * sizeof(float));
		std::memcpy(&s->int_conds_h[r * S], &conds[(size_t)kv.second * S], S);
		r++;
	}
	// the step graphs and kernels in flight use the current overwrite list
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	free_graphs(s);
	return rebuild_dirichlet(s);
}

int bfvm_store_densities(bfvm_solver* s, const float* host)
{
	CHECK_SOLVER(s);
	if (!host)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null host buffer");
	BFVM_CUDA(cudaMemcpyAsync(s->dens, host, (size_t)s->V * s->S * sizeof(float), cudaMemcpyHostToDevice, s->stream));
	return BFVM_OK;
}

int bfvm_load_densities(bfvm_solver* s, float* host)
{
	CHECK_SOLVER(s);
	if (!host)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null host buffer");
	BFVM_CUDA(cudaMemcpyAsync(host, s->dens, (size_t)s->V * s->S * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
	return check_device_errors(s);
}

int bfvm_store_densities_device(bfvm_solver* s, const float* device_densities)
{
	CHECK_SOLVER(s);
	if (!device_densities)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null device buffer");
	BFVM_CUDA(cudaMemcpyAsync(s->dens, device_densities, (size_t)s->V * s->S * sizeof(float), cudaMemcpyDeviceToDevice,
							  s->stream));
	return BFVM_OK;
}

int bfvm_load_densities_device(bfvm_solver* s, float* device_densities)
{
	CHECK_SOLVER(s);
	if (!device_densities)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null device buffer");
	BFVM_CUDA(cudaMemcpyAsync(device_densities, s->dens, (size_t)s->V * s->S * sizeof(float), cudaMemcpyDeviceToDevice,
							  s->stream));
	return BFVM_OK;
}

int bfvm_load_gradients(bfvm_solver* s, float* host)
{
	CHECK_SOLVER(s);
	if (!host)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null host buffer");
	BFVM_CUDA(cudaMemcpyAsync(host, s->grad, (size_t)s->V * s->S * s->dims * sizeof(float), cudaMemcpyDeviceToHost,
							  s->stream));
	return check_device_errors(s);
}

int bfvm_store_agents(bfvm_solver* s, int32_t count, const float* secretion_rates, const float* saturation_densities,
					  const float* uptake_rates, const float* net_export_rates, const float* internalized_substrates,
					  const float* fraction_released_at_death, const float* volumes, const float* positions)
{
	CHECK_SOLVER(s);
	if (count < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "count must not be negative");
	if (count > 0
		&& (!secretion_rates || !saturation_densities || !uptake_rates || !net_export_rates || !internalized_substrates
			|| !volumes || !positions))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent arrays must not be null");
	int rc;
	if ((rc = order_after_copies(s)))
		return rc;
	const bool resized = count != s->ag.count;
	if (resized || count > s->ag.capacity)
	{
		BFVM_CUDA(cudaStreamSynchronize(s->stream));
		free_graphs(s);
	}
	int st;
	if (count == 0)
	{
		s->ag.count = 0;
		s->ag.binned = false;
		return BFVM_OK;
	}
	if ((st = cell_alloc(s, count)))
		return st;
	agent_state& a = s->ag;
	const size_t AS = (size_t)count * s->S * sizeof(float);
	BFVM_CUDA(cudaMemcpyAsync(a.sec, secretion_rates, AS, cudaMemcpyHostToDevice, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.sat, saturation_densities, AS, cudaMemcpyHostToDevice, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.upt, uptake_rates, AS, cudaMemcpyHostToDevice, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.nex, net_export_rates, AS, cudaMemcpyHostToDevice, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.intern, internalized_substrates, AS, cudaMemcpyHostToDevice, s->stream));
	if (fraction_released_at_death)
		BFVM_CUDA(cudaMemcpyAsync(a.frac, fraction_released_at_death, AS, cudaMemcpyHostToDevice, s->stream));
	else
		BFVM_CUDA(cudaMemsetAsync(a.frac, 0, AS, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.vol, volumes, (size_t)count * sizeof(float), cudaMemcpyHostToDevice, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.pos, positions, (size_t)count * s->dims * sizeof(float), cudaMemcpyHostToDevice,
							  s->stream));
	if (resized)
	{
		a.binned = false;
		a.sorted = false; // the stored amounts are the master until the next binning sorts them
	}
	else if ((st = agents_resort_internalized(s)))
		return st;
	return BFVM_OK;
}

int bfvm_store_agent_positions(bfvm_solver* s, int32_t count, const float* positions)
{
	CHECK_SOLVER(s);
	if (count != s->ag.count)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "count " + std::to_string(count) + " differs from the "
												   + std::to_string(s->ag.count) + " stored agents");
	if (count == 0)
		return BFVM_OK;
	if (!positions)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null positions");
	int rc;
	if ((rc = order_after_copies(s)))
		return rc;
	BFVM_CUDA(cudaMemcpyAsync(s->ag.pos, positions, (size_t)count * s->dims * sizeof(float), cudaMemcpyHostToDevice,
							  s->stream));
	return BFVM_OK;
}

int bfvm_store_agent_positions_async(bfvm_solver* s, int32_t count, const float* positions)
{
	CHECK_SOLVER(s);
	if (count != s->ag.count)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "count " + std::to_string(count) + " differs from the "
												   + std::to_string(s->ag.count) + " stored agents");
	if (count == 0)
		return BFVM_OK;
	if (!positions)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null positions");
	int rc;
	if ((rc = begin_async_copy(s)))
		return rc;
	BFVM_CUDA(cudaMemcpyAsync(s->ag.pos, positions, (size_t)count * s->dims * sizeof(float), cudaMemcpyHostToDevice,
							  s->copy_stream));
	return end_async_copy(s);
}

int bfvm_load_internalized_async(bfvm_solver* s, float* host)
{
	CHECK_SOLVER(s);
	if (s->ag.count == 0)
		return BFVM_OK;
	if (!host)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null host buffer");
	int rc;
	// amounts held in sorted order are written to agent order first, after earlier copies read it
	if (s->ag.sorted && ((rc = order_after_copies(s)) || (rc = agents_unsort(s, true))))
		return rc;
	if ((rc = begin_async_copy(s)))
		return rc;
	BFVM_CUDA(cudaMemcpyAsync(host, s->ag.intern, (size_t)s->ag.count * s->S * sizeof(float), cudaMemcpyDeviceToHost,
							  s->copy_stream));
	return end_async_copy(s);
}

int bfvm_load_internalized(bfvm_solver* s, float* host)
{
	CHECK_SOLVER(s);
	if (s->ag.count == 0)
		return BFVM_OK;
	if (!host)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null host buffer");
	int rc;
	if ((rc = order_after_copies(s)) || (rc = agents_unsort(s, true)))
		return rc;
	BFVM_CUDA(cudaMemcpyAsync(host, s->ag.intern, (size_t)s->ag.count * s->S * sizeof(float), cudaMemcpyDeviceToHost,
							  s->stream));
	return check_device_errors(s);
}

int bfvm_diffusion_solve(bfvm_solver* s)
{
	CHECK_SOLVER(s);
	REFUSE_SLABS(s, "bfvm_diffusion_solve");
	return diffusion(s);
}

int bfvm_diffusion_sweep(bfvm_solver* s, int axis)
{
	CHECK_SOLVER(s);
	if (axis < 0 || axis >= s->dims)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "axis must be in [0, dims)");
	if (axis == 2)
		REFUSE_SLABS(s, "the z sweep");
	return launch_sweep(s, axis, axis == s->dims - 1);
}

int bfvm_dirichlet_solve(bfvm_solver* s)
{
	CHECK_SOLVER(s);
	return launch_dirichlet(s);
}

int bfvm_diffusion_gradient_solve(bfvm_solver* s)
{
	CHECK_SOLVER(s);
	REFUSE_SLABS(s, "bfvm_diffusion_gradient_solve");
	bool done = false;
	int st = launch_diffusion(s, true, &done);
	if (st)
		return st;
	return done ? BFVM_OK : launch_gradient(s);
}

int bfvm_gradient_solve(bfvm_solver* s)
{
	CHECK_SOLVER(s);
	REFUSE_SLABS(s, "bfvm_gradient_solve");
	return launch_gradient(s);
}

int bfvm_secretion_solve(bfvm_solver* s, int recompute)
{
	CHECK_SOLVER(s);
	int rc;
	if ((rc = order_after_copies(s)))
		return rc;
	return launch_secretion(s, recompute != 0);
}

int bfvm_set_bulk_rates(bfvm_solver* s, int per_voxel, const float* supply_rates, const float* uptake_rates,
						const float* supply_target_densities)
{
	CHECK_SOLVER(s);
	if (supply_rates && (!uptake_rates || !supply_target_densities))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "uptake rates and supply target densities must accompany supply rates");
	free_graphs(s);
	return set_bulk_rates(s, per_voxel ? 1 : 0, supply_rates, uptake_rates, supply_target_densities);
}

int bfvm_bulk_solve(bfvm_solver* s)
{
	CHECK_SOLVER(s);
	return launch_bulk(s);
}

int bfvm_release_internalized(bfvm_solver* s, int32_t index)
{
	CHECK_SOLVER(s);
	if (index < 0 || index >= s->ag.count)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent index out of range");
	int rc;
	if ((rc = order_after_copies(s)))
		return rc;
	return launch_release(s, index);
}

int bfvm_add_agents(bfvm_solver* s, int32_t count, const float* secretion_rates, const float* saturation_densities,
					const float* uptake_rates, const float* net_export_rates, const float* internalized_substrates,
					const float* fraction_released_at_death, const float* volumes, const float* positions)
{
	CHECK_SOLVER(s);
	if (count < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "count must not be negative");
	if (count == 0)
		return BFVM_OK;
	if ((long long)s->ag.count + count > INT32_MAX)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "more than 2^31 - 1 agents");
	int st;
	if ((st = order_after_copies(s)) || (st = agents_unsort(s, false)))
		return st;
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	free_graphs(s);
	const int old = s->ag.count;
	if ((st = cell_grow(s, old + count)))
		return st;
	agent_state& a = s->ag;
	const float* src[8] = { secretion_rates, saturation_densities, uptake_rates, net_export_rates,
							internalized_substrates, fraction_released_at_death, volumes, positions };
	float* dst[8] = { a.sec, a.sat, a.upt, a.nex, a.intern, a.frac, a.vol, a.pos };
	const size_t row[8] = { (size_t)s->S, (size_t)s->S, (size_t)s->S, (size_t)s->S, (size_t)s->S, (size_t)s->S, 1,
							(size_t)s->dims };
	for (int k = 0; k < 8; k++)
	{
		float* d = dst[k] + (size_t)old * row[k];
		const size_t bytes = (size_t)count * row[k] * sizeof(float);
		if (src[k])
			BFVM_CUDA(cudaMemcpyAsync(d, src[k], bytes, cudaMemcpyHostToDevice, s->stream));
		else
			BFVM_CUDA(cudaMemsetAsync(d, 0, bytes, s->stream));
	}
	a.binned = false;
	return BFVM_OK;
}

// The moves that sequential agent_data::remove calls amount to.  Only agents at or above the final
// count ever move (a removal moves the then-last agent, and the last slot never falls below the
// final count), and each moves down into a slot below it: so the stored order needs one move per
// slot below the final count whose occupant changed, from that occupant's original row.
static int plan_removal(int agents, int count, const int32_t* indices, int& remaining, std::vector<int>& dst,
						std::vector<int>& src)
{
	if (agents < 0 || count < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent and removal counts must not be negative");
	if (count > 0 && !indices)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null indices");
	std::unordered_map<int, int> at; // slot -> original row of its agent, for slots whose agent changed
	int c = agents;
	for (int k = 0; k < count; k++)
	{
		const int i = indices[k];
		if (i < 0 || i >= c)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "removal " + std::to_string(k) + ": index " + std::to_string(i)
													   + " is not below the agent count " + std::to_string(c));
		const int last = c - 1;
		if (i != last)
		{
			const auto it = at.find(last);
			at[i] = it != at.end() ? it->second : last;
		}
		at.erase(last);
		c--;
	}
	remaining = c;
	dst.clear();
	src.clear();
	std::vector<std::pair<int, int>> mv(at.begin(), at.end());
	std::sort(mv.begin(), mv.end());
	for (const auto& m : mv)
	{
		dst.push_back(m.first);
		src.push_back(m.second);
	}
	return BFVM_OK;
}

int bfvm_plan_agent_removal(int32_t agents, int32_t count, const int32_t* indices, int32_t* remaining,
							int32_t* moves, int32_t* dst, int32_t* src)
{
	if (!remaining || !moves || (count > 0 && (!dst || !src)))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null output");
	int r;
	std::vector<int> d, f;
	const int st = plan_removal(agents, count, indices, r, d, f);
	if (st)
		return st;
	*remaining = r;
	*moves = (int32_t)d.size();
	std::copy(d.begin(), d.end(), dst);
	std::copy(f.begin(), f.end(), src);
	return BFVM_OK;
}

int bfvm_remove_agents(bfvm_solver* s, int32_t count, const int32_t* indices)
{
	CHECK_SOLVER(s);
	int remaining, st;
	std::vector<int> dst, src;
	if ((st = plan_removal(s->ag.count, count, indices, remaining, dst, src)))
		return st;
	if (count == 0)
		return BFVM_OK;
	if ((st = order_after_copies(s)) || (st = agents_unsort(s, false)))
		return st;
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	free_graphs(s);
	if ((st = launch_agent_moves(s, dst, src)))
		return st;
	s->ag.count = remaining;
	s->ag.binned = false;
	return BFVM_OK;
}

int bfvm_run_steps(bfvm_solver* s, int32_t steps, int32_t first_step)
{
	CHECK_SOLVER(s);
	if (steps < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "steps must not be negative");
	REFUSE_SLABS(s, "bfvm_run_steps");
	// agent copies issued on the copy stream are waited for inside each step, right before its
	// secretion (one_step); the events exist before any graph is captured, so every graph holds
	// that wait
	int oc;
	if (s->ag.count > 0 && (oc = ensure_copy_stream(s)))
		return oc;
	if (s->grad_fused && (oc = grad_fuse_buffers(s)))
		return oc;
	for (int i = 0; i < steps; i++)
	{
		const int rc = ((first_step + i) % 10 == 0) ? 1 : 0;
		// the first non-recompute step after new agents needs a binning pass; run it eagerly
		if (!rc && s->ag.count > 0 && !s->ag.binned)
		{
			int st = one_step(s, false);
			if (st)
				return st;
			continue;
		}
		// what a step launches depends on whether the agent terms are sorted when it starts (a
		// recompute step writes sorted amounts back first; a step after a batch sorts them), so
		// there is a graph per (recompute, sorted before) and the host state advances as the
		// captured step did
		const int gi = 2 * rc + (s->ag.sorted ? 1 : 0);
		if (!s->step_graph[gi])
		{
			cudaGraph_t g = nullptr;
			const bool sorted_before = s->ag.sorted;
			BFVM_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
			const long long before = s->launches;
			int st = one_step(s, rc == 1);
			cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
			if (st)
			{
				if (g)
					cudaGraphDestroy(g);
				return st;
			}
			if (ce != cudaSuccess)
				return cuda_fail(ce, "cudaStreamEndCapture");
			s->graph_kernels[gi] = s->launches - before;
			s->graph_sorted_after[gi] = s->ag.sorted;
			s->launches = before;
			s->ag.sorted = sorted_before; // set again below, as after every launch of the graph
			ce = cudaGraphInstantiate(&s->step_graph[gi], g, 0);
			cudaGraphDestroy(g);
			if (ce != cudaSuccess)
			{
				s->step_graph[gi] = nullptr;
				return cuda_fail(ce, "cudaGraphInstantiate");
			}
		}
		BFVM_CUDA(cudaGraphLaunch(s->step_graph[gi], s->stream));
		s->launches += s->graph_kernels[gi];
		if (s->ag.count > 0)
		{
			s->ag.binned = true;
			s->ag.sorted = s->graph_sorted_after[gi];
		}
	}
	return BFVM_OK;
}

int bfvm_synchronize(bfvm_solver* s)
{
	CHECK_SOLVER(s);
	if (s->copy_stream)
		BFVM_CUDA(cudaStreamSynchronize(s->copy_stream));
	s->copy_pending = false;
	BFVM_CUDA(cudaStreamSynchronize(s->stream));
	return check_device_errors(s);
}

int bfvm_set_option(bfvm_solver* s, const char* name, int64_t value)
{
	CHECK_SOLVER(s);
	if (!name)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null option name");
	const std::string n(name);
	if (n == "tma_sweeps")
		s->use_tma = value != 0;
	else if (n == "tma_prefetch")
		s->tma_prefetch = value != 0;
	else if (n == "chunk_elements")
	{
		if (value != 0 && (value < 64 || value > 512))
			return fail(BFVM_ERR_INVALID_ARGUMENT, "chunk_elements must be 0 (automatic) or lie in [64, 512]");
		s->chunk_elements = (int)value;
		free_graphs(s);
		return rebuild_chunks(s);
	}
	else if (n == "tma_pairs")
	{
		if (value < 0 || value > 2)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "tma_pairs takes 0, 1 or 2");
		s->tma_pairs = (int)value;
	}
	else if (n == "fused_dirichlet")
		s->dir_fused = value != 0;
	else if (n == "fused_gradient")
		s->grad_fused = value != 0;
	else if (n == "face_dirichlet")
		s->face_dirichlet = value != 0;
	else if (n == "fused_gradient_evict_first")
		s->grad_evict_first = value != 0;
	else if (n == "xy_band_planes" || n == "zg_band_rows")
	{
		if (value < 0 || value > (1 << 20))
			return fail(BFVM_ERR_INVALID_ARGUMENT, n + " must lie in [0, 2^20]");
		(n == "xy_band_planes" ? s->xy_band_planes : s->zg_band_rows) = (int)value;
	}
	else if (n == "wait_limit_cycles")
	{
		if (value < 10000 || value > 40000000000LL)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "wait_limit_cycles must lie in [1e4, 4e10]");
		s->wait_limit_cycles = value;
	}
	else if (n == "test_drop_tile_copy")
	{
		if (value < -1)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "test_drop_tile_copy takes a tile index or -1");
		s->drop_tile_copy = value;
	}
	else
		return fail(BFVM_ERR_INVALID_ARGUMENT, "unknown option " + n);
	free_graphs(s);
	return BFVM_OK;
}

int bfvm_device_densities(bfvm_solver* s, float** ptr, int64_t* count)
{
	if (!s || !ptr)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	*ptr = s->dens;
	if (count)
		*count = s->V * s->S;
	return BFVM_OK;
}

int bfvm_device_gradients(bfvm_solver* s, float** ptr, int64_t* count)
{
	if (!s || !ptr)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	*ptr = s->grad;
	if (count)
		*count = s->V * s->S * s->dims;
	return BFVM_OK;
}

int bfvm_launch_count(const bfvm_solver* s, int64_t* launches)
{
	if (!s || !launches)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null argument");
	*launches = s->launches;
	return BFVM_OK;
}

} // extern "C"
