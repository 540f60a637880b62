// Agent secretion and uptake (paraBioFVM src/solver/host/cell_solver.cpp:15-373).
//
// Per agent i and substrate s (recompute steps, :63-85):
//   num = S*T*dt*vol/Vv     den = (U+S)*dt*vol/Vv     fac = N*dt/Vv
// Per voxel, over the agents in it, the reference reduces into the slot of a "winner" agent:
//   Rnum = sum num,  Rden = (den_w + 1) + sum_{others} den,  Rfac = sum fac        (:87-135)
// and every step (:197-245) updates
//   D = (D + Rnum) / Rden + Rfac
// with, when internalized substrates are tracked,
//   I -= Vv*(((1-Rden)*D + Rnum)/Rden + Rfac)              if no voxel holds two agents (:173-195)
//   I -= Vv*((-den*D + num)/(1+den) + fac), per agent       otherwise (:137-152)
// using the density from before the update.
//
// The reference picks the winner with a parallel compare-and-swap, so winner and summation order
// depend on thread timing.  Here agents are binned by a stable radix sort of their voxel index:
// the winner is the lowest agent index of the voxel and the sums run in agent index order, which
// is the reference's single-thread result.  One thread then owns one (voxel, substrate) pair, so
// the update needs no atomics and repeats bit for bit.  All arithmetic uses explicitly rounded
// operations in the reference's association.

#include <algorithm>

#include "agent_kernels.cuh"
#include "sweep_common.cuh"

namespace bfvm {

// ---------------------------------------------------------------------------------------------
// voxel keys

__device__ __forceinline__ bool voxel_of(const float* pos, int dims, int3 bmin, int3 vox, int3 grid, int3& c)
{
	// truncating (pos - min) / dx as in src/mesh.cpp:35-53; positions in (-dx, 0) truncate to 0 there
	// too.  Anything outside the mesh is rejected instead of indexing out of bounds.
	c = make_int3(0, 0, 0);
	const int bm[3] = { bmin.x, bmin.y, bmin.z };
	const int vx[3] = { vox.x, vox.y, vox.z };
	const int gr[3] = { grid.x, grid.y, grid.z };
	int out[3] = { 0, 0, 0 };
	for (int d = 0; d < dims; d++)
	{
		const float t = __fdiv_rn(__fsub_rn(pos[d], (float)bm[d]), (float)vx[d]);
		if (!(t > -1.0f && t < (float)gr[d]))
			return false;
		out[d] = (int)t;
	}
	c = make_int3(out[0], out[1], out[2]);
	return true;
}

__global__ void agent_keys_kernel(const float* __restrict__ pos, int A, int dims, int3 bmin, int3 vox, int3 grid,
								  unsigned int* __restrict__ keys, int* __restrict__ vals, unsigned int invalid_key,
								  int* err)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= A)
		return;
	int3 c;
	if (voxel_of(pos + (size_t)i * dims, dims, bmin, vox, grid, c))
		keys[i] = (unsigned int)c.x + (unsigned int)grid.x * ((unsigned int)c.y + (unsigned int)grid.y * (unsigned int)c.z);
	else
	{
		keys[i] = invalid_key;
		atomicOr(err, DEVERR_AGENT_OUTSIDE);
	}
	vals[i] = i;
}

// ---------------------------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits, tiles of 4096 keys

__global__ void __launch_bounds__(SORT_THREADS) radix_hist_kernel(const unsigned int* __restrict__ keys, int n,
																	 int shift, int* __restrict__ hist, int tiles)
{
	__shared__ int h[256];
	h[threadIdx.x] = 0;
	__syncthreads();
	const long long base = (long long)blockIdx.x * SORT_TILE;
	for (int r = 0; r < SORT_ROUNDS; r++)
	{
		const long long idx = base + r * SORT_THREADS + threadIdx.x;
		if (idx < n)
			atomicAdd(&h[(keys[idx] >> shift) & 255u], 1);
	}
	__syncthreads();
	hist[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(SORT_THREADS) radix_scatter_kernel(
	const unsigned int* __restrict__ keys_in, const int* __restrict__ vals_in, unsigned int* __restrict__ keys_out,
	int* __restrict__ vals_out, int n, int shift, const int* __restrict__ offsets, int tiles)
{
	__shared__ int run[256];
	__shared__ int wcnt[SORT_THREADS / 32][256];
	__shared__ int tot[256];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	run[tid] = offsets[(size_t)tid * tiles + blockIdx.x];
	const long long base = (long long)blockIdx.x * SORT_TILE;

	for (int r = 0; r < SORT_ROUNDS; r++)
	{
#pragma unroll
		for (int w = 0; w < SORT_THREADS / 32; w++)
			wcnt[w][tid] = 0;
		__syncthreads();

		const long long idx = base + r * SORT_THREADS + tid;
		const bool valid = idx < n;
		const unsigned int key = valid ? keys_in[idx] : 0u;
		const int val = valid ? vals_in[idx] : 0;
		const int digit = valid ? (int)((key >> shift) & 255u) : 256 + lane;
		const unsigned int peers = __match_any_sync(0xffffffffu, digit);
		const int rank = __popc(peers & ((1u << lane) - 1u));
		if (valid && lane == __ffs(peers) - 1)
			wcnt[warp][digit] = __popc(peers);
		__syncthreads();

		int acc = 0;
#pragma unroll
		for (int w = 0; w < SORT_THREADS / 32; w++)
		{
			const int c = wcnt[w][tid];
			wcnt[w][tid] = acc;
			acc += c;
		}
		tot[tid] = acc;
		__syncthreads();

		if (valid)
		{
			const int p = run[digit] + wcnt[warp][digit] + rank;
			keys_out[p] = key;
			vals_out[p] = val;
		}
		__syncthreads();
		run[tid] += tot[tid];
	}
}

// ---------------------------------------------------------------------------------------------
// voxel segments of the sorted keys

__global__ void seg_flags_kernel(const unsigned int* __restrict__ keys, int n, unsigned int invalid_key,
								 int* __restrict__ flags)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n)
		return;
	const unsigned int k = keys[p];
	flags[p] = (k != invalid_key && (p == 0 || keys[p - 1] != k)) ? 1 : 0;
}

// counts[0] = segments, counts[1] = agents inside the mesh, counts[2] = 1 if a voxel holds 2+ agents
__global__ void seg_finish_kernel(const unsigned int* __restrict__ keys, const int* __restrict__ flags,
								  const int* __restrict__ seg_id, int n, unsigned int invalid_key,
								  int* __restrict__ seg_start, int* __restrict__ counts)
{
	const int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n)
		return;
	const unsigned int k = keys[p];
	if (flags[p])
		seg_start[seg_id[p]] = p;
	if (k != invalid_key && (p == n - 1 || keys[p + 1] == invalid_key))
	{
		const int nseg = seg_id[p] + flags[p];
		counts[0] = nseg;
		counts[1] = p + 1;
		counts[2] = (p + 1 > nseg) ? 1 : 0;
		seg_start[nseg] = p + 1;
	}
}

// ---------------------------------------------------------------------------------------------
// intermediates and reductions (recompute steps)

__global__ void intermediates_kernel(long long total, int S, const float* __restrict__ sec,
									 const float* __restrict__ sat, const float* __restrict__ upt,
									 const float* __restrict__ nex, const float* __restrict__ vol, float voxel_volume,
									 float dt, float* __restrict__ num, float* __restrict__ den, float* __restrict__ fac)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	const long long i = t / S;
	const float v = vol[i];
	num[t] = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(sec[t], sat[t]), dt), v), voxel_volume);
	den[t] = __fdiv_rn(__fmul_rn(__fmul_rn(__fadd_rn(upt[t], sec[t]), dt), v), voxel_volume);
	fac[t] = __fdiv_rn(__fmul_rn(nex[t], dt), voxel_volume);
}

__global__ void reduce_kernel(long long total, int S, const int* __restrict__ counts,
							  const int* __restrict__ seg_start, const int* __restrict__ order,
							  const float* __restrict__ num, const float* __restrict__ den,
							  const float* __restrict__ fac, float* __restrict__ red_num, float* __restrict__ red_den,
							  float* __restrict__ red_fac)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	const int seg = (int)(t / S);
	const int s = (int)(t % S);
	if (seg >= counts[0])
		return;
	const int b = seg_start[seg], e = seg_start[seg + 1];
	const size_t w = (size_t)order[b] * S + s;
	float rn = __fadd_rn(0.f, num[w]);
	float rd = __fadd_rn(0.f, __fadd_rn(den[w], 1.f));
	float rf = __fadd_rn(0.f, fac[w]);
	for (int p = b + 1; p < e; p++)
	{
		const size_t k = (size_t)order[p] * S + s;
		rn = __fadd_rn(rn, num[k]);
		rd = __fadd_rn(rd, den[k]);
		rf = __fadd_rn(rf, fac[k]);
	}
	red_num[t] = rn;
	red_den[t] = rd;
	red_fac[t] = rf;
}

// The same sums over rows in the binning's sorted order (row p is the agent at sorted position p).
__global__ void reduce_sorted_kernel(long long total, int S, const int* __restrict__ counts,
									 const int* __restrict__ seg_start, const float* __restrict__ num,
									 const float* __restrict__ den, const float* __restrict__ fac,
									 float* __restrict__ red_num, float* __restrict__ red_den,
									 float* __restrict__ red_fac)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	const int seg = (int)(t / S);
	const int s = (int)(t % S);
	if (seg >= counts[0])
		return;
	const int b = seg_start[seg], e = seg_start[seg + 1];
	const size_t w = (size_t)b * S + s;
	float rn = __fadd_rn(0.f, num[w]);
	float rd = __fadd_rn(0.f, __fadd_rn(den[w], 1.f));
	float rf = __fadd_rn(0.f, fac[w]);
	for (int p = b + 1; p < e; p++)
	{
		const size_t k = (size_t)p * S + s;
		rn = __fadd_rn(rn, num[k]);
		rd = __fadd_rn(rd, den[k]);
		rf = __fadd_rn(rf, fac[k]);
	}
	red_num[t] = rn;
	red_den[t] = rd;
	red_fac[t] = rf;
}

// Row p of the sorted copies takes row order[p] of the agent-order arrays, and rank[order[p]] = p
// (t over A * S; every agent, those outside the mesh included, has a row).
__global__ void sort_agent_terms_kernel(long long total, int S, const int* __restrict__ order,
										const float* __restrict__ num, const float* __restrict__ den,
										const float* __restrict__ fac, const float* __restrict__ intern,
										float* __restrict__ snum, float* __restrict__ sden, float* __restrict__ sfac,
										float* __restrict__ sintern, int* __restrict__ rank)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	const int p = (int)(t / S);
	const int s = (int)(t - (long long)p * S);
	const int i = order[p];
	const size_t k = (size_t)i * S + s;
	snum[t] = num[k];
	sden[t] = den[k];
	sfac[t] = fac[k];
	sintern[t] = intern[k];
	if (s == 0)
		rank[i] = p;
}

// One array between the two orders: to_sorted, row p of `sorted` takes row order[p] of `agent`;
// otherwise row order[p] of `agent` takes row p of `sorted`.
__global__ void permute_rows_kernel(long long total, int S, const int* __restrict__ order, float* __restrict__ agent,
									float* __restrict__ sorted, int to_sorted)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	const int p = (int)(t / S);
	const size_t k = (size_t)order[p] * S + (t - (long long)p * S);
	if (to_sorted)
		sorted[t] = agent[k];
	else
		agent[k] = sorted[t];
}

// ---------------------------------------------------------------------------------------------
// the per-step update (compute_result)

__global__ void secrete_kernel(long long total, int S, float* __restrict__ dens, const int* __restrict__ counts,
							   const int* __restrict__ seg_start, const int* __restrict__ order,
							   const unsigned int* __restrict__ keys, const float* __restrict__ num,
							   const float* __restrict__ den, const float* __restrict__ fac,
							   const float* __restrict__ red_num, const float* __restrict__ red_den,
							   const float* __restrict__ red_fac, float* __restrict__ intern, int internalized,
							   float voxel_volume)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	secrete_element(t, S, dens, counts, seg_start, order, keys, num, den, fac, red_num, red_den, red_fac, intern,
					internalized, voxel_volume);
}

// The same update with the per-agent rows in the binning's sorted order: an agent's rows are read
// and written where its voxel's segment lies, so a warp touches contiguous memory.
__global__ void secrete_sorted_kernel(long long total, int S, float* __restrict__ dens, const int* __restrict__ counts,
									  const int* __restrict__ seg_start, const unsigned int* __restrict__ keys,
									  const float* __restrict__ snum, const float* __restrict__ sden,
									  const float* __restrict__ sfac, const float* __restrict__ red_num,
									  const float* __restrict__ red_den, const float* __restrict__ red_fac,
									  float* __restrict__ sintern, float voxel_volume)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total)
		return;
	secrete_element<true>(t, S, dens, counts, seg_start, nullptr, keys, snum, sden, sfac, red_num, red_den, red_fac,
						  sintern, 1, voxel_volume);
}

// release_internalized_substrates (:301-346): D += I*F/Vv at the agent's current voxel, I = 0
__global__ void release_kernel(int index, int S, int dims, const float* __restrict__ pos, int3 bmin, int3 vox,
							   int3 grid, float* __restrict__ dens, float* __restrict__ intern,
							   const float* __restrict__ frac, float voxel_volume, int* err)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= S)
		return;
	int3 c;
	if (!voxel_of(pos + (size_t)index * dims, dims, bmin, vox, grid, c))
	{
		if (s == 0)
			atomicOr(err, DEVERR_AGENT_OUTSIDE);
		return;
	}
	const size_t v = (size_t)c.x + (size_t)grid.x * ((size_t)c.y + (size_t)grid.y * c.z);
	const size_t k = (size_t)index * S + s;
	dens[v * S + s] = __fadd_rn(dens[v * S + s], __fdiv_rn(__fmul_rn(intern[k], frac[k]), voxel_volume));
	intern[k] = 0.f;
}

// The sorted update four substrates at a time (S % 4 == 0; secrete_sorted4_element).  Its threads
// stride over the segments the binning found (counts[0], read on the device), so no thread is
// launched for agents that share a voxel.
__global__ void __launch_bounds__(256) secrete_sorted4_kernel(int S, float* __restrict__ dens,
															  const int* __restrict__ counts,
															  const int* __restrict__ seg_start,
															  const unsigned int* __restrict__ keys,
															  const float* __restrict__ snum, const float* __restrict__ sden,
															  const float* __restrict__ sfac,
															  const float* __restrict__ red_num,
															  const float* __restrict__ red_den,
															  const float* __restrict__ red_fac,
															  float* __restrict__ sintern, float voxel_volume)
{
	const long long n = (long long)counts[0] * (S >> 2);
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
		secrete_sorted4_element(t, S, dens, counts, seg_start, keys, snum, sden, sfac, red_num, red_den, red_fac, sintern,
								voxel_volume);
}

// The same release with the internalized amounts in sorted order: agent `index` is at row rank[index].
__global__ void release_sorted_kernel(int index, int S, int dims, const float* __restrict__ pos, int3 bmin, int3 vox,
									  int3 grid, float* __restrict__ dens, float* __restrict__ sintern,
									  const int* __restrict__ rank, const float* __restrict__ frac, float voxel_volume,
									  int* err)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= S)
		return;
	int3 c;
	if (!voxel_of(pos + (size_t)index * dims, dims, bmin, vox, grid, c))
	{
		if (s == 0)
			atomicOr(err, DEVERR_AGENT_OUTSIDE);
		return;
	}
	const size_t v = (size_t)c.x + (size_t)grid.x * ((size_t)c.y + (size_t)grid.y * c.z);
	const size_t k = (size_t)rank[index] * S + s;
	const float f = frac[(size_t)index * S + s];
	dens[v * S + s] = __fadd_rn(dens[v * S + s], __fdiv_rn(__fmul_rn(sintern[k], f), voxel_volume));
	sintern[k] = 0.f;
}

// ---------------------------------------------------------------------------------------------
// host side

void cell_free(bfvm_solver* s)
{
	agent_state& a = s->ag;
	for (float** p : { &a.sec, &a.sat, &a.upt, &a.nex, &a.intern, &a.frac, &a.vol, &a.pos, &a.num, &a.den, &a.fac,
					   &a.red_num, &a.red_den, &a.red_fac, &a.snum, &a.sden, &a.sfac, &a.sintern })
		device_free(*p);
	device_free(a.rank);
	a.sorted = false;
	device_free(a.keys);
	device_free(a.keys_alt);
	device_free(a.vals);
	device_free(a.vals_alt);
	device_free(a.hist);
	device_free(a.flags);
	device_free(a.seg_id);
	device_free(a.seg_start);
	device_free(a.seg_count_dev);
	scan_plan_free(a.hist_scan);
	scan_plan_free(a.flag_scan);
	device_free(a.move_idx);
	a.move_capacity = 0;
	a.capacity = 0;
	a.count = 0;
	a.binned = false;
}

int cell_alloc(bfvm_solver* s, int count)
{
	agent_state& a = s->ag;
	if (count <= a.capacity && a.capacity > 0)
	{
		a.count = count;
		return BFVM_OK;
	}
	cell_free(s);
	const size_t AS = (size_t)count * s->S;
	int st = 0;
	for (float** p : { &a.sec, &a.sat, &a.upt, &a.nex, &a.intern, &a.frac, &a.num, &a.den, &a.fac, &a.red_num,
					   &a.red_den, &a.red_fac })
		if ((st = device_alloc(p, AS)))
			return st;
	if ((st = device_alloc(&a.vol, (size_t)count)) || (st = device_alloc(&a.pos, (size_t)count * s->dims)))
		return st;
	if (s->internalized)
	{
		for (float** p : { &a.snum, &a.sden, &a.sfac, &a.sintern })
			if ((st = device_alloc(p, AS)))
				return st;
		if ((st = device_alloc(&a.rank, (size_t)count)))
			return st;
	}
	a.tiles = (int)((count + SORT_TILE - 1) / SORT_TILE);
	if ((st = device_alloc(&a.keys, (size_t)count)) || (st = device_alloc(&a.keys_alt, (size_t)count))
		|| (st = device_alloc(&a.vals, (size_t)count)) || (st = device_alloc(&a.vals_alt, (size_t)count))
		|| (st = device_alloc(&a.hist, (size_t)256 * a.tiles)) || (st = device_alloc(&a.flags, (size_t)count))
		|| (st = device_alloc(&a.seg_id, (size_t)count)) || (st = device_alloc(&a.seg_start, (size_t)count + 1))
		|| (st = device_alloc(&a.seg_count_dev, 4)))
		return st;
	if ((st = scan_plan_build(a.hist_scan, 256LL * a.tiles)) || (st = scan_plan_build(a.flag_scan, count)))
		return st;
	a.capacity = count;
	a.count = count;
	return BFVM_OK;
}

int rebuild_bins(bfvm_solver* s, bool sorted)
{
	agent_state& a = s->ag;
	const int A = a.count;
	const int3 bmin = make_int3(s->bbox_min[0], s->bbox_min[1], s->bbox_min[2]);
	const int3 vox = make_int3(s->voxel[0], s->voxel[1], s->voxel[2]);
	const int3 grid = make_int3(s->grid[0], s->grid[1], s->grid[2]);
	const unsigned int invalid = (unsigned int)s->V;
	int st;

	BFVM_CUDA(cudaMemsetAsync(a.seg_count_dev, 0, 4 * sizeof(int), s->stream));
	// The sort ping-pongs between the two buffers once per pass; starting in the buffer that makes
	// it end in keys/vals keeps those pointers fixed, so graphs and ensemble descriptors that hold
	// them stay valid.
	const int passes = sort_passes(s->V);
	unsigned int* kin = (passes % 2) ? a.keys_alt : a.keys;
	unsigned int* kout = (passes % 2) ? a.keys : a.keys_alt;
	int* vin = (passes % 2) ? a.vals_alt : a.vals;
	int* vout = (passes % 2) ? a.vals : a.vals_alt;
	agent_keys_kernel<<<(A + 255) / 256, 256, 0, s->stream>>>(a.pos, A, s->dims, bmin, vox, grid, kin, vin, invalid,
															   s->dev_error);
	if ((st = check_launch(s, "agent_keys_kernel")))
		return st;

	const int tiles = (A + SORT_TILE - 1) / SORT_TILE;
	for (int pass = 0; pass < passes; pass++)
	{
		radix_hist_kernel<<<tiles, SORT_THREADS, 0, s->stream>>>(kin, A, 8 * pass, a.hist, tiles);
		if ((st = check_launch(s, "radix_hist_kernel")))
			return st;
		if ((st = launch_exclusive_scan(s, a.hist_scan, a.hist, a.hist, 256LL * tiles)))
			return st;
		radix_scatter_kernel<<<tiles, SORT_THREADS, 0, s->stream>>>(kin, vin, kout, vout, A, 8 * pass, a.hist, tiles);
		if ((st = check_launch(s, "radix_scatter_kernel")))
			return st;
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	// the sorted result is in a.keys / a.vals now (kin == a.keys)

	seg_flags_kernel<<<(A + 255) / 256, 256, 0, s->stream>>>(a.keys, A, invalid, a.flags);
	if ((st = check_launch(s, "seg_flags_kernel")))
		return st;
	if ((st = launch_exclusive_scan(s, a.flag_scan, a.flags, a.seg_id, A)))
		return st;
	seg_finish_kernel<<<(A + 255) / 256, 256, 0, s->stream>>>(a.keys, a.flags, a.seg_id, A, invalid, a.seg_start,
															   a.seg_count_dev);
	if ((st = check_launch(s, "seg_finish_kernel")))
		return st;

	const long long AS = (long long)A * s->S;
	const unsigned blocks = (unsigned)((AS + 255) / 256);
	intermediates_kernel<<<blocks, 256, 0, s->stream>>>(AS, s->S, a.sec, a.sat, a.upt, a.nex, a.vol,
														 (float)(s->voxel[0] * s->voxel[1] * s->voxel[2]), s->dt,
														 a.num, a.den, a.fac);
	if ((st = check_launch(s, "intermediates_kernel")))
		return st;
	if (sorted)
	{
		sort_agent_terms_kernel<<<blocks, 256, 0, s->stream>>>(AS, s->S, a.vals, a.num, a.den, a.fac, a.intern, a.snum,
																a.sden, a.sfac, a.sintern, a.rank);
		if ((st = check_launch(s, "sort_agent_terms_kernel")))
			return st;
		reduce_sorted_kernel<<<blocks, 256, 0, s->stream>>>(AS, s->S, a.seg_count_dev, a.seg_start, a.snum, a.sden,
															 a.sfac, a.red_num, a.red_den, a.red_fac);
		if ((st = check_launch(s, "reduce_sorted_kernel")))
			return st;
	}
	else
	{
		reduce_kernel<<<blocks, 256, 0, s->stream>>>(AS, s->S, a.seg_count_dev, a.seg_start, a.vals, a.num, a.den,
													 a.fac, a.red_num, a.red_den, a.red_fac);
		if ((st = check_launch(s, "reduce_kernel")))
			return st;
	}
	a.binned = true;
	return BFVM_OK;
}

// One per-agent array between agent order and the binning's sorted order.
static int permute_rows(bfvm_solver* s, float* agent, float* sorted, bool to_sorted)
{
	const long long AS = (long long)s->ag.count * s->S;
	permute_rows_kernel<<<(unsigned)((AS + 255) / 256), 256, 0, s->stream>>>(AS, s->S, s->ag.vals, agent, sorted,
																			  to_sorted ? 1 : 0);
	return check_launch(s, "permute_rows_kernel");
}

// While the agent terms are sorted, the internalized amounts live in sintern: write them back to
// agent order (intern).  keep_sorted: as a copy for a load (sintern stays the master); otherwise
// agent order becomes the master.
int agents_unsort(bfvm_solver* s, bool keep_sorted)
{
	agent_state& a = s->ag;
	if (!a.sorted || a.count == 0)
		return BFVM_OK;
	const int st = permute_rows(s, a.intern, a.sintern, false);
	if (!st && !keep_sorted)
		a.sorted = false;
	return st;
}

// Internalized amounts just stored in agent order: into sorted order, when the terms are sorted.
int agents_resort_internalized(bfvm_solver* s)
{
	agent_state& a = s->ag;
	if (!a.sorted || a.count == 0)
		return BFVM_OK;
	return permute_rows(s, a.intern, a.sintern, true);
}

// With internalized substrates the secretion runs on sorted agent terms, alone or in a batch: a
// rebinning sorts them (after writing the internalized amounts back to agent order with the old
// order), and a solver binned but not sorted (stored amounts of an unchanged count) sorts them
// once.  Solvers without internalized substrates keep agent order (only the per-voxel sums are
// read then).
int prepare_agent_terms(bfvm_solver* s, bool recompute)
{
	agent_state& a = s->ag;
	if (a.count == 0)
		return BFVM_OK;
	const bool use_sorted = s->internalized;
	int st;
	if (recompute || !a.binned || (a.sorted && !use_sorted))
	{
		if ((st = agents_unsort(s, false)))
			return st;
	}
	if (recompute || !a.binned)
	{
		if ((st = rebuild_bins(s, use_sorted)))
			return st;
		a.sorted = use_sorted;
	}
	else if (use_sorted && !a.sorted)
	{
		const long long AS = (long long)a.count * s->S;
		sort_agent_terms_kernel<<<(unsigned)((AS + 255) / 256), 256, 0, s->stream>>>(
			AS, s->S, a.vals, a.num, a.den, a.fac, a.intern, a.snum, a.sden, a.sfac, a.sintern, a.rank);
		if ((st = check_launch(s, "sort_agent_terms_kernel")))
			return st;
		a.sorted = true;
	}
	return BFVM_OK;
}

int launch_secretion(bfvm_solver* s, bool recompute)
{
	agent_state& a = s->ag;
	if (a.count == 0)
		return BFVM_OK;
	int st;
	if ((st = prepare_agent_terms(s, recompute)))
		return st;
	const long long AS = (long long)a.count * s->S;
	const float vv = (float)(s->voxel[0] * s->voxel[1] * s->voxel[2]);
	if (a.sorted && s->S % 4 == 0)
	{
		// up to the threads of every segment (at most one per agent), resident at once
		const long long threads = AS / 4;
		const unsigned grid = (unsigned)std::max<long long>(
			1, std::min<long long>((threads + 255) / 256, (long long)sm_count_impl(s->device) * 8));
		secrete_sorted4_kernel<<<grid, 256, 0, s->stream>>>(s->S, s->dens, a.seg_count_dev, a.seg_start, a.keys,
															 a.snum, a.sden, a.sfac, a.red_num, a.red_den, a.red_fac,
															 a.sintern, vv);
		return check_launch(s, "secrete_sorted4_kernel");
	}
	if (a.sorted)
	{
		secrete_sorted_kernel<<<(unsigned)((AS + 255) / 256), 256, 0, s->stream>>>(
			AS, s->S, s->dens, a.seg_count_dev, a.seg_start, a.keys, a.snum, a.sden, a.sfac, a.red_num, a.red_den,
			a.red_fac, a.sintern, vv);
		return check_launch(s, "secrete_sorted_kernel");
	}
	secrete_kernel<<<(unsigned)((AS + 255) / 256), 256, 0, s->stream>>>(
		AS, s->S, s->dens, a.seg_count_dev, a.seg_start, a.vals, a.keys, a.num, a.den, a.fac, a.red_num, a.red_den,
		a.red_fac, a.intern, s->internalized ? 1 : 0, vv);
	return check_launch(s, "secrete_kernel");
}

int launch_release(bfvm_solver* s, int index)
{
	agent_state& a = s->ag;
	if (!s->internalized)
		return BFVM_OK;
	const int3 bmin = make_int3(s->bbox_min[0], s->bbox_min[1], s->bbox_min[2]);
	const int3 vox = make_int3(s->voxel[0], s->voxel[1], s->voxel[2]);
	const int3 grid = make_int3(s->grid[0], s->grid[1], s->grid[2]);
	const float vv = (float)(s->voxel[0] * s->voxel[1] * s->voxel[2]);
	if (a.sorted)
	{
		release_sorted_kernel<<<(s->S + 127) / 128, 128, 0, s->stream>>>(index, s->S, s->dims, a.pos, bmin, vox, grid,
																		  s->dens, a.sintern, a.rank, a.frac, vv,
																		  s->dev_error);
		return check_launch(s, "release_sorted_kernel");
	}
	release_kernel<<<(s->S + 127) / 128, 128, 0, s->stream>>>(index, s->S, s->dims, a.pos, bmin, vox, grid, s->dens,
															  a.intern, a.frac, vv, s->dev_error);
	return check_launch(s, "release_kernel");
}

// Agent storage for `count` agents that keeps the stored agents' rows (bfvm_add_agents).  Growth
// takes at least half the capacity again, so repeated additions copy each row a bounded number of
// times; the binning buffers are rebuilt empty, as the next secretion call rebins.
int cell_grow(bfvm_solver* s, int count)
{
	agent_state& a = s->ag;
	if (count <= a.capacity && a.capacity > 0)
	{
		a.count = count;
		return BFVM_OK;
	}
	const int old = a.count;
	const int cap = (int)std::min<long long>(INT32_MAX, std::max<long long>(count, (long long)a.capacity * 3 / 2));
	float* keep[8] = { a.sec, a.sat, a.upt, a.nex, a.intern, a.frac, a.vol, a.pos };
	for (float** p : { &a.sec, &a.sat, &a.upt, &a.nex, &a.intern, &a.frac, &a.vol, &a.pos })
		*p = nullptr;
	cell_free(s);
	int st = cell_alloc(s, cap);
	if (!st && old > 0)
	{
		float* now[8] = { a.sec, a.sat, a.upt, a.nex, a.intern, a.frac, a.vol, a.pos };
		const size_t rows[8] = { (size_t)s->S, (size_t)s->S, (size_t)s->S, (size_t)s->S, (size_t)s->S, (size_t)s->S, 1,
								 (size_t)s->dims };
		for (int k = 0; k < 8 && !st; k++)
		{
			const cudaError_t e = cudaMemcpyAsync(now[k], keep[k], (size_t)old * rows[k] * sizeof(float),
												  cudaMemcpyDeviceToDevice, s->stream);
			if (e != cudaSuccess)
				st = cuda_fail(e, "cudaMemcpyAsync");
		}
		const cudaError_t e = cudaStreamSynchronize(s->stream);
		if (!st && e != cudaSuccess)
			st = cuda_fail(e, "cudaStreamSynchronize");
	}
	for (float* p : keep)
		device_free(p);
	if (!st)
		a.count = count;
	return st;
}

struct agent_rows
{
	float* v[6]; // [A][S]: secretion, saturation, uptake, net export, internalized, fraction released
	float* vol;	 // [A]
	float* pos;	 // [A][dims]
};

// Row dst[k] of every per-agent array takes row src[k] (the moves of a batch of agent removals;
// no source is a destination, so the moves run in any order).
__global__ void __launch_bounds__(256) agent_move_kernel(const int* __restrict__ dst, const int* __restrict__ src,
														  int moves, int S, int dims, agent_rows r)
{
	const int per = 6 * S + 1 + dims;
	const long long n = (long long)moves * per;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
	{
		const int k = (int)(t / per), e = (int)(t - (long long)k * per);
		const long long d = __ldg(&dst[k]), f = __ldg(&src[k]);
		if (e < 6 * S)
		{
			float* p = r.v[e / S];
			const int j = e % S;
			p[d * S + j] = p[f * S + j];
		}
		else if (e == 6 * S)
			r.vol[d] = r.vol[f];
		else
		{
			const int j = e - 6 * S - 1;
			r.pos[d * dims + j] = r.pos[f * dims + j];
		}
	}
}

int launch_agent_moves(bfvm_solver* s, const std::vector<int>& dst, const std::vector<int>& src)
{
	agent_state& a = s->ag;
	const int moves = (int)dst.size();
	if (moves == 0)
		return BFVM_OK;
	int st;
	if (2 * moves > a.move_capacity)
	{
		BFVM_CUDA(cudaStreamSynchronize(s->stream));
		device_free(a.move_idx);
		a.move_capacity = 0;
		if ((st = device_alloc(&a.move_idx, (size_t)2 * moves)))
			return st;
		a.move_capacity = 2 * moves;
	}
	BFVM_CUDA(cudaMemcpyAsync(a.move_idx, dst.data(), (size_t)moves * sizeof(int), cudaMemcpyHostToDevice, s->stream));
	BFVM_CUDA(cudaMemcpyAsync(a.move_idx + moves, src.data(), (size_t)moves * sizeof(int), cudaMemcpyHostToDevice,
							  s->stream));
	agent_rows r{ { a.sec, a.sat, a.upt, a.nex, a.intern, a.frac }, a.vol, a.pos };
	const long long n = (long long)moves * (6 * s->S + 1 + s->dims);
	const int threads = 256;
	const long long blocks = std::min<long long>((n + threads - 1) / threads, 148LL * 8);
	agent_move_kernel<<<(unsigned)blocks, threads, 0, s->stream>>>(a.move_idx, a.move_idx + moves, moves, s->S,
																	s->dims, r);
	return check_launch(s, "agent_move_kernel");
}

} // namespace bfvm
