// Exclusive prefix sum of int32 arrays: each CTA scans 4096 elements (1024 threads x 4), writes its
// total, the totals are scanned recursively, and a second pass adds the scanned totals back.
// All buffers are allocated when the plan is built, so a scan can be captured in a CUDA graph.

#include "agent_kernels.cuh"

namespace bfvm {

__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_kernel(const int* in, int* out, long long n, int* tile_sums)
{
	__shared__ int warp_sums[SCAN_THREADS / 32];
	const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
	int v[SCAN_ITEMS];
	int local = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++)
	{
		v[k] = (base + k < n) ? in[base + k] : 0;
		local += v[k];
	}
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = local;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1)
	{
		const int t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o)
			incl += t;
	}
	if (lane == 31)
		warp_sums[warp] = incl;
	__syncthreads();
	if (warp == 0)
	{
		int ws = warp_sums[lane];
		int wi = ws;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			const int t = __shfl_up_sync(0xffffffffu, wi, o);
			if (lane >= o)
				wi += t;
		}
		warp_sums[lane] = wi - ws; // exclusive
		if (lane == 31 && tile_sums)
			tile_sums[blockIdx.x] = wi;
	}
	__syncthreads();
	int run = warp_sums[warp] + incl - local;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++)
	{
		if (base + k < n)
			out[base + k] = run;
		run += v[k];
	}
}

__global__ void scan_add_kernel(int* out, long long n, const int* tile_offsets)
{
	const long long tile = blockIdx.x;
	const int add = tile_offsets[tile];
	const long long base = tile * SCAN_TILE;
	for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x)
		if (base + k < n)
			out[base + k] += add;
}

int scan_plan_build(scan_plan& p, long long n)
{
	scan_plan_free(p);
	long long m = n;
	while (m > SCAN_TILE)
	{
		const long long tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
		int* buf = nullptr;
		int st = device_alloc(&buf, (size_t)tiles);
		if (st)
			return st;
		p.level_sizes.push_back(tiles);
		p.level_sums.push_back(buf);
		m = tiles;
	}
	return BFVM_OK;
}

void scan_plan_free(scan_plan& p)
{
	for (int* b : p.level_sums)
		device_free(b);
	p.level_sums.clear();
	p.level_sizes.clear();
}

static int scan_level(bfvm_solver* s, scan_plan& p, size_t level, const int* in, int* out, long long n)
{
	const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
	int* sums = level < p.level_sums.size() ? p.level_sums[level] : nullptr;
	if (tiles > 1 && !sums)
		return fail(BFVM_ERR_STATE, "scan plan too small");
	scan_tile_kernel<<<(unsigned)tiles, SCAN_THREADS, 0, s->stream>>>(in, out, n, tiles > 1 ? sums : nullptr);
	int st = check_launch(s, "scan_tile_kernel");
	if (st || tiles == 1)
		return st;
	st = scan_level(s, p, level + 1, sums, sums, tiles);
	if (st)
		return st;
	scan_add_kernel<<<(unsigned)tiles, 256, 0, s->stream>>>(out, n, sums);
	return check_launch(s, "scan_add_kernel");
}

int launch_exclusive_scan(bfvm_solver* s, scan_plan& p, const int* in, int* out, long long n)
{
	if (n <= 0)
		return BFVM_OK;
	return scan_level(s, p, 0, in, out, n);
}

} // namespace bfvm
