// Kernels of the agent binning and secretion pipeline (cell.cu) and of the exclusive scan
// (scan.cu), declared for the launchers in other files.
#pragma once

#include "bfvm_internal.h"

namespace bfvm {

// radix sort of the agents' voxel keys: 256-thread CTAs, each ranking 16 rounds of 256 keys
static constexpr int SORT_THREADS = 256;
static constexpr int SORT_ROUNDS = 16;
static constexpr int SORT_TILE = SORT_THREADS * SORT_ROUNDS;

// exclusive scan: 1024-thread CTAs, 4 elements per thread
static constexpr int SCAN_THREADS = 1024;
static constexpr int SCAN_ITEMS = 4;
static constexpr long long SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ void agent_keys_kernel(const float* __restrict__ pos, int A, int dims, int3 bmin, int3 vox, int3 grid,
								  unsigned int* __restrict__ keys, int* __restrict__ vals, unsigned int invalid_key,
								  int* err);
__global__ void __launch_bounds__(SORT_THREADS) radix_hist_kernel(const unsigned int* __restrict__ keys, int n, int shift, int* __restrict__ hist,
								  int tiles);
__global__ void __launch_bounds__(SORT_THREADS) radix_scatter_kernel(const unsigned int* __restrict__ keys_in, const int* __restrict__ vals_in,
									 unsigned int* __restrict__ keys_out, int* __restrict__ vals_out, int n, int shift,
									 const int* __restrict__ offsets, int tiles);
__global__ void seg_flags_kernel(const unsigned int* __restrict__ keys, int n, unsigned int invalid_key,
								 int* __restrict__ flags);
__global__ void seg_finish_kernel(const unsigned int* __restrict__ keys, const int* __restrict__ flags,
								  const int* __restrict__ seg_id, int n, unsigned int invalid_key,
								  int* __restrict__ seg_start, int* __restrict__ counts);
__global__ void intermediates_kernel(long long total, int S, const float* __restrict__ sec,
									 const float* __restrict__ sat, const float* __restrict__ upt,
									 const float* __restrict__ nex, const float* __restrict__ vol, float voxel_volume,
									 float dt, float* __restrict__ num, float* __restrict__ den, float* __restrict__ fac);
__global__ void reduce_kernel(long long total, int S, const int* __restrict__ counts,
							  const int* __restrict__ seg_start, const int* __restrict__ order,
							  const float* __restrict__ num, const float* __restrict__ den,
							  const float* __restrict__ fac, float* __restrict__ red_num, float* __restrict__ red_den,
							  float* __restrict__ red_fac);
__global__ void secrete_kernel(long long total, int S, float* __restrict__ dens, const int* __restrict__ counts,
							   const int* __restrict__ seg_start, const int* __restrict__ order,
							   const unsigned int* __restrict__ keys, const float* __restrict__ num,
							   const float* __restrict__ den, const float* __restrict__ fac,
							   const float* __restrict__ red_num, const float* __restrict__ red_den,
							   const float* __restrict__ red_fac, float* __restrict__ intern, int internalized,
							   float voxel_volume);

// One (voxel segment, substrate) pair of the secretion update; t < segments * S (secrete_kernel of
// cell.cu, and the ensemble update of batch_kernels.cu).  See cell.cu for the formulas.  SORTED:
// the per-agent rows num/den/fac/intern are in the binning's sorted order (row p is the agent at
// sorted position p), otherwise in agent order (row order[p]).
template <bool SORTED = false>
__device__ __forceinline__ void secrete_element(long long t, int S, float* __restrict__ dens,
												const int* __restrict__ counts, const int* __restrict__ seg_start,
												const int* __restrict__ order, const unsigned int* __restrict__ keys,
												const float* __restrict__ num, const float* __restrict__ den,
												const float* __restrict__ fac, const float* __restrict__ red_num,
												const float* __restrict__ red_den, const float* __restrict__ red_fac,
												float* __restrict__ intern, int internalized, float voxel_volume)
{
	const int seg = (int)(t / S);
	const int s = (int)(t % S);
	if (seg >= counts[0])
		return;
	const int b = seg_start[seg];
	const size_t dv = (size_t)keys[b] * S + s;
	const float D = dens[dv];
	const float rn = red_num[t], rd = red_den[t], rf = red_fac[t];

	if (internalized)
	{
		if (!counts[2])
		{
			// compute_fused: the voxel holds this one agent
			const size_t k = (size_t)(SORTED ? b : order[b]) * S + s;
			const float term = __fadd_rn(__fdiv_rn(__fadd_rn(__fmul_rn(__fsub_rn(1.f, rd), D), rn), rd), rf);
			intern[k] = __fsub_rn(intern[k], __fmul_rn(voxel_volume, term));
		}
		else
		{
			// compute_internalized for every agent of the voxel, with its own intermediates
			const int e = seg_start[seg + 1];
			for (int p = b; p < e; p++)
			{
				const size_t k = (size_t)(SORTED ? p : order[p]) * S + s;
				const float dk = den[k];
				const float term =
					__fadd_rn(__fdiv_rn(__fadd_rn(__fmul_rn(-dk, D), num[k]), __fadd_rn(1.f, dk)), fac[k]);
				intern[k] = __fsub_rn(intern[k], __fmul_rn(voxel_volume, term));
			}
		}
	}
	dens[dv] = __fadd_rn(__fdiv_rn(__fadd_rn(D, rn), rd), rf);
}

// The sorted update four substrates at a time (S % 4 == 0): thread t < segments * S / 4 owns a
// (segment, four substrates) pair and moves every row as 16-byte accesses (secrete_sorted4_kernel of
// cell.cu, and the ensemble update of batch_kernels.cu).  The arithmetic is secrete_element's, per
// substrate, in the same order.
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

__device__ __forceinline__ float fused_term(float D, float rn, float rd, float rf)
{
	return __fadd_rn(__fdiv_rn(__fadd_rn(__fmul_rn(__fsub_rn(1.f, rd), D), rn), rd), rf);
}

__device__ __forceinline__ float agent_term(float D, float num, float den, float fac)
{
	return __fadd_rn(__fdiv_rn(__fadd_rn(__fmul_rn(-den, D), num), __fadd_rn(1.f, den)), fac);
}

__device__ __forceinline__ void secrete_sorted4_element(long long t, int S, float* __restrict__ dens,
														const int* __restrict__ counts,
														const int* __restrict__ seg_start,
														const unsigned int* __restrict__ keys,
														const float* __restrict__ snum, const float* __restrict__ sden,
														const float* __restrict__ sfac, const float* __restrict__ red_num,
														const float* __restrict__ red_den,
														const float* __restrict__ red_fac, float* __restrict__ sintern,
														float voxel_volume)
{
	const int S4 = S >> 2;
	const int seg = (int)(t / S4);
	const int s0 = (int)(t - (long long)seg * S4) * 4;
	const int b = seg_start[seg];
	const size_t dv = (size_t)keys[b] * S + s0;
	const size_t r = (size_t)seg * S + s0;
	const float4 D = ld4(dens + dv);
	const float4 rn = ld4(red_num + r), rd = ld4(red_den + r), rf = ld4(red_fac + r);
	if (counts[2] == 0)
	{
		// compute_fused: the voxel holds this one agent
		float* ip = sintern + (size_t)b * S + s0;
		float4 I = ld4(ip);
		I.x = __fsub_rn(I.x, __fmul_rn(voxel_volume, fused_term(D.x, rn.x, rd.x, rf.x)));
		I.y = __fsub_rn(I.y, __fmul_rn(voxel_volume, fused_term(D.y, rn.y, rd.y, rf.y)));
		I.z = __fsub_rn(I.z, __fmul_rn(voxel_volume, fused_term(D.z, rn.z, rd.z, rf.z)));
		I.w = __fsub_rn(I.w, __fmul_rn(voxel_volume, fused_term(D.w, rn.w, rd.w, rf.w)));
		st4(ip, I);
	}
	else
	{
		// compute_internalized for every agent of the voxel, with its own intermediates
		const int e = seg_start[seg + 1];
		for (int p = b; p < e; p++)
		{
			const size_t k = (size_t)p * S + s0;
			const float4 nu = ld4(snum + k), de = ld4(sden + k), fa = ld4(sfac + k);
			float4 I = ld4(sintern + k);
			I.x = __fsub_rn(I.x, __fmul_rn(voxel_volume, agent_term(D.x, nu.x, de.x, fa.x)));
			I.y = __fsub_rn(I.y, __fmul_rn(voxel_volume, agent_term(D.y, nu.y, de.y, fa.y)));
			I.z = __fsub_rn(I.z, __fmul_rn(voxel_volume, agent_term(D.z, nu.z, de.z, fa.z)));
			I.w = __fsub_rn(I.w, __fmul_rn(voxel_volume, agent_term(D.w, nu.w, de.w, fa.w)));
			st4(sintern + k, I);
		}
	}
	st4(dens + dv, make_float4(__fadd_rn(__fdiv_rn(__fadd_rn(D.x, rn.x), rd.x), rf.x),
							   __fadd_rn(__fdiv_rn(__fadd_rn(D.y, rn.y), rd.y), rf.y),
							   __fadd_rn(__fdiv_rn(__fadd_rn(D.z, rn.z), rd.z), rf.z),
							   __fadd_rn(__fdiv_rn(__fadd_rn(D.w, rn.w), rd.w), rf.w)));
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_kernel(const int* in, int* out, long long n, int* tile_sums);
__global__ void scan_add_kernel(int* out, long long n, const int* tile_offsets);

// cell.cu: keys, sort, segments, intermediates, reductions; `sorted`: also the sorted copies of the
// per-agent terms (agent_state::snum ...), from which the reductions are then summed
int rebuild_bins(bfvm_solver* s, bool sorted = false);

// number of 8-bit radix passes for keys in [0, V] (V marks agents outside the mesh)
inline int sort_passes(long long V)
{
	int bits = 1;
	while (bits < 32 && ((1ull << bits) <= (unsigned long long)V))
		bits++;
	return (bits + 7) / 8;
}

} // namespace bfvm
