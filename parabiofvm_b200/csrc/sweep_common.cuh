// Pieces shared by the sweep kernels: arguments, the block partition, the block-level Thomas
// solve and the staging of the coefficient tables in shared memory.
#pragma once

#include <algorithm>
#include <string>

#include "bfvm_internal.h"

namespace bfvm {

struct sweep_args
{
	float* data;
	const float* bp; // [n][S] in global memory; staged into shared memory by the kernels
	const float* c;	 // [S]
	const float* gq; // [P][S] whole-block forward carry products
	const float* Gp; // [P][S] whole-block backward carry products
	int n, P, base_len, extra, S;
	const float* vtab; // front-padded tables of the staged sweeps (precompute_padded)
	int vP, pad;
	int X, Y, Z;
	int* err; // device error flags (DEVERR_*)
	// the solve pass of a z-slab (sweep_tma.cu): per-line carries in [2][slab_lines] (C, X); null
	// for every other sweep
	const float* slab_carry;
	long long slab_lines;
	// staged sweeps (sweep_tma.cu): the bound of every wait on a tile copy, in clock64 cycles; and,
	// for tests of that bound only, a tile whose stage barrier is armed but whose copies are never
	// issued (-1: none), so that the wait on it runs out
	long long wait_limit;
	long long drop_tile_copy;
	// staged sweeps of the LOD step: the Dirichlet overwrite that follows this sweep, grouped by its
	// tiles; each tile's entries are written right after the tile (items 0: no overwrite here)
	dirichlet_tiles dir;
	// staged sweeps of the LOD step: nonzero to write the Dirichlet face conditions by position into
	// the stored values (the faces of the overwrite after this sweep).  face_bits [S], face_vals
	// [6][S], face_tiles: per tile, whether a line of the tile lies on a face of another axis
	int face_apply;
	const int* face_bits;
	const float* face_vals;
	const unsigned char* face_tiles;
};

__device__ __forceinline__ void block_range(int j, int base_len, int extra, int& p, int& L)
{
	p = j * base_len + min(j, extra);
	L = base_len + (j < extra ? 1 : 0);
}

// Thomas solve of one register block of a line with carries exchanged through shared memory.
// `bp` points at b'_0 of this line's substrate with element stride `bstride`; gq / Gp hold the
// whole-block carry products with the same stride; carry_f / carry_t hold one value per block
// of this line at index k * cstride.  UNI: every block of the line has exactly M elements.  All
// threads of the CTA must call it (two __syncthreads).
template <int M, bool UNI>
__device__ __forceinline__ void thomas_block(float (&d)[M], int L, int p, int j, int P, const float* bp,
											 const float* gq, const float* Gp, int bstride, float cs, bool active,
											 float* carry_f, float* carry_t, int cstride)
{
	// forward elimination from a zero carry: f_i = d_i - e_{i-1} f_{i-1},  e_{i-1} = c b'_{i-1}
	// (the float product the reference stores as e)
#pragma unroll
	for (int k = 1; k < M; k++)
		if (UNI || k < L)
			d[k] = __fsub_rn(d[k], __fmul_rn(__fmul_rn(cs, bp[(p + k - 1) * bstride]), d[k - 1]));

	if (active)
	{
		if (UNI)
			carry_f[j * cstride] = d[M - 1];
		else
		{
#pragma unroll
			for (int k = 0; k < M; k++)
				if (k == L - 1)
					carry_f[j * cstride] = d[k];
		}
	}
	__syncthreads();

	if (active && j > 0)
	{
		// d'_{p-1} = C_{j-1}: fold the blocks to the left, C_k = f^k_q + gq_k C_{k-1}
		float C = carry_f[0];
		for (int k = 1; k < j; k++)
			C = fmaf(gq[k * bstride], C, carry_f[k * cstride]);
		// d'_i = f_i + g_i C with the running product g_i = prod_{m=p-1}^{i-1} (-c b'_m)
		float g = 1.f;
#pragma unroll
		for (int k = 0; k < M; k++)
			if (UNI || k < L)
			{
				g = __fmul_rn(g, -__fmul_rn(cs, bp[(p + k - 1) * bstride]));
				d[k] = fmaf(g, C, d[k]);
			}
	}

	// backward substitution from a zero carry: t_q = d'_q b'_q, t_i = (d'_i - c t_{i+1}) b'_i
#pragma unroll
	for (int k = M - 1; k >= 0; k--)
	{
		if (UNI || k < L)
		{
			const float bpk = bp[(p + k) * bstride];
			if (UNI ? (k == M - 1) : (k == L - 1))
				d[k] = __fmul_rn(d[k], bpk);
			else
				d[k] = __fmul_rn(__fsub_rn(d[k], __fmul_rn(cs, d[k + 1 < M ? k + 1 : k])), bpk);
		}
	}

	if (active)
		carry_t[j * cstride] = d[0];
	__syncthreads();

	if (active && j < P - 1)
	{
		// x_{q+1} = X_{j+1}: fold the blocks to the right, X_k = t^k_p + Gp_k X_{k+1}
		float Xc = carry_t[(P - 1) * cstride];
		for (int k = P - 2; k > j; k--)
			Xc = fmaf(Gp[k * bstride], Xc, carry_t[k * cstride]);
		// x_i = t_i + G_i X with the running product G_i = prod_{m=i}^{q} (-c b'_m)
		float G = 1.f;
#pragma unroll
		for (int k = M - 1; k >= 0; k--)
			if (UNI || k < L)
			{
				G = __fmul_rn(G, -__fmul_rn(cs, bp[(p + k) * bstride]));
				d[k] = fmaf(G, Xc, d[k]);
			}
	}
}

// Stage the coefficients of substrates s0 .. s0+Sc-1 into shared memory: b' [n][Sc], c [Sc],
// gq [P][Sc], Gp [P][Sc] (consecutive in `tab`).  Ends with __syncthreads.
__device__ __forceinline__ void stage_table(const sweep_args& a, float* tab, int s0, int Sc)
{
	const int nt = blockDim.x * blockDim.y;
	const int t0 = threadIdx.x + threadIdx.y * blockDim.x;
	for (int t = t0; t < a.n * Sc; t += nt)
	{
		const int i = t / Sc, sl = t % Sc;
		tab[t] = (s0 + sl < a.S) ? a.bp[(size_t)i * a.S + s0 + sl] : 0.f;
	}
	float* ctab = tab + a.n * Sc;
	for (int t = t0; t < Sc; t += nt)
		ctab[t] = (s0 + t < a.S) ? a.c[s0 + t] : 0.f;
	float* gtab = ctab + Sc;
	float* Gtab = gtab + a.P * Sc;
	for (int t = t0; t < a.P * Sc; t += nt)
	{
		const int k = t / Sc, sl = t % Sc;
		const bool ok = s0 + sl < a.S;
		gtab[t] = ok ? a.gq[(size_t)k * a.S + s0 + sl] : 0.f;
		Gtab[t] = ok ? a.Gp[(size_t)k * a.S + s0 + sl] : 0.f;
	}
	__syncthreads();
}

__host__ __device__ __forceinline__ int table_floats(int n, int P, int Sc) { return n * Sc + Sc + 2 * P * Sc; }

// host helpers for persistent launches
inline int sm_count_impl(int device)
{
	static int cached[64] = { 0 };
	if (device >= 0 && device < 64 && cached[device])
		return cached[device];
	int n = 0;
	cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
	if (n <= 0)
		n = 148;
	if (device >= 0 && device < 64)
		cached[device] = n;
	return n;
}

template <typename K>
inline int persistent_grid(K kernel, int threads, size_t smem, long long items, int device)
{
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
	if (per_sm <= 0)
		per_sm = 1;
	const long long g = (long long)per_sm * sm_count_impl(device);
	return (int)std::max<long long>(1, std::min<long long>(g, items));
}

template <typename K>
inline int set_smem(K kernel, size_t smem)
{
	int dev = 0, optin = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
	if (optin > 0 && smem > (size_t)optin)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "axis length x substrates too large for the staged coefficient table ("
												   + std::to_string(smem) + " bytes of shared memory)");
	if (smem > 48 * 1024)
	{
		cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess)
			return cuda_fail(e, "cudaFuncSetAttribute(max dynamic shared memory)");
	}
	return BFVM_OK;
}

// The gradient computed inside the z sweep of the step (sweep_tma.cu).  Tile w's final values (its
// stores and the Dirichlet entries written after them) are published in tile_done[w]; the group
// that swept tile w then computes the gradient of tile w - lag from the field, whose planes are
// still in L2, once the tiles holding that tile's x and y neighbours are published.  A group that
// finds a neighbour unpublished after spin_limit cycles leaves the tile to grad_deferred_kernel,
// which runs after the sweep (deferred[0] counts the tiles, deferred[1 ...] lists them).
struct grad_fuse
{
	float* g;		 // [3][Z][Y][X][S]
	int* tile_done;	 // [z tiles], zero before the sweep
	int* deferred;	 // [1 + z tiles], deferred[0] zero before the sweep
	long long lag;	 // in tiles
	long long total; // V * S
	int X, Y, Z, S;
	float bx, cx, by, cy, bz, cz;
	long long spin_limit;
};

// Chunks of the lines along an axis (a line longer than the staged sweep takes, cut into chunks
// that it does take), swept in one launch: chunk k holds elements [e0[k], e0[k] + len) of every
// line, with its tables vtab[k] (precompute_padded_range; every chunk of a launch has the same
// length, so the same blocks and front), and the carries that enter each line, carry[k][2][lines]
// (C, X), indexed by line: x, row * S + s; y, z * X * S + column; z, column of the y*x*s plane.
struct line_chunks
{
	int count = 0;
	long long e0[8] = {};
	long long len = 0;
	const float* vtab[8] = {};
	int vP = 1, pad = 0;
	const float* carry = nullptr;
	long long lines = 0;
};

// slab_solve (z axis only): the solve pass of a z-slab's sweep.  gf (z axis only): compute the
// gradient inside the sweep; `handled` then also means the gradient is (being) computed.
// [w_begin, w_end): sweep only these tiles (w_end -1: to the last tile; not with gf or slab_solve).
// The launch shape is the one chosen for the whole field.  chunks: sweep these chunks of every line
// (their solve pass, entering each line with the chunk's carries).
int launch_sweep_tma(bfvm_solver* st, int axis, const sweep_args& a, bool& handled,
					 const sweep_tuning* tune = nullptr, std::vector<sweep_tuning>* shapes = nullptr,
					 bool slab_solve = false, const grad_fuse* gf = nullptr, long long w_begin = 0,
					 long long w_end = -1, const line_chunks* chunk = nullptr);

// The tiles of the staged sweep along `axis` (sweep_tma.cu and the Dirichlet tile lists): x,
// R = 32 / S whole rows; y, 32 columns of the x*s plane of one z plane; z, 32 columns of the y*x*s
// plane.  items is 0 when the staged sweep cannot take the axis.
struct staged_tiling
{
	int axis = 0;
	long long XS = 0, YXS = 0, R = 1, col_tiles = 0, items = 0;

	long long tile(long long e) const
	{
		if (axis == 0)
			return (e / XS) / R;
		if (axis == 1)
			return (e / YXS) * col_tiles + (e % XS) / 32;
		return (e % YXS) / 32;
	}
};

staged_tiling staged_tiles(const bfvm_solver* s, int axis);

} // namespace bfvm
