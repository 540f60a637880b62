// LOD diffusion-decay sweeps along x, y and z, with the Dirichlet overwrites fused into them.
//
// The reference step (paraBioFVM src/solver/host/diffusion_solver.cpp:512-544) is
//   Dirichlet, x sweep, Dirichlet, y sweep, Dirichlet, z sweep, Dirichlet.
// Each sweep kernel here applies the Dirichlet overwrite that precedes it while loading, and the
// last sweep also applies the final one while storing, so the field is read and written exactly
// once per sweep.
//
// Every line is split into P register blocks of at most M elements; one thread owns one block of
// one line.  A block runs the Thomas forward and backward recurrences on its registers, and the
// blocks of a line exchange one carry each way through shared memory (see precompute.cpp for
// the carry algebra).  With P == 1 the arithmetic is exactly the reference's Thomas solve.
//
// The only per-element coefficient is b'_i: e_{i-1} = c b'_{i-1} is recomputed with the same
// float product the reference stores, and the carry products are accumulated as running products
// of -c b'_i.  The kernels are persistent: each CTA stages the b' table of the axis in shared
// memory once and then loops over its share of the lines.
//
// Thread layouts (the field is [z][y][x][s], substrate fastest):
//   y and z sweeps ("columns"): a CTA owns 32 adjacent columns of the x*s (or y*x*s) plane and
//     all P blocks of their lines: blockDim = (32, P).  Warp w holds block w of 32 columns, so
//     every element step is one 128-byte coalesced load or store per warp.
//   x sweep ("rows"): lines are the S interleaved substrate lines of a row; thread t holds
//     substrate s = t % Sc of block j = (t / Sc) % P of row t / (Sc*P).  A warp touches S
//     consecutive floats of one or two blocks per element step.

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
	int X, Y, Z;
	dirichlet_dev dir;
	int pre_dirichlet;
	int post_dirichlet;
};

__device__ __forceinline__ float apply_dirichlet(const dirichlet_dev& d, float v, int x, int y, int z, int s, int S,
												 int X, int Y, int Z)
{
	// faces: x-min, x-max, y-min, y-max, z-min, z-max; the later write wins
	// (src/solver/host/dirichlet_solver.cpp:122-141)
	const int fm = d.face_mask;
	if (fm)
	{
		if ((fm & 1) && x == 0 && d.face_conds[0 * S + s])
			v = d.face_vals[0 * S + s];
		if ((fm & 2) && x == X - 1 && d.face_conds[1 * S + s])
			v = d.face_vals[1 * S + s];
		if ((fm & 4) && y == 0 && d.face_conds[2 * S + s])
			v = d.face_vals[2 * S + s];
		if ((fm & 8) && y == Y - 1 && d.face_conds[3 * S + s])
			v = d.face_vals[3 * S + s];
		if ((fm & 16) && z == 0 && d.face_conds[4 * S + s])
			v = d.face_vals[4 * S + s];
		if ((fm & 32) && z == Z - 1 && d.face_conds[5 * S + s])
			v = d.face_vals[5 * S + s];
	}
	// interior voxels last (dirichlet_solver.cpp:53-75)
	if (d.has_interior)
	{
		const long long vid = (long long)x + (long long)X * ((long long)y + (long long)Y * z);
		const unsigned int w = __ldg(&d.bits[vid >> 5]);
		const unsigned int b = (unsigned int)(vid & 31);
		if ((w >> b) & 1u)
		{
			const long long row = (long long)__ldg(&d.rank[vid >> 5]) + __popc(w & ((1u << b) - 1u));
			if (d.iconds[row * S + s])
				v = d.ivals[row * S + s];
		}
	}
	return v;
}

// The Dirichlet overwrite seen by one (line, substrate): faces of the other two axes cover a line
// either entirely or not at all, faces of the sweep axis touch only its first and last element, and
// interior voxels are looked up in the rank bitmap.  Resolved once per thread so the per-element
// cost is a select plus one bitmap probe.
struct line_dirichlet
{
	bool any;			 // anything to apply on this line
	bool line_face;		 // a face of another axis covers the line (after own faces in precedence)
	float line_val;
	bool own_min, own_max; // sweep-axis faces at element 0 / n-1 (already merged with line faces)
	float min_val, max_val;
	long long base_vid, vid_stride;
	int n;

	template <int AXIS>
	__device__ __forceinline__ void init(const dirichlet_dev& d, int i0, int i1, int s, int S, int X, int Y, int Z,
										 int n_)
	{
		// (i0, i1) are the line's fixed coordinates: AXIS 0 -> (y, z); 1 -> (x, z); 2 -> (x, y)
		n = n_;
		const int cx = AXIS == 0 ? 0 : i0;
		const int cy = AXIS == 0 ? i0 : (AXIS == 1 ? 0 : i1);
		const int cz = AXIS == 2 ? 0 : i1;
		// last applicable face of another axis, in precedence order x-min .. z-max
		int order = -1;
		line_val = 0.f;
#pragma unroll
		for (int f = 0; f < 6; f++)
		{
			const int ax = f >> 1;
			if (ax == AXIS || !(d.face_mask & (1 << f)))
				continue;
			const int c = ax == 0 ? cx : (ax == 1 ? cy : cz);
			const int e = ax == 0 ? X : (ax == 1 ? Y : Z);
			const bool on = (f & 1) ? c == e - 1 : c == 0;
			if (on && d.face_conds[f * S + s])
			{
				order = f;
				line_val = d.face_vals[f * S + s];
			}
		}
		line_face = order >= 0;
		// own-axis faces apply only where they come later than the covering face
		const int fmin = 2 * AXIS, fmax = 2 * AXIS + 1;
		own_min = (d.face_mask & (1 << fmin)) && d.face_conds[fmin * S + s];
		own_max = (d.face_mask & (1 << fmax)) && d.face_conds[fmax * S + s];
		min_val = own_min ? d.face_vals[fmin * S + s] : 0.f;
		max_val = own_max ? d.face_vals[fmax * S + s] : 0.f;
		if (n == 1)
		{
			// one voxel along the axis: min and max face hit the same element, max written last
			if (own_max)
				min_val = max_val;
			own_min = own_min || own_max;
			own_max = false;
		}
		if (line_face)
		{
			if (order > fmin)
			{
				own_min = true;
				min_val = line_val;
			}
			if (order > fmax && n > 1)
			{
				own_max = true;
				max_val = line_val;
			}
		}
		if (AXIS == 0)
		{
			vid_stride = 1;
			base_vid = (long long)X * ((long long)cy + (long long)Y * cz);
		}
		else if (AXIS == 1)
		{
			vid_stride = X;
			base_vid = (long long)cx + (long long)X * Y * cz;
		}
		else
		{
			vid_stride = (long long)X * Y;
			base_vid = (long long)cx + (long long)X * cy;
		}
		any = line_face || own_min || own_max || d.has_interior;
	}

	__device__ __forceinline__ float apply(const dirichlet_dev& d, int i, int s, int S, float v) const
	{
		if (line_face)
			v = line_val;
		if (i == 0 && own_min)
			v = min_val;
		if (i == n - 1 && own_max)
			v = max_val;
		if (d.has_interior)
		{
			const long long vid = base_vid + (long long)i * vid_stride;
			const unsigned int w = __ldg(&d.bits[vid >> 5]);
			const unsigned int b = (unsigned int)(vid & 31);
			if ((w >> b) & 1u)
			{
				const long long row = (long long)__ldg(&d.rank[vid >> 5]) + __popc(w & ((1u << b) - 1u));
				if (d.iconds[row * S + s])
					v = d.ivals[row * S + s];
			}
		}
		return v;
	}
};

__device__ __forceinline__ void block_range(int j, int base_len, int extra, int& p, int& L)
{
	p = j * base_len + min(j, extra);
	L = base_len + (j < extra ? 1 : 0);
}

// Solve block j of one line.  `line` points at element 0 of the line, `stride` is the element
// stride in floats.  `bp` is the b' column of this line's substrate (bp[i * bstride]).
// carry_f / carry_t hold one value per block of this line at index k*cstride.  All threads of the
// CTA must call this (it contains __syncthreads).
template <int M>
__device__ __forceinline__ void solve_block(const sweep_args& a, float* __restrict__ line, long long stride,
											const float* bp, const float* gq, const float* Gp, int bstride, float cs,
											int s, int j, bool active, float* carry_f, float* carry_t, int cstride,
											const line_dirichlet& ld)
{
	const int S = a.S;
	int p, L;
	block_range(j, a.base_len, a.extra, p, L);

	float d[M];
	{
		// running pointers keep one address live instead of M
		const float* ptr = line + (long long)p * stride;
#pragma unroll
		for (int k = 0; k < M; k++)
		{
			d[k] = (active && k < L) ? *ptr : 0.f;
			ptr += stride;
		}
	}
	if (a.pre_dirichlet && active && ld.any)
	{
#pragma unroll
		for (int k = 0; k < M; k++)
			if (k < L)
				d[k] = ld.apply(a.dir, p + k, s, S, d[k]);
	}

	// forward elimination from a zero carry: f_i = d_i - e_{i-1} f_{i-1},  e_{i-1} = c b'_{i-1}
#pragma unroll
	for (int k = 1; k < M; k++)
		if (active && k < L)
			d[k] = __fsub_rn(d[k], __fmul_rn(__fmul_rn(cs, bp[(p + k - 1) * bstride]), d[k - 1]));

	if (active)
	{
#pragma unroll
		for (int k = 0; k < M; k++)
			if (k == L - 1)
				carry_f[j * cstride] = d[k];
	}
	__syncthreads();

	if (active && j > 0)
	{
		// d'_{p-1} = C_{j-1}: fold the blocks to the left, C_k = f^k_q + g^k_q C_{k-1}, where
		// g^k_q = prod_{i=p_k-1}^{q_k-1} (-c b'_i)
		float C = carry_f[0];
		for (int k = 1; k < j; k++)
			C = fmaf(gq[k * bstride], C, carry_f[k * cstride]);
		// d'_i = f_i + g_i C with the running product g_i = prod_{m=p-1}^{i-1} (-c b'_m)
		float g = 1.f;
#pragma unroll
		for (int k = 0; k < M; k++)
			if (k < L)
			{
				g = __fmul_rn(g, -__fmul_rn(cs, bp[(p + k - 1) * bstride]));
				d[k] = fmaf(g, C, d[k]);
			}
	}

	// backward substitution from a zero carry: t_q = d'_q b'_q, t_i = (d'_i - c t_{i+1}) b'_i
#pragma unroll
	for (int k = M - 1; k >= 0; k--)
	{
		if (active && k < L)
		{
			const float bpk = bp[(p + k) * bstride];
			if (k == L - 1)
				d[k] = __fmul_rn(d[k], bpk);
			else
				d[k] = __fmul_rn(__fsub_rn(d[k], __fmul_rn(cs, d[k + 1 < M ? k + 1 : k])), bpk);
		}
	}

	if (active)
		carry_t[j * cstride] = d[0];
	__syncthreads();

	if (active && j < a.P - 1)
	{
		// x_{q+1} = X_{j+1}: fold the blocks to the right, X_k = t^k_p + G^k_p X_{k+1}, where
		// G^k_p = prod_{i=p_k}^{q_k} (-c b'_i)
		float Xc = carry_t[(a.P - 1) * cstride];
		for (int k = a.P - 2; k > j; k--)
			Xc = fmaf(Gp[k * bstride], Xc, carry_t[k * cstride]);
		// x_i = t_i + G_i X with the running product G_i = prod_{m=i}^{q} (-c b'_m)
		float G = 1.f;
#pragma unroll
		for (int k = M - 1; k >= 0; k--)
			if (k < L)
			{
				G = __fmul_rn(G, -__fmul_rn(cs, bp[(p + k) * bstride]));
				d[k] = fmaf(G, Xc, d[k]);
			}
	}

	if (a.post_dirichlet && active && ld.any)
	{
#pragma unroll
		for (int k = 0; k < M; k++)
			if (k < L)
				d[k] = ld.apply(a.dir, p + k, s, S, d[k]);
	}
	{
		float* ptr = line + (long long)(p + L - 1) * stride;
#pragma unroll
		for (int k = M - 1; k >= 0; k--)
			if (active && k < L)
			{
				*ptr = d[k];
				ptr -= stride;
			}
	}
}

// Stage the coefficients of substrates s0 .. s0+Sc-1 into shared memory: b' [n][Sc], c [Sc],
// gq [P][Sc], Gp [P][Sc] (consecutive in `tab`).
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

// y (AXIS 1) and z (AXIS 2) sweeps.  Work item w = outer * col_tiles + tile; the grid strides over
// items.  MAXT bounds the CTA size (32 * P) so the register budget follows the block count.
// Shared memory: b' table [n][S], c [S], carries [2][P][32].
template <int M, int AXIS, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
	sweep_columns(const __grid_constant__ sweep_args a, long long ncols, long long col_tiles, long long items,
				  long long outer_stride, long long line_stride)
{
	extern __shared__ float sh[];
	float* tab = sh;
	const float* ctab = tab + a.n * a.S;
	const float* gtab = ctab + a.S;
	const float* Gtab = gtab + a.P * a.S;
	float* carry_f = tab + table_floats(a.n, a.P, a.S);
	float* carry_t = carry_f + a.P * 32;
	stage_table(a, tab, 0, a.S);

	const int lane = threadIdx.x;
	const int j = threadIdx.y;
	const int S = a.S;
	for (long long w = blockIdx.x; w < items; w += gridDim.x)
	{
		const long long outer = w / col_tiles;
		const long long tile = w % col_tiles;
		const long long q = tile * 32 + lane;
		const bool active = q < ncols;
		const long long qq = active ? q : 0;
		const int s = (int)(qq % S);
		line_dirichlet ld;
		ld.any = false;
		if (a.pre_dirichlet)
		{
			if (AXIS == 1)
				ld.init<1>(a.dir, (int)(qq / S), (int)outer, s, S, a.X, a.Y, a.Z, a.n);
			else
			{
				const long long XS = (long long)a.X * S;
				ld.init<2>(a.dir, (int)((qq % XS) / S), (int)(qq / XS), s, S, a.X, a.Y, a.Z, a.n);
			}
		}
		float* line = a.data + outer * outer_stride + qq;
		solve_block<M>(a, line, line_stride, tab + s, gtab + s, Gtab + s, S, ctab[s], s, j, active, carry_f + lane,
					   carry_t + lane, 32, ld);
	}
}

// x sweep.  Work item = a group of rows_per_cta rows (blockIdx.y = substrate chunk of Sc lines);
// thread t holds substrate s0 + t % Sc, block (t / Sc) % P of row t / (Sc*P) of the group.
// Shared memory: b' table [n][Sc], c [Sc], carries [2][rows][P][Sc].
template <int M, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
	sweep_rows(const __grid_constant__ sweep_args a, long long nrows, int rows_per_cta, int Sc, long long groups)
{
	extern __shared__ float sh[];
	const int s0 = blockIdx.y * Sc;
	float* tab = sh;
	const float* ctab = tab + a.n * Sc;
	const float* gtab = ctab + Sc;
	const float* Gtab = gtab + a.P * Sc;
	float* carries = tab + table_floats(a.n, a.P, Sc);
	stage_table(a, tab, s0, Sc);

	const int t = threadIdx.x;
	const int P = a.P;
	const int sl = t % Sc;
	const int j = (t / Sc) % P;
	const int rl = t / (Sc * P);
	const int s = s0 + sl;
	float* carry_f = carries + (size_t)rl * P * Sc + sl;
	float* carry_t = carries + (size_t)rows_per_cta * P * Sc + (size_t)rl * P * Sc + sl;
	for (long long gi = blockIdx.x; gi < groups; gi += gridDim.x)
	{
		const long long r = gi * rows_per_cta + rl;
		const bool active = rl < rows_per_cta && r < nrows && s < a.S;
		const long long rr = active ? r : 0;
		const int ss = active ? s : 0;
		line_dirichlet ld;
		ld.any = false;
		if (a.pre_dirichlet)
			ld.init<0>(a.dir, (int)(rr % a.Y), (int)(rr / a.Y), ss, a.S, a.X, a.Y, a.Z, a.n);
		float* line = a.data + rr * (long long)a.X * a.S + ss;
		solve_block<M>(a, line, a.S, tab + sl, gtab + sl, Gtab + sl, Sc, ctab[sl], ss, j, active, carry_f, carry_t, Sc,
					   ld);
	}
}

static int sm_count(int device)
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
static int persistent_grid(K kernel, int threads, size_t smem, long long items, int device)
{
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
	if (per_sm <= 0)
		per_sm = 1;
	const long long g = (long long)per_sm * sm_count(device);
	return (int)std::max<long long>(1, std::min<long long>(g, items));
}

template <typename K>
static int set_smem(K kernel, size_t smem)
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

template <int M, int AXIS, int MAXT, int MINB>
static int launch_columns(bfvm_solver* st, const sweep_args& a)
{
	const long long X = st->grid[0], Y = st->grid[1], Z = st->grid[2], S = st->S;
	const long long ncols = AXIS == 1 ? X * S : Y * X * S;
	const long long tiles = (ncols + 31) / 32;
	const long long outers = AXIS == 1 ? Z : 1;
	const long long items = outers * tiles;
	const size_t smem = ((size_t)table_floats(a.n, a.P, (int)S) + 2 * (size_t)a.P * 32) * sizeof(float);
	auto kernel = sweep_columns<M, AXIS, MAXT, MINB>;
	int rc = set_smem(kernel, smem);
	if (rc)
		return rc;
	dim3 block(32, a.P);
	const int grid = persistent_grid(kernel, 32 * a.P, smem, items, st->device);
	kernel<<<grid, block, smem, st->stream>>>(a, ncols, tiles, items, AXIS == 1 ? Y * X * S : 0,
											  AXIS == 1 ? X * S : Y * X * S);
	return check_launch(st, AXIS == 1 ? "sweep_columns<y>" : "sweep_columns<z>");
}

template <int M>
static int launch_sweep_m(bfvm_solver* st, int axis, const sweep_args& a)
{
	const long long Y = st->grid[1], Z = st->grid[2], S = st->S;
	if (axis == 0)
	{
		const long long nrows = Y * Z;
		const int Sc = (int)std::min<long long>(S, std::max(1, 512 / a.P));
		const int per_row = Sc * a.P;
		// prefer CTAs of at most 320 threads (two resident per SM), else up to 512
		const int cap = per_row <= 320 ? 320 : 512;
		const int rows_per_cta = (int)std::min<long long>(std::max(1, cap / per_row), nrows);
		const int threads = rows_per_cta * per_row;
		const long long groups = (nrows + rows_per_cta - 1) / rows_per_cta;
		const int chunks = (int)((S + Sc - 1) / Sc);
		const size_t smem = ((size_t)table_floats(a.n, a.P, Sc) + 2 * (size_t)rows_per_cta * a.P * Sc) * sizeof(float);
		auto kernel = threads <= 320 ? sweep_rows<M, 320, 2> : sweep_rows<M, 512, 1>;
		int rc = set_smem(kernel, smem);
		if (rc)
			return rc;
		const int gx = persistent_grid(kernel, threads, smem, groups * chunks, st->device);
		dim3 grid((unsigned)std::max(1, (int)std::min<long long>(groups, (gx + chunks - 1) / chunks)), (unsigned)chunks);
		kernel<<<grid, threads, smem, st->stream>>>(a, nrows, rows_per_cta, Sc, groups);
		return check_launch(st, "sweep_rows");
	}
	const int threads = 32 * a.P;
	if (axis == 1)
		return threads <= 320 ? launch_columns<M, 1, 320, 2>(st, a)
							  : (threads <= 512 ? launch_columns<M, 1, 512, 1>(st, a) : launch_columns<M, 1, 1024, 1>(st, a));
	return threads <= 320 ? launch_columns<M, 2, 320, 2>(st, a)
						  : (threads <= 512 ? launch_columns<M, 2, 512, 1>(st, a) : launch_columns<M, 2, 1024, 1>(st, a));
}

int launch_sweep(bfvm_solver* st, int axis, bool final_dirichlet)
{
	const sweep_plan& pl = st->plan[axis];
	sweep_args a;
	a.data = st->dens;
	a.bp = pl.bp;
	a.c = pl.c;
	a.gq = pl.gq;
	a.Gp = pl.Gp;
	a.n = pl.n;
	a.P = pl.P;
	a.base_len = pl.base_len;
	a.extra = pl.extra;
	a.S = st->S;
	a.X = st->grid[0];
	a.Y = st->grid[1];
	a.Z = st->grid[2];
	a.dir = st->dirichlet();
	a.pre_dirichlet = (a.dir.face_mask != 0 || a.dir.has_interior) ? 1 : 0;
	a.post_dirichlet = final_dirichlet ? a.pre_dirichlet : 0;
	if (pl.M == 32)
		return launch_sweep_m<32>(st, axis, a);
	return launch_sweep_m<64>(st, axis, a);
}

// ------------------------------------------------------------------------------------------------
// standalone Dirichlet overwrite (dirichlet_solver::solve): one thread per field element

__global__ void dirichlet_kernel(float* __restrict__ data, long long total, int S, int X, int Y, int Z,
								 dirichlet_dev dir)
{
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= total)
		return;
	const int s = (int)(i % S);
	const long long v = i / S;
	const int x = (int)(v % X);
	const int y = (int)((v / X) % Y);
	const int z = (int)(v / ((long long)X * Y));
	const float old = data[i];
	const float nv = apply_dirichlet(dir, old, x, y, z, s, S, X, Y, Z);
	if (__float_as_uint(nv) != __float_as_uint(old))
		data[i] = nv;
}

int launch_dirichlet(bfvm_solver* st)
{
	dirichlet_dev d = st->dirichlet();
	if (!d.face_mask && !d.has_interior)
		return BFVM_OK;
	const long long total = st->V * st->S;
	const int threads = 256;
	dirichlet_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, st->stream>>>(
		st->dens, total, st->S, st->grid[0], st->grid[1], st->grid[2], d);
	return check_launch(st, "dirichlet_kernel");
}

} // namespace bfvm
