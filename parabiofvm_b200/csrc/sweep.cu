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

#include "sweep_common.cuh"

namespace bfvm {

int sm_count(int device) { return sm_count_impl(device); }

// Solve block j of one line read from and written to global memory.  `line` points at element 0
// of the line, `stride` is its element stride in floats.
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
		dirichlet_block<M, false>(ld, a.dir, d, p, L, s, S);

	thomas_block<M, false>(d, L, p, j, a.P, bp, gq, Gp, bstride, cs, active, carry_f, carry_t, cstride);

	if (a.post_dirichlet && active && ld.any)
		dirichlet_block<M, false>(ld, a.dir, d, p, L, s, S);
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
	float* fvals = const_cast<float*>(Gtab) + a.P * a.S;
	unsigned char* fconds = reinterpret_cast<unsigned char*>(fvals + 6 * a.S);
	float* carry_f = tab + table_floats(a.n, a.P, a.S, a.S);
	float* carry_t = carry_f + a.P * 32;
	stage_faces(a, fvals, fconds);
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
			{
				const int x = (int)(qq / S);
				ld.init<1>(a.dir, fvals, fconds, x, (int)outer, s, S, a.X, a.Y, a.Z, a.n);
				ld.load_mask<1>(a.dir, x + (long long)a.X * outer, j, a.P);
			}
			else
			{
				const long long XS = (long long)a.X * S;
				const int x = (int)((qq % XS) / S), y = (int)(qq / XS);
				ld.init<2>(a.dir, fvals, fconds, x, y, s, S, a.X, a.Y, a.Z, a.n);
				ld.load_mask<2>(a.dir, x + (long long)a.X * y, j, a.P);
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
	float* fvals = const_cast<float*>(Gtab) + a.P * Sc;
	unsigned char* fconds = reinterpret_cast<unsigned char*>(fvals + 6 * a.S);
	float* carries = tab + table_floats(a.n, a.P, Sc, a.S);
	stage_faces(a, fvals, fconds);
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
		{
			ld.init<0>(a.dir, fvals, fconds, (int)(rr % a.Y), (int)(rr / a.Y), ss, a.S, a.X, a.Y, a.Z, a.n);
			ld.load_mask<0>(a.dir, rr, j, a.P);
		}
		float* line = a.data + rr * (long long)a.X * a.S + ss;
		solve_block<M>(a, line, a.S, tab + sl, gtab + sl, Gtab + sl, Sc, ctab[sl], ss, j, active, carry_f, carry_t, Sc,
					   ld);
	}
}

template <int M, int AXIS, int MAXT, int MINB>
static int launch_columns(bfvm_solver* st, const sweep_args& a)
{
	const long long X = st->grid[0], Y = st->grid[1], Z = st->grid[2], S = st->S;
	const long long ncols = AXIS == 1 ? X * S : Y * X * S;
	const long long tiles = (ncols + 31) / 32;
	const long long outers = AXIS == 1 ? Z : 1;
	const long long items = outers * tiles;
	const size_t smem = ((size_t)table_floats(a.n, a.P, (int)S, (int)S) + 2 * (size_t)a.P * 32) * sizeof(float);
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
		const size_t smem =
			((size_t)table_floats(a.n, a.P, Sc, (int)S) + 2 * (size_t)rows_per_cta * a.P * Sc) * sizeof(float);
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
	a.err = st->dev_error;
	if (st->use_tma)
	{
		bool handled = false;
		int rc = launch_sweep_tma(st, axis, a, handled);
		if (rc || handled)
			return rc;
	}
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
