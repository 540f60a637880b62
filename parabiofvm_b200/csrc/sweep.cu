// LOD diffusion-decay sweeps along x, y and z (paraBioFVM src/solver/host/diffusion_solver.cpp:
// 297-544).  The reference step is
//   Dirichlet, x sweep, Dirichlet, y sweep, Dirichlet, z sweep, Dirichlet;
// the sweeps here are pure line solves and the overwrites run as the scatter kernel of
// dirichlet.cu at the same four points, touching only the conditioned elements.
//
// Every line is split into P register blocks of at most M elements; one thread owns one block of
// one line.  A block runs the Thomas forward and backward recurrences on its registers, and the
// blocks of a line exchange one carry each way through shared memory (see precompute.cpp for
// the carry algebra).  With P == 1 the arithmetic is exactly the reference's Thomas solve.
// The only per-element coefficient is b'_i: e_{i-1} = c b'_{i-1} is recomputed with the same
// float product the reference stores, and the carry products are accumulated as running products
// of -c b'_i.
//
// Two implementations: sweep_tma.cu stages tiles of 32 lines through shared memory with the
// TMA (used whenever the shape allows); the kernels in this file read and write the field
// directly and cover every other shape:
//   y and z sweeps ("columns"): a CTA owns 32 adjacent columns of the x*s (or y*x*s) plane and
//     all P blocks of their lines: blockDim = (32, P); warp j holds block j of 32 columns, so every
//     element step is one 128-byte coalesced access per warp.
//   x sweep ("rows"): lines are the S interleaved substrate lines of a row; thread t holds
//     substrate s = t % Sc of block j = (t / Sc) % P of row t / (Sc*P).

#include "ensemble.h"
#include "sweep_common.cuh"

namespace bfvm {

// Solve block j of one line read from and written to global memory.  `line` points at element 0
// of the line, `stride` is its element stride in floats.
template <int M>
__device__ __forceinline__ void solve_block(const sweep_args& a, float* __restrict__ line, long long stride,
											const float* bp, const float* gq, const float* Gp, int bstride, float cs,
											int j, bool active, float* carry_f, float* carry_t, int cstride)
{
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

	thomas_block<M, false>(d, L, p, j, a.P, bp, gq, Gp, bstride, cs, active, carry_f, carry_t, cstride);

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
// Shared memory: coefficient tables, carries [2][P][32].
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
		const long long q = (w % col_tiles) * 32 + lane;
		const bool active = q < ncols;
		const long long qq = active ? q : 0;
		const int s = (int)(qq % S);
		float* line = a.data + outer * outer_stride + qq;
		solve_block<M>(a, line, line_stride, tab + s, gtab + s, Gtab + s, S, ctab[s], j, active, carry_f + lane,
					   carry_t + lane, 32);
	}
}

// x sweep.  Work item = a group of rows_per_cta rows (blockIdx.y = substrate chunk of Sc lines);
// thread t holds substrate s0 + t % Sc, block (t / Sc) % P of row t / (Sc*P) of the group.
// Shared memory: coefficient tables of the chunk, carries [2][rows][P][Sc].
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
		float* line = a.data + rr * (long long)a.X * a.S + ss;
		solve_block<M>(a, line, a.S, tab + sl, gtab + sl, Gtab + sl, Sc, ctab[sl], j, active, carry_f, carry_t, Sc);
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

static sweep_args make_args(bfvm_solver* st, int axis)
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
	a.vtab = pl.vtab;
	a.vP = pl.vP;
	a.pad = pl.pad;
	a.S = st->S;
	a.X = st->grid[0];
	a.Y = st->grid[1];
	a.Z = st->grid[2];
	a.err = st->dev_error;
	a.slab_carry = nullptr;
	a.slab_lines = 0;
	a.wait_limit = st->wait_limit_cycles;
	a.drop_tile_copy = st->drop_tile_copy;
	a.dir = dirichlet_tiles();
	a.face_apply = 0;
	a.face_bits = st->face_bits;
	a.face_vals = st->face_vals_d;
	a.face_tiles = st->face_tiles[axis];
	return a;
}

int launch_staged_sweep(bfvm_solver* st, int axis, const sweep_tuning& tune, bool& handled)
{
	const sweep_args a = make_args(st, axis);
	return launch_sweep_tma(st, axis, a, handled, &tune);
}

std::vector<sweep_tuning> staged_sweep_shapes(bfvm_solver* st, int axis)
{
	std::vector<sweep_tuning> shapes;
	bool handled = false;
	const sweep_args a = make_args(st, axis);
	if (launch_sweep_tma(st, axis, a, handled, nullptr, &shapes))
		shapes.clear();
	return shapes;
}

int launch_slab_z(bfvm_solver* st)
{
	sweep_args a = make_args(st, 2);
	a.slab_lines = (long long)st->grid[0] * st->grid[1] * st->S;
	a.slab_carry = st->slab_carry;
	bool handled = false;
	int rc = BFVM_OK;
	if (st->use_tma)
		rc = launch_sweep_tma(st, 2, a, handled, &st->tune[2], nullptr, true);
	if (!rc && !handled)
		rc = fail(BFVM_ERR_INVALID_ARGUMENT, "the z sweep of a slab needs the TMA-staged kernel: at most 512 planes "
											 "per slab, X * substrates a multiple of 4, and the tma_sweeps option on");
	return rc;
}

// The sweep of one axis by the first kernel that takes its shape: the TMA-staged sweep (which sets
// `staged`; with gf, only if it also computes the gradient), the staged sweep of the line's chunks,
// the ensemble sweep on this mesh alone, or the direct kernels.
static int sweep_axis(bfvm_solver* st, int axis, const sweep_args& a, bool& staged, const grad_fuse* gf = nullptr)
{
	const sweep_plan& pl = st->plan[axis];
	int rc = BFVM_OK;
	bool handled = false;
	staged = false;
	// lines longer than the chunk length (chunk_elements; always beyond 512): the staged sweep of
	// their chunks with their carries (chunks.cu).  Not `staged` for the caller: the chunks write no
	// per-tile overwrite, face condition or gradient.
	if (st->use_tma && pl.chunks.count > 0)
	{
		rc = launch_chunked_sweep(st, axis, handled);
		if (rc || handled)
			return rc;
	}
	if (st->use_tma)
		rc = launch_sweep_tma(st, axis, a, handled, &st->tune[axis], nullptr, false, gf);
	if (!rc && !handled && gf)
		return sweep_axis(st, axis, a, staged); // the shape cannot take the gradient: sweep alone
	staged = handled;
	// the same front-padded block algebra without TMA staging, where the lines fit 16 blocks
	if (!rc && !handled && st->self_plan && pl.vtab && pl.vP <= ENS_MAX_P_ONE && (axis > 0 || st->S <= 32)
		&& ensemble_sweep_fits(*st->self_plan, axis))
	{
		rc = ensemble_sweep(*st->self_plan, axis, st->stream);
		if (!rc)
			st->launches++;
		handled = true;
	}
	if (!rc && !handled)
		rc = pl.M == 32 ? launch_sweep_m<32>(st, axis, a) : launch_sweep_m<64>(st, axis, a);
	return rc;
}

// One axis on its own (bfvm_diffusion_sweep): the Dirichlet overwrite that precedes the sweep,
// the sweep, and after the last axis the closing overwrite.
int launch_sweep(bfvm_solver* st, int axis, bool final_dirichlet)
{
	int rc = launch_dirichlet(st);
	if (rc)
		return rc;
	bool staged = false;
	rc = sweep_axis(st, axis, make_args(st, axis), staged);
	if (!rc && final_dirichlet)
		rc = launch_dirichlet(st);
	return rc;
}

// The tile flags and deferred-tile list of the gradient inside the z sweep, allocated outside any
// stream capture (bfvm_run_steps calls this before it captures a step); inside a capture nothing
// is allocated.
int grad_fuse_buffers(bfvm_solver* st)
{
	if (st->dims != 3)
		return BFVM_OK;
	const long long items = ((long long)st->grid[1] * st->grid[0] * st->S + 31) / 32; // z tiles
	if (st->grad_tiles >= items)
		return BFVM_OK;
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	BFVM_CUDA(cudaStreamIsCapturing(st->stream, &cs));
	if (cs != cudaStreamCaptureStatusNone)
		return BFVM_OK;
	device_free(st->grad_tile_done);
	device_free(st->grad_deferred);
	st->grad_tiles = 0;
	int rc;
	if ((rc = device_alloc(&st->grad_tile_done, (size_t)items)) || (rc = device_alloc(&st->grad_deferred, (size_t)items + 1)))
		return rc;
	st->grad_tiles = items;
	return BFVM_OK;
}

// The band modes of the step.  A band is a slab of the field small enough to stay in L2 between two
// kernels: the kernel after the first reads the band back from L2 instead of HBM.  The arithmetic of
// every element is the same as in whole-field launches (each tile is swept by the same code), so
// results are identical; only the order of tiles changes.  The Dirichlet overwrites between the
// sweeps come from the per-tile lists, written by the sweep of each tile, so the band modes need them
// wherever the mesh has Dirichlet nodes.
static bool band_overwrites_ready(const bfvm_solver* st, int axis)
{
	return st->dir_qcount + st->dir_count == 0 || st->dir_tiles[axis].items > 0;
}

// x then y sweep per band of `xy_band_planes` z planes: a band's y sweep reads what its x sweep
// wrote.  Needs whole x tiles per plane (rows % (32 / S) == 0).  *done: the band mode ran.
static int banded_xy(bfvm_solver* st, bool& done)
{
	done = false;
	const long long c = st->xy_band_planes;
	if (c <= 0 || st->dims != 3 || !st->use_tma || c >= st->grid[2])
		return BFVM_OK;
	const staged_tiling tx = staged_tiles(st, 0), ty = staged_tiles(st, 1);
	const long long Y = st->grid[1], Z = st->grid[2];
	if (tx.items == 0 || ty.items == 0 || Y % tx.R != 0 || !band_overwrites_ready(st, 0) || !band_overwrites_ready(st, 1)
		|| staged_sweep_shapes(st, 0).empty() || staged_sweep_shapes(st, 1).empty())
		return BFVM_OK;
	sweep_args ax = make_args(st, 0), ay = make_args(st, 1);
	ax.dir = st->dir_tiles[0];
	ay.dir = st->dir_tiles[1];
	for (long long z0 = 0; z0 < Z; z0 += c)
	{
		const long long z1 = std::min(Z, z0 + c);
		bool hx = false, hy = false;
		int rc = launch_sweep_tma(st, 0, ax, hx, &st->tune[0], nullptr, false, nullptr, z0 * Y / tx.R, z1 * Y / tx.R);
		if (!rc)
			rc = launch_sweep_tma(st, 1, ay, hy, &st->tune[1], nullptr, false, nullptr, z0 * ty.col_tiles,
								  z1 * ty.col_tiles);
		if (!rc && !(hx && hy))
			rc = fail(BFVM_ERR_STATE, "a band of the x and y sweeps was not staged");
		if (rc)
			return rc;
	}
	done = true;
	return BFVM_OK;
}

// z sweep then gradient per band of `zg_band_rows` y rows: after the z sweep of rows [0, y1) the
// gradient of rows [.., y1 - 1) has every neighbour final (row y reads y - 1 and y + 1).  Needs
// whole z tiles per row (x * substrates % 32 == 0) and the row-range gradient kernel.
static int banded_zgrad(bfvm_solver* st, bool& done)
{
	done = false;
	const long long c = st->zg_band_rows;
	if (c <= 0 || st->dims != 3 || !st->use_tma || c >= st->grid[1] || !gradient_rows_possible(st))
		return BFVM_OK;
	const staged_tiling tz = staged_tiles(st, 2);
	const long long Y = st->grid[1], XS = tz.XS;
	if (tz.items == 0 || XS % 32 != 0 || !band_overwrites_ready(st, 2) || staged_sweep_shapes(st, 2).empty())
		return BFVM_OK;
	sweep_args az = make_args(st, 2);
	az.dir = st->dir_tiles[2];
	const long long row_tiles = XS / 32;
	long long g0 = 0;
	for (long long y0 = 0; y0 < Y; y0 += c)
	{
		const long long y1 = std::min(Y, y0 + c);
		bool hz = false;
		int rc = launch_sweep_tma(st, 2, az, hz, &st->tune[2], nullptr, false, nullptr, y0 * row_tiles, y1 * row_tiles);
		if (!rc && !hz)
			rc = fail(BFVM_ERR_STATE, "a band of the z sweep was not staged");
		const long long g1 = y1 == Y ? Y : y1 - 1;
		if (!rc)
			rc = launch_gradient_rows(st, (int)g0, (int)g1);
		if (rc)
			return rc;
		g0 = g1;
	}
	done = true;
	return BFVM_OK;
}

// The whole LOD step (src/solver/host/diffusion_solver.cpp:512-544): overwrite, then per axis the
// sweep and the overwrite after it.  A staged sweep writes that overwrite itself, tile by tile
// right after storing the tile, from the list grouped by its tiles; other sweeps are followed by
// the scatter kernel.
int launch_diffusion(bfvm_solver* st, bool gradient, bool* gradient_done)
{
	if (gradient_done)
		*gradient_done = false;
	// the face conditions by position: each staged sweep writes them into the values it stores, and
	// the scatter after it keeps the interior elements alone.  An axis whose sweep is not staged is
	// followed by the whole list.
	const bool faces = faces_by_position(st) && st->xy_band_planes == 0 && st->zg_band_rows == 0;
	// the first overwrite stays a scatter of the whole list: inside the x sweep it would have to
	// reach the values before the recurrences, where the kernel has no registers to spare
	int rc = launch_dirichlet(st);
	int axis = 0;
	if (!rc)
	{
		bool banded = false;
		rc = banded_xy(st, banded);
		if (banded)
			axis = 2;
	}
	for (; axis < st->dims && !rc; axis++)
	{
		if (axis == 2 && gradient && gradient_done && !st->grad_fused && st->batch_refs == 0 && st->slab_count == 1)
		{
			bool banded = false;
			if ((rc = banded_zgrad(st, banded)))
				return rc;
			if (banded)
			{
				*gradient_done = true;
				break;
			}
		}
		sweep_args a = make_args(st, axis);
		if (st->dir_fused)
			a.dir = st->dir_tiles[axis];
		if (faces)
			a.face_apply = 1;
		// the gradient inside the z sweep needs the final field there: no overwrite after it, or
		// the overwrite written by the sweep itself
		const bool overwrite_after = st->dir_qcount + st->dir_count > 0;
		grad_fuse gf;
		bool fuse_grad = gradient && axis == 2 && st->grad_fused && st->batch_refs == 0 && st->slab_count == 1
							   && st->plan[2].vP > 1 && (!overwrite_after || a.dir.items > 0);
		if (fuse_grad && (rc = grad_fuse_buffers(st)))
			return rc;
		if (fuse_grad && st->grad_tiles < ((long long)st->grid[1] * st->grid[0] * st->S + 31) / 32)
			fuse_grad = false; // inside a capture before the buffers exist: the gradient kernel follows
		if (fuse_grad)
		{
			gf.g = st->grad;
			gf.tile_done = st->grad_tile_done;
			gf.deferred = st->grad_deferred;
			gf.lag = 0;
			gf.total = st->V * st->S;
			gf.X = st->grid[0];
			gf.Y = st->grid[1];
			gf.Z = st->grid[2];
			gf.S = st->S;
			// the factors of gradient.cu: 1/h at the ends, 1/(2h) inside, rounded to float
			gf.bx = 1.f / st->voxel[0];
			gf.cx = 1.f / (st->voxel[0] * 2);
			gf.by = 1.f / st->voxel[1];
			gf.cy = 1.f / (st->voxel[1] * 2);
			gf.bz = 1.f / st->voxel[2];
			gf.cz = 1.f / (st->voxel[2] * 2);
			gf.spin_limit = 200000; // about 0.1 ms, then the tile is deferred
		}
		bool staged = false;
		rc = sweep_axis(st, axis, a, staged, fuse_grad ? &gf : nullptr);
		if (!rc && fuse_grad && staged && gradient_done)
			*gradient_done = true;
		if (!rc && !(staged && a.dir.items > 0))
			rc = launch_dirichlet(st, staged && faces);
	}
	return rc;
}

} // namespace bfvm
