// Sweeps with the field staged through shared memory by the Tensor Memory Accelerator.
//
// A persistent CTA owns a tile of 32 lines at a time: 32 adjacent columns of the x*s plane (y
// sweep) or of the y*x*s plane (z sweep), or R = 32/S whole rows (x sweep, R rows x S substrate
// lines).  Warp j holds register block j of every line of the tile (blockDim = (32, P)).  Two
// shared-memory stages alternate: while the CTA solves the tile in one stage, the TMA copies the
// next tile into the other, so the HBM reads of the next tile overlap the recurrences of this one.
// Results are written straight from registers with coalesced stores.  The Dirichlet overwrites run
// before and after the sweeps (dirichlet.cu), so this kernel is a pure line solve.
//
//   y sweep: 3D tensor map over [Z][Y][XS], boxes of 32 columns x box_h rows
//   z sweep: 2D tensor map over [Z][Y*XS], boxes of 32 columns x box_h planes
//   x sweep: one 1D bulk copy per row, into rows padded so the 32 lanes hit distinct banks
//
// Copies complete on an mbarrier per stage; every wait is bounded by a clock limit, after which
// the kernel raises DEVERR_TIMEOUT, lets its copies in flight land (again bounded) and returns.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "sweep_common.cuh"

namespace bfvm {

static constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL; // about two seconds

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
				 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
				 "selp.u32 %0, 1, 0, p;\n}"
				 : "=r"(ok)
				 : "r"(smem_addr(bar)), "r"(parity)
				 : "memory");
	return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
	const long long t0 = clock64();
	while (!mbar_try_wait(bar, parity))
		if (clock64() - t0 > WAIT_LIMIT_CYCLES)
			return false;
	return true;
}

__device__ __forceinline__ void tma_load_2d(float* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
				 ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_addr(bar))
				 : "memory");
}

__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar)
{
	asm volatile(
		"cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
		::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
		: "memory");
}

__device__ __forceinline__ void bulk_load(float* dst, const float* src, uint32_t bytes, uint64_t* bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
				 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
				 : "memory");
}

struct tma_tile
{
	int axis;			 // 0 x (rows), 1 y, 2 z
	long long items;	 // tiles
	long long ncols;	 // columns of the plane (y, z)
	long long col_tiles; // 32-column tiles per plane (y, z)
	long long outer_stride, line_stride;
	int box_h, nbox;	 // TMA boxes along the line (y, z)
	int R, row_pitch;	 // rows per tile and padded row length in floats (x)
	long long nrows;
	long long XS;
	int stage_floats;
	int stages; // pipeline depth (NST)
};

// Issue the copies of tile w into `dst`, completing on `bar` (one thread).
__device__ __forceinline__ void issue_tile(const sweep_args& a, const CUtensorMap* map, const tma_tile& tt, long long w,
										   float* dst, uint64_t* bar)
{
	if (tt.axis == 0)
	{
		const long long row0 = w * tt.R;
		const int rows = (int)min((long long)tt.R, tt.nrows - row0);
		const uint32_t row_bytes = (uint32_t)(tt.XS * sizeof(float));
		mbar_expect_tx(bar, row_bytes * rows);
		for (int r = 0; r < rows; r++)
			bulk_load(dst + r * tt.row_pitch, a.data + (row0 + r) * tt.XS, row_bytes, bar);
		return;
	}
	const long long outer = w / tt.col_tiles;
	const int c0 = (int)((w % tt.col_tiles) * 32);
	mbar_expect_tx(bar, (uint32_t)(tt.nbox * tt.box_h * 32 * sizeof(float)));
	for (int b = 0; b < tt.nbox; b++)
	{
		if (tt.axis == 1)
			tma_load_3d(dst + b * tt.box_h * 32, map, c0, b * tt.box_h, (int)outer, bar);
		else
			tma_load_2d(dst + b * tt.box_h * 32, map, c0, b * tt.box_h, bar);
	}
}

// Where line `lane` of tile w lives: in the shared-memory stage (sbase + i*sstride) and in the
// field (line + i*gstride), and its Dirichlet conditions.
struct tile_line
{
	bool active;
	int s, sbase, sstride;
	float* line;
	long long gstride;
	long long rr;			// x sweep: row index y + Y*z
	long long outer, qq;	// y/z sweeps: plane and column

	__device__ __forceinline__ void locate(const sweep_args& a, const tma_tile& tt, long long w, int lane)
	{
		const int S = a.S;
		if (tt.axis == 0)
		{
			const int rl = lane / S;
			s = lane - rl * S;
			const long long row = w * tt.R + rl;
			active = rl < tt.R && row < tt.nrows;
			rr = active ? row : 0;
			sbase = (rl < tt.R ? rl : 0) * tt.row_pitch + s; // lanes past the last row read row 0
			sstride = S;
			line = a.data + rr * tt.XS + s;
			gstride = S;
		}
		else
		{
			outer = w / tt.col_tiles;
			const long long q = (w % tt.col_tiles) * 32 + lane;
			active = q < tt.ncols;
			qq = active ? q : 0;
			s = (int)(qq % S);
			sbase = lane;
			sstride = 32;
			line = a.data + outer * tt.outer_stride + qq;
			gstride = tt.line_stride;
		}
	}

};

template <bool UNI, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
	sweep_tma_kernel(const __grid_constant__ sweep_args a, const __grid_constant__ CUtensorMap map,
					 const __grid_constant__ tma_tile tt)
{
	constexpr int M = 32;
	extern __shared__ __align__(128) unsigned char smem_raw[];
	// NST stages on a 1024-byte boundary (TMA destinations), then tables, carries and barriers
	const int NST = tt.stages;
	float* const stages = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
	float* tab = stages + (size_t)NST * tt.stage_floats;
	const int S = a.S;
	const float* ctab = tab + a.n * S;
	const float* gtab = ctab + S;
	const float* Gtab = gtab + a.P * S;
	float* carry_f = tab + table_floats(a.n, a.P, S);
	float* carry_t = carry_f + a.P * 32;
	uint64_t* bars =
		reinterpret_cast<uint64_t*>((reinterpret_cast<uintptr_t>(carry_t + a.P * 32) + 7) & ~uintptr_t(7));

	const int lane = threadIdx.x;
	const int j = threadIdx.y;
	const bool leader = lane == 0 && j == 0;
	if (leader)
	{
		for (int k = 0; k < NST; k++)
			mbar_init(&bars[k], 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	stage_table(a, tab, 0, S); // ends with __syncthreads, which also publishes the barrier init

	int p, L;
	block_range(j, a.base_len, a.extra, p, L);

	// prologue: the first NST-1 tiles of this CTA
	if (leader)
		for (int k = 0; k < NST - 1; k++)
		{
			const long long wk = blockIdx.x + (long long)k * gridDim.x;
			if (wk < tt.items)
				issue_tile(a, &map, tt, wk, stages + (size_t)k * tt.stage_floats, &bars[k]);
		}

	bool failed = false;
	int it = 0;
	long long w = blockIdx.x;
	for (; w < tt.items; w += gridDim.x, it++)
	{
		const int st = it % NST;
		const uint32_t parity = (uint32_t)((it / NST) & 1);
		if (leader)
		{
			// keep NST-1 tiles in flight; that stage was released by the previous tile's final barrier
			const long long wn = w + (long long)(NST - 1) * gridDim.x;
			if (wn < tt.items)
			{
				const int sn = (it + NST - 1) % NST;
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				issue_tile(a, &map, tt, wn, stages + (size_t)sn * tt.stage_floats, &bars[sn]);
			}
		}

		// this thread's line in the tile
		const float* cur = stages + (size_t)st * tt.stage_floats;
		tile_line tl;
		tl.locate(a, tt, w, lane);

		const bool ok = mbar_wait(&bars[st], parity);
		if (!__syncthreads_and(ok))
		{
			failed = true;
			break;
		}

		float d[M];
#pragma unroll
		for (int k = 0; k < M; k++)
			d[k] = (UNI || k < L) ? cur[tl.sbase + (p + k) * tl.sstride] : 0.f;
		const int s_now = tl.s;
		const bool active_now = tl.active;

		thomas_block<M, UNI>(d, L, p, j, a.P, tab + s_now, gtab + s_now, Gtab + s_now, S, ctab[s_now], active_now,
							 carry_f + lane, carry_t + lane, 32);

		{
			// recompute the line from an opaque copy of the tile index, so nothing of the load
			// phase stays live across the solve
			long long w2;
			asm volatile("mov.b64 %0, %1;" : "=l"(w2) : "l"(w));
			tile_line tl2;
			tl2.locate(a, tt, w2, lane);
			if (tl2.active)
			{
				float* ptr = tl2.line + (long long)p * tl2.gstride;
#pragma unroll
				for (int k = 0; k < M; k++)
					if (UNI || k < L)
					{
						*ptr = d[k];
						ptr += tl2.gstride;
					}
			}
		}
		__syncthreads(); // stage st fully read before it is refilled
	}

	if (failed && leader)
	{
		atomicOr(a.err, DEVERR_TIMEOUT);
		// let the copies already issued land before the CTA exits (bounded waits)
		for (int k = 0; k < NST - 1; k++)
		{
			const long long wk = w + (long long)k * gridDim.x;
			if (wk < tt.items)
				mbar_wait(&bars[(it + k) % NST], (uint32_t)(((it + k) / NST) & 1));
		}
	}
}

// ------------------------------------------------------------------------------------------------
// host side

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	static bool tried = false;
	if (!tried)
	{
		tried = true;
		cudaDriverEntryPointQueryResult q;
		void* p = nullptr;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess
			&& q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
		else
			(void)cudaGetLastError();
	}
	return fn;
}

static constexpr int TMA_MAX_P = 16;

template <bool UNI, int MAXT, int MINB>
static int launch_tma_variant(bfvm_solver* st, const sweep_args& a, const CUtensorMap& map, const tma_tile& tt,
							  size_t smem)
{
	auto kernel = sweep_tma_kernel<UNI, MAXT, MINB>;
	int rc = set_smem(kernel, smem);
	if (rc)
		return rc;
	const int threads = 32 * a.P;
	const int grid = persistent_grid(kernel, threads, smem, tt.items, st->device);
	kernel<<<grid, dim3(32, a.P), smem, st->stream>>>(a, map, tt);
	return check_launch(st, tt.axis == 0 ? "sweep_tma<x>" : (tt.axis == 1 ? "sweep_tma<y>" : "sweep_tma<z>"));
}

int launch_sweep_tma(bfvm_solver* st, int axis, const sweep_args& a, bool& handled)
{
	handled = false;
	const long long X = st->grid[0], Y = st->grid[1], Z = st->grid[2], S = st->S;
	const long long XS = X * S;
	const sweep_plan& pl = st->plan[axis];
	// shapes the TMA path covers: 16-byte row strides, at most 16 blocks of 32 per line, and for
	// the x sweep whole rows of at most 32 substrate lines per tile
	if (pl.M != 32 || a.P > TMA_MAX_P || XS % 4 != 0 || (axis == 0 && S > 32) || a.n < 2)
		return BFVM_OK;
	auto encode = encode_fn();
	if (!encode)
		return BFVM_OK;

	tma_tile tt;
	std::memset(&tt, 0, sizeof(tt));
	tt.axis = axis;
	tt.XS = XS;
	CUtensorMap map;
	std::memset(&map, 0, sizeof(map));
	if (axis == 0)
	{
		tt.R = (int)(32 / S);
		tt.nrows = Y * Z;
		tt.items = (tt.nrows + tt.R - 1) / tt.R;
		// pad rows so that lane (r, s) = r*pitch + s spreads over the banks, keeping 16-byte rows
		int pad = (int)(((S % 32) - (XS % 32) + 64) % 32);
		pad = (pad + 3) / 4 * 4;
		tt.row_pitch = (int)XS + pad;
		tt.stage_floats = (tt.R * tt.row_pitch + 31) / 32 * 32;
	}
	else
	{
		const long long n = axis == 1 ? Y : Z;
		tt.nbox = (int)((n + 255) / 256);
		tt.box_h = (int)((n + tt.nbox - 1) / tt.nbox);
		tt.ncols = axis == 1 ? XS : Y * XS;
		tt.col_tiles = (tt.ncols + 31) / 32;
		tt.items = (axis == 1 ? Z : 1) * tt.col_tiles;
		tt.outer_stride = axis == 1 ? Y * XS : 0;
		tt.line_stride = axis == 1 ? XS : Y * XS;
		tt.stage_floats = tt.nbox * tt.box_h * 32;
		cuuint64_t dims[3], strides[2];
		cuuint32_t box[3], estr[3] = { 1, 1, 1 };
		cuuint32_t rank;
		if (axis == 1)
		{
			rank = 3;
			dims[0] = (cuuint64_t)XS;
			dims[1] = (cuuint64_t)Y;
			dims[2] = (cuuint64_t)Z;
			strides[0] = (cuuint64_t)(XS * sizeof(float));
			strides[1] = (cuuint64_t)(Y * XS * sizeof(float));
			box[0] = 32;
			box[1] = (cuuint32_t)tt.box_h;
			box[2] = 1;
		}
		else
		{
			rank = 2;
			dims[0] = (cuuint64_t)(Y * XS);
			dims[1] = (cuuint64_t)Z;
			strides[0] = (cuuint64_t)(Y * XS * sizeof(float));
			box[0] = 32;
			box[1] = (cuuint32_t)tt.box_h;
		}
		CUresult r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, st->dens, dims, strides, box, estr,
							CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
							CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
		if (r != CUDA_SUCCESS)
			return BFVM_OK; // fall back to the direct kernels
	}
	int dev = 0, optin = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
	// one CTA per SM (128 registers) with as many stages as fit, up to 4; or, on request, two
	// 320-thread CTAs per SM (96 registers) with two stages each
	const bool two_per_sm = a.P <= 10 && st->sweep_ctas_per_sm == 2;
	const size_t fixed = 1024 + (table_floats(a.n, a.P, (int)S) + 2 * (size_t)a.P * 32) * sizeof(float) + 8
						 + 4 * sizeof(uint64_t);
	const size_t stage_bytes = (size_t)tt.stage_floats * sizeof(float);
	const size_t budget = two_per_sm ? std::min<size_t>((size_t)optin, 110 * 1024) : (size_t)optin;
	if (fixed + 2 * stage_bytes > budget)
		return BFVM_OK;
	tt.stages = (int)std::min<size_t>(two_per_sm ? 2 : 4, (budget - fixed) / stage_bytes);
	const size_t smem = fixed + tt.stages * stage_bytes;

	handled = true;
	const bool uni = a.extra == 0 && a.base_len == 32 && st->sweep_uniform != 0;
	if (two_per_sm)
		return uni ? launch_tma_variant<true, 320, 2>(st, a, map, tt, smem)
				   : launch_tma_variant<false, 320, 2>(st, a, map, tt, smem);
	return uni ? launch_tma_variant<true, 512, 1>(st, a, map, tt, smem)
			   : launch_tma_variant<false, 512, 1>(st, a, map, tt, smem);
}

} // namespace bfvm
