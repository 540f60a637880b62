// The learned surrogate's kernels: 3x3x3 convolutions on the fifth-generation tensor cores and the
// element-wise steps around them.
//
// Activations are channels-last bf16 tensors [B][Z][Y][X][32]: every layer has 32 channels (inputs
// and outputs with fewer are zero-padded), so one kernel covers every convolution.  A convolution
// is an implicit GEMM:
//   out[v][co] = sum over taps t, ci of  W[t][co][ci] * in[v + off_t][ci]
// with M = 128 voxels along x (one tile), N = 32 output channels and K = 27 taps x 32 channels.
// The tile of tap t is a TMA box of 128 voxels x 32 channels at the shifted coordinates, so the
// copy engine does the im2col gather and the zero padding at the mesh edges (out-of-range boxes read
// zeros).  The boxes land 64B-swizzled, the layout the MMA reads K-major; the 27 weight taps stay in
// shared memory for the CTA's whole life.  One thread issues tcgen05.mma (M128 N32 K16, bf16 in,
// f32 accumulate) into tensor memory; four epilogue warps read the accumulator back with
// tcgen05.ld, add bias, a residual and the ReLU, and store bf16 (or the f32 field prediction).
//
// The backward pass of the input is the same kernel run on the output gradient with the weights
// flipped in space and transposed in channels (W'[26-t][ci][co] = W[t][co][ci]), with the ReLU
// mask of the layer's input applied in the epilogue.  The weight gradient
//   dW[t][co][ci] = sum over v of dY[v][co] * in[v + off_t][ci]
// is a GEMM with M = 4 taps x 32 input channels, N = 32 output channels and K = voxels; both
// operands are tiles of voxels x channels, read MN-major.
//
// Warp roles (192 threads): warp 0 issues the TMA copies, warp 1 owns the tensor memory and one
// of its threads issues the MMAs, warps 2-5 run the epilogue.  Every wait is bounded: a role that
// gives up sets DEVERR_TIMEOUT and a shared abort flag, the others leave their loops, the copies
// and MMAs in flight are waited for (bounded again) and the tensor memory is freed.

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "sm100_common.cuh"
#include "surrogate.h"
#include "sweep_common.cuh"

namespace bfvm {

// ------------------------------------------------------------------------------------------------
// tcgen05

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
				 "r"(ncols)
				 : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (bf16 operands, f32 accumulator)
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
										  uint32_t accumulate)
{
	asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
				 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
				 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
				 : "memory");
}

// arrive on `bar` once every MMA this thread issued so far has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
				 : "memory");
}

// 32 consecutive f32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
	uint32_t r[32];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
				 "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
				 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
				   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
				   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
				   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
				   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
				 : "r"(taddr)
				 : "memory");
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 32; i++)
		v[i] = __uint_as_float(r[i]);
}

// Shared-memory operand descriptor, 64-byte swizzle (rows of 64 bytes, 8-row atoms of 512 bytes;
// tiles start on 1024-byte boundaries).  lbo / sbo in bytes: for a K-major operand sbo is the step
// between 8-row groups and lbo is unused; for an MN-major operand lbo is the step between 32-element
// groups of M (or N) and sbo the step between 8-row groups of K.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
	d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
	d |= (uint64_t)1 << 46; // descriptor version of sm_100
	d |= (uint64_t)4 << 61; // 64-byte swizzle
	return d;
}

// Instruction descriptor: bf16 A and B, f32 D, M x N; a_mn / b_mn select MN-major operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16)
		   | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tap_offset(int t, int& dz, int& dy, int& dx)
{
	dz = t / 9 - 1;
	dy = (t / 3) % 3 - 1;
	dx = t % 3 - 1;
}

__device__ __forceinline__ bool aborted(volatile int* flag) { return *flag != 0; }

__device__ __forceinline__ void give_up(volatile int* flag, int* err)
{
	*flag = 1;
	atomicOr(err, DEVERR_TIMEOUT);
}

// ------------------------------------------------------------------------------------------------
// convolution (forward, and backward of the input with flipped weights)

static constexpr uint32_t A_TILE_BYTES = SUR_TILE * SUR_C * 2; // 8192: 128 voxels x 32 channels
static constexpr uint32_t W_TAP_BYTES = SUR_C * SUR_C * 2;	   // 2048
static constexpr uint32_t W_BYTES = SUR_TAPS * W_TAP_BYTES;	   // 55296 (54 x 1024)
// A stage holds the 130 voxels x0 - 1 .. x0 + 128 of one (y + dy, z + dz) row, which serve the three
// taps dx = -1, 0, +1 as 128-row operands starting 0, 1 and 2 rows (64 bytes each) into the box.
static constexpr int CONV_ROWS = SUR_TILE + 2;
static constexpr uint32_t A_BOX_BYTES = CONV_ROWS * SUR_C * 2; // 8320
static constexpr uint32_t A_STAGE_BYTES = 9216;					// rounded up to 1024
static constexpr int CONV_PIPES = 3;  // independent pipelines per CTA, sharing the weights
static constexpr int CONV_STAGES = 6; // stages per pipeline
static constexpr int CONV_THREADS = 32 * (2 * CONV_PIPES + 4 * CONV_PIPES);
// barriers per pipeline: full and empty per stage, 2 accumulator full, 2 accumulator empty, drain;
// then the shared weight barrier, the tensor-memory address and the abort flag
static constexpr int CONV_PIPE_BARS = 2 * CONV_STAGES + 5;
static constexpr size_t CONV_BAR_BYTES = (CONV_PIPES * CONV_PIPE_BARS + 1) * sizeof(uint64_t) + 2 * sizeof(uint32_t);
static constexpr size_t CONV_SMEM =
	1024 + W_BYTES + (size_t)CONV_PIPES * CONV_STAGES * A_STAGE_BYTES + CONV_BAR_BYTES;
static_assert(CONV_SMEM <= 227 * 1024, "convolution stages exceed the shared memory of a CTA");
static_assert(A_BOX_BYTES <= A_STAGE_BYTES && A_STAGE_BYTES % 1024 == 0, "stage layout");

__device__ __forceinline__ void decode_tile(long long tile, const conv_params& p, int& b, int& z, int& y, int& x0)
{
	const int xt = (int)(tile % p.x_tiles);
	long long r = tile / p.x_tiles;
	y = (int)(r % p.Y);
	r /= p.Y;
	z = (int)(r % p.Z);
	b = (int)(r / p.Z);
	x0 = xt * SUR_TILE;
}

__device__ __forceinline__ void load_bf16x32(const __nv_bfloat16* src, float (&v)[32])
{
	const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
	for (int i = 0; i < 4; i++)
	{
		const uint4 u = __ldg(s + i);
		const uint32_t w[4] = { u.x, u.y, u.z, u.w };
#pragma unroll
		for (int j = 0; j < 4; j++)
		{
			const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[j]);
			const float2 f = __bfloat1622float2(h);
			v[8 * i + 2 * j] = f.x;
			v[8 * i + 2 * j + 1] = f.y;
		}
	}
}

__device__ __forceinline__ void store_bf16x32(__nv_bfloat16* dst, const float (&v)[32])
{
	uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
	for (int i = 0; i < 4; i++)
	{
		uint32_t w[4];
#pragma unroll
		for (int j = 0; j < 4; j++)
		{
			const __nv_bfloat162 h = __floats2bfloat162_rn(v[8 * i + 2 * j], v[8 * i + 2 * j + 1]);
			w[j] = *reinterpret_cast<const uint32_t*>(&h);
		}
		d[i] = make_uint4(w[0], w[1], w[2], w[3]);
	}
}

// CTA = CONV_PIPES pipelines, each with its own producer thread (warp p), MMA thread (warp
// CONV_PIPES + p), four epilogue warps, CONV_STAGES stages and two tensor-memory accumulators of
// 32 columns; all share the 27 weight taps.  Pipeline p of CTA c takes tiles c * CONV_PIPES + p,
// then every gridDim.x * CONV_PIPES-th tile.
__global__ void __launch_bounds__(CONV_THREADS, 1) sur_conv_kernel(const __grid_constant__ CUtensorMap act,
																	const __grid_constant__ CUtensorMap wmap,
																	const __grid_constant__ conv_params p)
{
	extern __shared__ __align__(1024) unsigned char conv_smem[];
	unsigned char* base =
		reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(conv_smem) + 1023) & ~uintptr_t(1023));
	unsigned char* wsm = base; // 27 taps x [32 co][64 B]
	unsigned char* stages0 = base + W_BYTES;
	uint64_t* bars0 = reinterpret_cast<uint64_t*>(stages0 + (size_t)CONV_PIPES * CONV_STAGES * A_STAGE_BYTES);
	uint64_t* wbar = bars0 + CONV_PIPES * CONV_PIPE_BARS;
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(wbar + 1);
	volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

	const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
	if (threadIdx.x == 0)
	{
		for (int q = 0; q < CONV_PIPES; q++)
		{
			uint64_t* b = bars0 + q * CONV_PIPE_BARS;
			for (int s = 0; s < CONV_STAGES; s++)
			{
				mbar_init(b + s, 1);				// full
				mbar_init(b + CONV_STAGES + s, 1);	// empty
			}
			mbar_init(b + 2 * CONV_STAGES, 1);		// accumulator 0 full
			mbar_init(b + 2 * CONV_STAGES + 1, 1);	// accumulator 1 full
			mbar_init(b + 2 * CONV_STAGES + 2, 128); // accumulator 0 empty
			mbar_init(b + 2 * CONV_STAGES + 3, 128); // accumulator 1 empty
			mbar_init(b + 2 * CONV_STAGES + 4, 1);	// drain
		}
		mbar_init(wbar, 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == CONV_PIPES)
	{
		tmem_alloc(tmem_slot, 256); // 2 accumulators of 32 columns per pipeline (192 used)
		tmem_relinquish();
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tmem_slot;

	// this thread's role and pipeline
	int role, pipe;
	if (warp < CONV_PIPES)
	{
		role = 0;
		pipe = warp;
	}
	else if (warp < 2 * CONV_PIPES)
	{
		role = 1;
		pipe = warp - CONV_PIPES;
	}
	else
	{
		role = 2;
		pipe = (warp - 2 * CONV_PIPES) / 4;
	}
	uint64_t* bars = bars0 + pipe * CONV_PIPE_BARS;
	uint64_t* full = bars;
	uint64_t* empty = bars + CONV_STAGES;
	uint64_t* acc_full = bars + 2 * CONV_STAGES;
	uint64_t* acc_empty = acc_full + 2;
	uint64_t* drain = acc_empty + 2;
	unsigned char* stages = stages0 + (size_t)pipe * CONV_STAGES * A_STAGE_BYTES;
	const long long first = (long long)blockIdx.x * CONV_PIPES + pipe;
	const long long stride = (long long)gridDim.x * CONV_PIPES;
	const long long my_tiles = first < p.tiles ? (p.tiles - first + stride - 1) / stride : 0;
	const uint32_t acc_col = tmem + (uint32_t)(pipe * 2 * SUR_C);

	if (role == 0 && lane == 0)
	{
		// producer: the weights once (pipeline 0), then one 130-row box per (dy, dz) of each tile
		if (pipe == 0)
		{
			mbar_expect_tx(wbar, W_BYTES);
			for (int t = 0; t < SUR_TAPS; t++)
				tma_load_2d(wsm + t * W_TAP_BYTES, &wmap, 0, t * SUR_C, wbar);
		}
		long long n = 0;
		for (long long i = 0; i < my_tiles && !aborted(abort_flag); i++)
		{
			int b, z, y, x0;
			decode_tile(first + i * stride, p, b, z, y, x0);
			for (int r = 0; r < 9; r++, n++)
			{
				const int s = (int)(n % CONV_STAGES);
				if (!mbar_wait(empty + s, (uint32_t)(((n / CONV_STAGES) & 1) ^ 1)))
				{
					give_up(abort_flag, p.err);
					break;
				}
				mbar_expect_tx(full + s, A_BOX_BYTES);
				tma_load_5d(stages + s * A_STAGE_BYTES, &act, 0, x0 - 1, y + r % 3 - 1, z + r / 3 - 1, b, full + s);
			}
		}
		// the copies issued last land before the CTA exits
		for (long long k = (n > CONV_STAGES ? n - CONV_STAGES : 0); k < n; k++)
			mbar_wait(full + k % CONV_STAGES, (uint32_t)((k / CONV_STAGES) & 1));
		if (pipe == 0)
			mbar_wait(wbar, 0);
	}
	else if (role == 1 && lane == 0)
	{
		// MMA issuer: per box, taps dx = -1, 0, +1 from rows 0, 1, 2 of the box; two K steps of 16
		// channels (32 bytes) each
		constexpr uint32_t idesc = idesc_bf16(SUR_TILE, SUR_C, false, false);
		bool ok = mbar_wait(wbar, 0);
		if (!ok)
			give_up(abort_flag, p.err);
		tc_fence_after();
		long long n = 0;
		for (long long i = 0; ok && i < my_tiles && !aborted(abort_flag); i++)
		{
			const int a = (int)(i & 1);
			if (!mbar_wait(acc_empty + a, (uint32_t)(((i >> 1) & 1) ^ 1)))
			{
				give_up(abort_flag, p.err);
				break;
			}
			tc_fence_after();
			const uint32_t d = acc_col + (uint32_t)(a * SUR_C);
			for (int r = 0; r < 9; r++, n++)
			{
				const int s = (int)(n % CONV_STAGES);
				if (!mbar_wait(full + s, (uint32_t)((n / CONV_STAGES) & 1)))
				{
					give_up(abort_flag, p.err);
					ok = false;
					break;
				}
				tc_fence_after();
				const uint32_t a_addr = smem_addr(stages + s * A_STAGE_BYTES);
#pragma unroll
				for (int dx = 0; dx < 3; dx++)
				{
					const uint32_t b_addr = smem_addr(wsm + (3 * r + dx) * W_TAP_BYTES);
#pragma unroll
					for (int k = 0; k < 2; k++)
						umma_bf16(d, sw64_desc(a_addr + 64 * dx + 32 * k, 16, 512), sw64_desc(b_addr + 32 * k, 16, 512),
								  idesc, (r | dx | k) != 0);
				}
				umma_commit(empty + s); // the stage is free once these MMAs have read it
			}
			if (ok)
				umma_commit(acc_full + a);
		}
		// every MMA has completed before the tensor memory is freed
		umma_commit(drain);
		mbar_wait(drain, 0);
	}
	else if (role == 2)
	{
		// epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. +31, i.e. voxels x0 + 32 (w % 4) + lane
		const int q = warp & 3;
		const int m = q * 32 + lane;
		for (long long i = 0; i < my_tiles; i++)
		{
			if (aborted(abort_flag))
				break;
			const int a = (int)(i & 1);
			if (!mbar_wait(acc_full + a, (uint32_t)((i >> 1) & 1)))
			{
				give_up(abort_flag, p.err);
				break;
			}
			tc_fence_after();
			float v[32];
			tmem_ld32(acc_col + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * SUR_C), v);
			tc_fence_before();
			mbar_arrive(acc_empty + a);

			int b, z, y, x0;
			decode_tile(first + i * stride, p, b, z, y, x0);
			const int x = x0 + m;
			if (x >= p.X)
				continue;
			const long long vox = (((long long)b * p.Z + z) * p.Y + y) * p.X + x;
			if (p.bias)
			{
#pragma unroll
				for (int c = 0; c < 32; c++)
					v[c] += __ldg(&p.bias[c]);
			}
			if (p.residual)
			{
				float r[32];
				load_bf16x32(p.residual + vox * SUR_C, r);
#pragma unroll
				for (int c = 0; c < 32; c++)
					v[c] += r[c];
			}
			if (p.relu)
			{
#pragma unroll
				for (int c = 0; c < 32; c++)
					v[c] = fmaxf(v[c], 0.f);
			}
			if (p.mask)
			{
				float r[32];
				load_bf16x32(p.mask + vox * SUR_C, r);
#pragma unroll
				for (int c = 0; c < 32; c++)
					v[c] = r[c] > 0.f ? v[c] : 0.f;
			}
			if (p.out)
				store_bf16x32(p.out + vox * SUR_C, v);
			if (p.out_f32)
			{
#pragma unroll
				for (int c = 0; c < 32; c++)
					if (c < p.out_ch)
						p.out_f32[vox * p.out_ch + c] = v[c] + (p.base_f32 ? p.base_f32[vox * p.out_ch + c] : 0.f);
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == CONV_PIPES)
	{
		tc_fence_after();
		tmem_dealloc(tmem, 256);
	}
}

// ------------------------------------------------------------------------------------------------
// weight gradient: dW[t][co][ci] += sum_v dY[v][co] in[v + off_t][ci]
//
// A CTA owns one (dy, dz) row of the stencil, i.e. the three taps dx = -1, 0, +1, and a strided
// share of the 128-voxel rows of the mesh, split over WG_PIPES pipelines with their own
// accumulators.  For each voxel row a pipeline copies the 130 input voxels x0 - 1 .. x0 + 128 of
// row (y + dy, z + dz) and the 128 output-gradient voxels of row (y, z), and accumulates M128 N32
// K16 MMAs over the row: M = (dx, input channel), N = output channel, K = voxel.  Both operands are
// [voxels][32 channels] boxes read MN-major (the voxels along K, 8-row groups 512 bytes apart); the
// three dx taps are the same box one row (64 bytes) apart, so A's 32-channel groups of M start 64
// bytes apart (the fourth group, rows 96-127 of the accumulator, reads past the taps and is
// dropped).  At the end every pipeline adds its accumulator to dW with one atomic per weight.

static constexpr int WG_PIPES = 3;
static constexpr int WG_STAGES = 4;
static constexpr uint32_t WG_GRAD_OFFSET = A_STAGE_BYTES;					 // gradient box after the input box
static constexpr uint32_t WG_STAGE_BYTES = A_STAGE_BYTES + A_TILE_BYTES; // 17408 (17 x 1024)
static constexpr int WG_THREADS = 32 * (2 * WG_PIPES + 4 * WG_PIPES);
// barriers per pipeline: full and empty per stage, accumulator full, drain; then the tensor-memory
// address and the abort flag
static constexpr int WG_PIPE_BARS = 2 * WG_STAGES + 2;
static constexpr size_t WG_BAR_BYTES = WG_PIPES * WG_PIPE_BARS * sizeof(uint64_t) + 2 * sizeof(uint32_t);
static constexpr size_t WG_SMEM = 1024 + (size_t)WG_PIPES * WG_STAGES * WG_STAGE_BYTES + WG_BAR_BYTES;
static_assert(WG_SMEM <= 227 * 1024, "weight-gradient stages exceed the shared memory of a CTA");
// the dropped fourth M group reads rows 3 .. 130 of the input box: still inside the stage
static_assert((CONV_ROWS + 1) * SUR_C * 2 <= A_STAGE_BYTES, "wgrad input box overrun");

__global__ void __launch_bounds__(WG_THREADS, 1) sur_wgrad_kernel(const __grid_constant__ CUtensorMap act,
																   const __grid_constant__ CUtensorMap grad,
																   const __grid_constant__ conv_params p,
																   float* __restrict__ dW, int shares)
{
	extern __shared__ __align__(1024) unsigned char wg_smem[];
	unsigned char* base =
		reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(wg_smem) + 1023) & ~uintptr_t(1023));
	uint64_t* bars0 = reinterpret_cast<uint64_t*>(base + (size_t)WG_PIPES * WG_STAGES * WG_STAGE_BYTES);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars0 + WG_PIPES * WG_PIPE_BARS);
	volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

	const int row = blockIdx.x % 9; // (dy, dz) = (row % 3 - 1, row / 3 - 1): taps 3 row .. 3 row + 2
	const int share = blockIdx.x / 9;
	const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
	if (threadIdx.x == 0)
	{
		for (int q = 0; q < WG_PIPES; q++)
		{
			uint64_t* b = bars0 + q * WG_PIPE_BARS;
			for (int s = 0; s < WG_STAGES; s++)
			{
				mbar_init(b + s, 1);
				mbar_init(b + WG_STAGES + s, 1);
			}
			mbar_init(b + 2 * WG_STAGES, 1);	 // accumulator full
			mbar_init(b + 2 * WG_STAGES + 1, 1); // drain
		}
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == WG_PIPES)
	{
		tmem_alloc(tmem_slot, 128); // 32 columns per pipeline
		tmem_relinquish();
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tmem_slot;

	int role, pipe;
	if (warp < WG_PIPES)
	{
		role = 0;
		pipe = warp;
	}
	else if (warp < 2 * WG_PIPES)
	{
		role = 1;
		pipe = warp - WG_PIPES;
	}
	else
	{
		role = 2;
		pipe = (warp - 2 * WG_PIPES) / 4;
	}
	uint64_t* bars = bars0 + pipe * WG_PIPE_BARS;
	uint64_t* full = bars;
	uint64_t* empty = bars + WG_STAGES;
	uint64_t* acc_full = bars + 2 * WG_STAGES;
	uint64_t* drain = acc_full + 1;
	unsigned char* stages = base + (size_t)pipe * WG_STAGES * WG_STAGE_BYTES;
	const long long first = (long long)share * WG_PIPES + pipe;
	const long long stride = (long long)shares * WG_PIPES;
	const long long my_rows = first < p.tiles ? (p.tiles - first + stride - 1) / stride : 0;
	const uint32_t acc = tmem + (uint32_t)(pipe * SUR_C);
	const int dy = row % 3 - 1, dz = row / 3 - 1;

	if (role == 0 && lane == 0)
	{
		long long n = 0;
		for (long long i = 0; i < my_rows && !aborted(abort_flag); i++, n++)
		{
			int b, z, y, x0;
			decode_tile(first + i * stride, p, b, z, y, x0);
			const int s = (int)(n % WG_STAGES);
			if (!mbar_wait(empty + s, (uint32_t)(((n / WG_STAGES) & 1) ^ 1)))
			{
				give_up(abort_flag, p.err);
				break;
			}
			unsigned char* st = stages + s * WG_STAGE_BYTES;
			mbar_expect_tx(full + s, A_BOX_BYTES + A_TILE_BYTES);
			tma_load_5d(st, &act, 0, x0 - 1, y + dy, z + dz, b, full + s);
			tma_load_5d(st + WG_GRAD_OFFSET, &grad, 0, x0, y, z, b, full + s);
		}
		for (long long k = (n > WG_STAGES ? n - WG_STAGES : 0); k < n; k++)
			mbar_wait(full + k % WG_STAGES, (uint32_t)((k / WG_STAGES) & 1));
	}
	else if (role == 1 && lane == 0)
	{
		constexpr uint32_t idesc = idesc_bf16(SUR_TILE, SUR_C, true, true);
		bool ok = true;
		for (long long i = 0; i < my_rows && !aborted(abort_flag); i++)
		{
			const int s = (int)(i % WG_STAGES);
			if (!mbar_wait(full + s, (uint32_t)((i / WG_STAGES) & 1)))
			{
				give_up(abort_flag, p.err);
				ok = false;
				break;
			}
			tc_fence_after();
			const uint32_t a_addr = smem_addr(stages + s * WG_STAGE_BYTES);
			const uint32_t b_addr = a_addr + WG_GRAD_OFFSET;
#pragma unroll
			for (int k = 0; k < SUR_TILE / 16; k++) // 16 voxels (two 8-row groups, 1024 bytes) per MMA
				umma_bf16(acc, sw64_desc(a_addr + 1024 * k, 64, 512), sw64_desc(b_addr + 1024 * k, A_TILE_BYTES, 512),
						  idesc, (i | k) != 0);
			umma_commit(empty + s);
		}
		if (ok && my_rows > 0)
			umma_commit(acc_full);
		umma_commit(drain);
		mbar_wait(drain, 0);
	}
	else if (role == 2 && my_rows > 0)
	{
		const int q = warp & 3;
		const int m = q * 32 + lane; // tap 3 row + m / 32, input channel m % 32
		if (!aborted(abort_flag))
		{
			if (mbar_wait(acc_full, 0))
			{
				tc_fence_after();
				float v[32];
				tmem_ld32(acc + ((uint32_t)(q * 32) << 16), v);
				if (m < 3 * SUR_C)
				{
					const int t = 3 * row + m / 32, ci = m % 32;
#pragma unroll
					for (int co = 0; co < 32; co++)
						atomicAdd(&dW[((size_t)t * SUR_C + co) * SUR_C + ci], v[co]);
				}
			}
			else
				give_up(abort_flag, p.err);
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == WG_PIPES)
	{
		tc_fence_after();
		tmem_dealloc(tmem, 128);
	}
}

// ------------------------------------------------------------------------------------------------
// host side

static bool encode_act_map(CUtensorMap* map, const void* ptr, int X, int Y, int Z, int B, int rows = SUR_TILE)
{
	auto encode = tensor_map_encoder();
	if (!encode)
		return false;
	std::memset(map, 0, sizeof(*map));
	cuuint64_t dims[5] = { (cuuint64_t)SUR_C, (cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z, (cuuint64_t)B };
	const cuuint64_t row = SUR_C * 2;
	cuuint64_t strides[4] = { row, row * X, row * X * Y, row * X * Y * Z };
	cuuint32_t box[5] = { (cuuint32_t)SUR_C, (cuuint32_t)rows, 1, 1, 1 };
	cuuint32_t estr[5] = { 1, 1, 1, 1, 1 };
	return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(ptr), dims, strides, box, estr,
				  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
				  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
		   == CUDA_SUCCESS;
}

static bool encode_weight_map(CUtensorMap* map, const void* ptr)
{
	auto encode = tensor_map_encoder();
	if (!encode)
		return false;
	std::memset(map, 0, sizeof(*map));
	cuuint64_t dims[2] = { (cuuint64_t)SUR_C, (cuuint64_t)(SUR_TAPS * SUR_C) };
	cuuint64_t strides[1] = { SUR_C * 2 };
	cuuint32_t box[2] = { (cuuint32_t)SUR_C, (cuuint32_t)SUR_C };
	cuuint32_t estr[2] = { 1, 1 };
	return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
				  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
				  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
		   == CUDA_SUCCESS;
}

int sur_check_shape(int X, int Y, int Z, int B)
{
	if (X < SUR_TILE || Y < 1 || Z < 1 || B < 1)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "the surrogate's meshes need at least 128 voxels along x");
	if ((long long)X * Y * Z * B * SUR_C >= (1LL << 40))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "activation tensor too large");
	return BFVM_OK;
}

int launch_sur_conv(const __nv_bfloat16* in, const __nv_bfloat16* w, conv_params p, int device, cudaStream_t stream)
{
	int st;
	if ((st = sur_check_shape(p.X, p.Y, p.Z, p.B)))
		return st;
	CUtensorMap act, wmap;
	if (!encode_act_map(&act, in, p.X, p.Y, p.Z, p.B, CONV_ROWS) || !encode_weight_map(&wmap, w))
		return fail(BFVM_ERR_CUDA, "cuTensorMapEncodeTiled failed for a surrogate tensor");
	p.x_tiles = (p.X + SUR_TILE - 1) / SUR_TILE;
	p.tiles = (long long)p.x_tiles * p.Y * p.Z * p.B;
	if ((st = set_smem(sur_conv_kernel, CONV_SMEM)))
		return st;
	const long long grid =
		std::min<long long>((p.tiles + CONV_PIPES - 1) / CONV_PIPES, (long long)sm_count_impl(device));
	sur_conv_kernel<<<(unsigned)std::max(1LL, grid), CONV_THREADS, CONV_SMEM, stream>>>(act, wmap, p);
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? BFVM_OK : cuda_fail(e, "sur_conv_kernel");
}

int launch_sur_wgrad(const __nv_bfloat16* in, const __nv_bfloat16* grad, float* dW, conv_params p, int device,
					 cudaStream_t stream)
{
	int st;
	if ((st = sur_check_shape(p.X, p.Y, p.Z, p.B)))
		return st;
	CUtensorMap act, gmap;
	if (!encode_act_map(&act, in, p.X, p.Y, p.Z, p.B, CONV_ROWS) || !encode_act_map(&gmap, grad, p.X, p.Y, p.Z, p.B))
		return fail(BFVM_ERR_CUDA, "cuTensorMapEncodeTiled failed for a surrogate tensor");
	p.x_tiles = (p.X + SUR_TILE - 1) / SUR_TILE;
	p.tiles = (long long)p.x_tiles * p.Y * p.Z * p.B;
	if ((st = set_smem(sur_wgrad_kernel, WG_SMEM)))
		return st;
	const int sms = sm_count_impl(device);
	const int shares = (int)std::max<long long>(
		1, std::min<long long>((p.tiles + WG_PIPES - 1) / WG_PIPES, std::max(1, sms / 9)));
	sur_wgrad_kernel<<<9 * shares, WG_THREADS, WG_SMEM, stream>>>(act, gmap, p, dW, shares);
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? BFVM_OK : cuda_fail(e, "sur_wgrad_kernel");
}

} // namespace bfvm
