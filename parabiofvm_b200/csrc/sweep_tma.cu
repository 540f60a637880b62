// Sweeps with the field staged through shared memory by the Tensor Memory Accelerator.
//
// A persistent CTA owns a tile of 32 lines at a time: 32 adjacent columns of the x*s plane (y
// sweep) or of the y*x*s plane (z sweep), or R = 32/S whole rows (x sweep, R rows x S substrate
// lines).  Each warp group keeps up to four tiles in flight, one per shared-memory stage: a stage is
// refilled with the tile NST ahead as soon as the group holds its current tile in registers, so
// the HBM reads overlap the whole solve.
// Results are written straight from registers with coalesced stores (the x sweep of 16, 8 or 4
// substrates through a warp transpose, store_block_rows).  The Dirichlet overwrites run before and
// after the sweeps (dirichlet.cu; as options, the per-tile lists or the face conditions inside
// the sweeps), so this kernel is otherwise a pure line solve.  Instances also sweep the chunks of
// longer lines (chunks.cu) and the slabs of a split mesh (slab.cu), entering lines with carries.
//
// Lines use the front-padded partition of precompute.cpp: P blocks of exactly 32 elements, the
// first `pad` of them virtual (b' = 0, read as zeros from a front of the stage that the copies
// never write).  Warp j holds block j of every line of the tile (blockDim = (32, P)) and
//   1. runs the forward and the backward recurrence on its registers from zero carries,
//   2. barrier; folds the forward carries of the blocks to its left into C and publishes its
//      first element corrected by C,
//   3. barrier; folds those first elements of the blocks to its right into X and applies
//      x = t + C tg + X G with the precomputed responses tg and G.
// With P == 1 steps 2 and 3 vanish and the arithmetic is the reference's Thomas solve.
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

#include "sm100_common.cuh"
#include "sweep_common.cuh"

namespace bfvm {

struct tma_tile
{
	int axis;			 // 0 x (rows), 1 y, 2 z
	long long items;	 // tiles: this launch sweeps [first, items)
	long long first;
	long long ncols;	 // columns of the plane (y, z)
	long long col_tiles; // 32-column tiles per plane (y, z)
	long long outer_stride, line_stride;
	int box_h, nbox;	 // TMA boxes along the line (y, z)
	int R, row_pitch;	 // rows per tile and padded row length in floats (x)
	long long row_elems; // x: floats of a row that a tile stages (XS, or the chunk's part of it)
	int front;			 // x: floats before each staged row (holds its virtual front, 16-byte multiple)
	long long nrows;
	long long XS;
	int stage_floats;
	int groups; // warp groups per CTA, each solving its own tiles
	int stages; // pipeline depth of each group
	// zero-filled virtual fronts of a stage: `front_count` runs of `front_floats`, `front_pitch` apart
	int front_floats, front_count, front_pitch;
	// z tiles read with an L2 evict-first policy, so that the planes the sweep writes (which the
	// gradient inside it reads back) are the lines L2 keeps
	int evict_first;
	// with each refill, an L2 prefetch of the tile after it (option tma_prefetch)
	int prefetch;
	// y/z: two warp groups share each stage, which holds a pair of adjacent tiles (64 columns, one
	// TMA box row of 256 bytes per plane); slots = pairs then, else slots = items
	int pair;
	long long slots;
	// y: tile index / col_tiles as (umulhi(ct_magic, w) + w) >> ct_shift (Granlund and Montgomery,
	// "Division by invariant integers using multiplication", 1994: exact for w < 2^31)
	unsigned ct_magic;
	int ct_shift;
	// the equal chunks of longer lines in one launch (SLAB 2): CTA b sweeps chunk b % chunks, whose
	// elements start chunk_e0 elements along the line, chunk_e0 * e_stride floats into the field,
	// with the tables chunk_vtab
	int chunks;
	long long e_stride;
	long long chunk_e0[8];
	const float* chunk_vtab[8];
};

// Issue the copies of slot w (a tile, or with tt.pair the tile pair 2w, 2w + 1) into `dst`,
// completing on `bar` (one thread).  The line elements land after the virtual front: row rl of an
// x tile at rl * row_pitch + front, and the columns of a y/z slot from stage row `pad` on.
__device__ __forceinline__ void issue_tile(const sweep_args& a, const CUtensorMap* map, const tma_tile& tt, long long w,
										   float* dst, uint64_t* bar, long long coff = 0, int crow = 0)
{
	if (tt.axis == 0)
	{
		const long long row0 = w * tt.R;
		const int rows = (int)min((long long)tt.R, tt.nrows - row0);
		const uint32_t row_bytes = (uint32_t)(tt.row_elems * sizeof(float));
		mbar_expect_tx(bar, row_bytes * rows);
		if (w == a.drop_tile_copy)
			return; // test of the bounded wait: the barrier expects bytes that never come
		for (int r = 0; r < rows; r++)
			bulk_load(dst + r * tt.row_pitch + tt.front, a.data + coff + (row0 + r) * tt.XS, row_bytes, bar);
		return;
	}
	const int width = tt.pair ? 64 : 32;
	const long long t = tt.pair ? 2 * w : w; // first tile of the slot
	const long long outer = t / tt.col_tiles;
	const int c0 = (int)((t % tt.col_tiles) * 32);
	mbar_expect_tx(bar, (uint32_t)(tt.nbox * tt.box_h * width * sizeof(float)));
	if (t == a.drop_tile_copy || (tt.pair && t + 1 == a.drop_tile_copy))
		return; // test of the bounded wait: the barrier expects bytes that never come
	float* base = dst + a.pad * width;
	for (int b = 0; b < tt.nbox; b++)
	{
		if (tt.axis == 1)
			tma_load_3d(base + b * tt.box_h * width, map, c0, crow + b * tt.box_h, (int)outer, bar);
		else if (tt.evict_first)
			tma_load_2d_hint(base + b * tt.box_h * width, map, c0, crow + b * tt.box_h, bar, l2_evict_first_policy());
		else
			tma_load_2d(base + b * tt.box_h * width, map, c0, crow + b * tt.box_h, bar);
	}
}

// Where line `lane` of tile w lives: virtual element v at stage[sbase + v * sstride], real element
// i = v - pad at line[i * gstride] in the field.
struct tile_line
{
	bool active;
	int s, sbase, sstride;
	float* line;
	long long gstride;

	template <bool ROWS>
	__device__ __forceinline__ void locate(const sweep_args& a, const tma_tile& tt, long long w, int lane,
										   long long coff = 0)
	{
		const int S = a.S;
		if (ROWS)
		{
			const int rl = (32 % S == 0) ? lane >> (31 - __clz(S)) : lane / S;
			s = lane - rl * S;
			const long long row = w * tt.R + rl;
			active = rl < tt.R && row < tt.nrows;
			const long long rr = active ? row : 0;
			// lanes past the last row of the tile read row 0
			sbase = (rl < tt.R ? rl : 0) * tt.row_pitch + tt.front - a.pad * S + s;
			sstride = S;
			line = a.data + coff + rr * tt.XS + s;
			gstride = S;
		}
		else
		{
			// tile and column indices below 2^31 (launch_sweep_tma declines other shapes): 32-bit
			// divisions, several times cheaper than 64-bit ones, and this runs twice per tile
			// (the z sweep's tiles cover one plane; when S divides 32, a lane's substrate is fixed)
			const unsigned wu = (unsigned)w, ct = (unsigned)tt.col_tiles;
			const unsigned outer = tt.axis == 2 ? 0u : (__umulhi(tt.ct_magic, wu) + wu) >> tt.ct_shift;
			const unsigned q = (wu - outer * ct) * 32u + (unsigned)lane;
			active = q < (unsigned)tt.ncols;
			const unsigned qq = active ? q : 0u;
			s = (32 % S == 0) ? (lane & (S - 1)) : (int)(qq % (unsigned)S);
			sbase = lane;
			sstride = 32;
			line = a.data + coff + (long long)outer * tt.outer_stride + qq;
			gstride = tt.line_stride;
		}
	}
};

// Shared-memory tables of the padded partition: the per-element tables transposed to [S][NP],
// NP = 32P + 1, so that a thread reaches its substrate's column with immediate offsets and the
// substrates of a warp fall into distinct banks, and c.  The per-block tables (gq, tgp, Gp; a few
// hundred floats read only by the carry folds) stay in global memory and are served by L1.
__host__ __device__ __forceinline__ int staged_table_floats(int P, int S)
{
	const int NP = 32 * P + 1;
	return 3 * S * NP + S;
}

// Copy tile wn (if it exists) into a stage whose previous contents every thread has read.
// An L2 prefetch of tile w (no stage, no barrier): its reads start a tile earlier than its copy.
__device__ __forceinline__ void prefetch_tile(const sweep_args& a, const CUtensorMap* map, const tma_tile& tt, long long w)
{
	if (w >= tt.items)
		return;
	if (tt.axis == 0)
	{
		const long long row0 = w * tt.R;
		const int rows = (int)min((long long)tt.R, tt.nrows - row0);
		for (int r = 0; r < rows; r++)
			bulk_prefetch(a.data + (row0 + r) * tt.XS, (uint32_t)(tt.row_elems * sizeof(float)));
		return;
	}
	const long long outer = w / tt.col_tiles;
	const int c0 = (int)((w % tt.col_tiles) * 32);
	for (int b = 0; b < tt.nbox; b++)
	{
		if (tt.axis == 1)
			tma_prefetch_3d(map, c0, b * tt.box_h, (int)outer);
		else
			tma_prefetch_2d(map, c0, b * tt.box_h);
	}
}

__device__ __forceinline__ void refill(const sweep_args& a, const CUtensorMap& map, const tma_tile& tt, long long wn,
									   float* stage, uint64_t* bar, long long wstride, long long coff = 0, int crow = 0)
{
	if (wn >= tt.slots)
		return;
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	issue_tile(a, &map, tt, wn, stage, bar, coff, crow);
	if (tt.prefetch)
		prefetch_tile(a, &map, tt, wn + wstride);
}

// Barriers of one warp group (ids 1 + group; id 0 is the CTA-wide __syncthreads).
__device__ __forceinline__ void group_sync(int id, int nthreads)
{
	asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ bool group_sync_and(int id, int nthreads, bool pred)
{
	uint32_t r;
	asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
				 "selp.u32 %0, 1, 0, q;\n}"
				 : "=r"(r)
				 : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
				 : "memory");
	return r != 0;
}

// ROWS: x sweep (tiles of whole rows, runtime element stride S in the stage); otherwise y/z
// sweep (tiles of 32 columns, element stride 32).  CTA = (32, P, G) threads: G warp groups share
// the coefficient tables; group g solves its own tiles with its own stages and barriers, and warp
// j of a group holds block j (virtual elements 32j .. 32j+31) of the 32 lines of its tile.
// Global store of one solved element.  NOALLOC: without allocating the line in L1 (faster for the
// x and y sweeps; the z sweep, whose rows lie a whole plane apart, is faster with plain stores).
template <bool NOALLOC>
__device__ __forceinline__ void store_element(float* p, float v)
{
	if (NOALLOC)
		asm volatile("st.global.L1::no_allocate.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
	else
		*p = v;
}

// Stores of elements K.. of a register block at `p` + k * STRIDE floats, with the offsets as
// immediates of the store instructions (a stride fixed at compile time: the x sweep of SC
// substrates).
template <bool NOALLOC, int OFF>
__device__ __forceinline__ void store_element_at(float* p, float v)
{
	if (NOALLOC)
		asm volatile("st.global.L1::no_allocate.f32 [%0+%2], %1;" ::"l"(p), "f"(v), "n"(OFF * 4) : "memory");
	else
		p[OFF] = v;
}

template <bool NOALLOC, int STRIDE, int M, int K = 0>
__device__ __forceinline__ void store_block(float* p, const float (&d)[M])
{
	if constexpr (K < M)
	{
		store_element_at<NOALLOC, K * STRIDE>(p, d[K]);
		store_block<NOALLOC, STRIDE, M, K + 1>(p, d);
	}
}

// The x sweep of SC substrates (R = 32 / SC rows per tile): the stores of a block transposed
// across the warp, so that each store instruction writes 128 contiguous bytes of one row (R
// consecutive elements of its SC substrates) instead of SC * 4 bytes in each of R rows.  Lane
// L = g * SC + s holds row g, substrate s.  For each run of R elements K .. K + R - 1, a butterfly
// of log2 R shuffle stages turns lane (g, s)'s values v[m] = element K + m of row g into v[r] =
// element K + g of row r (substrate s), which row r's store then writes at lane L.  r0 points at
// element 0 of the block in row 0 plus the lane; rows are XS floats apart; `rows` of them exist.
template <bool NOALLOC, int SC, int M, int K = 0>
__device__ __forceinline__ void store_block_rows(float* r0, long long XS, float (&d)[M], int g, int rows)
{
	constexpr int R = 32 / SC;
	if constexpr (K < M)
	{
#pragma unroll
		for (int b = 1; b < R; b <<= 1)
		{
			const bool hi = (g & b) != 0;
#pragma unroll
			for (int m = 0; m < R; m++)
				if (!(m & b))
				{
					const float send = hi ? d[K + m] : d[K + m + b];
					const float got = __shfl_xor_sync(0xffffffffu, send, b * SC);
					if (hi)
						d[K + m] = got;
					else
						d[K + m + b] = got;
				}
		}
#pragma unroll
		for (int r = 0; r < R; r++)
			if (r < rows)
				store_element_at<NOALLOC, K * SC>(r0 + r * XS, d[K + r]);
		store_block_rows<NOALLOC, SC, M, K + R>(r0, XS, d, g, rows);
	}
}

// The Dirichlet entries of tile w (sweep_args::dir), written by the gthr threads of a warp group.
// The caller has ordered them after every store of the tile with a barrier of the group, so an
// entry's value replaces the solved one, as the overwrite after the sweep does.
__device__ __forceinline__ void overwrite_tile(const dirichlet_tiles& d, float* data, long long w, int gtid, int gthr)
{
	const int q1 = __ldg(&d.qoff[w + 1]);
	for (int e = __ldg(&d.qoff[w]) + gtid; e < q1; e += gthr)
		*reinterpret_cast<float4*>(data + __ldg(&d.qidx[e])) = __ldg(&d.qval[e]);
	const int s1 = __ldg(&d.soff[w + 1]);
	for (int e = __ldg(&d.soff[w]) + gtid; e < s1; e += gthr)
		data[__ldg(&d.sidx[e])] = __ldg(&d.sval[e]);
}

// One thread's share of a tile's Dirichlet entries held in registers: the run of four and the
// single element at position gtid of the tile's lists.  The sweep loads them a tile ahead of their
// use, so their latency hides behind the next tile's solve.
struct dir_regs
{
	int qi = -1, si = -1; // -1: no entry for this thread
	float4 qv;
	float sv = 0.f;

	__device__ __forceinline__ void load(const dirichlet_tiles& d, const int (&o)[4], int gtid)
	{
		qi = -1;
		si = -1;
		if (o[0] + gtid < o[1])
		{
			qi = __ldg(&d.qidx[o[0] + gtid]);
			qv = __ldg(&d.qval[o[0] + gtid]);
		}
		if (o[2] + gtid < o[3])
		{
			si = __ldg(&d.sidx[o[2] + gtid]);
			sv = __ldg(&d.sval[o[2] + gtid]);
		}
	}

	// these entries, then (rarely) those past one per thread of the group, straight from the lists
	__device__ __forceinline__ void store(const dirichlet_tiles& d, const int (&o)[4], float* data, int gtid,
										  int gthr) const
	{
		if (qi >= 0)
			*reinterpret_cast<float4*>(data + qi) = qv;
		if (si >= 0)
			data[si] = sv;
		for (int e = o[0] + gthr + gtid; e < o[1]; e += gthr)
			*reinterpret_cast<float4*>(data + __ldg(&d.qidx[e])) = __ldg(&d.qval[e]);
		for (int e = o[2] + gthr + gtid; e < o[3]; e += gthr)
			data[__ldg(&d.sidx[e])] = __ldg(&d.sval[e]);
	}
};

// The Dirichlet face conditions of one line, by its position (sweep_args::face_apply).  The
// reference writes the faces in the order x-min, x-max, y-min, y-max, z-min, z-max, a later face
// winning where faces meet.  A line along axis a meets the faces of a at its two ends (elements 0
// and n - 1) and lies wholly on a face of another axis or not at all; those faces order before a's
// faces or after them (which then also win at the ends).  The result is packed into one register,
// which the sweep holds through the solve: bits 0-1 the line's kind (0 on no conditioned face of
// another axis, 1 on one ordered before a's, 2 after), bits 2-3 whether a's min and max faces
// condition the substrate, bits 4-6 the face whose value the line takes.
template <bool ROWS>
__device__ __forceinline__ int face_code(const sweep_args& a, const tma_tile& tt, long long w, int lane, int s,
									 bool face_tile)
{
	const int m = __ldg(&a.face_bits[s]);
	const int ax = ROWS ? 0 : tt.axis;
	int code = ((m >> (2 * ax)) & 3) << 2;
	if (m == 0 || !face_tile)
		return code;
	long long c[3] = { 0, 0, 0 };
	if (ROWS)
	{
		const long long row = w * tt.R + lane / a.S;
		c[1] = row % a.Y;
		c[2] = row / a.Y;
	}
	else if (ax == 1)
	{
		const long long q = (w % tt.col_tiles) * 32 + lane;
		c[0] = q / a.S;
		c[2] = w / tt.col_tiles;
	}
	else
	{
		const long long q = w * 32 + lane;
		c[1] = q / tt.XS;
		c[0] = (q % tt.XS) / a.S;
	}
	const long long n[3] = { a.X, a.Y, a.Z };
	int lb = 0;
#pragma unroll
	for (int b = 0; b < 3; b++)
		if (b != ax)
			lb |= (c[b] == 0 ? 1 << (2 * b) : 0) | (c[b] == n[b] - 1 ? 2 << (2 * b) : 0);
	lb &= m;
	const int after = lb >> (2 * ax + 2), before = lb & ((1 << (2 * ax)) - 1);
	if (after)
		code |= 2 | ((31 - __clz(after) + 2 * ax + 2) << 4);
	else if (before)
		code |= 1 | ((31 - __clz(before)) << 4);
	return code;
}

// Write the face conditions of `code` into block j of the line (virtual elements 32j .. 32j + 31;
// real element 0 is virtual element pad of block 0, element n - 1 the last of block P - 1).
template <int M>
__device__ __forceinline__ void apply_faces(float (&d)[M], int code, const sweep_args& a, int axis, int s, int j,
											int P)
{
	if (code == 0)
		return;
	const int line = code & 3;
	if (line != 0)
	{
		const float lv = __ldg(&a.face_vals[(code >> 4) * a.S + s]);
#pragma unroll
		for (int k = 0; k < M; k++)
			d[k] = lv;
		if (line == 2)
			return;
	}
	if ((code & 4) && j == 0)
	{
		// element pad of the block, by a select per element: an indexed store would move the
		// block out of registers
		const float v = __ldg(&a.face_vals[(2 * axis) * a.S + s]);
#pragma unroll
		for (int k = 0; k < M; k++)
			asm("{\n\t.reg .pred p;\n\tsetp.eq.s32 p, %1, %2;\n\tselp.f32 %0, %3, %0, p;\n}"
				: "+f"(d[k])
				: "r"(k), "r"(a.pad), "f"(v));
	}
	if ((code & 8) && j == P - 1)
		d[M - 1] = __ldg(&a.face_vals[(2 * axis + 1) * a.S + s]);
}

// ------------------------------------------------------------------------------------------------
// the gradient inside the z sweep (grad_fuse in sweep_common.cuh)

__device__ __forceinline__ int ld_acquire(const int* p)
{
	int v;
	asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

// Tile t holds its final values: called by one thread after a barrier of its group that ordered
// every store of the tile (and the Dirichlet entries written over them).
__device__ __forceinline__ void publish_tile(const grad_fuse& f, long long t)
{
	__threadfence();
	asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(f.tile_done + t), "r"(1) : "memory");
}

// The gradient of z tile g: columns 32g .. 32g + 31 of the y*x*s plane over every plane, the same
// arithmetic as gradient.cu (bit for bit).  Thread (lane, j) of a group of P warps marches column
// 32g + lane over planes [j c, (j + 1) c), c = ceil(Z / P), GZU planes at a time with every load
// of those planes issued before their arithmetic, keeping u(z-1), u(z) in registers.  The field is
// read with ordinary loads after the neighbour tiles were acquired: a 128-byte line of a plane
// belongs to one tile, and no line is read before its tile is published, so L1 can only hold final
// values.  The three components are stored streaming.
static constexpr int GZU = 4;

__device__ __forceinline__ void gradient_tile(const grad_fuse& f, const float* u, long long g, int lane, int j, int P)
{
	const long long plane = (long long)f.Y * f.X * f.S;
	const long long q = g * 32 + lane;
	if (q >= plane)
		return;
	const int XS = f.X * f.S;
	const int y = (int)(q / XS);
	const int x = (int)(q - (long long)y * XS) / f.S;
	const int chunk = (f.Z + P - 1) / P;
	const int z0 = j * chunk;
	const int z1 = min(f.Z, z0 + chunk);
	if (z0 >= z1)
		return;
	const int xo_hi = x == f.X - 1 ? 0 : f.S, xo_lo = x == 0 ? 0 : f.S;
	const float fx = (x == 0 || x == f.X - 1) ? f.bx : f.cx;
	const int yo_hi = y == f.Y - 1 ? 0 : XS, yo_lo = y == 0 ? 0 : XS;
	const float fy = (y == 0 || y == f.Y - 1) ? f.by : f.cy;
	const bool hasx = f.X > 1, hasy = f.Y > 1;
	const float* p = u + (long long)z0 * plane + q;
	float* gp = f.g + (long long)z0 * plane + q;
	float prev = z0 > 0 ? p[-plane] : 0.f;
	float cur = *p;
	for (int z = z0; z < z1; z += GZU)
	{
		float nx[GZU], xa[GZU], xb[GZU], ya[GZU], yb[GZU];
#pragma unroll
		for (int k = 0; k < GZU; k++)
		{
			const int zz = z + k;
			const float* pk = p + (long long)k * plane;
			const bool in = zz < z1;
			nx[k] = (in && zz + 1 < f.Z) ? pk[plane] : 0.f;
			xa[k] = (in && hasx) ? pk[xo_hi] : 0.f;
			xb[k] = (in && hasx) ? pk[-xo_lo] : 0.f;
			ya[k] = (in && hasy) ? pk[yo_hi] : 0.f;
			yb[k] = (in && hasy) ? pk[-yo_lo] : 0.f;
		}
#pragma unroll
		for (int k = 0; k < GZU; k++)
		{
			const int zz = z + k;
			if (zz >= z1)
				break;
			const float next = zz + 1 < f.Z ? nx[k] : cur;
			const float gx = hasx ? __fmul_rn(__fsub_rn(xa[k], xb[k]), fx) : 0.f;
			const float gy = hasy ? __fmul_rn(__fsub_rn(ya[k], yb[k]), fy) : 0.f;
			float gz;
			if (zz == 0)
				gz = __fmul_rn(__fsub_rn(next, cur), f.bz);
			else if (zz == f.Z - 1)
				gz = __fmul_rn(__fsub_rn(cur, prev), f.bz);
			else
				gz = __fmul_rn(__fsub_rn(next, prev), f.cz);
			float* o = gp + (long long)k * plane;
			__stcs(o, gx);
			__stcs(o + f.total, gy);
			__stcs(o + 2 * f.total, gz);
			prev = cur;
			cur = next;
		}
		p += (long long)GZU * plane;
		gp += (long long)GZU * plane;
	}
}

// The same gradient four substrates at a time (S % 4 == 0), with 16-byte accesses: thread (lane, j)
// owns columns 32g + 4 (lane % 8) .. + 3, and the four lanes that share them (lane / 8) split warp
// j's planes between them.  Four times the bytes in flight per load of the scalar form.
static constexpr int GZU4 = 1;

__device__ __forceinline__ float4 grad4(float4 a, float4 b, float f)
{
	return make_float4(__fmul_rn(__fsub_rn(a.x, b.x), f), __fmul_rn(__fsub_rn(a.y, b.y), f),
					   __fmul_rn(__fsub_rn(a.z, b.z), f), __fmul_rn(__fsub_rn(a.w, b.w), f));
}

__device__ __forceinline__ void gradient_tile4(const grad_fuse& f, const float* u, long long g, int lane, int j, int P)
{
	const long long plane = (long long)f.Y * f.X * f.S;
	const long long q = g * 32 + 4 * (lane & 7);
	if (q >= plane)
		return;
	const int XS = f.X * f.S;
	const int y = (int)(q / XS);
	const int x = (int)(q - (long long)y * XS) / f.S;
	const int chunk = (f.Z + P - 1) / P;
	const int sub = (chunk + 3) / 4;
	const int zj = j * chunk, zj1 = min(f.Z, zj + chunk);
	const int z0 = zj + (lane >> 3) * sub;
	const int z1 = min(zj1, z0 + sub);
	if (z0 >= z1)
		return;
	const int xo_hi = x == f.X - 1 ? 0 : f.S, xo_lo = x == 0 ? 0 : f.S;
	const float fx = (x == 0 || x == f.X - 1) ? f.bx : f.cx;
	const int yo_hi = y == f.Y - 1 ? 0 : XS, yo_lo = y == 0 ? 0 : XS;
	const float fy = (y == 0 || y == f.Y - 1) ? f.by : f.cy;
	const bool hasx = f.X > 1, hasy = f.Y > 1;
	const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
	const float* p = u + (long long)z0 * plane + q;
	float* gp = f.g + (long long)z0 * plane + q;
	float4 prev = z0 > 0 ? *reinterpret_cast<const float4*>(p - plane) : zero;
	float4 cur = *reinterpret_cast<const float4*>(p);
	for (int z = z0; z < z1; z += GZU4)
	{
		float4 nx[GZU4], xa[GZU4], xb[GZU4], ya[GZU4], yb[GZU4];
#pragma unroll
		for (int k = 0; k < GZU4; k++)
		{
			const int zz = z + k;
			const float* pk = p + (long long)k * plane;
			const bool in = zz < z1;
			nx[k] = (in && zz + 1 < f.Z) ? *reinterpret_cast<const float4*>(pk + plane) : zero;
			xa[k] = (in && hasx) ? *reinterpret_cast<const float4*>(pk + xo_hi) : zero;
			xb[k] = (in && hasx) ? *reinterpret_cast<const float4*>(pk - xo_lo) : zero;
			ya[k] = (in && hasy) ? *reinterpret_cast<const float4*>(pk + yo_hi) : zero;
			yb[k] = (in && hasy) ? *reinterpret_cast<const float4*>(pk - yo_lo) : zero;
		}
#pragma unroll
		for (int k = 0; k < GZU4; k++)
		{
			const int zz = z + k;
			if (zz >= z1)
				break;
			const float4 next = zz + 1 < f.Z ? nx[k] : cur;
			const float4 gx = hasx ? grad4(xa[k], xb[k], fx) : zero;
			const float4 gy = hasy ? grad4(ya[k], yb[k], fy) : zero;
			float4 gz;
			if (zz == 0)
				gz = grad4(next, cur, f.bz);
			else if (zz == f.Z - 1)
				gz = grad4(cur, prev, f.bz);
			else
				gz = grad4(next, prev, f.cz);
			float* o = gp + (long long)k * plane;
			__stcs(reinterpret_cast<float4*>(o), gx);
			__stcs(reinterpret_cast<float4*>(o + f.total), gy);
			__stcs(reinterpret_cast<float4*>(o + 2 * f.total), gz);
			prev = cur;
			cur = next;
		}
		p += (long long)GZU4 * plane;
		gp += (long long)GZU4 * plane;
	}
}

// Whether the tiles holding the x and y neighbours of tile g (and g itself) are published: the
// group's threads each watch some of them, for at most spin_limit cycles.
__device__ __forceinline__ bool neighbours_ready(const grad_fuse& f, long long g, int gtid, int gthr, int bar_id)
{
	const long long plane = (long long)f.Y * f.X * f.S;
	const long long XS = (long long)f.X * f.S;
	const long long c0 = g * 32, c1 = min(c0 + 31, plane - 1);
	const long long lo[3] = { c0 - f.S, c0 - XS, c0 + XS }, hi[3] = { c1 + f.S, c1 - XS, c1 + XS };
	long long first[3];
	int count[3], total = 0;
	for (int r = 0; r < 3; r++)
	{
		const long long a = max(lo[r], 0LL), b = min(hi[r], plane - 1);
		first[r] = a >> 5;
		count[r] = a > b ? 0 : (int)((b >> 5) - (a >> 5) + 1);
		total += count[r];
	}
	bool ok = true;
	for (int k = gtid; k < total; k += gthr)
	{
		const long long t = k < count[0] ? first[0] + k
										 : (k < count[0] + count[1] ? first[1] + (k - count[0])
																	: first[2] + (k - count[0] - count[1]));
		const long long start = clock64();
		while (ld_acquire(f.tile_done + t) == 0)
		{
			if (clock64() - start > f.spin_limit)
			{
				ok = false;
				break;
			}
			__nanosleep(100);
		}
	}
	return group_sync_and(bar_id, gthr, ok);
}

// The gradient of tile g by a group: now if its neighbours are published, else left to
// grad_deferred_kernel.  VEC: the four-substrate form (S % 4 == 0).
template <bool VEC>
__device__ __forceinline__ void gradient_work(const grad_fuse& f, const float* u, long long g, int lane, int j, int P,
											  int bar_id)
{
	const int gtid = lane + 32 * j, gthr = 32 * P;
	if (!neighbours_ready(f, g, gtid, gthr, bar_id))
	{
		if (gtid == 0)
		{
			const int k = atomicAdd(f.deferred, 1);
			f.deferred[1 + k] = (int)g;
		}
	}
	else if (VEC)
		gradient_tile4(f, u, g, lane, j, P);
	else
		gradient_tile(f, u, g, lane, j, P);
}

// The tiles whose gradient the sweep left behind, after the sweep: CTAs of (32, P) threads.
__global__ void __launch_bounds__(512) grad_deferred_kernel(const __grid_constant__ grad_fuse f, const float* u)
{
	const int n = *(volatile int*)f.deferred;
	for (int k = blockIdx.x; k < n; k += gridDim.x)
	{
		if (f.S % 4 == 0)
			gradient_tile4(f, u, f.deferred[1 + k], threadIdx.x, threadIdx.y, blockDim.y);
		else
			gradient_tile(f, u, f.deferred[1 + k], threadIdx.x, threadIdx.y, blockDim.y);
	}
}

// SLAB: 0 a plain sweep; 1 the solve pass of a z-slab or of a chunk of longer lines
// (line_chunks), which enters every line with the carries C (left) and X (right) of slab_carry: it
// always runs the carry folds, from C and X instead of zero, with the tables of
// precompute_padded_range; 2 the same for all the equal chunks of longer lines in one launch, the
// CTAs split among the chunks (tma_tile::chunks).
// GRAD (z sweep, P > 1): the gradient of the step inside the sweep (grad_fuse); 1 the scalar form,
// 4 the four-substrate form (S % 4 == 0).
// PAIR (y/z, plain sweeps only): groups 2u and 2u + 1 share their stages, each slot a pair of tiles
// of which group 2u + h solves tile 2 * slot + h; the group that finishes reading a stage second
// refills it (a counter per stage in shared memory, arrivals acquire-release ordered).
// MODE: 0 the plain sweep, 1 with the per-tile Dirichlet lists (sweep_args::dir), 2 with the face
// conditions by position (sweep_args::face_apply); separate instances, so the plain sweep holds no
// registers for either.
// SC (x sweep): the substrate count when the launch fixes it at compile time (0: read at run time),
// so that the element strides in shared and global memory become immediate offsets.
template <bool ROWS, bool NOALLOC, int SLAB, int GRAD, int MODE, bool PAIR, int SC = 0>
__global__ void __launch_bounds__(640, 1)
	sweep_tma_kernel(const __grid_constant__ sweep_args a, const __grid_constant__ CUtensorMap map,
					 const __grid_constant__ tma_tile tt, const __grid_constant__ grad_fuse gf)
{
	constexpr int M = 32;
	extern __shared__ __align__(128) unsigned char smem_raw[];
	// G * NST stages on a 128-byte boundary (TMA destinations), then tables, carries, barriers
	const int NST = tt.stages;
	const int G = tt.groups;
	const int U = PAIR ? G / 2 : G; // stage owners: groups, or pairs of groups
	float* const stages0 = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
	const int S = a.S;
	const int P = a.vP;
	const int N = 32 * P;
	const int NP = N + 1;
	// SLAB 2: this CTA's chunk, its place among the chunk's CTAs, offsets, tables and carries
	const int kc = SLAB == 2 ? (int)(blockIdx.x % tt.chunks) : 0;
	const long long cta = SLAB == 2 ? blockIdx.x / tt.chunks : blockIdx.x;
	const long long ncta = SLAB == 2 ? gridDim.x / tt.chunks : gridDim.x;
	const long long coff = SLAB == 2 ? tt.chunk_e0[kc] * tt.e_stride : 0;
	const int crow = SLAB == 2 ? (int)tt.chunk_e0[kc] : 0;
	const float* const vtab = SLAB == 2 ? tt.chunk_vtab[kc] : a.vtab;
	const float* const carry_in = SLAB == 2 ? a.slab_carry + (size_t)kc * 2 * a.slab_lines : a.slab_carry;
	float* tab = stages0 + (size_t)U * NST * tt.stage_floats;
	float2* tgtab = reinterpret_cast<float2*>(tab); // [S][NP] (tg, G)
	float* btab = tab + 2 * S * NP;					// [S][NP] b'
	float* ctab = btab + S * NP;					// [S]
	const float* gqtab = vtab + (size_t)3 * N * S + S; // [P][S], global
	const float* tgptab = gqtab + P * S;				 // [P][S], global
	const float* Gptab = tgptab + P * S;				 // [P][S], global
	float* carries = tab + staged_table_floats(P, S); // [G][2][P][32]
	uint64_t* bars0 = reinterpret_cast<uint64_t*>(
		(reinterpret_cast<uintptr_t>(carries + (size_t)G * 2 * P * 32) + 7) & ~uintptr_t(7)); // [U][NST]
	unsigned* const pair_count = reinterpret_cast<unsigned*>(bars0 + U * NST);			   // [U][NST] (PAIR)

	const int lane = threadIdx.x;
	const int j = threadIdx.y;
	const int g = threadIdx.z;
	const int tid = lane + 32 * (j + P * g);
	const int nthr = 32 * P * G;
	const int gthr = 32 * P; // threads of a group
	const int bar_id = 1 + g;
	const bool leader = lane == 0 && j == 0; // of the group
	const int u = PAIR ? g >> 1 : g;
	const int h = PAIR ? g & 1 : 0;
	float* const stages = stages0 + (size_t)u * NST * tt.stage_floats;
	uint64_t* const bars = bars0 + u * NST;
	float* const carry_f = carries + (size_t)g * 2 * P * 32;
	float* const carry_t = carry_f + P * 32;

	if (tid == 0)
	{
		for (int k = 0; k < U * NST; k++)
		{
			mbar_init(&bars0[k], 1);
			if (PAIR)
				pair_count[k] = 0;
		}
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	{
		// tables: global [v][S] -> shared [S][NP]
		const float* gb = vtab;
		const float2* gt = reinterpret_cast<const float2*>(vtab + (size_t)N * S);
		for (int t = tid; t < N * S; t += nthr)
		{
			const int v = t / S, s = t - v * S;
			btab[s * NP + v] = gb[t];
			tgtab[s * NP + v] = gt[t];
		}
		const float* gr = vtab + (size_t)3 * N * S;
		for (int t = tid; t < S; t += nthr)
			ctab[t] = gr[t];
		// the virtual fronts read as zeros; the copies never write them
		for (int k = 0; k < U * NST; k++)
			for (int r = 0; r < tt.front_count; r++)
				for (int t = tid; t < tt.front_floats; t += nthr)
					stages0[(size_t)k * tt.stage_floats + r * tt.front_pitch + t] = 0.f;
	}
	__syncthreads(); // also publishes the barrier init

	// slots of this stage owner: sl0, sl0 + slstride, ...; this group's tiles w0, w0 + wstride, ...
	const long long sl0 = (PAIR ? tt.first / 2 : tt.first) + cta * U + u;
	const long long slstride = ncta * U;
	const long long w0 = PAIR ? 2 * sl0 + h : sl0;
	const long long wstride = PAIR ? 2 * slstride : slstride;

	// prologue: the first NST slots, one per stage
	if (leader && h == 0)
	{
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		for (int k = 0; k < NST; k++)
		{
			const long long sk = sl0 + (long long)k * slstride;
			if (sk < tt.slots)
				issue_tile(a, &map, tt, sk, stages + (size_t)k * tt.stage_floats, &bars[k], coff, crow);
		}
	}

	const int p = 32 * j;
	bool failed = false;
	int it = 0;
	long long w = w0, sl = sl0;
	// the Dirichlet entries of the previous tile (written after the first barrier of this one):
	// their list offsets, loaded an iteration before the entries, and the entries themselves
	int dir_prev[4] = { 0, 0, 0, 0 };
	dir_regs dir_hold;
	constexpr bool DIR = MODE == 1;
	constexpr bool FACES = MODE == 2 && SLAB == 0 && GRAD == 0;
	int face_tile_next = (FACES && a.face_apply && w < tt.items) ? __ldg(&a.face_tiles[w]) : 0;
	// stage st = it % NST and its phase parity (it / NST) & 1, advanced without divisions
	int st = 0;
	uint32_t parity = 0;
	for (; w < tt.items; w += wstride, sl += slstride, it++, st = st + 1 == NST ? 0 : st + 1, parity ^= st == 0 ? 1u : 0u)
	{
		int dir_cur[4] = { 0, 0, 0, 0 };
		if (DIR && a.dir.items > 0)
		{
			if (it > 0)
				dir_hold.load(a.dir, dir_prev, lane + 32 * j);
			dir_cur[0] = __ldg(&a.dir.qoff[w]);
			dir_cur[1] = __ldg(&a.dir.qoff[w + 1]);
			dir_cur[2] = __ldg(&a.dir.soff[w]);
			dir_cur[3] = __ldg(&a.dir.soff[w + 1]);
		}

		const float* cur = stages + (size_t)st * tt.stage_floats;
		int s, sbase, sstride;
		{
			tile_line tl;
			tl.template locate<ROWS>(a, tt, w, lane, coff);
			s = tl.s;
			sbase = PAIR ? tl.sbase + 32 * h : tl.sbase;
			sstride = ROWS ? (SC ? SC : tl.sstride) : (PAIR ? 64 : 32);
		}
		// the line's face conditions, looked up while the tile's copy is in flight
		// (face_tiles[w] was loaded a tile ahead, so its latency hides behind the previous tile)
		int faces = 0;
		if (FACES && a.face_apply)
		{
			const bool ftile = face_tile_next != 0;
			face_tile_next = w + wstride < tt.items ? __ldg(&a.face_tiles[w + wstride]) : 0;
			faces = face_code<ROWS>(a, tt, w, lane, s, ftile);
		}
		// SLAB: the line's carries, loaded while the tile's copy is in flight.  Lines: x, row * S + s;
		// y, plane * X * S + column; z, column of the y*x*s plane
		float slab_c = 0.f, slab_x = 0.f;
		if (SLAB != 0)
		{
			long long lid;
			bool active;
			if (ROWS)
			{
				const int rl = lane / S;
				const long long row = w * tt.R + rl;
				active = rl < tt.R && row < tt.nrows;
				lid = row * S + (lane - rl * S);
			}
			else
			{
				const unsigned wu = (unsigned)w, ct = (unsigned)tt.col_tiles;
				const unsigned outer = tt.axis == 2 ? 0u : (__umulhi(tt.ct_magic, wu) + wu) >> tt.ct_shift;
				const unsigned q = (wu - outer * ct) * 32u + (unsigned)lane;
				active = q < (unsigned)tt.ncols;
				lid = (long long)outer * tt.ncols + q;
			}
			if (active)
			{
				slab_c = __ldg(&carry_in[lid]);
				slab_x = __ldg(&carry_in[a.slab_lines + lid]);
			}
		}
		const bool ok = mbar_wait(&bars[st], parity, a.wait_limit);

		const float cs = ctab[s];
		const float* bcol = btab + s * NP + p; // b' of this block: bcol[k]
		float d[M];
		{
			const float* src = cur + sbase + p * sstride;
#pragma unroll
			for (int k = 0; k < M; k++)
				d[k] = src[k * sstride];
		}
		// forward elimination from a zero carry: f_v = d_v - e_{v-1} f_{v-1}, with e = c b' the
		// float product the reference stores
#pragma unroll
		for (int k = 1; k < M; k++)
			d[k] = __fsub_rn(d[k], __fmul_rn(__fmul_rn(cs, bcol[k - 1]), d[k - 1]));
		carry_f[j * 32 + lane] = d[M - 1];
		// backward substitution from a zero carry: t_q = f_q b'_q, t_v = (f_v - c t_{v+1}) b'_v
		d[M - 1] = __fmul_rn(d[M - 1], bcol[M - 1]);
#pragma unroll
		for (int k = M - 2; k >= 0; k--)
			d[k] = __fmul_rn(__fsub_rn(d[k], __fmul_rn(cs, d[k + 1])), bcol[k]);

		if (!group_sync_and(bar_id, gthr, ok))
		{
			failed = true;
			break;
		}
		// every thread of the group holds its elements of this tile in registers now (they were
		// consumed by the recurrences before the barrier): refill the stage with the tile NST
		// ahead, so NST tiles stay in flight through the rest of this tile's solve
		if (leader)
		{
			bool last_reader = true;
			if (PAIR)
			{
				// the second group of the pair to finish reading the stage refills it
				unsigned old;
				asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;"
							 : "=r"(old)
							 : "r"(smem_addr(&pair_count[u * NST + st]))
							 : "memory");
				last_reader = (old & 1) != 0;
			}
			if (last_reader)
				refill(a, map, tt, sl + (long long)NST * slstride, stages + (size_t)st * tt.stage_floats, &bars[st],
					   wstride, coff, crow);
		}
		// the barrier also ordered the previous tile's stores: its Dirichlet entries go on top
		if (DIR && a.dir.items > 0 && it > 0)
			dir_hold.store(a.dir, dir_prev, a.data, lane + 32 * j, gthr);

		if (SLAB != 0)
		{
			float C = slab_c, Xc = slab_x;
			// C_k = f^{k-1}_q + gq_{k-1} C_{k-1} from C_0 = the slab's left carry
			for (int k = 0; k < j; k++)
				C = fmaf(__ldg(&gqtab[k * S + s]), C, carry_f[k * 32 + lane]);
			carry_t[j * 32 + lane] = fmaf(C, __ldg(&tgptab[j * S + s]), d[0]);
			group_sync(bar_id, gthr);
			// X_k = x^{k+1}_p + Gp_{k+1} X_{k+1} from X_{P-1} = the slab's right carry
			for (int k = P - 1; k > j; k--)
				Xc = fmaf(__ldg(&Gptab[k * S + s]), Xc, carry_t[k * 32 + lane]);
			const float2* tcol = tgtab + s * NP + p;
#pragma unroll
			for (int k = 0; k < M; k++)
			{
				const float2 r = tcol[k];
				d[k] = fmaf(Xc, r.y, fmaf(C, r.x, d[k]));
			}
		}
		else if (P > 1)
		{
			// left carry C = d'_{p-1}: fold the blocks to the left, C_k = f^k_q + gq_k C_{k-1}
			float C = 0.f;
			if (j > 0)
			{
				C = carry_f[lane];
				for (int k = 1; k < j; k++)
					C = fmaf(__ldg(&gqtab[k * S + s]), C, carry_f[k * 32 + lane]);
			}
			// this block's first solution element without the right carry
			carry_t[j * 32 + lane] = fmaf(C, __ldg(&tgptab[j * S + s]), d[0]);
			group_sync(bar_id, gthr);
			// the previous tile's stores (before the first barrier) and its Dirichlet entries
			// (before this one) are all done
			if (GRAD && leader && it > 0)
				publish_tile(gf, w - wstride);
			// right carry X = x_{q+1}: fold the blocks to the right, X_k = x^k_p + Gp_k X_{k+1}
			float Xc = 0.f;
			if (j < P - 1)
			{
				Xc = carry_t[(P - 1) * 32 + lane];
				for (int k = P - 2; k > j; k--)
					Xc = fmaf(__ldg(&Gptab[k * S + s]), Xc, carry_t[k * 32 + lane]);
			}
			const float2* tcol = tgtab + s * NP + p;
#pragma unroll
			for (int k = 0; k < M; k++)
			{
				const float2 r = tcol[k];
				d[k] = fmaf(Xc, r.y, fmaf(C, r.x, d[k]));
			}
		}

		if (FACES && a.face_apply) // the overwrite after this sweep
			apply_faces(d, faces, a, ROWS ? 0 : tt.axis, s, j, P);
		{
			// recompute the line from an opaque copy of the tile index, so nothing of the load
			// phase stays live across the solve
			long long w2;
			asm volatile("mov.b64 %0, %1;" : "=l"(w2) : "l"(w));
			tile_line tl2;
			tl2.template locate<ROWS>(a, tt, w2, lane, coff);
			if (ROWS && SC >= 4 && (j > 0 || a.pad == 0))
			{
				// every lane takes part in the shuffles; the rows' existence predicates the stores
				constexpr int R = SC ? 32 / SC : 1;
				const long long row0 = w2 * R;
				float* r0 = a.data + coff + row0 * tt.XS + (long long)(p - a.pad) * SC + lane;
				const int rows = (int)min((long long)R, tt.nrows - row0);
				store_block_rows<NOALLOC, (SC ? SC : 32)>(r0, tt.XS, d, lane / (SC ? SC : 32), rows);
			}
			else if (tl2.active)
			{
				if ((j > 0 || a.pad == 0) && ROWS && SC)
					store_block<NOALLOC, SC>(tl2.line + (long long)(p - a.pad) * SC, d);
				else if (j > 0 || a.pad == 0)
				{
					float* ptr = tl2.line + (long long)(p - a.pad) * tl2.gstride;
#pragma unroll
					for (int k = 0; k < M; k++)
					{
						store_element<NOALLOC>(ptr, d[k]);
						ptr += tl2.gstride;
					}
				}
				else
				{
					// block 0 of a padded line: the first `pad` elements are virtual
					float* ptr = tl2.line;
#pragma unroll
					for (int k = 0; k < M; k++)
						if (k >= a.pad)
						{
							store_element<NOALLOC>(ptr, d[k]);
							ptr += tl2.gstride;
						}
				}
			}
		}
		if (GRAD && w >= gf.lag)
			gradient_work<GRAD == 4>(gf, a.data, w - gf.lag, lane, j, P, bar_id);
#pragma unroll
		for (int k = 0; k < 4; k++)
			dir_prev[k] = dir_cur[k];
	}

	if (DIR && !failed && a.dir.items > 0 && it > 0)
	{
		group_sync(bar_id, gthr); // the last tile's stores, then its entries
		overwrite_tile(a.dir, a.data, w - wstride, lane + 32 * j, gthr);
	}
	if (GRAD && !failed)
	{
		if (it > 0)
		{
			group_sync(bar_id, gthr);
			if (leader)
				publish_tile(gf, w - wstride);
		}
		// the gradients still owed: tiles w - lag of this group's stride past the last tile
		for (; w - gf.lag < tt.items; w += wstride)
			if (w >= gf.lag)
				gradient_work<GRAD == 4>(gf, a.data, w - gf.lag, lane, j, P, bar_id);
	}
	if (failed && leader)
	{
		atomicOr(a.err, DEVERR_TIMEOUT);
		// let the copies already issued (slots sl .. sl + (NST-1) * stride) land before the CTA
		// exits (bounded waits)
		for (int k = 0; k < NST; k++)
		{
			const long long sk = sl + (long long)k * slstride;
			if (sk < tt.slots)
				mbar_wait(&bars[(it + k) % NST], (uint32_t)(((it + k) / NST) & 1), a.wait_limit);
		}
	}
}

// ------------------------------------------------------------------------------------------------
// host side

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
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

// The tensor map of a y sweep (3D over [Z][n][XS] from `base`, planes Y * XS apart) or a z sweep
// (2D over [n][Y*XS]): boxes of `width` columns x box_h rows; n is the line length of the launch
// (Y or Z, or a chunk's).
static CUresult encode_box(PFN_cuTensorMapEncodeTiled_v12000 encode, CUtensorMap& map, int axis, float* base,
						   long long X, long long Y, long long Z, long long S, long long n, int width, int box_h)
{
	const long long XS = X * S;
	cuuint64_t dims[3], strides[2];
	cuuint32_t box[3], estr[3] = { 1, 1, 1 };
	cuuint32_t rank;
	if (axis == 1)
	{
		rank = 3;
		dims[0] = (cuuint64_t)XS;
		dims[1] = (cuuint64_t)n;
		dims[2] = (cuuint64_t)Z;
		strides[0] = (cuuint64_t)(XS * sizeof(float));
		strides[1] = (cuuint64_t)(Y * XS * sizeof(float));
		box[0] = (cuuint32_t)width;
		box[1] = (cuuint32_t)box_h;
		box[2] = 1;
	}
	else
	{
		rank = 2;
		dims[0] = (cuuint64_t)(Y * XS);
		dims[1] = (cuuint64_t)n;
		strides[0] = (cuuint64_t)(Y * XS * sizeof(float));
		box[0] = (cuuint32_t)width;
		box[1] = (cuuint32_t)box_h;
	}
	return encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, base, dims, strides, box, estr,
				  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
				  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

template <bool ROWS, bool NOALLOC, int SLAB = 0, int GRAD = 0, int MODE = 0, bool PAIR = false, int SC = 0>
static int launch_tma_variant(bfvm_solver* st, const sweep_args& a, const CUtensorMap& map, const tma_tile& tt,
							  size_t smem, const grad_fuse* gfp = nullptr)
{
	auto kernel = sweep_tma_kernel<ROWS, NOALLOC, SLAB, GRAD, MODE, PAIR, SC>;
	int rc = set_smem(kernel, smem);
	if (rc)
		return rc;
	const int threads = 32 * a.vP * tt.groups;
	// one CTA per G tiles (per G / 2 slots of two tiles when paired); chunks in one launch (SLAB 2)
	// split the resident CTAs evenly among them
	int grid =
		persistent_grid(kernel, threads, smem, (tt.items - tt.first + tt.groups - 1) / tt.groups, st->device);
	if (SLAB == 2)
	{
		const int resident = persistent_grid(kernel, threads, smem, 1LL << 40, st->device);
		const long long per_chunk = std::max<long long>(
			1, std::min<long long>(resident / tt.chunks, (tt.items + tt.groups - 1) / tt.groups));
		grid = (int)(per_chunk * tt.chunks);
	}
	grad_fuse gf;
	std::memset(&gf, 0, sizeof(gf));
	if (GRAD)
	{
		gf = *gfp;
		// lag: the widest neighbour reach in tiles (a row of the y*x*s plane, plus S) and two
		// strides of the persistent groups, so the neighbours are normally published in time
		const long long XS = (long long)gf.X * gf.S;
		const long long reach = (XS + gf.S + 31) / 32 + 1;
		gf.lag = reach + 2LL * grid * tt.groups + 32;
		BFVM_CUDA(cudaMemsetAsync(gf.tile_done, 0, (size_t)tt.items * sizeof(int), st->stream));
		BFVM_CUDA(cudaMemsetAsync(gf.deferred, 0, sizeof(int), st->stream));
	}
	kernel<<<grid, dim3(32, a.vP, tt.groups), smem, st->stream>>>(a, map, tt, gf);
	rc = check_launch(st, tt.axis == 0 ? "sweep_tma<x>"
									   : (tt.axis == 1 ? "sweep_tma<y>" : (SLAB ? "sweep_tma<z slab>" : "sweep_tma<z>")));
	if (rc || !GRAD)
		return rc;
	grad_deferred_kernel<<<sm_count_impl(st->device) * 2, dim3(32, a.vP), 0, st->stream>>>(gf, a.data);
	return check_launch(st, "grad_deferred_kernel");
}

// tune: launch shape to use (groups 0: the built-in choice).  shapes: when given, nothing is
// launched; the launch shapes that fit are listed instead.
int launch_sweep_tma(bfvm_solver* st, int axis, const sweep_args& a_in, bool& handled, const sweep_tuning* tune,
					 std::vector<sweep_tuning>* shapes, bool slab_solve, const grad_fuse* gf, long long w_begin,
					 long long w_end, const line_chunks* chunk)
{
	if (slab_solve && axis != 2)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "slab passes exist for the z sweep only");
	if ((w_begin != 0 || w_end >= 0) && (slab_solve || gf || chunk))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "a range of tiles is swept only by the plain staged sweeps");
	if (chunk && (slab_solve || gf))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "a chunk of the lines is swept by the plain staged sweeps only");
	handled = false;
	const long long X = st->grid[0], Y = st->grid[1], Z = st->grid[2], S = st->S;
	const long long XS = X * S;
	// the line length of this launch, and for a chunk its field view, tables and carries
	const long long n_line = chunk ? chunk->len : st->grid[axis];
	sweep_args a = a_in;
	float* base = st->dens;
	if (chunk)
	{
		if (chunk->count < 1 || chunk->count > 8)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "1 to 8 chunks per launch");
		a.data = st->dens;
		a.n = (int)chunk->len;
		a.vtab = chunk->vtab[0];
		a.vP = chunk->vP;
		a.pad = chunk->pad;
		a.slab_carry = chunk->carry;
		a.slab_lines = chunk->lines;
		// an x chunk's part of a row is one bulk copy: it must start and end on 16-byte boundaries
		for (int k = 0; k < chunk->count; k++)
			if (axis == 0 && ((chunk->e0[k] * S) % 4 != 0 || (chunk->len * S) % 4 != 0))
				return BFVM_OK;
	}
	// shapes the TMA path covers: 16-byte row strides, at most 16 blocks of 32 per line, and for
	// the x sweep whole rows of at most 32 substrate lines per tile
	if (!a.vtab || a.vP > TMA_MAX_P || XS % 4 != 0 || (axis == 0 && S > 32) || a.n < 2)
		return BFVM_OK;
	auto encode = tensor_map_encoder();
	if (!encode)
		return BFVM_OK;

	tma_tile tt;
	std::memset(&tt, 0, sizeof(tt));
	tt.axis = axis;
	tt.XS = XS;
	tt.row_elems = n_line * S;
	CUtensorMap map;
	std::memset(&map, 0, sizeof(map));
	if (axis == 0)
	{
		tt.R = (int)(32 / S);
		tt.nrows = Y * Z;
		tt.items = (tt.nrows + tt.R - 1) / tt.R;
		// each staged row: the virtual front rounded up to 16 bytes, the row, and padding so that
		// lane (r, s) -> r * pitch + s spreads over the banks
		tt.front = (int)((a.pad * S + 3) / 4 * 4);
		int bank = (int)(((S - tt.front - tt.row_elems) % 32 + 64) % 32);
		bank = (bank + 3) / 4 * 4;
		tt.row_pitch = tt.front + (int)tt.row_elems + bank;
		tt.stage_floats = (tt.R * tt.row_pitch + 31) / 32 * 32;
		tt.front_floats = tt.front;
		tt.front_count = tt.R;
		tt.front_pitch = tt.row_pitch;
	}
	else
	{
		const long long n = n_line;
		tt.nbox = (int)((n + 255) / 256);
		tt.box_h = (int)((n + tt.nbox - 1) / tt.nbox);
		tt.ncols = axis == 1 ? XS : Y * XS;
		tt.col_tiles = (tt.ncols + 31) / 32;
		tt.items = (axis == 1 ? Z : 1) * tt.col_tiles;
		// tile indices and columns within 31 bits (tile_line::locate; 2^31 columns of a plane is
		// far beyond any field that fits the device)
		if (tt.items >= (1LL << 31) || tt.col_tiles * 32 >= (1LL << 31))
			return BFVM_OK;
		// the multiplier and shift that divide a tile index by col_tiles
		{
			const unsigned long long d = (unsigned long long)tt.col_tiles;
			int l = 0;
			while ((1ULL << l) < d)
				l++;
			tt.ct_shift = l;
			tt.ct_magic = (unsigned)(((1ULL << 32) * ((1ULL << l) - d)) / d + 1);
		}
		tt.outer_stride = axis == 1 ? Y * XS : 0;
		tt.line_stride = axis == 1 ? XS : Y * XS;
		// stage rows: the virtual front, then the boxes (the last may run past the line end and is
		// zero-filled by the copy)
		tt.stage_floats = (a.pad + tt.nbox * tt.box_h) * 32;
		tt.front_floats = a.pad * 32;
		tt.front_count = 1;
		tt.front_pitch = 0;
		// (chunks: the map spans the whole line; each CTA's boxes start at its chunk's first row)
		if (encode_box(encode, map, axis, base, X, Y, Z, S, chunk ? (long long)st->grid[axis] : n, 32, tt.box_h)
			!= CUDA_SUCCESS)
			return BFVM_OK; // fall back to the direct kernels
	}
	int dev = 0, optin = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
	// warp groups per CTA: up to 640 threads (20 warps per SM) in at most 8 groups (named barriers
	// 1..8), fewer when their stages (at least two each) do not fit; each group then takes as many
	// stages as fit, up to 4
	const size_t stage_bytes = (size_t)tt.stage_floats * sizeof(float);
	auto fixed_bytes = [&](int G) {
		return 128 + (staged_table_floats(a.vP, (int)S) + (size_t)G * 2 * a.vP * 32) * sizeof(float) + 8
			   + (size_t)G * 4 * (sizeof(uint64_t) + sizeof(unsigned));
	};
	const int Gmax = std::max(1, std::min(8, 20 / a.vP));
	auto max_stages = [&](int G) { return (int)std::min<size_t>(4, ((size_t)optin - std::min((size_t)optin, fixed_bytes(G))) / ((size_t)G * stage_bytes)); };
	if (shapes)
	{
		shapes->clear();
		for (int G = 1; G <= Gmax; G++)
			for (int n = 2; n <= max_stages(G); n++)
				shapes->push_back({ G, n });
		return BFVM_OK;
	}
	int G = Gmax;
	// a field of few tiles runs as more, smaller CTAs (at least 4 tiles per group over all SMs),
	// which also leaves room on the SMs for the kernels of other meshes in a batch
	G = (int)std::max<long long>(1, std::min<long long>(G, tt.items / (4LL * sm_count_impl(st->device))));
	while (G > 1 && max_stages(G) < 2)
		G--;
	if (max_stages(G) < 2)
		return BFVM_OK;
	int NST = max_stages(G);
	sweep_tuning cached;
	const sweep_tuning* want = (tune && tune->groups > 0) ? tune : (cached_tuning(st, axis, cached) ? &cached : nullptr);
	if (want && want->groups <= Gmax && want->stages >= 2 && want->stages <= max_stages(want->groups))
	{
		G = want->groups;
		NST = want->stages;
	}
	tt.groups = G;
	tt.stages = NST;
	tt.prefetch = st->tma_prefetch ? 1 : 0;
	const size_t smem = fixed_bytes(G) + (size_t)G * tt.stages * stage_bytes;
	// pairs of groups sharing 64-column stages (the same shared memory: half the stages, twice the
	// width): the plain y and z sweeps over the whole field, an even number of groups, and for y an
	// even number of tiles per plane so that no pair spans two planes
	const int mode = a.dir.items > 0 ? 1 : (a.face_apply ? 2 : 0);
	const bool pair = (axis == 2 ? st->tma_pairs >= 1 : axis == 1 && st->tma_pairs == 2) && !slab_solve && !gf && !chunk
					  && mode != 1 && w_begin == 0 && w_end < 0 && G % 2 == 0 && (axis == 2 || tt.col_tiles % 2 == 0);
	if (pair)
	{
		CUtensorMap pmap;
		if (encode_box(encode, pmap, axis, base, X, Y, Z, S, n_line, 64, tt.box_h) != CUDA_SUCCESS)
			return BFVM_OK; // the unpaired map was accepted above; a refusal here is not expected
		map = pmap;
		tt.pair = 1;
		tt.prefetch = 0;
		tt.slots = (tt.items + 1) / 2;
		tt.stage_floats *= 2;
		tt.front_floats *= 2;
	}
	if (w_end >= 0 || w_begin != 0)
	{
		if (w_end < 0)
			w_end = tt.items;
		if (w_begin < 0 || w_end > tt.items || w_begin > w_end)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "tile range outside the sweep");
		handled = true;
		if (w_begin == w_end)
			return BFVM_OK;
		tt.first = w_begin;
		tt.items = w_end;
	}
	if (!tt.pair)
		tt.slots = tt.items;

	handled = true;
	if (chunk)
	{
		tt.chunks = chunk->count;
		tt.e_stride = axis == 0 ? S : (axis == 1 ? XS : Y * XS);
		for (int k = 0; k < chunk->count; k++)
		{
			tt.chunk_e0[k] = chunk->e0[k];
			tt.chunk_vtab[k] = chunk->vtab[k];
		}
		if (axis == 0)
			return S == 16  ? launch_tma_variant<true, true, 2, 0, 0, false, 16>(st, a, map, tt, smem)
				   : S == 8 ? launch_tma_variant<true, true, 2, 0, 0, false, 8>(st, a, map, tt, smem)
				   : S == 4 ? launch_tma_variant<true, true, 2, 0, 0, false, 4>(st, a, map, tt, smem)
							: launch_tma_variant<true, true, 2>(st, a, map, tt, smem);
		return axis == 1 ? launch_tma_variant<false, true, 2>(st, a, map, tt, smem)
						 : launch_tma_variant<false, false, 2>(st, a, map, tt, smem);
	}
	if (axis == 0)
		return mode == 1   ? launch_tma_variant<true, true, 0, 0, 1>(st, a, map, tt, smem)
			   : mode == 2 ? launch_tma_variant<true, true, 0, 0, 2>(st, a, map, tt, smem)
						   : (S == 16  ? launch_tma_variant<true, true, 0, 0, 0, false, 16>(st, a, map, tt, smem)
							  : S == 8 ? launch_tma_variant<true, true, 0, 0, 0, false, 8>(st, a, map, tt, smem)
							  : S == 4 ? launch_tma_variant<true, true, 0, 0, 0, false, 4>(st, a, map, tt, smem)
									   : launch_tma_variant<true, true>(st, a, map, tt, smem));
	if (axis == 1)
	{
		if (pair)
			return mode == 2 ? launch_tma_variant<false, true, 0, 0, 2, true>(st, a, map, tt, smem)
							 : launch_tma_variant<false, true, 0, 0, 0, true>(st, a, map, tt, smem);
		return mode == 1   ? launch_tma_variant<false, true, 0, 0, 1>(st, a, map, tt, smem)
			   : mode == 2 ? launch_tma_variant<false, true, 0, 0, 2>(st, a, map, tt, smem)
						   : launch_tma_variant<false, true>(st, a, map, tt, smem);
	}
	if (slab_solve)
		return launch_tma_variant<false, false, 1>(st, a, map, tt, smem);
	if (gf && a.vP > 1)
	{
		tt.evict_first = st->grad_evict_first ? 1 : 0;
		if (S % 4 == 0)
			return launch_tma_variant<false, false, 0, 4, 1>(st, a, map, tt, smem, gf);
		return launch_tma_variant<false, false, 0, 1, 1>(st, a, map, tt, smem, gf);
	}
	handled = !gf; // a gradient was asked for and this shape cannot compute it: the caller sweeps
	if (!handled)
		return BFVM_OK;
	if (pair)
		return mode == 2 ? launch_tma_variant<false, false, 0, 0, 2, true>(st, a, map, tt, smem)
						 : launch_tma_variant<false, false, 0, 0, 0, true>(st, a, map, tt, smem);
	return mode == 1   ? launch_tma_variant<false, false, 0, 0, 1>(st, a, map, tt, smem)
		   : mode == 2 ? launch_tma_variant<false, false, 0, 0, 2>(st, a, map, tt, smem)
					   : launch_tma_variant<false, false>(st, a, map, tt, smem);
}

} // namespace bfvm
