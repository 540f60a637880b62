// Ensemble kernels: one launch per phase of the step (Dirichlet overwrite, the sweeps, gradient,
// secretion update) for every mesh of a batch.  Each phase has a prefix list of work units over the
// meshes; a CTA maps its unit to the mesh that owns it (a unit -> mesh table, or for the sweeps a
// binary search of the prefix list when a CTA's run of tiles enters the next mesh) and runs that
// mesh's arithmetic, the same as the mesh's own kernels, so a batch reproduces every mesh stepped
// alone bit for bit.  The Dirichlet overwrites run on flat lists of (address, value), and the
// sweeps write the face conditions of the overwrites that follow them where a mesh allows it.
//
// The sweep kernel reads its lines straight from global memory (coalesced 128-byte rows, 32
// independent loads per thread) rather than through TMA stages: ensemble meshes are small, and
// many small CTAs keep the GPU busy where staging depth would not.  It uses the front-padded block
// algebra of sweep_tma.cu (precompute_padded), and also serves a single mesh whose shape the TMA
// path does not take.

#include <algorithm>

#include "agent_kernels.cuh"
#include "ensemble.h"
#include "sweep_common.cuh"

namespace bfvm {

// mesh that owns work unit u: the last i with first[i] <= u
__device__ __forceinline__ int find_mesh(const long long* __restrict__ first, int count, long long u)
{
	int lo = 0, hi = count - 1;
	while (lo < hi)
	{
		const int mid = (lo + hi + 1) >> 1;
		if (__ldg(&first[mid]) <= u)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

// ------------------------------------------------------------------------------------------------
// Dirichlet overwrite, gradient, secretion: 256-element blocks

// Dirichlet overwrite: the members' lists are gathered once per plan into flat lists of
// (address, value), so the overwrite is one load of an entry and one store, with no lookup of the
// entry's mesh.  Every position occurs once per mesh list, so the order of the stores does not
// matter.

// one mesh's list to gather: its runs of four and single elements and their place in the flat list
struct ens_dir_src
{
	float* dens;
	const long long* qidx;
	const float4* qval;
	long long qcount;
	const long long* idx;
	const float* val;
	long long count;
	long long qflat, sflat;
};

// unit u (256 entries) of the list of mesh umesh[u], whose units start at ufirst[mesh]
__global__ void __launch_bounds__(256) ens_dirichlet_flatten_kernel(const ens_dir_src* __restrict__ src,
																	 const long long* __restrict__ ufirst,
																	 const int* __restrict__ umesh, long long units,
																	 float4** __restrict__ qptr, float4* __restrict__ qval,
																	 float** __restrict__ sptr, float* __restrict__ sval)
{
	for (long long u = blockIdx.x; u < units; u += gridDim.x)
	{
		const int i = umesh[u];
		const ens_dir_src& m = src[i];
		const long long e = (u - ufirst[i]) * 256 + threadIdx.x;
		if (e < m.qcount)
		{
			qptr[m.qflat + e] = reinterpret_cast<float4*>(m.dens + m.qidx[e]);
			qval[m.qflat + e] = m.qval[e];
		}
		else if (e - m.qcount < m.count)
		{
			const long long k = e - m.qcount;
			sptr[m.sflat + k] = m.dens + m.idx[k];
			sval[m.sflat + k] = m.val[k];
		}
	}
}

// *ptr[t] = val[t] for t < n, grid-stride, four entries per thread loaded before their stores
template <typename V>
__device__ __forceinline__ void scatter_entries(V* const* __restrict__ ptr, const V* __restrict__ val, long long n)
{
	const long long T = (long long)gridDim.x * blockDim.x;
	long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned long long* praw = reinterpret_cast<const unsigned long long*>(ptr);
	for (; t + 3 * T < n; t += 4 * T)
	{
		V* p[4];
		V v[4];
#pragma unroll
		for (int k = 0; k < 4; k++)
		{
			p[k] = reinterpret_cast<V*>(__ldg(&praw[t + k * T]));
			v[k] = __ldg(&val[t + k * T]);
		}
#pragma unroll
		for (int k = 0; k < 4; k++)
			*p[k] = v[k];
	}
	for (; t < n; t += T)
		*reinterpret_cast<V*>(__ldg(&praw[t])) = __ldg(&val[t]);
}

__global__ void __launch_bounds__(256) ens_dirichlet_kernel(float4* const* __restrict__ qptr,
															 const float4* __restrict__ qval, long long nq,
															 float* const* __restrict__ sptr,
															 const float* __restrict__ sval, long long ns)
{
	scatter_entries(qptr, qval, nq);
	scatter_entries(sptr, sval, ns);
}

// central differences (gradient.cu); output layouts 1D [x][s][1], 2D [y][x][s][2], 3D [3][z][y][x][s].
// One unit is 256 consecutive columns of the (y, x, s) plane over up to ZC planes: each thread
// marches z keeping u(z-1), u(z), u(z+1) in registers (gradient3d_vec4_kernel of gradient.cu for
// any S), reading x and y neighbours from L1/L2.  A thread's x and y never change along z, so the
// one-sided or central form of each axis is fixed once as two neighbour offsets and a factor; z
// advances ZU planes at a time with every load of those planes issued before their arithmetic,
// which keeps enough loads in flight for small meshes to stream at HBM rate.  ZC and ZU are launch
// choices (ens_tuning).

// neighbour offsets lo, hi and factor of an axis at position pos of n: (u[1] - u[0]) / h at the
// first voxel, (u[n-1] - u[n-2]) / h at the last, (u[i+1] - u[i-1]) / (2h) inside; an axis of one
// voxel reads nothing past it (its gradient is 0, set by the caller)
__device__ __forceinline__ void axis_form(int pos, int n, long long stride, float border, float center, long long& lo,
										  long long& hi, float& f)
{
	if (n == 1)
	{
		lo = hi = 0;
		f = 0.f;
	}
	else if (pos == 0)
	{
		lo = 0;
		hi = stride;
		f = border;
	}
	else if (pos == n - 1)
	{
		lo = -stride;
		hi = 0;
		f = border;
	}
	else
	{
		lo = -stride;
		hi = stride;
		f = center;
	}
}

// The z march of one column of a 3-D mesh over planes [z0, z1): p and g point at plane z0 of the
// column in the field and in the x component of the gradient.  Planes that have a next plane run
// U at a time without guards, through pointers that advance a plane per step; the rest (up to
// U - 1 planes, and the mesh's last plane) run one at a time.
template <int U>
__device__ __forceinline__ void ens_gradient_3d(const ens_inst& m, const float* __restrict__ p, float* __restrict__ g,
												long long plane, int z0, int z1, long long xlo, long long xhi,
												float fx, long long ylo, long long yhi, float fy)
{
	const int Z = m.Z;
	const long long total = plane * Z;
	const bool hasx = m.X > 1, hasy = m.Y > 1;
	const float bz = m.bgrad[2], cz = m.cgrad[2];
	float prev = z0 > 0 ? __ldg(p - plane) : 0.f;
	float cur = __ldg(p);
	int z = z0;
	const int zmain = min(z1, Z - 1);
	for (; z + U <= zmain; z += U)
	{
		float nx[U], xa[U], xb[U], ya[U], yb[U];
#pragma unroll
		for (int k = 0; k < U; k++)
		{
			const float* q = p + k * plane;
			nx[k] = __ldg(q + plane);
			xa[k] = __ldg(q + xhi);
			xb[k] = __ldg(q + xlo);
			ya[k] = __ldg(q + yhi);
			yb[k] = __ldg(q + ylo);
		}
#pragma unroll
		for (int k = 0; k < U; k++)
		{
			const float next = nx[k];
			const float gx = hasx ? __fmul_rn(__fsub_rn(xa[k], xb[k]), fx) : 0.f;
			const float gy = hasy ? __fmul_rn(__fsub_rn(ya[k], yb[k]), fy) : 0.f;
			const float gz = z + k == 0 ? __fmul_rn(__fsub_rn(next, cur), bz) : __fmul_rn(__fsub_rn(next, prev), cz);
			float* o = g + k * plane;
			__stcs(o, gx);
			__stcs(o + total, gy);
			__stcs(o + 2 * total, gz);
			prev = cur;
			cur = next;
		}
		p += U * plane;
		g += U * plane;
	}
	for (; z < z1; z++)
	{
		const float next = z + 1 < Z ? __ldg(p + plane) : cur;
		const float gx = hasx ? __fmul_rn(__fsub_rn(__ldg(p + xhi), __ldg(p + xlo)), fx) : 0.f;
		const float gy = hasy ? __fmul_rn(__fsub_rn(__ldg(p + yhi), __ldg(p + ylo)), fy) : 0.f;
		float gz;
		if (Z == 1)
			gz = 0.f;
		else if (z == 0)
			gz = __fmul_rn(__fsub_rn(next, cur), bz);
		else if (z == Z - 1)
			gz = __fmul_rn(__fsub_rn(cur, prev), bz);
		else
			gz = __fmul_rn(__fsub_rn(next, prev), cz);
		__stcs(g, gx);
		__stcs(g + total, gy);
		__stcs(g + 2 * total, gz);
		prev = cur;
		cur = next;
		p += plane;
		g += plane;
	}
}

// The z march of a 3-D mesh of 4k substrates, four substrates per thread (gradient3d_vec4_kernel of
// gradient.cu): p4 and g4 point at plane z0 of the thread's float4 column; neighbour offsets in
// float4s.  The loads of the next D planes are kept in flight ahead of the plane being written
// (a ring of D registers, shifted and refilled as each plane is used), so D planes of each thread
// stream from memory at once; the x and y neighbours, cache hits mostly, are loaded plane by plane.  The same arithmetic per element as the scalar march, so the same bits.
__device__ __forceinline__ float4 ens_f4sub_mul(float4 a, float4 b, float f)
{
	return make_float4(__fmul_rn(__fsub_rn(a.x, b.x), f), __fmul_rn(__fsub_rn(a.y, b.y), f),
					   __fmul_rn(__fsub_rn(a.z, b.z), f), __fmul_rn(__fsub_rn(a.w, b.w), f));
}

template <int D>
__device__ __forceinline__ void ens_gradient_3d_vec4(const ens_inst& m, const float4* __restrict__ p4,
													 float4* __restrict__ g4, int plane4, int z0, int z1, int xlo,
													 int xhi, float fx, int ylo, int yhi, float fy)
{
	// offsets in float4s fit 31 bits: a mesh's elements do (ensemble_eligible)
	const int Z = m.Z;
	const int total4 = plane4 * Z;
	const bool hasx = m.X > 1, hasy = m.Y > 1;
	const float bz = m.bgrad[2], cz = m.cgrad[2];
	const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
	float4 prev = z0 > 0 ? __ldg(p4 - plane4) : zero;
	float4 cur = __ldg(p4);
	// ring[k]: plane z + 1 + k (the planes up to z1, the last plane's next, and no further)
	float4 ring[D];
#pragma unroll
	for (int k = 0; k < D; k++)
	{
		const int zz = z0 + 1 + k;
		ring[k] = (zz < Z && zz <= z1) ? __ldg(p4 + (k + 1) * plane4) : zero;
	}
	for (int z = z0; z < z1; z++)
	{
		const float4 next = z + 1 < Z ? ring[0] : cur;
		const float4 gx = hasx ? ens_f4sub_mul(__ldg(p4 + xhi), __ldg(p4 + xlo), fx) : zero;
		const float4 gy = hasy ? ens_f4sub_mul(__ldg(p4 + yhi), __ldg(p4 + ylo), fy) : zero;
		float4 gz;
		if (Z == 1)
			gz = zero;
		else if (z == 0)
			gz = ens_f4sub_mul(next, cur, bz);
		else if (z == Z - 1)
			gz = ens_f4sub_mul(cur, prev, bz);
		else
			gz = ens_f4sub_mul(next, prev, cz);
		__stcs(g4, gx);
		__stcs(g4 + total4, gy);
		__stcs(g4 + 2 * total4, gz);
#pragma unroll
		for (int k = 0; k + 1 < D; k++)
			ring[k] = ring[k + 1];
		const int zz = z + 1 + D;
		ring[D - 1] = (zz < Z && zz <= z1) ? __ldg(p4 + (1 + D) * plane4) : zero;
		prev = cur;
		cur = next;
		p4 += plane4;
		g4 += plane4;
	}
}

// ALL3D: every mesh is 3-D.  The kernel then holds the 3-D march alone, which fits 64 registers, so
// four CTAs share an SM: twice the loads in flight of the kernel that also holds the 1-D and 2-D
// forms (held to 128 registers, two CTAs).
template <bool ALL3D, int ZU>
__global__ void __launch_bounds__(256, ALL3D ? 4 : 2) ens_gradient_kernel(const ens_inst* __restrict__ inst,
																		   const long long* __restrict__ first,
																		   const int* __restrict__ umesh,
																		   long long units, int ZC)
{
	for (long long u = blockIdx.x; u < units; u += gridDim.x)
	{
		const int i = __ldg(&umesh[u]);
		const ens_inst& m = inst[i];
		const int S = m.S, X = m.X, Y = m.Y, Z = m.Z, dims = m.dims;
		const int XS = X * S;
		if (dims == 3 && (S & 3) == 0)
		{
			// four substrates per thread: a unit is 256 float4 columns of the (y, x, s) plane
			const int S4 = S >> 2, XS4 = XS >> 2;
			const int cols4 = XS4 * Y;
			const int ncx = (cols4 + 255) / 256;
			const int local = (int)(u - first[i]);
			const int z0 = (local / ncx) * ZC;
			const int c4 = (local % ncx) * 256 + threadIdx.x;
			if (c4 >= cols4)
				continue;
			const int y = c4 / XS4;
			const int q4 = c4 - y * XS4;
			const int x = q4 / S4;
			const int plane4 = cols4;
			long long xlo, xhi, ylo, yhi;
			float fx, fy;
			axis_form(x, X, S4, m.bgrad[0], m.cgrad[0], xlo, xhi, fx);
			axis_form(y, Y, XS4, m.bgrad[1], m.cgrad[1], ylo, yhi, fy);
			const int e4 = z0 * plane4 + c4;
			ens_gradient_3d_vec4<2>(m, reinterpret_cast<const float4*>(m.dens) + e4,
										 reinterpret_cast<float4*>(m.grad) + e4, plane4, z0, min(Z, z0 + ZC), (int)xlo,
										 (int)xhi, fx, (int)ylo, (int)yhi, fy);
			continue;
		}
		const int plane_cols = XS * Y;
		const int ncx = (plane_cols + 255) / 256;
		const int local = (int)(u - first[i]);
		const int cx = local % ncx;
		const int z0 = (local / ncx) * ZC;
		const int z1 = min(Z, z0 + ZC);
		const int c = cx * 256 + threadIdx.x; // column of the plane: y * XS + q
		if (c >= plane_cols)
			continue;
		const int y = c / XS;
		const int q = c - y * XS;
		const int x = q / S;
		const float* __restrict__ d = m.dens;
		float* __restrict__ g = m.grad;
		const long long plane = (long long)Y * XS;
		const long long total = plane * Z;
		const long long row = (long long)y * XS + q;
		long long xlo, xhi, ylo = 0, yhi = 0;
		float fx, fy = 0.f;
		axis_form(x, X, S, m.bgrad[0], m.cgrad[0], xlo, xhi, fx);
		if (dims >= 2)
			axis_form(y, Y, XS, m.bgrad[1], m.cgrad[1], ylo, yhi, fy);
		if (ALL3D || dims == 3)
		{
			const long long e0 = (long long)z0 * plane + row;
			ens_gradient_3d<ZU>(m, d + e0, g + e0, plane, z0, z1, xlo, xhi, fx, ylo, yhi, fy);
			continue;
		}
		float prev = z0 > 0 ? __ldg(&d[(long long)(z0 - 1) * plane + row]) : 0.f;
		float cur = __ldg(&d[(long long)z0 * plane + row]);
		for (int z = z0; z < z1; z += ZU)
		{
			// every load of these planes first
			float nx[ZU], xa[ZU], xb[ZU], ya[ZU], yb[ZU];
#pragma unroll
			for (int k = 0; k < ZU; k++)
			{
				const int zz = z + k;
				const long long e = (long long)zz * plane + row;
				const bool in = zz < z1;
				nx[k] = (in && zz + 1 < Z) ? __ldg(&d[e + plane]) : 0.f;
				xa[k] = in ? __ldg(&d[e + xhi]) : 0.f;
				xb[k] = in ? __ldg(&d[e + xlo]) : 0.f;
				ya[k] = (in && dims >= 2) ? __ldg(&d[e + yhi]) : 0.f;
				yb[k] = (in && dims >= 2) ? __ldg(&d[e + ylo]) : 0.f;
			}
#pragma unroll
			for (int k = 0; k < ZU; k++)
			{
				const int zz = z + k;
				if (zz >= z1)
					break;
				const long long e = (long long)zz * plane + row;
				const float next = zz + 1 < Z ? nx[k] : cur;
				const float gx = X == 1 ? 0.f : __fmul_rn(__fsub_rn(xa[k], xb[k]), fx);
				if (dims == 1)
					g[e] = gx;
				else
				{
					const float gy = Y == 1 ? 0.f : __fmul_rn(__fsub_rn(ya[k], yb[k]), fy);
					if (dims == 2)
					{
						g[2 * e] = gx;
						g[2 * e + 1] = gy;
					}
					else
					{
						float gz;
						if (Z == 1)
							gz = 0.f;
						else if (zz == 0)
							gz = __fmul_rn(__fsub_rn(next, cur), m.bgrad[2]);
						else if (zz == Z - 1)
							gz = __fmul_rn(__fsub_rn(cur, prev), m.bgrad[2]);
						else
							gz = __fmul_rn(__fsub_rn(next, prev), m.cgrad[2]);
						__stcs(&g[e], gx);
						__stcs(&g[total + e], gy);
						__stcs(&g[2 * total + e], gz);
					}
				}
				prev = cur;
				cur = next;
			}
		}
	}
}

__global__ void __launch_bounds__(256) ens_secretion_kernel(const ens_inst* __restrict__ inst,
															 const long long* __restrict__ first,
															 const int* __restrict__ umesh, long long units)
{
	for (long long u = blockIdx.x; u < units; u += gridDim.x)
	{
		const int i = __ldg(&umesh[u]);
		const ens_inst& m = inst[i];
		const long long t = (u - first[i]) * 256 + threadIdx.x;
		if (m.vec4)
		{
			if (t < (long long)__ldg(m.counts) * (m.S >> 2))
				secrete_sorted4_element(t, m.S, m.dens, m.counts, m.seg_start, m.keys, m.num, m.den, m.fac, m.red_num,
										m.red_den, m.red_fac, m.intern, m.voxel_volume);
		}
		else if (t < m.AS)
		{
			if (m.sorted)
				secrete_element<true>(t, m.S, m.dens, m.counts, m.seg_start, nullptr, m.keys, m.num, m.den, m.fac,
									  m.red_num, m.red_den, m.red_fac, m.intern, 1, m.voxel_volume);
			else
				secrete_element(t, m.S, m.dens, m.counts, m.seg_start, m.order, m.keys, m.num, m.den, m.fac,
								m.red_num, m.red_den, m.red_fac, m.intern, m.internalized, m.voxel_volume);
		}
	}
}

// ------------------------------------------------------------------------------------------------
// sweeps: one unit = one tile of 32 lines (the tiles of sweep_tma.cu), blockDim = (32, maxP)

// staged tables of one mesh and axis: (tg, G) pairs and b' as [S][NP], NP = 32P + 1, then c [S],
// the face bits [S] (0 where the sweeps write no faces) and the face values [6][S]
__device__ __forceinline__ void ens_stage_tables(const ens_inst& m, int AXIS, float* tab)
{
	const float* __restrict__ vtab = m.vtab[AXIS];
	const int P = m.vP[AXIS], S = m.S;
	const int N = 32 * P, NP = N + 1;
	float2* tgtab = reinterpret_cast<float2*>(tab);
	float* btab = tab + 2 * S * NP;
	float* ctab = btab + S * NP;
	int* fbits = reinterpret_cast<int*>(ctab + S);
	float* fvals = ctab + 2 * S;
	const float2* gt = reinterpret_cast<const float2*>(vtab + (size_t)N * S);
	const int nthr = blockDim.x * blockDim.y;
	const int tid = threadIdx.x + blockDim.x * threadIdx.y;
	for (int t = tid; t < N * S; t += nthr)
	{
		const int v = t / S, s = t - v * S;
		btab[s * NP + v] = __ldg(&vtab[t]);
		tgtab[s * NP + v] = __ldg(&gt[t]);
	}
	for (int t = tid; t < S; t += nthr)
	{
		ctab[t] = __ldg(&vtab[(size_t)3 * N * S + t]);
		fbits[t] = m.faces ? __ldg(&m.face_bits[t]) : 0;
	}
	for (int t = tid; t < 6 * S; t += nthr)
		fvals[t] = m.faces ? __ldg(&m.face_vals[t]) : 0.f;
}

// The face conditions of the line along AXIS at coordinates (cx, cy, cz) (AXIS's own is unused),
// for substrate bits `mb` (face_code of sweep_tma.cu): bits 2 and 3, the faces of AXIS at the
// line's first and last element; bits 0-1, 1 when a face of an earlier axis covers the whole line
// (the ends then take AXIS's faces), 2 when a face of a later axis does (it wins everywhere); bits
// 4+, that face, the latest of its kind (later faces win where faces meet).
template <int AXIS>
__device__ __forceinline__ int ens_face_code(int mb, int cx, int cy, int cz, int X, int Y, int Z)
{
	int code = ((mb >> (2 * AXIS)) & 3) << 2;
	int lb = 0;
	if (AXIS != 0)
		lb |= (cx == 0 ? 1 : 0) | (cx == X - 1 ? 2 : 0);
	if (AXIS != 1)
		lb |= (cy == 0 ? 4 : 0) | (cy == Y - 1 ? 8 : 0);
	if (AXIS != 2)
		lb |= (cz == 0 ? 16 : 0) | (cz == Z - 1 ? 32 : 0);
	lb &= mb;
	const int after = lb >> (2 * AXIS + 2), before = lb & ((1 << (2 * AXIS)) - 1);
	if (after)
		code |= 2 | ((31 - __clz(after) + 2 * AXIS + 2) << 4);
	else if (before)
		code |= 1 | ((31 - __clz(before)) << 4);
	return code;
}

// Store the face conditions over block j of a line whose solved values were just stored (the same
// thread stores both, so these win): the line's first element is element `pad` of block 0, its
// last element 31 of block P - 1 (apply_faces of sweep_tma.cu, here after the stores, so the
// solved block need not stay in registers).
template <int AXIS>
__device__ __forceinline__ void ens_store_faces(float* line, int stride, int code, const float* fvals, int S, int s,
												int j, int P, int pad)
{
	const int lk = code & 3;
	if (lk != 0)
	{
		const float lv = fvals[(code >> 4) * S + s];
		for (int k = 0; k < 32; k++)
		{
			const int r = 32 * j + k - pad;
			if (r >= 0)
				line[r * stride] = lv;
		}
		if (lk == 2)
			return;
	}
	if ((code & 4) && j == 0)
		line[0] = fvals[(2 * AXIS) * S + s];
	if ((code & 8) && j == P - 1)
		line[(32 * P - 1 - pad) * stride] = fvals[(2 * AXIS + 1) * S + s];
}

// x tiles: rows [row0, row0 + rows) of mesh m, contiguous in the field
__device__ __forceinline__ void x_tile_rows(const ens_inst& m, long long local, long long& row0, int& rows)
{
	const int R = 32 / m.S;
	row0 = local * R;
	rows = (int)min((long long)R, (long long)m.Y * m.Z - row0);
}

// x sweep: a tile is the R = 32/S rows that follow one another in the field, lane l walking
// substrate l % S of row l / S.  The lanes read the field directly: the 32 lines of a tile cover
// R whole rows, so the tile's loads touch each of its cache lines, which stay in L1/L2 between
// the lanes' neighbouring elements.  (Staging the rows through shared memory with cp.async,
// double-buffered, measured 8% slower over a 256-mesh ensemble.)
// Two CTAs of 512 threads per SM (64 registers): at 114 registers a mesh of 3 blocks per line ran 5
// CTAs of 3 warps per SM, too few warps to hide the loads and barriers.
// MINB 0: lines of 17 to 32 blocks (one mesh alone), CTAs of up to 1024 threads, one per SM; the
// register cap (64) is that of MINB 2.
template <int AXIS, int MINB>
__global__ void __launch_bounds__(MINB == 0 ? 1024 : 512, MINB == 0 ? 1 : MINB) ens_sweep_kernel(const ens_inst* __restrict__ inst,
														 const long long* __restrict__ first, int count,
														 long long units, long long chunk, int maxP)
{
	constexpr int M = 32;
	extern __shared__ __align__(16) float ens_smem[];
	const int lane = threadIdx.x;
	const int j = threadIdx.y;
	float* carry_f = ens_smem;				 // [maxP][32]
	float* carry_t = carry_f + maxP * 32;	 // [maxP][32]
	float* tab = carry_t + maxP * 32;		 // tables of the current mesh (16-byte aligned: maxP*64 floats)

	const long long u0 = (long long)blockIdx.x * chunk;
	const long long u1 = min(units, u0 + chunk);
	// the mesh of the current unit, looked up again only when the units cross into the next mesh
	// (a CTA's chunk of consecutive units mostly stays in one); element offsets within a mesh fit
	// 31 bits (ensemble_eligible), so the line arithmetic runs in 32-bit integers
	int cur = -1;
	long long first_i = 0, first_next = 0;
	for (long long u = u0; u < u1; u++)
	{
		if (u >= first_next)
		{
			const int i = find_mesh(first, count, u);
			first_i = __ldg(&first[i]);
			first_next = __ldg(&first[i + 1]);
			__syncthreads(); // the previous mesh's tables are no longer read
			ens_stage_tables(inst[i], AXIS, tab);
			__syncthreads();
			cur = i;
		}
		const ens_inst& m = inst[cur];
		const int S = m.S, P = m.vP[AXIS], pad = m.pad[AXIS];
		const float* vtab = m.vtab[AXIS];
		const int N = 32 * P, NP = N + 1;
		const float2* tgtab = reinterpret_cast<const float2*>(tab);
		const float* btab = tab + 2 * S * NP;
		const float* ctab = btab + S * NP;
		const float* gqtab = vtab + (size_t)3 * N * S + S;
		const float* tgptab = gqtab + P * S;
		const float* Gptab = tgptab + P * S;

		// the line of this lane
		const int local = (int)(u - first_i);
		const int XS = m.X * S;
		bool active;
		int s, stride;
		float* line;
		if (AXIS == 0)
		{
			const int R = 32 / S;
			const int rl = lane / S;
			s = lane - rl * S;
			const int row0 = local * R;
			active = rl < min(R, m.Y * m.Z - row0);
			line = m.dens + (active ? row0 + rl : 0) * XS + s;
			stride = S;
		}
		else
		{
			const int ncols = AXIS == 1 ? XS : XS * m.Y;
			const int col_tiles = (ncols + 31) / 32;
			const int outer = AXIS == 1 ? local / col_tiles : 0;
			const int q = (local - outer * col_tiles) * 32 + lane;
			active = q < ncols;
			const int qq = active ? q : 0;
			s = qq % S;
			line = m.dens + outer * XS * m.Y + qq;
			stride = AXIS == 1 ? XS : XS * m.Y;
		}
		const bool mine = j < P; // warps past this mesh's blocks only join the barriers
		const int p = 32 * j;
		float d[M];
		float C = 0.f;
		if (mine)
		{
			const float cs = ctab[s];
			const float* bcol = btab + s * NP + p;
#pragma unroll
			for (int k = 0; k < M; k++)
			{
				const int r = p + k - pad; // real element of virtual element p + k
				d[k] = (active && r >= 0) ? line[r * stride] : 0.f;
			}
			// forward and backward recurrences from zero carries (sweep_tma.cu)
#pragma unroll
			for (int k = 1; k < M; k++)
				d[k] = __fsub_rn(d[k], __fmul_rn(__fmul_rn(cs, bcol[k - 1]), d[k - 1]));
			carry_f[j * 32 + lane] = d[M - 1];
			d[M - 1] = __fmul_rn(d[M - 1], bcol[M - 1]);
#pragma unroll
			for (int k = M - 2; k >= 0; k--)
				d[k] = __fmul_rn(__fsub_rn(d[k], __fmul_rn(cs, d[k + 1])), bcol[k]);
		}
		__syncthreads();
		if (mine && P > 1)
		{
			if (j > 0)
			{
				C = carry_f[lane];
				for (int k = 1; k < j; k++)
					C = fmaf(__ldg(&gqtab[k * S + s]), C, carry_f[k * 32 + lane]);
			}
			carry_t[j * 32 + lane] = fmaf(C, __ldg(&tgptab[j * S + s]), d[0]);
		}
		__syncthreads();
		if (mine)
		{
			if (P > 1)
			{
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
			if (active)
			{
#pragma unroll
				for (int k = 0; k < M; k++)
				{
					const int r = p + k - pad;
					if (r >= 0)
						line[r * stride] = d[k];
				}
				// the face conditions of the overwrite after this sweep (meshes with ens_inst::faces):
				// the ends of the line from the faces of AXIS, and, on tiles that reach a face of
				// another axis (a test on the tile's first line), the whole line from that face
				const int mb = reinterpret_cast<const int*>(ctab + S)[s];
				if (mb != 0)
				{
					int code = ((mb >> (2 * AXIS)) & 3) << 2;
					if (mb & ~(3 << (2 * AXIS)))
					{
						bool touch;
						int cx = 0, cy = 0, cz = 0;
						if (AXIS == 0)
						{
							// x tiles: each line placed directly (the tile test would cost the kernel spills)
							touch = true;
							const int row = local * (32 / S) + lane / S;
							cz = row / m.Y;
							cy = row - cz * m.Y;
						}
						else if (AXIS == 1)
						{
							const int col_tiles = (XS + 31) / 32;
							const int z = local / col_tiles, c0 = (local - z * col_tiles) * 32;
							touch = z == 0 || z == m.Z - 1 || c0 < S || c0 + 31 >= XS - S;
							if (touch)
							{
								cz = z;
								cx = (c0 + lane) / S;
							}
						}
						else
						{
							const int q0 = local * 32, y0 = q0 / XS, r0 = q0 - y0 * XS;
							touch = y0 == 0 || q0 + 31 >= (m.Y - 1) * XS || r0 < S || r0 + 31 >= XS - S;
							if (touch)
							{
								const int q = q0 + lane;
								cy = q / XS;
								cx = (q - cy * XS) / S;
							}
						}
						if (touch)
							code = ens_face_code<AXIS>(mb, cx, cy, cz, m.X, m.Y, m.Z);
					}
					if (code != 0)
						ens_store_faces<AXIS>(line, stride, code, ctab + 2 * S, S, s, j, P, pad);
				}
			}
		}
		__syncthreads(); // carries of this tile read before the next tile writes them
	}
}

// ------------------------------------------------------------------------------------------------
// host side

bool ensemble_eligible(const bfvm_solver* s)
{
	for (int d = 0; d < s->dims; d++)
	{
		const sweep_plan& p = s->plan[d];
		if (!p.vtab || p.vP > ENS_MAX_P || p.n < 2)
			return false;
	}
	// x tiles hold whole rows of at most 32 substrate lines; element indices fit 31 bits
	return s->S <= 32 && s->V * s->S < (1LL << 31);
}

// the staged tables of ens_stage_tables: (tg, G) and b' as [S][NP], c [S], face bits [S], face values [6][S]
static size_t staged_floats(int P, int S) { return 3 * (size_t)S * (32 * P + 1) + 8 * (size_t)S; }

void ensemble_free(ensemble_plan& plan)
{
	device_free(plan.inst);
	for (auto& f : plan.first)
		device_free(f);
	for (auto& u : plan.unit_mesh)
		device_free(u);
	for (auto& f : plan.first_h)
		f.clear();
	for (ensemble_plan::flat_list& l : plan.dir)
	{
		device_free(l.qptr);
		device_free(l.qval);
		device_free(l.sptr);
		device_free(l.sval);
		for (int k = 0; k < 4; k++)
			l.q_ge[k] = l.s_ge[k] = 0;
	}
	plan.dir_built = false;
	plan.count = 0;
}

int ensemble_build(ensemble_plan& plan, const std::vector<bfvm_solver*>& meshes, const ens_tuning& tune,
				   const std::vector<std::pair<float*, float*>>* buffers, bool rebinned, bool faces)
{
	ensemble_free(plan);
	plan.tune = tune;
	const int n = (int)meshes.size();
	if (n == 0)
		return BFVM_OK;
	std::vector<ens_inst> h(n);
	for (auto& f : plan.first_h)
		f.assign(n + 1, 0);
	plan.maxP[0] = plan.maxP[1] = plan.maxP[2] = 1;
	plan.table_floats[0] = plan.table_floats[1] = plan.table_floats[2] = 0;
	plan.maxS = 1;
	plan.all3d = true;
	for (int i = 0; i < n; i++)
	{
		const bfvm_solver* s = meshes[i];
		ens_inst& m = h[i];
		m.dens = buffers ? (*buffers)[i].first : s->dens;
		m.grad = buffers ? (*buffers)[i].second : s->grad;
		m.dims = s->dims;
		plan.all3d = plan.all3d && s->dims == 3;
		m.S = s->S;
		m.X = s->grid[0];
		m.Y = s->grid[1];
		m.Z = s->grid[2];
		for (int d = 0; d < 3; d++)
		{
			m.bgrad[d] = d < s->dims ? 1.f / s->voxel[d] : 0.f;
			m.cgrad[d] = d < s->dims ? 1.f / (s->voxel[d] * 2) : 0.f;
			m.vtab[d] = d < s->dims ? s->plan[d].vtab : nullptr;
			m.vP[d] = d < s->dims ? s->plan[d].vP : 1;
			m.pad[d] = d < s->dims ? s->plan[d].pad : 0;
		}
		m.dir_qidx = s->dir_qidx;
		m.dir_qval = s->dir_qval;
		m.dir_qcount = s->dir_qcount;
		m.dir_idx = s->dir_idx;
		m.dir_val = s->dir_val;
		m.dir_count = s->dir_count;
		const bool fp = faces && s->face_pos_ok && s->face_bits && s->face_vals_d;
		m.faces = fp ? 1 : 0;
		m.face_bits = fp ? s->face_bits : nullptr;
		m.face_vals = fp ? s->face_vals_d : nullptr;
		m.dir_iqidx = fp ? s->dir_interior.qidx : nullptr;
		m.dir_iqval = fp ? s->dir_interior.qval : nullptr;
		m.dir_iqcount = fp ? s->dir_interior.qcount : 0;
		m.dir_iidx = fp ? s->dir_interior.idx : nullptr;
		m.dir_ival = fp ? s->dir_interior.val : nullptr;
		m.dir_icount = fp ? s->dir_interior.count : 0;
		const agent_state& a = s->ag;
		m.AS = (long long)a.count * s->S;
		m.internalized = s->internalized ? 1 : 0;
		m.voxel_volume = (float)(s->voxel[0] * s->voxel[1] * s->voxel[2]);
		m.counts = a.seg_count_dev;
		m.seg_start = a.seg_start;
		m.order = a.vals;
		m.keys = a.keys;
		const bool sorted = a.count > 0 && (rebinned ? s->internalized : a.sorted);
		m.sorted = sorted ? 1 : 0;
		m.vec4 = sorted && s->S % 4 == 0 ? 1 : 0;
		m.num = sorted ? a.snum : a.num;
		m.den = sorted ? a.sden : a.den;
		m.fac = sorted ? a.sfac : a.fac;
		m.red_num = a.red_num;
		m.red_den = a.red_den;
		m.red_fac = a.red_fac;
		m.intern = sorted ? a.sintern : a.intern;

		const long long X = m.X, Y = m.Y, Z = m.Z, S = m.S, XS = X * S;
		long long units[ENS_PHASES] = { 0, 0, 0, 0, 0, 0 };
		units[ENS_DIRICHLET] = (m.dir_qcount + m.dir_count + 255) / 256;
		const long long R = 32 / S; // x tiles: rows of at most 32 substrate lines
		units[ENS_SWEEP_X] = R > 0 ? (Y * Z + R - 1) / R : 0;
		units[ENS_SWEEP_Y] = s->dims >= 2 ? Z * ((XS + 31) / 32) : 0;
		units[ENS_SWEEP_Z] = s->dims >= 3 ? (Y * XS + 31) / 32 : 0;
		// 3-D meshes of 4k substrates: 256 float4 columns per unit (ens_gradient_kernel)
		const long long grad_cols = (s->dims == 3 && S % 4 == 0) ? XS * Y / 4 : XS * Y;
		units[ENS_GRADIENT] = ((grad_cols + 255) / 256) * ((Z + tune.grad_zc - 1) / tune.grad_zc);
		units[ENS_SECRETION] = ((m.vec4 ? m.AS / 4 : m.AS) + 255) / 256;
		for (int ph = 0; ph < ENS_PHASES; ph++)
			plan.first_h[ph][i + 1] = plan.first_h[ph][i] + units[ph];
		for (int d = 0; d < s->dims; d++)
		{
			plan.maxP[d] = std::max(plan.maxP[d], m.vP[d]);
			plan.table_floats[d] = std::max(plan.table_floats[d], staged_floats(m.vP[d], m.S));
		}
		plan.maxS = std::max(plan.maxS, m.S);
	}
	int st;
	if ((st = device_alloc(&plan.inst, (size_t)n)))
		return st;
	BFVM_CUDA(cudaMemcpy(plan.inst, h.data(), n * sizeof(ens_inst), cudaMemcpyHostToDevice));
	for (int ph = 0; ph < ENS_PHASES; ph++)
	{
		if ((st = device_alloc(&plan.first[ph], (size_t)n + 1)))
			return st;
		BFVM_CUDA(cudaMemcpy(plan.first[ph], plan.first_h[ph].data(), (n + 1) * sizeof(long long),
							 cudaMemcpyHostToDevice));
	}
	for (int ph : { (int)ENS_DIRICHLET, (int)ENS_GRADIENT, (int)ENS_SECRETION })
	{
		const std::vector<long long>& f = plan.first_h[ph];
		std::vector<int> um((size_t)std::max<long long>(f[n], 1), 0);
		for (int i = 0; i < n; i++)
			std::fill(um.begin() + f[i], um.begin() + f[i + 1], i);
		if ((st = device_alloc(&plan.unit_mesh[ph], um.size())))
			return st;
		BFVM_CUDA(cudaMemcpy(plan.unit_mesh[ph], um.data(), um.size() * sizeof(int), cudaMemcpyHostToDevice));
	}
	plan.count = n;
	return BFVM_OK;
}

static int current_device_sms()
{
	int dev = 0;
	cudaGetDevice(&dev);
	return sm_count_impl(dev);
}

static unsigned element_grid(long long units)
{
	return (unsigned)std::max<long long>(1, std::min<long long>(units, (long long)current_device_sms() * 16));
}

static int launched(const char* what)
{
	cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? BFVM_OK : cuda_fail(e, what);
}

// Gather the lists `src` (meshes in the order of the flat list: qflat / sflat set) into `out`.
static int flatten_lists(const std::vector<ens_dir_src>& src, ensemble_plan::flat_list& out, long long nq, long long ns)
{
	int st;
	if ((st = device_alloc(&out.qptr, (size_t)std::max(nq, 1LL))) || (st = device_alloc(&out.qval, (size_t)std::max(nq, 1LL)))
		|| (st = device_alloc(&out.sptr, (size_t)std::max(ns, 1LL))) || (st = device_alloc(&out.sval, (size_t)std::max(ns, 1LL))))
		return st;
	const int n = (int)src.size();
	std::vector<long long> ufirst(n + 1, 0);
	for (int i = 0; i < n; i++)
		ufirst[i + 1] = ufirst[i] + (src[i].qcount + src[i].count + 255) / 256;
	const long long units = ufirst[n];
	if (units == 0)
		return BFVM_OK;
	std::vector<int> um((size_t)units);
	for (int i = 0; i < n; i++)
		std::fill(um.begin() + ufirst[i], um.begin() + ufirst[i + 1], i);
	ens_dir_src* src_d = nullptr;
	long long* ufirst_d = nullptr;
	int* um_d = nullptr;
	if ((st = device_alloc(&src_d, (size_t)n)) || (st = device_alloc(&ufirst_d, (size_t)n + 1))
		|| (st = device_alloc(&um_d, (size_t)units)))
	{
		device_free(src_d);
		device_free(ufirst_d);
		return st;
	}
	cudaError_t e = cudaMemcpy(src_d, src.data(), n * sizeof(ens_dir_src), cudaMemcpyHostToDevice);
	if (e == cudaSuccess)
		e = cudaMemcpy(ufirst_d, ufirst.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice);
	if (e == cudaSuccess)
		e = cudaMemcpy(um_d, um.data(), units * sizeof(int), cudaMemcpyHostToDevice);
	if (e == cudaSuccess)
	{
		ens_dirichlet_flatten_kernel<<<element_grid(units), 256>>>(src_d, ufirst_d, um_d, units, out.qptr, out.qval,
																	out.sptr, out.sval);
		e = cudaGetLastError();
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(0);
	}
	device_free(src_d);
	device_free(ufirst_d);
	device_free(um_d);
	return e == cudaSuccess ? BFVM_OK : cuda_fail(e, "ens_dirichlet_flatten_kernel");
}

int ensemble_build_dirichlet(ensemble_plan& plan)
{
	const int n = plan.count;
	plan.dir_built = true;
	if (n == 0)
		return BFVM_OK;
	std::vector<ens_inst> h(n);
	BFVM_CUDA(cudaMemcpy(h.data(), plan.inst, n * sizeof(ens_inst), cudaMemcpyDeviceToHost));
	for (int which = 0; which < 2; which++)
	{
		// meshes of 3, 2, then 1 dimensions; list 1 takes the interior elements alone where the
		// sweeps write the faces
		std::vector<ens_dir_src> src;
		long long nq = 0, ns = 0;
		ensemble_plan::flat_list& out = plan.dir[which];
		for (int d = 3; d >= 0; d--)
		{
			for (int i = 0; i < n; i++)
			{
				const ens_inst& m = h[i];
				if (m.dims != d)
					continue;
				const bool inner = which == 1 && m.faces;
				ens_dir_src x;
				x.dens = m.dens;
				x.qidx = inner ? m.dir_iqidx : m.dir_qidx;
				x.qval = inner ? m.dir_iqval : m.dir_qval;
				x.qcount = inner ? m.dir_iqcount : m.dir_qcount;
				x.idx = inner ? m.dir_iidx : m.dir_idx;
				x.val = inner ? m.dir_ival : m.dir_val;
				x.count = inner ? m.dir_icount : m.dir_count;
				x.qflat = nq;
				x.sflat = ns;
				nq += x.qcount;
				ns += x.count;
				src.push_back(x);
			}
			out.q_ge[d] = nq;
			out.s_ge[d] = ns;
		}
		int st;
		if ((st = flatten_lists(src, out, nq, ns)))
			return st;
	}
	return BFVM_OK;
}

long long ensemble_dirichlet_entries(const ensemble_plan& plan, int phase)
{
	const int k = std::min(std::max(phase, 0), 3);
	const ensemble_plan::flat_list& l = plan.dir[k == 0 ? 0 : 1];
	return l.q_ge[k] + l.s_ge[k];
}

int ensemble_dirichlet(const ensemble_plan& plan, int phase, cudaStream_t stream)
{
	const int k = std::min(std::max(phase, 0), 3);
	if (!plan.dir_built && plan.count && plan.first_h[ENS_DIRICHLET][plan.count] > 0)
		return fail(BFVM_ERR_STATE, "ensemble Dirichlet lists not built");
	const ensemble_plan::flat_list& l = plan.dir[k == 0 ? 0 : 1];
	const long long nq = l.q_ge[k], ns = l.s_ge[k];
	if (nq + ns == 0)
		return BFVM_OK;
	// four entries per thread, at most 8 CTAs of 256 per SM
	const long long blocks = (std::max(nq, ns) + 1023) / 1024;
	const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(blocks, (long long)current_device_sms() * 8));
	ens_dirichlet_kernel<<<grid, 256, 0, stream>>>(l.qptr, l.qval, nq, l.sptr, l.sval, ns);
	return launched("ens_dirichlet_kernel");
}

template <int ZU>
static void launch_ens_gradient(const ensemble_plan& plan, long long units, cudaStream_t stream)
{
	if (plan.all3d)
		ens_gradient_kernel<true, ZU><<<element_grid(units), 256, 0, stream>>>(
			plan.inst, plan.first[ENS_GRADIENT], plan.unit_mesh[ENS_GRADIENT], units, plan.tune.grad_zc);
	else
		ens_gradient_kernel<false, ZU><<<element_grid(units), 256, 0, stream>>>(
			plan.inst, plan.first[ENS_GRADIENT], plan.unit_mesh[ENS_GRADIENT], units, plan.tune.grad_zc);
}

int ensemble_gradient(const ensemble_plan& plan, cudaStream_t stream)
{
	const long long units = plan.count ? plan.first_h[ENS_GRADIENT][plan.count] : 0;
	if (units == 0)
		return BFVM_OK;
	if (plan.tune.grad_zu == 4)
		launch_ens_gradient<4>(plan, units, stream);
	else
		launch_ens_gradient<8>(plan, units, stream);
	return launched("ens_gradient_kernel");
}

int ensemble_secretion(const ensemble_plan& plan, cudaStream_t stream)
{
	const long long units = plan.count ? plan.first_h[ENS_SECRETION][plan.count] : 0;
	if (units == 0)
		return BFVM_OK;
	ens_secretion_kernel<<<element_grid(units), 256, 0, stream>>>(plan.inst, plan.first[ENS_SECRETION],
																   plan.unit_mesh[ENS_SECRETION], units);
	return launched("ens_secretion_kernel");
}

static size_t ens_sweep_smem(const ensemble_plan& plan, int axis)
{
	return (2 * (size_t)plan.maxP[axis] * 32 + plan.table_floats[axis]) * sizeof(float);
}

template <int AXIS, int MINB>
static int launch_ens_sweep(const ensemble_plan& plan, long long units, cudaStream_t stream)
{
	auto kernel = ens_sweep_kernel<AXIS, MINB>;
	const int P = plan.maxP[AXIS];
	const size_t smem = ens_sweep_smem(plan, AXIS);
	int rc = set_smem(kernel, smem);
	if (rc)
		return rc;
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * P, smem);
	const long long slots = (long long)std::max(per_sm, 1) * current_device_sms() * plan.tune.sweep_split[AXIS];
	const long long chunk = std::max<long long>(1, (units + slots - 1) / slots);
	const unsigned grid = (unsigned)((units + chunk - 1) / chunk);
	kernel<<<grid, dim3(32, P), smem, stream>>>(plan.inst, plan.first[ENS_SWEEP_X + AXIS], plan.count, units, chunk, P);
	return launched("ens_sweep_kernel");
}

bool ensemble_sweep_fits(const ensemble_plan& plan, int axis)
{
	int dev = 0, optin = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
	return plan.maxP[axis] <= ENS_MAX_P_ONE && ens_sweep_smem(plan, axis) <= (size_t)optin;
}

int ensemble_sweep(const ensemble_plan& plan, int axis, cudaStream_t stream)
{
	const long long units = plan.count ? plan.first_h[ENS_SWEEP_X + axis][plan.count] : 0;
	if (units == 0)
		return BFVM_OK;
	if (plan.maxP[axis] > ENS_MAX_P)
	{
		if (axis == 0)
			return launch_ens_sweep<0, 0>(plan, units, stream);
		if (axis == 1)
			return launch_ens_sweep<1, 0>(plan, units, stream);
		return launch_ens_sweep<2, 0>(plan, units, stream);
	}
	const bool one = plan.tune.sweep_minb[axis] == 1;
	if (axis == 0)
		return one ? launch_ens_sweep<0, 1>(plan, units, stream) : launch_ens_sweep<0, 2>(plan, units, stream);
	if (axis == 1)
		return one ? launch_ens_sweep<1, 1>(plan, units, stream) : launch_ens_sweep<1, 2>(plan, units, stream);
	return one ? launch_ens_sweep<2, 1>(plan, units, stream) : launch_ens_sweep<2, 2>(plan, units, stream);
}

} // namespace bfvm
