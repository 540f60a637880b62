// Pieces shared by the sweep kernels: arguments, the Dirichlet overwrite as seen by one line, the
// block partition and the staging of the coefficient tables in shared memory.
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
	int X, Y, Z;
	dirichlet_dev dir;
	int pre_dirichlet;
	int post_dirichlet;
	int* err; // device error flags (DEVERR_*)
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
	// every field has a neutral default: a line with no conditions applies nothing
	bool any = false;		// anything to apply on this line
	bool line_face = false; // a face of another axis covers the line (after own faces in precedence)
	float line_val = 0.f;
	bool own_min = false, own_max = false; // sweep-axis faces at element 0 / n-1 (merged with line faces)
	float min_val = 0.f, max_val = 0.f;
	long long base_vid = 0, vid_stride = 0;
	int n = 0;
	unsigned long long mask = 0ull; // interior Dirichlet elements of this thread's block
	long long row0 = 0;				// row of its first marked element in the axis tables
	const float* avals = nullptr;
	const unsigned char* aconds = nullptr;

	// fvals / fconds: the face values and conditions [6][S] staged in shared memory
	template <int AXIS>
	__device__ __forceinline__ void init(const dirichlet_dev& d, const float* fvals, const unsigned char* fconds,
										 int i0, int i1, int s, int S, int X, int Y, int Z, int n_)
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
			if (on && fconds[f * S + s])
			{
				order = f;
				line_val = fvals[f * S + s];
			}
		}
		line_face = order >= 0;
		// own-axis faces apply only where they come later than the covering face
		const int fmin = 2 * AXIS, fmax = 2 * AXIS + 1;
		own_min = (d.face_mask & (1 << fmin)) && fconds[fmin * S + s];
		own_max = (d.face_mask & (1 << fmax)) && fconds[fmax * S + s];
		min_val = own_min ? fvals[fmin * S + s] : 0.f;
		max_val = own_max ? fvals[fmax * S + s] : 0.f;
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
		mask = 0ull;
		row0 = 0;
		avals = nullptr;
		aconds = nullptr;
		any = line_face || own_min || own_max;
	}

	// interior Dirichlet elements of block j of line `line` for this sweep axis
	template <int AXIS>
	__device__ __forceinline__ void load_mask(const dirichlet_dev& d, long long line, int j, int P)
	{
		if (d.has_interior)
		{
			const ulonglong2 desc = d.block_desc[AXIS][line * P + j];
			mask = desc.x;
			row0 = (long long)desc.y;
			avals = d.axis_vals[AXIS];
			aconds = d.axis_conds[AXIS];
			any = any || mask != 0ull;
		}
	}

	// interior Dirichlet value of marked element k of this block (substrate s), or v
	__device__ __forceinline__ float marked(int k, int s, int S, float v) const
	{
		const long long row = row0 + __popcll(mask & ((1ull << k) - 1ull));
		return aconds[row * S + s] ? avals[row * S + s] : v;
	}

	// the interior Dirichlet value of line element i (substrate s), or v if it has no condition
	__device__ __forceinline__ float interior(const dirichlet_dev& d, int i, int s, int S, float v) const
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
		return v;
	}

	// element k of the block starting at line position p
	__device__ __forceinline__ float apply(const dirichlet_dev& d, int p, int k, int s, int S, float v) const
	{
		const int i = p + k;
		if (line_face)
			v = line_val;
		if (i == 0 && own_min)
			v = min_val;
		if (i == n - 1 && own_max)
			v = max_val;
		if ((mask >> k) & 1ull)
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

// The Dirichlet overwrite on the M register values of one block (elements p .. p+L-1 of the
// line).  UNI: every block of the line has exactly M elements.  Faces of other axes cover the
// whole line, the sweep axis's own faces only its first and last element, and the interior mask
// marks the few elements that need the bitmap lookup, so the common case costs two predicates.
template <int M, bool UNI>
__device__ __forceinline__ void dirichlet_block(const line_dirichlet& ld, const dirichlet_dev& dir, float (&d)[M],
												int p, int L, int s, int S)
{
	if (ld.line_face)
	{
#pragma unroll
		for (int k = 0; k < M; k++)
			if (UNI || k < L)
				d[k] = ld.line_val;
	}
	if (ld.own_min && p == 0)
		d[0] = ld.min_val;
	if (ld.own_max && p + L == ld.n)
	{
		if (UNI)
			d[M - 1] = ld.max_val;
		else
		{
#pragma unroll
			for (int k = 0; k < M; k++)
				if (k == L - 1)
					d[k] = ld.max_val;
		}
	}
	if (ld.mask)
	{
#pragma unroll
		for (int k = 0; k < M; k++)
			if ((ld.mask >> k) & 1ull)
				d[k] = ld.marked(k, s, S, d[k]);
	}
}

// faces only (the interior marks are applied separately by the TMA kernels)
template <int M, bool UNI>
__device__ __forceinline__ void dirichlet_faces(const line_dirichlet& ld, float (&d)[M], int p, int L)
{
	if (ld.line_face)
	{
#pragma unroll
		for (int k = 0; k < M; k++)
			if (UNI || k < L)
				d[k] = ld.line_val;
	}
	if (ld.own_min && p == 0)
		d[0] = ld.min_val;
	if (ld.own_max && p + L == ld.n)
	{
		if (UNI)
			d[M - 1] = ld.max_val;
		else
		{
#pragma unroll
			for (int k = 0; k < M; k++)
				if (k == L - 1)
					d[k] = ld.max_val;
		}
	}
}

// Thomas solve of one register block of a line with carries exchanged through shared memory.
// `bp` points at b'_0 of this line's substrate with element stride `bstride`; gq / Gp hold the
// whole-block carry products with the same stride; carry_f / carry_t hold one value per block
// of this line at index k * cstride.  All threads of the CTA must call it (two __syncthreads).
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

	asm volatile("" ::: "memory"); // keep the next pass's table loads from being hoisted here
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
	asm volatile("" ::: "memory");
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

	asm volatile("" ::: "memory");
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

// Solve block j of one line.  `line` points at element 0 of the line, `stride` is the element
// stride in floats.  `bp` is the b' column of this line's substrate (bp[i * bstride]).
// carry_f / carry_t hold one value per block of this line at index k*cstride.  All threads of the
// CTA must call this (it contains __syncthreads).
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

// face values [6][S] and conditions [6][S] follow the coefficient tables in shared memory
__host__ __device__ __forceinline__ int table_floats(int n, int P, int Sc, int S)
{
	return n * Sc + Sc + 2 * P * Sc + 6 * S + (6 * S + 3) / 4;
}

__device__ __forceinline__ void stage_faces(const sweep_args& a, float* fvals, unsigned char* fconds)
{
	const int nt = blockDim.x * blockDim.y;
	const int t0 = threadIdx.x + threadIdx.y * blockDim.x;
	for (int t = t0; t < 6 * a.S; t += nt)
	{
		const bool on = (a.dir.face_mask >> (t / a.S)) & 1;
		fvals[t] = on ? a.dir.face_vals[t] : 0.f;
		fconds[t] = on ? a.dir.face_conds[t] : 0;
	}
}


// host helpers for persistent launches
int sm_count(int device);
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


int launch_sweep_tma(bfvm_solver* st, int axis, const sweep_args& a, bool& handled);

} // namespace bfvm
