// Dirichlet overwrite (paraBioFVM src/solver/host/dirichlet_solver.cpp:11-151).
//
// The reference writes the boundary faces in the order x-min, x-max, y-min, y-max, z-min, z-max
// (a later face wins on shared edges and corners) and then the interior Dirichlet voxels.  Here
// one thread owns one voxel that carries a condition and writes, for each substrate that has one,
// the value the reference's order leaves there; elements without a condition are not touched.
// Work items are the voxels of every face that exists followed by the interior Dirichlet voxels,
// so an overwrite costs the conditioned elements only, not a pass over the field.  A voxel listed
// by two work items (a face edge, or a face voxel also listed as interior) receives the same value
// from both.

#include "bfvm_internal.h"

namespace bfvm {

struct dirichlet_work
{
	long long face_start[7]; // work item ranges of the six faces (empty when the face is absent)
	int face_w[6];			 // extent of the faster of the two free axes of each face
	long long n_items;		 // faces + interior voxels
};

__device__ __forceinline__ bool interior_value(const dirichlet_dev& d, long long vid, int s, int S, float& v)
{
	if (!d.has_interior)
		return false;
	const unsigned int w = __ldg(&d.bits[vid >> 5]);
	const unsigned int b = (unsigned int)(vid & 31);
	if (!((w >> b) & 1u))
		return false;
	const long long row = (long long)__ldg(&d.rank[vid >> 5]) + __popc(w & ((1u << b) - 1u));
	if (!d.iconds[row * S + s])
		return false;
	v = d.ivals[row * S + s];
	return true;
}

__global__ void __launch_bounds__(256) dirichlet_scatter_kernel(float* __restrict__ data, const dirichlet_dev dir,
																const dirichlet_work wk, int S, int X, int Y, int Z,
																const long long* __restrict__ rows_vid)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= wk.n_items)
		return;
	long long vid;
	if (t < wk.face_start[6])
	{
		int f = 0;
		while (t >= wk.face_start[f + 1])
			f++;
		const long long r = t - wk.face_start[f];
		const int ax = f >> 1;
		const int fixed = (f & 1) ? (ax == 0 ? X : (ax == 1 ? Y : Z)) - 1 : 0;
		const int a0 = (int)(r % wk.face_w[f]);
		const int a1 = (int)(r / wk.face_w[f]);
		// the two free axes in x, y, z order
		const int x = ax == 0 ? fixed : a0;
		const int y = ax == 1 ? fixed : (ax == 0 ? a0 : a1);
		const int z = ax == 2 ? fixed : a1;
		vid = (long long)x + (long long)X * ((long long)y + (long long)Y * z);
		for (int s = 0; s < S; s++)
		{
			bool hit = false;
			float v = 0.f;
			// faces in the reference's order; a later one overwrites
#pragma unroll
			for (int g = 0; g < 6; g++)
			{
				if (!((dir.face_mask >> g) & 1))
					continue;
				const int gax = g >> 1;
				const int cg = gax == 0 ? x : (gax == 1 ? y : z);
				const int eg = gax == 0 ? X : (gax == 1 ? Y : Z);
				const bool on = (g & 1) ? cg == eg - 1 : cg == 0;
				if (on && dir.face_conds[g * S + s])
				{
					v = dir.face_vals[g * S + s];
					hit = true;
				}
			}
			float iv;
			if (interior_value(dir, vid, s, S, iv))
			{
				v = iv;
				hit = true;
			}
			if (hit)
				data[vid * S + s] = v;
		}
		return;
	}
	// interior voxel: written last by the reference, so its conditions are final
	const long long row = t - wk.face_start[6];
	vid = rows_vid[row];
	for (int s = 0; s < S; s++)
		if (dir.iconds[row * S + s])
			data[vid * S + s] = dir.ivals[row * S + s];
}

int launch_dirichlet(bfvm_solver* st)
{
	const dirichlet_dev d = st->dirichlet();
	if (!d.face_mask && !d.has_interior)
		return BFVM_OK;
	const long long X = st->grid[0], Y = st->grid[1], Z = st->grid[2];
	dirichlet_work wk;
	long long acc = 0;
	for (int f = 0; f < 6; f++)
	{
		wk.face_start[f] = acc;
		const int ax = f >> 1;
		// free axes in x, y, z order: x face -> (y, z); y face -> (x, z); z face -> (x, y)
		const long long w0 = ax == 0 ? Y : X;
		const long long w1 = ax == 2 ? Y : Z;
		wk.face_w[f] = (int)w0;
		if ((d.face_mask >> f) & 1)
			acc += w0 * w1;
	}
	wk.face_start[6] = acc;
	wk.n_items = acc + (d.has_interior ? st->n_interior : 0);
	if (wk.n_items == 0)
		return BFVM_OK;
	const int threads = 256;
	dirichlet_scatter_kernel<<<(unsigned)((wk.n_items + threads - 1) / threads), threads, 0, st->stream>>>(
		st->dens, d, wk, st->S, (int)X, (int)Y, (int)Z, st->dir_rows_vid);
	return check_launch(st, "dirichlet_scatter_kernel");
}

} // namespace bfvm
