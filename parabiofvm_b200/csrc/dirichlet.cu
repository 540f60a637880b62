// Dirichlet overwrite (paraBioFVM src/solver/host/dirichlet_solver.cpp:11-151).
//
// The reference writes the boundary faces in the order x-min, x-max, y-min, y-max, z-min, z-max
// (a later face wins on shared edges and corners) and then the interior Dirichlet voxels.  The
// conditions change only through the set-up calls, so the host resolves that order once, when
// they are set: the result is a list of (element index, value) pairs holding every conditioned
// element once with the value the reference leaves there.  The overwrite is then a scatter of the
// list, touching only the conditioned elements; it runs four times per step (before each sweep
// and after the last).

#include <algorithm>
#include <cstring>

#include "bfvm_internal.h"

namespace bfvm {

__global__ void __launch_bounds__(256) dirichlet_scatter_kernel(float* __restrict__ data,
																const long long* __restrict__ idx,
																const float* __restrict__ val, long long count)
{
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (long long)gridDim.x * blockDim.x)
		data[__ldg(&idx[t])] = __ldg(&val[t]);
}

int launch_dirichlet(bfvm_solver* st)
{
	if (st->dir_count == 0)
		return BFVM_OK;
	const int threads = 256;
	const long long blocks = std::min<long long>((st->dir_count + threads - 1) / threads, 148LL * 16);
	dirichlet_scatter_kernel<<<(unsigned)blocks, threads, 0, st->stream>>>(st->dens, st->dir_idx, st->dir_val,
																			st->dir_count);
	return check_launch(st, "dirichlet_scatter_kernel");
}

void free_dirichlet(bfvm_solver* s)
{
	device_free(s->dir_idx);
	device_free(s->dir_val);
	s->dir_count = 0;
}

// Resolve the faces and interior voxels into the overwrite list and upload it.
int rebuild_dirichlet(bfvm_solver* s)
{
	const int S = s->S;
	const long long X = s->grid[0], Y = s->grid[1], Z = s->grid[2];
	const long long ext[3] = { X, Y, Z };

	// voxels on any face that has conditions, each once, ascending
	std::vector<long long> face_vox;
	for (int f = 0; f < 6; f++)
	{
		if (!((s->face_mask >> f) & 1))
			continue;
		const int ax = f >> 1;
		const int a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2; // the free axes, faster first
		long long c[3];
		c[ax] = (f & 1) ? ext[ax] - 1 : 0;
		for (c[a2] = 0; c[a2] < ext[a2]; c[a2]++)
			for (c[a1] = 0; c[a1] < ext[a1]; c[a1]++)
				face_vox.push_back(c[0] + X * (c[1] + Y * c[2]));
	}
	std::sort(face_vox.begin(), face_vox.end());
	face_vox.erase(std::unique(face_vox.begin(), face_vox.end()), face_vox.end());

	std::vector<long long> idx;
	std::vector<float> val;
	idx.reserve(face_vox.size() * S + s->int_vids_h.size() * S);
	val.reserve(idx.capacity());
	const auto& iv = s->int_vids_h;
	for (long long vid : face_vox)
	{
		const long long c[3] = { vid % X, (vid / X) % Y, vid / (X * Y) };
		const auto it = std::lower_bound(iv.begin(), iv.end(), vid);
		const long long row = (it != iv.end() && *it == vid) ? (long long)(it - iv.begin()) : -1;
		for (int k = 0; k < S; k++)
		{
			bool hit = false;
			float v = 0.f;
			for (int f = 0; f < 6; f++) // the reference's face order; a later face overwrites
			{
				if (!((s->face_mask >> f) & 1))
					continue;
				const int ax = f >> 1;
				const bool on = (f & 1) ? c[ax] == ext[ax] - 1 : c[ax] == 0;
				if (on && s->face_conds_h[(size_t)f * S + k])
				{
					v = s->face_vals_h[(size_t)f * S + k];
					hit = true;
				}
			}
			if (row >= 0 && s->int_conds_h[(size_t)row * S + k]) // interior voxels come last
			{
				v = s->int_vals_h[(size_t)row * S + k];
				hit = true;
			}
			if (hit)
			{
				idx.push_back(vid * S + k);
				val.push_back(v);
			}
		}
	}
	for (size_t r = 0; r < iv.size(); r++)
	{
		if (std::binary_search(face_vox.begin(), face_vox.end(), iv[r]))
			continue; // resolved with the faces
		for (int k = 0; k < S; k++)
			if (s->int_conds_h[r * S + k])
			{
				idx.push_back(iv[r] * S + k);
				val.push_back(s->int_vals_h[r * S + k]);
			}
	}

	free_dirichlet(s);
	if (idx.empty())
		return BFVM_OK;
	int st;
	if ((st = device_alloc(&s->dir_idx, idx.size())) || (st = device_alloc(&s->dir_val, val.size())))
	{
		free_dirichlet(s);
		return st;
	}
	BFVM_CUDA(cudaMemcpy(s->dir_idx, idx.data(), idx.size() * sizeof(long long), cudaMemcpyHostToDevice));
	BFVM_CUDA(cudaMemcpy(s->dir_val, val.data(), val.size() * sizeof(float), cudaMemcpyHostToDevice));
	s->dir_count = (long long)idx.size();
	return BFVM_OK;
}

} // namespace bfvm
