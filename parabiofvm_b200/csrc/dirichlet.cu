// Dirichlet overwrite (paraBioFVM src/solver/host/dirichlet_solver.cpp:11-151).
//
// The reference writes the boundary faces in the order x-min, x-max, y-min, y-max, z-min, z-max
// (a later face wins on shared edges and corners) and then the interior Dirichlet voxels.  The
// conditions change only through the set-up calls, so the host resolves that order once, when
// they are set: the result holds every conditioned element once with the value the reference
// leaves there, split into aligned runs of four consecutive elements (interior voxels usually
// pin every substrate; one 16-byte store per run) and single elements.  The overwrite is then a
// scatter of the list, touching only the conditioned elements; it runs four times per step
// (before each sweep and after the last).

#include <algorithm>
#include <cstring>

#include "bfvm_internal.h"

namespace bfvm {

__global__ void __launch_bounds__(256) dirichlet_scatter_kernel(float* __restrict__ data,
																const long long* __restrict__ qidx,
																const float4* __restrict__ qval, long long qcount,
																const long long* __restrict__ idx,
																const float* __restrict__ val, long long count)
{
	const long long n = qcount + count;
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
	{
		if (t < qcount)
			*reinterpret_cast<float4*>(data + __ldg(&qidx[t])) = __ldg(&qval[t]);
		else
			data[__ldg(&idx[t - qcount])] = __ldg(&val[t - qcount]);
	}
}

int launch_dirichlet(bfvm_solver* st)
{
	const long long n = st->dir_qcount + st->dir_count;
	if (n == 0)
		return BFVM_OK;
	const int threads = 256;
	const long long blocks = std::min<long long>((n + threads - 1) / threads, 148LL * 16);
	dirichlet_scatter_kernel<<<(unsigned)blocks, threads, 0, st->stream>>>(
		st->dens, st->dir_qidx, st->dir_qval, st->dir_qcount, st->dir_idx, st->dir_val, st->dir_count);
	return check_launch(st, "dirichlet_scatter_kernel");
}

void free_dirichlet(bfvm_solver* s)
{
	device_free(s->dir_qidx);
	device_free(s->dir_qval);
	device_free(s->dir_idx);
	device_free(s->dir_val);
	s->dir_qcount = 0;
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

	// aligned runs of four consecutive elements, and the rest one by one
	std::vector<size_t> order(idx.size());
	for (size_t k = 0; k < order.size(); k++)
		order[k] = k;
	std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return idx[a] < idx[b]; });
	std::vector<long long> qidx, sidx;
	std::vector<float4> qval;
	std::vector<float> sval;
	for (size_t k = 0; k < order.size();)
	{
		const long long e = idx[order[k]];
		if (e % 4 == 0 && k + 3 < order.size() && idx[order[k + 3]] == e + 3)
		{
			qidx.push_back(e);
			qval.push_back(make_float4(val[order[k]], val[order[k + 1]], val[order[k + 2]], val[order[k + 3]]));
			k += 4;
		}
		else
		{
			sidx.push_back(e);
			sval.push_back(val[order[k]]);
			k++;
		}
	}

	free_dirichlet(s);
	int st;
	if ((st = device_alloc(&s->dir_qidx, qidx.size())) || (st = device_alloc(&s->dir_qval, qval.size()))
		|| (st = device_alloc(&s->dir_idx, sidx.size())) || (st = device_alloc(&s->dir_val, sval.size())))
	{
		free_dirichlet(s);
		return st;
	}
	if (!qidx.empty())
	{
		BFVM_CUDA(cudaMemcpy(s->dir_qidx, qidx.data(), qidx.size() * sizeof(long long), cudaMemcpyHostToDevice));
		BFVM_CUDA(cudaMemcpy(s->dir_qval, qval.data(), qval.size() * sizeof(float4), cudaMemcpyHostToDevice));
	}
	if (!sidx.empty())
	{
		BFVM_CUDA(cudaMemcpy(s->dir_idx, sidx.data(), sidx.size() * sizeof(long long), cudaMemcpyHostToDevice));
		BFVM_CUDA(cudaMemcpy(s->dir_val, sval.data(), sval.size() * sizeof(float), cudaMemcpyHostToDevice));
	}
	s->dir_qcount = (long long)qidx.size();
	s->dir_count = (long long)sidx.size();
	return BFVM_OK;
}

} // namespace bfvm
