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

static void free_tiles(dirichlet_tiles& t)
{
	device_free(t.qoff);
	device_free(t.qidx);
	device_free(t.qval);
	device_free(t.soff);
	device_free(t.sidx);
	device_free(t.sval);
	t.items = 0;
}

void free_dirichlet(bfvm_solver* s)
{
	device_free(s->dir_qidx);
	device_free(s->dir_qval);
	device_free(s->dir_idx);
	device_free(s->dir_val);
	s->dir_qcount = 0;
	s->dir_count = 0;
	for (auto& t : s->dir_tiles)
		free_tiles(t);
}

// The tiles of the staged sweep along `axis` (sweep_tma.cu): x, R = 32 / S whole rows; y, 32
// columns of the x*s plane of one z plane; z, 32 columns of the y*x*s plane.  Returns the tile
// count (0 when the staged sweep cannot take the axis) and sets tile(e) for element e.
struct staged_tiling
{
	int axis = 0;
	long long XS = 0, YXS = 0, R = 1, col_tiles = 0, items = 0;

	long long tile(long long e) const
	{
		if (axis == 0)
			return (e / XS) / R;
		if (axis == 1)
			return (e / YXS) * col_tiles + (e % XS) / 32;
		return (e % YXS) / 32;
	}
};

static staged_tiling staged_tiles(const bfvm_solver* s, int axis)
{
	staged_tiling t;
	t.axis = axis;
	const long long X = s->grid[0], Y = s->grid[1], Z = s->grid[2], S = s->S;
	t.XS = X * S;
	t.YXS = Y * X * S;
	if (axis >= s->dims || t.XS % 4 != 0 || (axis == 0 && S > 32))
		return t;
	if (axis == 0)
	{
		t.R = 32 / S;
		t.items = (Y * Z + t.R - 1) / t.R;
	}
	else if (axis == 1)
	{
		t.col_tiles = (t.XS + 31) / 32;
		t.items = Z * t.col_tiles;
	}
	else
		t.items = (t.YXS + 31) / 32;
	return t;
}

// Group the sorted runs and singles by the tiles of each axis (a counting sort keeps each tile's
// entries in ascending element order) and upload them.
static int build_tile_lists(bfvm_solver* s, const std::vector<long long>& qidx, const std::vector<float4>& qval,
							const std::vector<long long>& sidx, const std::vector<float>& sval)
{
	for (int axis = 0; axis < s->dims; axis++)
	{
		const staged_tiling tl = staged_tiles(s, axis);
		if (tl.items == 0 || tl.items > INT32_MAX || s->V * s->S > INT32_MAX)
			continue;
		dirichlet_tiles& t = s->dir_tiles[axis];
		std::vector<int> qoff(tl.items + 1, 0), soff(tl.items + 1, 0);
		for (long long e : qidx)
			qoff[tl.tile(e) + 1]++;
		for (long long e : sidx)
			soff[tl.tile(e) + 1]++;
		for (long long w = 0; w < tl.items; w++)
		{
			qoff[w + 1] += qoff[w];
			soff[w + 1] += soff[w];
		}
		std::vector<int> qi(qidx.size()), si(sidx.size());
		std::vector<float4> qv(qval.size());
		std::vector<float> sv(sval.size());
		{
			std::vector<int> at(qoff.begin(), qoff.end() - 1);
			for (size_t k = 0; k < qidx.size(); k++)
			{
				const int p = at[tl.tile(qidx[k])]++;
				qi[p] = (int)qidx[k];
				qv[p] = qval[k];
			}
			std::vector<int> as(soff.begin(), soff.end() - 1);
			for (size_t k = 0; k < sidx.size(); k++)
			{
				const int p = as[tl.tile(sidx[k])]++;
				si[p] = (int)sidx[k];
				sv[p] = sval[k];
			}
		}
		int st;
		if ((st = device_alloc(&t.qoff, qoff.size())) || (st = device_alloc(&t.soff, soff.size()))
			|| (st = device_alloc(&t.qidx, qi.size())) || (st = device_alloc(&t.qval, qv.size()))
			|| (st = device_alloc(&t.sidx, si.size())) || (st = device_alloc(&t.sval, sv.size())))
		{
			free_tiles(t);
			return st;
		}
		BFVM_CUDA(cudaMemcpy(t.qoff, qoff.data(), qoff.size() * sizeof(int), cudaMemcpyHostToDevice));
		BFVM_CUDA(cudaMemcpy(t.soff, soff.data(), soff.size() * sizeof(int), cudaMemcpyHostToDevice));
		if (!qi.empty())
		{
			BFVM_CUDA(cudaMemcpy(t.qidx, qi.data(), qi.size() * sizeof(int), cudaMemcpyHostToDevice));
			BFVM_CUDA(cudaMemcpy(t.qval, qv.data(), qv.size() * sizeof(float4), cudaMemcpyHostToDevice));
		}
		if (!si.empty())
		{
			BFVM_CUDA(cudaMemcpy(t.sidx, si.data(), si.size() * sizeof(int), cudaMemcpyHostToDevice));
			BFVM_CUDA(cudaMemcpy(t.sval, sv.data(), sv.size() * sizeof(float), cudaMemcpyHostToDevice));
		}
		t.items = tl.items;
	}
	return BFVM_OK;
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
	if (s->slab_count > 1 || qidx.size() + sidx.size() == 0)
		return BFVM_OK; // slabs step axis by axis through the unfused calls
	const int st2 = build_tile_lists(s, qidx, qval, sidx, sval);
	if (st2)
		free_dirichlet(s);
	return st2;
}

} // namespace bfvm
