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
#include "sweep_common.cuh"

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

// interior_only: the interior elements alone, when the sweeps write the face conditions
// (faces_by_position); otherwise every conditioned element
int launch_dirichlet(bfvm_solver* st, bool interior_only)
{
	overwrite_list full;
	full.qidx = st->dir_qidx;
	full.qval = st->dir_qval;
	full.qcount = st->dir_qcount;
	full.idx = st->dir_idx;
	full.val = st->dir_val;
	full.count = st->dir_count;
	const overwrite_list& l = interior_only && st->face_pos_ok ? st->dir_interior : full;
	const long long n = l.qcount + l.count;
	if (n == 0)
		return BFVM_OK;
	const int threads = 256;
	const long long blocks = std::min<long long>((n + threads - 1) / threads, 148LL * 16);
	dirichlet_scatter_kernel<<<(unsigned)blocks, threads, 0, st->stream>>>(st->dens, l.qidx, l.qval, l.qcount, l.idx,
																		   l.val, l.count);
	return check_launch(st, "dirichlet_scatter_kernel");
}

bool faces_by_position(const bfvm_solver* s)
{
	return s->face_pos_ok && s->face_dirichlet && !s->dir_fused && s->slab_count == 1;
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
	s->face_pos_ok = false;
	device_free(s->face_bits);
	device_free(s->face_vals_d);
	for (auto& t : s->face_tiles)
		device_free(t);
	overwrite_list& l = s->dir_interior;
	device_free(l.qidx);
	device_free(l.qval);
	device_free(l.idx);
	device_free(l.val);
	l = overwrite_list();
}

// Elements sorted by index, split into aligned runs of four consecutive elements and the rest.
struct split_list
{
	std::vector<long long> qidx, sidx;
	std::vector<float4> qval;
	std::vector<float> sval;
};

static split_list split_runs(const std::vector<long long>& idx, const std::vector<float>& val)
{
	std::vector<size_t> order(idx.size());
	for (size_t k = 0; k < order.size(); k++)
		order[k] = k;
	std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return idx[a] < idx[b]; });
	split_list r;
	for (size_t k = 0; k < order.size();)
	{
		const long long e = idx[order[k]];
		if (e % 4 == 0 && k + 3 < order.size() && idx[order[k + 3]] == e + 3)
		{
			r.qidx.push_back(e);
			r.qval.push_back(make_float4(val[order[k]], val[order[k + 1]], val[order[k + 2]], val[order[k + 3]]));
			k += 4;
		}
		else
		{
			r.sidx.push_back(e);
			r.sval.push_back(val[order[k]]);
			k++;
		}
	}
	return r;
}

template <typename T>
static int upload(T** dst, const std::vector<T>& v)
{
	int st = device_alloc(dst, v.size());
	if (st || v.empty())
		return st;
	BFVM_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
	return BFVM_OK;
}

// The face conditions by position (face_pos_ok): the per-substrate face bits and values, the
// interior elements as their own list, and per staged tile of each axis whether a line of the tile
// lies on a conditioned face of another axis.
static int build_face_tables(bfvm_solver* s, const std::vector<long long>& iidx, const std::vector<float>& ival)
{
	const int S = s->S;
	const long long X = s->grid[0], Y = s->grid[1], Z = s->grid[2];
	std::vector<int> bits(S, 0);
	std::vector<float> vals((size_t)6 * S, 0.f);
	for (int f = 0; f < 6; f++)
		for (int k = 0; k < S; k++)
			if (((s->face_mask >> f) & 1) && s->face_conds_h[(size_t)f * S + k])
			{
				bits[k] |= 1 << f;
				vals[(size_t)f * S + k] = s->face_vals_h[(size_t)f * S + k];
			}
	int st;
	if ((st = upload(&s->face_bits, bits)) || (st = upload(&s->face_vals_d, vals)))
		return st;
	const split_list r = split_runs(iidx, ival);
	overwrite_list& l = s->dir_interior;
	if ((st = upload(&l.qidx, r.qidx)) || (st = upload(&l.qval, r.qval)) || (st = upload(&l.idx, r.sidx))
		|| (st = upload(&l.val, r.sval)))
		return st;
	l.qcount = (long long)r.qidx.size();
	l.count = (long long)r.sidx.size();
	auto on = [&](int f) { return ((s->face_mask >> f) & 1) != 0; };
	for (int axis = 0; axis < s->dims; axis++)
	{
		const staged_tiling tl = staged_tiles(s, axis);
		if (tl.items == 0)
			continue;
		std::vector<unsigned char> t(tl.items, 0);
		const long long XS = tl.XS;
		if (axis == 0)
		{
			// rows (y, z) on a y or z face
			for (long long z = 0; z < Z; z++)
				for (long long y = 0; y < Y; y++)
					if ((y == 0 && on(2)) || (y == Y - 1 && on(3)) || (z == 0 && on(4)) || (z == Z - 1 && on(5)))
						t[(z * Y + y) / tl.R] = 1;
		}
		else if (axis == 1)
		{
			// columns (x, s) of a plane on an x face, and every column of a z-face plane
			for (long long z = 0; z < Z; z++)
				for (long long q = 0; q < XS; q++)
				{
					const long long x = q / S;
					if ((x == 0 && on(0)) || (x == X - 1 && on(1)) || (z == 0 && on(4)) || (z == Z - 1 && on(5)))
						t[z * tl.col_tiles + q / 32] = 1;
				}
		}
		else
		{
			// columns (y, x, s) on an x or y face
			for (long long y = 0; y < Y; y++)
				for (long long q = 0; q < XS; q++)
				{
					const long long x = q / S;
					if ((x == 0 && on(0)) || (x == X - 1 && on(1)) || (y == 0 && on(2)) || (y == Y - 1 && on(3)))
						t[(y * XS + q) / 32] = 1;
				}
		}
		if ((st = upload(&s->face_tiles[axis], t)))
			return st;
	}
	s->face_pos_ok = true;
	return BFVM_OK;
}

staged_tiling staged_tiles(const bfvm_solver* s, int axis)
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
	// the face conditions can be written by position only if no interior voxel lies on a
	// conditioned face (then the interior list never meets a face element)
	bool by_position = s->face_mask != 0;
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
	std::vector<long long> iidx;
	std::vector<float> ival;
	for (size_t r = 0; r < iv.size(); r++)
	{
		if (std::binary_search(face_vox.begin(), face_vox.end(), iv[r]))
		{
			by_position = false;
			continue; // resolved with the faces
		}
		for (int k = 0; k < S; k++)
			if (s->int_conds_h[r * S + k])
			{
				idx.push_back(iv[r] * S + k);
				val.push_back(s->int_vals_h[r * S + k]);
				iidx.push_back(iv[r] * S + k);
				ival.push_back(s->int_vals_h[r * S + k]);
			}
	}

	// aligned runs of four consecutive elements, and the rest one by one
	const split_list runs = split_runs(idx, val);
	const std::vector<long long>& qidx = runs.qidx;
	const std::vector<float4>& qval = runs.qval;
	const std::vector<long long>& sidx = runs.sidx;
	const std::vector<float>& sval = runs.sval;

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
	int st2 = build_tile_lists(s, qidx, qval, sidx, sval);
	if (!st2 && by_position)
		st2 = build_face_tables(s, iidx, ival);
	if (st2)
		free_dirichlet(s);
	return st2;
}

} // namespace bfvm
