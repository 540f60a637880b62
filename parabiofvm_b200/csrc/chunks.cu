// Lines longer than the staged sweep takes (more than 16 blocks of 32 elements), cut into chunks
// that it does take, the way a z line is cut into slabs (slab.cu), here along any axis of one mesh.
//
// Every line is one tridiagonal system (src/solver/host/diffusion_solver.cpp:297-334).  Chunk k
// holds elements [b_k, b_{k+1}) of every line.  The sweep of the axis runs in two passes:
//   1. carries: per line, each chunk's A (its last forward value) and B (its first solution), both
//      from zero carries, are weighted sums over the elements near the chunk's two ends
//      (slab_reduce_weights: the weights shrink geometrically away from the end they belong to),
//      one thread per sum.  The true carries follow from them by the recurrences of
//      slab_coefficients,
//        C_{k+1} = A_k + Gamma_k C_k (C_0 = 0),   X_{k-1} = B_k + beta_k C_k + Lambda_k X_k (X_{K-1} = 0),
//      one thread per line, written to carry[k][2][lines];
//   2. solve: the staged sweep of each chunk (sweep_tma.cu, the slab variant) enters every line with
//      the chunk's carries and writes the field.
// In exact arithmetic this is the Thomas solve of the whole line; in float it agrees with it to
// rounding.  The first pass reads a few dozen elements per chunk end, the second one reads and
// writes the field once, at the staged sweep's rate.

#include <algorithm>
#include <cstring>
#include <numeric>
#include <type_traits>

#include "bfvm_internal.h"
#include "sweep_common.cuh"

namespace bfvm {

static constexpr int CHUNK_MAX = 8;

struct chunk_meta
{
	int count;
	int a_first[CHUNK_MAX], na[CHUNK_MAX], b0[CHUNK_MAX], nb[CHUNK_MAX];
	long long w_off[CHUNK_MAX];
};

// Element i of line l lies at u[base(l) + i * es]: z lines, base = l, es = Y X S; y lines
// (l = z X S + column), base = z Y X S + column, es = X S; x lines (l = row S + s), base = row X S
// + s, es = S.
template <int AXIS>
__device__ __forceinline__ long long line_base(long long l, int S, long long XS, long long YXS)
{
	if (AXIS == 2)
		return l;
	if (AXIS == 1)
	{
		const long long z = l / XS;
		return z * YXS + (l - z * XS);
	}
	return (l / S) * XS + l % S;
}

// The end sums of the chunks, one thread per (V lines, chunk boundary, side): at boundary k
// (between chunks k and k + 1), side 0 is chunk k's A (its last forward value), side 1 chunk
// k + 1's B (its first solution), both from zero carries; ex[k][side][lines].  Each sum runs from
// its smallest weights to its largest (towards the end it belongs to), the order of the slab
// reduce pass.  V = 4 when S % 4 == 0: four consecutive lines, whose elements (and weights) are
// four consecutive floats, read as one 16-byte load.
template <int V>
__device__ __forceinline__ void load_v(const float* p, float (&x)[V])
{
	if constexpr (V == 4)
	{
		const float4 v = __ldg(reinterpret_cast<const float4*>(p));
		x[0] = v.x;
		x[1] = v.y;
		x[2] = v.z;
		x[3] = v.w;
	}
	else
		x[0] = __ldg(p);
}

template <int AXIS, int V>
__global__ void __launch_bounds__(256) chunk_sums_kernel(const float* __restrict__ u, const float* __restrict__ rw,
														  float* __restrict__ ex, long long lines, int S, long long XS,
														  long long YXS, chunk_meta m)
{
	const long long groups = lines / V;
	const long long total = groups * 2 * (m.count - 1);
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
		 t += (long long)gridDim.x * blockDim.x)
	{
		const long long l = (t % groups) * V;
		const int bs = (int)(t / groups); // 2 * boundary + side
		const int k = bs >> 1, side = bs & 1;
		const int s = (int)(l % S);
		const long long es = AXIS == 2 ? YXS : (AXIS == 1 ? XS : S);
		const long long base = line_base<AXIS>(l, S, XS, YXS);
		float acc[V];
#pragma unroll
		for (int v = 0; v < V; v++)
			acc[v] = 0.f;
		if (side == 0)
		{
			const float* wa = rw + m.w_off[k];
			const float* p = u + base + (long long)m.a_first[k] * es;
#pragma unroll 8
			for (int i = 0; i < m.na[k]; i++)
			{
				float x[V], w[V];
				load_v<V>(p + (long long)i * es, x);
				load_v<V>(wa + (size_t)i * S + s, w);
#pragma unroll
				for (int v = 0; v < V; v++)
					acc[v] = fmaf(w[v], x[v], acc[v]);
			}
		}
		else
		{
			const float* wb = rw + m.w_off[k + 1] + (size_t)m.na[k + 1] * S;
			const float* p = u + base + (long long)m.b0[k + 1] * es;
#pragma unroll 8
			for (int i = m.nb[k + 1] - 1; i >= 0; i--)
			{
				float x[V], w[V];
				load_v<V>(p + (long long)i * es, x);
				load_v<V>(wb + (size_t)i * S + s, w);
#pragma unroll
				for (int v = 0; v < V; v++)
					acc[v] = fmaf(w[v], x[v], acc[v]);
			}
		}
#pragma unroll
		for (int v = 0; v < V; v++)
			ex[(size_t)bs * lines + l + v] = acc[v];
	}
}

// The chunks' carries from the end sums, one thread per line: C_{k+1} = A_k + Gamma_k C_k from
// C_0 = 0, X_{k-1} = B_k + beta_k C_k + Lambda_k X_k from X_{K-1} = 0; carry[k][2][lines] = (C, X).
__global__ void __launch_bounds__(256) chunk_combine_kernel(const float* __restrict__ ex, const float* __restrict__ coef,
															 float* __restrict__ carry, long long lines, int S, int count)
{
	for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < lines;
		 l += (long long)gridDim.x * blockDim.x)
	{
		const int s = (int)(l % S);
		float Ck[CHUNK_MAX];
		Ck[0] = 0.f;
		float C = 0.f;
		for (int k = 0; k + 1 < count; k++)
		{
			C = fmaf(__ldg(&coef[(size_t)k * 3 * S + s]), C, __ldg(&ex[(size_t)(2 * k) * lines + l]));
			Ck[k + 1] = C;
		}
		float X = 0.f;
		carry[((size_t)(count - 1) * 2 + 1) * lines + l] = 0.f;
		for (int k = count - 1; k > 0; k--)
		{
			const float* ck = coef + (size_t)k * 3 * S;
			X = fmaf(__ldg(&ck[2 * S + s]), X, fmaf(__ldg(&ck[S + s]), Ck[k], __ldg(&ex[(size_t)(2 * k - 1) * lines + l])));
			carry[((size_t)(k - 1) * 2 + 1) * lines + l] = X;
		}
		for (int k = 0; k < count; k++)
			carry[(size_t)k * 2 * lines + l] = Ck[k];
	}
}

void free_chunks(sweep_plan& p)
{
	auto& ch = p.chunks;
	for (float*& t : ch.vtab)
		device_free(t);
	device_free(ch.rw);
	device_free(ch.coef);
	device_free(ch.carry);
	device_free(ch.ex);
	ch = sweep_plan::chunks_t();
}

// Chunk bounds for a line of n elements: chunks of at most max_len elements, each bound a multiple
// of `align` (x lines: a chunk's part of a row must start on a 16-byte boundary); equal chunks when
// that takes at most twice the fewest, else the fewest of near-equal lengths.  Empty when no such
// cut exists within CHUNK_MAX chunks.
static std::vector<int> chunk_bounds(int n, int align, int max_len)
{
	// equal chunks first (one launch sweeps them all), within twice the fewest chunks
	const int K0 = (n + max_len - 1) / max_len;
	for (int K = K0; K <= std::min(CHUNK_MAX, 2 * K0); K++)
		if (n % K == 0 && (n / K) % align == 0 && n / K >= 2)
		{
			std::vector<int> b(K + 1);
			for (int k = 0; k <= K; k++)
				b[k] = k * (n / K);
			return b;
		}
	for (int K = K0; K <= CHUNK_MAX; K++)
	{
		std::vector<int> b(K + 1);
		b[0] = 0;
		b[K] = n;
		bool ok = true;
		for (int k = 1; k < K; k++)
			b[k] = (int)(((long long)n * k / K) / align * align);
		for (int k = 0; k < K && ok; k++)
			ok = b[k + 1] - b[k] >= 2 && b[k + 1] - b[k] <= max_len;
		if (ok)
			return b;
	}
	return {};
}

int build_chunks(bfvm_solver* s, int axis, const std::vector<float>& bp, const std::vector<float>& c)
{
	sweep_plan& p = s->plan[axis];
	free_chunks(p);
	const int n = s->grid[axis];
	const long long S = s->S, XS = (long long)s->grid[0] * S;
	// chunk_elements 0 (automatic): lines beyond 512 elements (the staged sweep's 16 blocks of 32) in
	// chunks of at most 320 along x and 512 along y and z, the fastest measured at 640-1024
	// elements (an x chunk of 512 and 4 substrates is 64 KB of stage); otherwise lines beyond
	// chunk_elements in chunks of at most that
	const int max_len = s->chunk_elements > 0 ? s->chunk_elements : (axis == 0 ? 320 : 512);
	const int longest_whole = s->chunk_elements > 0 ? s->chunk_elements : 512;
	if (axis >= s->dims || n <= longest_whole || XS % 4 != 0 || (axis == 0 && S > 32) || s->slab_global_z > 0)
		return BFVM_OK;
	const int align = axis == 0 ? 4 / std::gcd(4, (int)S) : 1;
	const std::vector<int> bounds = chunk_bounds(n, align, max_len);
	if (bounds.empty())
		return BFVM_OK;
	auto& ch = p.chunks;
	const int K = (int)bounds.size() - 1;
	ch.bounds = bounds;
	ch.lines = s->V * S / n;
	std::vector<float> rw_all, coef;
	int st;
	for (int k = 0; k < K; k++)
	{
		std::vector<float> vt, w;
		int vP, pad, af, na, nb;
		precompute_padded_range(n, bounds[k], bounds[k + 1], (int)S, bp, c, vP, pad, vt);
		float* dv = nullptr;
		if ((st = device_alloc(&dv, vt.size())))
		{
			free_chunks(p);
			return st;
		}
		ch.vtab.push_back(dv);
		BFVM_CUDA(cudaMemcpy(dv, vt.data(), vt.size() * sizeof(float), cudaMemcpyHostToDevice));
		ch.vP.push_back(vP);
		ch.pad.push_back(pad);
		// end sums truncated where the dropped weights total 2^-36 of the line's largest value, 12 bits
		// below the rounding of a float (the slabs keep 2^-50; this reads a third fewer elements)
		slab_reduce_weights(n, bounds[k], bounds[k + 1], (int)S, bp, c, w, af, na, nb, -36);
		ch.a_first.push_back(af);
		ch.na.push_back(na);
		ch.nb.push_back(nb);
		ch.w_off.push_back((long long)rw_all.size());
		rw_all.insert(rw_all.end(), w.begin(), w.end());
	}
	slab_coefficients(n, (int)S, bp, c, K, bounds.data(), coef);
	if ((st = device_alloc(&ch.rw, std::max<size_t>(rw_all.size(), 4))) || (st = device_alloc(&ch.coef, coef.size()))
		|| (st = device_alloc(&ch.carry, (size_t)K * 2 * ch.lines))
		|| (st = device_alloc(&ch.ex, (size_t)(K - 1) * 2 * ch.lines)))
	{
		free_chunks(p);
		return st;
	}
	if (!rw_all.empty())
		BFVM_CUDA(cudaMemcpy(ch.rw, rw_all.data(), rw_all.size() * sizeof(float), cudaMemcpyHostToDevice));
	BFVM_CUDA(cudaMemcpy(ch.coef, coef.data(), coef.size() * sizeof(float), cudaMemcpyHostToDevice));
	ch.count = K;
	return BFVM_OK;
}

int rebuild_chunks(bfvm_solver* s)
{
	for (int axis = 0; axis < s->dims; axis++)
	{
		const int n = s->grid[axis];
		if (n < 2)
			continue;
		std::vector<float> bp, ep, g, G, c, gq, Gp;
		int P, bl, ex;
		precompute_axis(n, s->voxel[axis], s->dims, s->S, s->dt, s->D.data(), s->decay.data(), 32, bp, ep, g, G, c, gq,
						Gp, P, bl, ex);
		int st = build_chunks(s, axis, bp, c);
		if (st)
			return st;
	}
	return BFVM_OK;
}

// The chunks of a launch: all of them when they have one length (one launch), else chunk k alone.
static line_chunks chunk_set(const sweep_plan& p, int k)
{
	const auto& ch = p.chunks;
	line_chunks lc;
	const bool equal = std::all_of(ch.vP.begin(), ch.vP.end(), [&](int v) { return v == ch.vP[0]; })
					   && std::all_of(ch.pad.begin(), ch.pad.end(), [&](int v) { return v == ch.pad[0]; });
	const int k0 = equal ? 0 : k, k1 = equal ? ch.count : k + 1;
	lc.count = k1 - k0;
	for (int i = k0; i < k1; i++)
	{
		lc.e0[i - k0] = ch.bounds[i];
		lc.vtab[i - k0] = ch.vtab[i];
	}
	lc.len = ch.bounds[k0 + 1] - ch.bounds[k0];
	lc.vP = ch.vP[k0];
	lc.pad = ch.pad[k0];
	lc.carry = ch.carry + (size_t)k0 * 2 * ch.lines;
	lc.lines = ch.lines;
	return lc;
}

// launches of a chunked sweep: 1 when the chunks have one length
static int chunk_launches(const sweep_plan& p) { return chunk_set(p, 0).count == p.chunks.count ? 1 : p.chunks.count; }

int launch_chunked_sweep(bfvm_solver* st, int axis, bool& handled)
{
	handled = false;
	const sweep_plan& p = st->plan[axis];
	const auto& ch = p.chunks;
	// y and z lines of few lines per mesh (fewer than 2^17: 128 x 128 x 4 or smaller cross-sections)
	// sweep faster whole in the ensemble sweep, whose one launch has no carries pass (measured at
	// 1024-element lines: 3.26-3.28 against 2.99-3.16 TB/s)
	if (ch.count < 2 || !st->use_tma || (axis > 0 && ch.lines < (1LL << 17)))
		return BFVM_OK;
	sweep_args a;
	std::memset(&a, 0, sizeof(a));
	a.data = st->dens;
	a.S = st->S;
	a.X = st->grid[0];
	a.Y = st->grid[1];
	a.Z = st->grid[2];
	a.err = st->dev_error;
	a.wait_limit = st->wait_limit_cycles;
	a.drop_tile_copy = st->drop_tile_copy;
	a.face_bits = st->face_bits;
	a.face_vals = st->face_vals_d;
	// every chunk must be one the staged sweep takes, before anything is launched
	const int launches = chunk_launches(p);
	for (int k = 0; k < launches; k++)
	{
		const line_chunks lc = chunk_set(p, k);
		std::vector<sweep_tuning> shapes;
		bool h = false;
		int rc = launch_sweep_tma(st, axis, a, h, nullptr, &shapes, false, nullptr, 0, -1, &lc);
		if (rc || shapes.empty())
			return rc;
	}
	chunk_meta m;
	std::memset(&m, 0, sizeof(m));
	m.count = ch.count;
	for (int k = 0; k < ch.count; k++)
	{
		m.a_first[k] = ch.a_first[k];
		m.na[k] = ch.na[k];
		m.b0[k] = ch.bounds[k];
		m.nb[k] = ch.nb[k];
		m.w_off[k] = ch.w_off[k];
	}
	const long long XS = (long long)st->grid[0] * st->S, YXS = XS * st->grid[1];
	const int threads = 256;
	// four lines per thread when S % 4 == 0 (their elements and weights are 16-byte aligned runs)
	const int V = st->S % 4 == 0 ? 4 : 1;
	const long long sums = ch.lines / V * 2 * (ch.count - 1);
	const unsigned blocks = (unsigned)std::min<long long>((sums + threads - 1) / threads, 148LL * 32);
	auto sums_kernel = [&](auto axis_tag, auto v_tag) {
		constexpr int AX = decltype(axis_tag)::value, VV = decltype(v_tag)::value;
		chunk_sums_kernel<AX, VV><<<blocks, threads, 0, st->stream>>>(st->dens, ch.rw, ch.ex, ch.lines, st->S, XS, YXS, m);
	};
	using A0 = std::integral_constant<int, 0>;
	using A1 = std::integral_constant<int, 1>;
	using A2 = std::integral_constant<int, 2>;
	using V1 = std::integral_constant<int, 1>;
	using V4 = std::integral_constant<int, 4>;
	if (axis == 0)
		V == 4 ? sums_kernel(A0(), V4()) : sums_kernel(A0(), V1());
	else if (axis == 1)
		V == 4 ? sums_kernel(A1(), V4()) : sums_kernel(A1(), V1());
	else
		V == 4 ? sums_kernel(A2(), V4()) : sums_kernel(A2(), V1());
	int rc = check_launch(st, "chunk_sums_kernel");
	if (rc)
		return rc;
	const unsigned cblocks = (unsigned)std::min<long long>((ch.lines + threads - 1) / threads, 148LL * 16);
	chunk_combine_kernel<<<cblocks, threads, 0, st->stream>>>(ch.ex, ch.coef, ch.carry, ch.lines, st->S, ch.count);
	rc = check_launch(st, "chunk_combine_kernel");
	for (int k = 0; k < launches && !rc; k++)
	{
		const line_chunks lc = chunk_set(p, k);
		bool h = false;
		rc = launch_sweep_tma(st, axis, a, h, nullptr, nullptr, false, nullptr, 0, -1, &lc);
		if (!rc && !h)
			rc = fail(BFVM_ERR_STATE, "a chunk of the lines was not staged");
	}
	if (!rc)
		handled = true;
	return rc;
}

} // namespace bfvm
