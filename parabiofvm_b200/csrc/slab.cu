// z-slabs: one mesh split along z into slabs, each held by its own solver (normally one per GPU).
//
// The x and y sweeps, the Dirichlet overwrites, secretion and release never cross a z plane, so
// each slab runs them on its own planes unchanged.  Two parts of the step couple the slabs:
//
// * The z sweep.  Every z line is one tridiagonal system over the whole mesh.  A slab holds the
//   whole line's Thomas coefficients for its planes (precompute_padded_range) and solves its part
//   of every line in two passes around one exchange:
//     1. reduce: publish, per line, A = the forward value at the slab's last plane and B = the
//        solution at its first plane, both from zero carries (2 floats per line).  Both are linear
//        in the slab's field, with weights that shrink geometrically away from the plane each
//        belongs to (slab_reduce_weights), so slab_reduce_kernel forms them as sums over the
//        planes near the slab's edges alone;
//     2. the caller gathers every slab's (A, B) (an all-gather over NCCL, or copies on one GPU);
//     3. combine: the slab's true carries follow from the gathered values by the recurrences of
//        slab_coefficients, C_{k+1} = A_k + Gamma_k C_k and X_{k-1} = B_k + beta_k C_k + Lambda_k X_k;
//     4. solve: the staged sweep enters every line with those carries and writes the field.
//   In exact arithmetic this is the Thomas solve of the whole line; in float it agrees with the
//   single-solver sweep to rounding.
// * The gradient.  The z difference at a slab's first and last plane needs the neighbouring
//   slabs' edge planes: the caller passes them in and an edge kernel rewrites those two planes of
//   the z component after the ordinary gradient kernel.
//
// No kernel here waits on another GPU: the exchange happens between launches, on the caller's
// side, so slabs can be emulated as several solvers on one GPU.

#include <algorithm>

#include "bfvm_internal.h"

namespace bfvm {

static constexpr int SLAB_MAX = 64;

// carry[0][q] = C and carry[1][q] = X of slab `me` for every z line q, from every slab's (A, B)
// in ex[count][2][lines] and the coefficients coef[count][3][S] (Gamma, beta, Lambda).
__global__ void __launch_bounds__(256) slab_combine_kernel(const float* __restrict__ ex,
															const float* __restrict__ coef, float* __restrict__ carry,
															long long lines, int S, int count, int me)
{
	float Ck[SLAB_MAX];
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < lines;
		 q += (long long)gridDim.x * blockDim.x)
	{
		const int s = (int)(q % S);
		float C = 0.f;
		Ck[0] = 0.f;
		for (int k = 0; k + 1 < count; k++)
		{
			C = fmaf(__ldg(&coef[(size_t)k * 3 * S + s]), C, __ldg(&ex[(size_t)k * 2 * lines + q]));
			Ck[k + 1] = C;
		}
		float X = 0.f;
		for (int k = count - 1; k > me; k--)
		{
			const float* ck = coef + (size_t)k * 3 * S;
			X = fmaf(__ldg(&ck[2 * S + s]), X,
					 fmaf(__ldg(&ck[S + s]), Ck[k], __ldg(&ex[((size_t)k * 2 + 1) * lines + q])));
		}
		carry[q] = Ck[me];
		carry[lines + q] = X;
	}
}

// The reduce pass of a slab's z sweep.  For every z line q (s = q mod S):
//   out[q] = A = sum_{k < na} wa[k][s] u[a0 + k][q],   out[lines + q] = B = sum_{k < nb} wb[k][s] u[k][q],
// each summed from its smallest weights to its largest (towards the slab edge it belongs to).
// V lines per thread: 4 when S is a multiple of 4 (16-byte loads of the field and the weights).
template <int V>
__global__ void __launch_bounds__(256) slab_reduce_kernel(const float* __restrict__ u, const float* __restrict__ wa,
														   const float* __restrict__ wb, float* __restrict__ out,
														   long long lines, int S, int a0, int na, int nb)
{
	const long long q = (blockIdx.x * (long long)blockDim.x + threadIdx.x) * V;
	if (q >= lines)
		return;
	const int s = (int)(q % S);
	auto load = [](const float* p, float (&x)[V]) {
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
	};
	float A[V], B[V];
#pragma unroll
	for (int i = 0; i < V; i++)
		A[i] = B[i] = 0.f;
	const float* ua = u + (long long)a0 * lines + q;
#pragma unroll 8
	for (int k = 0; k < na; k++)
	{
		float x[V], w[V];
		load(ua + (long long)k * lines, x);
		load(wa + (size_t)k * S + s, w);
#pragma unroll
		for (int i = 0; i < V; i++)
			A[i] = fmaf(w[i], x[i], A[i]);
	}
#pragma unroll 8
	for (int k = nb - 1; k >= 0; k--)
	{
		float x[V], w[V];
		load(u + (long long)k * lines + q, x);
		load(wb + (size_t)k * S + s, w);
#pragma unroll
		for (int i = 0; i < V; i++)
			B[i] = fmaf(w[i], x[i], B[i]);
	}
#pragma unroll
	for (int i = 0; i < V; i++)
	{
		out[q + i] = A[i];
		out[lines + q + i] = B[i];
	}
}

static int launch_slab_reduce(bfvm_solver* s, float* out)
{
	const long long lines = (long long)s->grid[0] * s->grid[1] * s->S;
	const int V = s->S % 4 == 0 ? 4 : 1;
	const int threads = 256;
	const long long blocks = (lines / V + threads - 1) / threads;
	const float* wa = s->slab_rw;
	const float* wb = s->slab_rw + (size_t)s->slab_na * s->S;
	if (V == 4)
		slab_reduce_kernel<4><<<(unsigned)blocks, threads, 0, s->stream>>>(s->dens, wa, wb, out, lines, s->S,
																		   s->slab_a0, s->slab_na, s->slab_nb);
	else
		slab_reduce_kernel<1><<<(unsigned)blocks, threads, 0, s->stream>>>(s->dens, wa, wb, out, lines, s->S,
																		   s->slab_a0, s->slab_na, s->slab_nb);
	return check_launch(s, "slab_reduce_kernel");
}

// The z component of the gradient on a slab's first plane (edge 0, when `below` is given) and last
// plane (edge 1, when `above` is given), with the neighbour's plane in place of the missing one:
// the central difference (u[z+1] - u[z-1]) * (1/(2h)) of gradient.cu, here across the slab edge.
__global__ void __launch_bounds__(256) slab_gradient_edges_kernel(const float* __restrict__ u, float* __restrict__ gz,
																   const float* __restrict__ below,
																   const float* __restrict__ above, long long plane,
																   int Zl, float cz)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i >= plane)
		return;
	const int edge = blockIdx.y;
	if (edge == 0 && below)
		gz[i] = __fmul_rn(__fsub_rn(__ldg(&u[plane + i]), __ldg(&below[i])), cz);
	if (edge == 1 && above)
	{
		const long long last = (long long)(Zl - 1) * plane;
		gz[last + i] = __fmul_rn(__fsub_rn(__ldg(&above[i]), __ldg(&u[last - plane + i])), cz);
	}
}

static int slab_state(bfvm_solver* s)
{
	if (!s)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null solver");
	if (s->slab_global_z == 0)
		return fail(BFVM_ERR_STATE, "not a slab solver (bfvm_create_slab)");
	if (cudaSetDevice(s->device) != cudaSuccess)
		return cuda_fail(cudaGetLastError(), "cudaSetDevice");
	return BFVM_OK;
}

} // namespace bfvm

using namespace bfvm;

extern "C" {

int bfvm_slab_coefficients(int32_t planes, int32_t voxel_z, int32_t substrates, float time_step,
						   const float* diffusion_coefficients, const float* decay_rates, int32_t slab_count,
						   const int32_t* slab_planes, float* coefficients)
{
	if (planes < 2 || voxel_z <= 0 || substrates < 1 || !diffusion_coefficients || !decay_rates || !coefficients)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "bad mesh or substrate arguments");
	if (slab_count < 1 || slab_count > SLAB_MAX || !slab_planes)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "slab_count must be 1.." + std::to_string(SLAB_MAX));
	if (slab_planes[0] != 0 || slab_planes[slab_count] != planes)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "slab_planes must run from 0 to the mesh's plane count");
	for (int k = 0; k < slab_count; k++)
		if (slab_planes[k + 1] <= slab_planes[k])
			return fail(BFVM_ERR_INVALID_ARGUMENT, "slab_planes must increase");
	std::vector<float> bp, ep, g, G, c, gq, Gp, out;
	int P, bl, ex;
	precompute_axis(planes, voxel_z, 3, substrates, time_step, diffusion_coefficients, decay_rates, 32, bp, ep, g, G,
					c, gq, Gp, P, bl, ex);
	slab_coefficients(planes, substrates, bp, c, slab_count, slab_planes, out);
	std::copy(out.begin(), out.end(), coefficients);
	return BFVM_OK;
}

int bfvm_slab_reduce_weights(int32_t planes, int32_t voxel_z, int32_t substrates, float time_step,
							 const float* diffusion_coefficients, const float* decay_rates, int32_t first_plane,
							 int32_t end_plane, float* weights, int32_t* a_first, int32_t* a_count, int32_t* b_count)
{
	if (planes < 2 || voxel_z <= 0 || substrates < 1 || !diffusion_coefficients || !decay_rates || !weights || !a_first
		|| !a_count || !b_count)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "bad mesh, substrate or output arguments");
	if (first_plane < 0 || end_plane <= first_plane || end_plane > planes)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "the slab's planes must lie within the mesh");
	std::vector<float> bp, ep, g, G, c, gq, Gp, w;
	int P, bl, ex, af, na, nb;
	precompute_axis(planes, voxel_z, 3, substrates, time_step, diffusion_coefficients, decay_rates, 32, bp, ep, g, G,
					c, gq, Gp, P, bl, ex);
	slab_reduce_weights(planes, first_plane, end_plane, substrates, bp, c, w, af, na, nb);
	std::copy(w.begin(), w.end(), weights);
	*a_first = af;
	*a_count = na;
	*b_count = nb;
	return BFVM_OK;
}

int bfvm_slab_info(const bfvm_solver* s, int32_t* slab_count, int32_t* slab, int32_t* first_plane,
				   int32_t* mesh_planes)
{
	if (!s)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "null solver");
	const bool is_slab = s->slab_global_z > 0;
	if (slab_count)
		*slab_count = s->slab_count;
	if (slab)
		*slab = s->slab_index;
	if (first_plane)
		*first_plane = s->slab_z0;
	if (mesh_planes)
		*mesh_planes = is_slab ? s->slab_global_z : s->grid[2];
	return BFVM_OK;
}

int bfvm_slab_diffusion_begin(bfvm_solver* s, float* exchange)
{
	int st;
	if ((st = slab_state(s)))
		return st;
	if (!exchange)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "exchange buffer is null");
	if (s->slab_phase)
		return fail(BFVM_ERR_STATE, "bfvm_slab_diffusion_begin called twice without bfvm_slab_diffusion_end");
	if ((st = launch_sweep(s, 0, false)) || (st = launch_sweep(s, 1, false)) || (st = launch_dirichlet(s))
		|| (st = launch_slab_reduce(s, exchange)))
		return st;
	s->slab_phase = 1;
	return BFVM_OK;
}

int bfvm_slab_diffusion_end(bfvm_solver* s, const float* exchange_all)
{
	int st;
	if ((st = slab_state(s)))
		return st;
	if (!exchange_all)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "gathered exchange buffer is null");
	if (!s->slab_phase)
		return fail(BFVM_ERR_STATE, "bfvm_slab_diffusion_end without bfvm_slab_diffusion_begin");
	const long long lines = (long long)s->grid[0] * s->grid[1] * s->S;
	const int threads = 256;
	const long long blocks = std::min<long long>((lines + threads - 1) / threads, 148LL * 16);
	slab_combine_kernel<<<(unsigned)blocks, threads, 0, s->stream>>>(exchange_all, s->slab_coef, s->slab_carry, lines,
																	 s->S, s->slab_count, s->slab_index);
	if ((st = check_launch(s, "slab_combine_kernel")) || (st = launch_slab_z(s))
		|| (st = launch_dirichlet(s)))
		return st;
	s->slab_phase = 0;
	return BFVM_OK;
}

int bfvm_slab_edge_planes(bfvm_solver* s, float* first_plane, float* last_plane)
{
	int st;
	if ((st = slab_state(s)))
		return st;
	const size_t plane = (size_t)s->grid[0] * s->grid[1] * s->S;
	if (first_plane)
		BFVM_CUDA(cudaMemcpyAsync(first_plane, s->dens, plane * sizeof(float), cudaMemcpyDeviceToDevice, s->stream));
	if (last_plane)
		BFVM_CUDA(cudaMemcpyAsync(last_plane, s->dens + (size_t)(s->grid[2] - 1) * plane, plane * sizeof(float),
								  cudaMemcpyDeviceToDevice, s->stream));
	return BFVM_OK;
}

int bfvm_slab_gradient_solve(bfvm_solver* s, const float* plane_below, const float* plane_above)
{
	int st;
	if ((st = slab_state(s)))
		return st;
	const bool has_below = s->slab_index > 0, has_above = s->slab_index < s->slab_count - 1;
	if ((has_below && !plane_below) || (has_above && !plane_above))
		return fail(BFVM_ERR_INVALID_ARGUMENT, "a neighbouring slab's edge plane is missing");
	if ((st = launch_gradient(s)))
		return st;
	if (!has_below && !has_above)
		return BFVM_OK;
	const long long plane = (long long)s->grid[0] * s->grid[1] * s->S;
	const float cz = 1.f / (s->voxel[2] * 2);
	const int threads = 256;
	const dim3 blocks((unsigned)((plane + threads - 1) / threads), 2);
	slab_gradient_edges_kernel<<<blocks, threads, 0, s->stream>>>(s->dens, s->grad + 2 * (size_t)s->V * s->S,
																  has_below ? plane_below : nullptr,
																  has_above ? plane_above : nullptr, plane,
																  s->grid[2], cz);
	return check_launch(s, "slab_gradient_edges_kernel");
}

} // extern "C"
