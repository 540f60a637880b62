// Central-difference gradients of the field (paraBioFVM src/solver/host/gradient_solver.cpp:10-291).
//
// g = (u[i+1] - u[i-1]) * (1/(2h)) inside, (u[1] - u[0]) * (1/h) and (u[n-1] - u[n-2]) * (1/h) at
// the ends, with both factors rounded to float as in the reference (:17-18).  A 3D grid walks the
// field: blockIdx.y = y, blockIdx.z = z, and threads run along the contiguous x*s row, so every load
// and store of a warp is coalesced and no per-element 64-bit division is needed; the x and y
// neighbours hit L1/L2 and each plane is read from DRAM about once.  Output layouts (src/traits.h):
// 1D [x][s][1], 2D [y][x][s][2], 3D [3][z][y][x][s].  An axis of length 1 has gradient 0.

#include "bfvm_internal.h"

namespace bfvm {

__device__ __forceinline__ float axis_grad(const float* __restrict__ u, long long i, int pos, int n, long long stride,
										   float border, float center)
{
	if (n == 1)
		return 0.f;
	if (pos == 0)
		return __fmul_rn(__fsub_rn(__ldg(&u[i + stride]), __ldg(&u[i])), border);
	if (pos == n - 1)
		return __fmul_rn(__fsub_rn(__ldg(&u[i]), __ldg(&u[i - stride])), border);
	return __fmul_rn(__fsub_rn(__ldg(&u[i + stride]), __ldg(&u[i - stride])), center);
}

template <int DIMS>
__global__ void __launch_bounds__(256) gradient_kernel(const float* __restrict__ u, float* __restrict__ g,
													   long long total, int S, int X, int Y, int Z, float bx, float cx,
													   float by, float cy, float bz, float cz)
{
	const int XS = X * S;
	const int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= XS)
		return;
	const int y = blockIdx.y, z = blockIdx.z;
	const long long i = ((long long)z * Y + y) * XS + q;
	const int x = q / S;
	const float gx = axis_grad(u, i, x, X, S, bx, cx);
	if (DIMS == 1)
	{
		g[i] = gx;
		return;
	}
	const float gy = axis_grad(u, i, y, Y, XS, by, cy);
	if (DIMS == 2)
	{
		reinterpret_cast<float2*>(g)[i] = make_float2(gx, gy);
		return;
	}
	const float gz = axis_grad(u, i, z, Z, (long long)XS * Y, bz, cz);
	g[i] = gx;
	g[total + i] = gy;
	g[2 * total + i] = gz;
}

// 3D gradients when S % 4 == 0: a thread owns a float4 of four consecutive substrates of one voxel
// column (x, y) and walks ZC planes of z, keeping u(z-1), u(z), u(z+1) in registers, so each
// element costs one streamed 16-byte load of u(z+1) plus the x and y neighbours (L1/L2 hits) and
// three 16-byte stores.  All four substrates share x, so the border logic is per thread.
static constexpr int GRAD_ZC = 32;

__device__ __forceinline__ float4 f4sub_mul(float4 a, float4 b, float f)
{
	return make_float4(__fmul_rn(__fsub_rn(a.x, b.x), f), __fmul_rn(__fsub_rn(a.y, b.y), f),
					   __fmul_rn(__fsub_rn(a.z, b.z), f), __fmul_rn(__fsub_rn(a.w, b.w), f));
}

__global__ void __launch_bounds__(256) gradient3d_vec4_kernel(const float4* __restrict__ u, float4* __restrict__ g,
															   long long total4, int S4, int X, int Y, int Z, float bx,
															   float cx, float by, float cy, float bz, float cz, int y0)
{
	const int XS4 = X * S4;
	const int q4 = blockIdx.x * blockDim.x + threadIdx.x;
	if (q4 >= XS4)
		return;
	const int y = y0 + blockIdx.y;
	const int z0 = blockIdx.z * GRAD_ZC;
	const int z1 = min(Z, z0 + GRAD_ZC);
	const int x = q4 / S4;
	const long long plane = (long long)Y * XS4;
	const long long row = (long long)y * XS4 + q4;

	// x neighbours: +-S4 float4s; y neighbours: +-XS4
	const int xo_hi = x == X - 1 ? 0 : S4, xo_lo = x == 0 ? 0 : S4;
	const float fx = (x == 0 || x == X - 1) ? bx : cx;
	const int yo_hi = y == Y - 1 ? 0 : XS4, yo_lo = y == 0 ? 0 : XS4;
	const float fy = (y == 0 || y == Y - 1) ? by : cy;

	float4 prev = z0 > 0 ? __ldg(&u[(long long)(z0 - 1) * plane + row]) : make_float4(0, 0, 0, 0);
	float4 cur = __ldg(&u[(long long)z0 * plane + row]);
	for (int z = z0; z < z1; z++)
	{
		const long long i = (long long)z * plane + row;
		const float4 next = z + 1 < Z ? __ldg(&u[i + plane]) : cur;
		float4 gx, gy, gz;
		if (X == 1)
			gx = make_float4(0, 0, 0, 0);
		else
			gx = f4sub_mul(__ldg(&u[i + xo_hi]), __ldg(&u[i - xo_lo]), fx);
		if (Y == 1)
			gy = make_float4(0, 0, 0, 0);
		else
			gy = f4sub_mul(__ldg(&u[i + yo_hi]), __ldg(&u[i - yo_lo]), fy);
		if (Z == 1)
			gz = make_float4(0, 0, 0, 0);
		else if (z == 0)
			gz = f4sub_mul(next, cur, bz);
		else if (z == Z - 1)
			gz = f4sub_mul(cur, prev, bz);
		else
			gz = f4sub_mul(next, prev, cz);
		__stcs(&g[i], gx);
		__stcs(&g[total4 + i], gy);
		__stcs(&g[2 * total4 + i], gz);
		prev = cur;
		cur = next;
	}
}

static void gradient_factors(const bfvm_solver* st, float (&f)[6])
{
	for (int d = 0; d < 6; d++)
		f[d] = 0.f;
	for (int d = 0; d < st->dims; d++)
	{
		f[2 * d] = 1.f / st->voxel[d];
		f[2 * d + 1] = 1.f / (st->voxel[d] * 2);
	}
}

bool gradient_rows_possible(const bfvm_solver* st) { return st->dims == 3 && st->S % 4 == 0; }

int launch_gradient_rows(bfvm_solver* st, int y0, int y1)
{
	if (!gradient_rows_possible(st) || y0 < 0 || y1 > st->grid[1] || y0 > y1)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "gradient rows outside the mesh or not a 3D mesh of 4k substrates");
	if (y0 == y1)
		return BFVM_OK;
	float f[6];
	gradient_factors(st, f);
	const int threads = 256;
	const int S = st->S, X = st->grid[0], Y = st->grid[1], Z = st->grid[2];
	const int XS4 = X * (S / 4);
	const dim3 blocks((unsigned)((XS4 + threads - 1) / threads), (unsigned)(y1 - y0), (unsigned)((Z + GRAD_ZC - 1) / GRAD_ZC));
	gradient3d_vec4_kernel<<<blocks, threads, 0, st->stream>>>(reinterpret_cast<const float4*>(st->dens),
															   reinterpret_cast<float4*>(st->grad), st->V * S / 4, S / 4,
															   X, Y, Z, f[0], f[1], f[2], f[3], f[4], f[5], y0);
	return check_launch(st, "gradient3d_vec4_kernel");
}

int launch_gradient(bfvm_solver* st)
{
	const long long total = st->V * st->S;
	float f[6];
	gradient_factors(st, f);
	const int threads = 256;
	const int S = st->S, X = st->grid[0], Y = st->grid[1], Z = st->grid[2];
	if (gradient_rows_possible(st))
		return launch_gradient_rows(st, 0, Y);
	const dim3 blocks((unsigned)((X * S + threads - 1) / threads), (unsigned)Y, (unsigned)Z);
	if (st->dims == 1)
		gradient_kernel<1><<<blocks, threads, 0, st->stream>>>(st->dens, st->grad, total, S, X, Y, Z, f[0], f[1], f[2],
															   f[3], f[4], f[5]);
	else if (st->dims == 2)
		gradient_kernel<2><<<blocks, threads, 0, st->stream>>>(st->dens, st->grad, total, S, X, Y, Z, f[0], f[1], f[2],
															   f[3], f[4], f[5]);
	else
		gradient_kernel<3><<<blocks, threads, 0, st->stream>>>(st->dens, st->grad, total, S, X, Y, Z, f[0], f[1], f[2],
															   f[3], f[4], f[5]);
	return check_launch(st, "gradient_kernel");
}

} // namespace bfvm
