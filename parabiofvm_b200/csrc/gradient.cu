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

int launch_gradient(bfvm_solver* st)
{
	const long long total = st->V * st->S;
	float f[6] = { 0, 0, 0, 0, 0, 0 };
	for (int d = 0; d < st->dims; d++)
	{
		f[2 * d] = 1.f / st->voxel[d];
		f[2 * d + 1] = 1.f / (st->voxel[d] * 2);
	}
	const int threads = 256;
	const int S = st->S, X = st->grid[0], Y = st->grid[1], Z = st->grid[2];
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
