// The learned surrogate: shapes, the convolution launch parameters and the launchers of
// surrogate.cu, used by the network in surrogate_net.cu.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace bfvm {

constexpr int SUR_C = 32;	  // channels of every activation tensor
constexpr int SUR_TILE = 128; // voxels of a tile along x (the MMA's M)
constexpr int SUR_TAPS = 27;  // 3 x 3 x 3 stencil
constexpr int SUR_LAYERS = 10; // lift, 4 residual blocks of 2 convolutions, projection
constexpr int SUR_LAYER_PARAMS = SUR_TAPS * SUR_C * SUR_C + SUR_C; // W[27][co][ci] then b[co]

struct conv_params
{
	int X, Y, Z, B;
	int x_tiles;	// set by the launcher
	long long tiles; // set by the launcher
	const float* bias;				// [32] added first, or null
	const __nv_bfloat16* residual;	// [voxels][32] added next, or null
	int relu;						// then max(v, 0)
	const __nv_bfloat16* mask;		// [voxels][32]: then v where mask > 0 else 0, or null
	__nv_bfloat16* out;				// [voxels][32], or null
	float* out_f32;					// [voxels][out_ch] = v[:out_ch] (+ base_f32), or null
	const float* base_f32;			// [voxels][out_ch] or null
	int out_ch;
	int* err; // device error flags
};

int sur_check_shape(int X, int Y, int Z, int B);
// out = epilogue(conv(in, w)), w bf16 [27][co][ci]
int launch_sur_conv(const __nv_bfloat16* in, const __nv_bfloat16* w, conv_params p, int device, cudaStream_t stream);
// dW[27][co][ci] += sum over voxels of grad[v][co] in[v + off_t][ci] (p: shape and err only)
int launch_sur_wgrad(const __nv_bfloat16* in, const __nv_bfloat16* grad, float* dW, conv_params p, int device,
					 cudaStream_t stream);

} // namespace bfvm
