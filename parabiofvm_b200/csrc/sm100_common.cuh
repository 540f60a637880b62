// Shared-memory barriers and Tensor Memory Accelerator copies for the sm_100a kernels (the staged
// sweeps of sweep_tma.cu and the surrogate's convolutions of surrogate.cu).
//
// Every wait is bounded by WAIT_LIMIT_CYCLES of clock64 (about two seconds): a caller that gives
// up raises a device error flag and returns instead of spinning forever.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace bfvm {

static constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL; // about two seconds

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
				 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
				 "selp.u32 %0, 1, 0, p;\n}"
				 : "=r"(ok)
				 : "r"(smem_addr(bar)), "r"(parity)
				 : "memory");
	return ok != 0;
}

// Wait for the phase of `bar` with the given parity for at most `limit` cycles of clock64; false
// when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = WAIT_LIMIT_CYCLES)
{
	const long long t0 = clock64();
	while (!mbar_try_wait(bar, parity))
		if (clock64() - t0 > limit)
			return false;
	return true;
}

__device__ __forceinline__ void tma_load_2d(float* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
				 ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_addr(bar))
				 : "memory");
}

// An L2 policy that marks lines as the first to evict (for data read once).
__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
	uint64_t p;
	asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
	return p;
}

__device__ __forceinline__ void tma_load_2d_hint(float* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar,
												 uint64_t policy)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, "
				 "{%2, %3}], [%4], %5;" ::"r"(smem_addr(dst)),
				 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_addr(bar)), "l"(policy)
				 : "memory");
}

// Prefetches into L2 of a tensor-map box, or of a contiguous range (no shared memory, no barrier).
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int c0, int c1)
{
	asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(reinterpret_cast<uint64_t>(map)),
				 "r"(c0), "r"(c1)
				 : "memory");
}

__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int c0, int c1, int c2)
{
	asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
					 reinterpret_cast<uint64_t>(map)),
				 "r"(c0), "r"(c1), "r"(c2)
				 : "memory");
}

__device__ __forceinline__ void bulk_prefetch(const void* src, uint32_t bytes)
{
	asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar)
{
	asm volatile(
		"cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
		::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
		: "memory");
}

__device__ __forceinline__ void bulk_load(float* dst, const float* src, uint32_t bytes, uint64_t* bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
				 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
				 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar)
{
	tma_load_2d(static_cast<float*>(dst), map, c0, c1, bar);
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
											uint64_t* bar)
{
	asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
				 "%5, %6}], [%7];" ::"r"(smem_addr(dst)),
				 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
				 : "memory");
}

} // namespace bfvm

// cuTensorMapEncodeTiled from the driver (sweep_tma.cu); null when the driver does not offer it
#include <cudaTypedefs.h>
namespace bfvm {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();
} // namespace bfvm
