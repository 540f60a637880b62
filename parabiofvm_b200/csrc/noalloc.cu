// bfvm_secretion_solve_noalloc: the secretion/uptake step with recompute for callers that cannot
// allocate GPU memory.  It runs the same kernels as bfvm_secretion_solve (agent keys, stable radix
// sort, voxel segments, intermediates, reductions, update) in the same order, so its results are
// the same bit for bit; the binning scratch lives in one static device array instead of buffers a
// solver allocates.

#include <mutex>

#include "agent_kernels.cuh"

namespace bfvm {

static constexpr long long NA_MAX_AGENTS = BFVM_NOALLOC_MAX_AGENTS;
static constexpr long long NA_MAX_AS = BFVM_NOALLOC_MAX_AGENT_SUBSTRATES;
static constexpr long long NA_SORT_TILES = (NA_MAX_AGENTS + SORT_TILE - 1) / SORT_TILE;
static constexpr long long NA_FLAG_TILES = (NA_MAX_AGENTS + SCAN_TILE - 1) / SCAN_TILE;
// the histogram scan fits one scan tile, and the flag scan needs one level of tile sums
static_assert(256 * NA_SORT_TILES <= SCAN_TILE, "histogram scan must fit one scan tile");
static_assert(NA_FLAG_TILES <= SCAN_TILE, "flag scan tile sums must fit one scan tile");

static constexpr size_t na_align(size_t b) { return (b + 255) / 256 * 256; }

// byte offsets of the pieces of the scratch array
static constexpr size_t NA_COUNTS = 0;											  // int [4]
static constexpr size_t NA_FLAGWORD = NA_COUNTS + na_align(4 * sizeof(int));		  // int, when no error_flags
static constexpr size_t NA_KEYS = NA_FLAGWORD + na_align(sizeof(int));			  // uint [A]
static constexpr size_t NA_KEYS_ALT = NA_KEYS + na_align(NA_MAX_AGENTS * 4);		  // uint [A]
static constexpr size_t NA_VALS = NA_KEYS_ALT + na_align(NA_MAX_AGENTS * 4);		  // int [A]
static constexpr size_t NA_VALS_ALT = NA_VALS + na_align(NA_MAX_AGENTS * 4);		  // int [A]
static constexpr size_t NA_FLAGS = NA_VALS_ALT + na_align(NA_MAX_AGENTS * 4);		  // int [A]
static constexpr size_t NA_SEG_ID = NA_FLAGS + na_align(NA_MAX_AGENTS * 4);		  // int [A]
static constexpr size_t NA_SEG_START = NA_SEG_ID + na_align(NA_MAX_AGENTS * 4);	  // int [A+1]
static constexpr size_t NA_HIST = NA_SEG_START + na_align((NA_MAX_AGENTS + 1) * 4); // int [256][tiles]
static constexpr size_t NA_SUMS = NA_HIST + na_align(256 * NA_SORT_TILES * 4);	  // int [flag tiles]
static constexpr size_t NA_F0 = NA_SUMS + na_align(NA_FLAG_TILES * 4);			  // 6 x float [A*S]
static constexpr size_t NA_FSTRIDE = na_align(NA_MAX_AS * 4);
static constexpr size_t NA_TOTAL = NA_F0 + 6 * NA_FSTRIDE;
static_assert(NA_TOTAL == BFVM_NOALLOC_SCRATCH_BYTES, "BFVM_NOALLOC_SCRATCH_BYTES in bfvm.h is out of date");

static __device__ __align__(256) unsigned char noalloc_scratch[NA_TOTAL];

// Device address of noalloc_scratch on the current device.  In host code the name noalloc_scratch
// is a host-side stand-in, not a device address.  Outside stream capture the address is looked up
// on every call (cheap), so a device reset or a re-created primary context, which may move the
// array, never leaves a stale address behind; the last address found on each device is kept for
// calls made while `stream` is capturing, where the lookup (which may load the module) is not
// allowed.  So the first call on a device must come before any capture.
static int scratch_address(cudaStream_t stream, unsigned char** out)
{
	static std::mutex lock;
	static void* addr[64] = {};
	int dev = 0;
	BFVM_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 64)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "device index beyond 63");
	cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess)
	{
		(void)cudaGetLastError();
		capture = cudaStreamCaptureStatusActive; // cannot tell: do not risk a lookup during a capture
	}
	std::lock_guard<std::mutex> guard(lock);
	if (capture == cudaStreamCaptureStatusNone)
	{
		void* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
		if (e != cudaSuccess)
			return cuda_fail(e, "cudaGetSymbolAddress(noalloc_scratch)");
		addr[dev] = p;
	}
	else if (!addr[dev])
		return fail(BFVM_ERR_STATE, "the first bfvm_secretion_solve_noalloc call on a device must come before any "
									"stream capture");
	*out = static_cast<unsigned char*>(addr[dev]);
	return BFVM_OK;
}

static int launched(const char* what)
{
	cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? BFVM_OK : cuda_fail(e, what);
}

} // namespace bfvm

using namespace bfvm;

extern "C" int bfvm_secretion_solve_noalloc(float* densities, int dims, const int32_t bounding_box_mins[3],
											const int32_t voxel_shape[3], const int32_t grid_shape[3],
											int32_t substrates, float time_step, int32_t agent_count,
											const float* secretion_rates, const float* saturation_densities,
											const float* uptake_rates, const float* net_export_rates,
											float* internalized_substrates, const float* volumes,
											const float* positions, int32_t* error_flags, void* stream_handle)
{
	if (!densities || !bounding_box_mins || !voxel_shape || !grid_shape)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "densities, bounding_box_mins, voxel_shape and grid_shape are required");
	if (dims < 1 || dims > 3)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "dims must be 1, 2 or 3");
	if (substrates < 1)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "at least one substrate is required");
	if (agent_count < 0)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent_count must not be negative");
	if (agent_count > NA_MAX_AGENTS)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent_count " + std::to_string(agent_count) + " exceeds the limit of "
												   + std::to_string(NA_MAX_AGENTS) + " agents");
	if ((long long)agent_count * substrates > NA_MAX_AS)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "agent_count x substrates " + std::to_string((long long)agent_count * substrates)
												   + " exceeds the limit of " + std::to_string(NA_MAX_AS));
	int grid[3] = { 1, 1, 1 };
	long long V = 1;
	for (int d = 0; d < dims; d++)
	{
		if (grid_shape[d] < 1 || voxel_shape[d] < 1)
			return fail(BFVM_ERR_INVALID_ARGUMENT, "grid_shape and voxel_shape must be positive along every used axis");
		grid[d] = grid_shape[d];
		V *= grid[d];
	}
	if (V >= 0xffffffffLL)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "mesh too large for 32-bit voxel keys");
	if (agent_count == 0)
		return BFVM_OK;
	if (!secretion_rates || !saturation_densities || !uptake_rates || !net_export_rates || !volumes || !positions)
		return fail(BFVM_ERR_INVALID_ARGUMENT, "the agent arrays are required");

	cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
	unsigned char* base = nullptr;
	int st = scratch_address(stream, &base);
	if (st)
		return st;
	int* counts = reinterpret_cast<int*>(base + NA_COUNTS);
	int* err = error_flags ? error_flags : reinterpret_cast<int*>(base + NA_FLAGWORD);
	unsigned int* keys = reinterpret_cast<unsigned int*>(base + NA_KEYS);
	unsigned int* keys_alt = reinterpret_cast<unsigned int*>(base + NA_KEYS_ALT);
	int* vals = reinterpret_cast<int*>(base + NA_VALS);
	int* vals_alt = reinterpret_cast<int*>(base + NA_VALS_ALT);
	int* flags = reinterpret_cast<int*>(base + NA_FLAGS);
	int* seg_id = reinterpret_cast<int*>(base + NA_SEG_ID);
	int* seg_start = reinterpret_cast<int*>(base + NA_SEG_START);
	int* hist = reinterpret_cast<int*>(base + NA_HIST);
	int* sums = reinterpret_cast<int*>(base + NA_SUMS);
	float* num = reinterpret_cast<float*>(base + NA_F0);
	float* den = reinterpret_cast<float*>(base + NA_F0 + NA_FSTRIDE);
	float* fac = reinterpret_cast<float*>(base + NA_F0 + 2 * NA_FSTRIDE);
	float* red_num = reinterpret_cast<float*>(base + NA_F0 + 3 * NA_FSTRIDE);
	float* red_den = reinterpret_cast<float*>(base + NA_F0 + 4 * NA_FSTRIDE);
	float* red_fac = reinterpret_cast<float*>(base + NA_F0 + 5 * NA_FSTRIDE);

	const int A = agent_count;
	const int S = substrates;
	const int3 bmin = make_int3(bounding_box_mins[0], bounding_box_mins[1], bounding_box_mins[2]);
	const int3 vox = make_int3(voxel_shape[0], voxel_shape[1], voxel_shape[2]);
	const int3 gr = make_int3(grid[0], grid[1], grid[2]);
	const unsigned int invalid = (unsigned int)V;
	const float voxel_volume = (float)(voxel_shape[0] * voxel_shape[1] * voxel_shape[2]);

	// the array keeps the previous call's contents: the segment counters must start at zero
	BFVM_CUDA(cudaMemsetAsync(counts, 0, 4 * sizeof(int), stream));
	agent_keys_kernel<<<(A + 255) / 256, 256, 0, stream>>>(positions, A, dims, bmin, vox, gr, keys, vals, invalid, err);
	if ((st = launched("agent_keys_kernel")))
		return st;

	// stable LSD radix sort of (key, agent index)
	unsigned int* kin = keys;
	unsigned int* kout = keys_alt;
	int* vin = vals;
	int* vout = vals_alt;
	const int tiles = (A + SORT_TILE - 1) / SORT_TILE;
	for (int pass = 0; pass < sort_passes(V); pass++)
	{
		radix_hist_kernel<<<tiles, SORT_THREADS, 0, stream>>>(kin, A, 8 * pass, hist, tiles);
		if ((st = launched("radix_hist_kernel")))
			return st;
		scan_tile_kernel<<<1, SCAN_THREADS, 0, stream>>>(hist, hist, 256LL * tiles, nullptr);
		if ((st = launched("scan_tile_kernel")))
			return st;
		radix_scatter_kernel<<<tiles, SORT_THREADS, 0, stream>>>(kin, vin, kout, vout, A, 8 * pass, hist, tiles);
		if ((st = launched("radix_scatter_kernel")))
			return st;
		std::swap(kin, kout);
		std::swap(vin, vout);
	}

	// voxel segments of the sorted keys
	seg_flags_kernel<<<(A + 255) / 256, 256, 0, stream>>>(kin, A, invalid, flags);
	if ((st = launched("seg_flags_kernel")))
		return st;
	const long long ftiles = (A + SCAN_TILE - 1) / SCAN_TILE;
	scan_tile_kernel<<<(unsigned)ftiles, SCAN_THREADS, 0, stream>>>(flags, seg_id, A, ftiles > 1 ? sums : nullptr);
	if ((st = launched("scan_tile_kernel")))
		return st;
	if (ftiles > 1)
	{
		scan_tile_kernel<<<1, SCAN_THREADS, 0, stream>>>(sums, sums, ftiles, nullptr);
		if ((st = launched("scan_tile_kernel")))
			return st;
		scan_add_kernel<<<(unsigned)ftiles, 256, 0, stream>>>(seg_id, A, sums);
		if ((st = launched("scan_add_kernel")))
			return st;
	}
	seg_finish_kernel<<<(A + 255) / 256, 256, 0, stream>>>(kin, flags, seg_id, A, invalid, seg_start, counts);
	if ((st = launched("seg_finish_kernel")))
		return st;

	// intermediates, per-voxel reductions and the update
	const long long AS = (long long)A * S;
	const unsigned blocks = (unsigned)((AS + 255) / 256);
	intermediates_kernel<<<blocks, 256, 0, stream>>>(AS, S, secretion_rates, saturation_densities, uptake_rates,
													 net_export_rates, volumes, voxel_volume, time_step, num, den, fac);
	if ((st = launched("intermediates_kernel")))
		return st;
	reduce_kernel<<<blocks, 256, 0, stream>>>(AS, S, counts, seg_start, vin, num, den, fac, red_num, red_den, red_fac);
	if ((st = launched("reduce_kernel")))
		return st;
	secrete_kernel<<<blocks, 256, 0, stream>>>(AS, S, densities, counts, seg_start, vin, kin, num, den, fac, red_num,
											   red_den, red_fac, internalized_substrates,
											   internalized_substrates ? 1 : 0, voxel_volume);
	return launched("secrete_kernel");
}
