// Internal state of a bfvm_solver and the launchers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bfvm.h"

namespace bfvm {

struct ensemble_plan;

// Launch shape of the staged sweep of one axis: warp groups per CTA and pipeline stages per group
// (0: the built-in choice).  Set by bfvm_autotune, or from its process-wide cache of shapes.
struct sweep_tuning
{
	int groups = 0;
	int stages = 0;
};

// ------------------------------------------------------------------------------------------------
// errors

void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define BFVM_CUDA(call)                                                                                                \
	do                                                                                                                 \
	{                                                                                                                  \
		cudaError_t e_ = (call);                                                                                       \
		if (e_ != cudaSuccess)                                                                                         \
			return ::bfvm::cuda_fail(e_, #call);                                                                       \
	} while (0)

// device-side error flag bits
enum device_error_bits : int
{
	DEVERR_AGENT_OUTSIDE = 1,
	DEVERR_TIMEOUT = 2, // a bounded wait on an asynchronous copy gave up
};

// ------------------------------------------------------------------------------------------------
// One sweep axis: the precomputed Thomas coefficients of src/solver/host/diffusion_solver.cpp:72-142
// (only b' is stored; e = c b' is recomputed) plus the whole-block carry products of the
// partitioned solve.
struct sweep_plan
{
	int n = 0;		   // line length
	int P = 1;		   // blocks per line
	int base_len = 0;  // blocks 0..extra-1 have base_len+1 elements, the rest base_len
	int extra = 0;
	int M = 32;		   // register block capacity (kernel template)
	float* bp = nullptr;	// [n][S] b'_i
	float* c = nullptr;		// [S] off-diagonal
	float* gq = nullptr;	// [P][S] forward carry product of each whole block
	float* Gp = nullptr;	// [P][S] backward carry product of each whole block
	// front-padded partition of the staged sweeps (precompute_padded): vP blocks of exactly 32
	int vP = 1;
	int pad = 0;
	float* vtab = nullptr; // padded_table_floats(vP, S) floats
	// lines longer than the staged sweep takes, cut into chunks that it takes (chunks.cu): chunk k
	// holds elements [bounds[k], bounds[k + 1]) of every line; count 0 when the axis is not chunked
	struct chunks_t
	{
		int count = 0;
		std::vector<int> bounds;
		std::vector<float*> vtab; // per chunk, the tables of precompute_padded_range
		std::vector<int> vP, pad;
		// the carries pass (slab_reduce_weights): per chunk, A over elements [a_first, a_first + na)
		// and B over [bounds[k], bounds[k] + nb), with weights at rw + w_off[k] ([na][S], then [nb][S])
		std::vector<int> a_first, na, nb;
		std::vector<long long> w_off;
		float* rw = nullptr;
		float* coef = nullptr;	// [count][3][S] (slab_coefficients)
		float* carry = nullptr; // [count][2][lines]: each chunk's carries C, X of every line
		float* ex = nullptr;	// [count - 1][2][lines]: the end sums A, B at each chunk boundary
		long long lines = 0;
	} chunks;
};

// Radix-sort / scan scratch for the agent binning.
struct scan_plan
{
	std::vector<long long> level_sizes; // element count at each level
	std::vector<int*> level_sums;		// block sums per level (device)
};

// A Dirichlet overwrite list grouped by the tiles of one axis's staged sweep (dirichlet.cu): the
// runs of four and single elements of tile w are [qoff[w], qoff[w + 1]) and [soff[w], soff[w + 1]).
struct dirichlet_tiles
{
	long long items = 0; // tiles of the sweep; 0 when the axis has no grouped list
	int* qoff = nullptr;
	int* qidx = nullptr; // element indices (the lists exist for fields of fewer than 2^31 elements)
	float4* qval = nullptr;
	int* soff = nullptr;
	int* sidx = nullptr;
	float* sval = nullptr;
};

// A Dirichlet overwrite list (dirichlet.cu): aligned runs of four consecutive elements (one float4
// store each) and single elements, by element index.
struct overwrite_list
{
	long long* qidx = nullptr;
	float4* qval = nullptr;
	long long qcount = 0;
	long long* idx = nullptr;
	float* val = nullptr;
	long long count = 0;
};

struct agent_state
{
	int count = 0;
	int capacity = 0;
	float *sec = nullptr, *sat = nullptr, *upt = nullptr, *nex = nullptr, *intern = nullptr, *frac = nullptr;
	float *vol = nullptr, *pos = nullptr;

	// binning (rebuilt on recompute)
	unsigned int *keys = nullptr, *keys_alt = nullptr;
	int *vals = nullptr, *vals_alt = nullptr;
	int* hist = nullptr;		 // [256][tiles]
	int* flags = nullptr;		 // [A]
	int* seg_id = nullptr;		 // [A]
	int* seg_start = nullptr;	 // [A+1]
	int* seg_count_dev = nullptr; // [2]: number of segments, number of valid agents
	float *num = nullptr, *den = nullptr, *fac = nullptr;			 // [A][S]
	float *red_num = nullptr, *red_den = nullptr, *red_fac = nullptr; // [A][S] by segment
	int tiles = 0;
	scan_plan hist_scan, flag_scan;
	bool binned = false;		 // a recompute has run since the last store

	// A solver stepping alone with internalized substrates keeps its per-agent terms in the
	// binning's sorted order (cell.cu): row p of snum/sden/sfac/sintern is row vals[p] of
	// num/den/fac/intern, and rank[i] is agent i's row there, so the per-step update reads and
	// writes contiguous rows.  While `sorted` is set, sintern holds the internalized amounts and
	// intern is only a copy, refreshed when they are loaded.
	float *snum = nullptr, *sden = nullptr, *sfac = nullptr, *sintern = nullptr; // [A][S] sorted
	int* rank = nullptr;																// [A]
	bool sorted = false;

	int* move_idx = nullptr; // [2][moves]: destinations, then sources of bfvm_remove_agents
	int move_capacity = 0;
};

} // namespace bfvm

struct bfvm_solver
{
	int device = 0;
	cudaStream_t stream = nullptr;
	cudaStream_t own_stream = nullptr;

	int dims = 3;
	int bbox_min[3] = { 0, 0, 0 }, bbox_max[3] = { 0, 0, 0 }, voxel[3] = { 1, 1, 1 }, grid[3] = { 1, 1, 1 };
	int S = 1;
	float dt = 0;
	std::vector<float> D, decay;
	bool internalized = false;
	long long V = 0;

	float* dens = nullptr;
	float* grad = nullptr;

	bfvm::sweep_plan plan[3];

	// Dirichlet conditions as set (host), and the resolved overwrite list on the device: every
	// conditioned element once, with the value the reference's order leaves there
	std::vector<float> face_vals_h;			 // [6][S]
	std::vector<unsigned char> face_conds_h; // [6][S]
	int face_mask = 0;
	std::vector<long long> int_vids_h;		// interior voxels, ascending linear index
	std::vector<float> int_vals_h;			// [voxel][S]
	std::vector<unsigned char> int_conds_h; // [voxel][S]
	// ... as aligned runs of four consecutive elements (one float4 store each) and single elements
	long long* dir_qidx = nullptr; // first element index of each run, a multiple of 4
	float4* dir_qval = nullptr;
	long long dir_qcount = 0;
	long long* dir_idx = nullptr; // element index vid * S + s
	float* dir_val = nullptr;
	long long dir_count = 0;
	// the same list grouped by the tiles of each axis's staged sweep, which applies a tile's entries
	// right after storing the tile (the overwrite that follows the sweep in the LOD step)
	bfvm::dirichlet_tiles dir_tiles[3];
	// The face conditions by position: when no interior Dirichlet voxel lies on a conditioned face,
	// the staged sweeps of the LOD step write the face conditions themselves (the x sweep also right
	// after its loads, for the overwrite before it) and the scatter takes the interior elements alone
	bool face_pos_ok = false;
	bool face_dirichlet = false;		  // option face_dirichlet (measured no faster than the scatter)
	int* face_bits = nullptr;			  // [S]: bit f set when face f conditions the substrate
	float* face_vals_d = nullptr;		  // [6][S]
	unsigned char* face_tiles[3] = {};	  // per staged tile of each axis: a line lies on a face of another axis
	bfvm::overwrite_list dir_interior;	  // the interior elements of the list

	bfvm::agent_state ag;

	// bulk supply/uptake: prepared terms, [bulk_rows][S] (bulk_rows 1: one row for every voxel)
	float* bulk_add = nullptr;
	float* bulk_den = nullptr;
	long long bulk_rows = 0;

	int* dev_error = nullptr; // device error flags
	int* host_error = nullptr; // pinned mirror

	long long launches = 0;
	bool use_tma = true;		 // stage sweeps through shared memory with the TMA where the shape allows
	bool tma_prefetch = false;	 // staged sweeps also prefetch into L2 the tile after the one they copy
	// staged sweeps whose two warp groups share 64-column stages (sweep_tma.cu): 0 none, 1 the z
	// sweep (measured 2-3 % faster), 2 the y and z sweeps (the y sweep measured 2 % slower)
	int tma_pairs = 1;
	// measured slower than the scatter kernel and the gradient kernel at 320^3 x 16 (the extra work
	// in every tile of a latency-bound sweep costs more than the launches it saves), so off unless
	// asked for with bfvm_set_option
	bool dir_fused = false;		 // staged sweeps of the LOD step write the overwrite that follows them
	bool grad_fused = false;	 // the z sweep of a step computes the gradient (sweep_tma.cu)
	bool grad_evict_first = true; // ... reading its tiles with an L2 evict-first policy
	// the LOD step in bands that stay in L2 between two kernels (0: whole-field launches): the x and
	// y sweeps band by band of `xy_band_planes` z planes, the z sweep and the gradient band by band
	// of `zg_band_rows` y rows (sweep.cu)
	int xy_band_planes = 0;
	// the longest chunk of a line that the staged sweep takes as a chunk (chunks.cu): lines longer
	// than this are cut into chunks; 0: automatic (lines beyond 512 elements, x chunks of at most 320)
	int chunk_elements = 0;
	int zg_band_rows = 0;
	int* grad_tile_done = nullptr; // [z tiles] and [1 + z tiles] of the gradient inside the z sweep
	int* grad_deferred = nullptr;
	long long grad_tiles = 0;
	long long wait_limit_cycles = 4000000000LL; // bound of the staged sweeps' waits on tile copies (clock64 cycles;
												// the default is the kernels' WAIT_LIMIT_CYCLES)
	long long drop_tile_copy = -1;				// tests only: a staged-sweep tile whose copies are never issued
	bfvm::sweep_tuning tune[3];	 // staged sweep launch shape per axis

	// graphs for run_steps: [2 * recompute + agent terms sorted before the step]
	cudaGraphExec_t step_graph[4] = { nullptr, nullptr, nullptr, nullptr };
	long long graph_kernels[4] = { 0, 0, 0, 0 }; // kernel nodes per step graph
	bool graph_sorted_after[4] = { false, false, false, false }; // agent terms sorted after the step
	int batch_refs = 0; // batches holding this solver (its own step graphs leave the gradient unfused then)
	bool graphs_dirty = true;
	long long graph_epoch = 0; // advances whenever captured buffers or launch shapes may have changed

	// this mesh alone as an ensemble: its sweeps run the ensemble sweep kernel on shapes the TMA
	// path does not take (built at creation, so never inside a stream capture)
	bfvm::ensemble_plan* self_plan = nullptr;

	// z-slab of a larger mesh (bfvm_create_slab): planes [slab_z0, slab_z0 + grid[2]) of a mesh of
	// slab_global_z planes, slab slab_index of slab_count.  Its z tables are the whole line's,
	// restricted to the slab (precompute_padded_range), and its z sweep runs as two passes around
	// an exchange of 2 floats per z line with the other slabs.
	int slab_count = 1;
	int slab_index = 0;
	int slab_z0 = 0;
	int slab_global_z = 0;
	float* slab_coef = nullptr;	 // device [slab_count][3][S]: Gamma, beta, Lambda of slab_coefficients
	float* slab_carry = nullptr; // device [2][X*Y*S]: this slab's left and right carries of the step
	// the reduce pass's weights (slab_reduce_weights): A over local planes [slab_a0, slab_a0 +
	// slab_na), B over local planes [0, slab_nb); device [slab_na + slab_nb][S]
	float* slab_rw = nullptr;
	int slab_a0 = 0, slab_na = 0, slab_nb = 0;
	int slab_phase = 0;			 // 1 between bfvm_slab_diffusion_begin and _end

	// asynchronous agent copies (bfvm_store_agent_positions_async, bfvm_load_internalized_async) run
	// on copy_stream, each ordered after the work queued on `stream` when it was called; the next
	// call that touches agent data makes `stream` wait for them (order_after_copies)
	cudaStream_t copy_stream = nullptr;
	cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
	bool copy_pending = false;
};

namespace bfvm {

// precompute.cpp
void precompute_axis(int n, int h, int dims, int S, float dt, const float* D, const float* decay, int M,
					 std::vector<float>& bp, std::vector<float>& eprev, std::vector<float>& g, std::vector<float>& G,
					 std::vector<float>& c, std::vector<float>& gq, std::vector<float>& Gp, int& P, int& base_len,
					 int& extra);
int padded_table_floats(int P, int S);
void precompute_padded(int n, int S, const std::vector<float>& bp, const std::vector<float>& c, int& P, int& pad,
					   std::vector<float>& tab);
// the tables of elements [i0, i1) of a line of n, with the responses to carries across i0 and i1
void precompute_padded_range(int n, int i0, int i1, int S, const std::vector<float>& bp, const std::vector<float>& c,
							 int& P, int& pad, std::vector<float>& tab);
void slab_coefficients(int n, int S, const std::vector<float>& bp, const std::vector<float>& c, int count,
					   const int* bounds, std::vector<float>& out);
// the weights of A and B of the slab holding elements [i0, i1), over the planes that matter
void slab_reduce_weights(int n, int i0, int i1, int S, const std::vector<float>& bp, const std::vector<float>& c,
						 std::vector<float>& w, int& a_first, int& na, int& nb, int drop_log2 = -50);

// bfvm_api.cu
int one_step(bfvm_solver* s, bool recompute); // diffusion, gradient, secretion on the solver's stream
int order_after_copies(bfvm_solver* s);		  // the solver's stream waits for pending asynchronous copies
int check_device_errors(bfvm_solver* s);	  // waits for the stream, reports device-side error flags

// sweep.cu
int launch_sweep(bfvm_solver* s, int axis, bool final_dirichlet);
// the LOD step, overwrites fused into the staged sweeps; with `gradient`, the z sweep also
// computes the gradient where it can, and *gradient_done tells whether it did
int launch_diffusion(bfvm_solver* s, bool gradient = false, bool* gradient_done = nullptr);
int grad_fuse_buffers(bfvm_solver* s); // buffers of the gradient inside the z sweep (outside a capture)
// the staged sweep of one axis alone, with launch shape `tune` (groups 0: built-in choice);
// `handled` is false when the staged path does not take the shape
int launch_staged_sweep(bfvm_solver* s, int axis, const sweep_tuning& tune, bool& handled);
// launch shapes the staged sweep of `axis` can take on this mesh (empty if none)
std::vector<sweep_tuning> staged_sweep_shapes(bfvm_solver* s, int axis);
// autotune.cu: a tuned launch shape of an equal mesh, from the process-wide cache
bool cached_tuning(const bfvm_solver* s, int axis, sweep_tuning& out);
// chunks.cu: the chunk plan of an axis whose lines the staged sweep cannot take whole (from the
// line's b' and c), its release, and the chunked sweep (`handled` false when it cannot run)
int build_chunks(bfvm_solver* s, int axis, const std::vector<float>& bp, const std::vector<float>& c);
int rebuild_chunks(bfvm_solver* s); // every axis, after the chunk length changed (outside any capture)
void free_chunks(sweep_plan& p);
int launch_chunked_sweep(bfvm_solver* s, int axis, bool& handled);
// the solve pass of a slab solver's z sweep, with the carries in s->slab_carry
int launch_slab_z(bfvm_solver* s);
// dirichlet.cu
int launch_dirichlet(bfvm_solver* s, bool interior_only = false);
// the step's staged sweep of `axis` can write the face conditions (face_pos_ok and the option)
bool faces_by_position(const bfvm_solver* s);
int rebuild_dirichlet(bfvm_solver* s);
void free_dirichlet(bfvm_solver* s);

// gradient.cu
int launch_gradient(bfvm_solver* s);
// the 3D gradient of rows [y0, y1) of every plane, when substrates % 4 == 0 (false: not this shape)
bool gradient_rows_possible(const bfvm_solver* s);
int launch_gradient_rows(bfvm_solver* s, int y0, int y1);

// bulk.cu
int set_bulk_rates(bfvm_solver* s, int per_voxel, const float* supply, const float* uptake, const float* target);
int launch_bulk(bfvm_solver* s);
void free_bulk(bfvm_solver* s);

// cell.cu
int cell_alloc(bfvm_solver* s, int count);
void cell_free(bfvm_solver* s);
int launch_secretion(bfvm_solver* s, bool recompute);
// the binning and the agent terms' order a secretion update needs (a rebinning when `recompute`)
int prepare_agent_terms(bfvm_solver* s, bool recompute);
int agents_unsort(bfvm_solver* s, bool keep_sorted); // internalized amounts back to agent order (cell.cu)
int solver_drop_graphs(bfvm_solver* s);			  // after queued work, drop the step graphs (bfvm_api.cu)
int agents_resort_internalized(bfvm_solver* s);	  // stored internalized amounts into sorted order
int launch_release(bfvm_solver* s, int index);
// storage for `count` agents keeping the stored rows; the moves dst[k] <- src[k] of every agent row
int cell_grow(bfvm_solver* s, int count);
int launch_agent_moves(bfvm_solver* s, const std::vector<int>& dst, const std::vector<int>& src);

// scan.cu
int scan_plan_build(scan_plan& p, long long n);
void scan_plan_free(scan_plan& p);
int launch_exclusive_scan(bfvm_solver* s, scan_plan& p, const int* in, int* out, long long n);

template <typename T>
int device_alloc(T** ptr, size_t count)
{
	*ptr = nullptr;
	if (count == 0)
		return BFVM_OK;
	cudaError_t e = cudaMalloc((void**)ptr, count * sizeof(T));
	if (e != cudaSuccess)
	{
		*ptr = nullptr;
		(void)cudaGetLastError();
		return fail(BFVM_ERR_OUT_OF_MEMORY, std::string("device allocation of ") + std::to_string(count * sizeof(T))
												+ " bytes failed: " + cudaGetErrorString(e));
	}
	return BFVM_OK;
}

template <typename T>
void device_free(T*& ptr)
{
	if (ptr)
		cudaFree((void*)ptr);
	ptr = nullptr;
}

inline int check_launch(bfvm_solver* s, const char* what)
{
	s->launches++;
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess)
		return cuda_fail(e, what);
	return BFVM_OK;
}

} // namespace bfvm
