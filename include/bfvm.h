/*
 * bfvm.h -- C ABI of the B200 microenvironment solver (libbfvm_cuda.so).
 *
 * One bfvm_solver holds one microenvironment on one GPU: the substrate field, its gradients, the
 * Dirichlet conditions, the agents' secretion/uptake data and the precomputed solver state.  The
 * entry points mirror the device solver of paraBioFVM (paths relative to that project's root):
 *
 *   solver::initialize / store_data_to_solver / load_data_from_solver / wait_for_all
 *                                        src/solver/device/CUDA/solver.cpp:7-23
 *   diffusion_solver::solve              src/solver/host/diffusion_solver.cpp:60-70, 512-544
 *   dirichlet_solver::solve              src/solver/host/dirichlet_solver.cpp:143-151
 *   gradient_solver::solve               src/solver/host/gradient_solver.cpp:275-291
 *   cell_solver::simulate_secretion_and_uptake / release_internalized_substrates
 *                                        src/solver/host/cell_solver.cpp:272-346
 *
 * Memory layouts are the reference's (src/traits.h:9-93): densities [z][y][x][s] with the
 * substrate index fastest; gradients [x][s][1] (1D), [y][x][s][2] (2D), [3][z][y][x][s] (3D);
 * agent arrays [agent][substrate], volumes [agent], positions [agent][dims].  All values are
 * 32-bit floats (the reference's default real_t), indices 32-bit ints.
 *
 * Calls are ordered on the solver's CUDA stream and return before the GPU finishes unless they
 * say otherwise; a solver is not safe to use from two host threads at once.  Every function
 * returns a bfvm_status; on failure bfvm_last_error() describes the problem.  Nothing aborts the
 * process.
 */
#ifndef BFVM_H
#define BFVM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bfvm_solver bfvm_solver;

typedef enum bfvm_status
{
	BFVM_OK = 0,
	BFVM_ERR_INVALID_ARGUMENT = 1, /* bad size, index, pointer or mesh */
	BFVM_ERR_OUT_OF_MEMORY = 2,    /* device or pinned host allocation failed */
	BFVM_ERR_CUDA = 3,             /* a CUDA runtime call failed */
	BFVM_ERR_NO_DEVICE = 4,        /* no usable CUDA device / library built for another arch */
	BFVM_ERR_STATE = 5,            /* call out of order (e.g. agents not stored) */
	BFVM_ERR_AGENT_OUTSIDE = 6,    /* an agent position maps outside the mesh */
	BFVM_ERR_TIMEOUT = 7           /* a kernel's bounded wait on an asynchronous copy gave up */
} bfvm_status;

/* Message for the last failing call on this host thread ("" if none). */
const char* bfvm_last_error(void);
const char* bfvm_status_string(int status);
/* Library version as major*10000 + minor*100 + patch. */
int bfvm_version(void);

/*
 * Create a solver on CUDA device `device` (replaces microenvironment_builder::build + solver::
 * initialize, src/microenvironment_builder.cpp:146-193, src/solver/device/CUDA/solver.cpp:7-13).
 * The mesh follows cartesian_mesh (src/mesh.cpp:7-30): grid_shape[d] = ceil((max-min)/voxel).
 * diffusion_coefficients and decay_rates hold `substrates` values.  The field starts at zero.
 */
int bfvm_create(bfvm_solver** out, int device, int dims, const int32_t bounding_box_mins[3],
				const int32_t bounding_box_maxs[3], const int32_t voxel_shape[3], int32_t substrates,
				float time_step, const float* diffusion_coefficients, const float* decay_rates,
				int compute_internalized_substrates);
int bfvm_destroy(bfvm_solver* s);

/* grid_shape[3] as computed from the mesh; voxel count; substrate count; dims. */
int bfvm_get_shape(const bfvm_solver* s, int32_t grid_shape[3], int64_t* voxel_count, int32_t* substrates,
				   int32_t* dims);

/* Run the solver's work on `stream` (a cudaStream_t; NULL = the solver's own stream). */
int bfvm_set_stream(bfvm_solver* s, void* stream);

/*
 * Boundary Dirichlet conditions of one face (microenvironment.h:47-50): `dim` 0..dims-1,
 * `is_max` 0 for the min face.  values/conditions hold `substrates` entries; values == NULL removes
 * the face.  Faces are applied x-min, x-max, y-min, y-max, z-min, z-max, later faces winning
 * (src/solver/host/dirichlet_solver.cpp:91-141).
 */
int bfvm_set_boundary_dirichlet(bfvm_solver* s, int dim, int is_max, const float* values, const uint8_t* conditions);

/*
 * Interior Dirichlet voxels (microenvironment.h:41-44): voxels [count][dims], values and
 * conditions [count][substrates].  Replaces any previous set; count == 0 clears.  Applied after
 * the faces; a voxel listed twice takes, per substrate, the last listed condition that is set.
 */
int bfvm_set_interior_dirichlet(bfvm_solver* s, int32_t count, const int32_t* voxels, const float* values,
								const uint8_t* conditions);

/* Host <-> device copies of the field (solver::store/load_data_to/from_solver). load_* wait for
 * the stream and check the device error flags before returning. */
int bfvm_store_densities(bfvm_solver* s, const float* host_densities);
int bfvm_load_densities(bfvm_solver* s, float* host_densities);
int bfvm_load_gradients(bfvm_solver* s, float* host_gradients);
/* The field from / to device memory of the solver's device, ordered on its stream (no wait): for
 * callers whose data already lives on the GPU. */
int bfvm_store_densities_device(bfvm_solver* s, const float* device_densities);
int bfvm_load_densities_device(bfvm_solver* s, float* device_densities);

/*
 * Replace the agent set (device_context::copy_to_device, src/solver/device/CUDA/device_context.cpp:
 * 56-97).  Arrays are [count][substrates] except volumes [count] and positions [count][dims].
 * fraction_released_at_death may be NULL (taken as zero).  A new agent count forces the next
 * secretion call to rebuild the voxel binning.
 */
int bfvm_store_agents(bfvm_solver* s, int32_t count, const float* secretion_rates, const float* saturation_densities,
					  const float* uptake_rates, const float* net_export_rates, const float* internalized_substrates,
					  const float* fraction_released_at_death, const float* volumes, const float* positions);
/*
 * Positions alone ([count][dims]) of the stored agents, count equal to the stored count: the
 * per-step input of a model whose agents move.  No counterpart in the reference, whose
 * store_data_to_solver copies every agent array (src/solver/device/CUDA/cell_solver.cpp:172-178).
 * As with bfvm_store_agents, new positions enter the voxel binning at the next recompute.
 */
int bfvm_store_agent_positions(bfvm_solver* s, int32_t count, const float* positions);
int bfvm_load_internalized(bfvm_solver* s, float* host_internalized);
/*
 * Asynchronous variants for step loops that move agent data every step (no counterpart in the
 * reference, whose loads are synchronous).  The copy runs on a copy stream of the solver, after the
 * work queued on the solver's stream when it is called, so it overlaps the work queued afterwards
 * (the next step's diffusion and gradient); the next call that uses agent data (secretion, release,
 * agent stores and loads, run_steps, batches) waits for it on the GPU.  The host buffer must stay
 * valid, and for an overlapping copy be pinned, until bfvm_synchronize returns.
 */
int bfvm_store_agent_positions_async(bfvm_solver* s, int32_t count, const float* positions);
int bfvm_load_internalized_async(bfvm_solver* s, float* host_internalized);

/* One LOD diffusion-decay step with the Dirichlet overwrites between sweeps
 * (diffusion_solver::solve). */
int bfvm_diffusion_solve(bfvm_solver* s);
/* One axis (0 = x, 1 = y, 2 = z) of the diffusion step: the Dirichlet overwrite, that axis's
 * Thomas sweep, and for the last axis the closing overwrite.  bfvm_diffusion_solve is these calls
 * for axes 0 .. dims-1 (diffusion_solver.cpp:512-544); one axis alone serves operator-split
 * orderings and per-kernel timing. */
int bfvm_diffusion_sweep(bfvm_solver* s, int axis);
/* Dirichlet overwrite alone (dirichlet_solver::solve). */
int bfvm_dirichlet_solve(bfvm_solver* s);
/* Central-difference gradients of the current field (gradient_solver::solve). */
int bfvm_gradient_solve(bfvm_solver* s);
/* bfvm_diffusion_solve followed by bfvm_gradient_solve (diffusion_solver::solve then
 * gradient_solver::solve, as src/main.cpp:76-90 calls them), with the gradient computed inside the
 * z sweep when the option "fused_gradient" is set and the staged sweep takes the mesh: each tile's
 * gradient is computed from the planes the sweep just wrote, while they are still in L2.  The
 * results are the same bits as the two calls. */
int bfvm_diffusion_gradient_solve(bfvm_solver* s);
/* Secretion and uptake (cell_solver::simulate_secretion_and_uptake); recompute != 0 rebuilds the
 * per-voxel reductions from the current agent data and positions. */
int bfvm_secretion_solve(bfvm_solver* s, int recompute);
/* cell_solver::release_internalized_substrates for agent `index`. */
int bfvm_release_internalized(bfvm_solver* s, int32_t index);
/*
 * Agents added and removed on the GPU, without moving the stored agents through the host (the
 * reference re-copies every agent array after any change, src/solver/device/CUDA/cell_solver.cpp:
 * 172-178).  The next secretion call rebuilds the voxel binning, as after bfvm_store_agents with a
 * new count.
 *
 * bfvm_add_agents: agent_data::add() (src/agent_data.cpp:10-25) `count` times, the new agents
 * taking indices [stored, stored + count) with the values of the host arrays given (shapes as in
 * bfvm_store_agents, `count` rows each).  A NULL array leaves that quantity 0 for the new agents,
 * as add() does.  Only the new rows cross the host link; grown storage is copied on the device.
 * If the storage cannot grow, the call returns BFVM_ERR_OUT_OF_MEMORY and the solver is left
 * without agents, as after a failed bfvm_store_agents.
 *
 * bfvm_remove_agents: agent_data::remove (src/agent_data.cpp:27-53) of indices[0], then
 * indices[1], ... in that order, each moving the then-last agent into the freed slot.  Every index
 * must lie below the agent count at its turn; otherwise nothing changes and the call returns
 * BFVM_ERR_INVALID_ARGUMENT.  Only the indices cross the host link.
 *
 * bfvm_plan_agent_removal: the host part of bfvm_remove_agents, without a solver or a device.  For
 * `agents` agents and the removals indices[0 .. count), it returns the agents left and the moves
 * that bring the stored rows into the order sequential agent_data::remove calls leave: row dst[k]
 * takes row src[k] for k < *moves (dst and src hold `count` entries; sources lie at or above
 * *remaining and destinations below it, so the moves are independent).
 */
int bfvm_add_agents(bfvm_solver* s, int32_t count, const float* secretion_rates, const float* saturation_densities,
					const float* uptake_rates, const float* net_export_rates, const float* internalized_substrates,
					const float* fraction_released_at_death, const float* volumes, const float* positions);
int bfvm_remove_agents(bfvm_solver* s, int32_t count, const int32_t* indices);
int bfvm_plan_agent_removal(int32_t agents, int32_t count, const int32_t* indices, int32_t* remaining,
							int32_t* moves, int32_t* dst, int32_t* src);

/*
 * `steps` full steps of the reference driver's loop (src/main.cpp:68-107): diffusion, gradient,
 * then secretion with recompute = ((first_step + i) % 10 == 0).  Replayed from CUDA graphs.
 */
int bfvm_run_steps(bfvm_solver* s, int32_t steps, int32_t first_step);

/* Wait for the stream and the asynchronous copies (solver::wait_for_all) and report device-side
 * errors. */
int bfvm_synchronize(bfvm_solver* s);

/*
 * Tuning options (no counterpart in the reference; they replace the reference's abort() on a
 * device error, src/solver/device/CUDA/device_context.h:12-21, with a bounded wait and a status):
 * - "tma_sweeps" 0/1 stages sweep tiles through shared memory with the TMA (default 1; 0 selects
 *   the kernels that read the field directly).  Results agree to rounding either way.
 * - "tma_prefetch" 0/1: each staged-sweep refill also prefetches into L2 the tile after the one it
 *   copies (default 0).  Results are identical either way.
 * - "chunk_elements" N in [64, 512], or 0 (the default, automatic): lines longer than N are swept as
 *   chunks of at most N elements by the staged sweep, joined by per-line carries; automatic cuts
 *   lines longer than 512 into chunks of at most 320 along x and 512 along y and z.  Results agree
 *   to rounding with the sweep of whole lines.
 * - "tma_pairs" 0/1/2: staged sweeps whose two warp groups share each shared-memory stage, which then
 *   holds two adjacent tiles copied as one 64-column box: 1 (the default) the z sweep, 2 the y and z
 *   sweeps, 0 neither.  Results are identical either way.
 * - "fused_dirichlet" 0/1: in the LOD step (bfvm_diffusion_solve, bfvm_run_steps) a staged sweep
 *   writes the Dirichlet overwrite that follows it, tile by tile (default 0: the scatter kernel
 *   after the sweep, measured faster).  Results are identical either way.
 * - "fused_gradient" 0/1: in bfvm_run_steps and bfvm_diffusion_gradient_solve the z sweep computes
 *   the gradient from the planes it has just written (default 0: the gradient kernel after the
 *   sweep, measured faster).  Results are identical either way.  "fused_gradient_evict_first" 0/1
 *   (default 1): that sweep reads its tiles with an L2 evict-first policy.
 * - "face_dirichlet" 0/1: in the LOD step the staged sweeps write the Dirichlet face conditions by
 *   position into the values they store (the reference's face order decides where faces meet), and
 *   the scatter after each sweep keeps the interior elements alone (default 0: the scatter of every
 *   conditioned element).  Taken only when no interior Dirichlet voxel lies on a conditioned face.
 *   Results are identical either way.
 * - "xy_band_planes" N, "zg_band_rows" N (default 0: off): the LOD step in bands that stay in L2
 *   between two kernels: the x and y sweeps band by band of N z planes, the z sweep and the gradient
 *   band by band of N y rows.  Results are identical either way; measured slower at 320^3 x 16.
 * - "wait_limit_cycles" bounds every wait of the staged sweeps on a tile copy, in GPU clock cycles
 *   (default 4e9, about two seconds; accepted range [1e4, 4e10]).  A wait that runs out makes the
 *   kernel give up its tile, let its copies in flight land and return; the next synchronising call
 *   returns BFVM_ERR_TIMEOUT, and the field is then not valid until it is stored again.
 * - "test_drop_tile_copy" (tests of that bound only) names a staged-sweep tile whose stage barrier
 *   is armed but whose copies are never issued, so its wait runs out; -1 (the default) turns it off.
 */
int bfvm_set_option(bfvm_solver* s, const char* name, int64_t value);

/*
 * Autotuning (no counterpart in the reference): for every axis whose sweep is staged through
 * shared memory, time each launch shape that fits (warp groups per CTA x pipeline stages per group)
 * on a scratch copy of the field, and keep the fastest.  The choice is also recorded for the rest
 * of the process under the mesh shape, so solvers of the same shape use it without measuring.
 * choices, if not NULL, receives [dims][2] = (groups, stages), (0, 0) for an axis the staged path
 * does not take.  Results do not depend on the launch shape.  Needs one field's worth of scratch.
 */
int bfvm_autotune(bfvm_solver* s, int32_t* choices);

/* Device pointers to the resident field and gradients, for zero-copy use by other GPU code. */
int bfvm_device_densities(bfvm_solver* s, float** ptr, int64_t* count);
int bfvm_device_gradients(bfvm_solver* s, float** ptr, int64_t* count);

/*
 * Bulk supply and uptake (bulk_solver::initialize / solve, src/solver/host/bulk_solver.cpp:8-98):
 * D = (D + dt*S*T) / (1 + dt*(U+S)) for every voxel and substrate.  The reference calls three
 * callbacks per voxel; here their values are tabulated: per_voxel != 0 takes [voxels][substrates]
 * arrays, per_voxel == 0 one [substrates] row for every voxel.  supply_rates == NULL removes the
 * tables.  bfvm_bulk_solve applies one step (BFVM_ERR_STATE before any rates are set); it is not
 * part of bfvm_run_steps, as the reference's driver does not call it either.
 */
int bfvm_set_bulk_rates(bfvm_solver* s, int per_voxel, const float* supply_rates, const float* uptake_rates,
                        const float* supply_target_densities);
int bfvm_bulk_solve(bfvm_solver* s);

/* Number of this library's kernel launches issued so far on this solver (graph replays count
 * every kernel node). */
int bfvm_launch_count(const bfvm_solver* s, int64_t* launches);

/*
 * Batched ensembles (no counterpart in the reference): independent solvers of one device, with
 * uneven meshes, substrate and agent counts, stepped together.  bfvm_batch_run_steps runs
 * `steps` steps of every instance (each exactly what bfvm_run_steps runs on that solver alone)
 * as one CUDA graph whose branches are the instances, so their kernels share the GPU; it is
 * ordered after work already queued on the instances' streams, and later calls on a solver see
 * its results.  The batch does not own the solvers; destroy it before them.
 * bfvm_batch_synchronize waits and returns the first instance's device-side error, if any.
 */
typedef struct bfvm_batch bfvm_batch;
int bfvm_batch_create(bfvm_batch** out, int32_t count, bfvm_solver* const* solvers);
int bfvm_batch_destroy(bfvm_batch* b);
int bfvm_batch_run_steps(bfvm_batch* b, int32_t steps, int32_t first_step);
int bfvm_batch_synchronize(bfvm_batch* b);
/*
 * Autotuning of a batch (no counterpart in the reference): time each launch choice of the
 * ensemble kernels on scratch copies of the instances' fields and gradients, phase by phase, and
 * keep the fastest for this batch and, for the rest of the process, for batches of the same
 * meshes.  The choices: per sweep axis the register cap (1 or 2 CTAs of up to 512 threads per SM)
 * and CTAs per slot of tiles (1, 2, 4); for the gradient the planes per work unit (32, 64, 128)
 * and per batch of loads (4, 8).  choices, if not NULL, receives [8] = minb x/y/z, split x/y/z,
 * gradient planes, gradient load batch.  Results do not depend on the choices.  Needs one
 * field-and-gradient's worth of scratch for every instance.
 */
int bfvm_batch_autotune(bfvm_batch* b, int32_t* choices);

/*
 * z-slabs (no counterpart in the reference, whose solvers hold a whole mesh on one device): one 3D
 * mesh split along z into slab_count slabs, each held by its own solver, normally one per GPU.
 * slab_planes[slab_count + 1] lists the plane boundaries, 0 = slab_planes[0] < ... <
 * slab_planes[slab_count] = the mesh's z plane count; slab k holds planes [slab_planes[k],
 * slab_planes[k + 1]), at least 2 and, with more than one slab, at most 512 of them, and X *
 * substrates must then be a multiple of 4.  bfvm_create_slab takes the whole mesh as bfvm_create
 * does (dims 3) and creates the solver of slab `slab`: its grid_shape, field, gradients and
 * Dirichlet conditions are the slab's planes only (local z = mesh z - slab_planes[slab]; agent
 * positions stay in mesh coordinates).  The caller gives each slab its part of the conditions (the
 * z-min face to slab 0, the z-max face to the last) and the agents whose voxel it holds.
 *
 * The x and y sweeps, Dirichlet overwrites, secretion and release stay within a slab.  The z sweep
 * and the z gradient cross slabs, so with slab_count > 1 bfvm_diffusion_solve, the z axis of
 * bfvm_diffusion_sweep, bfvm_gradient_solve and bfvm_run_steps return BFVM_ERR_STATE, and a step
 * of the split mesh is, on every slab in the same order:
 *   bfvm_slab_diffusion_begin(s, mine)   Dirichlet, x sweep, Dirichlet, y sweep, Dirichlet, and the
 *                                        reduce pass of the z sweep, writing mine [2][X*Y*S]
 *   (the caller gathers every slab's `mine`, in slab order, into all [slab_count][2][X*Y*S])
 *   bfvm_slab_diffusion_end(s, all)      the rest of the z sweep, closing Dirichlet overwrite
 *   bfvm_slab_edge_planes(s, lo, hi)     copies the slab's first and last planes [Y][X][S]
 *   (the caller hands slab k's `hi` to slab k+1 as plane_below, its `lo` to slab k-1 as plane_above)
 *   bfvm_slab_gradient_solve(s, below, above)
 *   bfvm_secretion_solve(s, recompute)
 * Buffers are device memory of the slab's device; the exchanges between the calls are the caller's
 * (an all-gather and a neighbour exchange over NCCL, or copies between solvers of one GPU), ordered
 * on the solver's stream.  The result is the single-solver step of the whole mesh up to float
 * rounding in the z sweep.  A solver created with slab_count 1 is an ordinary solver.
 */
int bfvm_create_slab(bfvm_solver** out, int device, const int32_t bounding_box_mins[3],
                     const int32_t bounding_box_maxs[3], const int32_t voxel_shape[3], int32_t substrates,
                     float time_step, const float* diffusion_coefficients, const float* decay_rates,
                     int compute_internalized_substrates, int32_t slab_count, const int32_t* slab_planes, int32_t slab);
/* slab_count, this solver's slab, its first plane in the mesh and the mesh's plane count (1, 0, 0,
 * grid z for a solver made by bfvm_create).  Any output may be NULL. */
int bfvm_slab_info(const bfvm_solver* s, int32_t* slab_count, int32_t* slab, int32_t* first_plane,
                   int32_t* mesh_planes);
int bfvm_slab_diffusion_begin(bfvm_solver* s, float* exchange);
int bfvm_slab_diffusion_end(bfvm_solver* s, const float* exchange_all);
/* Either output may be NULL. */
int bfvm_slab_edge_planes(bfvm_solver* s, float* first_plane, float* last_plane);
/* plane_below is required except on slab 0, plane_above except on the last slab. */
int bfvm_slab_gradient_solve(bfvm_solver* s, const float* plane_below, const float* plane_above);
/*
 * Host only (no GPU needed): the coefficients that couple the slabs of a z line, [slab_count][3]
 * [substrates] = (Gamma, beta, Lambda) per slab.  Slab k, solved from zero carries, yields A (its
 * last forward-eliminated value) and B (its first solution value); with the true carries C_k
 * (forward value before the slab) and X_k (solution after it),
 *   C_{k+1} = A_k + Gamma_k C_k  (C_0 = 0),   X_{k-1} = B_k + beta_k C_k + Lambda_k X_k  (X_last = 0).
 * This is what bfvm_slab_diffusion_end evaluates per line.
 */
int bfvm_slab_coefficients(int32_t planes, int32_t voxel_z, int32_t substrates, float time_step,
                           const float* diffusion_coefficients, const float* decay_rates, int32_t slab_count,
                           const int32_t* slab_planes, float* coefficients);
/*
 * Host only: the weights of the reduce pass of the slab holding planes [first_plane, end_plane) of
 * a mesh of `planes` planes.  A = sum_k weights[k][s] u[*a_first - first_plane + k] over k <
 * *a_count, and B = sum_k weights[*a_count + k][s] u[k] over k < *b_count, with u the slab's
 * planes (line by line).  Planes whose weights sum to at most 2^-50 (the largest over the
 * substrates) are left out; A is empty for the last slab and B for the first.  `weights` must hold
 * 2 * (end_plane - first_plane) * substrates floats (both sums may keep every plane).
 */
int bfvm_slab_reduce_weights(int32_t planes, int32_t voxel_z, int32_t substrates, float time_step,
                             const float* diffusion_coefficients, const float* decay_rates, int32_t first_plane,
                             int32_t end_plane, float* weights, int32_t* a_first, int32_t* a_count, int32_t* b_count);

/*
 * The learned surrogate (no counterpart in the reference): a 3D convolutional operator that
 * advances a field of `substrates` (1..10) by 16 steps at once,
 *   field(t + 16 dt) = field(t) + net(field(t), 16 x sources, 16 x sinks)
 * where sources and sinks are one step's secretion terms per voxel (bfvm_sur_agent_rates).  The
 * network: a 3x3x3 convolution to 32 channels with ReLU, 4 residual blocks of two 3x3x3 convolutions
 * (ReLU between), a 3x3x3 projection to the substrates; bf16 weights and activations, f32
 * accumulation on the tensor cores, f32 master weights trained with Adam on the mean squared error.
 * The mesh needs at least 128 voxels along x.  Fields, sources, sinks, targets and predictions are
 * device arrays [batch][voxels][substrates], f32, voxels in the field's [z][y][x] order; batch is
 * 1..max_batch.  Parameters: bfvm_sur_parameter_count floats, layer by layer, each W[27][32 out][32
 * in] (tap t = 9 (dz+1) + 3 (dy+1) + (dx+1)) then b[32].  Work runs on the surrogate's stream; calls
 * that return a loss (non-NULL) or host data wait for it.
 */
typedef struct bfvm_surrogate bfvm_surrogate;
int bfvm_sur_create(bfvm_surrogate** out, int device, const int32_t grid_shape[3], int32_t substrates,
                    int32_t max_batch, uint64_t seed);
int bfvm_sur_destroy(bfvm_surrogate* n);
int bfvm_sur_set_stream(bfvm_surrogate* n, void* stream);
int bfvm_sur_parameter_count(const bfvm_surrogate* n, int64_t* count);
/* Replace the parameters (host array) and reset the optimiser; save copies them out. */
int bfvm_sur_load(bfvm_surrogate* n, const float* parameters);
int bfvm_sur_save(bfvm_surrogate* n, float* parameters);
/* prediction of field(t + 16 dt) into out */
int bfvm_sur_infer(bfvm_surrogate* n, int32_t batch, const float* field, const float* sources, const float* sinks,
                   float* out);
/* forward and backward: prediction, the parameters' gradients (bfvm_sur_load_gradients) and the mean
 * squared error against target */
int bfvm_sur_gradients(bfvm_surrogate* n, int32_t batch, const float* field, const float* sources, const float* sinks,
                       const float* target, float* prediction, float* loss);
int bfvm_sur_load_gradients(bfvm_surrogate* n, float* gradients);
/* bfvm_sur_gradients, then one Adam step (beta 0.9, 0.999, eps 1e-8) */
int bfvm_sur_train_step(bfvm_surrogate* n, int32_t batch, const float* field, const float* sources,
                        const float* sinks, const float* target, float* prediction, float learning_rate, float* loss);
/* wait for the stream; BFVM_ERR_TIMEOUT if a kernel's bounded wait gave up */
int bfvm_sur_synchronize(bfvm_surrogate* n);
/* One step's secretion terms per voxel, summed over the agents (cell_solver.cpp:63-85 of the
 * reference): sources = sum S T dt vol / V_vox + N dt / V_vox, sinks = sum (U + S) dt vol / V_vox.
 * Device arrays; sources and sinks [voxels][substrates] are overwritten.  Positions [agents][3]. */
int bfvm_sur_agent_rates(const int32_t bounding_box_mins[3], const int32_t voxel_shape[3], const int32_t grid_shape[3],
                         int32_t substrates, float time_step, int32_t agent_count, const float* secretion_rates,
                         const float* saturation_densities, const float* uptake_rates, const float* net_export_rates,
                         const float* volumes, const float* positions, float* sources, float* sinks,
                         int32_t* error_flags, void* stream);
/* field [voxels][substrates] (device) = sum of Gaussian bumps, bump_params (host, read during the
 * call) [substrates][bumps][5] = (x, y, z, width, amplitude) in voxel units; 1..10 substrates, 1..16
 * bumps; ordered on `stream` */
int bfvm_sur_random_field(const int32_t grid_shape[3], int32_t substrates, int32_t bumps, const float* bump_params,
                          float* field, void* stream);
/*
 * One convolution layer on device tensors, the kernels the network runs (exported for tests and
 * other networks).  shape = (X, Y, Z, batch); tensors [batch][Z][Y][X][32] bf16; weights bf16
 * [27][32 out][32 in].  out = mask(relu(conv + bias + residual)) as bf16 and/or out_f32[voxel]
 * [:out_channels] (+ base_f32); any of bias, residual, mask, base_f32 may be NULL.  The weight
 * gradient adds sum_v grad[v][co] input[v + off_t][ci] into weight_grad [27][32][32] (f32).
 */
int bfvm_sur_conv3d(const int32_t shape[4], const void* input, const void* weights, const float* bias,
                    const void* residual, int32_t relu, const void* mask, void* out, float* out_f32,
                    const float* base_f32, int32_t out_channels, int32_t* error_flags, void* stream);
int bfvm_sur_conv3d_wgrad(const int32_t shape[4], const void* input, const void* grad, float* weight_grad,
                          int32_t* error_flags, void* stream);

/*
 * Secretion and uptake with recompute, for callers that cannot allocate GPU memory: code that runs
 * under a memory budget planned ahead of time, inside a host framework that owns every device
 * allocation, or while another library's stream capture forbids cudaMalloc.  No counterpart in the
 * reference; it does what bfvm_secretion_solve(s, 1) does for a solver holding the same field and
 * agents, on buffers the caller owns, and allocates nothing: no cudaMalloc, no cudaFree, no
 * allocating library routine.
 *
 * Every pointer except `error_flags` and `internalized_substrates` is required (the agent arrays
 * when agent_count > 0) and is device memory of the current device: densities [voxels][substrates]
 * (updated in place), the four rate arrays [agent_count][substrates], internalized_substrates
 * (updated in place, or NULL when internalized substrates are not tracked), volumes
 * [agent_count], positions [agent_count][dims].  The mesh is given as in bfvm_create by its
 * minimum corner and voxel shape, plus grid_shape (1 along unused axes).  Work is enqueued on
 * `stream` (a cudaStream_t; NULL is the legacy default stream) and the call returns without
 * waiting.  An agent outside the mesh is skipped and sets the value 1 (bit 0) in *error_flags
 * (device int) when error_flags is not NULL.
 *
 * Its scratch memory is one static device array of BFVM_NOALLOC_SCRATCH_BYTES (about 8 MB), held
 * by every GPU that loads the library until the process exits; the call rejects more than
 * BFVM_NOALLOC_MAX_AGENTS agents or more than BFVM_NOALLOC_MAX_AGENT_SUBSTRATES agent x substrate
 * pairs with BFVM_ERR_INVALID_ARGUMENT.  A call outside stream capture looks up the array's device
 * address (cudaGetSymbolAddress) and keeps it for calls made while `stream` is capturing, which
 * reuse it: make the first call on each device before any capture (a call captured first returns
 * BFVM_ERR_STATE), and after a device reset make one call outside capture again.  All calls share
 * the array, so calls that overlap on the GPU (other streams, other host threads) race: order
 * them on one stream.
 */
#define BFVM_NOALLOC_MAX_AGENTS 65536
#define BFVM_NOALLOC_MAX_AGENT_SUBSTRATES 262144
#define BFVM_NOALLOC_SCRATCH_BYTES 8143872
int bfvm_secretion_solve_noalloc(float* densities, int dims, const int32_t bounding_box_mins[3],
                                 const int32_t voxel_shape[3], const int32_t grid_shape[3], int32_t substrates,
                                 float time_step, int32_t agent_count, const float* secretion_rates,
                                 const float* saturation_densities, const float* uptake_rates,
                                 const float* net_export_rates, float* internalized_substrates, const float* volumes,
                                 const float* positions, int32_t* error_flags, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BFVM_H */
