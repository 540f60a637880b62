// Ensemble kernels of a batch (batch_kernels.cu): one launch per phase of the step for every mesh
// of the batch, driven by work lists, instead of one launch per phase and mesh.
#pragma once

#include <vector>

#include "bfvm_internal.h"

namespace bfvm {

static constexpr int ENS_MAX_P = 16;	 // blocks of 32 per line the ensemble sweep handles in a batch
static constexpr int ENS_MAX_P_ONE = 32; // ... for one mesh alone (CTAs of up to 1024 threads)

// Everything a kernel needs of one mesh (device copy in ensemble_plan::inst).
struct ens_inst
{
	float* dens;
	float* grad;
	int dims, S, X, Y, Z;
	float bgrad[3], cgrad[3]; // gradient factors 1/h and 1/(2h) per axis (float, as the reference)
	// sweeps: front-padded tables of each axis (precompute_padded)
	const float* vtab[3];
	int vP[3], pad[3];
	// Dirichlet overwrite list
	const long long* dir_qidx; // runs of four (dirichlet.cu)
	const float4* dir_qval;
	long long dir_qcount;
	const long long* dir_idx; // single elements
	const float* dir_val;
	long long dir_count;
	// faces by position (dirichlet.cu, face_pos_ok): each sweep writes the face conditions into the
	// values it stores, so the overwrites after the sweeps take only the interior list (dir_i*).
	// face_bits[s]: bit f when face f conditions substrate s; face_vals [6][S].  faces 0: none.
	int faces;
	const int* face_bits;
	const float* face_vals;
	const long long* dir_iqidx;
	const float4* dir_iqval;
	long long dir_iqcount;
	const long long* dir_iidx;
	const float* dir_ival;
	long long dir_icount;
	// secretion (the binning of the mesh's cell solver).  sorted: num/den/fac/intern are the agent
	// terms in the binning's sorted order (agent_state::snum ...), else in agent order; vec4: sorted
	// with S % 4 == 0, a unit is 256 (segment, four substrates) pairs
	long long AS; // agents * S (0 without agents)
	int internalized;
	int sorted, vec4;
	float voxel_volume;
	const int* counts;
	const int* seg_start;
	const int* order;
	const unsigned int* keys;
	const float *num, *den, *fac, *red_num, *red_den, *red_fac;
	float* intern;
};

// Per phase, a prefix list over the meshes: mesh i owns work units [first[i], first[i+1]).
// Units are 256-element blocks (Dirichlet, gradient, secretion) or 32-line tiles (sweeps).
enum ens_phase : int
{
	ENS_DIRICHLET = 0,
	ENS_SWEEP_X = 1,
	ENS_SWEEP_Y = 2,
	ENS_SWEEP_Z = 3,
	ENS_GRADIENT = 4,
	ENS_SECRETION = 5,
	ENS_PHASES = 6
};

// Launch choices of the ensemble kernels (batch_kernels.cu), picked by bfvm_batch_autotune:
// per sweep axis, the register cap (CTAs of up to 512 threads resident per SM: 1 or 2) and how many
// CTAs share a slot's run of tiles (1, 2 or 4: shorter runs balance better, longer runs restage
// the coefficient tables less often); for the gradient, the planes per work unit and the planes
// whose loads are issued together.
struct ens_tuning
{
	int sweep_minb[3] = { 2, 2, 2 };
	int sweep_split[3] = { 1, 1, 1 };
	int grad_zc = 64;
	int grad_zu = 8;
};

struct ensemble_plan
{
	int count = 0;					 // meshes in the ensemble
	ens_inst* inst = nullptr;		 // device [count]
	long long* first[ENS_PHASES] = {}; // device [count + 1]
	// the mesh of every unit of the per-element phases (Dirichlet, gradient, secretion), so a unit
	// finds its mesh with one load instead of a binary search over `first`; device [units]
	int* unit_mesh[ENS_PHASES] = {};
	std::vector<long long> first_h[ENS_PHASES];
	int maxP[3] = { 1, 1, 1 };		 // largest vP per axis
	int maxS = 1;
	size_t table_floats[3] = { 0, 0, 0 }; // largest staged table per axis
	bool all3d = true;					  // every mesh is 3-D (the gradient kernel without the 1-D/2-D forms)
	ens_tuning tune;					  // launch choices (the gradient units follow tune.grad_zc)
	// the Dirichlet overwrites of every mesh as flat lists of (address, value), runs of four and
	// single elements (ensemble_build_dirichlet; device).  List 0 holds every mesh's whole list, for
	// the overwrite before the x sweep; list 1 the lists of the overwrites after the sweeps (the
	// interior elements alone for meshes whose sweeps write the faces).  Meshes of more dimensions
	// come first, so that overwrite k covers the meshes with dims >= k: the first q_ge[k] / s_ge[k]
	// entries.
	struct flat_list
	{
		float4** qptr = nullptr;
		float4* qval = nullptr;
		float** sptr = nullptr;
		float* sval = nullptr;
		long long q_ge[4] = { 0, 0, 0, 0 }, s_ge[4] = { 0, 0, 0, 0 };
	};
	flat_list dir[2];
	bool dir_built = false;
};

// Which meshes the ensemble kernels cover: every axis with n >= 2 and at most ENS_MAX_P blocks,
// at most 32 substrates.
bool ensemble_eligible(const bfvm_solver* s);
// buffers: when given, the field and gradient buffers of each mesh instead of the solvers' own
// (the autotuner times candidates on scratch copies).  rebinned: the secretion update runs after
// a rebinning of every mesh with agents (prepare_agent_terms), so it finds their agent terms in
// the order that leaves (sorted with internalized substrates) rather than in today's.  faces: the
// sweeps write the face conditions of the meshes that allow it (a batch step; the plan then holds
// pointers to the members' Dirichlet tables and is rebuilt whenever they change).
int ensemble_build(ensemble_plan& plan, const std::vector<bfvm_solver*>& meshes, const ens_tuning& tune = ens_tuning(),
				   const std::vector<std::pair<float*, float*>>* buffers = nullptr, bool rebinned = false,
				   bool faces = false);
void ensemble_free(ensemble_plan& plan);
// The flat Dirichlet lists of a built plan, for ensemble_dirichlet (complete on return; never
// inside a stream capture).
int ensemble_build_dirichlet(ensemble_plan& plan);
// One phase for every mesh of the plan, on `stream`.  `dirichlet_phase` k applies the overwrite to
// meshes with k <= dims (before sweep k, or after the last sweep); it launches nothing when
// ensemble_dirichlet_entries is 0.
int ensemble_dirichlet(const ensemble_plan& plan, int dirichlet_phase, cudaStream_t stream);
long long ensemble_dirichlet_entries(const ensemble_plan& plan, int dirichlet_phase);
int ensemble_sweep(const ensemble_plan& plan, int axis, cudaStream_t stream);
// whether the ensemble sweep of `axis` fits the shared memory of a CTA on this device
bool ensemble_sweep_fits(const ensemble_plan& plan, int axis);
int ensemble_gradient(const ensemble_plan& plan, cudaStream_t stream);
int ensemble_secretion(const ensemble_plan& plan, cudaStream_t stream);

} // namespace bfvm
