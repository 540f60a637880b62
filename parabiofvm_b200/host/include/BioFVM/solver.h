// The solver classes of the reference's device path (include/BioFVM/solver.h,
// src/solver/device/CUDA/solver.h:12-31) on the B200 library's C ABI (include/bfvm.h).
//
//   biofvm::solver s;
//   s.initialize(m);                  // creates the GPU state: mesh, coefficients, Dirichlet
//   s.store_data_to_solver(m);        // field and agents to the GPU
//   s.diffusion.solve(m);             // Dirichlet + x/y/z sweeps + Dirichlet
//   s.gradient.solve(m);              // central differences of the current field
//   s.cell.simulate_secretion_and_uptake(m, recompute);
//   s.load_data_from_solver(m);       // field, gradients and internalized substrates back
//
// Failures throw std::runtime_error with the library's message (the reference aborts on CUDA
// errors).  Calls are ordered on the solver's stream; loads wait for the work before them.
#pragma once

#include <memory>
#include <vector>

#include "microenvironment.h"

struct bfvm_solver;

namespace biofvm {
namespace solvers::b200 {

// the shared GPU state of one solver
struct context
{
	bfvm_solver* handle = nullptr;
	int device = 0;
};

class diffusion_solver
{
	context& ctx_;

public:
	explicit diffusion_solver(context& ctx) : ctx_(ctx) {}
	void initialize(microenvironment& m);
	void solve(microenvironment& m);
	// one axis: its Dirichlet overwrite and sweep (and the closing overwrite after the last axis)
	void solve_axis(microenvironment& m, index_t axis);
};

class dirichlet_solver
{
	context& ctx_;

public:
	explicit dirichlet_solver(context& ctx) : ctx_(ctx) {}
	void solve(microenvironment& m);
};

class gradient_solver
{
	context& ctx_;

public:
	explicit gradient_solver(context& ctx) : ctx_(ctx) {}
	void solve(microenvironment& m);
};

// Bulk supply/uptake (src/solver/host/bulk_solver.h of the reference).  initialize() evaluates the
// microenvironment's three callbacks once for every voxel and keeps the table on the GPU;
// call it again when the rates change.  solve() applies one step.
class bulk_solver
{
	context& ctx_;

public:
	explicit bulk_solver(context& ctx) : ctx_(ctx) {}
	void initialize(microenvironment& m);
	void solve(microenvironment& m);
};

class cell_solver
{
	context& ctx_;

public:
	explicit cell_solver(context& ctx) : ctx_(ctx) {}
	void initialize(microenvironment& m);
	void simulate_secretion_and_uptake(microenvironment& m, bool recompute);
	void release_internalized_substrates(microenvironment& m, index_t index);
	// Agents added and removed on the GPU copy alone, keeping it in step with the host agent data
	// without copying the stored agents again.  add_agents: the host agents [first, first + count)
	// (added with agent_data::add and filled in) are appended; first must equal the GPU's count.
	// remove_agents: agent_data::remove of indices[0], indices[1], ... in order, as the host
	// container did them.
	void add_agents(microenvironment& m, index_t first, index_t count);
	void remove_agents(microenvironment& m, const std::vector<index_t>& indices);
};

class solver
{
	context ctx_;

public:
	static constexpr bool is_device_solver = true;

	// device: CUDA device index for initialize()
	explicit solver(int device = 0);
	~solver();
	solver(const solver&) = delete;
	solver& operator=(const solver&) = delete;

	cell_solver cell;
	diffusion_solver diffusion;
	gradient_solver gradient;
	dirichlet_solver dirichlet;
	bulk_solver bulk;

	void initialize(microenvironment& m);

	void store_data_to_solver(microenvironment& m);
	void load_data_from_solver(microenvironment& m);

	void wait_for_all();

	// time the staged sweeps' launch shapes on a scratch copy of the field and keep the fastest
	void autotune();

	// `steps` steps of the reference driver's loop (diffusion, gradient, secretion with recompute
	// every 10th step), replayed from CUDA graphs
	void run_steps(microenvironment& m, index_t steps, index_t first_step = 0);

	bfvm_solver* handle() const { return ctx_.handle; }
};

} // namespace solvers::b200

// the names the reference's device backends use (include/BioFVM/solver.h of the reference), for
// code written against solvers::device::solver directly
namespace solvers {
namespace device = b200;
}

using solver = solvers::b200::solver;
using cell_solver = solvers::b200::cell_solver;

} // namespace biofvm
