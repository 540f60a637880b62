// The solver classes of the host API on the C ABI of the GPU library
// (src/solver/device/CUDA/solver.cpp:7-23 and the sub-solvers' public calls in the reference).

#include "BioFVM/solver.h"

#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/bfvm.h"

static_assert(sizeof(bool) == 1, "the C ABI reads Dirichlet conditions as one byte per flag");

namespace biofvm::solvers::b200 {

static void check(int status, const char* what)
{
	if (status != BFVM_OK)
		throw std::runtime_error(std::string(what) + ": " + bfvm_last_error());
}

static bfvm_solver* require(const context& ctx)
{
	if (!ctx.handle)
		throw std::runtime_error("solver used before initialize()");
	return ctx.handle;
}

// ------------------------------------------------------------------------------------------------
// solver

solver::solver(int device)
	: ctx_ { nullptr, device }, cell(ctx_), diffusion(ctx_), gradient(ctx_), dirichlet(ctx_), bulk(ctx_)
{}

solver::~solver()
{
	if (ctx_.handle)
		bfvm_destroy(ctx_.handle);
}

void solver::initialize(microenvironment& m)
{
	if (ctx_.handle)
	{
		bfvm_destroy(ctx_.handle);
		ctx_.handle = nullptr;
	}
	const cartesian_mesh& mesh = m.mesh;
	check(bfvm_create(&ctx_.handle, ctx_.device, mesh.dims, mesh.bounding_box_mins.data(),
					  mesh.bounding_box_maxs.data(), mesh.voxel_shape.data(), m.substrates_count, m.diffusion_time_step,
					  m.diffusion_coefficients.get(), m.decay_rates.get(), m.compute_internalized_substrates ? 1 : 0),
		  "bfvm_create");
	for (index_t d = 0; d < mesh.dims; d++)
	{
		if (m.dirichlet_min_boundary_values[d])
			check(bfvm_set_boundary_dirichlet(ctx_.handle, d, 0, m.dirichlet_min_boundary_values[d].get(),
											  reinterpret_cast<const uint8_t*>(m.dirichlet_min_boundary_conditions[d].get())),
				  "bfvm_set_boundary_dirichlet");
		if (m.dirichlet_max_boundary_values[d])
			check(bfvm_set_boundary_dirichlet(ctx_.handle, d, 1, m.dirichlet_max_boundary_values[d].get(),
											  reinterpret_cast<const uint8_t*>(m.dirichlet_max_boundary_conditions[d].get())),
				  "bfvm_set_boundary_dirichlet");
	}
	if (m.dirichlet_interior_voxels_count > 0)
		check(bfvm_set_interior_dirichlet(ctx_.handle, m.dirichlet_interior_voxels_count,
										  m.dirichlet_interior_voxels.get(), m.dirichlet_interior_values.get(),
										  reinterpret_cast<const uint8_t*>(m.dirichlet_interior_conditions.get())),
			  "bfvm_set_interior_dirichlet");
	diffusion.initialize(m);
	cell.initialize(m);
}

void solver::store_data_to_solver(microenvironment& m)
{
	bfvm_solver* h = require(ctx_);
	check(bfvm_store_densities(h, m.substrate_densities.get()), "bfvm_store_densities");
	agent_data& a = m.agents->get_agent_data();
	check(bfvm_store_agents(h, a.agents_count, a.secretion_rates.data(), a.saturation_densities.data(),
							a.uptake_rates.data(), a.net_export_rates.data(), a.internalized_substrates.data(),
							a.fraction_released_at_death.data(), a.volumes.data(), a.positions.data()),
		  "bfvm_store_agents");
}

void solver::load_data_from_solver(microenvironment& m)
{
	bfvm_solver* h = require(ctx_);
	check(bfvm_load_densities(h, m.substrate_densities.get()), "bfvm_load_densities");
	check(bfvm_load_gradients(h, m.gradients.get()), "bfvm_load_gradients");
	agent_data& a = m.agents->get_agent_data();
	if (a.agents_count > 0)
		check(bfvm_load_internalized(h, a.internalized_substrates.data()), "bfvm_load_internalized");
	check(bfvm_synchronize(h), "bfvm_synchronize");
}

void solver::wait_for_all() { check(bfvm_synchronize(require(ctx_)), "bfvm_synchronize"); }

void solver::autotune() { check(bfvm_autotune(require(ctx_), nullptr), "bfvm_autotune"); }

void solver::run_steps(microenvironment&, index_t steps, index_t first_step)
{
	check(bfvm_run_steps(require(ctx_), steps, first_step), "bfvm_run_steps");
}

// ------------------------------------------------------------------------------------------------
// sub-solvers: their GPU state is created by solver::initialize

void diffusion_solver::initialize(microenvironment&) {}

void diffusion_solver::solve(microenvironment&) { check(bfvm_diffusion_solve(require(ctx_)), "bfvm_diffusion_solve"); }

void diffusion_solver::solve_axis(microenvironment&, index_t axis)
{
	check(bfvm_diffusion_sweep(require(ctx_), axis), "bfvm_diffusion_sweep");
}

void dirichlet_solver::solve(microenvironment&) { check(bfvm_dirichlet_solve(require(ctx_)), "bfvm_dirichlet_solve"); }

void gradient_solver::solve(microenvironment&) { check(bfvm_gradient_solve(require(ctx_)), "bfvm_gradient_solve"); }

void bulk_solver::initialize(microenvironment& m)
{
	bfvm_solver* h = require(ctx_);
	if (!m.supply_rate_func || !m.uptake_rate_func || !m.supply_target_densities_func)
	{
		check(bfvm_set_bulk_rates(h, 0, nullptr, nullptr, nullptr), "bfvm_set_bulk_rates");
		return;
	}
	const cartesian_mesh& mesh = m.mesh;
	const std::size_t S = m.substrates_count;
	const std::size_t n = mesh.voxel_count() * S;
	std::vector<real_t> supply(n), uptake(n), target(n);
	std::size_t v = 0;
	for (index_t z = 0; z < mesh.grid_shape[2]; z++)
		for (index_t y = 0; y < mesh.grid_shape[1]; y++)
			for (index_t x = 0; x < mesh.grid_shape[0]; x++, v++)
			{
				m.supply_rate_func(m, { x, y, z }, supply.data() + v * S);
				m.uptake_rate_func(m, { x, y, z }, uptake.data() + v * S);
				m.supply_target_densities_func(m, { x, y, z }, target.data() + v * S);
			}
	check(bfvm_set_bulk_rates(h, 1, supply.data(), uptake.data(), target.data()), "bfvm_set_bulk_rates");
}

void bulk_solver::solve(microenvironment&) { check(bfvm_bulk_solve(require(ctx_)), "bfvm_bulk_solve"); }

void cell_solver::initialize(microenvironment&) {}

void cell_solver::simulate_secretion_and_uptake(microenvironment&, bool recompute)
{
	check(bfvm_secretion_solve(require(ctx_), recompute ? 1 : 0), "bfvm_secretion_solve");
}

void cell_solver::release_internalized_substrates(microenvironment&, index_t index)
{
	check(bfvm_release_internalized(require(ctx_), index), "bfvm_release_internalized");
}

void cell_solver::add_agents(microenvironment& m, index_t first, index_t count)
{
	agent_data& a = m.agents->get_agent_data();
	if (first < 0 || count < 0 || first + count > a.agents_count)
		throw std::runtime_error("add_agents: agents [first, first + count) are not all in the host agent data");
	const std::size_t S = (std::size_t)m.substrates_count, d = (std::size_t)m.mesh.dims;
	check(bfvm_add_agents(require(ctx_), count, a.secretion_rates.data() + first * S,
						  a.saturation_densities.data() + first * S, a.uptake_rates.data() + first * S,
						  a.net_export_rates.data() + first * S, a.internalized_substrates.data() + first * S,
						  a.fraction_released_at_death.data() + first * S, a.volumes.data() + first,
						  a.positions.data() + first * d),
		  "bfvm_add_agents");
}

void cell_solver::remove_agents(microenvironment&, const std::vector<index_t>& indices)
{
	std::vector<int32_t> idx(indices.begin(), indices.end());
	check(bfvm_remove_agents(require(ctx_), (int32_t)idx.size(), idx.data()), "bfvm_remove_agents");
}

} // namespace biofvm::solvers::b200
