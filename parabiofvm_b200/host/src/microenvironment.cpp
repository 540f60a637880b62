// The microenvironment and its builder (src/microenvironment.cpp:14-53,
// src/microenvironment_builder.cpp:112-193 of the reference).

#include <algorithm>
#include <iostream>
#include <stdexcept>

#include "BioFVM/microenvironment.h"
#include "BioFVM/microenvironment_builder.h"

namespace biofvm {

// ------------------------------------------------------------------------------------------------
// microenvironment

microenvironment::microenvironment(cartesian_mesh mesh, index_t substrates_count, real_t time_step,
								   const real_t* initial_conditions)
	: mesh(mesh),
	  agents(std::make_unique<agent_container>(*this)),
	  substrates_count(substrates_count),
	  diffusion_time_step(time_step),
	  substrate_densities(std::make_unique<real_t[]>((std::size_t)substrates_count * mesh.voxel_count())),
	  gradients(std::make_unique<real_t[]>((std::size_t)mesh.dims * substrates_count * mesh.voxel_count())),
	  dirichlet_interior_voxels_count(0),
	  compute_internalized_substrates(false),
	  data_residency(solvers::data_residency::host)
{
	// every voxel starts at the initial conditions: [voxel][s]
	const std::size_t V = mesh.voxel_count();
	real_t* d = substrate_densities.get();
	for (std::size_t v = 0; v < V; v++)
		std::copy_n(initial_conditions, substrates_count, d + v * substrates_count);
	std::fill_n(gradients.get(), (std::size_t)mesh.dims * substrates_count * V, real_t(0));
}

// The agents refer back to their microenvironment, so a move is only possible before any agent
// exists; the moved-to microenvironment gets a fresh, empty container.
microenvironment::microenvironment(microenvironment&& o)
	: name(std::move(o.name)),
	  time_units(std::move(o.time_units)),
	  space_units(std::move(o.space_units)),
	  substrates_names(std::move(o.substrates_names)),
	  substrates_units(std::move(o.substrates_units)),
	  mesh(o.mesh),
	  agents(nullptr),
	  substrates_count(o.substrates_count),
	  diffusion_time_step(o.diffusion_time_step),
	  substrate_densities(std::move(o.substrate_densities)),
	  diffusion_coefficients(std::move(o.diffusion_coefficients)),
	  decay_rates(std::move(o.decay_rates)),
	  gradients(std::move(o.gradients)),
	  dirichlet_interior_voxels_count(o.dirichlet_interior_voxels_count),
	  dirichlet_interior_voxels(std::move(o.dirichlet_interior_voxels)),
	  dirichlet_interior_values(std::move(o.dirichlet_interior_values)),
	  dirichlet_interior_conditions(std::move(o.dirichlet_interior_conditions)),
	  dirichlet_min_boundary_values(std::move(o.dirichlet_min_boundary_values)),
	  dirichlet_max_boundary_values(std::move(o.dirichlet_max_boundary_values)),
	  dirichlet_min_boundary_conditions(std::move(o.dirichlet_min_boundary_conditions)),
	  dirichlet_max_boundary_conditions(std::move(o.dirichlet_max_boundary_conditions)),
	  supply_rate_func(std::move(o.supply_rate_func)),
	  uptake_rate_func(std::move(o.uptake_rate_func)),
	  supply_target_densities_func(std::move(o.supply_target_densities_func)),
	  compute_internalized_substrates(o.compute_internalized_substrates),
	  data_residency(o.data_residency)
{
	if (o.agents && o.agents->agents_count() > 0)
		throw std::logic_error("a microenvironment that holds agents cannot be moved");
	agents = std::make_unique<agent_container>(*this);
}

index_t microenvironment::find_substrate_index(const std::string& name) const
{
	for (index_t i = 0; i < (index_t)substrates_names.size(); i++)
		if (substrates_names[i] == name)
			return i;
	return -1;
}

real_t microenvironment::substrate_density_value(point_t<index_t, 3> position, index_t substrate_index) const
{
	const std::size_t v = (std::size_t)position[0]
						  + (std::size_t)mesh.grid_shape[0]
								* ((std::size_t)position[1] + (std::size_t)mesh.grid_shape[1] * position[2]);
	return substrate_densities[v * substrates_count + substrate_index];
}

void microenvironment::display_info()
{
	mesh.display_info();
	std::cout << "Microenvironment " << name << ": " << substrates_count << " substrates, time step "
			  << diffusion_time_step << " " << time_units << std::endl;
	for (index_t s = 0; s < substrates_count; s++)
		std::cout << "   " << (s < (index_t)substrates_names.size() ? substrates_names[s] : std::string("?"))
				  << ": D = " << diffusion_coefficients[s] << ", decay = " << decay_rates[s] << std::endl;
}

// ------------------------------------------------------------------------------------------------
// microenvironment_builder

void microenvironment_builder::set_name(const std::string& n) { name = n; }
void microenvironment_builder::set_time_units(const std::string& u) { time_units = u; }
void microenvironment_builder::set_space_units(const std::string& u) { space_units = u; }
void microenvironment_builder::set_time_step(real_t dt) { time_step = dt; }

void microenvironment_builder::resize(index_t dims, point_t<index_t, 3> bounding_box_mins,
									  point_t<index_t, 3> bounding_box_maxs, point_t<index_t, 3> voxel_shape)
{
	mesh_.emplace(dims, bounding_box_mins, bounding_box_maxs, voxel_shape);
}

void microenvironment_builder::add_density(const std::string& n, const std::string& units,
										   real_t diffusion_coefficient, real_t decay_rate, real_t initial_condition)
{
	substrates_names.push_back(n);
	substrates_units.push_back(units);
	diffusion_coefficients.push_back(diffusion_coefficient);
	decay_rates.push_back(decay_rate);
	initial_conditions.push_back(initial_condition);
	// no boundary condition until one is added
	boundary_dirichlet_mins_values.push_back({ 0, 0, 0 });
	boundary_dirichlet_maxs_values.push_back({ 0, 0, 0 });
	boundary_dirichlet_mins_conditions.push_back({ false, false, false });
	boundary_dirichlet_maxs_conditions.push_back({ false, false, false });
}

std::size_t microenvironment_builder::get_density_index(const std::string& n) const
{
	const auto it = std::find(substrates_names.begin(), substrates_names.end(), n);
	if (it == substrates_names.end())
		throw std::runtime_error("Density " + n + " not found");
	return (std::size_t)(it - substrates_names.begin());
}

void microenvironment_builder::add_dirichlet_node(point_t<index_t, 3> voxel_index, std::vector<real_t> values,
												  std::vector<bool> conditions)
{
	if (values.size() != substrates_names.size())
		throw std::runtime_error("Dirichlet node values size does not match the number of densities");
	if (!conditions.empty() && conditions.size() != substrates_names.size())
		throw std::runtime_error("Dirichlet node conditions size does not match the number of densities");
	if (!mesh_)
		throw std::runtime_error("Dirichlet node cannot be added without a mesh");
	for (index_t d = 0; d < mesh_->dims; d++)
		dirichlet_voxels.push_back(voxel_index[d]);
	dirichlet_values.insert(dirichlet_values.end(), values.begin(), values.end());
	if (conditions.empty())
		conditions.assign(values.size(), true);
	dirichlet_conditions.insert(dirichlet_conditions.end(), conditions.begin(), conditions.end());
}

void microenvironment_builder::add_boundary_dirichlet_conditions(std::size_t density_index,
																 point_t<real_t, 3> mins_values,
																 point_t<real_t, 3> maxs_values,
																 point_t<bool, 3> mins_conditions,
																 point_t<bool, 3> maxs_conditions)
{
	if (density_index >= substrates_names.size())
		throw std::runtime_error("Density index out of bounds");
	boundary_dirichlet_mins_values[density_index] = mins_values;
	boundary_dirichlet_maxs_values[density_index] = maxs_values;
	boundary_dirichlet_mins_conditions[density_index] = mins_conditions;
	boundary_dirichlet_maxs_conditions[density_index] = maxs_conditions;
}

void microenvironment_builder::set_bulk_functions(bulk_func_t supply, bulk_func_t uptake, bulk_func_t targets)
{
	supply_rate_func = std::move(supply);
	uptake_rate_func = std::move(uptake);
	supply_target_densities_func = std::move(targets);
}

void microenvironment_builder::do_compute_internalized_substrates() { compute_internalized_substrates = true; }

// One face's arrays exist only when at least one substrate is conditioned there.
static void fill_face(index_t axis, index_t S, const std::vector<point_t<real_t, 3>>& values,
					  const std::vector<point_t<bool, 3>>& conditions, std::unique_ptr<real_t[]>& out_values,
					  std::unique_ptr<bool[]>& out_conditions)
{
	bool any = false;
	for (index_t s = 0; s < S; s++)
		any = any || conditions[s][axis];
	if (!any)
		return;
	out_values = std::make_unique<real_t[]>(S);
	out_conditions = std::make_unique<bool[]>(S);
	for (index_t s = 0; s < S; s++)
	{
		out_values[s] = values[s][axis];
		out_conditions[s] = conditions[s][axis];
	}
}

void microenvironment_builder::fill_dirichlet_vectors(microenvironment& m)
{
	for (index_t d = 0; d < m.mesh.dims; d++)
	{
		fill_face(d, m.substrates_count, boundary_dirichlet_mins_values, boundary_dirichlet_mins_conditions,
				  m.dirichlet_min_boundary_values[d], m.dirichlet_min_boundary_conditions[d]);
		fill_face(d, m.substrates_count, boundary_dirichlet_maxs_values, boundary_dirichlet_maxs_conditions,
				  m.dirichlet_max_boundary_values[d], m.dirichlet_max_boundary_conditions[d]);
	}
}

microenvironment microenvironment_builder::build()
{
	if (!mesh_)
		throw std::runtime_error("Microenvironment cannot be built without a mesh");
	if (substrates_names.empty())
		throw std::runtime_error("Microenvironment cannot be built with no densities");

	const index_t S = (index_t)substrates_names.size();
	microenvironment m(*mesh_, S, time_step, initial_conditions.data());
	m.name = name;
	m.time_units = time_units;
	m.space_units = space_units;
	m.substrates_names = substrates_names;
	m.substrates_units = substrates_units;

	m.diffusion_coefficients = std::make_unique<real_t[]>(S);
	std::copy(diffusion_coefficients.begin(), diffusion_coefficients.end(), m.diffusion_coefficients.get());
	m.decay_rates = std::make_unique<real_t[]>(S);
	std::copy(decay_rates.begin(), decay_rates.end(), m.decay_rates.get());

	m.dirichlet_interior_voxels_count = (index_t)(dirichlet_voxels.size() / m.mesh.dims);
	m.dirichlet_interior_voxels = std::make_unique<index_t[]>(dirichlet_voxels.size());
	std::copy(dirichlet_voxels.begin(), dirichlet_voxels.end(), m.dirichlet_interior_voxels.get());
	m.dirichlet_interior_values = std::make_unique<real_t[]>(dirichlet_values.size());
	std::copy(dirichlet_values.begin(), dirichlet_values.end(), m.dirichlet_interior_values.get());
	m.dirichlet_interior_conditions = std::make_unique<bool[]>(dirichlet_conditions.size());
	std::copy(dirichlet_conditions.begin(), dirichlet_conditions.end(), m.dirichlet_interior_conditions.get());

	fill_dirichlet_vectors(m);

	m.supply_rate_func = supply_rate_func;
	m.uptake_rate_func = uptake_rate_func;
	m.supply_target_densities_func = supply_target_densities_func;
	m.compute_internalized_substrates = compute_internalized_substrates;
	return m;
}

} // namespace biofvm
