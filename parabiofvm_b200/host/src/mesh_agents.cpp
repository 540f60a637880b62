// Mesh, agent data and agent views of the host API (src/mesh.cpp:7-53, src/agent_data.cpp:10-53,
// src/agent.cpp of the reference).

#include <algorithm>
#include <iostream>

#include "BioFVM/agent.h"
#include "BioFVM/agent_data.h"
#include "BioFVM/mesh.h"
#include "BioFVM/microenvironment.h"

namespace biofvm {

// ------------------------------------------------------------------------------------------------
// cartesian_mesh

cartesian_mesh::cartesian_mesh(index_t dims, point_t<index_t, 3> bounding_box_mins,
							   point_t<index_t, 3> bounding_box_maxs, point_t<index_t, 3> voxel_shape)
	: dims(dims),
	  bounding_box_mins(bounding_box_mins),
	  bounding_box_maxs(bounding_box_maxs),
	  voxel_shape(voxel_shape),
	  grid_shape { 1, 1, 1 }
{
	for (index_t d = 0; d < dims && d < 3; d++)
		grid_shape[d] = (bounding_box_maxs[d] - bounding_box_mins[d] + voxel_shape[d] - 1) / voxel_shape[d];
}

std::size_t cartesian_mesh::voxel_count() const
{
	return (std::size_t)grid_shape[0] * (std::size_t)grid_shape[1] * (std::size_t)grid_shape[2];
}

index_t cartesian_mesh::voxel_volume() const { return voxel_shape[0] * voxel_shape[1] * voxel_shape[2]; }

template <index_t dims_>
point_t<index_t, 3> cartesian_mesh::voxel_position(const real_t* position) const
{
	static_assert(dims_ >= 1 && dims_ <= 3);
	point_t<index_t, 3> v { 0, 0, 0 };
	for (index_t d = 0; d < dims_; d++)
		v[d] = (index_t)((position[d] - bounding_box_mins[d]) / voxel_shape[d]);
	return v;
}

template point_t<index_t, 3> cartesian_mesh::voxel_position<1>(const real_t*) const;
template point_t<index_t, 3> cartesian_mesh::voxel_position<2>(const real_t*) const;
template point_t<index_t, 3> cartesian_mesh::voxel_position<3>(const real_t*) const;

point_t<real_t, 3> cartesian_mesh::voxel_center(point_t<index_t, 3> position) const
{
	point_t<real_t, 3> c;
	for (int d = 0; d < 3; d++)
		c[d] = (real_t)(position[d] * voxel_shape[d] + voxel_shape[d] / 2.0 + bounding_box_mins[d]);
	return c;
}

void cartesian_mesh::display_info()
{
	std::cout << "\nMesh information:\n   dimensions: " << dims << "\n   domain: ";
	for (int d = 0; d < 3; d++)
		std::cout << (d ? " x " : "") << "[" << bounding_box_mins[d] << "," << bounding_box_maxs[d] << "]";
	std::cout << "\n   resolution: " << voxel_shape[0] << " x " << voxel_shape[1] << " x " << voxel_shape[2]
			  << "\n   voxels: " << voxel_count() << std::endl;
}

// ------------------------------------------------------------------------------------------------
// agent_data

agent_data::agent_data(microenvironment& m) : agents_count(0), m(m) {}

void agent_data::add()
{
	agents_count++;
	const std::size_t rows = (std::size_t)agents_count * m.substrates_count;
	for (auto* v : { &secretion_rates, &saturation_densities, &uptake_rates, &net_export_rates,
					 &internalized_substrates, &fraction_released_at_death, &fraction_transferred_when_ingested })
		v->resize(rows, 0);
	volumes.resize(agents_count, 0);
	positions.resize((std::size_t)agents_count * m.mesh.dims, 0);
}

void agent_data::remove(index_t index)
{
	agents_count--;
	if (index == agents_count)
		return; // the last agent: the arrays keep their (now unused) tail
	const std::size_t S = m.substrates_count;
	for (auto* v : { &secretion_rates, &saturation_densities, &uptake_rates, &net_export_rates,
					 &internalized_substrates, &fraction_released_at_death, &fraction_transferred_when_ingested })
		std::copy_n(v->data() + (std::size_t)agents_count * S, S, v->data() + (std::size_t)index * S);
	volumes[index] = volumes[agents_count];
	std::copy_n(positions.data() + (std::size_t)agents_count * m.mesh.dims, m.mesh.dims,
				positions.data() + (std::size_t)index * m.mesh.dims);
}

// ------------------------------------------------------------------------------------------------
// agent

agent::agent(agent_id_t id, agent_data& data, index_t index) : index_(index), data_(data), id(id) {}

static real_t* row(std::vector<real_t>& v, index_t index, index_t width) { return v.data() + (std::size_t)index * width; }

real_t* agent::secretion_rates() { return row(data_.secretion_rates, index_, data_.m.substrates_count); }
real_t* agent::saturation_densities() { return row(data_.saturation_densities, index_, data_.m.substrates_count); }
real_t* agent::uptake_rates() { return row(data_.uptake_rates, index_, data_.m.substrates_count); }
real_t* agent::net_export_rates() { return row(data_.net_export_rates, index_, data_.m.substrates_count); }
real_t* agent::internalized_substrates()
{
	return row(data_.internalized_substrates, index_, data_.m.substrates_count);
}
real_t* agent::fraction_released_at_death()
{
	return row(data_.fraction_released_at_death, index_, data_.m.substrates_count);
}
real_t* agent::fraction_transferred_when_ingested()
{
	return row(data_.fraction_transferred_when_ingested, index_, data_.m.substrates_count);
}

real_t& agent::volume() { return data_.volumes[index_]; }

real_t* agent::position() { return row(data_.positions, index_, data_.m.mesh.dims); }

point_t<real_t, 3> agent::get_position() const
{
	point_t<real_t, 3> p { 0, 0, 0 };
	const index_t dims = data_.m.mesh.dims;
	for (index_t d = 0; d < dims; d++)
		p[d] = data_.positions[(std::size_t)index_ * dims + d];
	return p;
}

point_t<index_t, 3> agent::voxel_index() const
{
	const auto p = get_position();
	switch (data_.m.mesh.dims)
	{
		case 1:
			return data_.m.mesh.voxel_position<1>(p.data());
		case 2:
			return data_.m.mesh.voxel_position<2>(p.data());
		default:
			return data_.m.mesh.voxel_position<3>(p.data());
	}
}

// linear voxel index x + X (y + Y z) of a voxel of the mesh
static std::size_t linear_voxel(const cartesian_mesh& mesh, point_t<index_t, 3> v)
{
	return (std::size_t)v[0] + (std::size_t)mesh.grid_shape[0] * ((std::size_t)v[1] + (std::size_t)mesh.grid_shape[1] * v[2]);
}

real_t* agent::nearest_density_vector()
{
	const microenvironment& m = data_.m;
	return m.substrate_densities.get() + linear_voxel(m.mesh, voxel_index()) * m.substrates_count;
}

point_t<real_t, 3> agent::nearest_gradient(index_t substrate_index) const
{
	// gradient layouts (src/traits.h:33-93): 1D [x][s][1], 2D [y][x][s][2], 3D [3][z][y][x][s]
	const microenvironment& m = data_.m;
	const std::size_t e = linear_voxel(m.mesh, voxel_index()) * m.substrates_count + substrate_index;
	const index_t dims = m.mesh.dims;
	point_t<real_t, 3> g { 0, 0, 0 };
	for (index_t d = 0; d < dims; d++)
		g[d] = dims == 3 ? m.gradients[(std::size_t)d * m.mesh.voxel_count() * m.substrates_count + e]
						 : m.gradients[e * dims + d];
	return g;
}

index_t agent::index() const { return index_; }

} // namespace biofvm
