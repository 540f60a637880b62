// Cartesian mesh (include/BioFVM/mesh.h, src/mesh.cpp:7-53 of the reference).
#pragma once

#include <cstddef>

#include "types.h"

namespace biofvm {

struct cartesian_mesh
{
	index_t dims; // 1, 2 or 3

	point_t<index_t, 3> bounding_box_mins;
	point_t<index_t, 3> bounding_box_maxs;
	point_t<index_t, 3> voxel_shape;
	point_t<index_t, 3> grid_shape; // ceil((max - min) / voxel) along used axes, 1 along the others

	cartesian_mesh(index_t dims, point_t<index_t, 3> bounding_box_mins, point_t<index_t, 3> bounding_box_maxs,
				   point_t<index_t, 3> voxel_shape);

	std::size_t voxel_count() const;
	// product of all three voxel edges, as in the reference
	index_t voxel_volume() const;

	// voxel holding `position` ([dims] reals): truncating (position - min) / voxel per used axis
	template <index_t dims_>
	point_t<index_t, 3> voxel_position(const real_t* position) const;

	point_t<real_t, 3> voxel_center(point_t<index_t, 3> position) const;

	void display_info();
};

} // namespace biofvm
