// Cases of the reference's tests written against the C++20 host API (parabiofvm_b200/host),
// the way a paraBioFVM user writes them: microenvironment_builder, agent container, solver.
// Each mode prints one JSON object; tests/test_cpp_facade.py checks it against the goldens of the
// reference's test/test.cpp or against the oracle.
//
//   facade_cases host       mesh, builder and agent-container behaviour (no GPU)
//   facade_cases uniform3d  one diffusion step of the uniform 3D case (test/test.cpp:98-113)
//   facade_cases step       steps with boundary and interior Dirichlet and agents, plus a release
//   facade_cases bulk       bulk supply/uptake from the builder's callbacks
//   facade_cases lifecycle_device / lifecycle_host
//                           agents released, removed and added between steps, on the GPU copy or
//                           through load/store round trips

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "BioFVM/agent_container_base.h"
#include "BioFVM/microenvironment.h"
#include "BioFVM/microenvironment_builder.h"
#include "BioFVM/solver.h"

using namespace biofvm;

// the reference's spellings of the solver types name the same classes
static_assert(std::is_same_v<solvers::device::solver, biofvm::solver>);
static_assert(std::is_same_v<solvers::device::cell_solver, biofvm::cell_solver>);

static void print_array(const char* name, const real_t* p, std::size_t n, bool last = false)
{
	std::printf("\"%s\": [", name);
	for (std::size_t i = 0; i < n; i++)
		std::printf(i ? ",%.9g" : "%.9g", (double)p[i]);
	std::printf("]%s", last ? "" : ", ");
}

static void print_ints(const char* name, const index_t* p, std::size_t n, bool last = false)
{
	std::printf("\"%s\": [", name);
	for (std::size_t i = 0; i < n; i++)
		std::printf(i ? ",%d" : "%d", p[i]);
	std::printf("]%s", last ? "" : ", ");
}

// test/utils.cpp default_microenv: 2 substrates, dt 5, D {4, 2}, decay {5, 3}, initial 1
static microenvironment default_microenv(cartesian_mesh mesh)
{
	microenvironment_builder b;
	b.set_name("test");
	b.set_time_step(5);
	b.resize(mesh.dims, mesh.bounding_box_mins, mesh.bounding_box_maxs, mesh.voxel_shape);
	b.add_density("first", "g/cm^3", 4, 5, 1);
	b.add_density("second", "g/cm^3", 2, 3, 1);
	return b.build();
}

static int mode_host()
{
	cartesian_mesh mesh(3, { 0, 0, 0 }, { 210, 100, 60 }, { 20, 20, 30 });

	microenvironment_builder b;
	b.resize(2, { 0, 0, 0 }, { 100, 60, 0 }, { 20, 20, 20 });
	b.add_density("a", "u", 1, 0.5f, 3);
	b.add_density("b", "u", 2, 0.25f, 4);
	b.add_boundary_dirichlet_conditions(1, { 7, 8, 9 }, { 10, 11, 12 }, { false, true, false }, { true, false, false });
	b.add_dirichlet_node({ 1, 2, 0 }, { 5, 6 }, { true, false });
	b.add_dirichlet_node({ 3, 1, 0 }, { 9, 10 });
	microenvironment m = b.build();

	// agents: create four, remove the second; the last one moves into its slot
	auto& agents = *m.agents;
	for (int i = 0; i < 4; i++)
	{
		agent* a = agents.create_agent();
		a->volume() = 100.f + i;
		a->position()[0] = 10.f * i + 1;
		a->position()[1] = 5.f * i + 2;
		a->secretion_rates()[0] = (real_t)i;
		a->secretion_rates()[1] = (real_t)(10 + i);
	}
	agents.remove_at(1);
	agent* moved = agents.get_agent_at(1);

	std::printf("{");
	print_ints("grid", mesh.grid_shape.data(), 3);
	std::printf("\"voxel_count\": %zu, \"voxel_volume\": %d, ", mesh.voxel_count(), mesh.voxel_volume());
	const point_t<real_t, 3> pos { 45.f, 59.f, 91.f };
	const auto vp = mesh.voxel_position<3>(pos.data());
	print_ints("voxel_position", vp.data(), 3);
	const auto vc = mesh.voxel_center({ 1, 2, 3 });
	print_array("voxel_center", vc.data(), 3);
	std::printf("\"grid2\": [%d,%d,%d], ", m.mesh.grid_shape[0], m.mesh.grid_shape[1], m.mesh.grid_shape[2]);
	std::printf("\"initial\": [%g,%g], ", m.substrate_densities[0], m.substrate_densities[1]);
	std::printf("\"faces\": [%d,%d,%d,%d], ", (int)!!m.dirichlet_min_boundary_values[0],
				(int)!!m.dirichlet_max_boundary_values[0], (int)!!m.dirichlet_min_boundary_values[1],
				(int)!!m.dirichlet_max_boundary_values[1]);
	std::printf("\"xmax_face\": [%g,%g,%d,%d], ", m.dirichlet_max_boundary_values[0][0],
				m.dirichlet_max_boundary_values[0][1], (int)m.dirichlet_max_boundary_conditions[0][0],
				(int)m.dirichlet_max_boundary_conditions[0][1]);
	std::printf("\"ymin_face\": [%g,%g,%d,%d], ", m.dirichlet_min_boundary_values[1][0],
				m.dirichlet_min_boundary_values[1][1], (int)m.dirichlet_min_boundary_conditions[1][0],
				(int)m.dirichlet_min_boundary_conditions[1][1]);
	print_ints("interior_voxels", m.dirichlet_interior_voxels.get(), 2 * m.dirichlet_interior_voxels_count);
	std::printf("\"interior_conditions\": [%d,%d,%d,%d], ", (int)m.dirichlet_interior_conditions[0],
				(int)m.dirichlet_interior_conditions[1], (int)m.dirichlet_interior_conditions[2],
				(int)m.dirichlet_interior_conditions[3]);
	std::printf("\"agents\": %d, \"moved_id\": %u, \"moved_index\": %d, \"moved_volume\": %g, ",
				agents.agents_count(), moved->id, moved->index(), moved->volume());
	print_array("moved_secretion", moved->secretion_rates(), 2);
	const auto vi = moved->voxel_index();
	print_ints("moved_voxel", vi.data(), 3);
	std::printf("\"host_resident\": %d", (int)(m.data_residency == solvers::data_residency::host));
	std::printf("}\n");
	return 0;
}

static int mode_uniform3d()
{
	auto m = default_microenv(cartesian_mesh(3, { 0, 0, 0 }, { 200, 200, 200 }, { 20, 20, 20 }));
	solver s;
	s.initialize(m);
	s.store_data_to_solver(m);
	s.diffusion.solve(m);
	s.load_data_from_solver(m);
	std::printf("{");
	print_array("densities", m.substrate_densities.get(), m.mesh.voxel_count() * m.substrates_count, true);
	std::printf("}\n");
	return 0;
}

// A small 3D scene with boundary and interior Dirichlet conditions and agents that share voxels,
// stepped like the reference driver (src/main.cpp:76-96), then one agent releases its
// internalized substrates.  The inputs are printed with the results so the test can rebuild the
// same scene for the oracle.
static microenvironment step_scene()
{
	microenvironment_builder b;
	b.set_time_step(0.01f);
	b.resize(3, { 0, 0, 0 }, { 120, 100, 80 }, { 20, 20, 20 });
	b.add_density("o2", "mmHg", 1000, 0.1f, 1);
	b.add_density("drug", "uM", 100, 0.5f, 0.5f);
	b.add_density("signal", "nM", 10, 1, 0);
	b.add_boundary_dirichlet_conditions(0, { 1, 0, 0 }, { 0, 0, 0 }, { true, false, false }, { false, false, false });
	b.add_boundary_dirichlet_conditions(2, { 0, 0, 0 }, { 0, 0, 2 }, { false, false, false }, { false, false, true });
	b.add_dirichlet_node({ 2, 2, 1 }, { 3, 4, 5 }, { true, false, true });
	b.add_dirichlet_node({ 4, 1, 2 }, { 6, 7, 8 });
	b.do_compute_internalized_substrates();
	microenvironment m = b.build();

	const index_t S = m.substrates_count;
	for (int i = 0; i < 40; i++)
	{
		agent* a = m.agents->create_agent();
		a->volume() = 500.f + 25.f * (i % 7);
		// positions on a coarse lattice so that several agents share a voxel
		a->position()[0] = 7.f + 13.f * (i % 9);
		a->position()[1] = 5.f + 11.f * (i % 8);
		a->position()[2] = 3.f + 19.f * (i % 4);
		for (index_t s = 0; s < S; s++)
		{
			a->secretion_rates()[s] = 0.5f * ((i + s) % 5);
			a->saturation_densities()[s] = 1.f + 0.25f * ((i * 3 + s) % 4);
			a->uptake_rates()[s] = 0.1f * ((i + 2 * s) % 6);
			a->net_export_rates()[s] = 0.01f * ((i + s) % 3);
			a->fraction_released_at_death()[s] = 0.2f * ((i + s) % 5);
		}
	}
	return m;
}

static int mode_step()
{
	microenvironment m = step_scene();
	const index_t S = m.substrates_count;
	solver s;
	s.initialize(m);
	s.store_data_to_solver(m);
	for (index_t step = 0; step < 3; step++)
	{
		s.diffusion.solve(m);
		s.gradient.solve(m);
		s.cell.simulate_secretion_and_uptake(m, step % 10 == 0);
	}
	s.cell.release_internalized_substrates(m, 5);
	s.load_data_from_solver(m);

	const agent_data& d = static_cast<const agent_container&>(*m.agents).data();
	const std::size_t AS = (std::size_t)d.agents_count * S;
	std::printf("{");
	print_array("secretion_rates", d.secretion_rates.data(), AS);
	print_array("saturation_densities", d.saturation_densities.data(), AS);
	print_array("uptake_rates", d.uptake_rates.data(), AS);
	print_array("net_export_rates", d.net_export_rates.data(), AS);
	print_array("fraction_released", d.fraction_released_at_death.data(), AS);
	print_array("volumes", d.volumes.data(), d.agents_count);
	print_array("positions", d.positions.data(), (std::size_t)d.agents_count * 3);
	print_ints("interior_voxels", m.dirichlet_interior_voxels.get(), 3 * m.dirichlet_interior_voxels_count);
	print_array("interior_values", m.dirichlet_interior_values.get(), (std::size_t)S * m.dirichlet_interior_voxels_count);
	std::vector<real_t> conds(S * m.dirichlet_interior_voxels_count);
	for (std::size_t i = 0; i < conds.size(); i++)
		conds[i] = m.dirichlet_interior_conditions[i] ? 1.f : 0.f;
	print_array("interior_conditions", conds.data(), conds.size());
	print_array("densities", m.substrate_densities.get(), m.mesh.voxel_count() * S);
	print_array("gradients", m.gradients.get(), 3 * m.mesh.voxel_count() * S);
	print_array("internalized", d.internalized_substrates.data(), AS, true);
	std::printf("}\n");
	return 0;
}

// Agents that die, appear and leave between steps, as a model's agent loop has them.  The host
// container does every change; the GPU copy follows either by cell.add_agents / cell.remove_agents
// (`on_device`) or by the reference's round trip, load_data_from_solver, the change, then
// store_data_to_solver.  Both must end identical.
static int mode_lifecycle(bool on_device)
{
	microenvironment m = step_scene();
	const index_t S = m.substrates_count;
	solver s;
	s.initialize(m);
	s.store_data_to_solver(m);
	auto steps = [&](index_t from, index_t to) {
		for (index_t step = from; step < to; step++)
		{
			s.diffusion.solve(m);
			s.gradient.solve(m);
			s.cell.simulate_secretion_and_uptake(m, step % 10 == 0);
		}
	};
	auto remove = [&](const std::vector<index_t>& indices) {
		if (!on_device)
			s.load_data_from_solver(m);
		for (index_t i : indices)
			m.agents->remove_at(i);
		if (on_device)
			s.cell.remove_agents(m, indices);
		else
			s.store_data_to_solver(m);
	};
	steps(0, 3);
	// agent 5 dies: it releases its internalized substrates and leaves
	s.cell.release_internalized_substrates(m, 5);
	remove({ 5 });
	steps(3, 5);
	// six agents appear, two of them in an occupied voxel
	if (!on_device)
		s.load_data_from_solver(m);
	const index_t first = m.agents->agents_count();
	for (int i = 0; i < 6; i++)
	{
		agent* a = m.agents->create_agent();
		a->volume() = 300.f + 50.f * i;
		a->position()[0] = i < 2 ? 7.f : 11.f + 17.f * i;
		a->position()[1] = i < 2 ? 5.f : 9.f + 13.f * i;
		a->position()[2] = 3.f + 12.f * i;
		for (index_t s2 = 0; s2 < S; s2++)
		{
			a->secretion_rates()[s2] = 0.3f * ((i + s2) % 4);
			a->saturation_densities()[s2] = 1.5f;
			a->uptake_rates()[s2] = 0.05f * (i + 1);
			a->net_export_rates()[s2] = 0.02f * s2;
			a->internalized_substrates()[s2] = 0.1f * i;
			a->fraction_released_at_death()[s2] = 0.5f;
		}
	}
	if (on_device)
		s.cell.add_agents(m, first, 6);
	else
		s.store_data_to_solver(m);
	steps(5, 8);
	// three agents leave at once: the first, one of the new ones, and the then-last
	remove({ 0, first + 2, m.agents->agents_count() - 3 });
	steps(8, 11);
	s.load_data_from_solver(m);

	const agent_data& d = static_cast<const agent_container&>(*m.agents).data();
	std::printf("{\"agents\": %d, ", d.agents_count);
	print_array("volumes", d.volumes.data(), d.agents_count);
	print_array("densities", m.substrate_densities.get(), m.mesh.voxel_count() * S);
	print_array("gradients", m.gradients.get(), 3 * m.mesh.voxel_count() * S);
	print_array("internalized", d.internalized_substrates.data(), (std::size_t)d.agents_count * S, true);
	std::printf("}\n");
	return 0;
}

// Bulk supply/uptake through the builder's callbacks (src/solver/host/bulk_solver.cpp): two
// steps on a 2D mesh with rates that depend on the voxel and the substrate.
static int mode_bulk()
{
	microenvironment_builder b;
	b.set_time_step(0.5f);
	b.resize(2, { 0, 0, 0 }, { 140, 100, 0 }, { 20, 20, 20 });
	b.add_density("a", "u", 10, 0.1f, 2);
	b.add_density("b", "u", 20, 0.2f, 0.5f);
	b.add_density("c", "u", 30, 0.3f, 0);
	b.set_bulk_functions(
		[](microenvironment& m, point_t<index_t, 3> v, real_t* out) {
			for (index_t s = 0; s < m.substrates_count; s++)
				out[s] = 0.1f * (real_t)(v[0] + 1) + 0.01f * (real_t)s;
		},
		[](microenvironment& m, point_t<index_t, 3> v, real_t* out) {
			for (index_t s = 0; s < m.substrates_count; s++)
				out[s] = 0.05f * (real_t)(v[1] + 1);
		},
		[](microenvironment& m, point_t<index_t, 3> v, real_t* out) {
			for (index_t s = 0; s < m.substrates_count; s++)
				out[s] = (real_t)(1 + v[0] + 2 * v[1] + s);
		});
	microenvironment m = b.build();
	solver sv;
	sv.initialize(m);
	sv.store_data_to_solver(m);
	sv.bulk.initialize(m);
	sv.bulk.solve(m);
	sv.bulk.solve(m);
	sv.load_data_from_solver(m);
	std::printf("{");
	print_array("densities", m.substrate_densities.get(), m.mesh.voxel_count() * m.substrates_count, true);
	std::printf("}\n");
	return 0;
}

int main(int argc, char** argv)
{
	const std::string mode = argc > 1 ? argv[1] : "host";
	try
	{
		if (mode == "host")
			return mode_host();
		if (mode == "uniform3d")
			return mode_uniform3d();
		if (mode == "step")
			return mode_step();
		if (mode == "bulk")
			return mode_bulk();
		if (mode == "lifecycle_device" || mode == "lifecycle_host")
			return mode_lifecycle(mode == "lifecycle_device");
	}
	catch (const std::exception& e)
	{
		std::fprintf(stderr, "error: %s\n", e.what());
		return 2;
	}
	std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
	return 1;
}
