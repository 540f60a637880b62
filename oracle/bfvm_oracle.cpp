// CPU oracle for the paraBioFVM microenvironment step -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++20 + OpenMP, the reference's host solvers for the per-step
// microenvironment update so that the CUDA path can be checked against it.  It is the parity
// checker and the timed CPU baseline; the product library never links, loads or calls it.
//
// Reference files restated here (paths relative to the asmelko/paraBioFVM project root):
//   mesh                 src/mesh.cpp:7-53                (grid shape, voxel volume, voxel position)
//   microenvironment     src/microenvironment.cpp:14-53  (initial densities)
//   layouts              src/traits.h:9-93                (density [z][y][x][s]; gradient layout per dims)
//   diffusion precompute src/solver/host/diffusion_solver.cpp:72-142
//   diffusion sweeps     src/solver/host/diffusion_solver.cpp:297-544
//   dirichlet            src/solver/host/dirichlet_solver.cpp:11-144
//   gradient             src/solver/host/gradient_solver.cpp:10-291
//   secretion/uptake     src/solver/host/cell_solver.cpp:15-373
//   step order           src/main.cpp:64-107
//
// The noarr-structures layout library used by the reference is not available, so its index maps
// are written out as explicit arithmetic.  The arithmetic of every update keeps the reference's
// operation order and association; build with -ffp-contract=off so no multiply-add is fused
// (the reference's default x86-64 build has no FMA either).
//
// Determinism: the reference's secretion ballot is a parallel compare-and-swap whose winner and
// summation order depend on thread timing (src/solver/host/cell_solver.cpp:98-134).  Run with
// one thread, the winner is the lowest agent index of each voxel and the sums run in agent
// index order.  This oracle always uses that single-thread order, whatever the thread count.

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

namespace {

template <typename real_t>
struct oracle_state
{
	// mesh (src/mesh.cpp:7-30)
	int dims;
	int bbox_min[3], bbox_max[3], voxel[3], grid[3];

	int S;
	real_t dt;
	std::vector<real_t> D, decay;

	std::vector<real_t> dens; // [z][y][x][s]
	std::vector<real_t> grad; // layout of src/traits.h gradient_layout per dims

	// Dirichlet (include/BioFVM/microenvironment.h:41-50)
	int n_interior = 0;
	bool interior_duplicates = false; // a voxel listed twice
	std::vector<int> interior_voxels;
	std::vector<real_t> interior_values;
	std::vector<uint8_t> interior_conds;
	bool has_min[3] = { false, false, false }, has_max[3] = { false, false, false };
	std::vector<real_t> min_vals[3], max_vals[3];
	std::vector<uint8_t> min_conds[3], max_conds[3];

	bool internalized = false;

	// agents (include/BioFVM/agent_data.h:14-24)
	int A = 0;
	std::vector<real_t> secretion, saturation, uptake, net_export, intern, frac_released, volumes, positions;

	// diffusion precompute (src/solver/host/diffusion_solver.h:40-44)
	std::vector<real_t> b[3], c[3], e[3];

	// cell solver state (src/solver/host/cell_solver.h:51-63)
	std::vector<real_t> numerators, denominators, factors;
	std::vector<real_t> red_num, red_den, red_fac;
	std::vector<int> ballots;
	bool is_conflict = false;

	std::size_t voxel_count() const { return (std::size_t)grid[0] * grid[1] * grid[2]; }
	int voxel_volume() const { return voxel[0] * voxel[1] * voxel[2]; } // src/mesh.cpp:32

	// src/mesh.cpp:35-53: truncating division, no bounds check
	void voxel_position(const real_t* pos, int out[3]) const
	{
		out[0] = out[1] = out[2] = 0;
		for (int d = 0; d < dims; d++)
			out[d] = (int)((pos[d] - bbox_min[d]) / voxel[d]);
	}

	std::size_t dens_index(int x, int y, int z, int s) const
	{
		return (((std::size_t)z * grid[1] + y) * grid[0] + x) * S + s;
	}
};

// ---------------------------------------------------------------------------------------------
// diffusion precompute: src/solver/host/diffusion_solver.cpp:72-142 (copies = 1: the substrate
// factor only duplicates identical values for vectorisation, so it never changes a result)
template <typename real_t>
void precompute_values(oracle_state<real_t>& m, int axis)
{
	const int n = m.grid[axis];
	const int shape = m.voxel[axis];
	const int dims = m.dims;
	auto& b = m.b[axis];
	auto& c = m.c[axis];
	auto& e = m.e[axis];

	if (n == 1)
	{
		b.assign(m.S, 0);
		for (int s = 0; s < m.S; s++)
			b[s] = 1 / (1 + m.decay[s] * m.dt / dims);
		c.clear();
		e.clear();
		return;
	}

	b.assign((std::size_t)n * m.S, 0);
	e.assign((std::size_t)(n - 1) * m.S, 0);
	c.assign(m.S, 0);

	for (int s = 0; s < m.S; s++)
		c[s] = -m.dt * m.D[s] / (shape * shape);

	for (int i : { 0, n - 1 })
		for (int s = 0; s < m.S; s++)
			b[(std::size_t)i * m.S + s] = 1 + m.decay[s] * m.dt / dims + m.dt * m.D[s] / (shape * shape);
	for (int i = 1; i < n - 1; i++)
		for (int s = 0; s < m.S; s++)
			b[(std::size_t)i * m.S + s] = 1 + m.decay[s] * m.dt / dims + 2 * m.dt * m.D[s] / (shape * shape);

	for (int s = 0; s < m.S; s++)
		b[s] = 1 / b[s];
	for (int i = 1; i < n; i++)
		for (int s = 0; s < m.S; s++)
		{
			b[(std::size_t)i * m.S + s] =
				1 / (b[(std::size_t)i * m.S + s] - c[s] * c[s] * b[(std::size_t)(i - 1) * m.S + s]);
			e[(std::size_t)(i - 1) * m.S + s] = c[s] * b[(std::size_t)(i - 1) * m.S + s];
		}
}

// ---------------------------------------------------------------------------------------------
// Dirichlet: src/solver/host/dirichlet_solver.cpp:11-144.  Faces in the order x-min, x-max,
// y-min, y-max, z-min, z-max, then interior voxels; a later write wins.
template <typename real_t>
void solve_boundary_face(oracle_state<real_t>& m, int axis, bool is_max)
{
	const auto& vals = is_max ? m.max_vals[axis] : m.min_vals[axis];
	const auto& conds = is_max ? m.max_conds[axis] : m.min_conds[axis];
	if (!(is_max ? m.has_max[axis] : m.has_min[axis]))
		return;

	const int fixed = is_max ? m.grid[axis] - 1 : 0;
	int lo[3] = { 0, 0, 0 }, hi[3] = { m.grid[0], m.grid[1], m.grid[2] };
	lo[axis] = fixed;
	hi[axis] = fixed + 1;

	// omp_trav_for_each distributes the outermost remaining dimension (include/BioFVM/omp_utils.h:6-12)
#pragma omp for collapse(2)
	for (int z = lo[2]; z < hi[2]; z++)
		for (int y = lo[1]; y < hi[1]; y++)
			for (int x = lo[0]; x < hi[0]; x++)
				for (int s = 0; s < m.S; s++)
					if (conds[s])
						m.dens[m.dens_index(x, y, z, s)] = vals[s];
}

template <typename real_t>
void apply_interior_entry(oracle_state<real_t>& m, int v)
{
	int idx[3] = { 0, 0, 0 };
	for (int d = 0; d < m.dims; d++)
		idx[d] = m.interior_voxels[(std::size_t)v * m.dims + d];
	for (int s = 0; s < m.S; s++)
		if (m.interior_conds[(std::size_t)v * m.S + s])
			m.dens[m.dens_index(idx[0], idx[1], idx[2], s)] = m.interior_values[(std::size_t)v * m.S + s];
}

template <typename real_t>
void solve_interior(oracle_state<real_t>& m)
{
	if (m.n_interior == 0)
		return;
	if (m.interior_duplicates)
	{
		// The reference distributes the list over threads (dirichlet_solver.cpp:63), so two entries
		// for one voxel race; in list order the later entry wins, as with one thread.
#pragma omp single
		for (int v = 0; v < m.n_interior; v++)
			apply_interior_entry(m, v);
		return;
	}
#pragma omp for
	for (int v = 0; v < m.n_interior; v++)
	{
		int idx[3] = { 0, 0, 0 };
		for (int d = 0; d < m.dims; d++)
			idx[d] = m.interior_voxels[(std::size_t)v * m.dims + d];
		for (int s = 0; s < m.S; s++)
			if (m.interior_conds[(std::size_t)v * m.S + s])
				m.dens[m.dens_index(idx[0], idx[1], idx[2], s)] = m.interior_values[(std::size_t)v * m.S + s];
	}
}

template <typename real_t>
void dirichlet_solve(oracle_state<real_t>& m)
{
	for (int d = 0; d < m.dims; d++)
	{
		solve_boundary_face(m, d, false);
		solve_boundary_face(m, d, true);
	}
	solve_interior(m);
}

// ---------------------------------------------------------------------------------------------
// Thomas sweeps: src/solver/host/diffusion_solver.cpp:297-480.
// A line of n elements with element stride `stride` starting at `base`, substrate s.

// x sweep of one row (solve_slice<'x'>, :297-334): the substrate loop is innermost
template <typename real_t>
void solve_row_x(real_t* __restrict__ row, const real_t* __restrict__ b, const real_t* __restrict__ c,
				 const real_t* __restrict__ e, int n, int S)
{
	for (int i = 1; i < n; i++)
		for (int s = 0; s < S; s++)
			row[(std::size_t)i * S + s] = row[(std::size_t)i * S + s] - e[(std::size_t)(i - 1) * S + s] * row[(std::size_t)(i - 1) * S + s];

	for (int s = 0; s < S; s++)
		row[(std::size_t)(n - 1) * S + s] = row[(std::size_t)(n - 1) * S + s] * b[(std::size_t)(n - 1) * S + s];

	for (int i = n - 2; i >= 0; i--)
		for (int s = 0; s < S; s++)
			row[(std::size_t)i * S + s] =
				(row[(std::size_t)i * S + s] - c[s] * row[(std::size_t)(i + 1) * S + s]) * b[(std::size_t)i * S + s];
}

// y/z sweep of a plane of lines (solve_slice_yz, :378-414): the merged x*s plane is innermost;
// element (i, q) of the plane sits at base[i * stride + q], q = x*S + s.
template <typename real_t>
void solve_plane_yz(real_t* __restrict__ base, const real_t* __restrict__ b, const real_t* __restrict__ c,
					const real_t* __restrict__ e, int n, std::size_t stride, int XS, int S)
{
	for (int i = 1; i < n; i++)
		for (int q = 0; q < XS; q++)
		{
			const int s = q % S;
			base[i * stride + q] = base[i * stride + q] - e[(std::size_t)(i - 1) * S + s] * base[(i - 1) * stride + q];
		}
	for (int q = 0; q < XS; q++)
	{
		const int s = q % S;
		base[(n - 1) * stride + q] = base[(n - 1) * stride + q] * b[(std::size_t)(n - 1) * S + s];
	}
	for (int i = n - 2; i >= 0; i--)
		for (int q = 0; q < XS; q++)
		{
			const int s = q % S;
			base[i * stride + q] = (base[i * stride + q] - c[s] * base[(i + 1) * stride + q]) * b[(std::size_t)i * S + s];
		}
}

template <typename real_t>
void diffusion_solve(oracle_state<real_t>& m)
{
	const int X = m.grid[0], Y = m.grid[1], Z = m.grid[2], S = m.S;
	real_t* dens = m.dens.data();

	if (m.dims == 1)
	{
		// solve_1d (:482-491) with solve_slice_omp<'x'> (:336-376)
		dirichlet_solve(m);
		const real_t *b = m.b[0].data(), *c = m.c[0].data(), *e = m.e[0].data();
		const int n = X;
#pragma omp for
		for (int s = 0; s < S; s++)
			for (int i = 1; i < n; i++)
				dens[(std::size_t)i * S + s] = dens[(std::size_t)i * S + s] - e[(std::size_t)(i - 1) * S + s] * dens[(std::size_t)(i - 1) * S + s];
#pragma omp for
		for (int s = 0; s < S; s++)
			dens[(std::size_t)(n - 1) * S + s] = dens[(std::size_t)(n - 1) * S + s] * b[(std::size_t)(n - 1) * S + s];
#pragma omp for
		for (int s = 0; s < S; s++)
			for (int i = n - 2; i >= 0; i--)
				dens[(std::size_t)i * S + s] = (dens[(std::size_t)i * S + s] - c[s] * dens[(std::size_t)(i + 1) * S + s]) * b[(std::size_t)i * S + s];
		dirichlet_solve(m);
		return;
	}

	const std::size_t XS = (std::size_t)X * S;

	// x sweep (:519-527 for 3D, :500-502 for 2D)
	dirichlet_solve(m);
#pragma omp for collapse(2)
	for (int z = 0; z < Z; z++)
		for (int y = 0; y < Y; y++)
			solve_row_x(dens + ((std::size_t)z * Y + y) * XS, m.b[0].data(), m.c[0].data(), m.e[0].data(), X, S);
	dirichlet_solve(m);

	// y sweep: 3D uses an omp for over z of solve_slice_yz (:532-537); 2D uses solve_slice_yz_omp
	// (:507), parallel across the x*s plane.  The per-element arithmetic is the same in both.
	if (m.dims == 3)
	{
#pragma omp for
		for (int z = 0; z < Z; z++)
			solve_plane_yz(dens + (std::size_t)z * Y * XS, m.b[1].data(), m.c[1].data(), m.e[1].data(), Y, XS, (int)XS, S);
	}
	else
	{
		// chunks of whole substrate groups keep q % S aligned with the chunk start
		const int chunk = 64 * S;
		const int chunks = (int)((XS + chunk - 1) / chunk);
#pragma omp for
		for (int ch = 0; ch < chunks; ch++)
		{
			const int q0 = ch * chunk;
			const int width = (int)std::min<std::size_t>(chunk, XS - q0);
			solve_plane_yz(dens + q0, m.b[1].data(), m.c[1].data(), m.e[1].data(), Y, XS, width, S);
		}
	}
	dirichlet_solve(m);

	if (m.dims == 2)
		return;

	// z sweep: solve_slice_yz_omp<'z'> (:416-480) -- parallel over y inside every z step
	{
		const int n = Z;
		const std::size_t stride = (std::size_t)Y * XS;
		const real_t *b = m.b[2].data(), *c = m.c[2].data(), *e = m.e[2].data();
		for (int i = 1; i < n; i++)
		{
#pragma omp for nowait
			for (int y = 0; y < Y; y++)
			{
				real_t* row = dens + (std::size_t)y * XS;
				for (std::size_t q = 0; q < XS; q++)
				{
					const int s = (int)(q % S);
					row[i * stride + q] = row[i * stride + q] - e[(std::size_t)(i - 1) * S + s] * row[(i - 1) * stride + q];
				}
			}
		}
#pragma omp barrier
#pragma omp for
		for (int y = 0; y < Y; y++)
		{
			real_t* row = dens + (std::size_t)y * XS;
			for (std::size_t q = 0; q < XS; q++)
			{
				const int s = (int)(q % S);
				row[(n - 1) * stride + q] = row[(n - 1) * stride + q] * b[(std::size_t)(n - 1) * S + s];
			}
		}
		for (int i = n - 2; i >= 0; i--)
		{
#pragma omp for nowait
			for (int y = 0; y < Y; y++)
			{
				real_t* row = dens + (std::size_t)y * XS;
				for (std::size_t q = 0; q < XS; q++)
				{
					const int s = (int)(q % S);
					row[i * stride + q] = (row[i * stride + q] - c[s] * row[(i + 1) * stride + q]) * b[(std::size_t)i * S + s];
				}
			}
		}
#pragma omp barrier
	}
	dirichlet_solve(m);
}

// ---------------------------------------------------------------------------------------------
// gradient: src/solver/host/gradient_solver.cpp:10-291.  Factors are computed as float
// (1.f / h) even when real_t is double (:17-18).
//
// Gradient layout (src/traits.h): 1D [x][s][d=1]; 2D [y][x][s][d=2]; 3D [d=3][z][y][x][s].
template <typename real_t>
std::size_t grad_index(const oracle_state<real_t>& m, int d, int x, int y, int z, int s)
{
	if (m.dims == 3)
		return (std::size_t)d * m.voxel_count() * m.S + m.dens_index(x, y, z, s);
	return m.dens_index(x, y, z, s) * m.dims + d;
}

template <typename real_t>
void gradient_solve(oracle_state<real_t>& m)
{
	const int X = m.grid[0], Y = m.grid[1], Z = m.grid[2], S = m.S;
	const real_t* u = m.dens.data();
	real_t* g = m.grad.data();

	auto axis_grad = [&](int axis, int x, int y, int z, int s) -> real_t {
		const int n = m.grid[axis];
		const int h = m.voxel[axis];
		const real_t border_factor = 1.f / h;
		const real_t center_factor = 1.f / (h * 2);
		int pos[3] = { x, y, z };
		const int i = pos[axis];
		int lo[3] = { x, y, z }, hi[3] = { x, y, z };
		if (n == 1)
			return 0; // the reference reads out of bounds here; a single-voxel axis has no gradient
		if (i == 0)
		{
			hi[axis] = 1;
			lo[axis] = 0;
			return (u[m.dens_index(hi[0], hi[1], hi[2], s)] - u[m.dens_index(lo[0], lo[1], lo[2], s)]) * border_factor;
		}
		if (i == n - 1)
		{
			hi[axis] = n - 1;
			lo[axis] = n - 2;
			return (u[m.dens_index(hi[0], hi[1], hi[2], s)] - u[m.dens_index(lo[0], lo[1], lo[2], s)]) * border_factor;
		}
		hi[axis] = i + 1;
		lo[axis] = i - 1;
		return (u[m.dens_index(hi[0], hi[1], hi[2], s)] - u[m.dens_index(lo[0], lo[1], lo[2], s)]) * center_factor;
	};

#pragma omp for collapse(2)
	for (int z = 0; z < Z; z++)
		for (int y = 0; y < Y; y++)
			for (int x = 0; x < X; x++)
				for (int s = 0; s < S; s++)
					for (int d = 0; d < m.dims; d++)
						g[grad_index(m, d, x, y, z, s)] = axis_grad(d, x, y, z, s);
}

// ---------------------------------------------------------------------------------------------
// secretion / uptake: src/solver/host/cell_solver.cpp:15-373
template <typename real_t>
void cell_resize(oracle_state<real_t>& m)
{
	const std::size_t n = (std::size_t)m.A * m.S;
	m.numerators.assign(n, 0);
	m.denominators.assign(n, 0);
	m.factors.assign(n, 0);
	m.red_num.assign(n, 0);
	m.red_den.assign(n, 0);
	m.red_fac.assign(n, 0);
}

template <typename real_t>
std::size_t agent_voxel(const oracle_state<real_t>& m, int i)
{
	int idx[3];
	m.voxel_position(m.positions.data() + (std::size_t)i * m.dims, idx);
	return ((std::size_t)idx[2] * m.grid[1] + idx[1]) * m.grid[0] + idx[0];
}

template <typename real_t>
void cell_simulate(oracle_state<real_t>& m, bool recompute)
{
	const int S = m.S;
	const int A = m.A;

#pragma omp single
	if (recompute)
	{
		cell_resize(m);
		m.is_conflict = false;
	}

	if (recompute)
	{
		// compute_intermediates (:63-85)
		const real_t voxel_volume = m.voxel_volume();
		const real_t time_step = m.dt;
#pragma omp for
		for (int i = 0; i < A; i++)
			for (int s = 0; s < S; s++)
			{
				const std::size_t k = (std::size_t)i * S + s;
				m.numerators[k] = m.secretion[k] * m.saturation[k] * time_step * m.volumes[i] / voxel_volume;
				m.denominators[k] = (m.uptake[k] + m.secretion[k]) * time_step * m.volumes[i] / voxel_volume;
				m.factors[k] = m.net_export[k] * time_step / voxel_volume;
			}

		// clear_ballots (:35-61) + ballot_and_sum (:87-135) in single-thread order
#pragma omp single
		{
			for (int i = 0; i < A; i++)
			{
				m.ballots[agent_voxel(m, i)] = -1;
				for (int s = 0; s < S; s++)
				{
					m.red_num[(std::size_t)i * S + s] = 0;
					m.red_den[(std::size_t)i * S + s] = 0;
					m.red_fac[(std::size_t)i * S + s] = 0;
				}
			}
			for (int i = 0; i < A; i++)
			{
				int& ballot = m.ballots[agent_voxel(m, i)];
				if (ballot == -1)
				{
					ballot = i;
					for (int s = 0; s < S; s++)
					{
						const std::size_t k = (std::size_t)i * S + s;
						m.red_num[k] += m.numerators[k];
						m.red_den[k] += m.denominators[k] + 1;
						m.red_fac[k] += m.factors[k];
					}
				}
				else
				{
					m.is_conflict = true;
					const int w = ballot;
					for (int s = 0; s < S; s++)
					{
						const std::size_t k = (std::size_t)i * S + s;
						const std::size_t kw = (std::size_t)w * S + s;
						m.red_num[kw] += m.numerators[k];
						m.red_den[kw] += m.denominators[k];
						m.red_fac[kw] += m.factors[k];
					}
				}
			}
		}
	}

	// compute_result (:197-245)
	const bool with_internalized = m.internalized;
	const bool is_conflict = m.is_conflict;
	real_t* dens = m.dens.data();

	if (with_internalized && !is_conflict)
	{
		// compute_fused (:173-195): the voxel volume stays an integer until it meets a real_t
		const int voxel_volume = m.voxel_volume();
#pragma omp for
		for (int i = 0; i < A; i++)
		{
			const std::size_t v = agent_voxel(m, i);
			for (int s = 0; s < S; s++)
			{
				const std::size_t k = (std::size_t)i * S + s;
				real_t& d = dens[v * S + s];
				m.intern[k] -= voxel_volume * (((1 - m.red_den[k]) * d + m.red_num[k]) / (m.red_den[k]) + m.red_fac[k]);
				d = (d + m.red_num[k]) / m.red_den[k] + m.red_fac[k];
			}
		}
		return;
	}

	if (with_internalized)
	{
		// compute_internalized (:137-152) with a real_t voxel volume
		const real_t voxel_volume = m.voxel_volume();
#pragma omp for
		for (int i = 0; i < A; i++)
		{
			const std::size_t v = agent_voxel(m, i);
			for (int s = 0; s < S; s++)
			{
				const std::size_t k = (std::size_t)i * S + s;
				m.intern[k] -= voxel_volume
							   * (((-m.denominators[k]) * dens[v * S + s] + m.numerators[k]) / (1 + m.denominators[k])
								  + m.factors[k]);
			}
		}
	}

	// compute_densities (:154-171) by the ballot winner
#pragma omp for
	for (int i = 0; i < A; i++)
	{
		const std::size_t v = agent_voxel(m, i);
		if (m.ballots[v] != i)
			continue;
		for (int s = 0; s < S; s++)
		{
			const std::size_t k = (std::size_t)i * S + s;
			dens[v * S + s] = (dens[v * S + s] + m.red_num[k]) / m.red_den[k] + m.red_fac[k];
		}
	}
}

// release_internalized_substrates (:301-346)
template <typename real_t>
void cell_release(oracle_state<real_t>& m, int index)
{
	if (!m.internalized)
		return;
	const real_t voxel_volume = m.voxel_volume();
	const std::size_t v = agent_voxel(m, index);
	for (int s = 0; s < m.S; s++)
	{
		const std::size_t k = (std::size_t)index * m.S + s;
		m.dens[v * m.S + s] += m.intern[k] * m.frac_released[k] / voxel_volume;
		m.intern[k] = 0;
	}
}

template <typename real_t>
oracle_state<real_t>* create(int dims, const int* bbox_min, const int* bbox_max, const int* voxel, int S, real_t dt,
							 const real_t* D, const real_t* decay, const real_t* initial, int internalized)
{
	auto m = std::make_unique<oracle_state<real_t>>();
	m->dims = dims;
	for (int d = 0; d < 3; d++)
	{
		m->bbox_min[d] = bbox_min[d];
		m->bbox_max[d] = bbox_max[d];
		m->voxel[d] = voxel[d];
		m->grid[d] = 1;
	}
	// src/mesh.cpp:11-25
	for (int d = 0; d < dims; d++)
		m->grid[d] = (bbox_max[d] - bbox_min[d] + voxel[d] - 1) / voxel[d];
	m->S = S;
	m->dt = dt;
	m->D.assign(D, D + S);
	m->decay.assign(decay, decay + S);
	m->internalized = internalized != 0;
	const std::size_t V = m->voxel_count();
	m->dens.resize(V * S);
	for (std::size_t v = 0; v < V; v++)
		for (int s = 0; s < S; s++)
			m->dens[v * S + s] = initial[s]; // src/microenvironment.cpp:14-25
	m->grad.assign(V * S * dims, 0);
	m->ballots.assign(V, 0); // value-initialised atomics (src/solver/host/cell_solver.cpp:372)
	return m.release();
}

template <typename real_t>
void initialize(oracle_state<real_t>& m)
{
	for (int d = 0; d < m.dims; d++)
		precompute_values(m, d);
	cell_resize(m);
}

template <typename real_t>
void set_agents(oracle_state<real_t>& m, int count, const real_t* sec, const real_t* sat, const real_t* upt,
				const real_t* nex, const real_t* intern, const real_t* frac, const real_t* vol, const real_t* pos)
{
	m.A = count;
	const std::size_t n = (std::size_t)count * m.S;
	m.secretion.assign(sec, sec + n);
	m.saturation.assign(sat, sat + n);
	m.uptake.assign(upt, upt + n);
	m.net_export.assign(nex, nex + n);
	m.intern.assign(intern, intern + n);
	m.frac_released.assign(frac, frac + n);
	m.volumes.assign(vol, vol + count);
	m.positions.assign(pos, pos + (std::size_t)count * m.dims);
}

// agent_data::add (src/agent_data.cpp:10-25) `count` times: every per-agent array grows by one row,
// value-initialised (0), and the caller's values then fill the new rows (the reference sets them
// through the agent afterwards); a null array leaves its rows at 0.
template <typename real_t>
void add_agents(oracle_state<real_t>& m, int count, const real_t* sec, const real_t* sat, const real_t* upt,
				const real_t* nex, const real_t* intern, const real_t* frac, const real_t* vol, const real_t* pos)
{
	const std::size_t S = (std::size_t)m.S, D = (std::size_t)m.dims, old = (std::size_t)m.A;
	auto grow = [&](std::vector<real_t>& v, std::size_t row, const real_t* src) {
		v.resize((old + count) * row, 0);
		if (src)
			std::copy(src, src + (std::size_t)count * row, v.begin() + old * row);
	};
	grow(m.secretion, S, sec);
	grow(m.saturation, S, sat);
	grow(m.uptake, S, upt);
	grow(m.net_export, S, nex);
	grow(m.intern, S, intern);
	grow(m.frac_released, S, frac);
	grow(m.volumes, 1, vol);
	grow(m.positions, D, pos);
	m.A += count;
}

// agent_data::remove (src/agent_data.cpp:27-53): the last agent's rows move into the freed slot.
template <typename real_t>
void remove_agent(oracle_state<real_t>& m, int index)
{
	m.A--;
	auto shrink = [&](std::vector<real_t>& v, std::size_t row) {
		if ((std::size_t)index != (std::size_t)m.A)
			std::copy(v.begin() + (std::size_t)m.A * row, v.begin() + ((std::size_t)m.A + 1) * row,
					  v.begin() + (std::size_t)index * row);
		v.resize((std::size_t)m.A * row);
	};
	const std::size_t S = (std::size_t)m.S;
	shrink(m.secretion, S);
	shrink(m.saturation, S);
	shrink(m.uptake, S);
	shrink(m.net_export, S);
	shrink(m.intern, S);
	shrink(m.frac_released, S);
	shrink(m.volumes, 1);
	shrink(m.positions, (std::size_t)m.dims);
}

// Bulk supply and uptake (src/solver/host/bulk_solver.cpp:20-33, solve_single), for every voxel:
//   D = (D + dt * S * T) / (1 + dt * (U + S))
// with the rates the reference's three callbacks return for the voxel, given here as tables:
// [voxel][s] when per_voxel, else one [s] row for every voxel.
template <typename real_t>
void bulk_solve(oracle_state<real_t>& m, const real_t* supply, const real_t* uptake, const real_t* target, int per_voxel)
{
	const std::size_t V = m.voxel_count();
	const int S = m.S;
	const real_t dt = m.dt;
#pragma omp for
	for (std::size_t v = 0; v < V; v++)
	{
		const std::size_t row = per_voxel ? v * S : 0;
		for (int s = 0; s < S; s++)
		{
			real_t& d = m.dens[v * S + s];
			d = (d + dt * supply[row + s] * target[row + s]) / (1 + dt * (uptake[row + s] + supply[row + s]));
		}
	}
}

template <typename real_t>
void run_steps(oracle_state<real_t>& m, int steps, int first_step)
{
	// src/main.cpp:68-107: one parallel region per step; diffusion -> gradient -> secretion
	for (int i = 0; i < steps; i++)
	{
		const bool recompute = ((first_step + i) % 10) == 0;
#pragma omp parallel
		{
			diffusion_solve(m);
			gradient_solve(m);
			cell_simulate(m, recompute);
		}
	}
}

} // namespace

#define ORACLE_EXPORTS(SUFFIX, T)                                                                                     \
	extern "C" void* oracle_##SUFFIX##_create(int dims, const int* bbox_min, const int* bbox_max, const int* voxel,    \
											   int S, T dt, const T* D, const T* decay, const T* initial,             \
											   int internalized)                                                      \
	{                                                                                                                  \
		return create<T>(dims, bbox_min, bbox_max, voxel, S, dt, D, decay, initial, internalized);                     \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_destroy(void* h) { delete static_cast<oracle_state<T>*>(h); }                    \
	extern "C" void oracle_##SUFFIX##_grid_shape(void* h, int* out)                                                    \
	{                                                                                                                  \
		for (int d = 0; d < 3; d++)                                                                                    \
			out[d] = static_cast<oracle_state<T>*>(h)->grid[d];                                                        \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_set_boundary_dirichlet(void* h, int dim, int is_max, const T* values,           \
															  const uint8_t* conds)                                   \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		auto& has = is_max ? m.has_max[dim] : m.has_min[dim];                                                          \
		auto& vals = is_max ? m.max_vals[dim] : m.min_vals[dim];                                                       \
		auto& cs = is_max ? m.max_conds[dim] : m.min_conds[dim];                                                       \
		if (!values)                                                                                                   \
		{                                                                                                              \
			has = false;                                                                                               \
			vals.clear();                                                                                              \
			cs.clear();                                                                                                \
			return;                                                                                                    \
		}                                                                                                              \
		has = true;                                                                                                    \
		vals.assign(values, values + m.S);                                                                             \
		cs.assign(conds, conds + m.S);                                                                                 \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_set_interior_dirichlet(void* h, int count, const int* voxels, const T* values,   \
															  const uint8_t* conds)                                   \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		m.n_interior = count;                                                                                          \
		m.interior_voxels.assign(voxels, voxels + (std::size_t)count * m.dims);                                        \
		{                                                                                                              \
			std::vector<long long> lin(count);                                                                         \
			for (int v = 0; v < count; v++)                                                                            \
			{                                                                                                          \
				long long key = 0;                                                                                     \
				for (int d = m.dims - 1; d >= 0; d--)                                                                  \
					key = key * m.grid[d] + voxels[(std::size_t)v * m.dims + d];                                       \
				lin[v] = key;                                                                                          \
			}                                                                                                          \
			std::sort(lin.begin(), lin.end());                                                                         \
			m.interior_duplicates = std::adjacent_find(lin.begin(), lin.end()) != lin.end();                           \
		}                                                                                                              \
		m.interior_values.assign(values, values + (std::size_t)count * m.S);                                           \
		m.interior_conds.assign(conds, conds + (std::size_t)count * m.S);                                              \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_initialize(void* h) { initialize(*static_cast<oracle_state<T>*>(h)); }           \
	extern "C" void oracle_##SUFFIX##_set_densities(void* h, const T* src)                                            \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		std::memcpy(m.dens.data(), src, m.dens.size() * sizeof(T));                                                    \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_get_densities(void* h, T* dst)                                                  \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		std::memcpy(dst, m.dens.data(), m.dens.size() * sizeof(T));                                                    \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_get_gradients(void* h, T* dst)                                                  \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		std::memcpy(dst, m.grad.data(), m.grad.size() * sizeof(T));                                                   \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_set_agents(void* h, int count, const T* sec, const T* sat, const T* upt,         \
												  const T* nex, const T* intern, const T* frac, const T* vol,          \
												  const T* pos)                                                        \
	{                                                                                                                  \
		set_agents(*static_cast<oracle_state<T>*>(h), count, sec, sat, upt, nex, intern, frac, vol, pos);              \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_add_agents(void* h, int count, const T* sec, const T* sat, const T* upt,         \
												  const T* nex, const T* intern, const T* frac, const T* vol,          \
												  const T* pos)                                                        \
	{                                                                                                                  \
		add_agents(*static_cast<oracle_state<T>*>(h), count, sec, sat, upt, nex, intern, frac, vol, pos);              \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_remove_agent(void* h, int index)                                                 \
	{                                                                                                                  \
		remove_agent(*static_cast<oracle_state<T>*>(h), index);                                                        \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_get_internalized(void* h, T* dst)                                               \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		std::memcpy(dst, m.intern.data(), m.intern.size() * sizeof(T));                                                \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_diffusion(void* h)                                                               \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		_Pragma("omp parallel") diffusion_solve(m);                                                                    \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_dirichlet(void* h)                                                               \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		_Pragma("omp parallel") dirichlet_solve(m);                                                                    \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_gradient(void* h)                                                                \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		_Pragma("omp parallel") gradient_solve(m);                                                                     \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_secretion(void* h, int recompute)                                                \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		_Pragma("omp parallel") cell_simulate(m, recompute != 0);                                                      \
	}                                                                                                                  \
	extern "C" void oracle_##SUFFIX##_release(void* h, int index) { cell_release(*static_cast<oracle_state<T>*>(h), index); } \
	extern "C" void oracle_##SUFFIX##_run_steps(void* h, int steps, int first_step)                                    \
	{                                                                                                                  \
		run_steps(*static_cast<oracle_state<T>*>(h), steps, first_step);                                               \
	}                                                                                                                  \
	extern "C" int oracle_##SUFFIX##_is_conflict(void* h) { return static_cast<oracle_state<T>*>(h)->is_conflict; } \
	extern "C" void oracle_##SUFFIX##_bulk(void* h, const T* supply, const T* uptake, const T* target, int per_voxel) \
	{                                                                                                                  \
		auto& m = *static_cast<oracle_state<T>*>(h);                                                                   \
		_Pragma("omp parallel") bulk_solve(m, supply, uptake, target, per_voxel);                                      \
	}

ORACLE_EXPORTS(f32, float)
ORACLE_EXPORTS(f64, double)

extern "C" void oracle_set_threads(int n)
{
	if (n > 0)
		omp_set_num_threads(n);
}

extern "C" int oracle_max_threads() { return omp_get_max_threads(); }
