// Host precompute of the tridiagonal coefficients for one sweep axis.
//
// The LOD step solves, along each axis of length n with voxel size h, the constant tridiagonal
// system  c x_{i-1} + b_i x_i + c x_{i+1} = d_i  with
//   c   = -dt*D/h^2
//   b_i = 1 + dt*lambda/dims + 2*dt*D/h^2   (interior)   and   1 + dt*lambda/dims + dt*D/h^2  (ends),
// and Thomas coefficients b'_0 = 1/b_0, b'_i = 1/(b_i - c^2 b'_{i-1}), e_{i-1} = c b'_{i-1}
// (paraBioFVM src/solver/host/diffusion_solver.cpp:72-142).  These are evaluated in float with the
// same operation order as the reference, so a line solved as a single block reproduces the
// reference's sequential Thomas bit for bit.
//
// Lines longer than one register block are split into P blocks.  Each block runs the Thomas
// recurrences locally and is corrected with carries from its neighbours:
//   forward   d'_i = f_i + g_i * d'_{p-1},  g_i = prod_{k=p-1}^{i-1} (-e_k)          (block start p)
//   backward  x_i  = t_i + G_i * x_{q+1},   G_i = prod_{k=i}^{q} (-c b'_k)           (block end q)
// where f and t are the block-local recurrences started from zero.  g and G are computed here in
// double precision and rounded once.

#include <algorithm>
#include <cmath>
#include <vector>

namespace bfvm {

void precompute_axis(int n, int h, int dims, int S, float dt, const float* D, const float* decay, int M,
					 std::vector<float>& bp, std::vector<float>& eprev, std::vector<float>& g, std::vector<float>& G,
					 std::vector<float>& c, std::vector<float>& gq, std::vector<float>& Gp, int& P, int& base_len,
					 int& extra)
{
	bp.assign((size_t)n * S, 0.f);
	eprev.assign((size_t)n * S, 0.f);
	g.assign((size_t)n * S, 0.f);
	G.assign((size_t)n * S, 0.f);
	c.assign(S, 0.f);

	if (n == 1)
	{
		// single voxel along the axis: only the decay part remains (diffusion_solver.cpp:76-85)
		for (int s = 0; s < S; s++)
			bp[s] = 1 / (1 + decay[s] * dt / dims);
		P = 1;
		base_len = 1;
		extra = 0;
		gq.assign(S, 0.f);
		Gp.assign(S, 0.f);
		return;
	}

	for (int s = 0; s < S; s++)
		c[s] = -dt * D[s] / (h * h);

	std::vector<float> b((size_t)n * S);
	for (int i : { 0, n - 1 })
		for (int s = 0; s < S; s++)
			b[(size_t)i * S + s] = 1 + decay[s] * dt / dims + dt * D[s] / (h * h);
	for (int i = 1; i < n - 1; i++)
		for (int s = 0; s < S; s++)
			b[(size_t)i * S + s] = 1 + decay[s] * dt / dims + 2 * dt * D[s] / (h * h);

	for (int s = 0; s < S; s++)
		bp[s] = 1 / b[s];
	for (int i = 1; i < n; i++)
		for (int s = 0; s < S; s++)
		{
			bp[(size_t)i * S + s] = 1 / (b[(size_t)i * S + s] - c[s] * c[s] * bp[(size_t)(i - 1) * S + s]);
			eprev[(size_t)i * S + s] = c[s] * bp[(size_t)(i - 1) * S + s];
		}

	// block partition: P blocks of base_len or base_len + 1 elements, at most M each
	P = (n + M - 1) / M;
	base_len = n / P;
	extra = n % P;

	// whole-block products used by the carry folds: gq[j] = g at the block end, Gp[j] = G at the
	// block start
	gq.assign((size_t)P * S, 0.f);
	Gp.assign((size_t)P * S, 0.f);
	for (int j = 0; j < P; j++)
	{
		const int p = j * base_len + std::min(j, extra);
		const int L = base_len + (j < extra ? 1 : 0);
		const int q = p + L - 1;
		for (int s = 0; s < S; s++)
		{
			if (j > 0)
			{
				double acc = 1.0;
				for (int i = p; i <= q; i++)
				{
					acc *= -(double)eprev[(size_t)i * S + s];
					g[(size_t)i * S + s] = (float)acc;
				}
				gq[(size_t)j * S + s] = (float)acc;
			}
			if (j < P - 1)
			{
				double acc = 1.0;
				for (int i = q; i >= p; i--)
				{
					acc *= -(double)c[s] * (double)bp[(size_t)i * S + s];
					G[(size_t)i * S + s] = (float)acc;
				}
				Gp[(size_t)j * S + s] = (float)acc;
			}
		}
	}
}

} // namespace bfvm
