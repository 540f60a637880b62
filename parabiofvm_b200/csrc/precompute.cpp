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

// Tables of the front-padded partition used by the staged sweeps (sweep_tma.cu).  The line is
// extended at its front by pad = 32 P - n virtual elements with b' = 0, so every one of the P
// blocks holds exactly 32 elements.  A virtual element has e = c * 0 = 0 and so couples nothing
// into the first real element: a line that fits one block still runs the reference's recurrences
// bit for bit, and longer lines need no per-element predicates.
//
// Each block first runs the forward and backward recurrences from zero carries (f, then t).  The
// backward substitution is linear, so the effect of the left carry C = d'_{p-1} on the block is
// the backward substitution tg of g, and the exact solution is
//   x_i = t_i + C tg_i + X G_i,    X = x_{q+1}.
// Layout, one float buffer that the kernels copy to shared memory as is (virtual index v < 32 P):
//   b' [32P][S] | (tg, G) pairs [32P][S][2] | c [S] | gq [P][S] | tgp [P][S] | Gp [P][S]
// with gq = g at each block end, tgp = tg and Gp = G at each block start.  g, tg and G are
// evaluated in double from the float b' and e = c b' and rounded once.
int padded_table_floats(int P, int S) { return 3 * 32 * P * S + S + 3 * P * S; }

void precompute_padded_range(int n, int i0, int i1, int S, const std::vector<float>& bp, const std::vector<float>& c,
							 int& P, int& pad, std::vector<float>& tab)
{
	const int nl = i1 - i0;
	P = (nl + 31) / 32;
	pad = 32 * P - nl;
	const int N = 32 * P;
	tab.assign((size_t)padded_table_floats(P, S), 0.f);
	float* vbp = tab.data();
	float* tgG = vbp + (size_t)N * S;
	float* ct = tgG + (size_t)2 * N * S;
	float* gq = ct + S;
	float* tgp = gq + (size_t)P * S;
	float* Gp = tgp + (size_t)P * S;
	for (int v = pad; v < N; v++)
		for (int s = 0; s < S; s++)
			vbp[(size_t)v * S + s] = bp[(size_t)(i0 + v - pad) * S + s];
	for (int s = 0; s < S; s++)
		ct[s] = c[s];
	const bool left_carry = i0 > 0, right_carry = i1 < n;
	if (P == 1 && !left_carry && !right_carry)
		return; // a single block uses no carries
	double gd[32];
	for (int j = 0; j < P; j++)
	{
		const int p = 32 * j, q = p + 31;
		for (int s = 0; s < S; s++)
		{
			const double cs = (double)c[s];
			if (j < P - 1 || right_carry)
			{
				// response to the right carry: G_v = prod_{m=v}^{q} (-c b'_m)
				double acc = 1.0;
				for (int v = q; v >= p; v--)
				{
					acc *= -cs * (double)vbp[(size_t)v * S + s];
					tgG[((size_t)v * S + s) * 2 + 1] = (float)acc;
				}
				Gp[(size_t)j * S + s] = (float)acc;
			}
			if (j > 0 || left_carry)
			{
				// forward response g_v = prod_{m=p-1}^{v-1} (-e_m), e_m = c b'_m the float product.  In
				// block 0 of a sub-line the carry enters at its first real element, v = pad, through
				// e of the element before the sub-line; the virtual elements before it stay 0.
				double acc = 1.0;
				for (int v = p; v <= q; v++)
				{
					if (v < pad)
					{
						gd[v - p] = 0.0;
						continue;
					}
					const float e = (j == 0 && v == pad) ? c[s] * bp[(size_t)(i0 - 1) * S + s]
														 : c[s] * vbp[(size_t)(v - 1) * S + s];
					acc *= -(double)e;
					gd[v - p] = acc;
				}
				gq[(size_t)j * S + s] = (float)acc;
				// tg: the backward substitution of g within the block
				double t = 0.0;
				for (int v = q; v >= p; v--)
				{
					const double b = (double)vbp[(size_t)v * S + s];
					t = (v == q) ? gd[v - p] * b : (gd[v - p] - cs * t) * b;
					tgG[((size_t)v * S + s) * 2] = (float)t;
				}
				tgp[(size_t)j * S + s] = (float)t;
			}
		}
	}
}

void precompute_padded(int n, int S, const std::vector<float>& bp, const std::vector<float>& c, int& P, int& pad,
					   std::vector<float>& tab)
{
	precompute_padded_range(n, 0, n, S, bp, c, P, pad, tab);
}

// Coefficients of the system that couples the slabs of a line split at bounds[0] = 0 < bounds[1] <
// ... < bounds[count] = n.  Slab k holds elements [i0, i1) and, solved from zero carries, yields A
// = its last forward value d'_{i1-1} and B = its first solution x_{i0}.  With the true carries C_k
// = d'_{i0-1} (left) and X_k = x_{i1} (right), both are linear:
//   d'_{i1-1} = A + Gamma C_k,   x_{i0} = B + beta C_k + Lambda X_k,
// so C_{k+1} = A_k + Gamma_k C_k from C_0 = 0, and X_{k-1} = B_k + beta_k C_k + Lambda_k X_k from
// X_{count-1} = 0.  out[k][3][S] = (Gamma, beta, Lambda), evaluated in double from the float b' and
// e = c b' of the whole line: Gamma = prod (-e), Lambda = prod (-c b'), and beta the Thomas solve
// of the slab for a unit left carry.  Terms without a neighbour are 0.
void slab_coefficients(int n, int S, const std::vector<float>& bp, const std::vector<float>& c, int count,
					   const int* bounds, std::vector<float>& out)
{
	out.assign((size_t)count * 3 * S, 0.f);
	std::vector<double> u;
	for (int k = 0; k < count; k++)
	{
		const int i0 = bounds[k], i1 = bounds[k + 1];
		for (int s = 0; s < S; s++)
		{
			const double cs = (double)c[s];
			auto b = [&](int i) { return (double)bp[(size_t)i * S + s]; };
			auto e = [&](int i) { return (double)(c[s] * bp[(size_t)i * S + s]); };
			float* o = out.data() + (size_t)k * 3 * S;
			if (i0 > 0)
			{
				// forward response of the slab to C = 1, then its backward substitution
				u.assign((size_t)(i1 - i0), 0.0);
				double acc = 1.0;
				for (int i = i0; i < i1; i++)
				{
					acc *= -e(i - 1);
					u[i - i0] = acc;
				}
				o[s] = (float)acc;
				double t = 0.0;
				for (int i = i1 - 1; i >= i0; i--)
					t = (i == i1 - 1) ? u[i - i0] * b(i) : (u[i - i0] - cs * t) * b(i);
				o[S + s] = (float)t;
			}
			if (i1 < n)
			{
				double acc = 1.0;
				for (int i = i1 - 1; i >= i0; i--)
					acc *= -cs * b(i);
				o[2 * S + s] = (float)acc;
			}
		}
	}
}

// Weights of the reduce pass of a z-slab holding elements [i0, i1) of lines of n elements
// (slab_reduce_kernel).  Solved from zero carries, the slab's last forward value A and its first
// solution B are linear in the slab's right-hand sides d_i:
//   A = sum_i alpha_i d_i,   alpha_i = prod_{m=i}^{i1-2} (-e_m),
//   B = sum_i omega_i d_i,   omega_{i1-1} = phi_{i1-1},  omega_i = phi_i - e_i omega_{i+1},
// with e = c b' (the float product) and phi_k = b'_k prod_{m=i0}^{k-1} (-c b'_m), the weight of the
// forward value f_k in the backward substitution's first element.  The weights shrink
// geometrically away from the end each sum belongs to, so the sums keep only the planes whose
// weights matter: planes are dropped from the far end while the dropped weights (the largest over
// the substrates, summed) stay at most 2^drop_log2 (2^-50 by default).  That moves A and B by at
// most that fraction of the line's largest |d|.  A is needed only below a neighbour (i1 < n), B only above one (i0 > 0); a sum not
// needed keeps no planes.
// Output w = alpha of planes [a_first, i1) as [na][S], then omega of planes [i0, i0 + nb) as
// [nb][S], evaluated in double from the float b' and e and rounded once.
void slab_reduce_weights(int n, int i0, int i1, int S, const std::vector<float>& bp, const std::vector<float>& c,
						 std::vector<float>& w, int& a_first, int& na, int& nb, int drop_log2)
{
	const int nl = i1 - i0;
	const double drop = std::ldexp(1.0, drop_log2);
	std::vector<double> alpha((size_t)nl * S), omega((size_t)nl * S), phi((size_t)nl);
	for (int s = 0; s < S; s++)
	{
		const double cs = (double)c[s];
		auto b = [&](int i) { return (double)bp[(size_t)i * S + s]; };
		auto e = [&](int i) { return (double)(c[s] * bp[(size_t)i * S + s]); };
		double acc = 1.0;
		for (int i = i1 - 1; i >= i0; i--)
		{
			alpha[(size_t)(i - i0) * S + s] = acc;
			if (i > i0)
				acc *= -e(i - 1);
		}
		double pr = 1.0;
		for (int k = i0; k < i1; k++)
		{
			phi[k - i0] = b(k) * pr;
			pr *= -cs * b(k);
		}
		double om = 0.0;
		for (int i = i1 - 1; i >= i0; i--)
		{
			om = (i == i1 - 1) ? phi[i - i0] : phi[i - i0] - e(i) * om;
			omega[(size_t)(i - i0) * S + s] = om;
		}
	}
	auto largest = [&](const std::vector<double>& v, int i) {
		double m = 0.0;
		for (int s = 0; s < S; s++)
			m = std::max(m, std::fabs(v[(size_t)(i - i0) * S + s]));
		return m;
	};
	a_first = i1;
	if (i1 < n)
	{
		double tail = 0.0;
		a_first = i0;
		for (int i = i0; i < i1; i++)
		{
			tail += largest(alpha, i);
			if (tail > drop)
				break;
			a_first = i + 1;
		}
	}
	na = i1 - a_first;
	int b_end = i0;
	if (i0 > 0)
	{
		double tail = 0.0;
		b_end = i1;
		for (int i = i1 - 1; i >= i0; i--)
		{
			tail += largest(omega, i);
			if (tail > drop)
				break;
			b_end = i;
		}
	}
	nb = b_end - i0;
	w.assign((size_t)(na + nb) * S, 0.f);
	for (int i = a_first; i < i1; i++)
		for (int s = 0; s < S; s++)
			w[(size_t)(i - a_first) * S + s] = (float)alpha[(size_t)(i - i0) * S + s];
	for (int i = i0; i < b_end; i++)
		for (int s = 0; s < S; s++)
			w[(size_t)(na + i - i0) * S + s] = (float)omega[(size_t)(i - i0) * S + s];
}

} // namespace bfvm
