// CPU ORACLE — test infrastructure only. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load this library, and only as the checker or
// the timed CPU baseline; the GPU product never links or calls it.
//
// A dependency-free C++17 restatement of PolyFEM's NeoHookean assembly path
// (iiiian/polyfem), following these reference files:
//   assembler/NeoHookeanElasticity.cpp:337-388   compute_energy_aux<double,n,3>
//   assembler/NeoHookeanElasticity.cpp:453-545   compute_energy_aux_gradient_fast<n,3>
//   assembler/NeoHookeanElasticity.cpp:547-658   compute_energy_hessian_aux_fast<n,3>
//   assembler/NeoHookeanElasticity.cpp:660-680   compute_stress_grad_multiply_mat
//   assembler/NeoHookeanElasticity.cpp:747-762   compute_dstress_dmu_dlambda
//   assembler/Assembler.cpp:495-771              NLAssembler energy/gradient/hessian loops
//   assembler/ElementAssemblyValues.cpp:65-104,164-237   geometry (J, det, J^-T)
//   assembler/AssemblyValsCache.cpp:52-67        per-element cache copy
//   utils/MatrixCache.cpp:88-228                 SparseMatrixCache (triplets -> CSC, slot map)
//   utils/par_for.cpp:10-31                      contiguous std::thread split
//   optimization/force_derivatives/ElasticForceDerivative.cpp:91-132,207-260
//   io/Evaluator.cpp:727-757                     interpolate_at_local_vals
//   quadrature/{Tet,Hex,Line}Quadrature.cpp, autogen/auto_tetrahedron.ipp,
//   autogen/auto_p_bases.cpp:1101-1306, autogen/auto_q_bases_3d_grad_1.cpp:7-53
//
// Parity status: the reference cannot be built here (no Eigen/oneTBB), so no
// vectors produced by the reference itself exist.  This oracle is pinned by the
// reference's own known-answer test for SparseMatrixCache (tests/test_matrix.cpp:
// 202-249, restated), by its autodiff-equality and finite-difference test
// methods (tests/test_assembler.cpp:127-286, tests/test_form_derivatives.cpp:
// 166-226) applied to this code, and by closed-form known answers of the
// NeoHookean law.  Eigen's summation order inside small products is not
// reproduced, so agreement with the reference is expected to ~1e-15 relative,
// not bit-for-bit.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace orc
{
enum ElemType
{
	P1_TET = 1,
	P2_TET = 2,
	Q1_HEX = 3
};

constexpr int MAXN = 10;
constexpr int MAXQ = 8;

// ---------------------------------------------------------------------------
// Reference-element tables: quadrature and basis gradients
// ---------------------------------------------------------------------------

// P2 tetrahedron gradients (autogen/auto_p_bases.cpp:1248-1306)
static void p2_grad(int i, double x, double y, double z, double *g)
{
	switch (i)
	{
	case 0: g[0] = 4 * x + 4 * y + 4 * z - 3; g[1] = 4 * x + 4 * y + 4 * z - 3; g[2] = 4 * x + 4 * y + 4 * z - 3; break;
	case 1: g[0] = 4 * x - 1; g[1] = 0; g[2] = 0; break;
	case 2: g[0] = 0; g[1] = 4 * y - 1; g[2] = 0; break;
	case 3: g[0] = 0; g[1] = 0; g[2] = 4 * z - 1; break;
	case 4: g[0] = 4 * (-2 * x - y - z + 1); g[1] = -4 * x; g[2] = -4 * x; break;
	case 5: g[0] = 4 * y; g[1] = 4 * x; g[2] = 0; break;
	case 6: g[0] = -4 * y; g[1] = 4 * (-x - 2 * y - z + 1); g[2] = -4 * y; break;
	case 7: g[0] = -4 * z; g[1] = -4 * z; g[2] = 4 * (-x - y - 2 * z + 1); break;
	case 8: g[0] = 4 * z; g[1] = 0; g[2] = 4 * x; break;
	case 9: g[0] = 0; g[1] = 4 * z; g[2] = 4 * y; break;
	}
}

// P1 tetrahedron gradients (autogen/auto_p_bases.cpp:1101-1123)
static void p1_grad(int i, double, double, double, double *g)
{
	static const double t[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
	g[0] = t[i][0]; g[1] = t[i][1]; g[2] = t[i][2];
}

// Q1 hexahedron gradients (autogen/auto_q_bases_3d_grad_1.cpp:7-53)
static void q1_grad(int i, double x, double y, double z, double *g)
{
	switch (i)
	{
	case 0: g[0] = -1.0 * (y - 1) * (z - 1); g[1] = -1.0 * (x - 1) * (z - 1); g[2] = -1.0 * (x - 1) * (y - 1); break;
	case 1: g[0] = 1.0 * (y - 1) * (z - 1); g[1] = 1.0 * x * (z - 1); g[2] = 1.0 * x * (y - 1); break;
	case 2: g[0] = -1.0 * y * (z - 1); g[1] = -1.0 * x * (z - 1); g[2] = -1.0 * x * y; break;
	case 3: g[0] = 1.0 * y * (z - 1); g[1] = 1.0 * (x - 1) * (z - 1); g[2] = 1.0 * y * (x - 1); break;
	case 4: g[0] = 1.0 * z * (y - 1); g[1] = 1.0 * z * (x - 1); g[2] = 1.0 * (x - 1) * (y - 1); break;
	case 5: g[0] = -1.0 * z * (y - 1); g[1] = -1.0 * x * z; g[2] = -1.0 * x * (y - 1); break;
	case 6: g[0] = 1.0 * y * z; g[1] = 1.0 * x * z; g[2] = 1.0 * x * y; break;
	case 7: g[0] = -1.0 * y * z; g[1] = -1.0 * z * (x - 1); g[2] = -1.0 * y * (x - 1); break;
	}
}

struct Tables
{
	int type = 0, n = 0, ng = 0, nq = 0;
	double qp[MAXQ][3];
	double qw[MAXQ];
	double grad[MAXQ][MAXN][3];  // FE basis, reference coordinates
	double ggrad[MAXQ][MAXN][3]; // geometric basis, reference coordinates
};

static Tables make_tables(int type)
{
	Tables t;
	t.type = type;
	void (*fe)(int, double, double, double, double *) = nullptr;
	void (*ge)(int, double, double, double, double *) = nullptr;
	if (type == P1_TET)
	{
		// order 1: GrundmannMoeller(tet, 0), weights / 6 (TetQuadrature.cpp:43-55)
		t.n = 4; t.ng = 4; t.nq = 1;
		t.qp[0][0] = t.qp[0][1] = t.qp[0][2] = 0.25;
		t.qw[0] = 1.0 / 6.0;
		fe = p1_grad; ge = p1_grad;
	}
	else if (type == P2_TET)
	{
		// order 2: HammerMarloweStroud(1) (autogen/auto_tetrahedron.ipp:7-12)
		t.n = 10; t.ng = 4; t.nq = 4;
		const double a = 0.13819660112501053195188660538406111299991607666015625;
		const double b = 0.58541019662496840414434018384781666100025177001953125;
		const double P[4][3] = {{a, a, b}, {a, b, a}, {b, a, a}, {a, a, a}};
		for (int q = 0; q < 4; ++q)
		{
			for (int d = 0; d < 3; ++d) t.qp[q][d] = P[q][d];
			t.qw[q] = 0.25 / 6.0;
		}
		fe = p2_grad; ge = p1_grad;
	}
	else if (type == Q1_HEX)
	{
		// order 2 Gauss-Legendre on [0,1] (LineQuadrature.cpp:20-24, 4708-4740),
		// tensor product index (i*2+j)*2+k -> point (x_k, x_j, x_i) (HexQuadrature.cpp:17-44)
		t.n = 8; t.ng = 8; t.nq = 8;
		double x1[2] = {-0.57735026918962576450914878050195745564760175127012687601860232648397767230293334569371539558574952522520871380513556767665664836499965082627055183736479121617603107730076852735599160670036155830775501, 0.57735026918962576450914878050195745564760175127012687601860232648397767230293334569371539558574952522520871380513556767665664836499965082627055183736479121617603107730076852735599160670036155830775501};
		double w1[2] = {1.0, 1.0};
		double ws = 0;
		for (int i = 0; i < 2; ++i)
		{
			w1[i] /= 2;
			x1[i] /= 2;
			x1[i] += 0.5;
			ws += w1[i];
		}
		for (int i = 0; i < 2; ++i) w1[i] /= ws;
		for (int i = 0; i < 2; ++i)
			for (int j = 0; j < 2; ++j)
				for (int k = 0; k < 2; ++k)
				{
					const int idx = (i * 2 + j) * 2 + k;
					t.qp[idx][0] = x1[k]; t.qp[idx][1] = x1[j]; t.qp[idx][2] = x1[i];
					t.qw[idx] = w1[i] * w1[j] * w1[k];
				}
		fe = q1_grad; ge = q1_grad;
	}
	else
		throw std::runtime_error("unknown element type");
	for (int q = 0; q < t.nq; ++q)
	{
		for (int i = 0; i < t.n; ++i) fe(i, t.qp[q][0], t.qp[q][1], t.qp[q][2], t.grad[q][i]);
		for (int i = 0; i < t.ng; ++i) ge(i, t.qp[q][0], t.qp[q][1], t.qp[q][2], t.ggrad[q][i]);
	}
	return t;
}

// ---------------------------------------------------------------------------
// 3x3 helpers (row-major m[r][c])
// ---------------------------------------------------------------------------
struct M3
{
	double a[3][3];
};

static inline double det3(const M3 &m)
{
	// cofactor expansion along the first column
	return m.a[0][0] * (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1])
		 - m.a[1][0] * (m.a[0][1] * m.a[2][2] - m.a[0][2] * m.a[2][1])
		 + m.a[2][0] * (m.a[0][1] * m.a[1][2] - m.a[0][2] * m.a[1][1]);
}

static inline M3 inv3(const M3 &m)
{
	M3 r;
	const double d = det3(m);
	r.a[0][0] = (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) / d;
	r.a[0][1] = (m.a[0][2] * m.a[2][1] - m.a[0][1] * m.a[2][2]) / d;
	r.a[0][2] = (m.a[0][1] * m.a[1][2] - m.a[0][2] * m.a[1][1]) / d;
	r.a[1][0] = (m.a[1][2] * m.a[2][0] - m.a[1][0] * m.a[2][2]) / d;
	r.a[1][1] = (m.a[0][0] * m.a[2][2] - m.a[0][2] * m.a[2][0]) / d;
	r.a[1][2] = (m.a[0][2] * m.a[1][0] - m.a[0][0] * m.a[1][2]) / d;
	r.a[2][0] = (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]) / d;
	r.a[2][1] = (m.a[0][1] * m.a[2][0] - m.a[0][0] * m.a[2][1]) / d;
	r.a[2][2] = (m.a[0][0] * m.a[1][1] - m.a[0][1] * m.a[1][0]) / d;
	return r;
}

static inline M3 transpose(const M3 &m)
{
	M3 r;
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) r.a[i][j] = m.a[j][i];
	return r;
}

// ---------------------------------------------------------------------------
// ElementAssemblyValues restatement
// ---------------------------------------------------------------------------
struct ElementValues
{
	int nq = 0, n = 0, ng = 0;
	int global[MAXN];
	int gglobal[MAXN];
	double det[MAXQ];
	double w[MAXQ];
	M3 jac_it[MAXQ];
	double grad[MAXQ][MAXN][3];      // reference gradients (AssemblyValues::grad)
	double grad_t_m[MAXQ][MAXN][3];  // physical gradients grad * jac_it
	double ggrad_t_m[MAXQ][MAXN][3]; // geometric-basis physical gradients (gvals)
};

// ElementAssemblyValues::compute + finalize3d (ElementAssemblyValues.cpp:65-104,164-237)
static void compute_values(const Tables &t, const int *conn, const int *gconn, const double *X, int e, ElementValues &v)
{
	v.nq = t.nq; v.n = t.n; v.ng = t.ng;
	for (int i = 0; i < t.n; ++i) v.global[i] = conn[(size_t)e * t.n + i];
	for (int i = 0; i < t.ng; ++i) v.gglobal[i] = gconn[(size_t)e * t.ng + i];
	for (int k = 0; k < t.nq; ++k)
	{
		M3 tmp;
		std::memset(&tmp, 0, sizeof(tmp));
		for (int j = 0; j < t.ng; ++j)
		{
			const double *node = X + (size_t)v.gglobal[j] * 3;
			for (int r = 0; r < 3; ++r)
				for (int c = 0; c < 3; ++c) tmp.a[r][c] += t.ggrad[k][j][r] * node[c];
		}
		v.det[k] = det3(tmp);
		v.w[k] = t.qw[k];
		v.jac_it[k] = transpose(inv3(tmp));
		for (int j = 0; j < t.n; ++j)
			for (int c = 0; c < 3; ++c)
			{
				v.grad[k][j][c] = t.grad[k][j][c];
				double s = 0;
				for (int r = 0; r < 3; ++r) s += t.grad[k][j][r] * v.jac_it[k].a[r][c];
				v.grad_t_m[k][j][c] = s;
			}
		for (int j = 0; j < t.ng; ++j)
			for (int c = 0; c < 3; ++c)
			{
				double s = 0;
				for (int r = 0; r < 3; ++r) s += t.ggrad[k][j][r] * v.jac_it[k].a[r][c];
				v.ggrad_t_m[k][j][c] = s;
			}
	}
}

// ---------------------------------------------------------------------------
// NeoHookean element kernels (NeoHookeanElasticity.cpp)
// ---------------------------------------------------------------------------
template <int N>
static double element_energy(const ElementValues &v, const double *x, double lambda, double mu)
{
	double local_disp[N][3];
	for (int i = 0; i < N; ++i)
		for (int d = 0; d < 3; ++d) local_disp[i][d] = x[(size_t)v.global[i] * 3 + d];
	double energy = 0;
	for (int p = 0; p < v.nq; ++p)
	{
		const double da = v.det[p] * v.w[p];
		// def_grad = (local_disp^T * grad) * jac_it + I
		M3 A;
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c)
			{
				double s = 0;
				for (int i = 0; i < N; ++i) s += local_disp[i][r] * v.grad[p][i][c];
				A.a[r][c] = s;
			}
		M3 F;
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c)
			{
				double s = 0;
				for (int k = 0; k < 3; ++k) s += A.a[r][k] * v.jac_it[p].a[k][c];
				F.a[r][c] = s + (r == c ? 1.0 : 0.0);
			}
		const double J = det3(F);
		const double log_det_j = std::log(J);
		double sq = 0;
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c) sq += F.a[r][c] * F.a[r][c];
		const double val = mu / 2 * (sq - 3 - 2 * log_det_j) + lambda / 2 * log_det_j * log_det_j;
		energy += val * da;
	}
	return energy;
}

static inline void cross(const double *x, const double *y, double *z)
{
	z[0] = x[1] * y[2] - x[2] * y[1];
	z[1] = x[2] * y[0] - x[0] * y[2];
	z[2] = x[0] * y[1] - x[1] * y[0];
}

// F = local_disp^T * delF_delU + I with delF_delU = grad * jac_it; returns delF_delU too.
template <int N>
static void def_grad_fast(const ElementValues &v, int p, const double (*local_disp)[3], double (*delF_delU)[3], M3 &F)
{
	for (int i = 0; i < N; ++i)
		for (int c = 0; c < 3; ++c)
		{
			double s = 0;
			for (int r = 0; r < 3; ++r) s += v.grad[p][i][r] * v.jac_it[p].a[r][c];
			delF_delU[i][c] = s;
		}
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			double s = 0;
			for (int i = 0; i < N; ++i) s += local_disp[i][r] * delF_delU[i][c];
			F.a[r][c] = s + (r == c ? 1.0 : 0.0);
		}
}

// delJ_delF columns: (v x w, w x u, u x v), u,v,w = columns of F
static inline void del_j_del_f(const M3 &F, M3 &D)
{
	double u[3] = {F.a[0][0], F.a[1][0], F.a[2][0]};
	double v[3] = {F.a[0][1], F.a[1][1], F.a[2][1]};
	double w[3] = {F.a[0][2], F.a[1][2], F.a[2][2]};
	double c0[3], c1[3], c2[3];
	cross(v, w, c0);
	cross(w, u, c1);
	cross(u, v, c2);
	for (int r = 0; r < 3; ++r)
	{
		D.a[r][0] = c0[r];
		D.a[r][1] = c1[r];
		D.a[r][2] = c2[r];
	}
}

template <int N>
static void element_gradient(const ElementValues &v, const double *x, double lambda, double mu, double *G_flat)
{
	double local_disp[N][3];
	for (int i = 0; i < N; ++i)
		for (int d = 0; d < 3; ++d) local_disp[i][d] = x[(size_t)v.global[i] * 3 + d];
	double G[N][3];
	std::memset(G, 0, sizeof(G));
	for (int p = 0; p < v.nq; ++p)
	{
		const double da = v.det[p] * v.w[p];
		double delF_delU[N][3];
		M3 F;
		def_grad_fast<N>(v, p, local_disp, delF_delU, F);
		const double J = det3(F);
		const double log_det_j = std::log(J);
		M3 D;
		del_j_del_f(F, D);
		M3 gt; // mu*F - mu*(1/J)*D + lambda*logJ*(1/J)*D
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c)
				gt.a[r][c] = mu * F.a[r][c] - mu * (1 / J) * D.a[r][c] + lambda * log_det_j * (1 / J) * D.a[r][c];
		// gradient = delF_delU * gt^T
		for (int i = 0; i < N; ++i)
			for (int d = 0; d < 3; ++d)
			{
				double s = 0;
				for (int k = 0; k < 3; ++k) s += delF_delU[i][k] * gt.a[d][k];
				G[i][d] += s * da;
			}
	}
	for (int i = 0; i < N; ++i)
		for (int d = 0; d < 3; ++d) G_flat[i * 3 + d] = G[i][d];
}

// Dense per-qp B^T C B, as written in the reference (H is 3N x 3N, row-major).
template <int N>
static void element_hessian(const ElementValues &v, const double *x, double lambda, double mu, double *H)
{
	constexpr int ND = 3 * N;
	double local_disp[N][3];
	for (int i = 0; i < N; ++i)
		for (int d = 0; d < 3; ++d) local_disp[i][d] = x[(size_t)v.global[i] * 3 + d];
	std::fill(H, H + ND * ND, 0.0);
	for (int p = 0; p < v.nq; ++p)
	{
		const double da = v.det[p] * v.w[p];
		double delF_delU[N][3];
		M3 F;
		def_grad_fast<N>(v, p, local_disp, delF_delU, F);
		const double J = det3(F);
		const double log_det_j = std::log(J);
		M3 D;
		del_j_del_f(F, D);
		double u[3] = {F.a[0][0], F.a[1][0], F.a[2][0]};
		double vv[3] = {F.a[0][1], F.a[1][1], F.a[2][1]};
		double w[3] = {F.a[0][2], F.a[1][2], F.a[2][2]};
		double d2[9][9];
		std::memset(d2, 0, sizeof(d2));
		// hat(x) = [[0,-x2,x1],[x2,0,-x0],[-x1,x0,0]] blocks (NeoHookeanElasticity.cpp:621-626)
		auto put_hat = [&](int r0, int c0, const double *xx, double s) {
			d2[r0 + 0][c0 + 1] += s * -xx[2];
			d2[r0 + 0][c0 + 2] += s * xx[1];
			d2[r0 + 1][c0 + 0] += s * xx[2];
			d2[r0 + 1][c0 + 2] += s * -xx[0];
			d2[r0 + 2][c0 + 0] += s * -xx[1];
			d2[r0 + 2][c0 + 1] += s * xx[0];
		};
		put_hat(0, 6, vv, 1.0);
		put_hat(6, 0, vv, -1.0);
		put_hat(0, 3, w, -1.0);
		put_hat(3, 0, w, 1.0);
		put_hat(3, 6, u, -1.0);
		put_hat(6, 3, u, 1.0);
		double g[9]; // column-major flattening of delJ_delF
		for (int c = 0; c < 3; ++c)
			for (int r = 0; r < 3; ++r) g[c * 3 + r] = D.a[r][c];
		const double c1 = (mu + lambda * (1 - log_det_j)) / (J * J);
		const double c2 = (lambda * log_det_j - mu) / (J);
		double C[9][9];
		for (int a = 0; a < 9; ++a)
			for (int b = 0; b < 9; ++b)
				C[a][b] = (a == b ? mu : 0.0) + c1 * (g[a] * g[b]) + c2 * d2[a][b];
		// B (9 x 3N): column i*3+j = vec_colmajor(E_j (x) delF_delU.row(i))
		static thread_local double B[9][3 * MAXN];
		for (int a = 0; a < 9; ++a)
			for (int b = 0; b < ND; ++b) B[a][b] = 0;
		for (int i = 0; i < N; ++i)
			for (int j = 0; j < 3; ++j)
				for (int k = 0; k < 3; ++k) B[k * 3 + j][i * 3 + j] = delF_delU[i][k];
		// (B^T C) B
		double BtC[3 * MAXN][9];
		for (int a = 0; a < ND; ++a)
			for (int b = 0; b < 9; ++b)
			{
				double s = 0;
				for (int k = 0; k < 9; ++k) s += B[k][a] * C[k][b];
				BtC[a][b] = s;
			}
		for (int a = 0; a < ND; ++a)
			for (int b = 0; b < ND; ++b)
			{
				double s = 0;
				for (int k = 0; k < 9; ++k) s += BtC[a][k] * B[k][b];
				H[a * ND + b] += s * da;
			}
	}
}

// ---------------------------------------------------------------------------
// SparseMatrixCache restatement (utils/MatrixCache.cpp:8-228, 289-322)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Other materials of the GenericElastic family (assembler/GenericElastic.hpp:93-130):
// energy = sum_q psi(F_q) da_q with F = I + grad u (real_def_grad, the default);
// gradient and Hessian with AutodiffType::STRESS (GenericElastic.hpp:70): dpsi/dF
// and d2psi/dF2 by second-order forward-mode dual numbers over the 9 entries of F
// (the reference's DScalar2 over def_grad, GenericElastic.cpp:502-511), contracted
// with the physical basis gradients.
//   MAT_ISO_NEOHOOKEAN: IsochoricNeoHookean::elastic_energy (IsochoricNeoHookean.hpp:19-33)
//   MAT_SAINT_VENANT  : SaintVenantElasticity::compute_energy_aux (SaintVenantElasticity.cpp:
//                       209-267) with the isotropic tensor of ElasticityTensor::set_from_lambda_mu
//                       (MatParams.cpp:211-260); per element (lambda, mu) here.
//   MAT_LINEAR_ELASTICITY: LinearElasticity::compute_energy_aux (LinearElasticity.cpp:113-139),
//                       differentiated over the nodal values there (gradient_from_energy /
//                       hessian_from_energy), over F here: the same derivatives, since F is
//                       linear in the nodal values.
//   MAT_MOONEY_RIVLIN : MooneyRivlinElasticity::elastic_energy (MooneyRivlinElasticity.hpp:25-46)
//   MAT_MOONEY_RIVLIN_3PARAM: MooneyRivlin3ParamElasticity::elastic_energy
//                       (MooneyRivlin3ParamElasticity.hpp:26-49)
//   MAT_VOLUME_PENALTY: VolumePenalty::elastic_energy (VolumePenalty.hpp:20-34)
//   MAT_HOOKE         : HookeLinearElasticity::compute_energy_aux (HookeLinearElasticity.cpp:
//                       372-421), one anisotropic tensor (orc_set_elasticity_tensor)
//   MAT_SAINT_VENANT_TENSOR: SaintVenantElasticity::compute_energy_aux with that tensor
// The material parameters of an element are prm[0..3]: (lambda, mu) for the first
// four, the GenericMatParam values for the others (orc_set_material_params).
// ---------------------------------------------------------------------------
enum
{
	MAT_NEOHOOKEAN = 0,
	MAT_ISO_NEOHOOKEAN = 1,
	MAT_SAINT_VENANT = 2,
	MAT_LINEAR_ELASTICITY = 3,
	MAT_MOONEY_RIVLIN = 4,
	MAT_MOONEY_RIVLIN_3PARAM = 5,
	MAT_VOLUME_PENALTY = 6,
	MAT_HOOKE = 7,
	MAT_SAINT_VENANT_TENSOR = 8,
	MAT_UNCONSTRAINED_OGDEN = 9,
	MAT_INCOMPRESSIBLE_OGDEN = 10,
	MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC = 11
};
constexpr int PRM_MAX = 21; // material parameters of an element: 21 tensor entries for MAT_HOOKE and
                            // MAT_SAINT_VENANT_TENSOR
constexpr int PRM_COUNT = PRM_MAX - 1; // the Ogden formulations: prm[PRM_COUNT] = number of values set

// value, gradient and Hessian with respect to the 9 entries F(r, c) (index 3r + c)
struct D2
{
	double v = 0, g[9] = {}, h[9][9] = {};
	D2() = default;
	D2(double x) : v(x) {}
	static D2 var(double x, int k)
	{
		D2 d(x);
		d.g[k] = 1.0;
		return d;
	}
};
static D2 operator+(const D2 &a, const D2 &b)
{
	D2 r(a.v + b.v);
	for (int i = 0; i < 9; ++i)
	{
		r.g[i] = a.g[i] + b.g[i];
		for (int j = 0; j < 9; ++j) r.h[i][j] = a.h[i][j] + b.h[i][j];
	}
	return r;
}
static D2 operator*(double s, const D2 &a)
{
	D2 r(s * a.v);
	for (int i = 0; i < 9; ++i)
	{
		r.g[i] = s * a.g[i];
		for (int j = 0; j < 9; ++j) r.h[i][j] = s * a.h[i][j];
	}
	return r;
}
static D2 operator-(const D2 &a, const D2 &b) { return a + (-1.0) * b; }
static D2 operator*(const D2 &a, const D2 &b)
{
	D2 r(a.v * b.v);
	for (int i = 0; i < 9; ++i)
	{
		r.g[i] = a.g[i] * b.v + a.v * b.g[i];
		for (int j = 0; j < 9; ++j)
			r.h[i][j] = a.h[i][j] * b.v + a.v * b.h[i][j] + a.g[i] * b.g[j] + b.g[i] * a.g[j];
	}
	return r;
}
// f(a) for a scalar function with f' = d1, f'' = d2 at a.v
static D2 chain(const D2 &a, double f, double d1, double d2)
{
	D2 r(f);
	for (int i = 0; i < 9; ++i)
	{
		r.g[i] = d1 * a.g[i];
		for (int j = 0; j < 9; ++j) r.h[i][j] = d1 * a.h[i][j] + d2 * a.g[i] * a.g[j];
	}
	return r;
}
static D2 dpow(const D2 &a, double p)
{
	return chain(a, std::pow(a.v, p), p * std::pow(a.v, p - 1), p * (p - 1) * std::pow(a.v, p - 2));
}
static D2 operator/(const D2 &a, const D2 &b) { return a * dpow(b, -1.0); }
static double dpow(double a, double p) { return std::pow(a, p); }
static D2 dlog(const D2 &a) { return chain(a, std::log(a.v), 1.0 / a.v, -1.0 / (a.v * a.v)); }
static double dlog(double a) { return std::log(a); }
static D2 dsqrt(const D2 &a)
{
	const double f = std::sqrt(a.v);
	return chain(a, f, 0.5 / f, -0.25 / (f * a.v));
}
static double dsqrt(double a) { return std::sqrt(a); }
static D2 dacos(const D2 &a)
{
	const double d = 1.0 - a.v * a.v;
	return chain(a, std::acos(a.v), -1.0 / std::sqrt(d), -a.v / (d * std::sqrt(d)));
}
static double dacos(double a) { return std::acos(a); }
static D2 dcos(const D2 &a) { return chain(a, std::cos(a.v), -std::sin(a.v), -std::cos(a.v)); }
static double dcos(double a) { return std::cos(a); }
static double dval(const D2 &a) { return a.v; }
static double dval(double a) { return a; }

template <class S>
static S det3s(const S (&F)[3][3])
{
	return F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
		   F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
}

// IsochoricNeoHookean: Cbar = F^T F / J^(2/3), psi = mu/2 (tr Cbar - 3)
template <class S>
static S psi_iso_neohookean(const S (&F)[3][3], double, double mu)
{
	const S J = det3s(F);
	const S jp = dpow(J, 2.0 / 3.0);
	S tr = S(0.0);
	for (int k = 0; k < 3; ++k)
		for (int i = 0; i < 3; ++i) tr = tr + F[i][k] * F[i][k] / jp; // (F^T F)(k,k) / J^(2/3)
	return (mu / 2.0) * (tr - S(3.0));
}

// SaintVenant: strain from the displacement gradient, Voigt strain with doubled
// shears, stress = C eps with C = [2mu+lambda, lambda, lambda; ...; mu, mu, mu],
// psi = 1/2 tr(stress * strain)
template <class S>
static S psi_saint_venant_tensor(const S (&F)[3][3], const double (&C)[6][6]);

template <class S>
static S psi_saint_venant(const S (&F)[3][3], double lambda, double mu)
{
	const double C[6][6] = {{2 * mu + lambda, lambda, lambda, 0, 0, 0}, {lambda, 2 * mu + lambda, lambda, 0, 0, 0},
							{lambda, lambda, 2 * mu + lambda, 0, 0, 0}, {0, 0, 0, mu, 0, 0},
							{0, 0, 0, 0, mu, 0},                       {0, 0, 0, 0, 0, mu}};
	return psi_saint_venant_tensor(F, C);
}

// SaintVenant with any elasticity tensor C (ElasticityTensor::set_from_entries):
// the Green strain of the displacement gradient, its Voigt form, stress = C eps
template <class S>
static S psi_saint_venant_tensor(const S (&F)[3][3], const double (&C)[6][6])
{
	S G[3][3], E[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) G[r][c] = F[r][c] - S(r == c ? 1.0 : 0.0);
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			S gtg = S(0.0);
			for (int k = 0; k < 3; ++k) gtg = gtg + G[k][r] * G[k][c];
			E[r][c] = 0.5 * (gtg + G[r][c] + G[c][r]);
		}
	const S eps[6] = {E[0][0], E[1][1], E[2][2], 2.0 * E[1][2], 2.0 * E[0][2], 2.0 * E[0][1]};
	S st[6];
	for (int j = 0; j < 6; ++j)
	{
		st[j] = C[j][0] * eps[0];
		for (int k = 1; k < 6; ++k) st[j] = st[j] + C[j][k] * eps[k];
	}
	const S sig[3][3] = {{st[0], st[5], st[4]}, {st[5], st[1], st[3]}, {st[4], st[3], st[2]}};
	S tr = S(0.0);
	for (int r = 0; r < 3; ++r)
		for (int k = 0; k < 3; ++k) tr = tr + sig[r][k] * E[k][r];
	return 0.5 * tr;
}

// LinearElasticity: strain = (G + G^T) / 2 of the displacement gradient G = F - I,
// psi = mu tr(strain^T strain) + lambda/2 tr(strain)^2
template <class S>
static S psi_linear_elasticity(const S (&F)[3][3], double lambda, double mu)
{
	S eps[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
			eps[r][c] = 0.5 * ((F[r][c] - S(r == c ? 1.0 : 0.0)) + (F[c][r] - S(r == c ? 1.0 : 0.0)));
	S ee = S(0.0), tr = S(0.0);
	for (int r = 0; r < 3; ++r)
	{
		tr = tr + eps[r][r];
		for (int k = 0; k < 3; ++k) ee = ee + eps[k][r] * eps[k][r]; // (strain^T strain)(r, r)
	}
	return mu * ee + (lambda / 2.0) * (tr * tr);
}

// tr(A) and (tr(A)^2 - tr(A A)) / 2 of a 3 x 3 matrix (first_invariant and
// second_invariant of utils/ElasticityUtils.hpp:140-149)
template <class S>
static void invariants12(const S (&A)[3][3], S &i1, S &i2)
{
	i1 = A[0][0] + A[1][1] + A[2][2];
	S trAA = S(0.0);
	for (int r = 0; r < 3; ++r)
		for (int k = 0; k < 3; ++k) trAA = trAA + A[r][k] * A[k][r];
	i2 = 0.5 * (i1 * i1 - trAA);
}

// MooneyRivlin: F~ = F / J^(1/3), C~ = F~ F~^T,
// psi = c1 (tr C~ - 3) + c2 (I2(C~) - 3) + k/2 ln^2 J
template <class S>
static S psi_mooney_rivlin(const S (&F)[3][3], double c1, double c2, double k)
{
	const S J = det3s(F);
	const S lj = dlog(J);
	const S s = dpow(J, -1.0 / 3.0);
	S Ft[3][3], Ct[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) Ft[r][c] = F[r][c] * s;
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			Ct[r][c] = S(0.0);
			for (int m = 0; m < 3; ++m) Ct[r][c] = Ct[r][c] + Ft[r][m] * Ft[c][m];
		}
	S i1, i2;
	invariants12(Ct, i1, i2);
	return c1 * (i1 - S(3.0)) + c2 * (i2 - S(3.0)) + (k / 2.0) * (lj * lj);
}

// MooneyRivlin3Param: B = F F^T, I1~ = J^(-2/3) tr B - 3, I2~ = J^(-4/3) I2(B) - 3,
// psi = c1 I1~ + (c2 + c3 I1~) I2~ + d1 (J - 1)^2
template <class S>
static S psi_mooney_rivlin_3param(const S (&F)[3][3], double c1, double c2, double c3, double d1)
{
	const S J = det3s(F);
	S B[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			B[r][c] = S(0.0);
			for (int m = 0; m < 3; ++m) B[r][c] = B[r][c] + F[r][m] * F[c][m];
		}
	const S pj = dpow(J, -2.0 / 3.0);
	S trB, i2;
	invariants12(B, trB, i2);
	const S I1t = pj * trB - S(3.0);
	const S I2t = (pj * pj) * i2 - S(3.0);
	const S jm = J - S(1.0);
	return c1 * I1t + (S(c2) + c3 * I1t) * I2t + d1 * (jm * jm);
}

// MooneyRivlin3ParamSymbolic (MooneyRivlin3ParamSymbolic.cpp:317-340): B = F F^T,
// I1~ = J^(-2/3) tr B, I2~ = J^(-4/3) I2(B),
// psi = c1 (I1~ - 3) + c2 (I2~ - 3) + c3 (I1~ - 3)(I2~ - 3) + d1 ln^2 J
template <class S>
static S psi_mooney_rivlin_3param_symbolic(const S (&F)[3][3], double c1, double c2, double c3, double d1)
{
	const S J = det3s(F);
	const S lj = dlog(J);
	S B[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			B[r][c] = S(0.0);
			for (int m = 0; m < 3; ++m) B[r][c] = B[r][c] + F[r][m] * F[c][m];
		}
	S trB, i2;
	invariants12(B, trB, i2);
	const S I1t = dpow(J, -2.0 / 3.0) * trB;
	const S I2t = dpow(J, -4.0 / 3.0) * i2;
	return c1 * (I1t - S(3.0)) + c2 * (I2t - S(3.0)) + c3 * ((I1t - S(3.0)) * (I2t - S(3.0))) + d1 * (lj * lj);
}

// VolumePenalty: psi = k/2 ((J^2 - 1)/2 - ln J)
template <class S>
static S psi_volume_penalty(const S (&F)[3][3], double k)
{
	const S J = det3s(F);
	return (k / 2.0) * (0.5 * (J * J - S(1.0)) - dlog(J));
}

// HookeLinearElasticity::compute_energy_aux (HookeLinearElasticity.cpp:372-421): the
// small strain of the displacement gradient G = F - I, its Voigt form with doubled
// shears, stress(j) = sum_k C(j, k) eps[k] (ElasticityTensor::compute_stress,
// MatParams.cpp:336-344, C(j, k) = C(k, j) read from the upper triangle), and
// psi = 1/2 tr(stress_tensor * strain).  c21: C(i, j), i <= j, row by row.
template <class S>
static S psi_hooke(const S (&F)[3][3], const double *c21)
{
	double C[6][6];
	for (int i = 0, k = 0; i < 6; ++i)
		for (int j = i; j < 6; ++j, ++k) C[i][j] = C[j][i] = c21[k];
	S E[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
			E[r][c] = 0.5 * ((F[r][c] - S(r == c ? 1.0 : 0.0)) + (F[c][r] - S(c == r ? 1.0 : 0.0)));
	const S eps[6] = {E[0][0], E[1][1], E[2][2], 2.0 * E[1][2], 2.0 * E[0][2], 2.0 * E[0][1]};
	S st[6];
	for (int j = 0; j < 6; ++j)
	{
		st[j] = S(0.0);
		for (int k = 0; k < 6; ++k) st[j] = st[j] + C[j][k] * eps[k];
	}
	const S sig[3][3] = {{st[0], st[5], st[4]}, {st[5], st[1], st[3]}, {st[4], st[3], st[2]}};
	S tr = S(0.0);
	for (int r = 0; r < 3; ++r)
		for (int k = 0; k < 3; ++k) tr = tr + sig[r][k] * E[k][r];
	return 0.5 * tr;
}

// utils::autogen::eigs_3d (autogen/auto_eigs.hpp:33-76): the eigenvalues of a symmetric
// 3 x 3 matrix by the trigonometric solution of its characteristic cubic, from the
// entries m(0,0), m(1,1), m(2,2), m(0,1), m(0,2), m(1,2); all three the trace / 3 when
// the deviator vanishes (below 1e-10), the arc cosine's argument clamped to [-1, 1].
template <class S>
static void eigs_3d(const S (&m)[3][3], S (&res)[3])
{
	const S t01 = m[0][0] + m[1][1];
	const S tr = t01 + m[2][2];
	const S off = m[0][1] * m[0][1] + m[0][2] * m[0][2] + m[1][2] * m[1][2];
	const S d02 = m[0][0] - m[2][2], d12 = m[1][1] - m[2][2], d01 = m[0][0] - m[1][1];
	// 9 p: three times the sum of squared off-diagonal entries plus half the squared diagonal differences
	const S p9 = 3.0 * off + 0.5 * (d02 * d02) + 0.5 * (d12 * d12) + 0.5 * (d01 * d01);
	const S sp9 = dsqrt(p9);
	if (2.0 * dval(sp9) < 1e-10)
	{
		res[0] = res[1] = res[2] = (1.0 / 3.0) * tr;
		return;
	}
	// 27 det(m - tr/3 I) / 2 over (9 p)^(3/2): the cosine of three times the angle
	const S num = -1.5 * (t01 * (m[0][0] + m[2][2]) * (m[1][1] + m[2][2])) + 4.5 * (tr * off) -
				  13.5 * (m[0][1] * m[0][1] * m[2][2]) - 13.5 * (m[0][2] * m[0][2] * m[1][1]) -
				  13.5 * (m[1][2] * m[1][2] * m[0][0]) + m[0][0] * m[0][0] * m[0][0] + 9.0 * (m[0][0] * m[1][1] * m[2][2]) +
				  27.0 * (m[0][1] * m[0][2] * m[1][2]) + m[1][1] * m[1][1] * m[1][1] + m[2][2] * m[2][2] * m[2][2];
	const S c3 = num / dpow(p9, 1.5);
	const S ang = (1.0 / 3.0) * (dval(c3) >= 1.0 ? S(0.0) : dval(c3) <= -1.0 ? S(M_PI) : dacos(c3));
	const S r = (2.0 / 3.0) * sp9, mean = (1.0 / 3.0) * tr;
	res[0] = r * dcos(ang) + mean;
	res[1] = r * dcos(ang + S(2.0 * M_PI / 3.0)) + mean;
	res[2] = r * dcos(ang - S(2.0 * M_PI / 3.0)) + mean;
}

// UnconstrainedOgden (OgdenElasticity.tpp:8-57): the principal stretches sqrt(eig(F^T F)),
// scaled by J^(-1/3), K terms (alpha_t, mu_t, D_t) in prm = alphas, mus, Ds:
//   psi = sum_t 2 mu_t / alpha_t^2 (sum_i s_i^alpha_t - 3) + sum_t (J - 1)^(2(t+1)) / D_t
template <class S>
static S psi_unconstrained_ogden(const S (&F)[3][3], const double *prm, int K)
{
	S C[3][3], ev[3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			C[r][c] = S(0.0);
			for (int k = 0; k < 3; ++k) C[r][c] = C[r][c] + F[k][r] * F[k][c];
		}
	eigs_3d(C, ev);
	for (int i = 0; i < 3; ++i) ev[i] = dsqrt(ev[i]);
	const S J = det3s(F);
	const S jd = dpow(J, -1.0 / 3.0);
	for (int i = 0; i < 3; ++i) ev[i] = ev[i] * jd;
	S val = S(0.0);
	for (int t = 0; t < K; ++t)
	{
		const double alpha = prm[t], mu = prm[K + t];
		S tmp = S(-3.0);
		for (int i = 0; i < 3; ++i) tmp = tmp + dpow(ev[i], alpha);
		val = val + (2.0 * mu / (alpha * alpha)) * tmp;
	}
	for (int t = 0; t < K; ++t) val = val + (1.0 / prm[2 * K + t]) * dpow(J - S(1.0), 2.0 * (t + 1));
	return val;
}

// IncompressibleOgden (OgdenElasticity.tpp:59-94): F~ = F / J^(1/3), the stretches
// sqrt(eig(F~ F~^T)), K terms (c_t, m_t) and k in prm = cs, ms, k:
//   psi = sum_t c_t / m_t^2 (sum_j s_j^m_t - 3) + k/2 ln^2 J
template <class S>
static S psi_incompressible_ogden(const S (&F)[3][3], const double *prm, int K)
{
	const S J = det3s(F);
	const S lj = dlog(J);
	const S s = dpow(J, 1.0 / 3.0);
	S Ft[3][3], Ct[3][3], ev[3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) Ft[r][c] = F[r][c] / s;
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			Ct[r][c] = S(0.0);
			for (int k = 0; k < 3; ++k) Ct[r][c] = Ct[r][c] + Ft[r][k] * Ft[c][k];
		}
	eigs_3d(Ct, ev);
	for (int i = 0; i < 3; ++i) ev[i] = dsqrt(ev[i]);
	S val = S(0.0);
	for (int t = 0; t < K; ++t)
	{
		const double c = prm[t], m = prm[K + t];
		S tmp = S(-3.0);
		for (int j = 0; j < 3; ++j) tmp = tmp + dpow(ev[j], m);
		val = val + (c / (m * m)) * tmp;
	}
	return val + (0.5 * prm[2 * K]) * (lj * lj);
}

template <class S>
static S psi_material(int mat, const S (&F)[3][3], const double *prm)
{
	switch (mat)
	{
	case MAT_HOOKE: return psi_hooke(F, prm);
	case MAT_SAINT_VENANT_TENSOR:
	{
		double C[6][6];
		for (int i = 0, k = 0; i < 6; ++i)
			for (int j = i; j < 6; ++j, ++k) C[i][j] = C[j][i] = prm[k];
		return psi_saint_venant_tensor(F, C);
	}
	case MAT_ISO_NEOHOOKEAN: return psi_iso_neohookean(F, prm[0], prm[1]);
	case MAT_SAINT_VENANT: return psi_saint_venant(F, prm[0], prm[1]);
	case MAT_LINEAR_ELASTICITY: return psi_linear_elasticity(F, prm[0], prm[1]);
	case MAT_MOONEY_RIVLIN: return psi_mooney_rivlin(F, prm[0], prm[1], prm[2]);
	case MAT_MOONEY_RIVLIN_3PARAM: return psi_mooney_rivlin_3param(F, prm[0], prm[1], prm[2], prm[3]);
	case MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC: return psi_mooney_rivlin_3param_symbolic(F, prm[0], prm[1], prm[2], prm[3]);
	case MAT_UNCONSTRAINED_OGDEN: return psi_unconstrained_ogden(F, prm, (int)prm[PRM_COUNT] / 3);
	case MAT_INCOMPRESSIBLE_OGDEN: return psi_incompressible_ogden(F, prm, ((int)prm[PRM_COUNT] - 1) / 2);
	default: return psi_volume_penalty(F, prm[0]);
	}
}

template <int N>
static void def_grad_plain(const ElementValues &v, const double *x, int p, double (&F)[3][3])
{
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c)
		{
			double s = 0;
			for (int i = 0; i < N; ++i) s += x[(size_t)v.global[i] * 3 + r] * v.grad_t_m[p][i][c];
			F[r][c] = s + (r == c ? 1.0 : 0.0);
		}
}

template <int N>
static double gen_element_energy(int mat, const ElementValues &v, const double *x, const double *prm)
{
	double energy = 0;
	for (int p = 0; p < v.nq; ++p)
	{
		double F[3][3];
		def_grad_plain<N>(v, x, p, F);
		energy += psi_material(mat, F, prm) * (v.det[p] * v.w[p]);
	}
	return energy;
}

// gradient (grad != nullptr, 3N) and Hessian (hess != nullptr, 3N x 3N row-major)
template <int N>
static void gen_element_derivatives(int mat, const ElementValues &v, const double *x, const double *prm, double *grad,
									double *hess)
{
	constexpr int ND = 3 * N;
	if (grad) std::fill(grad, grad + ND, 0.0);
	if (hess) std::fill(hess, hess + ND * ND, 0.0);
	for (int p = 0; p < v.nq; ++p)
	{
		double Fv[3][3];
		def_grad_plain<N>(v, x, p, Fv);
		D2 F[3][3];
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c) F[r][c] = D2::var(Fv[r][c], 3 * r + c);
		const D2 psi = psi_material(mat, F, prm);
		const double da = v.det[p] * v.w[p];
		const double(*g)[3] = v.grad_t_m[p];
		for (int i = 0; i < N; ++i)
			for (int r = 0; r < 3; ++r)
			{
				if (grad)
				{
					double s = 0;
					for (int c = 0; c < 3; ++c) s += psi.g[3 * r + c] * g[i][c];
					grad[i * 3 + r] += s * da;
				}
				if (hess)
					for (int j = 0; j < N; ++j)
						for (int t = 0; t < 3; ++t)
						{
							double s = 0;
							for (int c = 0; c < 3; ++c)
								for (int d = 0; d < 3; ++d) s += g[i][c] * psi.h[3 * r + c][3 * t + d] * g[j][d];
							hess[(i * 3 + r) * ND + j * 3 + t] += s * da;
						}
			}
	}
}

struct Triplet
{
	int r, c;
	double v;
};

struct CSC
{
	int rows = 0, cols = 0;
	std::vector<int> outer, inner;
	std::vector<double> values;
	size_t nnz() const { return inner.size(); }
	double coeff(int r, int c) const
	{
		const auto b = inner.begin() + outer[c], e = inner.begin() + outer[c + 1];
		auto it = std::lower_bound(b, e, r);
		if (it != e && *it == r) return values[it - inner.begin()];
		return 0.0;
	}
};

// Eigen::SparseMatrix::setFromTriplets: duplicates summed, inner indices sorted
static CSC csc_from_triplets(int rows, int cols, const std::vector<Triplet> &t)
{
	CSC m;
	m.rows = rows; m.cols = cols;
	std::vector<Triplet> s(t);
	std::stable_sort(s.begin(), s.end(), [](const Triplet &a, const Triplet &b) { return a.c != b.c ? a.c < b.c : a.r < b.r; });
	m.outer.assign(cols + 1, 0);
	for (size_t k = 0; k < s.size();)
	{
		size_t l = k;
		double v = 0;
		while (l < s.size() && s[l].c == s[k].c && s[l].r == s[k].r) v += s[l++].v;
		m.inner.push_back(s[k].r);
		m.values.push_back(v);
		m.outer[s[k].c + 1]++;
		k = l;
	}
	for (int c = 0; c < cols; ++c) m.outer[c + 1] += m.outer[c];
	return m;
}

// sparse + sparse keeps the union of stored entries (explicit zeros included)
static CSC csc_add(const CSC &a, const CSC &b)
{
	CSC m;
	m.rows = std::max(a.rows, b.rows);
	m.cols = std::max(a.cols, b.cols);
	m.outer.assign(m.cols + 1, 0);
	for (int c = 0; c < m.cols; ++c)
	{
		int ia = c < a.cols ? a.outer[c] : 0, ea = c < a.cols ? a.outer[c + 1] : 0;
		int ib = c < b.cols ? b.outer[c] : 0, eb = c < b.cols ? b.outer[c + 1] : 0;
		while (ia < ea || ib < eb)
		{
			if (ib >= eb || (ia < ea && a.inner[ia] < b.inner[ib]))
			{
				m.inner.push_back(a.inner[ia]); m.values.push_back(a.values[ia]); ++ia;
			}
			else if (ia >= ea || b.inner[ib] < a.inner[ia])
			{
				m.inner.push_back(b.inner[ib]); m.values.push_back(b.values[ib]); ++ib;
			}
			else
			{
				m.inner.push_back(a.inner[ia]); m.values.push_back(a.values[ia] + b.values[ib]); ++ia; ++ib;
			}
		}
		m.outer[c + 1] = (int)m.inner.size();
	}
	return m;
}

struct SparseMatrixCache
{
	size_t size_ = 0;
	CSC mat_;
	std::vector<Triplet> entries_;
	std::vector<std::vector<std::pair<int, size_t>>> mapping_;
	std::vector<int> inner_index_, outer_index_;
	std::vector<double> values_;
	const SparseMatrixCache *main_cache_ = nullptr;
	std::vector<std::vector<int>> second_cache_;
	std::vector<std::vector<std::pair<int, int>>> second_cache_entries_;
	int current_e_ = -1;
	int current_e_index_ = -1;

	const SparseMatrixCache *main_cache() const { return main_cache_ == nullptr ? this : main_cache_; }
	const std::vector<std::vector<std::pair<int, size_t>>> &mapping() const { return main_cache()->mapping_; }
	const std::vector<std::vector<int>> &second_cache() const { return main_cache()->second_cache_; }

	void init(size_t size)
	{
		size_ = size;
		mat_ = CSC();
		mat_.rows = mat_.cols = (int)size;
		mat_.outer.assign(size + 1, 0);
	}
	// init(other, copy_main_cache_ptr) (MatrixCache.cpp:56-77)
	void init(const SparseMatrixCache &other, bool copy_main_cache_ptr)
	{
		if (copy_main_cache_ptr)
			main_cache_ = other.main_cache_;
		else if (main_cache_ == nullptr)
			main_cache_ = other.main_cache();
		size_ = other.size_;
		values_.assign(other.values_.size(), 0.0);
		mat_ = CSC();
		mat_.rows = other.mat_.rows; mat_.cols = other.mat_.cols;
		mat_.outer.assign(mat_.cols + 1, 0);
	}
	void set_zero()
	{
		mat_.inner.clear(); mat_.values.clear();
		std::fill(mat_.outer.begin(), mat_.outer.end(), 0);
		std::fill(values_.begin(), values_.end(), 0.0);
	}
	void add_value(int e, int i, int j, double value)
	{
		if (mapping().empty())
		{
			entries_.push_back({i, j, value});
			if ((int)second_cache_entries_.size() <= e) second_cache_entries_.resize(e + 1);
			second_cache_entries_[e].emplace_back(i, j);
		}
		else
		{
			if (e != current_e_)
			{
				current_e_ = e;
				current_e_index_ = 0;
			}
			values_[second_cache()[e][current_e_index_]] += value;
			current_e_index_++;
		}
	}
	void prune()
	{
		if (mapping().empty())
		{
			CSC tmp = csc_from_triplets(mat_.rows, mat_.cols, entries_);
			mat_ = csc_add(mat_, tmp);
			entries_.clear();
		}
	}
	CSC get_matrix(bool compute_mapping = true)
	{
		prune();
		if (mapping().empty())
		{
			if (compute_mapping && size_ > 0)
			{
				values_.assign(mat_.nnz(), 0.0);
				inner_index_ = mat_.inner;
				outer_index_ = mat_.outer;
				mapping_.assign(mat_.rows, {});
				size_t index = 0;
				for (int i = 0; i < mat_.cols; ++i)
					for (int ii = outer_index_[i]; ii < outer_index_[i + 1]; ++ii)
						mapping_[inner_index_[ii]].emplace_back(i, index++);
				second_cache_.clear();
				second_cache_.resize(second_cache_entries_.size());
				for (size_t e = 0; e < second_cache_entries_.size(); ++e)
					for (const auto &p : second_cache_entries_[e])
					{
						const auto &map = mapping()[p.first];
						int idx = -1;
						for (const auto &q : map)
							if (q.first == p.second)
							{
								idx = (int)q.second;
								break;
							}
						if (idx < 0) throw std::runtime_error("slot not found");
						second_cache_[e].push_back(idx);
					}
				second_cache_entries_.resize(0);
			}
		}
		else
		{
			const SparseMatrixCache *mc = main_cache();
			mat_.rows = mat_.cols = (int)size_;
			mat_.outer = mc->outer_index_;
			mat_.inner = mc->inner_index_;
			mat_.values = values_;
			current_e_ = -1;
			current_e_index_ = -1;
		}
		std::fill(values_.begin(), values_.end(), 0.0);
		return mat_;
	}
	// operator+= (MatrixCache.cpp:289-322)
	void add_cache(const SparseMatrixCache &o, int n_threads);
};

static void par_for(int size, int n_threads, const std::function<void(int, int, int)> &func)
{
	if (n_threads <= 1)
	{
		func(0, size, 0);
		return;
	}
	std::vector<std::thread> threads(n_threads);
	for (int t = 0; t < n_threads; t++)
		threads[t] = std::thread(func, (int)((long long)t * size / n_threads),
								 (t + 1) == n_threads ? size : (int)((long long)(t + 1) * size / n_threads), t);
	for (auto &th : threads) th.join();
}

void SparseMatrixCache::add_cache(const SparseMatrixCache &o, int n_threads)
{
	if (mapping().empty() || o.mapping().empty())
	{
		mat_ = csc_add(mat_, o.mat_);
		const size_t this_e_size = second_cache_entries_.size();
		const size_t o_e_size = o.second_cache_entries_.size();
		second_cache_entries_.resize(std::max(this_e_size, o_e_size));
		for (size_t e = 0; e < o_e_size; ++e)
			second_cache_entries_[e].insert(second_cache_entries_[e].end(), o.second_cache_entries_[e].begin(), o.second_cache_entries_[e].end());
	}
	else
	{
		par_for((int)o.values_.size(), n_threads, [&](int s, int e, int) {
			for (int i = s; i < e; ++i) values_[i] += o.values_[i];
		});
	}
}

// ---------------------------------------------------------------------------
// Assembly context (NLAssembler + ElasticForm + ElasticForceDerivative)
// ---------------------------------------------------------------------------
struct Context
{
	Tables t;
	int E = 0, N = 0, Ng = 0;
	std::vector<int> conn, gconn;
	std::vector<double> X, lambda, mu;
	int n_threads = 1;
	bool use_cache = true;
	std::vector<ElementValues> cache; // AssemblyValsCache
	SparseMatrixCache mat_cache;
	bool fast_pattern = false; // build the first-call pattern by sorting instead of triplets
	bool project_psd = false;  // NLAssembler::assemble_hessian(project_to_psd = true)
	int material = 0;          // MAT_*: the assembler's formulation
	std::vector<double> mparams; // per-element parameters of the GenericMatParam materials, parameter-major
	double hooke[PRM_MAX] = {};  // MAT_HOOKE's elasticity tensor, 21 entries C(i, j), i <= j, row by row
	int n_mparams = 0;

	// the element's material parameters (lambda, mu) or GenericMatParam values
	void params(int e, double (&prm)[PRM_MAX]) const
	{
		for (int k = 0; k < PRM_MAX; ++k) prm[k] = 0.0;
		prm[0] = lambda[e];
		prm[1] = mu[e];
		if (material == MAT_HOOKE || material == MAT_SAINT_VENANT_TENSOR)
			for (int k = 0; k < PRM_MAX; ++k) prm[k] = hooke[k];
		else if (material >= MAT_MOONEY_RIVLIN)
		{
			for (int k = 0; k < 8; ++k) prm[k] = k < n_mparams ? mparams[(size_t)k * E + e] : 0.0;
			prm[PRM_COUNT] = n_mparams;
		}
	}
	CSC last;                  // last assembled Hessian
	CSC mass;                  // last assembled mass matrix
	std::string err;

	void vals(int e, ElementValues &v) const
	{
		if (cache.empty())
			compute_values(t, conn.data(), gconn.data(), X.data(), e, v);
		else
			v = cache[e];
	}
};

template <int N>
static double energy_impl(Context &c, const double *x, double *per_elem)
{
	std::vector<double> partial(c.n_threads, 0.0);
	par_for(c.E, c.n_threads, [&](int s, int e, int tid) {
		ElementValues v;
		double acc = 0;
		for (int el = s; el < e; ++el)
		{
			c.vals(el, v);
			double prm[PRM_MAX];
			c.params(el, prm);
			const double val = c.material ? gen_element_energy<N>(c.material, v, x, prm)
										  : element_energy<N>(v, x, c.lambda[el], c.mu[el]);
			if (per_elem) per_elem[el] = val;
			acc += val;
		}
		partial[tid] = acc;
	});
	double res = 0;
	for (double p : partial) res += p;
	return res;
}

template <int N>
static void gradient_impl(Context &c, const double *x, double *g)
{
	const size_t ndof = (size_t)c.N * 3;
	std::vector<std::vector<double>> local(c.n_threads);
	par_for(c.E, c.n_threads, [&](int s, int e, int tid) {
		local[tid].assign(ndof, 0.0);
		ElementValues v;
		double val[3 * N];
		for (int el = s; el < e; ++el)
		{
			c.vals(el, v);
			if (c.material)
			{
				double prm[PRM_MAX];
				c.params(el, prm);
				gen_element_derivatives<N>(c.material, v, x, prm, val, nullptr);
			}
			else
				element_gradient<N>(v, x, c.lambda[el], c.mu[el], val);
			for (int j = 0; j < N; ++j)
				for (int m = 0; m < 3; ++m) local[tid][(size_t)v.global[j] * 3 + m] += val[j * 3 + m];
		}
	});
	std::fill(g, g + ndof, 0.0);
	for (auto &l : local)
		if (!l.empty())
			for (size_t i = 0; i < ndof; ++i) g[i] += l[i];
}

// Fast first-call pattern: same CSC and slot order as the triplet path, built by sorting.
template <int N>
static void build_pattern_fast(Context &c)
{
	const int n = N;
	const int ndof = c.N * 3;
	// node adjacency
	std::vector<std::vector<int>> nbr(c.N);
	for (int e = 0; e < c.E; ++e)
		for (int a = 0; a < n; ++a)
			for (int b = 0; b < n; ++b) nbr[c.conn[(size_t)e * n + b]].push_back(c.conn[(size_t)e * n + a]);
	for (auto &v : nbr)
	{
		std::sort(v.begin(), v.end());
		v.erase(std::unique(v.begin(), v.end()), v.end());
	}
	SparseMatrixCache &mc = c.mat_cache;
	mc.outer_index_.assign(ndof + 1, 0);
	for (int B = 0; B < c.N; ++B)
		for (int nn = 0; nn < 3; ++nn) mc.outer_index_[3 * B + nn + 1] = mc.outer_index_[3 * B + nn] + 3 * (int)nbr[B].size();
	mc.inner_index_.resize(mc.outer_index_[ndof]);
	for (int B = 0; B < c.N; ++B)
		for (int nn = 0; nn < 3; ++nn)
		{
			int o = mc.outer_index_[3 * B + nn];
			for (int A : nbr[B])
				for (int m = 0; m < 3; ++m) mc.inner_index_[o++] = 3 * A + m;
		}
	mc.values_.assign(mc.inner_index_.size(), 0.0);
	mc.mapping_.assign(1, {{-1, 0}}); // marks the mapping as built; row lookups go through second_cache_
	mc.second_cache_.assign(c.E, {});
	for (int e = 0; e < c.E; ++e)
	{
		auto &sc = mc.second_cache_[e];
		sc.reserve((size_t)9 * n * n);
		const int *g = &c.conn[(size_t)e * n];
		for (int i = 0; i < n; ++i)
			for (int j = 0; j < n; ++j)
			{
				const auto &nb = nbr[g[j]];
				const int rank = (int)(std::lower_bound(nb.begin(), nb.end(), g[i]) - nb.begin());
				for (int nn = 0; nn < 3; ++nn)
					for (int m = 0; m < 3; ++m) sc.push_back(mc.outer_index_[3 * g[j] + nn] + 3 * rank + m);
			}
	}
}

// ---------------------------------------------------------------------------
// ipc::project_to_psd with the default PSDProjectionMethod::CLAMP, as called by
// NLAssembler::assemble_hessian (Assembler.cpp:693-694).  The function lives in
// ipc-toolkit (commit b40e9c0, cmake/recipes/ipc_toolkit.cmake:11), which is not
// part of the reference tree; its published algorithm is: eigendecompose the
// symmetric element matrix A = V diag(l) V^T (eigenvalues ascending); if the
// smallest eigenvalue is > 0 return A unchanged, else clamp every eigenvalue
// <= 0 to 0 and return V diag(l) V^T.  The projection onto the PSD cone is
// unique, so the eigensolver (Eigen's SelfAdjointEigenSolver there, cyclic
// Jacobi here) only changes rounding.
// ---------------------------------------------------------------------------
static void jacobi_eigen(std::vector<double> &A, int m, std::vector<double> &V, std::vector<double> &lam)
{
	V.assign((size_t)m * m, 0.0);
	for (int i = 0; i < m; ++i) V[(size_t)i * m + i] = 1.0;
	for (int sweep = 0; sweep < 60; ++sweep)
	{
		double off = 0.0, tot = 0.0;
		for (int i = 0; i < m; ++i)
			for (int j = 0; j < m; ++j)
			{
				const double a = A[(size_t)i * m + j];
				tot += a * a;
				if (i != j) off += a * a;
			}
		if (!(off > 1e-32 * tot)) break; // also stops on NaN
		for (int p = 0; p < m - 1; ++p)
			for (int q = p + 1; q < m; ++q)
			{
				const double apq = A[(size_t)p * m + q];
				if (apq == 0.0) continue;
				const double app = A[(size_t)p * m + p], aqq = A[(size_t)q * m + q];
				const double theta = (aqq - app) / (2.0 * apq);
				const double t = std::fabs(theta) > 1e100
									 ? 0.5 / theta
									 : (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
				const double cc = 1.0 / std::sqrt(t * t + 1.0), ss = t * cc;
				// A <- J^T A J with J = I except J_pp = J_qq = c, J_pq = s, J_qp = -s
				for (int k = 0; k < m; ++k)
				{
					const double akp = A[(size_t)k * m + p], akq = A[(size_t)k * m + q];
					A[(size_t)k * m + p] = cc * akp - ss * akq;
					A[(size_t)k * m + q] = ss * akp + cc * akq;
				}
				for (int k = 0; k < m; ++k)
				{
					const double apk = A[(size_t)p * m + k], aqk = A[(size_t)q * m + k];
					A[(size_t)p * m + k] = cc * apk - ss * aqk;
					A[(size_t)q * m + k] = ss * apk + cc * aqk;
				}
				A[(size_t)p * m + q] = A[(size_t)q * m + p] = 0.0;
				for (int k = 0; k < m; ++k)
				{
					const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
					V[(size_t)k * m + p] = cc * vkp - ss * vkq;
					V[(size_t)k * m + q] = ss * vkp + cc * vkq;
				}
			}
	}
	lam.resize(m);
	for (int i = 0; i < m; ++i) lam[i] = A[(size_t)i * m + i];
}

// In place on the row-major m x m symmetric matrix H.
static void project_to_psd(double *H, int m)
{
	std::vector<double> A(H, H + (size_t)m * m), V, lam;
	jacobi_eigen(A, m, V, lam);
	double lmin = lam[0];
	for (int i = 1; i < m; ++i) lmin = std::min(lmin, lam[i]);
	if (lmin > 0.0) return;
	if (std::isnan(lmin)) return; // NaN input propagates unchanged
	for (int i = 0; i < m; ++i)
		if (lam[i] <= 0.0) lam[i] = 0.0;
	for (int i = 0; i < m; ++i)
		for (int j = 0; j < m; ++j)
		{
			double s = 0.0;
			for (int k = 0; k < m; ++k) s += V[(size_t)i * m + k] * lam[k] * V[(size_t)j * m + k];
			H[(size_t)i * m + j] = s;
		}
}

template <int N>
static void hessian_impl(Context &c, const double *x)
{
	constexpr int ND = 3 * N;
	const int ndof = c.N * 3;
	SparseMatrixCache &mc = c.mat_cache;
	if (mc.mapping().empty() && c.fast_pattern) build_pattern_fast<N>(c);

	mc.init(ndof);
	mc.set_zero();
	std::vector<SparseMatrixCache> storage(c.n_threads);
	for (auto &s : storage)
	{
		s.main_cache_ = nullptr;
		s.init(mc, false);
	}
	par_for(c.E, c.n_threads, [&](int s, int e, int tid) {
		SparseMatrixCache &lc = storage[tid];
		ElementValues v;
		std::vector<double> H(ND * ND);
		for (int el = s; el < e; ++el)
		{
			c.vals(el, v);
			if (c.material)
			{
				double prm[PRM_MAX];
				c.params(el, prm);
				gen_element_derivatives<N>(c.material, v, x, prm, nullptr, H.data());
			}
			else
				element_hessian<N>(v, x, c.lambda[el], c.mu[el], H.data());
			if (c.project_psd) project_to_psd(H.data(), ND);
			for (int i = 0; i < N; ++i)
				for (int j = 0; j < N; ++j)
					for (int nn = 0; nn < 3; ++nn)
						for (int m = 0; m < 3; ++m)
						{
							lc.add_value(el, v.global[i] * 3 + m, v.global[j] * 3 + nn, H[(i * 3 + m) * ND + (j * 3 + nn)]);
							// max_triplets_size = 1e7 (Assembler.cpp:657,741-745)
							if (lc.entries_.size() >= 10000000) lc.prune();
						}
		}
	});
	for (auto &s : storage)
	{
		s.prune();
		mc.add_cache(s, c.n_threads);
	}
	c.last = mc.get_matrix();
}

// interpolate_at_local_vals gradient part (io/Evaluator.cpp:727-757): grad[q][d][k]
template <int N>
static void interp_grad(const ElementValues &v, const double *fun, double (*out)[3][3])
{
	for (int q = 0; q < v.nq; ++q)
		for (int d = 0; d < 3; ++d)
			for (int k = 0; k < 3; ++k) out[q][d][k] = 0;
	for (int i = 0; i < N; ++i)
		for (int d = 0; d < 3; ++d)
		{
			const double f = fun[(size_t)v.global[i] * 3 + d];
			for (int q = 0; q < v.nq; ++q)
				for (int k = 0; k < 3; ++k) out[q][d][k] += f * v.grad_t_m[q][i][k];
		}
}

template <int N>
static void material_vjp_impl(Context &c, const double *x, const double *adj, double *term)
{
	const int E = c.E;
	std::vector<std::vector<double>> local(c.n_threads);
	par_for(E, c.n_threads, [&](int s, int e, int tid) {
		local[tid].assign((size_t)2 * E, 0.0);
		ElementValues v;
		double gu[MAXQ][3][3], gp[MAXQ][3][3];
		for (int el = s; el < e; ++el)
		{
			c.vals(el, v);
			interp_grad<N>(v, x, gu);
			interp_grad<N>(v, adj, gp);
			for (int q = 0; q < v.nq; ++q)
			{
				const double da = v.det[q] * v.w[q];
				if (c.material == MAT_LINEAR_ELASTICITY)
				{
					// LinearElasticity::compute_dstress_dmu_dlambda (LinearElasticity.cpp:290-299):
					// dP/dmu = grad u + grad u^T, dP/dlambda = tr(grad u) I
					double imu = 0, tru = 0, trp = 0;
					for (int i = 0; i < 3; ++i)
					{
						tru += gu[q][i][i];
						trp += gp[q][i][i];
						for (int j = 0; j < 3; ++j) imu += (gu[q][i][j] + gu[q][j][i]) * gp[q][i][j];
					}
					local[tid][el + E] += -imu * da;
					local[tid][el] += -(tru * trp) * da;
					continue;
				}
				M3 F;
				for (int i = 0; i < 3; ++i)
					for (int j = 0; j < 3; ++j) F.a[i][j] = (i == j ? 1.0 : 0.0) + gu[q][i][j];
				const M3 FmT = transpose(inv3(F));
				const double lj = std::log(det3(F));
				double imu = 0, ila = 0;
				for (int i = 0; i < 3; ++i)
					for (int j = 0; j < 3; ++j)
					{
						imu += (F.a[i][j] - FmT.a[i][j]) * gp[q][i][j];
						ila += (lj * FmT.a[i][j]) * gp[q][i][j];
					}
				local[tid][el + E] += -imu * da;
				local[tid][el] += -ila * da;
			}
		}
	});
	std::fill(term, term + 2 * (size_t)E, 0.0);
	for (auto &l : local)
		if (!l.empty())
			for (size_t i = 0; i < l.size(); ++i) term[i] += l[i];
}

template <int N>
static void shape_vjp_impl(Context &c, const double *x, const double *adj, double *term)
{
	const size_t nout = (size_t)c.Ng * 3;
	std::vector<std::vector<double>> local(c.n_threads);
	par_for(c.E, c.n_threads, [&](int s, int e, int tid) {
		local[tid].assign(nout, 0.0);
		ElementValues v;
		double gu[MAXQ][3][3], gp[MAXQ][3][3];
		for (int el = s; el < e; ++el)
		{
			c.vals(el, v);
			interp_grad<N>(v, x, gu);
			interp_grad<N>(v, adj, gp);
			const double lambda = c.lambda[el], mu = c.mu[el];
			double prm[PRM_MAX];
			c.params(el, prm);
			for (int q = 0; q < v.nq; ++q)
			{
				const double da = v.det[q] * v.w[q];
				M3 F;
				for (int i = 0; i < 3; ++i)
					for (int j = 0; j < 3; ++j) F.a[i][j] = (i == j ? 1.0 : 0.0) + gu[q][i][j];
				if (c.material)
				{
					// the other formulations: P = dpsi/dF and C = d2psi/dF2 by dual numbers over F,
					// then compute_stress_grad_multiply_mat's C : (grad u V), as GenericElastic
					// evaluates it (GenericElastic.cpp:613-690)
					D2 Fd[3][3];
					for (int r = 0; r < 3; ++r)
						for (int cc = 0; cc < 3; ++cc) Fd[r][cc] = D2::var(F.a[r][cc], 3 * r + cc);
					const D2 psi = psi_material(c.material, Fd, prm);
					for (int vi = 0; vi < v.ng; ++vi)
						for (int d = 0; d < 3; ++d)
						{
							double V[3][3] = {}, Mm[3][3];
							for (int k = 0; k < 3; ++k) V[d][k] = v.ggrad_t_m[q][vi][k];
							for (int i = 0; i < 3; ++i)
								for (int j = 0; j < 3; ++j)
								{
									double s2 = 0;
									for (int k = 0; k < 3; ++k) s2 += gu[q][i][k] * V[k][j];
									Mm[i][j] = s2;
								}
							const double tr = V[0][0] + V[1][1] + V[2][2];
							double ip = 0;
							for (int i = 0; i < 3; ++i)
								for (int j = 0; j < 3; ++j)
								{
									double R = 0, PVt = 0;
									for (int k = 0; k < 3; ++k)
										for (int l = 0; l < 3; ++l) R += psi.h[3 * i + j][3 * k + l] * Mm[k][l];
									for (int k = 0; k < 3; ++k) PVt += psi.g[3 * i + k] * V[j][k];
									ip += (R + PVt - tr * psi.g[3 * i + j]) * gp[q][i][j];
								}
							local[tid][(size_t)v.gglobal[vi] * 3 + d] -= ip * da;
						}
					continue;
				}
				const M3 FmT = transpose(inv3(F));
				const double lj = std::log(det3(F));
				M3 P;
				for (int i = 0; i < 3; ++i)
					for (int j = 0; j < 3; ++j) P.a[i][j] = mu * (F.a[i][j] - FmT.a[i][j]) + lambda * lj * FmT.a[i][j];
				for (int vi = 0; vi < v.ng; ++vi)
					for (int d = 0; d < 3; ++d)
					{
						M3 V;
						std::memset(&V, 0, sizeof(V));
						for (int k = 0; k < 3; ++k) V.a[d][k] = v.ggrad_t_m[q][vi][k];
						M3 Mm; // grad_u * V
						for (int i = 0; i < 3; ++i)
							for (int j = 0; j < 3; ++j)
							{
								double s2 = 0;
								for (int k = 0; k < 3; ++k) s2 += gu[q][i][k] * V.a[k][j];
								Mm.a[i][j] = s2;
							}
						// result = mu*M + FmT*M^T*FmT*(mu - lambda*logJ) + lambda*(FmT:M)*FmT
						double fm = 0;
						for (int i = 0; i < 3; ++i)
							for (int j = 0; j < 3; ++j) fm += FmT.a[i][j] * Mm.a[i][j];
						M3 T1, T2;
						for (int i = 0; i < 3; ++i)
							for (int j = 0; j < 3; ++j)
							{
								double s2 = 0;
								for (int k = 0; k < 3; ++k) s2 += FmT.a[i][k] * Mm.a[j][k];
								T1.a[i][j] = s2;
							}
						for (int i = 0; i < 3; ++i)
							for (int j = 0; j < 3; ++j)
							{
								double s2 = 0;
								for (int k = 0; k < 3; ++k) s2 += T1.a[i][k] * FmT.a[k][j];
								T2.a[i][j] = s2;
							}
						const double tr = V.a[0][0] + V.a[1][1] + V.a[2][2];
						double ip = 0;
						for (int i = 0; i < 3; ++i)
							for (int j = 0; j < 3; ++j)
							{
								const double R = mu * Mm.a[i][j] + T2.a[i][j] * (mu - lambda * lj) + lambda * fm * FmT.a[i][j];
								double PVt = 0;
								for (int k = 0; k < 3; ++k) PVt += P.a[i][k] * V.a[j][k];
								const double tmp = PVt - tr * P.a[i][j];
								ip += (R + tmp) * gp[q][i][j];
							}
						local[tid][(size_t)v.gglobal[vi] * 3 + d] -= ip * da;
					}
			}
		}
	});
	std::fill(term, term + nout, 0.0);
	for (auto &l : local)
		if (!l.empty())
			for (size_t i = 0; i < nout; ++i) term[i] += l[i];
}

// ---------------------------------------------------------------------------
// MassMatrixAssembler: LinearAssembler::assemble with the Mass term
// (assembler/Assembler.cpp:157-260, assembler/Mass.cpp:5-24).  For every local pair
// j <= i the block rho int phi_i phi_j dV * I is added with all nine entries (zeros
// included), and its transpose for j < i; triplets summed into CSC.  The mass
// quadrature has order 2p (AssemblerUtils::quadrature_order, AssemblerUtils.cpp:
// 201-211): Q1 uses the 2x2x2 Gauss rule as the reference does; on the affine tets any
// rule exact to degree 2p gives the integral, here a conical-product Gauss rule
// (Gauss-Legendre nodes by Newton iteration on the Legendre recurrence, collapsed
// to the tetrahedron) instead of the reference's tabulated rules.
// ---------------------------------------------------------------------------
static void gauss_legendre01(int n, std::vector<double> &x, std::vector<double> &w)
{
	x.resize(n);
	w.resize(n);
	for (int i = 0; i < n; ++i)
	{
		double t = std::cos(3.14159265358979323846 * (i + 0.75) / (n + 0.5)), dp = 0;
		for (int it = 0; it < 100; ++it)
		{
			double p0 = 1, p1 = t;
			for (int k = 2; k <= n; ++k)
			{
				const double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			const double pn = n == 1 ? t : p1, pm = n == 1 ? 1.0 : p0;
			dp = n * (t * pn - pm) / (t * t - 1);
			const double dt = pn / dp;
			t -= dt;
			if (std::fabs(dt) < 1e-16) break;
		}
		x[i] = 0.5 * (1 - t);
		w[i] = 1.0 / ((1 - t * t) * dp * dp); // 2 / ((1 - t^2) P_n'(t)^2), halved for [0, 1]
	}
}

// points (x, y, z) and weights on the unit tetrahedron exact to degree `deg`
static void tet_rule(int deg, std::vector<std::array<double, 3>> &pts, std::vector<double> &wts)
{
	std::vector<double> xu, wu, xv, wv, xw, ww;
	// an n-point Gauss-Legendre rule is exact to degree 2n - 1
	gauss_legendre01(deg / 2 + 2, xu, wu); // with the weight (1-u)^2: degree deg + 2
	gauss_legendre01(deg / 2 + 1, xv, wv); // with the weight (1-v): degree deg + 1
	gauss_legendre01(deg / 2 + 1, xw, ww); // degree deg
	pts.clear();
	wts.clear();
	for (size_t i = 0; i < xu.size(); ++i)
		for (size_t j = 0; j < xv.size(); ++j)
			for (size_t k = 0; k < xw.size(); ++k)
			{
				const double u = xu[i], v = xv[j], t = xw[k];
				pts.push_back({u, v * (1 - u), t * (1 - u) * (1 - v)});
				wts.push_back(wu[i] * wv[j] * ww[k] * (1 - u) * (1 - u) * (1 - v));
			}
}

// FE basis values: P1 barycentric; P2 vertices lambda(2 lambda - 1), edges 4 lambda_i
// lambda_j (01, 12, 20, 03, 13, 23); Q1 trilinear (corners 000 100 110 010 001 101 111 011)
static double basis_value(int type, int i, double x, double y, double z)
{
	const double l[4] = {1 - x - y - z, x, y, z};
	if (type == P1_TET) return l[i];
	if (type == P2_TET)
	{
		static const int e[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
		return i < 4 ? l[i] * (2 * l[i] - 1) : 4 * l[e[i - 4][0]] * l[e[i - 4][1]];
	}
	static const int c[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
	return (c[i][0] ? x : 1 - x) * (c[i][1] ? y : 1 - y) * (c[i][2] ? z : 1 - z);
}

static void mass_impl(Context &c, const double *rho)
{
	const Tables &t = c.t;
	std::vector<std::array<double, 3>> pts;
	std::vector<double> wts;
	if (t.type == Q1_HEX)
		for (int q = 0; q < t.nq; ++q)
		{
			pts.push_back({t.qp[q][0], t.qp[q][1], t.qp[q][2]});
			wts.push_back(t.qw[q]);
		}
	else
		tet_rule(t.type == P1_TET ? 2 : 4, pts, wts);
	void (*const ge)(int, double, double, double, double *) = t.type == Q1_HEX ? q1_grad : p1_grad;
	std::vector<Triplet> trip;
	for (int e = 0; e < c.E; ++e)
	{
		const double r = rho ? rho[e] : 1.0;
		std::vector<double> m((size_t)t.n * t.n, 0.0);
		for (size_t q = 0; q < pts.size(); ++q)
		{
			// geometry Jacobian at the point from the geometric basis
			M3 J;
			std::memset(&J, 0, sizeof(J));
			for (int j = 0; j < t.ng; ++j)
			{
				double g[3];
				ge(j, pts[q][0], pts[q][1], pts[q][2], g);
				const double *node = c.X.data() + (size_t)c.gconn[(size_t)e * t.ng + j] * 3;
				for (int rr = 0; rr < 3; ++rr)
					for (int cc = 0; cc < 3; ++cc) J.a[rr][cc] += g[rr] * node[cc];
			}
			const double da = det3(J) * wts[q];
			for (int a = 0; a < t.n; ++a)
				for (int b = 0; b < t.n; ++b)
					m[(size_t)a * t.n + b] += r * basis_value(t.type, a, pts[q][0], pts[q][1], pts[q][2]) *
											  basis_value(t.type, b, pts[q][0], pts[q][1], pts[q][2]) * da;
		}
		for (int i = 0; i < t.n; ++i)
			for (int j = 0; j <= i; ++j)
				for (int n = 0; n < 3; ++n)
					for (int mm = 0; mm < 3; ++mm)
					{
						const double v = n == mm ? m[(size_t)i * t.n + j] : 0.0;
						const int gi = c.conn[(size_t)e * t.n + i] * 3 + mm, gj = c.conn[(size_t)e * t.n + j] * 3 + n;
						trip.push_back({gi, gj, v});
						if (j < i) trip.push_back({gj, gi, v});
					}
	}
	c.mass = csc_from_triplets(c.N * 3, c.N * 3, trip);
}

template <typename Fn>
static auto dispatch(int n, Fn &&fn)
{
	switch (n)
	{
	case 4: return fn(std::integral_constant<int, 4>());
	case 8: return fn(std::integral_constant<int, 8>());
	case 10: return fn(std::integral_constant<int, 10>());
	}
	throw std::runtime_error("unsupported nodes per element");
}
} // namespace orc

using namespace orc;

extern "C"
{
	void *orc_create(int elem_type, int n_elements, int n_nodes, const int *conn, int n_geom_nodes, const int *gconn,
					 const double *X, const double *lambda, const double *mu, int n_threads, int cache_size, int fast_pattern)
	{
		try
		{
			auto *c = new Context();
			c->t = make_tables(elem_type);
			c->E = n_elements; c->N = n_nodes; c->Ng = n_geom_nodes;
			c->conn.assign(conn, conn + (size_t)n_elements * c->t.n);
			const int *gc = gconn ? gconn : conn;
			c->gconn.assign(gc, gc + (size_t)n_elements * c->t.ng);
			c->X.assign(X, X + (size_t)n_geom_nodes * 3);
			c->lambda.assign(lambda, lambda + n_elements);
			c->mu.assign(mu, mu + n_elements);
			c->n_threads = std::max(1, n_threads);
			c->fast_pattern = fast_pattern != 0;
			// AssemblyValsCache is built only when n_bases <= cache_size (State.cpp:994-1010)
			c->use_cache = n_nodes <= cache_size;
			if (c->use_cache)
			{
				c->cache.resize(n_elements);
				par_for(n_elements, c->n_threads, [&](int s, int e, int) {
					for (int el = s; el < e; ++el) compute_values(c->t, c->conn.data(), c->gconn.data(), c->X.data(), el, c->cache[el]);
				});
			}
			return c;
		}
		catch (...)
		{
			return nullptr;
		}
	}

	void orc_destroy(void *h) { delete static_cast<Context *>(h); }
	// FE basis value (for the check of the values against the gradient tables)
	double orc_basis_value(int type, int i, double x, double y, double z) { return basis_value(type, i, x, y, z); }
	// MassMatrixAssembler (rho per element or NULL for 1); returns nnz, then orc_mass_copy
	long long orc_mass(void *h, const double *rho)
	{
		Context &c = *static_cast<Context *>(h);
		mass_impl(c, rho);
		return (long long)c.mass.inner.size();
	}
	void orc_mass_copy(void *h, int *outer, int *inner, double *values)
	{
		const CSC &m = static_cast<Context *>(h)->mass;
		std::copy(m.outer.begin(), m.outer.end(), outer);
		std::copy(m.inner.begin(), m.inner.end(), inner);
		std::copy(m.values.begin(), m.values.end(), values);
	}

	void orc_set_threads(void *h, int n) { static_cast<Context *>(h)->n_threads = std::max(1, n); }
	// later orc_hessian calls project every element matrix onto the PSD cone
	void orc_set_project_psd(void *h, int on) { static_cast<Context *>(h)->project_psd = on != 0; }
	// later calls use another material of the GenericElastic family (MAT_*); 0 = NeoHookean
	void orc_set_material(void *h, int mat) { static_cast<Context *>(h)->material = mat; }
	// per-element GenericMatParam values, parameter-major (params[k * E + e]), 1..8 of them
	void orc_set_material_params(void *h, const double *params, int n_params)
	{
		Context &c = *static_cast<Context *>(h);
		c.n_mparams = n_params;
		c.mparams.assign(params, params + (size_t)n_params * c.E);
	}
	// HookeLinearElasticity's tensor: 21 entries C(i, j), i <= j, row by row
	// (ElasticityTensor::set_from_entries, MatParams.cpp:180-205)
	void orc_set_elasticity_tensor(void *h, const double *c21)
	{
		Context &c = *static_cast<Context *>(h);
		for (int k = 0; k < PRM_MAX; ++k) c.hooke[k] = c21[k];
	}
	// ipc::project_to_psd (CLAMP) of one row-major m x m symmetric matrix, in place
	void orc_project_psd(double *H, int m) { project_to_psd(H, m); }

	double orc_energy(void *h, const double *x)
	{
		Context &c = *static_cast<Context *>(h);
		return dispatch(c.t.n, [&](auto N) { return energy_impl<decltype(N)::value>(c, x, nullptr); });
	}

	void orc_energy_per_element(void *h, const double *x, double *out)
	{
		Context &c = *static_cast<Context *>(h);
		dispatch(c.t.n, [&](auto N) { return energy_impl<decltype(N)::value>(c, x, out); });
	}

	void orc_gradient(void *h, const double *x, double *g)
	{
		Context &c = *static_cast<Context *>(h);
		dispatch(c.t.n, [&](auto N) { gradient_impl<decltype(N)::value>(c, x, g); return 0; });
	}

	// Assembles the Hessian; returns nnz of the result (call orc_hessian_copy next).
	long long orc_hessian(void *h, const double *x)
	{
		Context &c = *static_cast<Context *>(h);
		try
		{
			dispatch(c.t.n, [&](auto N) { hessian_impl<decltype(N)::value>(c, x); return 0; });
		}
		catch (const std::exception &e)
		{
			c.err = e.what();
			return -1;
		}
		return (long long)c.last.nnz();
	}

	void orc_hessian_copy(void *h, int *outer, int *inner, double *values)
	{
		Context &c = *static_cast<Context *>(h);
		if (outer) std::copy(c.last.outer.begin(), c.last.outer.end(), outer);
		if (inner) std::copy(c.last.inner.begin(), c.last.inner.end(), inner);
		if (values) std::copy(c.last.values.begin(), c.last.values.end(), values);
	}

	// Slot of the k-th add_value of element e (SparseMatrixCache second_cache_).
	int orc_slot(void *h, int e, int k)
	{
		Context &c = *static_cast<Context *>(h);
		const auto &sc = c.mat_cache.second_cache();
		if (e < 0 || e >= (int)sc.size() || k < 0 || k >= (int)sc[e].size()) return -1;
		return sc[e][k];
	}

	void orc_material_vjp(void *h, const double *x, const double *adj, double *term)
	{
		Context &c = *static_cast<Context *>(h);
		dispatch(c.t.n, [&](auto N) { material_vjp_impl<decltype(N)::value>(c, x, adj, term); return 0; });
	}

	void orc_shape_vjp(void *h, const double *x, const double *adj, double *term)
	{
		Context &c = *static_cast<Context *>(h);
		dispatch(c.t.n, [&](auto N) { shape_vjp_impl<decltype(N)::value>(c, x, adj, term); return 0; });
	}

	// Single-element kernels for autodiff / finite-difference checks.
	// x is the global displacement; H is (3n x 3n) row-major.
	int orc_element(void *h, int e, const double *x, double *energy, double *grad, double *hess)
	{
		Context &c = *static_cast<Context *>(h);
		ElementValues v;
		c.vals(e, v);
		return dispatch(c.t.n, [&](auto N) {
			constexpr int n = decltype(N)::value;
			if (c.material)
			{
				double prm[PRM_MAX];
				c.params(e, prm);
				if (energy) *energy = gen_element_energy<n>(c.material, v, x, prm);
				if (grad || hess) gen_element_derivatives<n>(c.material, v, x, prm, grad, hess);
				return 0;
			}
			if (energy) *energy = element_energy<n>(v, x, c.lambda[e], c.mu[e]);
			if (grad) element_gradient<n>(v, x, c.lambda[e], c.mu[e], grad);
			if (hess) element_hessian<n>(v, x, c.lambda[e], c.mu[e], hess);
			return 0;
		});
	}

	// Reference tables: quadrature points (nq x 3), weights (nq), gradients (nq x n x 3).
	int orc_tables(int elem_type, double *qp, double *qw, double *grad, double *ggrad)
	{
		Tables t = make_tables(elem_type);
		for (int q = 0; q < t.nq; ++q)
		{
			for (int d = 0; d < 3; ++d) qp[q * 3 + d] = t.qp[q][d];
			qw[q] = t.qw[q];
			for (int i = 0; i < t.n; ++i)
				for (int d = 0; d < 3; ++d) grad[(q * t.n + i) * 3 + d] = t.grad[q][i][d];
			for (int i = 0; i < t.ng; ++i)
				for (int d = 0; d < 3; ++d) ggrad[(q * t.ng + i) * 3 + d] = t.ggrad[q][i][d];
		}
		return t.nq;
	}

	// ---- bare SparseMatrixCache for the restated known-answer test ----
	void *orc_smc_new(int size)
	{
		auto *m = new SparseMatrixCache();
		m->init(size);
		return m;
	}
	void *orc_smc_copy(void *other)
	{
		auto *m = new SparseMatrixCache();
		m->init(*static_cast<SparseMatrixCache *>(other), false);
		return m;
	}
	void orc_smc_add(void *h, int e, int i, int j, double v) { static_cast<SparseMatrixCache *>(h)->add_value(e, i, j, v); }
	void orc_smc_prune(void *h) { static_cast<SparseMatrixCache *>(h)->prune(); }
	// get_matrix(); the returned matrix is kept for orc_smc_coeff
	long long orc_smc_get_matrix(void *h)
	{
		auto *m = static_cast<SparseMatrixCache *>(h);
		const CSC r = m->get_matrix(); // returns mat_, which stays addressable for orc_smc_coeff
		return (long long)r.nnz();
	}
	double orc_smc_coeff(void *h, int i, int j)
	{
		const auto *m = static_cast<SparseMatrixCache *>(h);
		return m->mat_.coeff(i, j);
	}
	void orc_smc_free(void *h) { delete static_cast<SparseMatrixCache *>(h); }
}
