// Energy-defined materials on the device (FP64).
//
// The reference assembles these formulations from an energy density alone:
// GenericElastic (assembler/GenericElastic.cpp:493-611, AutodiffType::STRESS) takes
// dpsi/dF and d2psi/dF2 by forward-mode autodiff over the 9 entries of F and
// contracts them with the physical basis gradients; LinearElasticity
// (LinearElasticity.cpp:65-139) differentiates its strain energy over the nodal
// values.  Both give, per quadrature point q and node pair (a, b),
//   gradient  G[a][r]    = sum_q da_q sum_c P[r][c] g_a[c]
//   Hessian   H_ab[r][k] = sum_q da_q sum_{c,d} g_a[c] C[(r,c),(k,d)] g_b[d]
// with P = dpsi/dF and C = d2psi/dF2 (index 3r + c for F(r, c)).
//
// MooneyRivlin, MooneyRivlin3Param and VolumePenalty are functions of the three
// invariants x = (I1, I2, J) of F, I1 = tr B, I2 = (tr^2 B - tr B^2)/2, J = det F,
// B = F F^T; their density psi(I1, I2, J) is written once, generic in its number
// type, and its derivatives psi_x, psi_xy come from hyper-dual numbers over the
// three scalars (Fike and Alonso, "The development of hyper-dual numbers for exact
// second-derivative calculations", AIAA 2011-886): six evaluations per point give
// all of them exactly.  The chain rule through the invariants then gives
//   P = sum_x psi_x dx/dF,
//   C = sum_x psi_x d2x/dF2 + sum_{x,y} psi_xy dx/dF (x) dy/dF,
// with, for i = (a, A), j = (b, B):
//   dI1/dF = 2F,  dI2/dF = 2 I1 F - 2 B F,  dJ/dF = cof F,
//   d2I1 = 2 delta_ij,
//   d2I2 = 4 F_aA F_bB + 2 I1 delta_ab delta_AB - 2 delta_ab (F^T F)_AB - 2 F_aB F_bA - 2 delta_AB B_ab,
//   d2J  = eps_abc eps_ABC F_cC.
// LinearElasticity is quadratic: P = 2 mu eps + lambda tr(eps) I and the constant
// C = mu (delta_ab delta_AB + delta_aB delta_Ab) + lambda delta_aA delta_bB.
// HookeLinearElasticity is quadratic too: with the Voigt strain v(G) = (G00, G11,
// G22, G12 + G21, G02 + G20, G01 + G10) of G = F - I and the 6 x 6 tensor T,
// psi = 1/2 v.T v, P(r, c) = (T v)[voigt(r, c)] and C = T[voigt(a, A)][voigt(b, B)].
// SaintVenant with that tensor takes the Green strain E = (F^T F - I)/2 in the same
// Voigt form e = (E00, E11, E22, 2E12, 2E02, 2E01): psi = 1/2 e.T e, the second
// Piola-Kirchhoff stress S(A, B) = (T e)[voigt(A, B)], P = F S and
//   C[(a,A),(b,B)] = delta_ab S(A, B) + sum_{I,J} F(a, I) F(b, J) T[voigt(I, A)][voigt(J, B)].
// In the blocks kernel the 45 entries i <= j of C at every point are spread over
// the lanes of the element's warp; the blocks are written as the packed block
// triangle of the element, which the PSD projection and the scatter of
// pfg_kernels.cu consume.
//
// Materials (per-element parameters, pfg_set_material_params / pfg_set_lame):
//   3 LinearElasticity    (lambda, mu)     psi = mu eps:eps + lambda/2 tr(eps)^2, eps = (G + G^T)/2, G = F - I
//                                          (LinearElasticity.cpp:113-139)
//   4 MooneyRivlin        (c1, c2, k)      psi = c1 (I1~ - 3) + c2 (I2~ - 3) + k/2 ln^2 J
//                                          (MooneyRivlinElasticity.hpp:25-46)
//   5 MooneyRivlin3Param  (c1, c2, c3, d1) psi = c1 (I1~ - 3) + (c2 + c3 (I1~ - 3)) (I2~ - 3) + d1 (J - 1)^2
//                                          (MooneyRivlin3ParamElasticity.hpp:26-49)
//  11 MooneyRivlin3ParamSymbolic (c1, c2, c3, d1): the same with d1 ln^2 J
//                                          (MooneyRivlin3ParamSymbolic.cpp:317-340)
//   6 VolumePenalty       (k)              psi = k/2 ((J^2 - 1)/2 - ln J)   (VolumePenalty.hpp:20-34)
//   7 HookeLinearElasticity (one tensor)  psi = 1/2 sigma:eps, sigma = T eps in Voigt form
//                                          (HookeLinearElasticity.cpp:372-421)
//   8 SaintVenant         (one tensor)     psi = 1/2 S:E, S = T E in Voigt form, E the Green strain
//                                          (SaintVenantElasticity.cpp:209-267)
//   9 UnconstrainedOgden  (alphas, mus, Ds; 1-2 terms)   psi of the principal stretches
//  10 IncompressibleOgden (cs, ms, k; 1-3 terms)          (OgdenElasticity.tpp:8-94)
// The Ogden densities are functions of the invariants too: the stretches are the
// square roots of the eigenvalues of F^T F, which the characteristic cubic gives from
// (I1, I2, J^2) (cauchy_green_eigs).
// with I1~ = J^-2/3 I1 and I2~ = J^-4/3 I2 (the invariants of F~ F~^T, F~ = J^-1/3 F).
#include "pfg_device.cuh"

#include <algorithm>
#include <cmath>

namespace pfg
{

constexpr int MAT_LINEAR_ELASTICITY = 3, MAT_MOONEY_RIVLIN = 4, MAT_MOONEY_RIVLIN_3PARAM = 5, MAT_VOLUME_PENALTY = 6,
			  MAT_HOOKE = 7, MAT_SAINT_VENANT_TENSOR = 8, MAT_UNCONSTRAINED_OGDEN = 9, MAT_INCOMPRESSIBLE_OGDEN = 10,
			  MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC = 11;
// An element's material parameters: up to eight values (pfg_set_material_params)
// and, for the Ogden formulations, the number of terms.
struct MatP
{
	double x, y, z, w, x2, y2, z2, w2;
	int nt;
};
// the quadratic densities: constant tangent, no invariants
template <int MAT>
__host__ __device__ constexpr bool quadratic_mat() { return MAT == MAT_LINEAR_ELASTICITY || MAT == MAT_HOOKE; }
// the densities of the principal stretches (Ogden), differentiated by dual and
// hyper-dual numbers over the nine entries of F as the reference differentiates them
template <int MAT>
__host__ __device__ constexpr bool entry_mat() { return MAT == MAT_UNCONSTRAINED_OGDEN || MAT == MAT_INCOMPRESSIBLE_OGDEN; }
// the densities of (I1, I2, J), differentiated by hyper-dual numbers
template <int MAT>
__host__ __device__ constexpr bool invariant_mat()
{
	return !quadratic_mat<MAT>() && MAT != MAT_SAINT_VENANT_TENSOR && !entry_mat<MAT>();
}
// Voigt index of F(r, c) in HookeLinearElasticity's strain (e00, e11, e22, 2e12, 2e02, 2e01)
__host__ __device__ constexpr int voigt(int r, int c) { return r == c ? r : 6 - r - c; }
// IsochoricNeoHookean (hand-derived tangent in pfg_kernels.cu) is also an invariant
// density; its shape derivative is taken here
constexpr int MAT_ISO_NEOHOOKEAN = 1;

// ---------------------------------------------------------------------------
// forward-mode numbers
// ---------------------------------------------------------------------------
struct Dual1
{
	double v, d; // value, derivative along one direction
};
struct HDual
{
	double v, a, b, ab; // value, d/de1, d/de2, d2/de1de2
};

__device__ __forceinline__ Dual1 operator+(Dual1 x, Dual1 y) { return {x.v + y.v, x.d + y.d}; }
__device__ __forceinline__ Dual1 operator-(Dual1 x, Dual1 y) { return {x.v - y.v, x.d - y.d}; }
__device__ __forceinline__ Dual1 operator*(Dual1 x, Dual1 y) { return {x.v * y.v, x.v * y.d + x.d * y.v}; }
__device__ __forceinline__ Dual1 operator*(double s, Dual1 x) { return {s * x.v, s * x.d}; }
__device__ __forceinline__ Dual1 operator-(Dual1 x, double s) { return {x.v - s, x.d}; }
__device__ __forceinline__ Dual1 operator+(Dual1 x, double s) { return {x.v + s, x.d}; }
// f(x) with f'(x.v) = f1
__device__ __forceinline__ Dual1 chain(Dual1 x, double f0, double f1, double) { return {f0, f1 * x.d}; }

__device__ __forceinline__ HDual operator+(HDual x, HDual y) { return {x.v + y.v, x.a + y.a, x.b + y.b, x.ab + y.ab}; }
__device__ __forceinline__ HDual operator-(HDual x, HDual y) { return {x.v - y.v, x.a - y.a, x.b - y.b, x.ab - y.ab}; }
__device__ __forceinline__ HDual operator*(HDual x, HDual y)
{
	return {x.v * y.v, x.v * y.a + x.a * y.v, x.v * y.b + x.b * y.v, x.v * y.ab + x.a * y.b + x.b * y.a + x.ab * y.v};
}
__device__ __forceinline__ HDual operator*(double s, HDual x) { return {s * x.v, s * x.a, s * x.b, s * x.ab}; }
__device__ __forceinline__ HDual operator-(HDual x, double s) { return {x.v - s, x.a, x.b, x.ab}; }
__device__ __forceinline__ HDual operator+(HDual x, double s) { return {x.v + s, x.a, x.b, x.ab}; }
// f(x) with f'(x.v) = f1, f''(x.v) = f2
__device__ __forceinline__ HDual chain(HDual x, double f0, double f1, double f2)
{
	return {f0, f1 * x.a, f1 * x.b, f1 * x.ab + f2 * x.a * x.b};
}

__device__ __forceinline__ double ad_log(double x) { return log(x); }
__device__ __forceinline__ double ad_pow(double x, double p) { return pow(x, p); }
template <class S>
__device__ __forceinline__ S ad_log(S x)
{
	const double r = 1.0 / x.v;
	return chain(x, log(x.v), r, -r * r);
}
// x^p: f' = p x^(p-1) = p f / x, f'' = (p - 1) f' / x
template <class S>
__device__ __forceinline__ S ad_pow(S x, double p)
{
	const double f = pow(x.v, p), r = 1.0 / x.v, f1 = p * f * r;
	return chain(x, f, f1, (p - 1.0) * f1 * r);
}

template <class S>
__device__ __forceinline__ S sq(S x) { return x * x; }
__device__ __forceinline__ double ad_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ double ad_recip(double x) { return 1.0 / x; }
__device__ __forceinline__ double ad_acos(double x) { return acos(x); }
__device__ __forceinline__ double ad_cos(double x) { return cos(x); }
// sqrt: f' = 1/(2f), f'' = -f'/(2x)
template <class S>
__device__ __forceinline__ S ad_sqrt(S x)
{
	const double f = sqrt(x.v), f1 = 0.5 / f;
	return chain(x, f, f1, -0.5 * f1 / x.v);
}
template <class S>
__device__ __forceinline__ S ad_recip(S x)
{
	const double r = 1.0 / x.v;
	return chain(x, r, -r * r, 2.0 * r * r * r);
}
// acos: f' = -(1 - x^2)^(-1/2), f'' = -x (1 - x^2)^(-3/2)
template <class S>
__device__ __forceinline__ S ad_acos(S x)
{
	const double d = 1.0 - x.v * x.v, rs = 1.0 / sqrt(d);
	return chain(x, acos(x.v), -rs, -x.v * rs / d);
}
template <class S>
__device__ __forceinline__ S ad_cos(S x)
{
	const double c = cos(x.v);
	return chain(x, c, -sin(x.v), -c);
}
__device__ __forceinline__ double ad_val(double x) { return x; }
__device__ __forceinline__ double ad_val(Dual1 x) { return x.v; }
__device__ __forceinline__ double ad_val(HDual x) { return x.v; }
template <class S>
__device__ __forceinline__ S ad_const(double c);
template <>
__device__ __forceinline__ double ad_const<double>(double c) { return c; }
template <>
__device__ __forceinline__ Dual1 ad_const<Dual1>(double c) { return {c, 0.0}; }
template <>
__device__ __forceinline__ HDual ad_const<HDual>(double c) { return {c, 0.0, 0.0, 0.0}; }


// The Ogden sums of K terms over the three stretches st; pv holds alphas, mus, Ds
// (unconstrained) or cs, ms, k (incompressible), K values per group.
template <int K, bool INC, class S>
__device__ __forceinline__ S ogden_terms(const S (&st)[3], S J, const double (&pv)[8])
{
	S val = ad_const<S>(0.0);
#pragma unroll
	for (int t = 0; t < K; ++t)
	{
		const double ex = INC ? pv[K + t] : pv[t];
		const double co = INC ? pv[t] / (ex * ex) : 2.0 * pv[K + t] / (ex * ex);
		S tmp = ad_const<S>(-3.0);
#pragma unroll
		for (int i = 0; i < 3; ++i) tmp = tmp + ad_pow(st[i], ex);
		val = val + co * tmp;
	}
	if constexpr (INC)
		val = val + (0.5 * pv[2 * K]) * sq(ad_log(J));
	else
	{
		const S jm2 = sq(J - 1.0);
		S w = jm2;
#pragma unroll
		for (int t = 0; t < K; ++t)
		{
			val = val + (1.0 / pv[2 * K + t]) * w; // (J - 1)^(2(t+1)) / D_t
			w = w * jm2;
		}
	}
	return val;
}

// The eigenvalues of a symmetric 3 x 3 matrix m, the closed form that
// utils::autogen::eigs_3d (autogen/auto_eigs.hpp:33-76) evaluates from the entries
// m00, m11, m22, m01, m02, m12: with 9p = 3 (m01^2 + m02^2 + m12^2) + ((m00 - m22)^2 +
// (m11 - m22)^2 + (m00 - m11)^2) / 2 and the angle t = acos(27 det(m - tr/3 I) / (2 (9p)^(3/2))) / 3,
//   eig = tr/3 + (2/3) sqrt(9p) cos(t + {0, 2pi/3, -2pi/3});
// all three tr/3 when 2 sqrt(9p) < 1e-10, t the constant 0 or pi/3 when the cosine's
// argument leaves [-1, 1], as there.
template <class S>
__device__ __forceinline__ void sym_eigs3(const S (&m)[3][3], S (&res)[3])
{
	const S t01 = m[0][0] + m[1][1];
	const S tr = t01 + m[2][2];
	const S off = m[0][1] * m[0][1] + m[0][2] * m[0][2] + m[1][2] * m[1][2];
	const S d02 = m[0][0] - m[2][2], d12 = m[1][1] - m[2][2], d01 = m[0][0] - m[1][1];
	const S p9 = 3.0 * off + 0.5 * (d02 * d02) + 0.5 * (d12 * d12) + 0.5 * (d01 * d01);
	if (2.0 * sqrt(ad_val(p9)) < 1e-10)
	{
		res[0] = res[1] = res[2] = (1.0 / 3.0) * tr;
		return;
	}
	const S sp9 = ad_sqrt(p9);
	const S num = -1.5 * (t01 * (m[0][0] + m[2][2]) * (m[1][1] + m[2][2])) + 4.5 * (tr * off) -
				  13.5 * (m[0][1] * m[0][1] * m[2][2]) - 13.5 * (m[0][2] * m[0][2] * m[1][1]) -
				  13.5 * (m[1][2] * m[1][2] * m[0][0]) + m[0][0] * m[0][0] * m[0][0] + 9.0 * (m[0][0] * m[1][1] * m[2][2]) +
				  27.0 * (m[0][1] * m[0][2] * m[1][2]) + m[1][1] * m[1][1] * m[1][1] + m[2][2] * m[2][2] * m[2][2];
	const S c3 = num * ad_recip(p9 * sp9);
	const double c3v = ad_val(c3);
	const S ang = (1.0 / 3.0) * (c3v >= 1.0 ? ad_const<S>(0.0) : c3v <= -1.0 ? ad_const<S>(M_PI) : ad_acos(c3));
	const S r = (2.0 / 3.0) * sp9, mean = (1.0 / 3.0) * tr;
	res[0] = r * ad_cos(ang) + mean;
	res[1] = r * ad_cos(ang + 2.0 * M_PI / 3.0) + mean;
	res[2] = r * ad_cos(ang - 2.0 * M_PI / 3.0) + mean;
}

template <class S>
__device__ __forceinline__ S det3s(const S (&F)[3][3])
{
	return F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
		   F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
}

// The Ogden densities of F, generic in the number type:
//   UnconstrainedOgden (OgdenElasticity.tpp:8-57): the stretches sqrt(eig(F^T F)) J^(-1/3);
//   IncompressibleOgden (OgdenElasticity.tpp:59-94): F~ = F / J^(1/3), the stretches
//   sqrt(eig(F~ F~^T)); both then ogden_terms.
template <int MAT, class S>
__device__ __forceinline__ S ogden_psi(const S (&F)[3][3], const MatP &p)
{
	constexpr bool inc = MAT == MAT_INCOMPRESSIBLE_OGDEN;
	const double pv[8] = {p.x, p.y, p.z, p.w, p.x2, p.y2, p.z2, p.w2};
	const S J = det3s(F);
	S Cm[3][3], st[3];
	if constexpr (inc)
	{
		const S is = ad_recip(ad_pow(J, 1.0 / 3.0));
		S Ft[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Ft[r][c] = F[r][c] * is;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Cm[r][c] = Ft[r][0] * Ft[c][0] + Ft[r][1] * Ft[c][1] + Ft[r][2] * Ft[c][2];
		sym_eigs3(Cm, st);
#pragma unroll
		for (int i = 0; i < 3; ++i) st[i] = ad_sqrt(st[i]);
	}
	else
	{
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Cm[r][c] = F[0][r] * F[0][c] + F[1][r] * F[1][c] + F[2][r] * F[2][c];
		sym_eigs3(Cm, st);
		const S jd = ad_pow(J, -1.0 / 3.0);
#pragma unroll
		for (int i = 0; i < 3; ++i) st[i] = ad_sqrt(st[i]) * jd;
	}
	if (p.nt == 1) return ogden_terms<1, inc>(st, J, pv);
	if (p.nt == 2) return ogden_terms<2, inc>(st, J, pv);
	return ogden_terms<3, inc>(st, J, pv);
}

// F with the dual parts of two directions: entry (r, c) carries d/de1 = [3r+c == i],
// d/de2 = W(r, c) (W may be a unit direction e_j)
__device__ __forceinline__ void hd_def_grad(const double F[3][3], int i, const double (&W)[9], HDual (&Fh)[3][3])
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) Fh[r][c] = {F[r][c], (3 * r + c) == i ? 1.0 : 0.0, W[3 * r + c], 0.0};
}

// ---------------------------------------------------------------------------
// energy densities of the invariant materials, generic in the number type
// ---------------------------------------------------------------------------
template <int MAT, class S>
__device__ __forceinline__ S inv_psi(S I1, S I2, S J, const MatP &p)
{
	if constexpr (MAT == MAT_ISO_NEOHOOKEAN) // psi = mu/2 (J^-2/3 I1 - 3), IsochoricNeoHookean.hpp:19-33
		return (0.5 * p.y) * (ad_pow(J, -2.0 / 3.0) * I1 - 3.0);
	else if constexpr (MAT == MAT_VOLUME_PENALTY)
		return (0.5 * p.x) * (0.5 * (sq(J) - 1.0) - ad_log(J));
	else
	{
		const S j23 = ad_pow(J, -2.0 / 3.0);
		const S I1t = j23 * I1 - 3.0, I2t = sq(j23) * I2 - 3.0;
		if constexpr (MAT == MAT_MOONEY_RIVLIN)
			return p.x * I1t + p.y * I2t + (0.5 * p.z) * sq(ad_log(J));
		else if constexpr (MAT == MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC) // its volumetric term is d1 ln^2 J
			return p.x * I1t + (p.z * I1t + p.y) * I2t + p.w * sq(ad_log(J));
		else // MAT_MOONEY_RIVLIN_3PARAM
			return p.x * I1t + (p.z * I1t + p.y) * I2t + p.w * sq(J - 1.0);
	}
}

// invariants of F and their derivatives: dx[x][3a + A] = dx/dF(a, A) for x = I1, I2, J;
// B = F F^T and Cr = F^T F (row-major 9)
struct Invariants
{
	double I1, I2, J;
	double B[9], Cr[9], dx[3][9];
};

__device__ __forceinline__ void invariants(const double F[3][3], Invariants &v)
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c)
		{
			v.B[3 * r + c] = F[r][0] * F[c][0] + F[r][1] * F[c][1] + F[r][2] * F[c][2];
			v.Cr[3 * r + c] = F[0][r] * F[0][c] + F[1][r] * F[1][c] + F[2][r] * F[2][c];
		}
	v.I1 = v.B[0] + v.B[4] + v.B[8];
	double trB2 = 0.0;
#pragma unroll
	for (int i = 0; i < 9; ++i) trB2 += v.B[i] * v.B[i];
	v.I2 = 0.5 * (v.I1 * v.I1 - trB2);
	v.J = det3(F);
	double cof[3][3];
	cofactor3(F, cof);
#pragma unroll
	for (int a = 0; a < 3; ++a)
#pragma unroll
		for (int A = 0; A < 3; ++A)
		{
			const double BF = v.B[3 * a] * F[0][A] + v.B[3 * a + 1] * F[1][A] + v.B[3 * a + 2] * F[2][A];
			v.dx[0][3 * a + A] = 2.0 * F[a][A];
			v.dx[1][3 * a + A] = 2.0 * (v.I1 * F[a][A] - BF);
			v.dx[2][3 * a + A] = cof[a][A];
		}
}

// psi_x (x = I1, I2, J) by three dual evaluations
template <int MAT>
__device__ __forceinline__ void inv_psi_first(const Invariants &v, const MatP &p, double d[3])
{
#pragma unroll 1
	for (int x = 0; x < 3; ++x)
		d[x] = inv_psi<MAT, Dual1>({v.I1, x == 0 ? 1.0 : 0.0}, {v.I2, x == 1 ? 1.0 : 0.0}, {v.J, x == 2 ? 1.0 : 0.0}, p).d;
}

template <int MAT>
__device__ __forceinline__ MatP ad_params(const DevMesh &m, int e)
{
	MatP p{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, m.mterms};
	if constexpr (MAT == MAT_HOOKE || MAT == MAT_SAINT_VENANT_TENSOR) // their one tensor is m.hooke
		return p;
	else if constexpr (MAT == MAT_LINEAR_ELASTICITY || MAT == MAT_ISO_NEOHOOKEAN)
	{
		const double2 lm = __ldg(m.lame + e);
		p.x = lm.x;
		p.y = lm.y;
		return p;
	}
	else
	{
		// eight values per element, 64 bytes: the Ogden formulations read all of them
		const double2 *q = reinterpret_cast<const double2 *>(m.mpar + 2 * (size_t)e);
		const double2 x = __ldg(q), y = __ldg(q + 1);
		p.x = x.x;
		p.y = x.y;
		p.z = y.x;
		p.w = y.y;
		if constexpr (MAT == MAT_UNCONSTRAINED_OGDEN || MAT == MAT_INCOMPRESSIBLE_OGDEN)
		{
			const double2 z = __ldg(q + 2), w = __ldg(q + 3);
			p.x2 = z.x;
			p.y2 = z.y;
			p.z2 = w.x;
			p.w2 = w.y;
		}
		return p;
	}
}

// HookeLinearElasticity: the Voigt strain v and the Voigt stress T v
__device__ __forceinline__ void hooke_strain_stress(const double F[3][3], const double *__restrict__ T, double v[6],
													double sv[6])
{
	v[0] = F[0][0] - 1.0;
	v[1] = F[1][1] - 1.0;
	v[2] = F[2][2] - 1.0;
	v[3] = F[1][2] + F[2][1];
	v[4] = F[0][2] + F[2][0];
	v[5] = F[0][1] + F[1][0];
#pragma unroll
	for (int j = 0; j < 6; ++j)
	{
		double s_ = 0.0;
#pragma unroll
		for (int k = 0; k < 6; ++k) s_ += __ldg(T + 6 * j + k) * v[k];
		sv[j] = s_;
	}
}

// SaintVenant with a tensor: the Voigt Green strain from F^T F and the Voigt stress T e
__device__ __forceinline__ void green_voigt_stress(const double Cr[9], const double *__restrict__ T, double e[6],
												   double sv[6])
{
	e[0] = 0.5 * (Cr[0] - 1.0);
	e[1] = 0.5 * (Cr[4] - 1.0);
	e[2] = 0.5 * (Cr[8] - 1.0);
	e[3] = Cr[5];
	e[4] = Cr[2];
	e[5] = Cr[1];
#pragma unroll
	for (int j = 0; j < 6; ++j)
	{
		double s_ = 0.0;
#pragma unroll
		for (int k = 0; k < 6; ++k) s_ += __ldg(T + 6 * j + k) * e[k];
		sv[j] = s_;
	}
}

__device__ __forceinline__ void right_cauchy_green(const double F[3][3], double Cr[9])
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) Cr[3 * r + c] = F[0][r] * F[0][c] + F[1][r] * F[1][c] + F[2][r] * F[2][c];
}

template <int MAT>
__device__ __forceinline__ double mat_energy(const double F[3][3], const MatP &p, const double *T)
{
	if constexpr (entry_mat<MAT>())
	{
		double Fc[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Fc[r][c] = F[r][c];
		return ogden_psi<MAT, double>(Fc, p);
	}
	else if constexpr (MAT == MAT_SAINT_VENANT_TENSOR)
	{
		double Cr[9], e[6], sv[6];
		right_cauchy_green(F, Cr);
		green_voigt_stress(Cr, T, e, sv);
		return 0.5 * (sv[0] * e[0] + sv[1] * e[1] + sv[2] * e[2] + sv[3] * e[3] + sv[4] * e[4] + sv[5] * e[5]);
	}
	else if constexpr (MAT == MAT_HOOKE)
	{
		double v[6], sv[6];
		hooke_strain_stress(F, T, v, sv);
		return 0.5 * (sv[0] * v[0] + sv[1] * v[1] + sv[2] * v[2] + sv[3] * v[3] + sv[4] * v[4] + sv[5] * v[5]);
	}
	else if constexpr (MAT == MAT_LINEAR_ELASTICITY)
	{
		// eps:eps = sum_r G_rr^2 + 1/2 sum_{r<c} (G_rc + G_cr)^2
		const double g0 = F[0][0] - 1.0, g1 = F[1][1] - 1.0, g2 = F[2][2] - 1.0, tr = g0 + g1 + g2;
		const double ee = g0 * g0 + g1 * g1 + g2 * g2 +
						  0.5 * (sq(F[0][1] + F[1][0]) + sq(F[0][2] + F[2][0]) + sq(F[1][2] + F[2][1]));
		return p.y * ee + 0.5 * p.x * tr * tr;
	}
	else
	{
		Invariants v;
		invariants(F, v);
		return inv_psi<MAT, double>(v.I1, v.I2, v.J, p);
	}
}

// P = dpsi/dF (row-major 9)
template <int MAT>
__device__ __forceinline__ void mat_stress(const double F[3][3], const MatP &p, const double *T, double P[9])
{
	if constexpr (entry_mat<MAT>())
	{
		// one dual evaluation per entry of F
#pragma unroll 1
		for (int i = 0; i < 9; ++i)
		{
			Dual1 Fd[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) Fd[r][c] = {F[r][c], (3 * r + c) == i ? 1.0 : 0.0};
			P[i] = ogden_psi<MAT, Dual1>(Fd, p).d;
		}
	}
	else if constexpr (MAT == MAT_SAINT_VENANT_TENSOR)
	{
		double Cr[9], e[6], sv[6];
		right_cauchy_green(F, Cr);
		green_voigt_stress(Cr, T, e, sv);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
				P[3 * r + c] = F[r][0] * sv[voigt(0, c)] + F[r][1] * sv[voigt(1, c)] + F[r][2] * sv[voigt(2, c)];
	}
	else if constexpr (MAT == MAT_HOOKE)
	{
		double v[6], sv[6];
		hooke_strain_stress(F, T, v, sv);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) P[3 * r + c] = sv[voigt(r, c)];
	}
	else if constexpr (MAT == MAT_LINEAR_ELASTICITY)
	{
		const double tr = F[0][0] + F[1][1] + F[2][2] - 3.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
				P[3 * r + c] = p.y * ((F[r][c] - (r == c)) + (F[c][r] - (r == c))) + (r == c ? p.x * tr : 0.0);
	}
	else
	{
		Invariants v;
		invariants(F, v);
		double d[3];
		inv_psi_first<MAT>(v, p, d);
#pragma unroll
		for (int i = 0; i < 9; ++i) P[i] = d[0] * v.dx[0][i] + d[1] * v.dx[1][i] + d[2] * v.dx[2][i];
	}
}

// ---------------------------------------------------------------------------
// energy and gradient: thread per element
// ---------------------------------------------------------------------------
template <class EL, int MAT>
__device__ __forceinline__ double ad_element_energy(const DevMesh &m, const double *__restrict__ u, int e,
													unsigned long long *inverted)
{
	double Xg[EL::NG][3], U[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	const MatP prm = ad_params<MAT>(m, e);
	double en = 0.0;
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		double Jit[3][3], detJ, F[3][3];
		geometry<EL, double>(q, Xg, Jit, detJ);
		gen_def_grad<EL>(q, U, Jit, F);
		bad |= !(det3(F) > 0.0);
		en += mat_energy<MAT>(F, prm, m.hooke) * (detJ * qweight<EL>(q));
	}
	if (bad) atomicAdd(inverted, 1ull);
	return en;
}

template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_ad_energy(DevMesh m, const double *__restrict__ u, double *__restrict__ partials,
												  double *__restrict__ result, unsigned int *ticket,
												  unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	double en = 0.0;
	if (e < m.E) en = ad_element_energy<EL, MAT>(m, u, e, inverted);
	reduce_to_result<NT>(en, partials, result, ticket);
}

template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_ad_energy_per_element(DevMesh m, const double *__restrict__ u,
															  double *__restrict__ out, unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e < m.E) out[e] = ad_element_energy<EL, MAT>(m, u, e, inverted);
}

// element gradient G[a][d] = sum_q da sum_c P[d][c] g_a[c], g_a = J^-T gref_a, one
// slot per incidence as the other gradient kernels stage it
template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_ad_gradient(DevMesh m, const double *__restrict__ u, double *__restrict__ stage,
													unsigned long long *inverted)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	double Xg[EL::NG][3], U[EL::N][3], Gacc[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	const MatP prm = ad_params<MAT>(m, e);
#pragma unroll
	for (int a = 0; a < EL::N; ++a) Gacc[a][0] = Gacc[a][1] = Gacc[a][2] = 0.0;
	bool bad = false;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		double Jit[3][3], detJ, F[3][3], P[9];
		geometry<EL, double>(q, Xg, Jit, detJ);
		gen_def_grad<EL>(q, U, Jit, F);
		bad |= !(det3(F) > 0.0);
		mat_stress<MAT>(F, prm, m.hooke, P);
		const double da = detJ * qweight<EL>(q);
		double Q[3][3]; // da P J^-1 = da P Jit^T: G[a][d] = sum_r gref(q, a, r) Q[d][r]
#pragma unroll
		for (int d = 0; d < 3; ++d)
#pragma unroll
			for (int r = 0; r < 3; ++r)
				Q[d][r] = da * (P[3 * d] * Jit[r][0] + P[3 * d + 1] * Jit[r][1] + P[3 * d + 2] * Jit[r][2]);
#pragma unroll
		for (int a = 0; a < EL::N; ++a)
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				const double gr = gref<EL>(q, a, r);
				if (gr != 0.0)
				{
#pragma unroll
					for (int d = 0; d < 3; ++d) Gacc[a][d] += gr * Q[d][r];
				}
			}
	}
	if (bad) atomicAdd(inverted, 1ull);
#pragma unroll
	for (int a = 0; a < EL::N; ++a)
	{
		const int k = __ldg(m.eb_inc + (size_t)e * EL::N + a);
		st_slot(stage + (size_t)k * 4, Gacc[a][0], Gacc[a][1], Gacc[a][2]);
	}
}

// ---------------------------------------------------------------------------
// element blocks: one warp per element
// ---------------------------------------------------------------------------
// Entry k (i <= j, tri_index(9, i, j) order) of the 9 x 9 table C, with i = 3a + A,
// j = 3b + B: the flat indices and 0/1 factors of its terms, so that the lanes of a
// warp, each at its own entry, form it without branches:
//   aB = 3a + B, bA = 3b + A, AB = 3A + B, ab = 3a + b (indices into F, F^T F, F F^T),
//   cC = 3c + C and sJ = eps_abc eps_ABC for the one nonzero term of d2J (a != b, A != B),
//   the deltas ab, AB and ij, and the two index patterns of the LinearElasticity tangent.
struct alignas(4) CEntry
{
	unsigned char i, j, aB, bA, AB, ab, cC, dab, dAB, dij, le_aBbA, le_aAbB;
	signed char sJ;
	unsigned char pad[3];
};
struct CEntryTable
{
	CEntry e[45];
};
constexpr CEntryTable make_centries()
{
	CEntryTable t{};
	int k = 0;
	for (int i = 0; i < 9; ++i)
		for (int j = i; j < 9; ++j)
		{
			const int a = i / 3, A = i % 3, b = j / 3, B = j % 3;
			CEntry &c = t.e[k++];
			c.i = (unsigned char)i;
			c.j = (unsigned char)j;
			c.aB = (unsigned char)(3 * a + B);
			c.bA = (unsigned char)(3 * b + A);
			c.AB = (unsigned char)(3 * A + B);
			c.ab = (unsigned char)(3 * a + b);
			c.dab = a == b;
			c.dAB = A == B;
			c.dij = i == j;
			c.le_aBbA = a == B && A == b;
			c.le_aAbB = a == A && b == B;
			if (a != b && A != B)
			{
				const int cc = 3 - a - b, CC = 3 - A - B;
				const bool p1 = (b - a + 3) % 3 == 1, p2 = (B - A + 3) % 3 == 1; // cyclic (a, b, c), (A, B, C)
				c.cC = (unsigned char)(3 * cc + CC);
				c.sJ = p1 == p2 ? 1 : -1;
			}
		}
	return t;
}
__constant__ CEntryTable c_ad_centries = make_centries();
// the pairs (x, y), x <= y, of the three invariants; the node pairs of the element
// block triangle (P1, P2, Q1)
__constant__ PairTable c_ad_x3 = make_pairs(3);
__constant__ PairTable c_ad_pairs[3] = {make_pairs(4), make_pairs(10), make_pairs(8)};

template <class EL>
struct AdWarp
{
	static constexpr int N = EL::N, NG = EL::NG, NQ = EL::NQ, TP = tri_pad(EL::N);
	double U[N][3], X[NG][3];
	double Jit[NQ][9], da[NQ];
	Invariants inv[NQ];
	double psi[NQ][9];              // psi_x (x = I1, I2, J), then psi_xy (x <= y) in tri_index(3, x, y) order
	double C[NQ][45];               // da d2psi/dF2 at point q, entry (i <= j) at tri_index(9, i, j)
	alignas(16) double g[NQ][N][4]; // physical basis gradients (x, y, z, 0): two 16-byte loads
	alignas(16) double tri[TP];     // the element's packed block triangle, copied out as double2
};

__host__ __device__ constexpr int c9(int i, int j) { return i <= j ? tri_index(9, i, j) : tri_index(9, j, i); }

// SaintVenant with a tensor, entry ce = ((a, A), (b, B)) of C, with sv the point's
// Voigt stress:
//   delta_ab S(A, B) + sum_{I,J} F(a, I) F(b, J) T[voigt(I, A)][voigt(J, B)]
__device__ __forceinline__ double svt_hessian_entry(const Invariants &v, const double *sv, const double *__restrict__ T,
													const CEntry &ce)
{
	const int a = ce.i / 3, A = ce.i % 3, b = ce.j / 3, B = ce.j % 3;
	const double *F = v.dx[0]; // dI1/dF = 2F
	double h = ce.dab ? sv[voigt(A, B)] : 0.0;
#pragma unroll
	for (int I = 0; I < 3; ++I)
#pragma unroll
		for (int J = 0; J < 3; ++J)
			h += (0.25 * F[3 * a + I] * F[3 * b + J]) * __ldg(T + 6 * voigt(I, A) + voigt(J, B));
	return h;
}

// d2psi/dF_i dF_j from the invariants' derivatives, entry ce of C
__device__ __forceinline__ double inv_hessian_entry(const Invariants &v, const double *psi, const CEntry &ce)
{
	const double *dx0 = v.dx[0], *dx1 = v.dx[1], *dx2 = v.dx[2];
	const int i = ce.i, j = ce.j;
	// F = dI1/dF / 2
	const double FaA = 0.5 * dx0[i], FbB = 0.5 * dx0[j], FaB = 0.5 * dx0[ce.aB], FbA = 0.5 * dx0[ce.bA];
	const double d2I2 = 4.0 * FaA * FbB - 2.0 * FaB * FbA + 2.0 * ce.dab * (ce.dAB * v.I1 - v.Cr[ce.AB]) -
						2.0 * ce.dAB * v.B[ce.ab];
	const double d2J = ce.sJ * 0.5 * dx0[ce.cC];
	const double xi[3] = {dx0[i], dx1[i], dx2[i]}, xj[3] = {dx0[j], dx1[j], dx2[j]};
	double h = psi[0] * (2.0 * ce.dij) + psi[1] * d2I2 + psi[2] * d2J;
#pragma unroll
	for (int x = 0; x < 3; ++x)
#pragma unroll
		for (int y = 0; y < 3; ++y) h += psi[3 + (x <= y ? tri_index(3, x, y) : tri_index(3, y, x))] * xi[x] * xj[y];
	return h;
}

template <class EL, int MAT, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_ad_blocks(DevMesh m, const double *__restrict__ u, double *__restrict__ stage)
{
	using W = AdWarp<EL>;
	constexpr int N = EL::N, NG = EL::NG, NQ = EL::NQ, NP = N * (N + 1) / 2, TP = W::TP;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	W &S = reinterpret_cast<W *>(smem_raw)[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	// the lookup tables in shared memory: lanes at different entries read them without
	// the serialisation of divergent constant-memory reads
	__shared__ CEntry s_ce[45];
	__shared__ unsigned char s_pa[NP], s_pb[NP], s_xa[6], s_xb[6];
	for (int t = threadIdx.x; t < 45; t += WPB * 32) s_ce[t] = c_ad_centries.e[t];
	for (int t = threadIdx.x; t < NP; t += WPB * 32)
	{
		s_pa[t] = c_ad_pairs[EL::ET - 1].a[t];
		s_pb[t] = c_ad_pairs[EL::ET - 1].b[t];
	}
	for (int t = threadIdx.x; t < 6; t += WPB * 32)
	{
		s_xa[t] = c_ad_x3.a[t];
		s_xb[t] = c_ad_x3.b[t];
	}
	__syncthreads();
	for (int e = blockIdx.x * WPB + (threadIdx.x >> 5); e < m.E; e += gridDim.x * WPB)
	{
		for (int i = lane; i < N * 3; i += 32)
			S.U[i / 3][i % 3] = __ldg(u + (size_t)__ldg(m.conn + (size_t)(i / 3) * m.E + e) * 3 + i % 3);
		for (int i = lane; i < NG * 3; i += 32)
			S.X[i / 3][i % 3] = __ldg(m.X + (size_t)__ldg(m.gconn + (size_t)(i / 3) * m.E + e) * 3 + i % 3);
		__syncwarp();
		const MatP prm = ad_params<MAT>(m, e);
		if (lane < NQ)
		{
			const int q = lane;
			double Jit[3][3], detJ, F[3][3];
			geometry<EL, double>(q, S.X, Jit, detJ);
			gen_def_grad<EL>(q, S.U, Jit, F);
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) S.Jit[q][3 * r + c] = Jit[r][c];
			S.da[q] = detJ * qweight<EL>(q);
			if constexpr (!quadratic_mat<MAT>()) invariants(F, S.inv[q]); // entry_mat: F = dI1/dF / 2
			if constexpr (MAT == MAT_SAINT_VENANT_TENSOR)
			{
				// the point's Voigt stress, shared by its 45 tangent entries (psi is unused here)
				double e[6];
				green_voigt_stress(S.inv[q].Cr, m.hooke, e, S.psi[q]);
			}
		}
		__syncwarp();
		// lanes over (point, node): g = J^-T gref
		for (int t = lane; t < NQ * N; t += 32)
		{
			const int q = t / N, a = t - q * N;
			double *g = S.g[q][a];
#pragma unroll
			for (int c = 0; c < 3; ++c)
				g[c] = gref<EL>(q, a, 0) * S.Jit[q][c] + gref<EL>(q, a, 1) * S.Jit[q][3 + c] + gref<EL>(q, a, 2) * S.Jit[q][6 + c];
			g[3] = 0.0;
		}
		if constexpr (invariant_mat<MAT>())
		{
			// lanes over (point, invariant pair x <= y): one hyper-dual evaluation each
			for (int t = lane; t < NQ * 6; t += 32)
			{
				const int q = t / 6, k = t - q * 6, x = s_xa[k], y = s_xb[k];
				const Invariants &v = S.inv[q];
				const HDual h = inv_psi<MAT, HDual>({v.I1, x == 0 ? 1.0 : 0.0, y == 0 ? 1.0 : 0.0, 0.0},
													{v.I2, x == 1 ? 1.0 : 0.0, y == 1 ? 1.0 : 0.0, 0.0},
													{v.J, x == 2 ? 1.0 : 0.0, y == 2 ? 1.0 : 0.0, 0.0}, prm);
				S.psi[q][3 + k] = h.ab;
				if (x == y) S.psi[q][x] = h.a;
			}
			__syncwarp();
		}
		// lanes over (point, entry i <= j of C)
		for (int t = lane; t < NQ * 45; t += 32)
		{
			const int q = t / 45, k = t - q * 45;
			const CEntry ce = s_ce[k];
			double h;
			if constexpr (MAT == MAT_SAINT_VENANT_TENSOR)
				h = svt_hessian_entry(S.inv[q], S.psi[q], m.hooke, ce);
			else if constexpr (MAT == MAT_HOOKE)
				h = __ldg(m.hooke + 6 * voigt(ce.i / 3, ce.i % 3) + voigt(ce.j / 3, ce.j % 3));
			else if constexpr (MAT == MAT_LINEAR_ELASTICITY)
				h = prm.y * (ce.dab * ce.dAB + ce.le_aBbA) + prm.x * ce.le_aAbB;
			else if constexpr (entry_mat<MAT>())
			{
				// one hyper-dual evaluation over the entries (i, j) of F
				double F[3][3], ej[9];
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int c = 0; c < 3; ++c) F[r][c] = 0.5 * S.inv[q].dx[0][3 * r + c];
#pragma unroll
				for (int l = 0; l < 9; ++l) ej[l] = l == ce.j ? 1.0 : 0.0;
				HDual Fh[3][3];
				hd_def_grad(F, ce.i, ej, Fh);
				h = ogden_psi<MAT, HDual>(Fh, prm).ab;
			}
			else
				h = inv_hessian_entry(S.inv[q], S.psi[q], ce);
			S.C[q][k] = S.da[q] * h;
		}
		__syncwarp();
		// lanes over node pairs (a <= b): H_ab[r][k] = sum_q sum_{c,d} g_a[c] C[(r,c),(k,d)] g_b[d]
		for (int p = lane; p < NP; p += 32)
		{
			const int a = s_pa[p], b = s_pb[p];
			double h[3][3] = {};
			for (int q = 0; q < NQ; ++q)
			{
				const double2 a01 = reinterpret_cast<const double2 *>(S.g[q][a])[0], a2 = reinterpret_cast<const double2 *>(S.g[q][a])[1];
				const double2 b01 = reinterpret_cast<const double2 *>(S.g[q][b])[0], b2 = reinterpret_cast<const double2 *>(S.g[q][b])[1];
				const double ga[3] = {a01.x, a01.y, a2.x}, gb[3] = {b01.x, b01.y, b2.x};
				const double *Cq = S.C[q];
#pragma unroll
				for (int r = 0; r < 3; ++r)
#pragma unroll
					for (int k = 0; k < 3; ++k)
					{
						double s_ = 0.0;
#pragma unroll
						for (int c = 0; c < 3; ++c)
						{
							const double w = Cq[c9(3 * r + c, 3 * k)] * gb[0] + Cq[c9(3 * r + c, 3 * k + 1)] * gb[1] +
											 Cq[c9(3 * r + c, 3 * k + 2)] * gb[2];
							s_ += ga[c] * w;
						}
						h[r][k] += s_;
					}
			}
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int k = 0; k < 3; ++k) S.tri[9 * p + 3 * k + r] = h[r][k];
		}
		__syncwarp();
		double2 *dst = reinterpret_cast<double2 *>(stage + (size_t)e * TP);
		const double2 *src = reinterpret_cast<const double2 *>(S.tri);
		for (int i = lane; i < TP / 2; i += 32) dst[i] = src[i];
		__syncwarp();
	}
}

// ---------------------------------------------------------------------------
// adjoint terms (ElasticForceDerivative.cpp:35-132, 134-260)
// ---------------------------------------------------------------------------
// The invariants and dx/dF of F, generic in the number type: with F + eps W in
// first-order dual numbers they carry their directional derivatives along W.
template <class S>
__device__ __forceinline__ void stress_invariants(const S F[3][3], S &I1, S &I2, S &J, S dx[3][9])
{
	S B[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) B[r][c] = F[r][0] * F[c][0] + F[r][1] * F[c][1] + F[r][2] * F[c][2];
	I1 = B[0][0] + B[1][1] + B[2][2];
	const S trB2 = sq(B[0][0]) + sq(B[1][1]) + sq(B[2][2]) + 2.0 * (sq(B[0][1]) + sq(B[0][2]) + sq(B[1][2]));
	I2 = 0.5 * (sq(I1) - trB2);
	J = det3(F);
	S cof[3][3];
	cofactor3(F, cof);
#pragma unroll
	for (int a = 0; a < 3; ++a)
#pragma unroll
		for (int A = 0; A < 3; ++A)
		{
			dx[0][3 * a + A] = 2.0 * F[a][A];
			dx[1][3 * a + A] = 2.0 * (I1 * F[a][A] - (B[a][0] * F[0][A] + B[a][1] * F[1][A] + B[a][2] * F[2][A]));
			dx[2][3 * a + A] = cof[a][A];
		}
}

// P = dpsi/dF and Q = C : W = dP/dF[W], the stress's directional derivative along W
// (compute_stress_grad_multiply_mat with mat = W): P = sum_x psi_x dx/dF and
// Q = sum_x (psi_x' dx/dF + psi_x (dx/dF)'), with ' the derivative along W; psi_x and
// psi_x' = sum_y psi_xy y' come from one hyper-dual evaluation per invariant x.
template <int MAT>
__device__ __forceinline__ void stress_and_directional(const double F[3][3], const double W[3][3], const MatP &p,
													   double P[9], double Q[9])
{
	if constexpr (MAT == MAT_LINEAR_ELASTICITY)
	{
		const double trG = F[0][0] + F[1][1] + F[2][2] - 3.0, trW = W[0][0] + W[1][1] + W[2][2];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c)
			{
				P[3 * r + c] = p.y * ((F[r][c] - (r == c)) + (F[c][r] - (r == c))) + (r == c ? p.x * trG : 0.0);
				Q[3 * r + c] = p.y * (W[r][c] + W[c][r]) + (r == c ? p.x * trW : 0.0);
			}
	}
	else if constexpr (entry_mat<MAT>())
	{
		// one hyper-dual evaluation per entry i of F, along e_i and W: P_i and (C W)_i
		double w9[9];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) w9[3 * r + c] = W[r][c];
#pragma unroll 1
		for (int i = 0; i < 9; ++i)
		{
			HDual Fh[3][3];
			hd_def_grad(F, i, w9, Fh);
			const HDual h = ogden_psi<MAT, HDual>(Fh, p);
			P[i] = h.a;
			Q[i] = h.ab;
		}
	}
	else
	{
		Dual1 Fd[3][3], I1, I2, J, dx[3][9];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) Fd[r][c] = {F[r][c], W[r][c]};
		stress_invariants(Fd, I1, I2, J, dx);
#pragma unroll
		for (int i = 0; i < 9; ++i) P[i] = Q[i] = 0.0;
#pragma unroll
		for (int x = 0; x < 3; ++x)
		{
			const HDual h = inv_psi<MAT, HDual>({I1.v, x == 0 ? 1.0 : 0.0, I1.d, 0.0}, {I2.v, x == 1 ? 1.0 : 0.0, I2.d, 0.0},
												{J.v, x == 2 ? 1.0 : 0.0, J.d, 0.0}, p);
#pragma unroll
			for (int i = 0; i < 9; ++i)
			{
				P[i] += h.a * dx[x][i].v;
				Q[i] += h.ab * dx[x][i].v + h.a * dx[x][i].d;
			}
		}
	}
}

// LinearElasticity's material derivative: dP/dmu = grad u + grad u^T, dP/dlambda =
// tr(grad u) I (LinearElasticity.cpp:290-299); out = [lambda block; mu block], each
// -sum_q da dP:grad p
template <class EL, int NT>
__global__ void __launch_bounds__(NT) k_le_material_vjp(DevMesh m, const double *__restrict__ u,
														const double *__restrict__ adj, double *__restrict__ out)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	double Xg[EL::NG][3], U[EL::N][3], Pn[EL::N][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	load_nodal<EL, double>(m, e, adj, Pn, nodes);
	double tl = 0.0, tm = 0.0;
#pragma unroll
	for (int q = 0; q < EL::NQ; ++q)
	{
		double Jit[3][3], detJ, gphi[EL::N][3], Gu[3][3], Gp[3][3];
		geometry<EL, double>(q, Xg, Jit, detJ);
		phys_grads<EL, double>(q, Jit, gphi);
		disp_grad<EL, double>(U, gphi, Gu);
		disp_grad<EL, double>(Pn, gphi, Gp);
		double imu = 0.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) imu += (Gu[r][c] + Gu[c][r]) * Gp[r][c];
		const double da = detJ * qweight<EL>(q);
		tl -= (Gu[0][0] + Gu[1][1] + Gu[2][2]) * (Gp[0][0] + Gp[1][1] + Gp[2][2]) * da;
		tm -= imu * da;
	}
	out[e] = tl;
	out[(size_t)m.E + e] = tm;
}

// Shape derivative (ElasticForceDerivative.cpp:207-260): for the rank-one V = e_d (x) g,
// g the physical gradient of geometric basis function v, and M = grad u V,
//   (C:M + P V^T - tr(V) P) : grad p = a.(Q g) + (P g).grad p[:, d] - g_d (P : grad p),
// with a = grad u[:, d] and Q = C : grad p (C is symmetric in its index pairs).
// Element contributions into one slot per geometric incidence.
template <class EL, int MAT, int NT>
__global__ void __launch_bounds__(NT) k_ad_shape_vjp(DevMesh m, const double *__restrict__ u,
													 const double *__restrict__ adj, double *__restrict__ stage)
{
	const int e = blockIdx.x * NT + threadIdx.x;
	if (e >= m.E) return;
	double Xg[EL::NG][3], U[EL::N][3], Pn[EL::N][3], acc[EL::NG][3];
	int nodes[EL::N];
	load_geom<EL, double>(m, e, Xg);
	load_nodal<EL, double>(m, e, u, U, nodes);
	load_nodal<EL, double>(m, e, adj, Pn, nodes);
	const MatP prm = ad_params<MAT>(m, e);
#pragma unroll
	for (int j = 0; j < EL::NG; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0;
#pragma unroll 1
	for (int q = 0; q < EL::NQ; ++q)
	{
		double Jit[3][3], detJ, gphi[EL::N][3], Gu[3][3], Gp[3][3], F[3][3], P[9], Q[9];
		geometry<EL, double>(q, Xg, Jit, detJ);
		phys_grads<EL, double>(q, Jit, gphi);
		disp_grad<EL, double>(U, gphi, Gu);
		disp_grad<EL, double>(Pn, gphi, Gp);
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) F[r][c] = Gu[r][c] + (r == c ? 1.0 : 0.0);
		stress_and_directional<MAT>(F, Gp, prm, P, Q);
		double PGp = 0.0;
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) PGp += P[3 * r + c] * Gp[r][c];
		const double da = detJ * qweight<EL>(q);
#pragma unroll
		for (int v = 0; v < EL::NG; ++v)
		{
			double g[3];
#pragma unroll
			for (int c = 0; c < 3; ++c)
				g[c] = ggref<EL>(q, v, 0) * Jit[0][c] + ggref<EL>(q, v, 1) * Jit[1][c] + ggref<EL>(q, v, 2) * Jit[2][c];
			double Qg[3], Pg[3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
			{
				Qg[r] = Q[3 * r] * g[0] + Q[3 * r + 1] * g[1] + Q[3 * r + 2] * g[2];
				Pg[r] = P[3 * r] * g[0] + P[3 * r + 1] * g[1] + P[3 * r + 2] * g[2];
			}
#pragma unroll
			for (int d = 0; d < 3; ++d)
			{
				const double t = Gu[0][d] * Qg[0] + Gu[1][d] * Qg[1] + Gu[2][d] * Qg[2] + Pg[0] * Gp[0][d] +
								 Pg[1] * Gp[1][d] + Pg[2] * Gp[2][d] - g[d] * PGp;
				acc[v][d] -= t * da;
			}
		}
	}
#pragma unroll
	for (int v = 0; v < EL::NG; ++v)
	{
		const int k = __ldg(m.g_eb_inc + (size_t)e * EL::NG + v);
		st_slot(stage + (size_t)k * 4, acc[v][0], acc[v][1], acc[v][2]);
	}
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline int ad_blocks_for(int n, int nt) { return (n + nt - 1) / nt; }

// f(element type, material) for the context's element type and material
template <class Fn>
static cudaError_t with_ad_material(const DevMesh &m, Fn &&f)
{
	auto by_mat = [&](auto el) -> cudaError_t {
		using EL = decltype(el);
		switch (m.mat)
		{
		case MAT_LINEAR_ELASTICITY: f(EL{}, std::integral_constant<int, MAT_LINEAR_ELASTICITY>{}); break;
		case MAT_MOONEY_RIVLIN: f(EL{}, std::integral_constant<int, MAT_MOONEY_RIVLIN>{}); break;
		case MAT_MOONEY_RIVLIN_3PARAM: f(EL{}, std::integral_constant<int, MAT_MOONEY_RIVLIN_3PARAM>{}); break;
		case MAT_VOLUME_PENALTY: f(EL{}, std::integral_constant<int, MAT_VOLUME_PENALTY>{}); break;
		case MAT_HOOKE: f(EL{}, std::integral_constant<int, MAT_HOOKE>{}); break;
		case MAT_SAINT_VENANT_TENSOR: f(EL{}, std::integral_constant<int, MAT_SAINT_VENANT_TENSOR>{}); break;
		case MAT_UNCONSTRAINED_OGDEN: f(EL{}, std::integral_constant<int, MAT_UNCONSTRAINED_OGDEN>{}); break;
		case MAT_INCOMPRESSIBLE_OGDEN: f(EL{}, std::integral_constant<int, MAT_INCOMPRESSIBLE_OGDEN>{}); break;
		case MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC:
			f(EL{}, std::integral_constant<int, MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC>{});
			break;
		default: return cudaErrorInvalidValue;
		}
		return cudaGetLastError();
	};
	switch (m.et)
	{
	case 1: return by_mat(P1Tet{});
	case 2: return by_mat(P2Tet{});
	case 3: return by_mat(Q1Hex{});
	}
	return cudaErrorInvalidValue;
}

cudaError_t launch_ad_energy(const DevMesh &m, const double *u, bool per_element, double *out, const Scratch &sc,
							 cudaStream_t s)
{
	if (m.E == 0) return per_element ? cudaSuccess : cudaMemsetAsync(out, 0, sizeof(double), s);
	return with_ad_material(m, [&](auto el, auto mat) {
		using EL = decltype(el);
		constexpr int MAT = decltype(mat)::value, NT = 256;
		const int nb = ad_blocks_for(m.E, NT);
		if (per_element)
			k_ad_energy_per_element<EL, MAT, NT><<<nb, NT, 0, s>>>(m, u, out, sc.inverted);
		else
			k_ad_energy<EL, MAT, NT><<<nb, NT, 0, s>>>(m, u, sc.partials, out, sc.ticket, sc.inverted);
	});
}

cudaError_t launch_ad_gradient_stage(const DevMesh &m, const double *u, const Scratch &sc, cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	return with_ad_material(m, [&](auto el, auto mat) {
		using EL = decltype(el);
		constexpr int MAT = decltype(mat)::value, NT = 128;
		k_ad_gradient<EL, MAT, NT><<<ad_blocks_for(m.E, NT), NT, 0, s>>>(m, u, sc.vec_stage, sc.inverted);
	});
}

cudaError_t launch_ad_blocks(const DevMesh &m, const double *u, double *stage, cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	cudaError_t err = cudaSuccess;
	cudaError_t st = with_ad_material(m, [&](auto el, auto mat) {
		using EL = decltype(el);
		constexpr int MAT = decltype(mat)::value, WPB = 4;
		const size_t bytes = WPB * sizeof(AdWarp<EL>);
		err = cudaFuncSetAttribute(k_ad_blocks<EL, MAT, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
		if (err != cudaSuccess) return;
		const int nb = std::min((m.E + WPB - 1) / WPB, 148 * 32);
		k_ad_blocks<EL, MAT, WPB><<<nb, WPB * 32, bytes, s>>>(m, u, stage);
	});
	return err != cudaSuccess ? err : st;
}


cudaError_t launch_ad_material_vjp(const DevMesh &m, const double *u, const double *adj, double *out, cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	if (m.mat != MAT_LINEAR_ELASTICITY) return cudaErrorInvalidValue;
	constexpr int NT = 128;
	const int nb = ad_blocks_for(m.E, NT);
	switch (m.et)
	{
	case 1: k_le_material_vjp<P1Tet, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	case 2: k_le_material_vjp<P2Tet, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	case 3: k_le_material_vjp<Q1Hex, NT><<<nb, NT, 0, s>>>(m, u, adj, out); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t launch_ad_shape_vjp_stage(const DevMesh &m, const double *u, const double *adj, const Scratch &sc,
									  cudaStream_t s)
{
	if (m.E == 0) return cudaSuccess;
	constexpr int NT = 128;
	const int nb = ad_blocks_for(m.E, NT);
	auto launch = [&](auto el, auto mat) {
		using EL = decltype(el);
		k_ad_shape_vjp<EL, decltype(mat)::value, NT><<<nb, NT, 0, s>>>(m, u, adj, sc.vec_stage);
	};
	auto by_el = [&](auto mat) -> cudaError_t {
		switch (m.et)
		{
		case 1: launch(P1Tet{}, mat); break;
		case 2: launch(P2Tet{}, mat); break;
		case 3: launch(Q1Hex{}, mat); break;
		default: return cudaErrorInvalidValue;
		}
		return cudaGetLastError();
	};
	switch (m.mat)
	{
	case MAT_ISO_NEOHOOKEAN: return by_el(std::integral_constant<int, MAT_ISO_NEOHOOKEAN>{});
	case MAT_LINEAR_ELASTICITY: return by_el(std::integral_constant<int, MAT_LINEAR_ELASTICITY>{});
	case MAT_MOONEY_RIVLIN: return by_el(std::integral_constant<int, MAT_MOONEY_RIVLIN>{});
	case MAT_MOONEY_RIVLIN_3PARAM: return by_el(std::integral_constant<int, MAT_MOONEY_RIVLIN_3PARAM>{});
	case MAT_VOLUME_PENALTY: return by_el(std::integral_constant<int, MAT_VOLUME_PENALTY>{});
	case MAT_UNCONSTRAINED_OGDEN: return by_el(std::integral_constant<int, MAT_UNCONSTRAINED_OGDEN>{});
	case MAT_INCOMPRESSIBLE_OGDEN: return by_el(std::integral_constant<int, MAT_INCOMPRESSIBLE_OGDEN>{});
	case MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC: return by_el(std::integral_constant<int, MAT_MOONEY_RIVLIN_3PARAM_SYMBOLIC>{});
	}
	return cudaErrorInvalidValue;
}

} // namespace pfg
